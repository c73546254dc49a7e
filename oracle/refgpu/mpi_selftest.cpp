// CPU self-test of the in-process MPI stand-in (TEST INFRASTRUCTURE ONLY).
//
// zr_mpi_selftest(P) runs P*P ranks on host buffers through the same call pattern as
// the reference: MPI_Comm_split into row and column communicators (fft.cu:561-567),
// MPI_Alltoall over each (fft.cu:221-241), the four halo MPI_Sendrecv of
// communicate_laplace (laplace.cu:194-256) and MPI_Reduce(MAX) of the timing macro
// (fft.cu:8-18).  Returns 0 when every received value is the one MPI would deliver,
// otherwise the number of wrong values (or -1 when a rendezvous timed out).
#include "mpi.h"

#include <atomic>
#include <vector>

namespace {

struct Ctx {
    int p = 0;
    std::atomic<int> errors{0};
};

// value rank `id` sends to communicator rank `dst`, element k
long long tag_value(int id, int dst, int k) { return 1000000LL * id + 1000LL * dst + k; }

void rank_main(int id, void* arg) {
    Ctx* c = static_cast<Ctx*>(arg);
    const int p = c->p;
    const int rid = id / p, cid = id % p;
    int wr = -1, ws = -1;
    MPI_Comm_rank(MPI_COMM_WORLD, &wr);
    MPI_Comm_size(MPI_COMM_WORLD, &ws);
    if (wr != id || ws != p * p) c->errors++;

    MPI_Comm row_comm, col_comm;
    MPI_Comm_split(MPI_COMM_WORLD, rid, id, &row_comm);
    MPI_Comm_split(MPI_COMM_WORLD, cid, id, &col_comm);
    int rr = -1, rs = -1, cr = -1, cs = -1;
    MPI_Comm_rank(row_comm, &rr);
    MPI_Comm_size(row_comm, &rs);
    MPI_Comm_rank(col_comm, &cr);
    MPI_Comm_size(col_comm, &cs);
    if (rr != cid || rs != p || cr != rid || cs != p) c->errors++;

    const int K = 3;   // elements per peer block
    for (int pass = 0; pass < 2; ++pass) {
        MPI_Comm comm = pass == 0 ? row_comm : col_comm;
        const int me = pass == 0 ? cid : rid;
        std::vector<long long> send(p * K), recv(p * K, -1);
        for (int d = 0; d < p; ++d)
            for (int k = 0; k < K; ++k) send[d * K + k] = tag_value(id, d, k);
        MPI_Alltoall(send.data(), K, MPI_LONG_LONG, recv.data(), K, MPI_LONG_LONG, comm);
        for (int s = 0; s < p; ++s) {
            const int src_id = pass == 0 ? rid * p + s : s * p + cid;
            for (int k = 0; k < K; ++k)
                if (recv[s * K + k] != tag_value(src_id, me, k)) c->errors++;
        }
    }

    // Halo pattern of communicate_laplace: send right / receive from left, and so on.
    const int left = (cid - 1 + p) % p, right = (cid + 1) % p;
    const int up = (rid - 1 + p) % p, down = (rid + 1) % p;
    long long out = id, in = -1;
    MPI_Sendrecv(&out, 1, MPI_LONG_LONG, right, 0, &in, 1, MPI_LONG_LONG, left, 0, row_comm,
                 MPI_STATUS_IGNORE);
    if (in != rid * p + left) c->errors++;
    MPI_Sendrecv(&out, 1, MPI_LONG_LONG, left, 1, &in, 1, MPI_LONG_LONG, right, 1, row_comm,
                 MPI_STATUS_IGNORE);
    if (in != rid * p + right) c->errors++;
    MPI_Sendrecv(&out, 1, MPI_LONG_LONG, up, 2, &in, 1, MPI_LONG_LONG, down, 2, col_comm,
                 MPI_STATUS_IGNORE);
    if (in != down * p + cid) c->errors++;
    MPI_Sendrecv(&out, 1, MPI_LONG_LONG, down, 3, &in, 1, MPI_LONG_LONG, up, 3, col_comm,
                 MPI_STATUS_IGNORE);
    if (in != up * p + cid) c->errors++;

    long long mine = 7 * id + 1, mx = -1;
    MPI_Reduce(&mine, &mx, 1, MPI_LONG_LONG, MPI_MAX, 0, MPI_COMM_WORLD);
    if (id == 0 && mx != 7LL * (p * p - 1) + 1) c->errors++;
    MPI_Barrier(MPI_COMM_WORLD);
}

}  // namespace

extern "C" int zr_mpi_selftest(int p) {
    Ctx c;
    c.p = p;
    if (zr_run_ranks(p * p, rank_main, &c) != 0) return -1;
    return c.errors.load();
}
