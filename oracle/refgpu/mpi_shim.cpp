// In-process, thread-per-rank stand-in for the MPI calls of the reference's zmodel
// sources.  TEST INFRASTRUCTURE ONLY (see mpi.h): never linked into the product library.
//
// Each communicator keeps a member list (world ranks, in communicator-rank order) and a
// rendezvous slot per member.  A collective posts the caller's arguments in its slot,
// waits for every member (bounded: a missing rank ends the run with an error instead
// of hanging), performs its copies, and waits again so that no member reuses its send
// buffer before the others have read it.
#include "mpi.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

namespace {

constexpr double kRendezvousLimitS = 300.0;   // a rank that never arrives: give up

struct Slot {
    const void* send = nullptr;
    void* recv = nullptr;
    long long count = 0;
    int dest = -1, tag = -1;
    int color = 0, key = 0;
    MPI_Comm made = nullptr;
};

}  // namespace

struct zr_comm {
    std::vector<int> members;            // world ranks, communicator-rank order
    std::vector<Slot> slots;
    std::mutex m;
    std::condition_variable cv;
    int arrived = 0;
    long long generation = 0;
};

namespace {

struct World {
    std::vector<std::unique_ptr<zr_comm>> comms;   // owned; freed when the run ends
    std::mutex comms_m;
    zr_comm* world = nullptr;
    std::atomic<int> failed{0};
};

World* g_world = nullptr;                // one run at a time (zr_run_ranks is serialised)
std::mutex g_run_m;
thread_local int tl_rank = -1;           // world rank of the calling thread

zr_comm* new_comm(std::vector<int> members) {
    auto c = std::make_unique<zr_comm>();
    c->members = std::move(members);
    c->slots.resize(c->members.size());
    zr_comm* raw = c.get();
    std::lock_guard<std::mutex> g(g_world->comms_m);
    g_world->comms.push_back(std::move(c));
    return raw;
}

int my_index(MPI_Comm c) {
    for (size_t i = 0; i < c->members.size(); ++i)
        if (c->members[i] == tl_rank) return (int)i;
    return -1;
}

// Bounded barrier over the communicator's members.  Returns false on timeout.
bool rendezvous(MPI_Comm c) {
    std::unique_lock<std::mutex> lk(c->m);
    long long gen = c->generation;
    if (++c->arrived == (int)c->members.size()) {
        c->arrived = 0;
        ++c->generation;
        c->cv.notify_all();
        return true;
    }
    bool ok = c->cv.wait_for(lk, std::chrono::duration<double>(kRendezvousLimitS),
                             [&] { return c->generation != gen || g_world->failed.load(); });
    if (!ok || c->generation == gen) {
        g_world->failed.store(1);
        c->cv.notify_all();
        return false;
    }
    return true;
}

[[noreturn]] void give_up(const char* what) {
    std::fprintf(stderr, "mpi stand-in: %s timed out on world rank %d (a rank never arrived)\n",
                 what, tl_rank);
    std::fflush(stderr);
    std::_Exit(97);
}

// Device (or managed) memory: the __GPU__AWARE__MPI__ path.  Without a device every
// pointer is host memory, which keeps the stand-in usable in CPU-only tests.
bool on_device(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

void copy_bytes(void* dst, const void* src, size_t bytes) {
    if (bytes == 0) return;
    if (!on_device(dst) && !on_device(src)) {
        std::memcpy(dst, src, bytes);
        return;
    }
    cudaError_t e = cudaMemcpy(dst, src, bytes, cudaMemcpyDefault);
    if (e != cudaSuccess) {
        std::fprintf(stderr, "mpi stand-in: cudaMemcpy failed: %s\n", cudaGetErrorString(e));
        std::_Exit(98);
    }
}

}  // namespace

extern "C" {

MPI_Comm zr_comm_world(void) { return g_world ? g_world->world : nullptr; }

int MPI_Init(int*, char***) { return MPI_SUCCESS; }
int MPI_Finalize(void) { return MPI_SUCCESS; }

int MPI_Comm_rank(MPI_Comm comm, int* rank) {
    *rank = my_index(comm);
    return MPI_SUCCESS;
}

int MPI_Comm_size(MPI_Comm comm, int* size) {
    *size = (int)comm->members.size();
    return MPI_SUCCESS;
}

int MPI_Barrier(MPI_Comm comm) {
    if (!rendezvous(comm)) give_up("MPI_Barrier");
    return MPI_SUCCESS;
}

// Members with the same colour form one communicator, ordered by (key, old rank).
// The first member of each new group creates it; the others pick it up from its slot.
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm* newcomm) {
    const int me = my_index(comm);
    comm->slots[me].color = color;
    comm->slots[me].key = key;
    comm->slots[me].made = nullptr;
    if (!rendezvous(comm)) give_up("MPI_Comm_split");
    std::vector<std::pair<std::pair<int, int>, int>> group;   // ((key, old rank), world rank)
    for (size_t i = 0; i < comm->members.size(); ++i)
        if (comm->slots[i].color == color)
            group.push_back({{comm->slots[i].key, (int)i}, comm->members[i]});
    std::sort(group.begin(), group.end());
    const int leader = group.front().first.second;
    if (leader == me) {
        std::vector<int> members;
        for (auto& g : group) members.push_back(g.second);
        comm->slots[me].made = new_comm(std::move(members));
    }
    if (!rendezvous(comm)) give_up("MPI_Comm_split");
    *newcomm = comm->slots[leader].made;
    if (!rendezvous(comm)) give_up("MPI_Comm_split");
    return MPI_SUCCESS;
}

// One process on one node: every rank shares the node, so the split is a copy of comm.
int MPI_Comm_split_type(MPI_Comm comm, int, int key, MPI_Info, MPI_Comm* newcomm) {
    return MPI_Comm_split(comm, 0, key, newcomm);
}

int MPI_Alltoall(const void* sendbuf, int sendcount, MPI_Datatype sendtype,
                 void* recvbuf, int recvcount, MPI_Datatype recvtype, MPI_Comm comm) {
    const int me = my_index(comm);
    const int n = (int)comm->members.size();
    const size_t sbytes = (size_t)sendcount * (size_t)sendtype;
    const size_t rbytes = (size_t)recvcount * (size_t)recvtype;
    if (sbytes != rbytes) {
        std::fprintf(stderr, "mpi stand-in: MPI_Alltoall send/recv sizes differ\n");
        std::_Exit(99);
    }
    comm->slots[me].send = sendbuf;
    if (!rendezvous(comm)) give_up("MPI_Alltoall");
    for (int j = 0; j < n; ++j)
        copy_bytes(static_cast<char*>(recvbuf) + (size_t)j * rbytes,
                   static_cast<const char*>(comm->slots[j].send) + (size_t)me * sbytes, rbytes);
    if (!rendezvous(comm)) give_up("MPI_Alltoall");
    return MPI_SUCCESS;
}

// Every member of comm calls the same Sendrecv together (the reference's halo
// exchanges are symmetric), so one rendezvous pairs each receive with its sender.
int MPI_Sendrecv(const void* sendbuf, int sendcount, MPI_Datatype sendtype, int dest, int sendtag,
                 void* recvbuf, int recvcount, MPI_Datatype recvtype, int source, int recvtag,
                 MPI_Comm comm, MPI_Status* status) {
    const int me = my_index(comm);
    Slot& s = comm->slots[me];
    s.send = sendbuf;
    s.count = (long long)sendcount * sendtype;
    s.dest = dest;
    s.tag = sendtag;
    if (!rendezvous(comm)) give_up("MPI_Sendrecv");
    const Slot& from = comm->slots[source];
    if (from.dest != me || from.tag != recvtag || from.count != (long long)recvcount * recvtype) {
        std::fprintf(stderr, "mpi stand-in: MPI_Sendrecv mismatch (rank %d from %d, tag %d/%d)\n",
                     me, source, from.tag, recvtag);
        std::_Exit(99);
    }
    copy_bytes(recvbuf, from.send, (size_t)from.count);
    if (status) { status->source = source; status->tag = recvtag; }
    if (!rendezvous(comm)) give_up("MPI_Sendrecv");
    return MPI_SUCCESS;
}

int MPI_Reduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type, MPI_Op op,
               int root, MPI_Comm comm) {
    const int me = my_index(comm);
    comm->slots[me].send = sendbuf;
    if (!rendezvous(comm)) give_up("MPI_Reduce");
    if (me == root) {
        const bool is_int = (type == MPI_LONG_LONG);   // 8-byte types: long long here
        for (int k = 0; k < count; ++k) {
            if (type == MPI_INT) {
                int acc = static_cast<const int*>(comm->slots[0].send)[k];
                for (size_t j = 1; j < comm->members.size(); ++j) {
                    int v = static_cast<const int*>(comm->slots[j].send)[k];
                    acc = (op == MPI_MAX) ? std::max(acc, v) : acc + v;
                }
                static_cast<int*>(recvbuf)[k] = acc;
            } else if (is_int) {
                long long acc = static_cast<const long long*>(comm->slots[0].send)[k];
                for (size_t j = 1; j < comm->members.size(); ++j) {
                    long long v = static_cast<const long long*>(comm->slots[j].send)[k];
                    acc = (op == MPI_MAX) ? std::max(acc, v) : acc + v;
                }
                static_cast<long long*>(recvbuf)[k] = acc;
            }
        }
    }
    if (!rendezvous(comm)) give_up("MPI_Reduce");
    return MPI_SUCCESS;
}

int zr_run_ranks(int nranks, void (*fn)(int, void*), void* arg) {
    std::lock_guard<std::mutex> run_lock(g_run_m);
    World w;
    g_world = &w;
    std::vector<int> all(nranks);
    for (int i = 0; i < nranks; ++i) all[i] = i;
    w.world = new_comm(all);
    std::vector<std::thread> threads;
    for (int r = 0; r < nranks; ++r)
        threads.emplace_back([r, fn, arg] { tl_rank = r; fn(r, arg); });
    for (auto& t : threads) t.join();
    int failed = w.failed.load();
    g_world = nullptr;
    return failed ? -1 : 0;
}

}  // extern "C"
