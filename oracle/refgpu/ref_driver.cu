// Driver for the reference's own GPU pipeline -- TEST INFRASTRUCTURE ONLY.
//
// Compiled together with the unmodified reference sources (zmodel/utils.cu,
// zmodel/transforms/fft.cu, fft3d.cu, zmodel/stencils/laplace.cu, laplace3d.cu, dx.cu,
// dy.cu), cuFFT and the in-process MPI stand-in of mpi_shim.cpp, for one compile-time
// (N_DIM, B_DIM, P_DIM), into oracle/_ref/libzref_gpu_*.so.  Each extern "C" entry runs
// every virtual rank of the reference as one host thread on the current GPU and calls
// the reference's entry points exactly as its test drivers do, once per fresh input
// (never test_fft's RUNS loop, which re-transforms the clobbered buf0, fft.cu:596-599):
//   2D FFT   fft.cu:518-612     (init_plans, init_buffers, forward_fft / inverse_fft)
//   3D FFT   fft3d.cu:637-745   (dep/row/col splits, init_plans_3d, forward_fft_3d ...)
//   2D Laplacian  laplace.cu:260-330  (pack_laplace, communicate_laplace, laplace)
//   3D Laplacian  laplace3d.cu:365-445
//   dx / dy  dx.cu:163-210, dy.cu:187-235 (halos packed on the host by the reference's own
//            pack_dx_* / pack_dy_* functions, from the neighbour ranks' actual data)
// Whole-grid arrays are rank-major: rank id's rank-local array at offset id * L^dim.
#include <mpi.h>

#include "transforms/fft.h"
#include "stencils/laplace.h"

#include <chrono>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

// Reference functions that its headers do not declare (defined in laplace3d.cu, dx.cu, dy.cu).
void init_laplace_buffers_3d(LaplaceBuffers3d& laplace_buffers);
void destroy_laplace_buffers_3d(LaplaceBuffers3d& laplace_buffers);
__global__ void pack_laplace_3d(Complex* device_in, LaplaceBuffers3d laplace_buffers);
__global__ void laplace_3d(Complex* device_in, Complex* device_out, LaplaceBuffers3d laplace_buffers,
                           int rid, int cid, int did);
void communicate_laplace_3d(LaplaceBuffers3d& laplace_buffers, MPI_Comm& row_comm, MPI_Comm& col_comm,
                            MPI_Comm& dep_comm, int rid, int cid, int did);
__global__ void dx(Scalar* device_in, Scalar* device_out, int rid, int cid, Scalar delta,
                   Scalar* device_packed_left0, Scalar* device_packed_left1,
                   Scalar* device_packed_right0, Scalar* device_packed_right1);
__global__ void dy(Scalar* device_in, Scalar* device_out, int rid, int cid, Scalar delta,
                   Scalar* device_packed_above0, Scalar* device_packed_above1,
                   Scalar* device_packed_below0, Scalar* device_packed_below1);
void pack_dx_left0(Scalar* in, Scalar* packed);
void pack_dx_left1(Scalar* in, Scalar* packed);
void pack_dx_right0(Scalar* in, Scalar* packed);
void pack_dx_right1(Scalar* in, Scalar* packed);
void pack_dy_top0(Scalar* in, Scalar* packed);
void pack_dy_top1(Scalar* in, Scalar* packed);
void pack_dy_bottom0(Scalar* in, Scalar* packed);
void pack_dy_bottom1(Scalar* in, Scalar* packed);

namespace {

enum Kind { FFT2D = 0, FFT3D = 1, LAP2D = 2, LAP3D = 3 };

struct Job {
    int kind = FFT2D;
    bool inverse = false;
    bool do_compute = true;
    Complex scale{1.0, 0.0};
    const Complex* in = nullptr;
    Complex* out = nullptr;
    int reps = 0;            // timed calls (after one untimed warm-up call when > 0)
    double ms_total = 0.0;   // rank 0: sum of the timed calls (barrier to barrier)
};

double now_ms() {
    return std::chrono::duration<double, std::milli>(
               std::chrono::steady_clock::now().time_since_epoch()).count();
}

#define ZR_CHECK(x)                                                                        \
    do {                                                                                   \
        cudaError_t e_ = (x);                                                              \
        if (e_ != cudaSuccess) {                                                           \
            std::fprintf(stderr, "ref driver: %s failed: %s\n", #x, cudaGetErrorString(e_)); \
            std::_Exit(96);                                                                \
        }                                                                                  \
    } while (0)

// One timed region per call, as the reference's TOTAL timer brackets it (fft.cu:202-338):
// world barrier, the call, device sync, world barrier.
template <typename Load, typename Call>
void timed_calls(int id, Job* j, Load&& load_input, Call&& call) {
    const int calls = j->reps > 0 ? j->reps + 1 : 1;
    for (int c = 0; c < calls; ++c) {
        load_input();
        MPI_Barrier(MPI_COMM_WORLD);
        const double t0 = now_ms();
        call();
        ZR_CHECK(cudaDeviceSynchronize());
        MPI_Barrier(MPI_COMM_WORLD);
        const double t1 = now_ms();
        if (id == 0 && j->reps > 0 && c > 0) j->ms_total += t1 - t0;
    }
}

}  // namespace

namespace {

template <bool C>
void fft2d_rank(int id, Job* j) {
    const int rid = id / P_DIM, cid = id % P_DIM;           // fft.cu:561-567
    MPI_Comm row_comm, col_comm;
    MPI_Comm_split(MPI_COMM_WORLD, rid, id, &row_comm);
    MPI_Comm_split(MPI_COMM_WORLD, cid, id, &col_comm);
    FftHostPlans host_plans;
    init_plans(host_plans);
    FftdxFft1Ctx ctx1;
    FftBuffers buffers;
    init_buffers<true>(buffers, rid, cid);
    const size_t n = (size_t)LOCAL_DIM * LOCAL_DIM;
    timed_calls(id, j,
        [&] { ZR_CHECK(cudaMemcpy(buffers.device_buf0, j->in + id * n, LOCAL_COMPLEX_BYTES,
                                  cudaMemcpyHostToDevice)); },
        [&] {
            if (j->inverse) inverse_fft<C>(buffers, row_comm, col_comm, id, j->scale, host_plans);
            else forward_fft<C>(buffers, row_comm, col_comm, id, host_plans, ctx1);
        });
    ZR_CHECK(cudaMemcpy(j->out + id * n, buffers.device_buf1, LOCAL_COMPLEX_BYTES, cudaMemcpyDeviceToHost));
    destroy_plans(host_plans);
    destroy_buffers<true>(buffers);
}

template <bool C>
void fft3d_rank(int id, Job* j) {
    const int did = id / (P_DIM * P_DIM);                   // fft3d.cu:676-697
    const int rid = (id % (P_DIM * P_DIM)) / P_DIM;
    const int cid = id % P_DIM;
    MPI_Comm row_comm, col_comm, dep_comm;
    MPI_Comm_split(MPI_COMM_WORLD, rid * P_DIM + cid, id, &dep_comm);
    MPI_Comm_split(MPI_COMM_WORLD, did * P_DIM + rid, id, &row_comm);
    MPI_Comm_split(MPI_COMM_WORLD, did * P_DIM + cid, id, &col_comm);
    FftHostPlans host_plans;
    init_plans_3d(host_plans);
    FftdxFft1Ctx ctx1;
    FftBuffers buffers;
    init_buffers_3d<true>(buffers, rid, cid, did);
    const size_t n = (size_t)LOCAL_DIM * LOCAL_DIM * LOCAL_DIM;
    timed_calls(id, j,
        [&] { ZR_CHECK(cudaMemcpy(buffers.device_buf0, j->in + id * n, LOCAL_COMPLEX_BYTES_3D,
                                  cudaMemcpyHostToDevice)); },
        [&] {
            if (j->inverse)
                inverse_fft_3d<C>(buffers, row_comm, col_comm, dep_comm, id, j->scale, host_plans);
            else
                forward_fft_3d<C>(buffers, row_comm, col_comm, dep_comm, id, host_plans, ctx1);
        });
    ZR_CHECK(cudaMemcpy(j->out + id * n, buffers.device_buf1, LOCAL_COMPLEX_BYTES_3D, cudaMemcpyDeviceToHost));
    destroy_plans_3d(host_plans);
    destroy_buffers_3d<true>(buffers);
}

void lap2d_rank(int id, Job* j) {
    const int rid = id / P_DIM, cid = id % P_DIM;           // laplace.cu:287-297
    MPI_Comm row_comm, col_comm;
    MPI_Comm_split(MPI_COMM_WORLD, rid, id, &row_comm);
    MPI_Comm_split(MPI_COMM_WORLD, cid, id, &col_comm);
    Complex *buf0 = nullptr, *buf1 = nullptr;
    ZR_CHECK(cudaMalloc((void**)&buf0, LOCAL_COMPLEX_BYTES));
    ZR_CHECK(cudaMalloc((void**)&buf1, LOCAL_COMPLEX_BYTES));
    LaplaceBuffers lb;
    init_laplace_buffers(lb);
    const size_t n = (size_t)LOCAL_DIM * LOCAL_DIM;
    timed_calls(id, j,
        [&] { ZR_CHECK(cudaMemcpy(buf0, j->in + id * n, LOCAL_COMPLEX_BYTES, cudaMemcpyHostToDevice)); },
        [&] {                                               // laplace.cu:317-330
            pack_laplace<<<LOCAL_DIM, LOCAL_DIM>>>(buf0, lb);
            ZR_CHECK(cudaDeviceSynchronize());
            communicate_laplace(lb, row_comm, col_comm, rid, cid);
            MPI_Barrier(MPI_COMM_WORLD);
            laplace<<<VEC_TOTAL, VEC>>>(buf0, buf1, lb, rid, cid);
        });
    ZR_CHECK(cudaMemcpy(j->out + id * n, buf1, LOCAL_COMPLEX_BYTES, cudaMemcpyDeviceToHost));
    destroy_laplace_buffers(lb);
    ZR_CHECK(cudaFree(buf0));
    ZR_CHECK(cudaFree(buf1));
}

void lap3d_rank(int id, Job* j) {
    const int did = id / (P_DIM * P_DIM);                   // laplace3d.cu:385-405
    const int rid = (id % (P_DIM * P_DIM)) / P_DIM;
    const int cid = id % P_DIM;
    MPI_Comm row_comm, col_comm, dep_comm;
    MPI_Comm_split(MPI_COMM_WORLD, rid * P_DIM + cid, id, &dep_comm);
    MPI_Comm_split(MPI_COMM_WORLD, did * P_DIM + rid, id, &row_comm);
    MPI_Comm_split(MPI_COMM_WORLD, did * P_DIM + cid, id, &col_comm);
    Complex *buf0 = nullptr, *buf1 = nullptr;
    ZR_CHECK(cudaMalloc((void**)&buf0, LOCAL_COMPLEX_BYTES_3D));
    ZR_CHECK(cudaMalloc((void**)&buf1, LOCAL_COMPLEX_BYTES_3D));
    LaplaceBuffers3d lb;
    init_laplace_buffers_3d(lb);
    const size_t n = (size_t)LOCAL_DIM * LOCAL_DIM * LOCAL_DIM;
    timed_calls(id, j,
        [&] { ZR_CHECK(cudaMemcpy(buf0, j->in + id * n, LOCAL_COMPLEX_BYTES_3D, cudaMemcpyHostToDevice)); },
        [&] {                                               // laplace3d.cu:430-445
            dim3 grid_pack(LOCAL_DIM, LOCAL_DIM);
            pack_laplace_3d<<<grid_pack, LOCAL_DIM>>>(buf0, lb);
            ZR_CHECK(cudaDeviceSynchronize());
            communicate_laplace_3d(lb, row_comm, col_comm, dep_comm, rid, cid, did);
            MPI_Barrier(MPI_COMM_WORLD);
            dim3 grid_stencil(LOCAL_DIM, VEC_TOTAL);
            laplace_3d<<<grid_stencil, VEC>>>(buf0, buf1, lb, rid, cid, did);
        });
    ZR_CHECK(cudaMemcpy(j->out + id * n, buf1, LOCAL_COMPLEX_BYTES_3D, cudaMemcpyDeviceToHost));
    destroy_laplace_buffers_3d(lb);
    ZR_CHECK(cudaFree(buf0));
    ZR_CHECK(cudaFree(buf1));
}

void run_rank(int id, void* arg) {
    Job* j = static_cast<Job*>(arg);
    switch (j->kind) {
        case FFT2D: j->do_compute ? fft2d_rank<true>(id, j) : fft2d_rank<false>(id, j); break;
        case FFT3D: j->do_compute ? fft3d_rank<true>(id, j) : fft3d_rank<false>(id, j); break;
        case LAP2D: lap2d_rank(id, j); break;
        case LAP3D: lap3d_rank(id, j); break;
    }
}

// Runs one job over all ranks with std::cout (the reference's stage-timing prints)
// captured into `log`.
int run_job(Job& j, int ranks, char* log, int loglen) {
    std::ostringstream captured;
    std::streambuf* old = std::cout.rdbuf(captured.rdbuf());
    const int rc = zr_run_ranks(ranks, run_rank, &j);
    std::cout.rdbuf(old);
    if (log && loglen > 0) {
        const std::string s = captured.str();
        const size_t k = std::min(s.size(), (size_t)loglen - 1);
        std::memcpy(log, s.data(), k);
        log[k] = '\0';
    }
    return rc;
}

}  // namespace

extern "C" {

// The layout this library was compiled for, and whether its All-to-Alls and halo
// exchanges pass device pointers (__GPU__AWARE__MPI__) or stage through host memory
// (the reference's default, utils.h:21).
int zr_config(int* n, int* b, int* p, int* gpu_aware) {
    *n = N_DIM;
    *b = B_DIM;
    *p = P_DIM;
#ifdef __GPU__AWARE__MPI__
    *gpu_aware = 1;
#else
    *gpu_aware = 0;
#endif
    return 0;
}

// forward_fft / inverse_fft (dim 2) or forward_fft_3d / inverse_fft_3d (dim 3) over the
// whole grid: `in` -> `out` (host arrays of N^dim complex128, rank-major).  reps > 0:
// one warm-up call, then `reps` timed calls; *ms = mean barrier-to-barrier time.
int zr_fft(int dim, const void* in, void* out, int inverse, int do_compute,
           double scale_re, double scale_im, int reps, double* ms, char* log, int loglen) {
    if (dim != 2 && dim != 3) return -2;
    Job j;
    j.kind = dim == 2 ? FFT2D : FFT3D;
    j.inverse = inverse != 0;
    j.do_compute = do_compute != 0;
    j.scale = Complex{scale_re, scale_im};
    j.in = static_cast<const Complex*>(in);
    j.out = static_cast<Complex*>(out);
    j.reps = reps;
    const int ranks = dim == 2 ? P_DIM * P_DIM : P_DIM * P_DIM * P_DIM;
    const int rc = run_job(j, ranks, log, loglen);
    if (ms) *ms = reps > 0 ? j.ms_total / reps : 0.0;
    return rc;
}

// pack_laplace + communicate_laplace + laplace (dim 2), or the 3D chain, `in` -> `out`.
int zr_laplace(int dim, const void* in, void* out, int reps, double* ms, char* log, int loglen) {
    if (dim != 2 && dim != 3) return -2;
    Job j;
    j.kind = dim == 2 ? LAP2D : LAP3D;
    j.in = static_cast<const Complex*>(in);
    j.out = static_cast<Complex*>(out);
    j.reps = reps;
    const int ranks = dim == 2 ? P_DIM * P_DIM : P_DIM * P_DIM * P_DIM;
    const int rc = run_job(j, ranks, log, loglen);
    if (ms) *ms = reps > 0 ? j.ms_total / reps : 0.0;
    return rc;
}

// The reference's dx (axis 0) or dy (axis 1) kernel on every rank of a real 2D field
// (N^2 doubles, rank-major).  The reference fills the halos of its one-rank test on the
// host (init_packed_dx, dx.cu:143-161; init_packed_dy, dy.cu:167-185); here the same host
// pack functions read the neighbour ranks' parts of `in`.  Needs B_DIM >= 2 (dx.cu:100).
int zr_dxdy(int axis, const double* in, double* out, double delta) {
    if (B_DIM < 2) return -3;
    const size_t n = (size_t)LOCAL_DIM * LOCAL_DIM;
    const size_t halo = axis == 0 ? (size_t)PACKED_COL_SCALAR_BYTES : (size_t)PACKED_ROW_SCALAR_BYTES;
    std::vector<Scalar> rank_in(n), h0(halo / sizeof(Scalar)), h1(h0.size()), h2(h0.size()), h3(h0.size());
    std::vector<Scalar> nb_a(n), nb_b(n);
    Scalar *d_in, *d_out, *d_h[4];
    ZR_CHECK(cudaMalloc((void**)&d_in, LOCAL_SCALAR_BYTES));
    ZR_CHECK(cudaMalloc((void**)&d_out, LOCAL_SCALAR_BYTES));
    for (auto& p : d_h) ZR_CHECK(cudaMalloc((void**)&p, halo));
    for (int rid = 0; rid < P_DIM; ++rid) {
        for (int cid = 0; cid < P_DIM; ++cid) {
            const int id = rid * P_DIM + cid;
            std::memcpy(rank_in.data(), in + id * n, LOCAL_SCALAR_BYTES);
            if (axis == 0) {
                const int left = rid * P_DIM + (cid + P_DIM - 1) % P_DIM;
                const int right = rid * P_DIM + (cid + 1) % P_DIM;
                std::memcpy(nb_a.data(), in + left * n, LOCAL_SCALAR_BYTES);
                std::memcpy(nb_b.data(), in + right * n, LOCAL_SCALAR_BYTES);
                pack_dx_right0(nb_a.data(), h0.data());   // left0
                pack_dx_right1(nb_a.data(), h1.data());   // left1
                pack_dx_left0(nb_b.data(), h2.data());    // right0
                pack_dx_left1(nb_b.data(), h3.data());    // right1
            } else {
                const int above = ((rid + P_DIM - 1) % P_DIM) * P_DIM + cid;
                const int below = ((rid + 1) % P_DIM) * P_DIM + cid;
                std::memcpy(nb_a.data(), in + above * n, LOCAL_SCALAR_BYTES);
                std::memcpy(nb_b.data(), in + below * n, LOCAL_SCALAR_BYTES);
                pack_dy_bottom0(nb_a.data(), h0.data());  // above0
                pack_dy_bottom1(nb_a.data(), h1.data());  // above1
                pack_dy_top0(nb_b.data(), h2.data());     // below0
                pack_dy_top1(nb_b.data(), h3.data());     // below1
            }
            ZR_CHECK(cudaMemcpy(d_in, rank_in.data(), LOCAL_SCALAR_BYTES, cudaMemcpyHostToDevice));
            ZR_CHECK(cudaMemcpy(d_h[0], h0.data(), halo, cudaMemcpyHostToDevice));
            ZR_CHECK(cudaMemcpy(d_h[1], h1.data(), halo, cudaMemcpyHostToDevice));
            ZR_CHECK(cudaMemcpy(d_h[2], h2.data(), halo, cudaMemcpyHostToDevice));
            ZR_CHECK(cudaMemcpy(d_h[3], h3.data(), halo, cudaMemcpyHostToDevice));
            if (axis == 0)
                dx<<<VEC_TOTAL, VEC>>>(d_in, d_out, rid, cid, delta, d_h[0], d_h[1], d_h[2], d_h[3]);
            else
                dy<<<VEC_TOTAL, VEC>>>(d_in, d_out, rid, cid, delta, d_h[0], d_h[1], d_h[2], d_h[3]);
            ZR_CHECK(cudaGetLastError());
            ZR_CHECK(cudaDeviceSynchronize());
            ZR_CHECK(cudaMemcpy(out + id * n, d_out, LOCAL_SCALAR_BYTES, cudaMemcpyDeviceToHost));
        }
    }
    ZR_CHECK(cudaFree(d_in));
    ZR_CHECK(cudaFree(d_out));
    for (auto p : d_h) ZR_CHECK(cudaFree(p));
    return 0;
}

}  // extern "C"
