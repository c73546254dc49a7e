// zmodel_compat.hpp -- C++ drop-in for StencilFFT's zmodel entry points on top of the
// libzmodel_b200 C ABI (zmodel_b200.h).
//
// The reference is SPMD over MPI: every rank calls, e.g.,
//   forward_fft<do_compute>(FftBuffers&, MPI_Comm& row, MPI_Comm& col, int id,
//                           FftHostPlans&, FftdxFft1Ctx&)          (zmodel/transforms/fft.h:36-38)
// on its own L x L slice.  Here the P x P (P^3) ranks are virtual ranks inside one
// GPU, so one call covers the whole grid: the buffers are whole-grid device buffers
// (rank-major, each rank in the reference's layout), and the communicator / rank-id
// arguments disappear into the plan.  Names, argument order and the buffer contract
// (input in device_buf0, output in device_buf1, buf0 used as scratch) follow the
// reference.  Errors end the process with a message, like the reference's
// DEVICE_RT_SAFE_CALL / DEVICE_FFT_SAFE_CALL (zmodel/device_macros.h:112-152); the C ABI
// underneath only returns status codes.
#pragma once

#include <cstdio>
#include <cstdlib>

#include "zmodel_b200.h"

namespace zmodel_b200 {

struct Complex { double x, y; };   // cufftDoubleComplex layout (zmodel/utils.h:9)

#define ZM_COMPAT_CHECK(call)                                                          \
    do {                                                                               \
        int zm_rc_ = (call);                                                           \
        if (zm_rc_ != ZM_OK) {                                                         \
            std::fprintf(stderr, "zmodel_b200 error %d (%s) at %s:%d: %s\n", zm_rc_,   \
                         zm_status_string(zm_rc_), __FILE__, __LINE__,                 \
                         zm_last_error_string());                                      \
            std::exit(1);                                                              \
        }                                                                              \
    } while (0)

// FftHostPlans (zmodel/transforms/fft_host_plans.h:6-10): the cuFFT plans and streams
// become one compute plan and one data-movement-only plan (do_compute = false).
struct FftHostPlans {
    zm_plan plan = nullptr;
    zm_plan permute = nullptr;
    int dim = 2;
};

// FftBuffers (zmodel/transforms/fft.h:9-26): only the device buffers remain; the
// pinned host staging buffers and the L x L twiddle tables are not needed.  `work`
// is optional: nullptr uses the plan's own workspace (init_plans default), or buf0 as
// scratch when the plan has none (the reference's behaviour).
struct FftBuffers {
    void *device_buf0 = nullptr;
    void *device_buf1 = nullptr;
    void *work = nullptr;
};

// The compute plan owns one field of workspace by default (ZM_FLAG_OWN_WORKSPACE), so
// forward_fft / inverse_fft with buffers.work == nullptr run the out-of-place
// configurations (the fast ones; buf0 is then left intact, which the reference's
// contract permits).  The reference's init_buffers holds more than that: two to three
// fields of L x L twiddle tables per rank (fft.cu:75-108).  own_workspace = false keeps
// device memory to the caller's buffers and uses buf0 as scratch.
inline void init_plans(FftHostPlans &p, long long n, long long b, long long pdim,
                       int dtype = ZM_C128, bool own_workspace = true) {
    p.dim = 2;
    ZM_COMPAT_CHECK(zm_plan_create(&p.plan, 2, n, b, pdim, dtype,
                                   own_workspace ? ZM_FLAG_OWN_WORKSPACE : 0u));
    ZM_COMPAT_CHECK(zm_plan_create(&p.permute, 2, n, b, pdim, dtype, ZM_FLAG_PERMUTE_ONLY));
}
inline void init_plans_3d(FftHostPlans &p, long long n, long long b, long long pdim,
                          int dtype = ZM_C128, bool own_workspace = true) {
    p.dim = 3;
    ZM_COMPAT_CHECK(zm_plan_create(&p.plan, 3, n, b, pdim, dtype,
                                   own_workspace ? ZM_FLAG_OWN_WORKSPACE : 0u));
    ZM_COMPAT_CHECK(zm_plan_create(&p.permute, 3, n, b, pdim, dtype, ZM_FLAG_PERMUTE_ONLY));
}
#if defined(N_DIM) && defined(B_DIM) && defined(P_DIM)
// The reference's compile-time sizes (zmodel/utils.h:27-38) as defaults.
inline void init_plans(FftHostPlans &p) { init_plans(p, N_DIM, B_DIM, P_DIM); }
inline void init_plans_3d(FftHostPlans &p) { init_plans_3d(p, N_DIM, B_DIM, P_DIM); }
#endif
inline void destroy_plans(FftHostPlans &p) {
    if (p.plan) ZM_COMPAT_CHECK(zm_plan_destroy(p.plan));
    if (p.permute) ZM_COMPAT_CHECK(zm_plan_destroy(p.permute));
    p.plan = p.permute = nullptr;
}
inline void destroy_plans_3d(FftHostPlans &p) { destroy_plans(p); }

// forward_fft<do_compute> / forward_fft_3d<do_compute> (fft.cu:199, fft3d.cu:234):
// device_buf0 (real layout) -> device_buf1 (reciprocal layout).
template <bool do_compute>
inline void forward_fft(FftBuffers &b, FftHostPlans &p, void *stream = nullptr) {
    ZM_COMPAT_CHECK(zm_fft_forward(do_compute ? p.plan : p.permute, b.device_buf0, b.device_buf1,
                                   b.work, stream));
}
template <bool do_compute>
inline void forward_fft_3d(FftBuffers &b, FftHostPlans &p, void *stream = nullptr) {
    forward_fft<do_compute>(b, p, stream);
}

// inverse_fft<do_compute> / inverse_fft_3d<do_compute> (fft.cu:409, fft3d.cu:508):
// device_buf0 (reciprocal layout) -> device_buf1 (real layout), times `scale`.
template <bool do_compute>
inline void inverse_fft(FftBuffers &b, Complex scale, FftHostPlans &p, void *stream = nullptr) {
    ZM_COMPAT_CHECK(zm_fft_inverse(do_compute ? p.plan : p.permute, b.device_buf0, b.device_buf1,
                                   b.work, scale.x, scale.y, stream));
}
template <bool do_compute>
inline void inverse_fft_3d(FftBuffers &b, Complex scale, FftHostPlans &p, void *stream = nullptr) {
    inverse_fft<do_compute>(b, scale, p, stream);
}

// laplace / laplace_3d (laplace.cu:73, laplace3d.cu:90) with pack + communicate folded in.
// inv_h2 = 1 reproduces the reference (it has no 1/h^2 factor).
inline void laplace(const void *device_in, void *device_out, FftHostPlans &p, double inv_h2 = 1.0,
                    void *stream = nullptr) {
    ZM_COMPAT_CHECK(zm_laplace(p.plan, device_in, device_out, inv_h2, stream));
}
inline void laplace_3d(const void *device_in, void *device_out, FftHostPlans &p,
                       double inv_h2 = 1.0, void *stream = nullptr) {
    laplace(device_in, device_out, p, inv_h2, stream);
}
// dx / dy (dx.cu:10, dy.cu:10) on the reference's real Scalar field.
inline void dx(const double *device_in, double *device_out, double delta, FftHostPlans &p,
               void *stream = nullptr) {
    ZM_COMPAT_CHECK(zm_dx_real(p.plan, device_in, device_out, delta, stream));
}
inline void dy(const double *device_in, double *device_out, double delta, FftHostPlans &p,
               void *stream = nullptr) {
    ZM_COMPAT_CHECK(zm_dy_real(p.plan, device_in, device_out, delta, stream));
}

// Index maps with the reference's argument order (zmodel/utils.h:166-320).
inline void real_to_global(FftHostPlans &p, int rid, int cid, int lr, int lc, int &gr, int &gc) {
    int64_t a, b, c;
    ZM_COMPAT_CHECK(zm_real_to_global(p.plan, rid, cid, 0, 0, lr, lc, &a, &b, &c));
    gr = (int)b; gc = (int)c;
}
inline void global_to_real(FftHostPlans &p, int gr, int gc, int &rid, int &cid, int &lr, int &lc) {
    int64_t r, c, d, ld, l1, l2;
    ZM_COMPAT_CHECK(zm_global_to_real(p.plan, 0, gr, gc, &r, &c, &d, &ld, &l1, &l2));
    rid = (int)r; cid = (int)c; lr = (int)l1; lc = (int)l2;
}
inline void reciprocal_to_global(FftHostPlans &p, int rid, int cid, int local_row, int local_col,
                                 int &ky, int &kx) {
    int64_t a, b, c;
    ZM_COMPAT_CHECK(zm_reciprocal_to_global(p.plan, rid, cid, 0, 0, local_row, local_col, &a, &b, &c));
    ky = (int)b; kx = (int)c;
}
inline void global_to_reciprocal(FftHostPlans &p, int ky, int kx, int &rid, int &cid, int &local_row,
                                 int &local_col) {
    int64_t r, c, d, ld, l1, l2;
    ZM_COMPAT_CHECK(zm_global_to_reciprocal(p.plan, 0, ky, kx, &r, &c, &d, &ld, &l1, &l2));
    rid = (int)r; cid = (int)c; local_row = (int)l1; local_col = (int)l2;
}
inline void reciprocal_to_global_3d(FftHostPlans &p, int rid, int cid, int did, int ld, int lr, int lc,
                                    int &kd, int &kr, int &kc) {
    int64_t a, b, c;
    ZM_COMPAT_CHECK(zm_reciprocal_to_global(p.plan, rid, cid, did, ld, lr, lc, &a, &b, &c));
    kd = (int)a; kr = (int)b; kc = (int)c;
}
inline void global_to_reciprocal_3d(FftHostPlans &p, int kd, int kr, int kc, int &rid, int &cid,
                                    int &did, int &ld, int &lr, int &lc) {
    int64_t r, c, d, l0, l1, l2;
    ZM_COMPAT_CHECK(zm_global_to_reciprocal(p.plan, kd, kr, kc, &r, &c, &d, &l0, &l1, &l2));
    rid = (int)r; cid = (int)c; did = (int)d; ld = (int)l0; lr = (int)l1; lc = (int)l2;
}
inline void real_to_global_3d(FftHostPlans &p, int rid, int cid, int did, int ld, int lr, int lc,
                              int &gd, int &gr, int &gc) {
    int64_t a, b, c;
    ZM_COMPAT_CHECK(zm_real_to_global(p.plan, rid, cid, did, ld, lr, lc, &a, &b, &c));
    gd = (int)a; gr = (int)b; gc = (int)c;
}
inline void global_to_real_3d(FftHostPlans &p, int gd, int gr, int gc, int &rid, int &cid, int &did,
                              int &ld, int &lr, int &lc) {
    int64_t r, c, d, l0, l1, l2;
    ZM_COMPAT_CHECK(zm_global_to_real(p.plan, gd, gr, gc, &r, &c, &d, &l0, &l1, &l2));
    rid = (int)r; cid = (int)c; did = (int)d; ld = (int)l0; lr = (int)l1; lc = (int)l2;
}

}  // namespace zmodel_b200
