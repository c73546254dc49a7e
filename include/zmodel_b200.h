/*
 * zmodel_b200.h -- C ABI of the B200 (sm_100a) interleaved block-cyclic FFT and
 * stencil library (libzmodel_b200.so).
 *
 * One plan describes a whole N x N (N^3) field dealt block-cyclically in B x B
 * blocks over a P x P (P^3) grid of *virtual ranks*, all held in one GPU's HBM:
 * the field is one contiguous device buffer of P^2 (P^3) rank sub-buffers in
 * rank-id order (2D id = rid*P + cid, 3D id = did*P^2 + rid*P + cid), each rank
 * holding exactly StencilFFT's rank-local L x L (L^3) array, L = N/P, with the
 * vector-packed columns of zmodel/utils.h:98-128.  Forward transforms take the
 * real-space layout to the reciprocal layout of zmodel/utils.h:254-320 (no final
 * digit reversal), inverse transforms the other way.  The MPI All-to-All and halo
 * exchanges of the reference become permutations inside the kernels.
 *
 * Elements are interleaved complex: complex128 = {double re, im} (16 bytes),
 * complex64 = {float re, im} (8 bytes).  All calls are asynchronous on the
 * caller's stream (a cudaStream_t passed as void*, NULL = legacy default stream),
 * allocate nothing and never synchronise the device, so they can be captured in
 * a CUDA graph.  Every call returns a status code (ZM_OK = 0) and never exits
 * the process; zm_last_error_string() describes the last failure of the calling
 * thread.  The reference instead aborts on any CUDA/cuFFT error
 * (zmodel/device_macros.h:112-152).
 */
#ifndef ZMODEL_B200_H
#define ZMODEL_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ status codes */
enum zm_status {
    ZM_OK = 0,
    ZM_ERR_INVALID_ARG = 1,   /* null plan/pointer, unknown dtype/flag, overlapping buffers */
    ZM_ERR_CONSTRAINT = 2,    /* N, B, P break the layout constraints (B | L, P | VEC, powers of two) */
    ZM_ERR_MISALIGNED = 3,    /* a field pointer is not 16-byte aligned */
    ZM_ERR_NO_MEMORY = 4,     /* device or host allocation failed (plan creation only) */
    ZM_ERR_CUDA = 5,          /* CUDA runtime / launch error */
    ZM_ERR_TIMEOUT = 6,       /* a bounded device-side wait gave up (batched launches) */
    ZM_ERR_UNSUPPORTED = 7,   /* valid request this build does not support (e.g. dx/dy with B < 2) */
    ZM_ERR_WORKSPACE = 8      /* workspace required but too small */
};

/* Element types. */
enum zm_dtype {
    ZM_C128 = 0,   /* complex128, FP64 arithmetic (the reference's Complex, zmodel/utils.h:9) */
    ZM_C64 = 1     /* complex64 bulk form; twiddles generated in FP64, stored as split
                      hi/lo FP32 pairs and applied as compensated products */
};

/* Plan flags. */
#define ZM_FLAG_PERMUTE_ONLY 0x1u  /* data movement only, no FFT arithmetic and unit twiddles:
                                      the reference built with __ZMODEL__COMPUTE__ off
                                      (zmodel/transforms/fft.cu:176-180, 211-213) */
#define ZM_FLAG_HOST_ONLY 0x2u     /* no device resources: the plan answers zm_plan_get_info and
                                      the index maps only (device calls return ZM_ERR_UNSUPPORTED) */
#define ZM_FLAG_OWN_WORKSPACE 0x4u /* the plan allocates one field of workspace at creation and
                                      uses it whenever a transform is called with work = NULL:
                                      the input is then preserved and the 2D transforms take their
                                      out-of-place configurations.  Calls that pass work = NULL
                                      share that workspace, so they must not overlap on the GPU
                                      (two streams at once); pass separate workspaces there. */

typedef struct zm_plan_s *zm_plan;

/* Derived sizes of a plan (zmodel/utils.h:45-71, fft_host_plans.h:25-60). */
typedef struct zm_plan_info {
    int dim;                 /* 2 or 3 */
    int dtype;               /* zm_dtype */
    int64_t n, b, p;         /* N_DIM, B_DIM, P_DIM */
    int64_t local_dim;       /* L = N / P */
    int64_t vec;             /* VEC = L / B: FFT1a length */
    int64_t vec_split;       /* VP = VEC / P: FFT1b stride */
    int64_t m;               /* M = B * P: FFT1b length */
    int64_t ranks;           /* P^2 or P^3 virtual ranks */
    int64_t rank_elems;      /* L^2 or L^3 */
    int64_t total_elems;     /* N^2 or N^3 */
    size_t elem_bytes;       /* 16 (c128) or 8 (c64) */
    size_t field_bytes;      /* total_elems * elem_bytes */
    size_t workspace_bytes;  /* see zm_plan_workspace_size */
} zm_plan_info;

/*
 * Plan lifetime.  Replaces init_plans / init_plans_3d (fft_host_plans.h:14,75),
 * init_buffers / init_buffers_3d twiddle setup (fft.cu:75-108, fft3d.cu:70-136),
 * init_laplace_buffers (laplace.cu:26) and the communicator setup
 * (fft.cu:561-567, fft3d.cu:685-697).  Creation validates N, B, P
 * (powers of two, B | L, P | VEC) and allocates the FP64-generated twiddle
 * table on the current device.  A plan is immutable after creation and may be
 * used concurrently from several streams given separate workspaces.
 */
int zm_plan_create(zm_plan *plan, int dim, int64_t n, int64_t b, int64_t p, int dtype,
                   unsigned flags);
int zm_plan_destroy(zm_plan plan);   /* destroy_plans / destroy_buffers (fft_host_plans.h:63, fft.cu:110) */
int zm_plan_get_info(zm_plan plan, zm_plan_info *info);
/* Synchronises the device and reports (then clears) the plan's device error word:
 * *timed_out = 1 when a bounded wait inside one of its kernels (the asynchronous-copy
 * waits of the persistent FFT passes) gave up since the last call; results computed
 * since then are not valid.  No reference counterpart. */
int zm_plan_device_status(zm_plan plan, int *timed_out);
/* Workspace a transform needs to leave its input untouched (one field, or 0). */
int zm_plan_workspace_size(zm_plan plan, size_t *bytes);
/*
 * Tile shapes of the fused FFT pass (no counterpart in the reference; the autotuner's
 * knob next to B_DIM): the number of size-specialised variants for this plan's
 * (VEC, M, dtype) -- cluster size, lines per tile, threads -- and the one to use
 * (0 = default).  Results do not depend on the variant beyond rounding.  Set it before
 * the plan is used, not while calls using the plan are in flight.
 */
int zm_plan_kernel_variants(zm_plan plan, int *count);
int zm_plan_set_kernel_variant(zm_plan plan, int variant);
/*
 * Autotuner (no counterpart in the reference, whose only tuning knob is the
 * compile-time B_DIM): times a forward + inverse round trip `reps` times per kernel
 * variant on `stream` (CUDA events, after one untimed round trip), makes the fastest
 * the plan's variant and returns it with its time per round trip in milliseconds
 * (either output may be NULL).  `a`, `b` and `work` are caller fields of the plan's
 * size; their contents are overwritten (a holds IFFT(FFT(a)) / n^dim at the end, equal
 * to the input up to rounding).  Synchronises `stream`; not capturable.
 */
int zm_plan_autotune(zm_plan plan, void *a, void *b, void *work, int reps, void *stream,
                     int *best_variant, float *best_ms);
/*
 * B autotuner (the reference's compile-time B_DIM, chosen here per size): for every B
 * the layout constraints allow (power of two, B | N/P, P | N/(P B)) creates a plan,
 * fills a seeded field and runs zm_plan_autotune on it; returns the B, kernel variant
 * and round-trip time of the fastest.  Allocates and frees three fields of its own and
 * synchronises the device.  Note that B fixes the layout: data must be produced in the
 * layout of the chosen B.
 */
int zm_autotune_b(int dim, int64_t n, int64_t p, int dtype, int reps, int64_t *best_b, int *best_variant,
                  float *best_ms);

/*
 * Transforms over all virtual ranks.
 *
 * zm_fft_forward replaces forward_fft<true> / forward_fft_3d<true>
 * (zmodel/transforms/fft.h:36-38, 54-56; fft.cu:199-339, fft3d.cu:234-412):
 * real layout `in` -> reciprocal layout `out`, unnormalised.
 * zm_fft_inverse replaces inverse_fft<true> / inverse_fft_3d<true>
 * (fft.h:40-42, 58-60; fft.cu:409-514, fft3d.cu:508-633): reciprocal -> real,
 * result multiplied by the complex `scale` (1/N^2 or 1/N^3 for a round trip).
 *
 * `in` and `out` must not overlap.  `work` may be NULL, in which case `in` is
 * used as scratch and clobbered -- the reference's own contract (input in
 * device_buf0, output in device_buf1, buf0 clobbered; fft.cu:189-198) -- unless the
 * plan was created with ZM_FLAG_OWN_WORKSPACE, whose workspace is then used; or a
 * buffer of zm_plan_workspace_size bytes, in which case `in` is preserved.  The
 * 2D forward transform never touches `in`.  With ZM_FLAG_PERMUTE_ONLY the calls
 * reproduce the reference's do_compute=false pipelines (pure data movement).
 */
int zm_fft_forward(zm_plan plan, const void *in, void *out, void *work, void *stream);
int zm_fft_inverse(zm_plan plan, const void *in, void *out, void *work, double scale_re,
                   double scale_im, void *stream);

/*
 * zm_fft_inverse for callers that cannot allocate device memory (no counterpart in the
 * reference).  zm_fft_inverse needs one field of intermediate storage: it overwrites
 * `in`, or it uses a workspace the caller allocated.  Some callers can do neither -- a
 * plugin whose host application owns every device allocation, or a loop under a fixed
 * memory budget that may not grow or wait on an allocator -- and still need `in` kept.
 * This call keeps `in` intact and takes the intermediate from a scratch array built
 * into the library: a file-scope device array of ZM_STATIC_SCRATCH_BYTES (16 MiB) that
 * every GPU which loads the library holds until the process exits.  It calls no
 * allocator (no cudaMalloc / cudaFree, no allocating library routine).
 *   - Limit: the field (zm_plan_info.field_bytes) must fit in 16 MiB, e.g. a 2D
 *     complex128 field up to N = 1024 or a 3D complex64 field up to N = 128; larger
 *     fields return ZM_ERR_WORKSPACE.
 *   - The first call on each device looks up the array's device address
 *     (cudaGetSymbolAddress) with that device current; make that first call before
 *     any stream capture.  The address is kept for the life of the process:
 *     cudaDeviceReset on a device makes it stale, so do not call this function on a
 *     device after resetting it.
 *   - All calls on a device share the one array, which keeps the previous call's
 *     contents.  Each call overwrites everything it later reads, so nothing needs
 *     clearing, but calls that overlap on the GPU (e.g. on two streams at once) race.
 */
#define ZM_STATIC_SCRATCH_BYTES (16u << 20)
int zm_fft_inverse_static(zm_plan plan, const void *in, void *out, double scale_re,
                          double scale_im, void *stream);

/*
 * Stencils on the real-space layout.  Periodic boundaries over the whole N x N
 * (N^3) field; halos are read straight from the neighbouring virtual ranks.
 *
 * zm_laplace replaces pack_laplace + communicate_laplace + laplace
 * (laplace.h:28-38; laplace.cu:73-256) and the 3D trio (laplace3d.cu:90-361):
 * out = inv_h2 * (sum of the 4 (6) neighbours - 4 (6) * centre).  The reference
 * has no 1/h^2 factor: inv_h2 = 1 reproduces it.
 * zm_dx / zm_dy replace dx / dy (dx.cu:10-82, dy.cu:10-103), the 4th-order
 * central differences (f[i-2] - 8 f[i-1] + 8 f[i+1] - f[i+2]) / (12 delta) along
 * x (columns) / y (rows) of a 2D field, applied to each complex component.  The
 * reference needs B >= 2 (dx.cu:100, dy.cu:123); these also accept B = 1.
 * zm_dx_real / zm_dy_real take a real field (double for ZM_C128 plans, float for
 * ZM_C64), the reference's Scalar form.
 */
int zm_laplace(zm_plan plan, const void *in, void *out, double inv_h2, void *stream);
int zm_dx(zm_plan plan, const void *in, void *out, double delta, void *stream);
int zm_dy(zm_plan plan, const void *in, void *out, double delta, void *stream);
int zm_dx_real(zm_plan plan, const void *in, void *out, double delta, void *stream);
int zm_dy_real(zm_plan plan, const void *in, void *out, double delta, void *stream);
/* The 2D Laplacian, dx and dy of one complex field in one launch (no reference
 * counterpart: the reference runs three kernels with three halo exchanges).  Each output
 * is bit-identical to zm_laplace(inv_h2) / zm_dx(delta) / zm_dy(delta); the field is read
 * once (4 field transfers instead of 6).  The four buffers must not overlap. */
int zm_laplace_dx_dy(zm_plan plan, const void *in, void *lap, void *dx, void *dy, double inv_h2,
                     double delta, void *stream);

/*
 * Vector-Jacobian products (no counterpart in the reference).  Gradients use the
 * convention dL/du = dL/dRe(u) + i dL/dIm(u), so each VJP applies the adjoint
 * (conjugate transpose) of its forward map to the incoming gradient:
 *   zm_fft_forward_vjp: reciprocal-layout gradient -> real-layout gradient, the
 *     conjugate-direction transform through the same layout (adjoints of the
 *     twiddle-unpack and repack-transpose included), unnormalised;
 *   zm_fft_inverse_vjp: real-layout gradient -> reciprocal-layout gradient,
 *     conj(scale) times the forward-direction transform;
 *   zm_laplace_vjp: the periodic Laplacian is self-adjoint;
 *   zm_dx_vjp / zm_dy_vjp: the central differences are anti-self-adjoint.
 * Nothing from the forward call is stored: intermediates are recomputed.
 * `work` follows the zm_fft_forward / zm_fft_inverse rules (NULL clobbers grad_out).
 */
int zm_fft_forward_vjp(zm_plan plan, const void *grad_out, void *grad_in, void *work, void *stream);
int zm_fft_inverse_vjp(zm_plan plan, const void *grad_out, void *grad_in, void *work,
                       double scale_re, double scale_im, void *stream);
int zm_laplace_vjp(zm_plan plan, const void *grad_out, void *grad_in, double inv_h2, void *stream);
int zm_dx_vjp(zm_plan plan, const void *grad_out, void *grad_in, double delta, void *stream);
int zm_dy_vjp(zm_plan plan, const void *grad_out, void *grad_in, double delta, void *stream);

/*
 * Layout converters between a natural row-major N x N (N^3) field and the
 * interleaved layouts (device kernels; the reference does this on the host with
 * init_host + vector_pack, utils.cu:9-36, utils.h:99-119).
 */
int zm_natural_to_real(zm_plan plan, const void *natural, void *interleaved, void *stream);
int zm_real_to_natural(zm_plan plan, const void *interleaved, void *natural, void *stream);
int zm_natural_to_reciprocal(zm_plan plan, const void *natural, void *interleaved, void *stream);
int zm_reciprocal_to_natural(zm_plan plan, const void *interleaved, void *natural, void *stream);

/*
 * Pointwise operators on the reciprocal layout (in place), indexing frequencies
 * through reciprocal_to_global (utils.h:265-268, 298-302; used as in
 * main.cu:66-71).  k is the signed frequency (k >= N/2 maps to k - N).
 *   ZM_SPECTRAL_GAUSSIAN: x *= exp(-|k|^2 / (2 a^2))
 *   ZM_SPECTRAL_POISSON:  x /= -(a^2 |k|^2), and the k = 0 mode is set to 0
 *                         (a = 2 pi / (N h) turns grid units into physical wavenumbers)
 *   ZM_SPECTRAL_SCALE:    x *= a
 */
enum zm_spectral_op { ZM_SPECTRAL_GAUSSIAN = 0, ZM_SPECTRAL_POISSON = 1, ZM_SPECTRAL_SCALE = 2 };
int zm_spectral_apply(zm_plan plan, void *data, int op, double a, void *stream);
/* VJP of zm_spectral_apply, in place on `grad` (no reference counterpart).  The
 * multipliers are real and diagonal, so the adjoint applies the same multiplier. */
int zm_spectral_apply_vjp(zm_plan plan, void *grad, int op, double a, void *stream);

/*
 * Seeded synthetic fields written straight into the real-space layout
 * (counter-based, identical on host and device):
 *   ZM_FIELD_UNIFORM:  Re, Im ~ U[-1,1)
 *   ZM_FIELD_GAUSSIAN: Re, Im ~ N(0,1)
 */
enum zm_field_kind { ZM_FIELD_UNIFORM = 0, ZM_FIELD_GAUSSIAN = 1 };
int zm_fill_field(zm_plan plan, void *interleaved, int kind, uint64_t seed, void *stream);
/* Sum of `nmodes` plane waves a_m exp(2 pi i (kx x + ky y) / N) (evaluated in FP64)
 * plus `noise` * N(0,1) complex noise from counter stream `seed`; 2D only.
 * modes = {kx, ky} pairs, amps = {re, im} pairs, both host arrays. */
int zm_fill_modes(zm_plan plan, void *interleaved, int nmodes, const int64_t *modes,
                  const double *amps, double noise, uint64_t seed, void *stream);

/* Index maps of zmodel/utils.h (host functions; argument meaning as in the reference). */
int zm_real_to_global(zm_plan plan, int64_t rid, int64_t cid, int64_t did, int64_t ld,
                      int64_t lr, int64_t lc, int64_t *gd, int64_t *gr, int64_t *gc);
int zm_global_to_real(zm_plan plan, int64_t gd, int64_t gr, int64_t gc, int64_t *rid,
                      int64_t *cid, int64_t *did, int64_t *ld, int64_t *lr, int64_t *lc);
int zm_reciprocal_to_global(zm_plan plan, int64_t rid, int64_t cid, int64_t did, int64_t ld,
                            int64_t lr, int64_t lc, int64_t *kd, int64_t *kr, int64_t *kc);
int zm_global_to_reciprocal(zm_plan plan, int64_t kd, int64_t kr, int64_t kc, int64_t *rid,
                            int64_t *cid, int64_t *did, int64_t *ld, int64_t *lr, int64_t *lc);

/*
 * Batches of independent 2D fields of uneven N (no reference counterpart: the reference
 * transforms one field per MPI job).  Every field has its own (N, B, P) and lives in the
 * reference layout of that plan at `offset` elements into a batch buffer (offsets are
 * multiples of 2 elements, so a 16-byte aligned buffer keeps every field aligned).  Each
 * call below is ONE cooperative persistent launch over all fields (grid = the resident
 * CTAs of the device, phases separated by a grid barrier whose waits are bounded); no
 * call allocates or synchronises, so a sequence of calls can be captured in a CUDA graph.
 * Fields need 64 <= N <= 4096 (complex64) or 32 <= N <= 2048 (complex128).  A grid
 * barrier that waits more than 2 s sets a device error flag instead of hanging:
 * zm_batch_status reads and clears it.  A timeout ends only the launch it happened in
 * (whose outputs are then incomplete); later calls run normally, and the flag stays set
 * until zm_batch_status is called, so check it before trusting a call's outputs.
 */
typedef struct zm_batch_s *zm_batch;
typedef struct {
    int64_t n, b, p;
    int64_t offset;   /* element offset of the field in a batch buffer */
    int64_t elems;    /* N * N */
} zm_batch_field;
int zm_batch_create(zm_batch *batch, int nfields, const int64_t *n, const int64_t *b,
                    const int64_t *p, int dtype);
int zm_batch_destroy(zm_batch batch);
int zm_batch_get_field(zm_batch batch, int i, zm_batch_field *info);
/* Elements of one batch buffer (sum of N^2 plus alignment padding). */
int zm_batch_total_elems(zm_batch batch, int64_t *elems);
/* Field i <- zm_fill_field(kind, first_seed + i) in its real layout. */
int zm_batch_fill(zm_batch batch, void *data, int kind, uint64_t first_seed, void *stream);
/* Per field: zm_fft_forward (in kept) / zm_fft_inverse with scale 1 / N^2 when
 * `normalise` is non-zero (work NULL: `in` is scratch). */
int zm_batch_forward(zm_batch batch, const void *in, void *out, void *stream);
int zm_batch_inverse(zm_batch batch, const void *in, void *out, void *work, int normalise,
                     void *stream);
/*
 * Spectral Poisson solve per field on a periodic square of side `length` (h = length / N):
 * phi = IFFT(FFT(rhs) / (-|k|^2)) with k = (2 pi / length) * (signed integer frequency),
 * the k = 0 mode set to 0, then (when `residual` is not NULL)
 * residual = Lap_h(phi) - rhs with the 5-point Laplacian / h^2.  The forward y pass, the
 * division and the inverse y pass are fused (the spectrum is never stored).  `work` holds
 * one batch buffer of scratch; rhs is kept.
 */
int zm_batch_poisson(zm_batch batch, const void *rhs, void *phi, void *residual, void *work,
                     double length, void *stream);
/* Synchronises the device and reports (then clears) the grid-barrier timeout flag:
 * *device_error = 1 when a barrier timed out since the last call. */
int zm_batch_status(zm_batch batch, int *device_error);
/*
 * Failure-detection probe of the batch kernel's grid barrier (no reference counterpart):
 * one launch whose single barrier waits for `missing` (0 or 1) arrivals more than the
 * grid has.  With 1 the barrier can never complete: every CTA gives up after the 2 s
 * limit, the kernel returns and zm_batch_status reports 1.  With 0 it completes.
 */
int zm_batch_barrier_probe(zm_batch batch, int missing, void *stream);
/*
 * B autotuner for batched fields (the reference's compile-time B_DIM knob): times
 * zm_batch_poisson on a batch of `count` fields of size N for every B allowed by the
 * layout constraints (power of two, B | N/P, P | N/(P B)), `reps` timed calls each after
 * one untimed call, and returns the fastest B and its time per call.  Allocates and frees
 * its own buffers and synchronises the device.
 */
int zm_batch_autotune_b(int64_t n, int64_t p, int dtype, int count, int reps, int64_t *best_b,
                        float *best_ms);

/* Diagnostics. */
const char *zm_last_error_string(void);
const char *zm_status_string(int status);
/* Number of kernels this library has launched in this process (all threads). */
uint64_t zm_launch_count(void);
const char *zm_version(void);

#ifdef __cplusplus
}
#endif
#endif /* ZMODEL_B200_H */
