// zm_api.cu -- the C ABI of libzmodel_b200: plan creation, validation, twiddle
// generation and the orchestration of the fused kernels.
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>

#include <atomic>
#include <cmath>
#include <mutex>
#include <string>
#include <vector>

#include "zm_internal.h"
#include "zmodel_b200.h"

namespace {

thread_local std::string g_err;
std::atomic<uint64_t> g_launches{0};

int fail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

int cuda_fail(cudaError_t e, const char *what) {
    return fail(ZM_ERR_CUDA, "%s: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e));
}

bool pow2(int64_t x) { return x > 0 && (x & (x - 1)) == 0; }
int ilog2(int64_t x) {
    int l = 0;
    while ((int64_t{1} << l) < x) l++;
    return l;
}

bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

int schedule(int64_t n, int rmax, int *rad) { return zm::radix_schedule(n, rmax, rad); }

}  // namespace

namespace zm {

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

// Radix schedule of a power-of-two length n with radices <= rmax: the
// remainder radix first, then rmax-radix stages.
int radix_schedule(int64_t n, int rmax, int *rad) {
    int ln = ilog2(n), lr = ilog2(rmax), k = 0;
    if (ln == 0) return 0;
    int rem = ln % lr;
    if (rem) rad[k++] = 1 << rem;
    for (int i = 0; i < ln / lr; i++) rad[k++] = rmax;
    return k;
}

int report_error(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

int max_dyn_smem() {
    static int cached[64];
    static std::once_flag once[64];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    std::call_once(once[dev], [dev]() {
        int v = 0;
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
            v = 48 * 1024;
        cached[dev] = v;
    });
    return cached[dev];
}

}  // namespace zm

using zm::Geom;
using zm::LineParams;

// ---------------------------------------------------------------- helpers

static cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

static int check_plan(zm_plan p) {
    if (!p) return fail(ZM_ERR_INVALID_ARG, "null plan");
    return ZM_OK;
}

static int check_device_plan(zm_plan p) {
    if (!p) return fail(ZM_ERR_INVALID_ARG, "null plan");
    if (p->flags & ZM_FLAG_HOST_ONLY)
        return fail(ZM_ERR_UNSUPPORTED, "plan was created with ZM_FLAG_HOST_ONLY");
    return ZM_OK;
}

static int check_field(zm_plan p, const void *ptr, const char *name) {
    if (!ptr) return fail(ZM_ERR_INVALID_ARG, "%s is NULL", name);
    if (!aligned16(ptr)) return fail(ZM_ERR_MISALIGNED, "%s is not 16-byte aligned", name);
    (void)p;
    return ZM_OK;
}

static bool overlap(const void *a, const void *b, size_t bytes) {
    const char *x = static_cast<const char *>(a), *y = static_cast<const char *>(b);
    return x < y + bytes && y < x + bytes;
}

// Lines per CTA of the fused pass: aim at 512 threads, at most 64 lines, at most L.
static int pick_lines(const zm_plan_s *p) {
    const int ept = zm::ept_for(p->dtype);
    int64_t t = (512 * (int64_t)ept) / p->g.n;
    if (t < 1) t = 1;
    while (t * p->g.n < ept) t *= 2;   // at least one thread
    if (t > 64) t = 64;
    if (t > p->g.L) t = (int)p->g.L;
    return (int)t;
}

static bool fft_supported(const zm_plan_s *p, std::string *why) {
    const bool permute = (p->flags & ZM_FLAG_PERMUTE_ONLY) != 0;
    if (p->nvariants > 0 && !permute) return true;
    const int ept = zm::ept_for(p->dtype);
    const int64_t threads = (int64_t)p->T[0] * p->g.n / ept;
    const int64_t smem = (int64_t)p->T[0] * p->g.n * (int64_t)p->elem_bytes;
    if (threads > 1024 || threads < 1 || smem + 2048 > zm::max_dyn_smem() || p->T[0] > p->g.L) {
        if (why) *why = "one global line does not fit one CTA (N too large for this dtype)";
        return false;
    }
    return true;
}

static LineParams line_params(const zm_plan_s *p, int kind, const void *in, void *out) {
    LineParams lp{};
    lp.g = p->g;
    lp.kind = kind;
    lp.T = p->T[kind == zm::PASS_X2 || kind == zm::PASS_X3 ? 0 : (kind == zm::PASS_Z3 ? 2 : 1)];
    lp.nlines = p->g.dim == 2 ? p->g.n : p->g.n * p->g.n;
    lp.in = in;
    lp.out = out;
    lp.twN = p->twN;
    lp.twd = p->twd;
    lp.twv = p->twv;
    lp.twm = p->twm;
    lp.scale_re = 1.0;
    lp.scale_im = 0.0;
    lp.apply_scale = 0;
    lp.variant = p->variant;
    lp.permute_only = (p->flags & ZM_FLAG_PERMUTE_ONLY) ? 1 : 0;
    lp.err = p->dev_err;
    // 2D transforms on the size-specialised passes keep the x -> y intermediate with
    // groups of G x-frequency rows interleaved, G up to the tile's line count (at most
    // 4): the x pass then writes G * TL consecutive elements per line group and the y
    // pass reads its G lines as one contiguous run.  G <= VP keeps a group inside one
    // rank chunk.  Both passes of one transform see the same plan state, so they agree.
    lp.lg_inter = 0;
    if (p->g.dim == 2 && !lp.permute_only && p->nvariants > 0) {
        int lg = p->dtype == ZM_C128 ? zm::fused_interleave_lg_c128(p->g.logVEC, p->g.logM, p->variant)
                                     : zm::fused_interleave_lg_c64(p->g.logVEC, p->g.logM, p->variant);
        if (lg > p->g.logVP) lg = p->g.logVP;
        lp.lg_inter = lg;
    }
    lp.nst_vec = schedule(p->g.vec, p->max_radix, lp.rad_vec);
    lp.nst_m = schedule(p->g.m, p->max_radix, lp.rad_m);
    return lp;
}

// The out-of-place forward configuration of a 2D plan (x pass in -> work, y pass
// work -> out, each pass with its own tile shape and a wider row interleave; the
// in-place y pass rules out interleaves wider than its tile), or false.
static bool fwd_oop_config(const zm_plan_s *p, int *vx, int *vy, int *lg, int *qint) {
    if (p->g.dim != 2 || (p->flags & ZM_FLAG_PERMUTE_ONLY) || p->nvariants == 0 || p->variant != 0) return false;
    const int ok = p->dtype == ZM_C128 ? zm::fused_fwd_oop_c128(p->g.logVEC, p->g.logM, vx, vy, lg, qint)
                                       : zm::fused_fwd_oop_c64(p->g.logVEC, p->g.logM, vx, vy, lg, qint);
    if (!ok) return false;
    if (*lg > p->g.logVP) *lg = p->g.logVP;
    return true;
}
// The out-of-place inverse configuration of a 2D plan (y pass in -> work, x pass
// work -> out), or false.
static bool inv_oop_config(const zm_plan_s *p, int *vx, int *vy, int *lg, int *qint) {
    if (p->g.dim != 2 || (p->flags & ZM_FLAG_PERMUTE_ONLY) || p->nvariants == 0 || p->variant != 0) return false;
    const int ok = p->dtype == ZM_C128 ? zm::fused_inv_oop_c128(p->g.logVEC, p->g.logM, vx, vy, lg, qint)
                                       : zm::fused_inv_oop_c64(p->g.logVEC, p->g.logM, vx, vy, lg, qint);
    if (!ok) return false;
    if (*lg > p->g.logVP) *lg = p->g.logVP;
    return true;
}

// `variant` / `lg` >= 0 override the plan's tile shape and row interleave for this pass;
// `qint` selects the y-position interleave of the intermediate.
static int run_pass(const zm_plan_s *p, int kind, bool inv, const void *in, void *out, bool scale,
                    double sre, double sim, cudaStream_t st, int variant = -1, int lg = -1, int qint = 0) {
    LineParams lp = line_params(p, kind, in, out);
    if (variant >= 0) lp.variant = variant;
    if (lg >= 0) lp.lg_inter = lg;
    lp.inter_q = (qint && lp.lg_inter > 0) ? 1 : 0;
    if (scale) {
        lp.apply_scale = 1;
        lp.scale_re = sre;
        lp.scale_im = sim;
    }
    cudaError_t e = zm::launch_line_pass(lp, p->dtype, inv, st);
    if (e != cudaSuccess) return cuda_fail(e, "line pass launch");
    return ZM_OK;
}

// Forward pipeline (fft.cu:199-339, fft3d.cu:234-412); `scale` is applied by the
// last pass when set (used by the inverse transform's VJP).
static int forward_impl(zm_plan p, const void *in, void *out, void *work, bool scale, double sre,
                        double sim, cudaStream_t st) {
    int rc;
    if ((rc = check_device_plan(p))) return rc;
    if (!work) work = p->own_work;   // NULL unless ZM_FLAG_OWN_WORKSPACE
    if ((rc = check_field(p, in, "in")) || (rc = check_field(p, out, "out"))) return rc;
    const size_t F = p->total * p->elem_bytes;
    if (overlap(in, out, F)) return fail(ZM_ERR_INVALID_ARG, "in and out overlap");
    std::string why;
    if (!fft_supported(p, &why)) return fail(ZM_ERR_UNSUPPORTED, "%s", why.c_str());
    if (work && (!aligned16(work))) return fail(ZM_ERR_MISALIGNED, "work is not 16-byte aligned");
    if (p->g.dim == 2) {
        int vx, vy, lg, qi;
        if (work && fwd_oop_config(p, &vx, &vy, &lg, &qi)) {
            if (overlap(work, in, F) || overlap(work, out, F))
                return fail(ZM_ERR_INVALID_ARG, "work overlaps in/out");
            // x pass in -> work, y pass work -> out (no in-place constraint on the tile)
            if ((rc = run_pass(p, zm::PASS_X2, false, in, work, false, 0, 0, st, vx, lg, qi))) return rc;
            return run_pass(p, zm::PASS_Y2, false, work, out, scale, sre, sim, st, vy, lg, qi);
        }
        // x pass: real layout -> REPACK layout (in -> out); y pass in place on out
        if ((rc = run_pass(p, zm::PASS_X2, false, in, out, false, 0, 0, st))) return rc;
        return run_pass(p, zm::PASS_Y2, false, out, out, scale, sre, sim, st);
    }
    void *tmp = work ? work : const_cast<void *>(in);
    if (work && (overlap(work, in, F) || overlap(work, out, F)))
        return fail(ZM_ERR_INVALID_ARG, "work overlaps in/out");
    if ((rc = run_pass(p, zm::PASS_X3, false, in, out, false, 0, 0, st))) return rc;
    if ((rc = run_pass(p, zm::PASS_Y3, false, out, tmp, false, 0, 0, st))) return rc;
    return run_pass(p, zm::PASS_Z3, false, tmp, out, scale, sre, sim, st);
}

// Inverse pipeline (fft.cu:409-514, fft3d.cu:508-633), scale applied by the last pass.
static int inverse_impl(zm_plan p, const void *in, void *out, void *work, double sre, double sim,
                        cudaStream_t st) {
    int rc;
    if ((rc = check_device_plan(p))) return rc;
    if (!work) work = p->own_work;   // NULL unless ZM_FLAG_OWN_WORKSPACE
    if ((rc = check_field(p, in, "in")) || (rc = check_field(p, out, "out"))) return rc;
    const size_t F = p->total * p->elem_bytes;
    if (overlap(in, out, F)) return fail(ZM_ERR_INVALID_ARG, "in and out overlap");
    std::string why;
    if (!fft_supported(p, &why)) return fail(ZM_ERR_UNSUPPORTED, "%s", why.c_str());
    if (work && (!aligned16(work))) return fail(ZM_ERR_MISALIGNED, "work is not 16-byte aligned");
    if (work && (overlap(work, in, F) || overlap(work, out, F)))
        return fail(ZM_ERR_INVALID_ARG, "work overlaps in/out");
    void *tmp = work ? work : const_cast<void *>(in);
    if (p->g.dim == 2) {
        int vx, vy, lg, qi;
        if (work && inv_oop_config(p, &vx, &vy, &lg, &qi)) {
            if ((rc = run_pass(p, zm::PASS_Y2, true, in, work, false, 0, 0, st, vy, lg, qi))) return rc;
            return run_pass(p, zm::PASS_X2, true, work, out, true, sre, sim, st, vx, lg, qi);
        }
        if ((rc = run_pass(p, zm::PASS_Y2, true, in, tmp, false, 0, 0, st))) return rc;
        return run_pass(p, zm::PASS_X2, true, tmp, out, true, sre, sim, st);
    }
    if ((rc = run_pass(p, zm::PASS_Z3, true, in, out, false, 0, 0, st))) return rc;
    if ((rc = run_pass(p, zm::PASS_Y3, true, out, tmp, false, 0, 0, st))) return rc;
    return run_pass(p, zm::PASS_X3, true, tmp, out, true, sre, sim, st);
}

// ================================================================== C ABI
extern "C" {

int zm_plan_create(zm_plan *plan, int dim, int64_t n, int64_t b, int64_t p, int dtype,
                   unsigned flags) {
    if (!plan) return fail(ZM_ERR_INVALID_ARG, "plan output pointer is NULL");
    *plan = nullptr;
    if (dim != 2 && dim != 3) return fail(ZM_ERR_INVALID_ARG, "dim must be 2 or 3 (got %d)", dim);
    if (dtype != ZM_C128 && dtype != ZM_C64) return fail(ZM_ERR_INVALID_ARG, "unknown dtype %d", dtype);
    if (flags & ~(ZM_FLAG_PERMUTE_ONLY | ZM_FLAG_HOST_ONLY | ZM_FLAG_OWN_WORKSPACE))
        return fail(ZM_ERR_INVALID_ARG, "unknown flags 0x%x", flags);
    if ((flags & ZM_FLAG_HOST_ONLY) && (flags & ZM_FLAG_OWN_WORKSPACE))
        return fail(ZM_ERR_INVALID_ARG, "ZM_FLAG_OWN_WORKSPACE needs device resources (not HOST_ONLY)");
    if (!pow2(n) || !pow2(b) || !pow2(p))
        return fail(ZM_ERR_CONSTRAINT, "N=%lld, B=%lld, P=%lld must be powers of two", (long long)n,
                    (long long)b, (long long)p);
    if (n % p) return fail(ZM_ERR_CONSTRAINT, "P=%lld does not divide N=%lld", (long long)p, (long long)n);
    const int64_t L = n / p;
    if (L % b) return fail(ZM_ERR_CONSTRAINT, "B=%lld does not divide L=N/P=%lld", (long long)b, (long long)L);
    const int64_t vec = L / b;
    if (vec % p)
        return fail(ZM_ERR_CONSTRAINT, "P=%lld does not divide VEC=L/B=%lld (need B <= N/P^2)",
                    (long long)p, (long long)vec);
    const int64_t total = dim == 2 ? n * n : n * n * n;
    if ((dim == 2 && n > (int64_t{1} << 20)) || (dim == 3 && n > 4096))
        return fail(ZM_ERR_CONSTRAINT, "N=%lld too large", (long long)n);

    zm_plan_s *P = new (std::nothrow) zm_plan_s();
    if (!P) return fail(ZM_ERR_NO_MEMORY, "host allocation failed");
    Geom &g = P->g;
    g.dim = dim;
    g.n = n; g.b = b; g.p = p; g.L = L; g.vec = vec; g.vp = vec / p; g.m = b * p;
    g.logN = ilog2(n); g.logB = ilog2(b); g.logP = ilog2(p); g.logL = ilog2(L);
    g.logVEC = ilog2(vec); g.logVP = ilog2(g.vp); g.logM = ilog2(g.m);
    P->dtype = dtype;
    P->flags = flags;
    P->ranks = dim == 2 ? p * p : p * p * p;
    P->rank_elems = dim == 2 ? L * L : L * L * L;
    P->total = total;
    P->elem_bytes = dtype == ZM_C128 ? 16 : 8;
    P->max_radix = zm::ept_for(dtype);
    cudaGetDevice(&P->device);
    const int t = pick_lines(P);
    P->T[0] = P->T[1] = P->T[2] = t;
    P->variant = 0;
    P->nvariants = dtype == ZM_C128 ? zm::fused_variants_c128(g.logVEC, g.logM)
                                    : zm::fused_variants_c64(g.logVEC, g.logM);

    // Twiddle table w_N^m = exp(-2 pi i m / N), m < N, generated in extended
    // precision and rounded once (FP64 for complex128; hi/lo FP32 split of the
    // FP64 value for complex64).  Replaces the L x L per-rank tables of
    // init_forward_twiddles / init_inverse_twiddles (fft.cu:37-73).
    // Also, for the size-specialised passes: w_N^m in FP64 for every dtype (the
    // inter-step twiddles are generated from it on the device) and the sub-transform
    // tables w_VEC^m, w_M^m.  All four tables share one allocation of 16-byte entries.
    P->twN = P->twv = P->twm = P->twd = nullptr;
    P->dev_err = nullptr;
    P->own_work = nullptr;
    if (flags & ZM_FLAG_HOST_ONLY) {
        *plan = P;
        return ZM_OK;
    }
    const int64_t entries = 2 * n + g.vec + g.m + 1;   // + one 16-byte slot for the error word
    std::vector<unsigned char> host((size_t)entries * 16);
    const long double pi = 3.141592653589793238462643383279502884L;
    auto put = [&](int64_t slot, int64_t m, int64_t len, bool fp64 = false) {   // w_len^m
        const long double th = -2.0L * pi * (long double)m / (long double)len;
        const double c = (double)cosl(th), s = (double)sinl(th);
        if (dtype == ZM_C128 || fp64) {
            double *d = reinterpret_cast<double *>(host.data()) + 2 * slot;
            d[0] = c; d[1] = s;
        } else {
            float *f = reinterpret_cast<float *>(host.data()) + 4 * slot;
            const float ch = (float)c, sh = (float)s;
            f[0] = ch; f[1] = sh;
            f[2] = (float)(c - (double)ch); f[3] = (float)(s - (double)sh);
        }
    };
    for (int64_t m = 0; m < n; m++) put(m, m, n);
    for (int64_t m = 0; m < n; m++) put(n + m, m, n, true);
    for (int64_t m = 0; m < g.vec; m++) put(2 * n + m, m, g.vec);
    for (int64_t m = 0; m < g.m; m++) put(2 * n + g.vec + m, m, g.m);
    void *tables = nullptr;
    cudaError_t e = cudaMalloc(&tables, host.size());
    if (e != cudaSuccess) {
        delete P;
        return fail(ZM_ERR_NO_MEMORY, "twiddle table allocation failed: %s", cudaGetErrorString(e));
    }
    e = cudaMemcpy(tables, host.data(), host.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(tables);
        delete P;
        return cuda_fail(e, "twiddle upload");
    }
    unsigned char *tb = static_cast<unsigned char *>(tables);
    P->twN = tb;
    P->twd = tb + (size_t)n * 16;
    P->twv = tb + (size_t)2 * n * 16;
    P->twm = tb + (size_t)(2 * n + g.vec) * 16;
    P->dev_err = reinterpret_cast<int *>(tb + (size_t)(2 * n + g.vec + g.m) * 16);   // zeroed by the upload
    if (flags & ZM_FLAG_OWN_WORKSPACE) {
        e = cudaMalloc(&P->own_work, (size_t)P->total * P->elem_bytes);
        if (e != cudaSuccess) {
            P->own_work = nullptr;
            cudaFree(tables);
            delete P;
            return fail(ZM_ERR_NO_MEMORY, "plan workspace allocation failed: %s", cudaGetErrorString(e));
        }
    }
    *plan = P;
    return ZM_OK;
}

int zm_plan_destroy(zm_plan plan) {
    if (!plan) return fail(ZM_ERR_INVALID_ARG, "null plan");
    if (plan->twN) cudaFree(plan->twN);
    if (plan->own_work) cudaFree(plan->own_work);
    delete plan;
    return ZM_OK;
}

int zm_plan_kernel_variants(zm_plan plan, int *count) {
    int rc;
    if ((rc = check_plan(plan))) return rc;
    if (!count) return fail(ZM_ERR_INVALID_ARG, "count is NULL");
    *count = plan->nvariants;
    return ZM_OK;
}

int zm_plan_set_kernel_variant(zm_plan plan, int variant) {
    int rc;
    if ((rc = check_plan(plan))) return rc;
    if (variant < 0 || (variant > 0 && variant >= plan->nvariants))
        return fail(ZM_ERR_INVALID_ARG, "variant %d out of range (%d available)", variant,
                    plan->nvariants);
    plan->variant = variant;
    return ZM_OK;
}

int zm_plan_autotune(zm_plan plan, void *a, void *b, void *work, int reps, void *stream,
                     int *best_variant, float *best_ms) {
    int rc;
    if ((rc = check_device_plan(plan))) return rc;
    if (reps < 1) return fail(ZM_ERR_INVALID_ARG, "reps must be >= 1 (got %d)", reps);
    if ((rc = check_field(plan, a, "a")) || (rc = check_field(plan, b, "b"))) return rc;
    if (work && (rc = check_field(plan, work, "work"))) return rc;
    const int nv = plan->nvariants > 0 ? plan->nvariants : 1;
    double inv_n = 1.0;
    for (int d = 0; d < plan->g.dim; d++) inv_n /= (double)plan->g.n;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t ce = cudaEventCreate(&e0);
    if (ce == cudaSuccess) ce = cudaEventCreate(&e1);
    if (ce != cudaSuccess) {
        if (e0) cudaEventDestroy(e0);
        return cuda_fail(ce, "autotune events");
    }
    const int saved = plan->variant;
    int best = 0;
    float best_t = 0.f;
    rc = ZM_OK;
    for (int v = 0; v < nv && rc == ZM_OK; v++) {
        plan->variant = v;
        for (int it = -1; it < reps && rc == ZM_OK; it++) {
            if (it == 0) cudaEventRecord(e0, (cudaStream_t)stream);
            rc = zm_fft_forward(plan, a, b, work, stream);
            if (rc == ZM_OK) rc = zm_fft_inverse(plan, b, a, work, inv_n, 0.0, stream);
        }
        if (rc != ZM_OK) break;
        cudaEventRecord(e1, (cudaStream_t)stream);
        if ((ce = cudaEventSynchronize(e1)) != cudaSuccess) {
            rc = cuda_fail(ce, "autotune timing");
            break;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        ms /= (float)reps;
        if (v == 0 || ms < best_t) {
            best = v;
            best_t = ms;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != ZM_OK) {
        plan->variant = saved;
        return rc;
    }
    plan->variant = best;
    if (best_variant) *best_variant = best;
    if (best_ms) *best_ms = best_t;
    return ZM_OK;
}

int zm_autotune_b(int dim, int64_t n, int64_t p, int dtype, int reps, int64_t *best_b, int *best_variant,
                  float *best_ms) {
    if (reps < 1) return fail(ZM_ERR_INVALID_ARG, "reps must be >= 1 (got %d)", reps);
    if (dim != 2 && dim != 3) return fail(ZM_ERR_INVALID_ARG, "dim must be 2 or 3 (got %d)", dim);
    if (!pow2(n) || !pow2(p) || n % p) return fail(ZM_ERR_CONSTRAINT, "N and P must be powers of two with P | N");
    const int64_t L = n / p;
    int64_t bb = 0;
    int bv = 0;
    float bms = 0.f;
    for (int64_t b = 1; b <= L / p; b *= 2) {
        zm_plan pl = nullptr;
        if (zm_plan_create(&pl, dim, n, b, p, dtype, 0) != ZM_OK) continue;   // B outside the constraints
        const size_t F = pl->total * pl->elem_bytes;
        void *buf = nullptr;
        cudaError_t e = cudaMalloc(&buf, 3 * F);
        if (e != cudaSuccess) {
            zm_plan_destroy(pl);
            return fail(ZM_ERR_NO_MEMORY, "autotune buffers (%zu bytes): %s", 3 * F, cudaGetErrorString(e));
        }
        char *c = static_cast<char *>(buf);
        int v = 0;
        float ms = 0.f;
        int rc = zm_fill_field(pl, c, ZM_FIELD_GAUSSIAN, 1, nullptr);
        if (rc == ZM_OK) rc = zm_plan_autotune(pl, c, c + F, c + 2 * F, reps, nullptr, &v, &ms);
        cudaFree(buf);
        zm_plan_destroy(pl);
        if (rc != ZM_OK) return rc;
        if (bb == 0 || ms < bms) {
            bb = b;
            bv = v;
            bms = ms;
        }
    }
    if (bb == 0) return fail(ZM_ERR_CONSTRAINT, "no B is valid for N=%lld, P=%lld", (long long)n, (long long)p);
    if (best_b) *best_b = bb;
    if (best_variant) *best_variant = bv;
    if (best_ms) *best_ms = bms;
    return ZM_OK;
}

int zm_plan_device_status(zm_plan plan, int *timed_out) {
    int rc;
    if ((rc = check_device_plan(plan))) return rc;
    if (!timed_out) return fail(ZM_ERR_INVALID_ARG, "timed_out is NULL");
    cudaError_t e = cudaDeviceSynchronize();
    int v = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&v, plan->dev_err, sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && v) e = cudaMemset(plan->dev_err, 0, sizeof(int));
    if (e != cudaSuccess) return cuda_fail(e, "device status");
    *timed_out = v ? 1 : 0;
    return ZM_OK;
}

int zm_plan_workspace_size(zm_plan plan, size_t *bytes) {
    int rc;
    if ((rc = check_plan(plan))) return rc;
    if (!bytes) return fail(ZM_ERR_INVALID_ARG, "bytes is NULL");
    *bytes = plan->total * plan->elem_bytes;
    return ZM_OK;
}

int zm_plan_get_info(zm_plan plan, zm_plan_info *info) {
    int rc;
    if ((rc = check_plan(plan))) return rc;
    if (!info) return fail(ZM_ERR_INVALID_ARG, "info is NULL");
    const Geom &g = plan->g;
    info->dim = g.dim;
    info->dtype = plan->dtype;
    info->n = g.n; info->b = g.b; info->p = g.p;
    info->local_dim = g.L; info->vec = g.vec; info->vec_split = g.vp; info->m = g.m;
    info->ranks = plan->ranks;
    info->rank_elems = plan->rank_elems;
    info->total_elems = plan->total;
    info->elem_bytes = plan->elem_bytes;
    info->field_bytes = plan->total * plan->elem_bytes;
    info->workspace_bytes = info->field_bytes;
    return ZM_OK;
}

int zm_fft_forward(zm_plan plan, const void *in, void *out, void *work, void *stream) {
    return forward_impl(plan, in, out, work, false, 1.0, 0.0, as_stream(stream));
}

int zm_fft_inverse(zm_plan plan, const void *in, void *out, void *work, double scale_re,
                   double scale_im, void *stream) {
    return inverse_impl(plan, in, out, work, scale_re, scale_im, as_stream(stream));
}

int zm_fft_forward_vjp(zm_plan plan, const void *grad_out, void *grad_in, void *work, void *stream) {
    // adjoint of the unnormalised forward DFT through the layouts: the
    // conjugate-direction transform, reciprocal -> real, no scale
    return inverse_impl(plan, grad_out, grad_in, work, 1.0, 0.0, as_stream(stream));
}

int zm_fft_inverse_vjp(zm_plan plan, const void *grad_out, void *grad_in, void *work,
                       double scale_re, double scale_im, void *stream) {
    return forward_impl(plan, grad_out, grad_in, work, true, scale_re, -scale_im, as_stream(stream));
}

static int stencil_call(zm_plan plan, int op, bool real_field, const void *in, void *out,
                        double coef, void *stream) {
    int rc;
    if ((rc = check_device_plan(plan))) return rc;
    if ((rc = check_field(plan, in, "in")) || (rc = check_field(plan, out, "out"))) return rc;
    const size_t bytes = plan->total * (real_field ? plan->elem_bytes / 2 : plan->elem_bytes);
    if (overlap(in, out, bytes)) return fail(ZM_ERR_INVALID_ARG, "in and out overlap");
    if (op != zm::ST_LAPLACE && plan->g.dim != 2)
        return fail(ZM_ERR_UNSUPPORTED, "dx / dy are defined on 2D plans only");
    if (op != zm::ST_LAPLACE && coef == 0.0) return fail(ZM_ERR_INVALID_ARG, "delta must be non-zero");
    cudaError_t e = zm::launch_stencil(plan, op, real_field, in, out, coef, as_stream(stream));
    if (e != cudaSuccess) return cuda_fail(e, "stencil launch");
    return ZM_OK;
}

int zm_laplace_dx_dy(zm_plan plan, const void *in, void *lap, void *dx, void *dy, double inv_h2,
                     double delta, void *stream) {
    int rc;
    if ((rc = check_device_plan(plan))) return rc;
    if ((rc = check_field(plan, in, "in")) || (rc = check_field(plan, lap, "lap")) ||
        (rc = check_field(plan, dx, "dx")) || (rc = check_field(plan, dy, "dy")))
        return rc;
    if (plan->g.dim != 2) return fail(ZM_ERR_UNSUPPORTED, "dx / dy are defined on 2D plans only");
    if (delta == 0.0) return fail(ZM_ERR_INVALID_ARG, "delta must be non-zero");
    const size_t F = plan->total * plan->elem_bytes;
    const void *bufs[4] = {in, lap, dx, dy};
    for (int a = 0; a < 4; a++)
        for (int b = a + 1; b < 4; b++)
            if (overlap(bufs[a], bufs[b], F)) return fail(ZM_ERR_INVALID_ARG, "in, lap, dx and dy must not overlap");
    cudaError_t e = zm::launch_stencil(plan, zm::ST_ALL, false, in, lap, inv_h2, as_stream(stream), dx, dy, delta);
    if (e != cudaSuccess) return cuda_fail(e, "stencil launch");
    return ZM_OK;
}

int zm_laplace(zm_plan plan, const void *in, void *out, double inv_h2, void *stream) {
    return stencil_call(plan, zm::ST_LAPLACE, false, in, out, inv_h2, stream);
}
int zm_dx(zm_plan plan, const void *in, void *out, double delta, void *stream) {
    return stencil_call(plan, zm::ST_DX, false, in, out, delta, stream);
}
int zm_dy(zm_plan plan, const void *in, void *out, double delta, void *stream) {
    return stencil_call(plan, zm::ST_DY, false, in, out, delta, stream);
}
int zm_dx_real(zm_plan plan, const void *in, void *out, double delta, void *stream) {
    return stencil_call(plan, zm::ST_DX, true, in, out, delta, stream);
}
int zm_dy_real(zm_plan plan, const void *in, void *out, double delta, void *stream) {
    return stencil_call(plan, zm::ST_DY, true, in, out, delta, stream);
}
int zm_laplace_vjp(zm_plan plan, const void *grad_out, void *grad_in, double inv_h2, void *stream) {
    // the periodic Laplacian is a symmetric real operator: its adjoint is itself
    return stencil_call(plan, zm::ST_LAPLACE, false, grad_out, grad_in, inv_h2, stream);
}
int zm_dx_vjp(zm_plan plan, const void *grad_out, void *grad_in, double delta, void *stream) {
    // antisymmetric: adjoint = -dx, i.e. the same stencil with delta -> -delta (exact negation)
    return stencil_call(plan, zm::ST_DX, false, grad_out, grad_in, -delta, stream);
}
int zm_dy_vjp(zm_plan plan, const void *grad_out, void *grad_in, double delta, void *stream) {
    return stencil_call(plan, zm::ST_DY, false, grad_out, grad_in, -delta, stream);
}

static int convert_call(zm_plan plan, bool recip, bool to_nat, const void *in, void *out, void *stream) {
    int rc;
    if ((rc = check_device_plan(plan))) return rc;
    if ((rc = check_field(plan, in, "in")) || (rc = check_field(plan, out, "out"))) return rc;
    if (overlap(in, out, plan->total * plan->elem_bytes)) return fail(ZM_ERR_INVALID_ARG, "in and out overlap");
    cudaError_t e = zm::launch_convert(plan, recip, to_nat, in, out, as_stream(stream));
    if (e != cudaSuccess) return cuda_fail(e, "layout conversion launch");
    return ZM_OK;
}
int zm_natural_to_real(zm_plan plan, const void *natural, void *interleaved, void *stream) {
    return convert_call(plan, false, false, natural, interleaved, stream);
}
int zm_real_to_natural(zm_plan plan, const void *interleaved, void *natural, void *stream) {
    return convert_call(plan, false, true, interleaved, natural, stream);
}
int zm_natural_to_reciprocal(zm_plan plan, const void *natural, void *interleaved, void *stream) {
    return convert_call(plan, true, false, natural, interleaved, stream);
}
int zm_reciprocal_to_natural(zm_plan plan, const void *interleaved, void *natural, void *stream) {
    return convert_call(plan, true, true, interleaved, natural, stream);
}

int zm_spectral_apply(zm_plan plan, void *data, int op, double a, void *stream) {
    int rc;
    if ((rc = check_device_plan(plan))) return rc;
    if ((rc = check_field(plan, data, "data"))) return rc;
    if (op < ZM_SPECTRAL_GAUSSIAN || op > ZM_SPECTRAL_SCALE) return fail(ZM_ERR_INVALID_ARG, "unknown op %d", op);
    if (op != ZM_SPECTRAL_SCALE && a == 0.0) return fail(ZM_ERR_INVALID_ARG, "parameter a must be non-zero");
    cudaError_t e = zm::launch_spectral(plan, data, op, a, as_stream(stream));
    if (e != cudaSuccess) return cuda_fail(e, "spectral launch");
    return ZM_OK;
}

int zm_spectral_apply_vjp(zm_plan plan, void *grad, int op, double a, void *stream) {
    // every operator is a real diagonal multiplier, hence self-adjoint
    return zm_spectral_apply(plan, grad, op, a, stream);
}

int zm_fill_field(zm_plan plan, void *interleaved, int kind, uint64_t seed, void *stream) {
    int rc;
    if ((rc = check_device_plan(plan))) return rc;
    if ((rc = check_field(plan, interleaved, "interleaved"))) return rc;
    if (kind != ZM_FIELD_UNIFORM && kind != ZM_FIELD_GAUSSIAN) return fail(ZM_ERR_INVALID_ARG, "unknown kind %d", kind);
    cudaError_t e = zm::launch_fill(plan, interleaved, kind, seed, as_stream(stream));
    if (e != cudaSuccess) return cuda_fail(e, "fill launch");
    return ZM_OK;
}

int zm_fill_modes(zm_plan plan, void *interleaved, int nmodes, const int64_t *modes,
                  const double *amps, double noise, uint64_t seed, void *stream) {
    int rc;
    if ((rc = check_device_plan(plan))) return rc;
    if ((rc = check_field(plan, interleaved, "interleaved"))) return rc;
    if (plan->g.dim != 2) return fail(ZM_ERR_UNSUPPORTED, "zm_fill_modes is 2D only");
    if (nmodes < 0 || nmodes > 64) return fail(ZM_ERR_INVALID_ARG, "nmodes must be in [0, 64]");
    if (nmodes > 0 && (!modes || !amps)) return fail(ZM_ERR_INVALID_ARG, "modes/amps NULL");
    cudaError_t e = zm::launch_fill_modes(plan, interleaved, nmodes, modes, amps, noise, seed,
                                          as_stream(stream));
    if (e != cudaSuccess) return cuda_fail(e, "fill_modes launch");
    return ZM_OK;
}

// ------------------------------------------------------------- index maps
int zm_real_to_global(zm_plan plan, int64_t rid, int64_t cid, int64_t did, int64_t ld, int64_t lr,
                      int64_t lc, int64_t *gd, int64_t *gr, int64_t *gc) {
    int rc;
    if ((rc = check_plan(plan))) return rc;
    if (!gd || !gr || !gc) return fail(ZM_ERR_INVALID_ARG, "null output");
    const Geom &g = plan->g;
    const int64_t L = g.L;
    if (rid < 0 || rid >= g.p || cid < 0 || cid >= g.p || lr < 0 || lr >= L || lc < 0 || lc >= L ||
        (g.dim == 3 && (did < 0 || did >= g.p || ld < 0 || ld >= L)))
        return fail(ZM_ERR_INVALID_ARG, "index out of range");
    const int64_t bcc = lc / g.vec + (lc % g.vec) * g.b;                         // utils.h:122-124
    *gr = (lr / g.b) * g.b * g.p + rid * g.b + (lr % g.b);                       // utils.h:168
    *gc = (bcc / g.b) * g.b * g.p + cid * g.b + (bcc % g.b);                     // utils.h:169
    *gd = g.dim == 3 ? (ld / g.b) * g.b * g.p + did * g.b + (ld % g.b) : 0;     // utils.h:195
    return ZM_OK;
}

int zm_global_to_real(zm_plan plan, int64_t gd, int64_t gr, int64_t gc, int64_t *rid, int64_t *cid,
                      int64_t *did, int64_t *ld, int64_t *lr, int64_t *lc) {
    int rc;
    if ((rc = check_plan(plan))) return rc;
    if (!rid || !cid || !did || !ld || !lr || !lc) return fail(ZM_ERR_INVALID_ARG, "null output");
    const Geom &g = plan->g;
    if (gr < 0 || gr >= g.n || gc < 0 || gc >= g.n || (g.dim == 3 && (gd < 0 || gd >= g.n)))
        return fail(ZM_ERR_INVALID_ARG, "index out of range");
    *rid = (gr / g.b) % g.p;                                                     // utils.h:178-186
    *lr = (gr / (g.b * g.p)) * g.b + (gr % g.b);
    *cid = (gc / g.b) % g.p;
    const int64_t bcc = (gc / (g.b * g.p)) * g.b + (gc % g.b);
    *lc = (bcc % g.b) * g.vec + bcc / g.b;
    if (g.dim == 3) {
        *did = (gd / g.b) % g.p;                                                 // utils.h:205-206
        *ld = (gd / (g.b * g.p)) * g.b + (gd % g.b);
    } else {
        *did = 0;
        *ld = 0;
    }
    return ZM_OK;
}

static int64_t h_lp(const Geom &g, int64_t i) { return i / g.vp + (i % g.vp) * g.m; }      // utils.h:232
static int64_t h_ct(const Geom &g, int64_t q) { return (q % g.m) * g.vec + q / g.m; }      // utils.h:238
static int64_t h_lp_inv(const Geom &g, int64_t j) { return (j % g.m) * g.vp + j / g.m; }  // utils.h:243
static int64_t h_ct_inv(const Geom &g, int64_t k) { return (k % g.vec) * g.m + k / g.vec; }  // utils.h:249

int zm_reciprocal_to_global(zm_plan plan, int64_t rid, int64_t cid, int64_t did, int64_t ld,
                            int64_t lr, int64_t lc, int64_t *kd, int64_t *kr, int64_t *kc) {
    int rc;
    if ((rc = check_plan(plan))) return rc;
    if (!kd || !kr || !kc) return fail(ZM_ERR_INVALID_ARG, "null output");
    const Geom &g = plan->g;
    const int64_t L = g.L;
    if (rid < 0 || rid >= g.p || cid < 0 || cid >= g.p || lr < 0 || lr >= L || lc < 0 || lc >= L ||
        (g.dim == 3 && (did < 0 || did >= g.p || ld < 0 || ld >= L)))
        return fail(ZM_ERR_INVALID_ARG, "index out of range");
    if (g.dim == 2) {                                                            // utils.h:265-268
        *kc = h_ct(g, cid * L + h_lp(g, lr));
        *kr = h_ct(g, rid * L + h_lp(g, lc));
        *kd = 0;
    } else {                                                                     // utils.h:298-302
        *kc = h_ct(g, cid * L + h_lp(g, lr));
        *kr = h_ct(g, rid * L + h_lp(g, ld));
        *kd = h_ct(g, did * L + h_lp(g, lc));
    }
    return ZM_OK;
}

int zm_global_to_reciprocal(zm_plan plan, int64_t kd, int64_t kr, int64_t kc, int64_t *rid,
                            int64_t *cid, int64_t *did, int64_t *ld, int64_t *lr, int64_t *lc) {
    int rc;
    if ((rc = check_plan(plan))) return rc;
    if (!rid || !cid || !did || !ld || !lr || !lc) return fail(ZM_ERR_INVALID_ARG, "null output");
    const Geom &g = plan->g;
    const int64_t L = g.L;
    if (kr < 0 || kr >= g.n || kc < 0 || kc >= g.n || (g.dim == 3 && (kd < 0 || kd >= g.n)))
        return fail(ZM_ERR_INVALID_ARG, "index out of range");
    const int64_t px = h_ct_inv(g, kc);                                          // utils.h:274-282
    *cid = px / L;
    *lr = h_lp_inv(g, px % L);
    const int64_t py = h_ct_inv(g, kr);
    *rid = py / L;
    if (g.dim == 2) {
        *lc = h_lp_inv(g, py % L);
        *did = 0;
        *ld = 0;
    } else {                                                                     // utils.h:308-320
        *ld = h_lp_inv(g, py % L);
        const int64_t pd = h_ct_inv(g, kd);
        *did = pd / L;
        *lc = h_lp_inv(g, pd % L);
    }
    return ZM_OK;
}

const char *zm_last_error_string(void) { return g_err.c_str(); }

const char *zm_status_string(int status) {
    switch (status) {
    case ZM_OK: return "ok";
    case ZM_ERR_INVALID_ARG: return "invalid argument";
    case ZM_ERR_CONSTRAINT: return "layout constraint violated";
    case ZM_ERR_MISALIGNED: return "misaligned pointer";
    case ZM_ERR_NO_MEMORY: return "out of memory";
    case ZM_ERR_CUDA: return "CUDA error";
    case ZM_ERR_TIMEOUT: return "device wait timed out";
    case ZM_ERR_UNSUPPORTED: return "unsupported";
    case ZM_ERR_WORKSPACE: return "workspace too small";
    default: return "unknown status";
    }
}

uint64_t zm_launch_count(void) { return g_launches.load(); }

const char *zm_version(void) { return "zmodel_b200 0.1 (sm_100a)"; }

}  // extern "C"
