// zm_batch.cu -- many independent 2D fields of uneven N in one persistent launch.
//
// A batch is a list of fields, each with its own (N, B, P) reference layout, packed one
// after the other in every batch buffer.  One call is one cooperative launch of
// batch_kernel: a grid of exactly the CTAs that fit on the device at once walks a short
// program of steps (an axis pass over all fields, a fused y pass, a stencil, a
// generator ...), with a grid barrier between steps.  Inside a pass step the work items
// are tiles of TL lines of one field, TL * N = a fixed number of points per tile, so the
// same CTA shape serves every N; a tile's field comes from a binary search over the
// fields' first tile numbers.  The tile code is the runtime-sized axis pass of
// zm_tile.cuh (the same Cooley-Tukey split and reference layouts as single-field plans).
#include <cuda/atomic>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <new>
#include <tuple>
#include <vector>

#include "zm_index.cuh"
#include "zm_internal.h"
#include "zm_tile.cuh"
#include "zmodel_b200.h"

namespace zm {

constexpr int kBatchThreads = 256;
constexpr int kMaxSteps = 6;
constexpr unsigned long long kBarrierTimeoutNs = 2000000000ull;   // 2 s

struct BatchField {
    Geom g;
    int64_t off;       // element offset in a batch buffer
    int64_t tile0;     // first tile of this field in a pass step's tile sequence
    const void *twN;   // the field plan's twiddle table w_N^m (tw<T> entries)
    int T;             // lines per tile
    int nst_vec, nst_m;
    int rad_vec[8], rad_m[8];
};

enum BatchOp : int {
    BOP_X_FWD = 0,     // x pass forward: real layout -> REPACK layout
    BOP_Y_FWD = 1,     // y pass forward: REPACK layout -> reciprocal layout
    BOP_Y_INV = 2,     // y pass inverse
    BOP_X_INV = 3,     // x pass inverse (scale 1/N^2 when step.scale)
    BOP_Y_POISSON = 4, // y pass forward, divide by -|k|^2, y pass inverse (in place)
    BOP_RESIDUAL = 5,  // out = Lap(in) / h^2 - aux (5-point, periodic)
    BOP_FILL = 6,      // out = generator(kind, seed + field) in the real layout
    BOP_NOP = 7        // nothing (barrier probe)
};

struct BatchStep {
    int op;
    int kind;          // BOP_FILL: zm_field_kind
    int scale;         // BOP_X_INV: apply 1/N^2
    const void *in;
    void *out;
    const void *aux;
    double a;          // BOP_Y_POISSON: 2 pi / length; BOP_RESIDUAL: 1 / length
    uint64_t seed;
};

struct BatchParams {
    const BatchField *fields;
    int nfields;
    int64_t tiles;
    int nsteps;
    BatchStep step[kMaxSteps];
    unsigned *bar;     // [0] arrivals, [1] generation
    int *abort;        // this launch only: set by a barrier that timed out, the others give up
    int *err;          // sticky: set by a barrier that timed out, read and cleared by zm_batch_status
    unsigned missing;  // arrivals a barrier waits for beyond the grid (0; > 0 only in the probe)
};

ZM_DEV unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Grid-wide barrier of a cooperative launch (all CTAs resident).  Sense by generation
// count; the last CTA to arrive resets the arrival count and releases the generation.
// A wait longer than kBarrierTimeoutNs, or an abort already raised by another CTA of
// this launch, makes every waiting CTA give up: returns false and the kernel returns.
// A timeout also raises the sticky error word that zm_batch_status reports; the abort
// word is cleared before every launch, so one timeout ends only its own launch.
ZM_DEV bool grid_barrier(unsigned *bar, unsigned nblocks, int *abort, int *err, int *s_ok) {
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        cuda::atomic_ref<unsigned, cuda::thread_scope_device> cnt(bar[0]), gen(bar[1]);
        cuda::atomic_ref<int, cuda::thread_scope_device> flag(*abort), sticky(*err);
        const unsigned g0 = gen.load(cuda::memory_order_acquire);
        if (cnt.fetch_add(1u, cuda::memory_order_acq_rel) == nblocks - 1) {
            cnt.store(0u, cuda::memory_order_relaxed);
            gen.fetch_add(1u, cuda::memory_order_release);
        } else {
            const unsigned long long t0 = globaltimer_ns();
            while (gen.load(cuda::memory_order_acquire) == g0) {
                if (flag.load(cuda::memory_order_relaxed) != 0 ||
                    globaltimer_ns() - t0 > kBarrierTimeoutNs) {
                    flag.store(1, cuda::memory_order_relaxed);
                    sticky.store(1, cuda::memory_order_relaxed);
                    ok = 0;
                    break;
                }
                __nanosleep(128);
            }
        }
        *s_ok = ok;
    }
    __syncthreads();
    return *s_ok != 0;
}

// largest f with fields[f].tile0 <= tile
ZM_DEV int field_of_tile(const BatchField *fields, int nfields, int64_t tile) {
    int lo = 0, hi = nfields - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (fields[mid].tile0 <= tile) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// global (row, col) -> element of the real layout (inverse of real_gidx, 2D)
ZM_DEV int64_t real_elem(int64_t gr, int64_t gc, const Geom &g) {
    const int64_t rid = (gr >> g.logB) & (g.p - 1);
    const int64_t lr = ((gr >> (g.logB + g.logP)) << g.logB) + (gr & (g.b - 1));
    const int64_t cid = (gc >> g.logB) & (g.p - 1);
    const int64_t pos = ((gc & (g.b - 1)) << g.logVEC) + (gc >> (g.logB + g.logP));
    return (((rid << g.logP) + cid) << (2 * g.logL)) + (lr << g.logL) + pos;
}

// Both sub-transforms of a tile: compile-time-sized stages (LMC = log2 M) for the
// complex64 tiles with VEC = 4 and P = 2 or 4 (the layout the B autotuner picks for the
// batch sizes, B = N / 8 at P = 2), or the runtime-sized stages (LMC = 0) for every other
// shape.  (LMC > 0: the column sub-transform only; the row stage runs fused with the
// vector-side sweep, tile_load_rows_v4 / tile_rows_store_v4)
template <typename T, int EPT, bool INV, int LM, typename SW>
__device__ __noinline__ void tile_transform_v4(cpx<T> *s, int tid, const tw<T> *twN) {
    tile_transform_ct<T, EPT, INV, 2, LM, kBatchThreads, SW, false>(s, tid, twN);
}
template <typename T, int EPT, bool INV, int LMC, typename SW>
ZM_DEV void batch_tile_transform(cpx<T> *s, const BatchField &f, int nthr, int tid, const tw<T> *twN) {
    if constexpr (LMC > 0) {
        tile_transform_v4<T, EPT, INV, LMC, SW>(s, tid, twN);
    } else {
        const Geom &g = f.g;
        tile_transform<T, EPT, INV>(s, g, f.rad_vec, f.nst_vec, f.rad_m, f.nst_m, nthr, tid, twN);
    }
}

// One tile of an axis-pass step: load, transform(s), store.  SW is the shared-memory
// slot permutation of the tile (SwzV4 for the compile-time VEC = 4 tiles).
template <typename T, int EPT, int LMC, typename SW, int LP = 0>
__device__ __noinline__ void batch_tile(int op, bool scale, double a, const BatchField &sf, const Tile c, cpx<T> *s,
                                        const cpx<T> *in, cpx<T> *out, int64_t l0, int nthr, int tid) {
    const Geom &g = sf.g;
    const tw<T> *twN = reinterpret_cast<const tw<T> *>(sf.twN);
    const bool xpass = op == BOP_X_FWD || op == BOP_X_INV;
    // vector-side sweeps: plain, or with the VEC = 4 row stage fused in and every size
    // fixed (LMC > 0, P = 2^LP); likewise the frequency-side sweeps
    auto load_vec = [&]() {
        if constexpr (LMC > 0) {
            if (xpass) tile_load_rows_v4<EPT, LMC, LP, true, kBatchThreads, SW>(c, s, in, tid);
            else tile_load_rows_v4<EPT, LMC, LP, false, kBatchThreads, SW>(c, s, in, tid);
        } else {
            tile_load_vec<EPT, SW>(c, g, s, in, nthr, tid);
        }
    };
    auto store_vec = [&](bool scl, T sc) {
        if constexpr (LMC > 0) {
            if (xpass) tile_rows_store_v4<EPT, LMC, LP, true, kBatchThreads, SW>(c, s, out, scl, sc, (T)0, twN, tid);
            else tile_rows_store_v4<EPT, LMC, LP, false, kBatchThreads, SW>(c, s, out, scl, sc, (T)0, twN, tid);
        } else {
            tile_store_vec<EPT, SW>(c, g, s, out, scl, sc, (T)0, nthr, tid);
        }
    };
    auto store_freq = [&]() {
        if constexpr (LMC > 0) {
            if (xpass) tile_freq_v4<EPT, LMC, LP, true, kBatchThreads, false, SW>(c, s, in, out, tid);
            else tile_freq_v4<EPT, LMC, LP, false, kBatchThreads, false, SW>(c, s, in, out, tid);
        } else {
            tile_store_freq<EPT, SW>(c, g, s, out, false, (T)1, (T)0, nthr, tid);
        }
    };
    auto load_freq = [&]() {
        if constexpr (LMC > 0) {
            if (xpass) tile_freq_v4<EPT, LMC, LP, true, kBatchThreads, true, SW>(c, s, in, out, tid);
            else tile_freq_v4<EPT, LMC, LP, false, kBatchThreads, true, SW>(c, s, in, out, tid);
        } else {
            tile_load_freq<EPT, SW>(c, g, s, in, nthr, tid);
        }
    };
    if (op == BOP_X_FWD || op == BOP_Y_FWD) {
        load_vec();
        __syncthreads();
        batch_tile_transform<T, EPT, false, LMC, SW>(s, sf, nthr, tid, twN);
        store_freq();
    } else if (op == BOP_X_INV || op == BOP_Y_INV) {
        load_freq();
        __syncthreads();
        batch_tile_transform<T, EPT, true, LMC, SW>(s, sf, nthr, tid, twN);
        const bool scl = scale && xpass;
        const T sc = (T)(1.0 / ((double)g.n * (double)g.n));
        store_vec(scl, sc);
    } else {   // BOP_Y_POISSON
        load_vec();
        __syncthreads();
        batch_tile_transform<T, EPT, false, LMC, SW>(s, sf, nthr, tid, twN);
        // slot (t, k1, k2) holds the frequency the y pass would store at rank
        // (rid = k2 / VP, cid), local row p, column pos = k1 VP + k2 % VP
        // (reciprocal_to_global, utils.h:265-268): along the transform that is
        // d_ct(rid L + d_lp(pos)) = d_ct(k2 M + k1) = k1 VEC + k2 = r, the slot position
        // itself; along the lines d_ct(cid L + d_lp(p)) of line l0 + t.  The factor
        // -1 / (a^2 |k|^2) in the working precision (|k|^2 an exact integer).
        const T a2 = (T)(a * a);
        auto divide = [&](int e, int ka, int r, int nh, int n) {
            const int sa = ka >= nh ? ka - n : ka, sb = r >= nh ? r - n : r;
            const int ksq = sa * sa + sb * sb;
            T fac;
            if constexpr (sizeof(T) == 4) fac = ksq == 0 ? 0.f : -__frcp_rn(a2 * (float)ksq);
            else fac = ksq == 0 ? 0.0 : -1.0 / (a2 * (double)ksq);
            const cpx<T> v = s[SW::f(e)];
            s[SW::f(e)] = {v.x * fac, v.y * fac};
        };
        if constexpr (LMC > 0) {
            // the same with the sizes fixed: ka = ct(cid L + lp(p)) in 32-bit constant shifts
            using G = V4Geom<LMC, LP, false>;
            constexpr int M = 1 << LMC, LVP = G::LVP, VP = G::VP;
#pragma unroll 4
            for (int e = tid; e < EPT * kBatchThreads; e += kBatchThreads) {
                const int t = e >> G::LN, r = e & (G::N - 1);
                const int l = (int)l0 + t, cid = l >> G::LL, p = l & (G::L - 1);
                const int q = (cid << G::LL) + (p >> LVP) + ((p & (VP - 1)) << LMC);
                divide(e, ((q & (M - 1)) << 2) + (q >> LMC), r, G::N / 2, G::N);
            }
        } else {
            const int tot = sf.T << g.logN;
            for (int e = tid; e < tot; e += nthr) {
                const int t = e >> g.logN, r = e & (int)(g.n - 1);
                const int64_t l = l0 + t, cid = l >> g.logL, p = l & (g.L - 1);
                divide(e, (int)d_ct(cid * g.L + d_lp(p, g), g), r, (int)(g.n >> 1), (int)g.n);
            }
        }
        __syncthreads();
        batch_tile_transform<T, EPT, true, LMC, SW>(s, sf, nthr, tid, twN);
        store_vec(false, (T)1);
    }
}

// One tile of the residual step, out = Lap_h(in) - rhs over elements [e0, e0 + TP) of a
// field (5-point, periodic, h = length / N, a = 1 / length); its own function so that its
// registers do not weigh on the rest of the persistent kernel.
template <typename T, int TP>
__device__ __noinline__ void residual_tile(const Geom &g, double a, const cpx<T> *in, const cpx<T> *rhs, cpx<T> *out,
                                           int64_t e0, int nthr, int tid) {
    const T inv_h2 = (T)((double)g.n * a * (double)g.n * a);
    const int64_t m = g.n - 1;
    auto resid = [&](const cpx<T> &up, const cpx<T> &dn, const cpx<T> &lf, const cpx<T> &rt,
                     const cpx<T> &c, const cpx<T> &r) -> cpx<T> {
        const T lx = up.x + dn.x + lf.x + rt.x - (T)4 * c.x;
        const T ly = up.y + dn.y + lf.y + rt.y - (T)4 * c.y;
        return {lx * inv_h2 - r.x, ly * inv_h2 - r.y};
    };
    if constexpr (sizeof(T) == 4) {
        // Pairs (e, e + 1), e even: the two share rank and row (L is even), so
        // their up / down neighbours are again two adjacent elements, and so
        // are left / right except at a block edge.  Adjacent 16-byte-aligned
        // pairs move as one 16-byte access, anything else element by element.
        auto ld2 = [](const cpx<T> *p0, const cpx<T> *p1, cpx<T> &v0, cpx<T> &v1) {
            if (p1 == p0 + 1 && ((uintptr_t)p0 & 15) == 0) {
                const float4 q = __ldg(reinterpret_cast<const float4 *>(p0));
                v0 = {q.x, q.y};
                v1 = {q.z, q.w};
            } else {
                v0 = ldg(p0);
                v1 = ldg(p1);
            }
        };
        // Inside a rank's B x B block (in-block column j = pos >> log VEC and
        // row lr mod B both off the block's edges) the four neighbours of the
        // pair sit in the same rank at -L, +L (rows) and -VEC, +VEC (columns:
        // the next global column is the next in-block column of the same
        // block cycle), adjacent pairs again when VEC >= 2.
        const bool fast = g.logVEC >= 1 &&
                          (((uintptr_t)in | (uintptr_t)rhs | (uintptr_t)out) & 15) == 0;
        // the geometry in registers (g lives in shared memory; a field holds < 2^31 elements)
        const int iL = (int)g.L, iV = (int)g.vec, bm = (int)g.b - 1, logL = g.logL, logV = g.logVEC;
        auto q4 = [](const cpx<T> *q) { return __ldg(reinterpret_cast<const float4 *>(q)); };
        for (int i = tid; i < TP / 2; i += nthr) {
            const int64_t e = e0 + 2 * i;
            const int pos = (int)e & (iL - 1), lr = ((int)e >> logL) & (iL - 1);
            const int j = pos >> logV, rb = lr & bm;
            if (fast && j > 0 && j < bm && rb > 0 && rb < bm) {
                const cpx<T> *pc = in + e;
                const float4 up = q4(pc - iL), dn = q4(pc + iL), lf = q4(pc - iV), rt = q4(pc + iV);
                const float4 cc = q4(pc), rr = q4(rhs + e);
                const cpx<T> o0 = resid({up.x, up.y}, {dn.x, dn.y}, {lf.x, lf.y}, {rt.x, rt.y},
                                        {cc.x, cc.y}, {rr.x, rr.y});
                const cpx<T> o1 = resid({up.z, up.w}, {dn.z, dn.w}, {lf.z, lf.w}, {rt.z, rt.w},
                                        {cc.z, cc.w}, {rr.z, rr.w});
                *reinterpret_cast<float4 *>(out + e) = make_float4(o0.x, o0.y, o1.x, o1.y);
                continue;
            }
            const int64_t gi0 = real_gidx(e, g), gc1 = real_gidx(e + 1, g) & m;
            const int64_t gr = gi0 >> g.logN, gc0 = gi0 & m;
            const int64_t au = real_elem((gr - 1) & m, gc0, g), ad = real_elem((gr + 1) & m, gc0, g);
            cpx<T> up0, up1, dn0, dn1, lf0, lf1, rt0, rt1, c0, c1, r0, r1;
            ld2(in + au, in + au + 1, up0, up1);
            ld2(in + ad, in + ad + 1, dn0, dn1);
            ld2(in + real_elem(gr, (gc0 - 1) & m, g), in + real_elem(gr, (gc1 - 1) & m, g), lf0, lf1);
            ld2(in + real_elem(gr, (gc0 + 1) & m, g), in + real_elem(gr, (gc1 + 1) & m, g), rt0, rt1);
            ld2(in + e, in + e + 1, c0, c1);
            ld2(rhs + e, rhs + e + 1, r0, r1);
            const cpx<T> o0 = resid(up0, dn0, lf0, rt0, c0, r0);
            const cpx<T> o1 = resid(up1, dn1, lf1, rt1, c1, r1);
            cpx<T> *po = out + e;
            if (((uintptr_t)po & 15) == 0) {
                *reinterpret_cast<float4 *>(po) = make_float4(o0.x, o0.y, o1.x, o1.y);
            } else {
                po[0] = o0;
                po[1] = o1;
            }
        }
    } else {
        for (int i = tid; i < TP; i += nthr) {
            const int64_t e = e0 + i;
            const int64_t gi = real_gidx(e, g);
            const int64_t gr = gi >> g.logN, gc = gi & m;
            const cpx<T> up = ldg(in + real_elem((gr - 1) & m, gc, g));
            const cpx<T> dn = ldg(in + real_elem((gr + 1) & m, gc, g));
            const cpx<T> lf = ldg(in + real_elem(gr, (gc - 1) & m, g));
            const cpx<T> rt = ldg(in + real_elem(gr, (gc + 1) & m, g));
            out[e] = resid(up, dn, lf, rt, ldg(in + e), ldg(rhs + e));
        }
    }
}

template <typename T, int EPT>
__global__ void __launch_bounds__(kBatchThreads, 4) batch_kernel(const BatchParams bp) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpx<T> *s = reinterpret_cast<cpx<T> *>(smem_raw);
    __shared__ int64_t s_abase[64], s_fbase[64];
    __shared__ BatchField sf;
    __shared__ int s_ok, s_f;
    const int tid = threadIdx.x, nthr = blockDim.x;

    for (int st = 0; st < bp.nsteps; st++) {
        if (st > 0 && !grid_barrier(bp.bar, gridDim.x + bp.missing, bp.abort, bp.err, &s_ok)) return;
        const BatchStep S = bp.step[st];
        if (S.op == BOP_NOP) continue;

        if (S.op == BOP_RESIDUAL || S.op == BOP_FILL) {
            // element-wise steps over the pass steps' tiles: tile `tile` of field f covers
            // elements [(tile - tile0) * TP, + TP) of the field's array (N^2 / TP tiles of a
            // field of N^2 elements), so every CTA has work whatever the field sizes
            constexpr int TP = kBatchThreads * EPT;
            for (int64_t tile = blockIdx.x; tile < bp.tiles; tile += gridDim.x) {
                __syncthreads();   // the previous tile is done with sf
                if (tid == 0) {
                    s_f = field_of_tile(bp.fields, bp.nfields, tile);
                    sf = bp.fields[s_f];
                }
                __syncthreads();
                const int f = s_f;
                const Geom g = sf.g;
                const int64_t e0 = (tile - sf.tile0) * TP;
                cpx<T> *out = reinterpret_cast<cpx<T> *>(S.out) + sf.off;
                if (S.op == BOP_FILL) {
                    const uint64_t seed = S.seed + (uint64_t)f;
                    for (int i = tid; i < TP; i += nthr) {
                        const int64_t e = e0 + i;
                        const uint64_t gi = (uint64_t)real_gidx(e, g);
                        double re, im;
                        if (S.kind == 0) {
                            re = u01(seed, gi, 0) * 2.0 - 1.0;
                            im = u01(seed, gi, 1) * 2.0 - 1.0;
                        } else {
                            re = gauss(seed, gi, 0);
                            im = gauss(seed, gi, 1);
                        }
                        out[e] = {(T)re, (T)im};
                    }
                    continue;
                }
                const cpx<T> *in = reinterpret_cast<const cpx<T> *>(S.in) + sf.off;
                const cpx<T> *rhs = reinterpret_cast<const cpx<T> *>(S.aux) + sf.off;
                residual_tile<T, TP>(sf.g, S.a, in, rhs, out, e0, nthr, tid);
            }
            continue;
        }

        // axis-pass steps: tiles of TL lines, TL * N = nthr * EPT points
        for (int64_t tile = blockIdx.x; tile < bp.tiles; tile += gridDim.x) {
            __syncthreads();   // the previous tile is done with sf, the bases and s
            if (tid == 0) sf = bp.fields[field_of_tile(bp.fields, bp.nfields, tile)];
            __syncthreads();
            const Geom &g = sf.g;
            const int64_t l0 = (tile - sf.tile0) * sf.T;
            const bool xpass = S.op == BOP_X_FWD || S.op == BOP_X_INV;
            const Tile c = tile_begin(g, xpass ? PASS_X2 : PASS_Y2, l0, sf.T, s_abase, s_fbase, nthr, tid);
            __syncthreads();
            const cpx<T> *in = reinterpret_cast<const cpx<T> *>(S.in) + sf.off;
            cpx<T> *out = reinterpret_cast<cpx<T> *>(S.out) + sf.off;
            // slot permutation per column length (SwzX, zm_tile.cuh)
#define ZM_BT(LMC, ...)                                                                                \
    (g.logP == 1 ? batch_tile<T, EPT, LMC, __VA_ARGS__, 1>(S.op, S.scale != 0, S.a, sf, c, s, in, out, l0, nthr, tid) \
                 : batch_tile<T, EPT, LMC, __VA_ARGS__, 2>(S.op, S.scale != 0, S.a, sf, c, s, in, out, l0, nthr, tid))
            bool done = false;
            if constexpr (sizeof(T) == 4 && EPT == 16) {
                if (g.logVEC == 2 && (g.logP == 1 || g.logP == 2)) {
                    done = true;
                    switch (g.logM) {
                    case 4: ZM_BT(4, SwzX<4, 8, 4, 6, 0>); break;
                    case 5: ZM_BT(5, SwzX<3, 9, 7, 4, 6>); break;
                    case 6: ZM_BT(6, SwzX<3, 8, 0, 4, 10>); break;
                    case 7: ZM_BT(7, SwzX<3, 4, 10, 5, 8>); break;
                    case 8: ZM_BT(8, SwzX<4, 9, 4, 6, 10>); break;
                    case 9: ZM_BT(9, SwzX<3, 10, 0, 4, 6>); break;
                    case 10: ZM_BT(10, SwzX<3, 0, 0, 4, 0>); break;
                    default: done = false; break;
                    }
                }
            }
#undef ZM_BT
            if (!done) batch_tile<T, EPT, 0, SwzNone>(S.op, S.scale != 0, S.a, sf, c, s, in, out, l0, nthr, tid);
        }
    }
}

template <typename T, int EPT>
static cudaError_t launch_batch_t(const BatchParams &bp, int grid, cudaStream_t st) {
    const size_t smem = sizeof(cpx<T>) * kBatchThreads * EPT;
    cudaError_t e = cudaMemsetAsync(bp.bar, 0, 3 * sizeof(unsigned), st);   // arrivals, generation, abort
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(kBatchThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    e = cudaLaunchKernelEx(&cfg, batch_kernel<T, EPT>, bp);
    count_launch();
    return e;
}

template <typename T, int EPT>
static int batch_grid_t(int device) {
    int per_sm = 0, sms = 0;
    const size_t smem = sizeof(cpx<T>) * kBatchThreads * EPT;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_kernel<T, EPT>, kBatchThreads, smem) !=
        cudaSuccess)
        return 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return 0;
    return per_sm * sms;
}

}  // namespace zm

// ================================================================== C ABI

struct zm_batch_s {
    int dtype;
    int device;
    int grid;
    std::vector<zm_plan> plans;            // distinct (N, B, P) plans (twiddle tables)
    std::vector<zm::BatchField> fields;    // host copy
    std::vector<int> field_plan;
    zm::BatchField *d_fields = nullptr;
    unsigned *d_sync = nullptr;            // [0..1] barrier, [2] abort (per launch), [3] sticky error flag
    int64_t tiles = 0, elems = 0;
};

namespace {

bool aligned16b(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

int check_batch(zm_batch b) {
    if (!b) return zm::report_error(ZM_ERR_INVALID_ARG, "null batch");
    return ZM_OK;
}

int check_buf(const void *p, const char *name) {
    if (!p) return zm::report_error(ZM_ERR_INVALID_ARG, "%s is NULL", name);
    if (!aligned16b(p)) return zm::report_error(ZM_ERR_MISALIGNED, "%s is not 16-byte aligned", name);
    return ZM_OK;
}

bool overlap_b(const void *a, const void *b, size_t bytes) {
    const char *x = static_cast<const char *>(a), *y = static_cast<const char *>(b);
    return x < y + bytes && y < x + bytes;
}

int launch(zm_batch b, const zm::BatchStep *steps, int nsteps, void *stream, unsigned missing = 0) {
    zm::BatchParams bp = {};
    bp.missing = missing;
    bp.fields = b->d_fields;
    bp.nfields = (int)b->fields.size();
    bp.tiles = b->tiles;
    bp.nsteps = nsteps;
    for (int i = 0; i < nsteps; i++) bp.step[i] = steps[i];
    bp.bar = b->d_sync;
    bp.abort = reinterpret_cast<int *>(b->d_sync + 2);
    bp.err = reinterpret_cast<int *>(b->d_sync + 3);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    cudaError_t e = b->dtype == ZM_C128 ? zm::launch_batch_t<double, 8>(bp, b->grid, st)
                                        : zm::launch_batch_t<float, 16>(bp, b->grid, st);
    if (e != cudaSuccess)
        return zm::report_error(ZM_ERR_CUDA, "batch launch: %s (%s)", cudaGetErrorName(e), cudaGetErrorString(e));
    return ZM_OK;
}

size_t batch_bytes(zm_batch b) { return (size_t)b->elems * (b->dtype == ZM_C128 ? 16 : 8); }

}  // namespace

extern "C" {

int zm_batch_create(zm_batch *batch, int nfields, const int64_t *n, const int64_t *b, const int64_t *p,
                    int dtype) {
    if (!batch) return zm::report_error(ZM_ERR_INVALID_ARG, "batch output pointer is NULL");
    *batch = nullptr;
    if (nfields < 1 || nfields > 65536) return zm::report_error(ZM_ERR_INVALID_ARG, "nfields=%d out of range [1, 65536]", nfields);
    if (!n || !b || !p) return zm::report_error(ZM_ERR_INVALID_ARG, "n, b and p must not be NULL");
    if (dtype != ZM_C128 && dtype != ZM_C64) return zm::report_error(ZM_ERR_INVALID_ARG, "unknown dtype %d", dtype);
    const int ept = zm::ept_for(dtype);
    const int64_t tile_pts = (int64_t)zm::kBatchThreads * ept;
    zm_batch_s *B = new (std::nothrow) zm_batch_s();
    if (!B) return zm::report_error(ZM_ERR_NO_MEMORY, "host allocation failed");
    B->dtype = dtype;
    cudaGetDevice(&B->device);
    std::map<std::tuple<int64_t, int64_t, int64_t>, int> seen;
    int rc = ZM_OK;
    for (int i = 0; i < nfields && rc == ZM_OK; i++) {
        if (n[i] < tile_pts / 64 || n[i] > tile_pts) {
            rc = zm::report_error(ZM_ERR_CONSTRAINT, "field %d: N=%lld outside the batch range [%lld, %lld]", i,
                                  (long long)n[i], (long long)(tile_pts / 64), (long long)tile_pts);
            break;
        }
        const auto key = std::make_tuple(n[i], b[i], p[i]);
        auto it = seen.find(key);
        int pi;
        if (it == seen.end()) {
            zm_plan pl = nullptr;
            rc = zm_plan_create(&pl, 2, n[i], b[i], p[i], dtype, 0);
            if (rc != ZM_OK) break;
            pi = (int)B->plans.size();
            B->plans.push_back(pl);
            seen.emplace(key, pi);
        } else {
            pi = it->second;
        }
        const zm_plan_s *pl = B->plans[pi];
        zm::BatchField f = {};
        f.g = pl->g;
        f.off = B->elems;
        f.tile0 = B->tiles;
        f.twN = pl->twN;
        f.T = (int)(tile_pts / n[i]);
        f.nst_vec = zm::radix_schedule(pl->g.vec, ept, f.rad_vec);
        f.nst_m = zm::radix_schedule(pl->g.m, ept, f.rad_m);
        B->fields.push_back(f);
        B->field_plan.push_back(pi);
        B->elems += (n[i] * n[i] + 1) & ~int64_t{1};
        B->tiles += n[i] / f.T;
    }
    if (rc == ZM_OK) {
        B->grid = dtype == ZM_C128 ? zm::batch_grid_t<double, 8>(B->device) : zm::batch_grid_t<float, 16>(B->device);
        if (B->grid <= 0) rc = zm::report_error(ZM_ERR_CUDA, "batch kernel occupancy query failed");
    }
    if (rc == ZM_OK) {
        const size_t fb = sizeof(zm::BatchField) * B->fields.size();
        cudaError_t e = cudaMalloc(&B->d_fields, fb);
        if (e == cudaSuccess) e = cudaMemcpy(B->d_fields, B->fields.data(), fb, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMalloc(&B->d_sync, 4 * sizeof(unsigned));
        if (e == cudaSuccess) e = cudaMemset(B->d_sync, 0, 4 * sizeof(unsigned));
        if (e != cudaSuccess)
            rc = zm::report_error(ZM_ERR_NO_MEMORY, "batch tables: %s", cudaGetErrorString(e));
    }
    if (rc != ZM_OK) {
        zm_batch_destroy(B);
        return rc;
    }
    *batch = B;
    return ZM_OK;
}

int zm_batch_destroy(zm_batch batch) {
    int rc;
    if ((rc = check_batch(batch))) return rc;
    for (zm_plan pl : batch->plans) zm_plan_destroy(pl);
    if (batch->d_fields) cudaFree(batch->d_fields);
    if (batch->d_sync) cudaFree(batch->d_sync);
    delete batch;
    return ZM_OK;
}

int zm_batch_get_field(zm_batch batch, int i, zm_batch_field *info) {
    int rc;
    if ((rc = check_batch(batch))) return rc;
    if (!info) return zm::report_error(ZM_ERR_INVALID_ARG, "info is NULL");
    if (i < 0 || i >= (int)batch->fields.size()) return zm::report_error(ZM_ERR_INVALID_ARG, "field %d out of range", i);
    const zm::BatchField &f = batch->fields[i];
    info->n = f.g.n;
    info->b = f.g.b;
    info->p = f.g.p;
    info->offset = f.off;
    info->elems = f.g.n * f.g.n;
    return ZM_OK;
}

int zm_batch_total_elems(zm_batch batch, int64_t *elems) {
    int rc;
    if ((rc = check_batch(batch))) return rc;
    if (!elems) return zm::report_error(ZM_ERR_INVALID_ARG, "elems is NULL");
    *elems = batch->elems;
    return ZM_OK;
}

int zm_batch_fill(zm_batch batch, void *data, int kind, uint64_t first_seed, void *stream) {
    int rc;
    if ((rc = check_batch(batch)) || (rc = check_buf(data, "data"))) return rc;
    if (kind != ZM_FIELD_UNIFORM && kind != ZM_FIELD_GAUSSIAN) return zm::report_error(ZM_ERR_INVALID_ARG, "unknown kind %d", kind);
    zm::BatchStep s = {};
    s.op = zm::BOP_FILL;
    s.kind = kind;
    s.out = data;
    s.seed = first_seed;
    return launch(batch, &s, 1, stream);
}

int zm_batch_forward(zm_batch batch, const void *in, void *out, void *stream) {
    int rc;
    if ((rc = check_batch(batch)) || (rc = check_buf(in, "in")) || (rc = check_buf(out, "out"))) return rc;
    if (overlap_b(in, out, batch_bytes(batch))) return zm::report_error(ZM_ERR_INVALID_ARG, "in and out overlap");
    zm::BatchStep s[2] = {};
    s[0].op = zm::BOP_X_FWD; s[0].in = in; s[0].out = out;
    s[1].op = zm::BOP_Y_FWD; s[1].in = out; s[1].out = out;
    return launch(batch, s, 2, stream);
}

int zm_batch_inverse(zm_batch batch, const void *in, void *out, void *work, int normalise, void *stream) {
    int rc;
    if ((rc = check_batch(batch)) || (rc = check_buf(in, "in")) || (rc = check_buf(out, "out"))) return rc;
    const size_t F = batch_bytes(batch);
    if (overlap_b(in, out, F)) return zm::report_error(ZM_ERR_INVALID_ARG, "in and out overlap");
    if (work) {
        if ((rc = check_buf(work, "work"))) return rc;
        if (overlap_b(work, in, F) || overlap_b(work, out, F))
            return zm::report_error(ZM_ERR_INVALID_ARG, "work overlaps in/out");
    }
    void *tmp = work ? work : const_cast<void *>(in);
    zm::BatchStep s[2] = {};
    s[0].op = zm::BOP_Y_INV; s[0].in = in; s[0].out = tmp;
    s[1].op = zm::BOP_X_INV; s[1].in = tmp; s[1].out = out; s[1].scale = normalise ? 1 : 0;
    return launch(batch, s, 2, stream);
}

int zm_batch_poisson(zm_batch batch, const void *rhs, void *phi, void *residual, void *work, double length,
                     void *stream) {
    int rc;
    if ((rc = check_batch(batch)) || (rc = check_buf(rhs, "rhs")) || (rc = check_buf(phi, "phi")) ||
        (rc = check_buf(work, "work")))
        return rc;
    if (residual && (rc = check_buf(residual, "residual"))) return rc;
    if (!(length > 0.0) || !std::isfinite(length)) return zm::report_error(ZM_ERR_INVALID_ARG, "length must be positive");
    const size_t F = batch_bytes(batch);
    if (overlap_b(rhs, phi, F) || overlap_b(rhs, work, F) || overlap_b(phi, work, F) ||
        (residual && (overlap_b(residual, rhs, F) || overlap_b(residual, phi, F) || overlap_b(residual, work, F))))
        return zm::report_error(ZM_ERR_INVALID_ARG, "rhs, phi, residual and work must not overlap");
    zm::BatchStep s[4] = {};
    const double two_pi = 6.283185307179586476925286766559;
    s[0].op = zm::BOP_X_FWD; s[0].in = rhs; s[0].out = work;
    s[1].op = zm::BOP_Y_POISSON; s[1].in = work; s[1].out = work; s[1].a = two_pi / length;
    s[2].op = zm::BOP_X_INV; s[2].in = work; s[2].out = phi; s[2].scale = 1;
    int ns = 3;
    if (residual) {
        s[3].op = zm::BOP_RESIDUAL; s[3].in = phi; s[3].aux = rhs; s[3].out = residual; s[3].a = 1.0 / length;
        ns = 4;
    }
    return launch(batch, s, ns, stream);
}

int zm_batch_status(zm_batch batch, int *device_error) {
    int rc;
    if ((rc = check_batch(batch))) return rc;
    if (!device_error) return zm::report_error(ZM_ERR_INVALID_ARG, "device_error is NULL");
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess)
        return zm::report_error(ZM_ERR_CUDA, "batch status: %s (%s)", cudaGetErrorName(e), cudaGetErrorString(e));
    int flag = 0;
    e = cudaMemcpy(&flag, batch->d_sync + 3, sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && flag) e = cudaMemset(batch->d_sync, 0, 4 * sizeof(unsigned));
    if (e != cudaSuccess)
        return zm::report_error(ZM_ERR_CUDA, "batch status: %s (%s)", cudaGetErrorName(e), cudaGetErrorString(e));
    *device_error = flag ? 1 : 0;
    return ZM_OK;
}

int zm_batch_barrier_probe(zm_batch batch, int missing, void *stream) {
    int rc;
    if ((rc = check_batch(batch))) return rc;
    if (missing < 0 || missing > 1) return zm::report_error(ZM_ERR_INVALID_ARG, "missing must be 0 or 1");
    zm::BatchStep s[2] = {};
    s[0].op = zm::BOP_NOP;
    s[1].op = zm::BOP_NOP;
    return launch(batch, s, 2, stream, (unsigned)missing);
}

int zm_batch_autotune_b(int64_t n, int64_t p, int dtype, int count, int reps, int64_t *best_b, float *best_ms) {
    if (count < 1 || reps < 1) return zm::report_error(ZM_ERR_INVALID_ARG, "count and reps must be >= 1");
    if (n <= 0 || p <= 0 || (n & (n - 1)) || (p & (p - 1)) || n % p)
        return zm::report_error(ZM_ERR_CONSTRAINT, "N and P must be powers of two with P | N");
    const int64_t L = n / p;
    int64_t best = 0;
    float best_t = 0.f;
    int rc = ZM_OK;
    for (int64_t b = 1; b <= L / p && rc == ZM_OK; b *= 2) {
        std::vector<int64_t> nv(count, n), bv(count, b), pv(count, p);
        zm_batch bt = nullptr;
        if (zm_batch_create(&bt, count, nv.data(), bv.data(), pv.data(), dtype) != ZM_OK) continue;   // B not allowed
        const size_t F = batch_bytes(bt);
        void *buf = nullptr;
        cudaError_t e = cudaMalloc(&buf, 4 * F);
        if (e != cudaSuccess) {
            zm_batch_destroy(bt);
            rc = zm::report_error(ZM_ERR_NO_MEMORY, "autotune buffers: %s", cudaGetErrorString(e));
            break;
        }
        char *c = static_cast<char *>(buf);
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        rc = zm_batch_fill(bt, c, ZM_FIELD_GAUSSIAN, 1, nullptr);
        for (int it = -1; it < reps && rc == ZM_OK; it++) {
            if (it == 0) cudaEventRecord(e0, nullptr);
            rc = zm_batch_poisson(bt, c, c + F, c + 2 * F, c + 3 * F, 1.0, nullptr);
        }
        cudaEventRecord(e1, nullptr);
        int flag = 0;
        if (rc == ZM_OK && (e = cudaEventSynchronize(e1)) != cudaSuccess)
            rc = zm::report_error(ZM_ERR_CUDA, "autotune timing: %s", cudaGetErrorString(e));
        if (rc == ZM_OK) rc = zm_batch_status(bt, &flag);
        if (rc == ZM_OK && flag) rc = zm::report_error(ZM_ERR_TIMEOUT, "autotune: batch barrier timed out");
        if (rc == ZM_OK) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            ms /= (float)reps;
            if (best == 0 || ms < best_t) {
                best = b;
                best_t = ms;
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaFree(buf);
        zm_batch_destroy(bt);
    }
    if (rc != ZM_OK) return rc;
    if (best == 0) return zm::report_error(ZM_ERR_CONSTRAINT, "no B is valid for N=%lld", (long long)n);
    if (best_b) *best_b = best;
    if (best_ms) *best_ms = best_t;
    return ZM_OK;
}

}  // extern "C"
