// zm_fft2.cuh -- size-specialised fused axis pass (the fast path of zm_fft.cu).
//
// Same computation as line_fft_kernel (see zm_fft.cu for how one pass replaces the
// reference's FFT1a / pack / All-to-All / unpack+twiddle / FFT1b / repack stages), with
// the sizes VEC = 2^LV and M = 2^LM fixed at compile time so every index, stride and
// radix is a constant:
//   * a tile of TL lines is held by a cluster of CL CTAs.  CTA rank r owns the rows
//     n1 in [r*M/CL, (r+1)*M/CL) for the VEC-point transforms and the columns
//     k2 in [r*VEC/CL, (r+1)*VEC/CL) for the M-point transforms; between the two the
//     rows' results are scattered to the owning CTA through distributed shared memory.
//     With CL = P this is the reference's row / column All-to-All, one CTA per virtual
//     rank; CL = 1 keeps the whole line in one CTA;
//   * each CTA's shared memory holds rows X[t][n1][p] and columns Y[t][k2][q] of its
//     slice -- one buffer, two views used at different times.  Rows are padded by one
//     element per RA1 points (columns by one per M), which keeps the Stockham write and
//     read patterns of every stage free of bank conflicts while every register of a
//     butterfly sits at a compile-time offset from its base;
//   * each sub-transform is at most two register stages of radix <= 16 (Stockham
//     indexing), with the stage twiddles w_VEC, w_M in shared memory and the inter-step
//     twiddle w_N^{n1 k2} as two compensated products in complex64 tiles held by one
//     CTA -- forward with two 16-point column stages: w_N^{j k2} w_N^{16 r k2} read
//     through L1 by lanes that share k2; otherwise two shared-memory factor tables --
//     or an FP64 power walk;
//   * one tile per cluster, the vector side moved through registers / 16-byte vectors;
//     or, for forward passes with two row stages in the persistent variants (PERS), a
//     cluster walks tiles c, c + clusters, ... and each CTA fetches the vector-side rows
//     of its NEXT tile with bulk asynchronous copies (cp.async.bulk, tracked by an
//     mbarrier with a bounded wait) into a staging buffer as soon as the current tile's
//     first row stage has read it, so HBM reads overlap the rest of the tile;
//   * the frequency side is read / written straight from registers with lanes ordered
//     so that a warp covers whole sectors;
//   * a forward tile asks for an L2 prefetch (cp.async.bulk.prefetch) of the vector
//     side of the tile one wave of clusters ahead.
#pragma once

#include <cooperative_groups.h>

#include "zm_common.cuh"

namespace zm {

template <typename T> ZM_DEV uint4 ldg16(const cpx<T> *p) {
    return __ldg(reinterpret_cast<const uint4 *>(p));
}

template <int CL> ZM_DEV void tile_sync() {
    if constexpr (CL > 1) cooperative_groups::this_cluster().sync();
    else __syncthreads();
}

// ------------------------------------------------ bulk copies tracked by an mbarrier
ZM_DEV unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
ZM_DEV void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
ZM_DEV void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
ZM_DEV void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
ZM_DEV bool mbar_try_wait(uint64_t *bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
ZM_DEV unsigned long long gtimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Wait for the mbarrier phase of the given parity; false after `limit_ns` without it.
ZM_DEV bool mbar_wait(uint64_t *bar, unsigned parity, unsigned long long limit_ns) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = gtimer_ns();
    while (!mbar_try_wait(bar, parity))
        if (gtimer_ns() - t0 > limit_ns) return false;
    return true;
}
// order this thread's earlier generic-proxy shared-memory accesses before its
// following async-proxy (bulk copy) accesses
ZM_DEV void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// global -> this CTA's shared memory, `bytes` a multiple of 16, both addresses 16-byte aligned
ZM_DEV void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"((unsigned long long)__cvta_generic_to_global(src)), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
constexpr unsigned long long kCopyWaitNs = 1000000000ull;   // 1 s
// hint: bring [src, src + bytes) into L2 (no completion to wait for); 16-byte aligned,
// bytes a multiple of 16
ZM_DEV void bulk_prefetch_l2(const void *src, unsigned bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"((unsigned long long)__cvta_generic_to_global(src)),
                 "r"(bytes)
                 : "memory");
}

// Shared-memory geometry and radix split of one CTA's slice.
template <int LV, int LM, int CL, int TL, int NT> struct SliceGeom {
    static constexpr int VEC = 1 << LV, M = 1 << LM, N = VEC * M;
    static constexpr int ML = M / CL, VL = VEC / CL;
    static constexpr int E = TL * N / CL;                    // elements per CTA
    static constexpr int EPT = E / NT;                       // elements per thread
    static constexpr int RA1 = VEC < EPT ? VEC : EPT, RA2 = VEC / RA1;
    static constexpr int RC1 = M < EPT ? M : EPT, RC2 = M / RC1;
    // rows: with two row stages one pad element per RA1 points (Stockham writes of
    // RA1 consecutive points by RA2 lanes land in distinct banks); else VEC + 2
    static constexpr bool PADX = RA2 > 1;
    static constexpr int XR = PADX ? VEC + RA2 : VEC + 2;
    static constexpr int YP = VEC <= 4 ? 1 : 0;              // pad per 16 in a column
    // padded column; for VEC <= 4 the column stages run with lanes over (VL columns) x
    // (16 / VL consecutive points), so the column stride is rounded up to 16 / VL (mod 16,
    // in 8-byte words of complex64) to keep those 16 lanes on 16 distinct bank pairs
    static constexpr int YR0 = M + M / 16;
    static constexpr int YRES = VL >= 16 ? 0 : 16 / VL;
    static constexpr int YR = VEC <= 4 ? YR0 + (((YRES - YR0) % 16) + 16) % 16 : M + 1;
    static constexpr int XE = TL * ML * XR, YE = TL * VL * YR;
    static constexpr int ELEMS = XE > YE ? XE : YE;
    static ZM_DEV int X(int t, int n1l, int p) { return (t * ML + n1l) * XR + p + (PADX ? p / RA1 : 0); }
    // rows of the inverse with one row stage (RA2 == 1) where every access is per element
    // or the element is 16 bytes: an odd stride VEC + 1, so that the column stage's
    // scatter, with lanes along 16 consecutive rows of one column, hits 16 distinct bank
    // pairs (the stride VEC + 2 of the 16-byte row reads repeats every 8 rows)
    static constexpr int XRI = VEC + 1;
    static_assert(PADX || XRI <= XR, "the odd-stride rows fit the slice");
    static ZM_DEV int XI(int t, int n1l, int p) { return (t * ML + n1l) * XRI + p; }
    // Column position swizzle for VEC <= 4 tiles of several lines: where lanes run over the
    // lines t first (a strided frequency side), lines t and t + 4 would sit on the same bank
    // pairs (their rows are 4 YR = 0 mod 16 words apart); q ^ ysw(t) spreads the eight
    // lines of a half-warp over the two quads of 16 that the second column (+ 4) leaves
    // free, and is a constant permutation inside each aligned 16 for every other access.
    static constexpr bool YSW = VEC <= 4 && TL >= 2;
    static_assert(!YSW || M >= 16, "swizzle stays inside an aligned run of 16 points");
    static ZM_DEV int ysw(int t) { return YSW ? ((t & 3) | (((t >> 2) & 1) << 3)) : 0; }
    static ZM_DEV int Y(int t, int k2l, int q) { return (t * VL + k2l) * YR + (q ^ ysw(t)) + (q >> 4) * YP; }
    // staging rows of the persistent forward pass: one row of sg interleaved lines
    // (sg VEC points, a bulk copy each); the stride keeps the first row stage's reads
    // (lanes over sg lines x RA2 points, then rows) free of bank conflicts
    static constexpr int SR(int sg) { return sg * VEC + (sg * RA2) % 16; }
    static constexpr int stage_elems(int sg) { return sg > TL ? 0 : (TL / sg) * ML * SR(sg); }
    // complex64 inter-step twiddles w_N^m = w_N^{(m >> TLO) 2^TLO} w_N^{m mod 2^TLO}:
    // two tables of NTA and NTB entries (hi/lo pairs) in shared memory.  Used by the
    // one-CTA-per-tile shapes; with a cluster the exchange through distributed shared
    // memory already saturates the shared-memory pipe, and the FP64 walk (FP64 and
    // conversion pipes) is faster there.
    static constexpr int LOGN = LV + LM, TLO = LOGN / 2;
    static constexpr int NTA = 1 << (LOGN - TLO), NTB = 1 << TLO;
    template <typename T> static constexpr bool twtab() { return sizeof(T) == 4 && CL == 1; }
    // complex64 one-CTA forward tiles with two 16-point column stages: the first column
    // stage runs with lanes along n1 mod 16 and splits w_N^{(j + 16 r) k2} into
    // w_N^{j k2} (once per unit) and w_N^{16 r k2} (the same for the 16 lanes of one k2),
    // both read through L1 from the plan's hi/lo table (no per-CTA table fill)
    template <typename T> static constexpr bool colq() { return twtab<T>() && RC2 == 16 && VEC > 4; }
    static constexpr int smax(int a, int b) { return a > b ? a : b; }
    static constexpr int STAGE_ELEMS = smax(stage_elems(1), smax(stage_elems(2), stage_elems(4)));
};

template <typename T, int LV, int LM, int CL, int TL, int NT>
constexpr size_t fused_tables_offset() {
    return sizeof(cpx<T>) * (size_t)SliceGeom<LV, LM, CL, TL, NT>::ELEMS;
}
// twiddle tables: w_VEC, w_M and, for complex64, the two inter-step tables
template <typename T, int LV, int LM, int CL, int TL, int NT>
constexpr size_t fused_twiddle_entries() {
    using SG = SliceGeom<LV, LM, CL, TL, NT>;
    return ((size_t)1 << LV) + ((size_t)1 << LM) + (SG::template twtab<T>() ? (size_t)(SG::NTA + SG::NTB) : 0);
}
template <typename T, int LV, int LM, int CL, int TL, int NT>
constexpr size_t fused_stage_offset() {
    return fused_tables_offset<T, LV, LM, CL, TL, NT>() + sizeof(tw<T>) * fused_twiddle_entries<T, LV, LM, CL, TL, NT>();
}

// Forward passes with two row stages can run persistent with a staging buffer (PERS,
// a tile-shape variant of its own) when it fits next to the slice in one CTA's 227 KB
// of shared memory.
template <typename T, int LV, int LM, int CL, int TL, int NT, bool INV, bool PERS>
constexpr bool fused_persistent() {
    return PERS && !INV && SliceGeom<LV, LM, CL, TL, NT>::RA2 > 1 &&
           fused_stage_offset<T, LV, LM, CL, TL, NT>() +
                   sizeof(cpx<T>) * (size_t)SliceGeom<LV, LM, CL, TL, NT>::STAGE_ELEMS <=
               (size_t)227 * 1024;
}

template <typename T, int LV, int LM, int CL, int TL, int NT, bool INV, bool PERS>
constexpr size_t fused_smem_bytes() {
    return fused_stage_offset<T, LV, LM, CL, TL, NT>() +
           (fused_persistent<T, LV, LM, CL, TL, NT, INV, PERS>()
                ? sizeof(cpx<T>) * (size_t)SliceGeom<LV, LM, CL, TL, NT>::STAGE_ELEMS
                : 0);
}

// CTAs per SM the register budget is sized for: 1024 / NT threads' worth, or fewer when
// shared memory cannot hold that many (the persistent passes with their staging buffer)
template <typename T, int LV, int LM, int CL, int TL, int NT, bool INV, bool PERS>
constexpr int fused_min_blocks() {
    constexpr int by_threads = NT < 1024 ? 1024 / NT : 1;
    constexpr int by_smem = (int)((size_t)228 * 1024 / (fused_smem_bytes<T, LV, LM, CL, TL, NT, INV, PERS>() + 1024));
    return by_smem < 1 ? 1 : (by_smem < by_threads ? by_smem : by_threads);
}

template <typename T, int LV, int LM, int CL, int TL, int NT, bool INV, bool PERS, bool TMS = false>
__global__ void __launch_bounds__(NT, (fused_min_blocks<T, LV, LM, CL, TL, NT, INV, PERS>()))
    fused_pass_kernel(const LineParams prm) {
    using SG = SliceGeom<LV, LM, CL, TL, NT>;
    constexpr int VEC = SG::VEC, M = SG::M;
    constexpr int ML = SG::ML, VL = SG::VL;
    constexpr int E = SG::E, EPT = SG::EPT;
    static_assert(ML >= 1 && VL >= 1 && ML * CL == M && VL * CL == VEC, "cluster split");
    static_assert(EPT * NT == E, "threads must divide the tile");
    constexpr int RA1 = SG::RA1, RA2 = SG::RA2, RC1 = SG::RC1, RC2 = SG::RC2;
    static_assert(RA2 <= EPT && RC2 <= EPT, "sub-transform needs more than two register stages");
    static_assert(EPT % RA1 == 0 && EPT % RA2 == 0 && EPT % RC1 == 0 && EPT % RC2 == 0, "radix");
    constexpr int DIR = INV ? 1 : -1;
    using C = cpx<T>;
    using Wt = tw<T>;

    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *S = reinterpret_cast<C *>(smem_raw);
    Wt *stv = reinterpret_cast<Wt *>(smem_raw + fused_tables_offset<T, LV, LM, CL, TL, NT>());  // w_VEC^m
    Wt *stm = stv + VEC;                                                                          // w_M^m
    Wt *sta = stm + M;                     // complex64: w_N^{a 2^TLO}, a < NTA
    Wt *stb = sta + SG::NTA;               // complex64: w_N^b, b < NTB
    __shared__ int64_t s_abase[TL], s_fbase[TL];
    __shared__ int64_t s_abase_n[TL], s_fbase_n[TL];   // TMS: the CTA's next tile
    __shared__ uint32_t s_tmem;                          // TMS: tensor-memory base address
    __shared__ uint64_t s_bar;

    int rank = 0;
    if constexpr (CL > 1) rank = (int)cooperative_groups::this_cluster().block_rank();
    const int n1_0 = rank * ML, k2_0 = rank * VL;   // first owned row / column
    const Geom &g = prm.g;
    int tid = threadIdx.x;   // not const: the TMS tile loop re-derives it opaquely per tile
    const C *in = reinterpret_cast<const C *>(prm.in);
    C *out = reinterpret_cast<C *>(prm.out);
    // strides of the pass (the same for every line)
    // (TMS: the pass's address form lives in shared memory, read where used, so that the
    // persistent tile loop does not hold it in registers)
    __shared__ LineAddr s_a0;
    const LineAddr a0r = line_addr(g, prm.kind, 0, prm.lg_inter);
    if constexpr (TMS) {
        if (tid == 0) s_a0 = a0r;
        __syncthreads();
    }
    const LineAddr &a0 = TMS ? s_a0 : a0r;
    {
        const Wt *tv = reinterpret_cast<const Wt *>(prm.twv);
        const Wt *tm = reinterpret_cast<const Wt *>(prm.twm);
        for (int i = tid; i < VEC + M; i += NT) stv[i] = i < VEC ? ldtw(tv, i) : ldtw(tm, i - VEC);
        if constexpr (SG::template twtab<T>() && (INV || !SG::template colq<T>())) {
            const double2 *td = reinterpret_cast<const double2 *>(prm.twd);
            for (int i = tid; i < SG::NTA + SG::NTB; i += NT)
                sta[i] = tw_from_d<T>(ldd2(td + (i < SG::NTA ? (i << SG::TLO) : i - SG::NTA)));
        }
    }
    // per-line bases of the tile starting at line l0 (the caller synchronises)
    auto set_tile = [&](int64_t l0) {
        if (tid < TL) {
            const LineAddr a = line_addr(g, prm.kind, l0 + tid, prm.lg_inter);
            s_abase[tid] = a.a_base;
            s_fbase[tid] = a.f_base;
        }
    };
    auto set_next = [&](int64_t l0) {   // TMS
        if (tid < TL) {
            const LineAddr a = line_addr(g, prm.kind, l0 + tid, prm.lg_inter);
            s_abase_n[tid] = a.a_base;
            s_fbase_n[tid] = a.f_base;
        }
    };
    const int logL = g.logL, logVP = g.logVP;
    const int64_t L = g.L, VP = g.vp;
    const bool scl = prm.apply_scale != 0;
    const T sre = (T)prm.scale_re, sim = (T)prm.scale_im;
    constexpr int VE = 16 / (int)sizeof(C);      // elements per 16-byte vector
    constexpr int VPT = E / VE / NT;             // vectors per thread
    static_assert(VPT * VE * NT == E, "vector copy");

    // frequency side: pointer to (t, k2 global, k1 = k1_0) and the step between k1 and k1 + kstep
    auto fptr_b = [&](auto *base, const int64_t *fb, int t, int k2, int k1_0) {
        const int64_t c = k2 >> logVP, f = k2 & (VP - 1);
        const int64_t pos = (int64_t)k1_0 * VP + f;
        return base + fb[t] + c * a0.f_chunk + (pos >> a0.f_lg) * a0.f_hi + (pos & ((1 << a0.f_lg) - 1));
    };
    auto fptr = [&](auto *base, int t, int k2, int k1_0) { return fptr_b(base, s_fbase, t, k2, k1_0); };
    // (VP is a multiple of the interleave 2^flg whenever flg > 0)
    // k1 += RC2 (column stage 1) / RC1 (column stage 2), recomputed where used
    auto fstep1 = [&]() -> int64_t { return (((int64_t)RC2 * VP) >> a0.f_lg) * a0.f_hi; };
    auto fstep2 = [&]() -> int64_t { return (((int64_t)RC1 * VP) >> a0.f_lg) * a0.f_hi; };
    // vector-side element e of this CTA's rows (row-major over [t][n1l][p]) -> global
    // (16-byte vector copies; used only where the vector side is contiguous, a_pos = 1)
    auto aaddr = [&](int e) {
        const int t = e / (ML * VEC), r = (e % (ML * VEC)) + n1_0 * VEC;   // concatenated position
        const int64_t c = r >> logL, pos = r & (L - 1);
        return s_abase[t] + c * a0.a_chunk + pos;
    };
    // vector side: global offset of the first element of local row n1l of line t;
    // consecutive positions of a row are a_pos apart
    const int64_t apos = a0.a_pos;
    auto arow_b = [&](const int64_t *ab, int t, int n1l) {
        const int r = (n1_0 + n1l) * VEC;
        return ab[t] + (int64_t)(r >> logL) * a0.a_chunk + (int64_t)(r & (L - 1)) * apos;
    };
    auto arow = [&](int t, int n1l) { return arow_b(s_abase, t, n1l); };
    // Lane orders.  Rows: (j, n1, t) -- or t first when the vector side interleaves
    // lines (apos > 1) so that the lines' elements pair up in memory.  Columns:
    // (k2, j, t) -- or (low interleave bits of k2, t, rest of k2, j) when the frequency
    // side is strided (x-type passes) so that lines and interleaved positions pair up.
    const bool tfirst_rows = TL > 1 && apos > 1;
    const bool tfirst_cols = TL > 1 && a0.f_hi != 1;
    auto rowunit = [&](int u, int nj, int &t, int &n1l, int &j) {
        if (tfirst_rows) {
            t = u % TL;
            const int rr = u / TL;
            j = rr % nj;
            n1l = (rr / nj) % ML;
        } else {
            j = u % nj;
            const int rr = u / nj;
            n1l = rr % ML;
            t = rr / ML;
        }
    };
    auto colunit = [&](int u, int nj, int &t, int &k2l, int &j) {
        if (tfirst_cols) {
            const int flg = a0.f_lg;
            const int gm = (1 << flg) - 1;
            const int lo = u & gm;
            const int rr = u >> flg;
            t = rr % TL;
            const int r2 = rr / TL;
            k2l = ((r2 % (VL >> flg)) << flg) | lo;
            j = r2 / (VL >> flg);
        } else {
            k2l = u % VL;
            const int rr = u / VL;
            j = rr % nj;
            t = rr / nj;
        }
    };
    // inter-step twiddles w_N^{(j + s r) k2}, r = 0, 1, ... applied to a point:
    //   complex128: FP64 power walk from the table w_N^m (m < 16 VEC);
    //   complex64, one CTA per tile: exponent m = (j + s r) k2 mod N stepped in integers
    //               and the point multiplied by the two shared-memory factors of w_N^m,
    //               each a compensated hi/lo product (no FP64 work or conversions);
    //   complex64 with a cluster: the FP64 walk, each twiddle split into hi/lo
    const double2 *Td = reinterpret_cast<const double2 *>(prm.twd);
    struct Walk {
        double2 w, step;   // complex128
        int m, dm;         // complex64
        const Wt *ta, *tb;
        ZM_DEV C apply(C x, bool conj) {   // conj: multiply by conj(w) (a constant at every call)
            if constexpr (SG::template twtab<T>()) {
                const Wt a = ta[m >> SG::TLO], b = tb[m & (SG::NTB - 1)];
                x = conj ? twmul<true>(twmul<true>(x, a), b) : twmul<false>(twmul<false>(x, a), b);
                m = (m + dm) & (SG::N - 1);
                return x;
            } else {
                const Wt t = tw_from_d<T>(w);
                const C r = conj ? twmul<true>(x, t) : twmul<false>(x, t);
                w = cmul_d(w, step);
                return r;
            }
        }
    };
    auto walk = [&](int j, int s, int k2) {
        Walk wk;
        if constexpr (SG::template twtab<T>()) {
            wk.m = (j * k2) & (SG::N - 1);
            wk.dm = (s * k2) & (SG::N - 1);
            wk.ta = sta;
            wk.tb = stb;
        } else {
            wk.w = ldd2(Td + j * k2);
            wk.step = ldd2(Td + s * k2);
        }
        return wk;
    };
    auto xidx_of_e = [](int e) {
        const int t = e / (ML * VEC), r = e % (ML * VEC);
        return SG::X(t, r >> LV, r & (VEC - 1));
    };
    // shared memory of the CTA that owns column k2 / row n1
    auto yowner = [&](int k2) -> C * {
        if constexpr (CL > 1) return cooperative_groups::this_cluster().map_shared_rank(S, k2 / VL);
        else return S;
    };
    auto xowner = [&](int n1) -> C * {
        if constexpr (CL > 1) return cooperative_groups::this_cluster().map_shared_rank(S, n1 / ML);
        else return S;
    };
    auto scale_c = [&](C o) -> C {
        return scl ? C{o.x * sre - o.y * sim, o.x * sim + o.y * sre} : o;
    };

    // ---- forward, second row stage (two row stages): local rows X -> twiddle w_VEC,
    //      RA2-point transforms, results scattered to the column owners
    auto fwd_row_stage2_scatter = [&]() {
        constexpr int NU2 = EPT / RA2;
        C w[NU2][RA2];
        int wt[NU2], wn1[NU2], wj[NU2];
#pragma unroll
        for (int i = 0; i < NU2; i++) {
            const int u = tid + i * NT;
            wj[i] = u & (RA1 - 1);
            const int rr = u / RA1;
            wn1[i] = rr % ML;
            wt[i] = rr / ML;
#pragma unroll
            for (int r = 0; r < RA2; r++) w[i][r] = S[SG::X(wt[i], wn1[i], wj[i] + RA1 * r)];
        }
#pragma unroll
        for (int i = 0; i < NU2; i++) {
#pragma unroll
            for (int r = 1; r < RA2; r++) w[i][r] = twmul<false>(w[i][r], stv[wj[i] * r]);
            dft<RA2, DIR, T>(w[i]);
        }
        tile_sync<CL>();   // every CTA has finished reading its rows
#pragma unroll
        for (int i = 0; i < NU2; i++)
#pragma unroll
            for (int r = 0; r < RA2; r++) {
                const int k2 = wj[i] + RA1 * r;
                yowner(k2)[SG::Y(wt[i], k2 % VL, n1_0 + wn1[i])] = w[i][r];
            }
    };

    // ---- forward: w_N^{n1 k2}, M-point column transforms over n1, frequency-side store
    // hook(2) runs between the two column stages (TMS prefetch; a no-op otherwise)
    auto fwd_columns = [&](auto &&hook) {
      if constexpr (SG::template colq<T>()) {
        // complex64, one CTA per tile, RC2 = 16: the first stage runs with lanes along
        // j = n1 mod RC2 (k2 = zk with CL = 1); unit (t, k2, j) transforms n1 = j + RC2 r,
        // twiddled by w_N^{j k2} (one lookup per unit) times w_N^{RC2 r k2} (a lookup
        // shared by the lanes of one k2); its outputs s go to column position s RC2 + j,
        // so the second stage reads each unit's RC2 points as one run
        const Wt *twn = reinterpret_cast<const Wt *>(prm.twN);   // hi/lo pairs of w_N^m
        constexpr int NU = EPT / RC1;
        C z[NU][RC1];
        int zt[NU], zk[NU], zj[NU];
#pragma unroll
        for (int i = 0; i < NU; i++) {
            const int u = tid + i * NT;
            zj[i] = u % RC2;
            const int rr = u / RC2;
            zk[i] = rr % VL;
            zt[i] = rr / VL;
            const Wt b = ldtw(twn, zj[i] * zk[i]);
#pragma unroll
            for (int r = 0; r < RC1; r++) {
                const C x = twmul<false>(S[SG::Y(zt[i], zk[i], zj[i] + RC2 * r)], b);
                z[i][r] = r == 0 ? x : twmul<false>(x, ldtw(twn, RC2 * r * zk[i]));
            }
        }
#pragma unroll
        for (int i = 0; i < NU; i++) dft<RC1, DIR, T>(z[i]);
        __syncthreads();
#pragma unroll
        for (int i = 0; i < NU; i++)
#pragma unroll
            for (int r = 0; r < RC1; r++) S[SG::Y(zt[i], zk[i], r * RC2 + zj[i])] = z[i][r];
        __syncthreads();
        hook(2);
        constexpr int NU2 = EPT / RC2;
#pragma unroll
        for (int i = 0; i < NU2; i++) {
            const int u = tid + i * NT;
            int t, k2l, j2;
            colunit(u, RC1, t, k2l, j2);
            C y[RC2];
#pragma unroll
            for (int r = 0; r < RC2; r++) y[r] = S[SG::Y(t, k2l, j2 * RC2 + r)];
#pragma unroll
            for (int r = 1; r < RC2; r++) y[r] = twmul<false>(y[r], stm[j2 * r]);
            dft<RC2, DIR, T>(y);
            C *op = fptr(out, t, k2l, j2);
#pragma unroll
            for (int r = 0; r < RC2; r++) op[fstep2() * r] = scale_c(y[r]);
        }
      } else {
        constexpr int NU = EPT / RC1;
        C z[NU][RC1];
        int zt[NU], zk[NU], zj[NU];
#pragma unroll
        for (int i = 0; i < NU; i++) {
            const int u = tid + i * NT;
            if constexpr (RC2 == 1) {
                colunit(u, RC2, zt[i], zk[i], zj[i]);   // this stage stores to global
            } else {
                zk[i] = u % VL;
                const int rr = u / VL;
                zj[i] = rr % RC2;
                zt[i] = rr / RC2;
            }
            Walk wk = walk(zj[i], RC2, k2_0 + zk[i]);               // n1 = zj + RC2 * r
#pragma unroll
            for (int r = 0; r < RC1; r++)
                z[i][r] = wk.apply(S[SG::Y(zt[i], zk[i], zj[i] + RC2 * r)], false);
        }
#pragma unroll
        for (int i = 0; i < NU; i++) dft<RC1, DIR, T>(z[i]);
        if constexpr (RC2 == 1) {
#pragma unroll
            for (int i = 0; i < NU; i++) {
                C *op = fptr(out, zt[i], k2_0 + zk[i], 0);
#pragma unroll
                for (int r = 0; r < RC1; r++) op[fstep1() * r] = scale_c(z[i][r]);
            }
        } else {
            __syncthreads();
#pragma unroll
            for (int i = 0; i < NU; i++)
#pragma unroll
                for (int r = 0; r < RC1; r++) S[SG::Y(zt[i], zk[i], zj[i] * RC1 + r)] = z[i][r];
            __syncthreads();
            hook(2);
            constexpr int NU2 = EPT / RC2;
#pragma unroll
            for (int i = 0; i < NU2; i++) {
                const int u = tid + i * NT;
                int t, k2l, j2;
                colunit(u, RC1, t, k2l, j2);
                C y[RC2];
#pragma unroll
                for (int r = 0; r < RC2; r++) y[r] = S[SG::Y(t, k2l, j2 + RC1 * r)];
#pragma unroll
                for (int r = 1; r < RC2; r++) y[r] = twmul<false>(y[r], stm[j2 * r]);
                dft<RC2, DIR, T>(y);
                C *op = fptr(out, t, k2_0 + k2l, j2);
#pragma unroll
                for (int r = 0; r < RC2; r++) op[fstep2() * r] = scale_c(y[r]);
            }
        }
      }
    };

    if constexpr (fused_persistent<T, LV, LM, CL, TL, NT, INV, PERS>()) {
        // ================= forward, two row stages: persistent, staged bulk copies
        C *stage = reinterpret_cast<C *>(smem_raw + fused_stage_offset<T, LV, LM, CL, TL, NT>());
        const int sg = (int)apos;                       // 1, or the y pass's row interleave
        const int lgs = sg >= 4 ? 2 : (sg == 2 ? 1 : 0);
        const int SR = sg >= 4 ? SG::SR(4) : (sg == 2 ? SG::SR(2) : SG::SR(1));
        const int ncopy = (TL >> lgs) * ML;            // staging rows per tile
        const unsigned cbytes = (unsigned)(sg * VEC * (int)sizeof(C));
        const int64_t ntiles = prm.nlines / TL;
        const int64_t ncl = gridDim.x / CL;
        if (tid == 0) {
            mbar_init(&s_bar, 1);
            mbar_fence_init();
        }
        __syncthreads();
        // staging row u = (line group tg, local row n1l) of tile `tile`: sg * VEC
        // consecutive global elements (the rows of sg interleaved lines)
        auto issue = [&](int64_t tile) {
            if (tid == 0) mbar_expect_tx(&s_bar, (unsigned)ncopy * cbytes);
            __syncthreads();
            for (int u = tid; u < ncopy; u += NT) {
                const int tg = u / ML, n1l = u - tg * ML;
                const LineAddr a = line_addr(g, prm.kind, tile * TL + (tg << lgs), prm.lg_inter);
                const int r = (n1_0 + n1l) * VEC;
                const C *src = in + a.a_base + (int64_t)(r >> logL) * a.a_chunk + (int64_t)(r & (L - 1)) * a.a_pos;
                fence_proxy_async();
                bulk_g2s(stage + u * SR, src, cbytes, &s_bar);
            }
        };
        unsigned parity = 0;
        // Set (block-uniformly) when a tile's copies did not land within two bounded
        // waits: the CTA then issues no further copies, so at most that one round can be
        // in flight when it exits, and it skips the waits of later tiles.  It still runs
        // its remaining tiles (on stale data, with the device error word raised) so that
        // the cluster's barriers stay matched.
        bool copies_lost = false;
        int64_t tile = blockIdx.x / CL;
        if (tile < ntiles) issue(tile);
        for (; tile < ntiles; tile += ncl) {
            __syncthreads();   // the previous tile is done with S and the bases
            set_tile(tile * TL);
            if (!copies_lost) {
                bool landed = mbar_wait(&s_bar, parity, kCopyWaitNs);
                if (!landed) {
                    if (prm.err) atomicExch(prm.err, 1);
                    landed = mbar_wait(&s_bar, parity, kCopyWaitNs);   // let copies in flight land, bounded
                }
                copies_lost = __syncthreads_or(!landed) != 0;
                parity ^= 1u;
            }
            // first row stage: staging -> RA1-point transforms -> rows X
            {
                constexpr int NU = EPT / RA1;
                C v[NU][RA1];
                int ut[NU], un1[NU], uj[NU];
#pragma unroll
                for (int i = 0; i < NU; i++) {
                    rowunit(tid + i * NT, RA2, ut[i], un1[i], uj[i]);
                    const C *row = stage + ((ut[i] >> lgs) * ML + un1[i]) * SR + (uj[i] << lgs) + (ut[i] & (sg - 1));
#pragma unroll
                    for (int r = 0; r < RA1; r++) v[i][r] = row[(RA2 * r) << lgs];
                }
#pragma unroll
                for (int i = 0; i < NU; i++) {
                    dft<RA1, DIR, T>(v[i]);
#pragma unroll
                    for (int r = 0; r < RA1; r++) S[SG::X(ut[i], un1[i], uj[i] * RA1 + r)] = v[i][r];
                }
            }
            __syncthreads();   // staging consumed, rows complete, bases visible
            if (!copies_lost && tile + ncl < ntiles) issue(tile + ncl);
            fwd_row_stage2_scatter();
            tile_sync<CL>();
            fwd_columns([](int) {});
        }
        return;
    } else if constexpr (!TMS) {
        set_tile((int64_t)(blockIdx.x / CL) * TL);
        // forward: L2 prefetch of the vector side of the tile one wave of clusters ahead,
        // so its HBM reads overlap this tile's work (for an interleaved intermediate the
        // first line of each group fetches the group's runs).  Measured on the inverse
        // passes' frequency side it did not pay, so they take none.
        const int64_t ft = (int64_t)(blockIdx.x / CL) + prm.pf_tiles;
        if (!INV && prm.pf_tiles > 0 && rank == 0 && ft < prm.nlines / TL) {
            const int nch = (int)(SG::N >> logL);                  // rank chunks per line
            if (tid < TL * nch) {
                const int t = tid / nch, c = tid - t * nch;
                const int64_t l = ft * TL + t;
                if (a0.a_pos == 1 || (l & (a0.a_pos - 1)) == 0) {
                    const LineAddr a = line_addr(g, prm.kind, l, prm.lg_inter);
                    const unsigned char *src = reinterpret_cast<const unsigned char *>(in + a.a_base + c * a.a_chunk);
                    const int64_t bytes = L * a0.a_pos * (int64_t)sizeof(C);
                    if (((uintptr_t)src & 15) == 0 && (bytes & 15) == 0)
                        for (int64_t o = 0; o < bytes; o += 32768)
                            bulk_prefetch_l2(src + o, (unsigned)(bytes - o < 32768 ? bytes - o : 32768));
                }
            }
        }
        __syncthreads();
    }

    // ---- TMS (tensor-memory staging): the grid is persistent and each CTA walks tiles
    //      c, c + clusters, ...  The EPT points a thread loads from global memory first in a
    //      tile (vector-side rows forward, frequency-side columns inverse) are, for its NEXT
    //      tile, fetched during the current one in NCH chunks of 16 words: asynchronous
    //      copies (cp.async, no registers held) into a two-slot shared-memory ring behind
    //      the slice, chunks 0 and 1 at phase boundary 0 of the tile and chunk k >= 2 at
    //      boundary k - 1; a chunk is moved on into this thread's columns of tensor memory
    //      one boundary after its copy was issued (k + 1), freeing its slot; the last one
    //      is read from its slot when the next tile starts, the others from tensor memory.
    //      So the tile's HBM reads overlap the previous tile's work.  One CTA per SM (the
    //      slice fills shared memory), so the NCOLS columns are free at once.
    constexpr int WPP = (int)sizeof(C) / 4;                // 32-bit words per point
    constexpr int PC = 16 / WPP;                           // points per chunk
    constexpr int NCH = EPT / PC;                          // chunks per thread
    constexpr int NCOLS = EPT * WPP * (NT / 128);          // columns of the CTA
    if constexpr (TMS) {
        static_assert(!PERS && (INV || RA2 > 1) && RC2 > 1 && (!INV || RA2 > 1), "TMS tile shape");
        static_assert(NCH >= 2 && NCH <= 4, "TMS chunk schedule: at most one move per phase boundary");
        static_assert(NT % 128 == 0 && NCOLS >= 32 && NCOLS <= 512 && (NCOLS & (NCOLS - 1)) == 0, "TMEM columns");
        static_assert(2 * (fused_smem_bytes<T, LV, LM, CL, TL, NT, INV, PERS>() + 1024) > 228 * 1024,
                      "TMS needs one CTA per SM");
    }
    const int warp = tid >> 5;
    // ring slot s, point q of this thread (thread-fastest: conflict-free 8 / 16-byte accesses)
    C *ring = reinterpret_cast<C *>(smem_raw + fused_smem_bytes<T, LV, LM, CL, TL, NT, INV, PERS>());
    auto ring_at = [&](int slot, int q) { return ring + ((size_t)slot * PC + q) * NT + tid; };
    bool has_next = false;                                 // block-uniform
    auto chunk_src = [&](int c, int q) -> const C * {      // point q of chunk c, next tile
        const int f = c * PC + q;
        if constexpr (!INV) {
            int t, n1l, j;
            rowunit(tid + (f / RA1) * NT, RA2, t, n1l, j);
            return in + arow_b(s_abase_n, t, n1l) + j * apos + RA2 * (f % RA1) * apos;
        } else {
            int t, k2l, j;
            colunit(tid + (f / RC1) * NT, RC2, t, k2l, j);
            return fptr_b(in, s_fbase_n, t, k2_0 + k2l, j) + fstep1() * (f % RC1);
        }
    };
    auto tm_addr = [&](int c) -> uint32_t {
        return s_tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)((warp >> 2) * EPT * WPP + c * 16);
    };
    auto issue_chunk = [&](int c) {                        // copies into slot c & 1, one group
#pragma unroll
        for (int q = 0; q < PC; q++) {
            if constexpr (sizeof(C) == 16) cp_async16(ring_at(c & 1, q), chunk_src(c, q));
            else cp_async8(ring_at(c & 1, q), chunk_src(c, q));
        }
        cp_async_commit();
    };
    auto move_chunk = [&](int c) {                         // slot c & 1 -> tensor memory
        cp_async_wait_one();                               // all groups but the newest landed
        uint32_t w[16];
#pragma unroll
        for (int q = 0; q < PC; q++) memcpy(w + q * WPP, ring_at(c & 1, q), sizeof(C));
        tmem_st16(tm_addr(c), w);
    };
    auto hook = [&](int k) {
        if constexpr (TMS) {
            if (!has_next) return;
            if (k == 0) {
                issue_chunk(0);
                issue_chunk(1);
            } else if (k - 1 <= NCH - 2) {
                move_chunk(k - 1);
                if (k + 1 < NCH) issue_chunk(k + 1);
            }
        }
    };
    auto tms_read = [&](C *dst) {   // this tile's EPT first-phase points, flat order
#pragma unroll
        for (int c = 0; c < NCH - 1; c++) {
            uint32_t w[16];
            tmem_ld16(tm_addr(c), w);
            memcpy(dst + c * PC, w, 64);
        }
        cp_async_wait_all();
#pragma unroll
        for (int q = 0; q < PC; q++) dst[(NCH - 1) * PC + q] = *ring_at((NCH - 1) & 1, q);
    };
    if constexpr (TMS) {
        if (warp == 0) tmem_alloc(&s_tmem, NCOLS);
        tmem_fence_before();
        __syncthreads();
        tmem_fence_after();
    }
    const int64_t tms_ntiles = prm.nlines / TL, tms_ncl = gridDim.x / CL;
    int64_t tms_tile = blockIdx.x / CL;
    bool tms_first = true;
    for (;;) {
    if constexpr (TMS) {
        if (tms_tile >= tms_ntiles) break;
        // an opaque copy of tid: the per-thread index and address arithmetic of the tile is
        // then recomputed in every tile instead of being hoisted out of the loop and held
        // in registers across it (which spilled 380-460 bytes at 128 registers)
        asm volatile("mov.u32 %0, %0;" : "+r"(tid));
        __syncthreads();   // the previous tile is done with S and the bases
        set_tile(tms_tile * TL);
        has_next = tms_tile + tms_ncl < tms_ntiles;
        if (has_next) set_next((tms_tile + tms_ncl) * TL);
        __syncthreads();
    }
    if constexpr (!INV && RA2 > 1) {
        // ================= forward, two row stages, one tile per cluster: the first row
        // stage reads the vector side straight from global memory (TMS: from tensor
        // memory after the CTA's first tile)
        {
            constexpr int NU = EPT / RA1;
            C v[NU][RA1];
            int ut[NU], un1[NU], uj[NU];
#pragma unroll
            for (int i = 0; i < NU; i++) rowunit(tid + i * NT, RA2, ut[i], un1[i], uj[i]);
            if (TMS && !tms_first) {
                tms_read(&v[0][0]);
            } else {
#pragma unroll
                for (int i = 0; i < NU; i++) {
                    const C *row = in + arow(ut[i], un1[i]) + uj[i] * apos;
#pragma unroll
                    for (int r = 0; r < RA1; r++) v[i][r] = ldg(row + RA2 * r * apos);
                }
            }
#pragma unroll
            for (int i = 0; i < NU; i++) {
                dft<RA1, DIR, T>(v[i]);
#pragma unroll
                for (int r = 0; r < RA1; r++) S[SG::X(ut[i], un1[i], uj[i] * RA1 + r)] = v[i][r];
            }
        }
        __syncthreads();
        hook(0);
        fwd_row_stage2_scatter();
        tile_sync<CL>();
        hook(1);
        fwd_columns(hook);
        hook(3);
    } else if constexpr (!INV) {
        // ================= forward, one row stage (RA2 == 1): one tile per cluster.  With a
        // contiguous vector side each thread reads its rows straight from global memory (two
        // or more 16-byte loads per row, lanes on consecutive rows: a warp covers one run);
        // otherwise the side moves through the rows X as 16-byte vectors first.
        const bool rows_direct = (RA1 * sizeof(C)) % 16 == 0 && apos == 1;   // block-uniform
        if (!rows_direct) {
            // ---- 1. vector side -> local rows X (16-byte vectors, all loads before stores)
            uint4 buf[VPT];
#pragma unroll
            for (int i = 0; i < VPT; i++) buf[i] = ldg16(in + aaddr((tid + i * NT) * VE));
#pragma unroll
            for (int i = 0; i < VPT; i++)
                *reinterpret_cast<uint4 *>(&S[xidx_of_e((tid + i * NT) * VE)]) = buf[i];
            __syncthreads();
        }
        // ---- 2. VEC-point row transforms over n2, results scattered to the column owners
        {
            constexpr int NU = EPT / RA1;
            C v[NU][RA1];
            int ut[NU], un1[NU];
#pragma unroll
            for (int i = 0; i < NU; i++) {
                const int u = tid + i * NT;
                un1[i] = u % ML;
                ut[i] = u / ML;
            }
            if (rows_direct) {
                if constexpr ((RA1 * sizeof(C)) % 16 == 0) {
                    uint4 buf[NU][RA1 * sizeof(C) / 16];
#pragma unroll
                    for (int i = 0; i < NU; i++) {
                        const uint4 *rp = reinterpret_cast<const uint4 *>(in + arow(ut[i], un1[i]));
#pragma unroll
                        for (int q = 0; q < RA1 * (int)sizeof(C) / 16; q++) buf[i][q] = __ldg(rp + q);
                    }
#pragma unroll
                    for (int i = 0; i < NU; i++) memcpy(&v[i][0], &buf[i][0], RA1 * sizeof(C));
                }
            } else {
#pragma unroll
                for (int i = 0; i < NU; i++) {
                    if constexpr ((RA1 * sizeof(C)) % 16 == 0 && (SG::XR * sizeof(C)) % 16 == 0) {
                        // the row as 16-byte vectors: lanes on consecutive rows of XR = VEC + 2
                        // points take distinct bank groups (8-byte reads of the same rows collide)
                        const uint4 *rp = reinterpret_cast<const uint4 *>(&S[SG::X(ut[i], un1[i], 0)]);
#pragma unroll
                        for (int q = 0; q < RA1 * (int)sizeof(C) / 16; q++)
                            *reinterpret_cast<uint4 *>(&v[i][q * 16 / (int)sizeof(C)]) = rp[q];
                    } else {
#pragma unroll
                        for (int r = 0; r < RA1; r++) v[i][r] = S[SG::X(ut[i], un1[i], r)];
                    }
                }
            }
#pragma unroll
            for (int i = 0; i < NU; i++) dft<RA1, DIR, T>(v[i]);
            // every CTA has finished reading its rows (the scatter overwrites them); with the
            // rows read from global memory only a cluster needs it (its CTAs must have started)
            if (!rows_direct || CL > 1) tile_sync<CL>();
#pragma unroll
            for (int i = 0; i < NU; i++)
#pragma unroll
                for (int r = 0; r < RA1; r++) yowner(r)[SG::Y(ut[i], r % VL, n1_0 + un1[i])] = v[i][r];
        }
        tile_sync<CL>();
        // ---- 3. columns
        fwd_columns([](int) {});
    } else {
        // ================= inverse: one tile per cluster
        // rows X in the odd-stride form (SliceGeom::XI) where nothing reads them as 16-byte
        // vectors of several elements: complex128, or complex64 rows stored straight to a
        // contiguous vector side (block-uniform)
        const bool xri = RA2 == 1 && (sizeof(C) == 16 || ((RA1 * sizeof(C)) % 16 == 0 && apos == 1));
        auto Xs = [&](int t, int n1l, int p) { return xri ? SG::XI(t, n1l, p) : SG::X(t, n1l, p); };
        // ---- 1. frequency side -> M-point inverse column transforms over k1 (local columns)
        {
            constexpr int NU = EPT / RC1;
            C z[NU][RC1];
            int zt[NU], zk[NU], zj[NU];
#pragma unroll
            for (int i = 0; i < NU; i++) colunit(tid + i * NT, RC2, zt[i], zk[i], zj[i]);
            if (TMS && !tms_first) {
                tms_read(&z[0][0]);
            } else {
#pragma unroll
                for (int i = 0; i < NU; i++) {
                    const C *ip = fptr(in, zt[i], k2_0 + zk[i], zj[i]);
#pragma unroll
                    for (int r = 0; r < RC1; r++) z[i][r] = ldg(ip + fstep1() * r);
                }
            }
#pragma unroll
            for (int i = 0; i < NU; i++) dft<RC1, DIR, T>(z[i]);
            if constexpr (RC2 == 1) {
                // n1 = r: conj(w_N^{n1 k2}), then to the row owners X[t][n1l][k2]
                tile_sync<CL>();
#pragma unroll
                for (int i = 0; i < NU; i++) {
                    const int k2 = k2_0 + zk[i];
                    Walk wk = walk(0, 1, k2);                            // n1 = r
#pragma unroll
                    for (int r = 0; r < RC1; r++)
                        xowner(r)[Xs(zt[i], r % ML, k2)] = wk.apply(z[i][r], true);
                }
            } else {
#pragma unroll
                for (int i = 0; i < NU; i++)
#pragma unroll
                    for (int r = 0; r < RC1; r++) S[SG::Y(zt[i], zk[i], zj[i] * RC1 + r)] = z[i][r];
                __syncthreads();
                hook(0);
                constexpr int NU2 = EPT / RC2;
                C y[NU2][RC2];
                int yt[NU2], yk[NU2], yj[NU2];
#pragma unroll
                for (int i = 0; i < NU2; i++) {
                    const int u = tid + i * NT;
                    if (xri) {   // lanes along the rows yj of one column (the scatter below)
                        yj[i] = u % RC1;
                        const int rr = u / RC1;
                        yk[i] = rr % VL;
                        yt[i] = rr / VL;
                    } else {
                        yk[i] = u % VL;
                        const int rr = u / VL;
                        yj[i] = rr % RC1;
                        yt[i] = rr / RC1;
                    }
#pragma unroll
                    for (int r = 0; r < RC2; r++) y[i][r] = S[SG::Y(yt[i], yk[i], yj[i] + RC1 * r)];
                }
#pragma unroll
                for (int i = 0; i < NU2; i++) {
#pragma unroll
                    for (int r = 1; r < RC2; r++) y[i][r] = twmul<true>(y[i][r], stm[yj[i] * r]);
                    dft<RC2, DIR, T>(y[i]);
                }
                tile_sync<CL>();   // every CTA has finished reading its columns
#pragma unroll
                for (int i = 0; i < NU2; i++) {
                    const int k2 = k2_0 + yk[i];
                    Walk wk = walk(yj[i], RC1, k2);                      // n1 = yj + RC1 * r
#pragma unroll
                    for (int r = 0; r < RC2; r++) {
                        const int n1 = yj[i] + RC1 * r;
                        xowner(n1)[Xs(yt[i], n1 % ML, k2)] = wk.apply(y[i][r], true);
                    }
                }
            }
        }
        tile_sync<CL>();
        hook(1);
        // ---- 2. VEC-point inverse row transforms over k2 -> local rows X[t][n1l][n2]
        //      (one row stage, RA2 == 1: each row is one thread's alone, read as 16-byte
        //      vectors where the row stride allows, and with a contiguous vector side stored
        //      straight from registers -- no barrier, no shared-memory write-back)
        constexpr bool ROWVEC = RA2 == 1 && (RA1 * sizeof(C)) % 16 == 0 && (SG::XR * sizeof(C)) % 16 == 0;
        // (complex64 only: complex128 rows of 64 bytes stored by one lane each were slower
        // than the coalesced 16-byte sweep of section 3, 3D N = 512 inverse 4.09 -> 4.17 ms)
        const bool rows_direct = RA2 == 1 && sizeof(C) == 8 && (RA1 * sizeof(C)) % 16 == 0 && apos == 1;
        {
            constexpr int NU = EPT / RA1;
            C v[NU][RA1];
            int ut[NU], un1[NU], uj[NU];
#pragma unroll
            for (int i = 0; i < NU; i++) {
                const int u = tid + i * NT;
                uj[i] = u & (RA2 - 1);
                const int rr = u / RA2;
                un1[i] = rr % ML;
                ut[i] = rr / ML;
                if (ROWVEC && !(xri && sizeof(C) < 16)) {
                    const uint4 *rp = reinterpret_cast<const uint4 *>(&S[Xs(ut[i], un1[i], 0)]);
#pragma unroll
                    for (int q = 0; q < RA1 * (int)sizeof(C) / 16; q++)
                        *reinterpret_cast<uint4 *>(&v[i][q * 16 / (int)sizeof(C)]) = rp[q];
                } else {
#pragma unroll
                    for (int r = 0; r < RA1; r++) v[i][r] = S[Xs(ut[i], un1[i], uj[i] + RA2 * r)];
                }
            }
            if constexpr (RA2 > 1) __syncthreads();
#pragma unroll
            for (int i = 0; i < NU; i++) dft<RA1, DIR, T>(v[i]);
            if (rows_direct) {
                // row (t, n1) of the vector side: VEC consecutive positions, 16-byte aligned
#pragma unroll
                for (int i = 0; i < NU; i++) {
                    C *row = out + arow(ut[i], un1[i]);
#pragma unroll
                    for (int r = 0; r < RA1; r++) {
                        const C o = v[i][r];
                        v[i][r] = scl ? C{sre * o.x - sim * o.y, sre * o.y + sim * o.x} : o;
                    }
#pragma unroll
                    for (int q = 0; q < RA1 * (int)sizeof(C) / 16; q++)
                        reinterpret_cast<uint4 *>(row)[q] = *reinterpret_cast<const uint4 *>(&v[i][q * 16 / (int)sizeof(C)]);
                }
            } else {
#pragma unroll
                for (int i = 0; i < NU; i++)
#pragma unroll
                    for (int r = 0; r < RA1; r++) S[Xs(ut[i], un1[i], uj[i] * RA1 + r)] = v[i][r];
            }
            if constexpr (RA2 > 1) {
                __syncthreads();
                hook(2);
                constexpr int NU2 = EPT / RA2;
                C w[NU2][RA2];
                int wt[NU2], wn1[NU2], wj[NU2];
#pragma unroll
                for (int i = 0; i < NU2; i++) {
                    const int u = tid + i * NT;
                    rowunit(u, RA1, wt[i], wn1[i], wj[i]);   // this stage stores to global
#pragma unroll
                    for (int r = 0; r < RA2; r++) w[i][r] = S[SG::X(wt[i], wn1[i], wj[i] + RA1 * r)];
                }
#pragma unroll
                for (int i = 0; i < NU2; i++) {
#pragma unroll
                    for (int r = 1; r < RA2; r++) w[i][r] = twmul<true>(w[i][r], stv[wj[i] * r]);
                    dft<RA2, DIR, T>(w[i]);
                    // last stage: n2 = wj + RA1 r straight to the vector side (lanes along n2)
                    C *row = out + arow(wt[i], wn1[i]) + wj[i] * apos;
#pragma unroll
                    for (int r = 0; r < RA2; r++) row[RA1 * r * apos] = scale_c(w[i][r]);
                }
            }
        }
        // ---- 3. single row stage, strided vector side: local rows -> vector side (16-byte
        //      vectors), scale applied here
        if constexpr (RA2 == 1) {
          if (!rows_direct) {
            __syncthreads();
#pragma unroll
            for (int i = 0; i < VPT; i++) {
                const int e = (tid + i * NT) * VE;
                const int et = e / (ML * VEC), er = e % (ML * VEC);
                uint4 v = *reinterpret_cast<const uint4 *>(&S[Xs(et, er >> LV, er & (VEC - 1))]);
                if (scl) {
                    C *cv = reinterpret_cast<C *>(&v);
#pragma unroll
                    for (int q = 0; q < VE; q++) {
                        const C o = cv[q];
                        cv[q] = {sre * o.x - sim * o.y, sre * o.y + sim * o.x};
                    }
                }
                *reinterpret_cast<uint4 *>(out + aaddr(e)) = v;
            }
          }
        }
        hook(3);
    }
    if constexpr (!TMS) break;
    tms_first = false;
    tms_tile += tms_ncl;
    }   // tile loop (one pass unless TMS)
    if constexpr (TMS) {
        cp_async_wait_all();   // nothing in flight when the CTA exits
        tmem_fence_before();
        __syncthreads();   // every tensor-memory access of the CTA is complete
        if (warp == 0) {
            tmem_fence_after();
            tmem_dealloc(s_tmem, NCOLS);
        }
    }
}

// Clusters (or CTAs) resident at once for a persistent launch of `kern`, per device.
template <int CL, int NT, typename K>
static int resident_clusters(K kern, size_t smem, int dev) {
    int n = 0;
    if constexpr (CL == 1) {
        int per_sm = 0, sms = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, smem) != cudaSuccess) return 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
        n = per_sm * sms;
    } else {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(CL);
        cfg.blockDim = dim3(NT);
        cfg.dynamicSmemBytes = smem;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = CL;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        if (cudaOccupancyMaxActiveClusters(&n, kern, &cfg) != cudaSuccess) return 0;
    }
    return n;
}

template <typename T, int LV, int LM, int CL, int TL, int NT, bool INV, bool PERS = false, bool TMS = false>
cudaError_t launch_fused(const LineParams &prm, cudaStream_t st) {
    // TMS: the two-slot ring of 16-word chunks behind the slice
    constexpr size_t smem = fused_smem_bytes<T, LV, LM, CL, TL, NT, INV, PERS>() + (TMS ? (size_t)2 * 64 * NT : 0);
    static_assert(smem <= 227 * 1024, "shared memory of one CTA");
    constexpr bool bulk_persistent = fused_persistent<T, LV, LM, CL, TL, NT, INV, PERS>();
    constexpr bool persistent = TMS || bulk_persistent;
    if (prm.inter_q) return cudaErrorInvalidValue;   // row-interleaved intermediates only
    // the staging rows of a persistent pass hold sg = 1, 2 or 4 interleaved lines and
    // are sized for sg <= TL: a wider interleave of the y pass's vector side is refused
    if (bulk_persistent && prm.kind == PASS_Y2 && prm.lg_inter > 0 &&
        ((1 << prm.lg_inter) > TL || prm.lg_inter > 2))
        return cudaErrorInvalidValue;
    auto kern = fused_pass_kernel<T, LV, LM, CL, TL, NT, INV, PERS, TMS>;
    static int attr_done[64], clusters[64];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!attr_done[dev]) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        clusters[dev] = resident_clusters<CL, NT>(kern, smem, dev);
        if (clusters[dev] <= 0) return cudaErrorInvalidConfiguration;
        attr_done[dev] = 1;
    }
    const int64_t ntiles = prm.nlines / TL;
    const int64_t nclus = persistent ? (ntiles < clusters[dev] ? ntiles : clusters[dev]) : ntiles;
    const unsigned grid = (unsigned)nclus * CL;
    LineParams lp = prm;
    lp.pf_tiles = persistent ? 0 : clusters[dev];   // one wave of resident clusters ahead
    if constexpr (CL == 1) {
        kern<<<grid, NT, smem, st>>>(lp);
    } else {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(grid);
        cfg.blockDim = dim3(NT);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = CL;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        cudaError_t e = cudaLaunchKernelEx(&cfg, kern, lp);
        if (e != cudaSuccess) return e;
    }
    count_launch();
    return cudaGetLastError();
}

}  // namespace zm
