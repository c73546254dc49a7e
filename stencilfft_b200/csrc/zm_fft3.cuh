// zm_fft3.cuh -- three-stage fused axis pass for complex64 lines of N = 2^14 points.
//
// The same pass as fused_pass_kernel (one whole global line per CTA, the reference's
// FFT1a / pack / All-to-All / unpack+twiddle / FFT1b / repack stages of one axis in one
// kernel, see zm_fft.cu), with the line's DFT factored as 16 x 32 x 32 instead of the
// reference's VEC x M split, so that 512 threads holding 32 points each need two
// shared-memory exchanges instead of three:
//
//   time index      n = d0 + 32 d1 + 1024 d2            (d0, d1 < 32, d2 < 16)
//   frequency index k = ka + 16 kb + 512 kc             (ka < 16, kb, kc < 32)
//   X[k] = sum_d0 w32^{d0 kc} w_N^{d0 (ka + 16 kb)}                         stage 3
//            sum_d1 w32^{d1 kb} w512^{d1 ka}                                 stage 2
//              sum_d2 w16^{d2 ka} x[d0 + 32 d1 + 1024 d2]                    stage 1
//
// Forward: stage 1 (two 16-point units per thread: v = n mod 1024 with the two
// vector-side positions n2, n2 + 1 adjacent in memory, read as one 16-byte vector where
// the vector side is contiguous), exchange 1, stage 2 (unit (d0, ka): d0 = lane, ka =
// warp; input twiddle w512^{d1 ka} is the same for a whole warp), output twiddle
// w_N^{d0 ka} (one per thread) times w1024^{d0 kb} (a table read by lanes along d0),
// exchange 2, stage 3 (unit k mod 512 = thread index; its 32 outputs kc are stored with
// lanes along k2 so that a warp writes whole sectors of the frequency side).  The
// inverse runs the transposed algorithm: the same stages in reverse order with
// conjugate twiddles, so it reads the frequency side with the forward's store pattern
// and writes the vector side with the forward's load pattern.  Every twiddle is a
// compensated product with a split hi/lo FP32 pair of an FP64-generated value.
//
// Exchange buffers (8-byte elements): S1[ka][d1][d0] (rows of 32, conflict-free for
// both sides) and S2[kb][d0][ka] with d0 rows padded to 17 (the stage-2 side writes
// lanes along d0, the stage-3 side reads lanes along ka).  One CTA per line, 512
// threads, one CTA per SM (the line and the tables fill 160 KB of shared memory).
#pragma once

#include <cooperative_groups.h>

#include "zm_common.cuh"
#include "zm_lines.cuh"

namespace zm {

struct K3Geom {
    static constexpr int N = 16384, NT = 512;
    static constexpr int R2 = 32 * 17;                 // one kb row of S2
    static constexpr int EX = 32 * R2;                 // exchange region, elements (>= 16384)
    static constexpr int NT512 = 512, NT1024 = 1024;   // twiddle table entries
    static constexpr size_t SMEM = 8 * (size_t)EX + 16 * (size_t)(NT512 + NT1024);
    static ZM_DEV int s1(int ka, int d1, int d0) { return (ka * 32 + d1) * 32 + d0; }
    static ZM_DEV int s2(int kb, int d0, int ka) { return kb * R2 + d0 * 17 + ka; }
};

ZM_DEV void prefetch_l2_bytes(const void *p, int64_t bytes) {
    const unsigned char *src = reinterpret_cast<const unsigned char *>(p);
    if (((uintptr_t)src & 15) != 0 || (bytes & 15) != 0) return;
    for (int64_t o = 0; o < bytes; o += 32768) {
        const unsigned nb = (unsigned)(bytes - o < 32768 ? bytes - o : 32768);
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(
                         (unsigned long long)__cvta_generic_to_global(src + o)),
                     "r"(nb)
                     : "memory");
    }
}

// PERS: one CTA per SM walks lines blockIdx.x, + gridDim.x, ...; while it runs stage 3
// (stage C) of a line, asynchronous copies (cp.async, completion waited per thread)
// bring the next line's input into the exchange region, in the layout its stage-1
// (stage-A) reads want: vector-side rows of VEC + 4 elements (conflict-free 16-byte
// reads of 16 rows per warp), or the frequency side as [kc][k mod 512].  Each thread
// reads back only what it copied itself.  The twiddle tables are filled once per CTA.
// VM, the vector side's address form: 0 contiguous (a_pos = 1), 1 a stride (the row
// interleave of the intermediate, a_pos = G), 2 runs of 2^a_lg positions a_hi apart (the
// y-position interleave).
// PAIR (forward, VM = 1, one line per CTA): clusters of two CTAs on the buddy lines 2i,
// 2i + 1, whose elements share every 16-byte pair of the row interleave.  Each CTA loads
// the pairs of one of its two stage-1 units for both lines, keeps its own element and
// stores its partner's into the partner's shared memory (distributed shared memory), so
// a line's strided reads need half the L2 sector requests.
template <int LV, int LM, bool INV, bool PERS, int VM, bool PAIR = false>
__global__ void __launch_bounds__(512, 1) k3_pass_kernel(const LineParams prm) {
    static_assert(LV + LM == 14, "lines of 2^14 points");
    static_assert(LM >= 5 && LM <= 9 && LV <= 9, "vector / column split of the line");
    using C = cpx<float>;
    using Wt = tw<float>;
    using KG = K3Geom;
    constexpr int DIR = INV ? 1 : -1;
    constexpr int M = 1 << LM, VEC = 1 << LV;
    constexpr int HP = 512 / M;                 // threads per vector-side row n1 (stage 1 / C)
    constexpr int DSTEP = 1024 / M;             // n2 step between consecutive d2
    static_assert(!PERS || M * (VEC + 4) <= KG::EX, "staging rows fit the exchange region");

    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *S = reinterpret_cast<C *>(smem_raw);
    Wt *t512 = reinterpret_cast<Wt *>(smem_raw + 8 * (size_t)KG::EX);   // w_N^{32 m}, m < 512
    Wt *t1024 = t512 + KG::NT512;                                        // [kb][d0]: w1024^{d0 kb}

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const Geom &g = prm.g;
    const Wt *twn = reinterpret_cast<const Wt *>(prm.twN);   // w_N^m, hi/lo pairs
    const C *in = reinterpret_cast<const C *>(prm.in);
    C *out = reinterpret_cast<C *>(prm.out);
    const int64_t nl = prm.nlines;
    const int64_t lstep = PERS ? (int64_t)gridDim.x : nl;
    const int kind = prm.kind, lgi = prm.lg_inter;

    // stage-1 / stage-C thread: vector-side row n1 and two units n2_lo = lo0, lo1 (the
    // line's positions n2 = n2_lo + DSTEP d2).  Contiguous vector side: lo1 = lo0 + 1, the
    // two points of one d2 are one 16-byte vector.  Strided vector side (an interleaved
    // intermediate): lanes h = 0, 1 take adjacent positions, so the 32 lanes of a load
    // touch 16 cache lines instead of 32.
    const int h = tid % HP, n1 = tid / HP;
    const bool qint = prm.inter_q != 0;
    const LineAddr a0 = line_addr(g, kind, 0, lgi, qint);
    // vector-side offset of position n2 within a row
    const int alg = VM == 2 ? a0.a_lg : 0;
    const int64_t ahi = VM == 0 ? 1 : a0.a_hi;
    auto voff = [&](int n2) -> int64_t {
        if constexpr (VM == 0) return n2;
        else if constexpr (VM == 1) return (int64_t)n2 * ahi;
        else return (int64_t)(n2 >> alg) * ahi + (n2 & ((1 << alg) - 1));
    };
    constexpr bool vcont = VM != 1;   // positions n2, n2 + 1 (n2 even) adjacent
    const int lo0 = vcont ? 2 * h : h, lo1 = vcont ? 2 * h + 1 : h + HP;
    const int d0v = n1 & 31;
    const int d1v0 = (n1 >> 5) + (M / 32) * lo0, d1v1 = (n1 >> 5) + (M / 32) * lo1;
    // staging row of the vector side (PERS): VEC + 4 elements keep the 16-byte reads of
    // 16 rows per warp conflict-free, VEC + 2 the 8-byte reads of the strided form
    const int srow = vcont ? VEC + 4 : VEC + 2;
    // stage-2 / stage-B thread: d0 = lane, ka = warp
    const int ka2 = warp;
    // stage-3 / stage-A thread: ka = tid & 15, kb = tid >> 4; k mod 512 = tid
    const int ka3 = tid & 15, kb3 = tid >> 4;

    // vector side: row base of n1 in line a (positions n2 of the row are a_pos apart)
    auto rowbase = [&](const LineAddr &a) {
        const int64_t r = (int64_t)n1 << LV;
        return a.a_base + (r >> g.logL) * a.a_chunk + ((r & (g.L - 1)) >> alg) * ahi;
    };
    // frequency side: element k = tid + 512 kc of line a is at fofs(a) + kc * fstep
    const int k2 = tid & (VEC - 1);
    const int64_t VP = g.vp;
    const int flg = a0.f_lg;
    const int64_t pos0 = (int64_t)(tid >> LV) * VP + (k2 & (VP - 1));
    auto fofs = [&](const LineAddr &a) {
        return a.f_base + (int64_t)(k2 >> g.logVP) * a.f_chunk + (pos0 >> flg) * a.f_hi + (pos0 & ((1 << flg) - 1));
    };
    const int64_t fstep = ((((int64_t)512 >> LV) * VP) >> flg) * a0.f_hi;
    // contiguous frequency side (inverse input): the elements of threads t, t + 1 (t even,
    // k2 even, so the same run of VP) are adjacent and 16-byte aligned
    const bool fpair = INV && PERS && a0.f_hi == 1 && flg == 0 && VP >= 2;
    const bool scl = prm.apply_scale != 0;
    const float sre = (float)prm.scale_re, sim = (float)prm.scale_im;
    auto scale_c = [&](C o) -> C { return scl ? C{o.x * sre - o.y * sim, o.x * sim + o.y * sre} : o; };

    // L2 prefetch of line l's input (forward: vector side, for an interleaved
    // intermediate by the first line of each group for the group's runs; inverse:
    // frequency side chunks of the line)
    auto prefetch = [&](int64_t l) {
        if (l >= nl) return;
        const int nch = (int)(g.n >> g.logL);
        if (tid >= nch) return;
        const LineAddr fa = line_addr(g, kind, l, lgi, qint);
        if (!INV) {
            if (VM == 0 || (VM == 1 && (l & (ahi - 1)) == 0))
                prefetch_l2_bytes(in + fa.a_base + tid * fa.a_chunk, g.L * ahi * (int64_t)sizeof(C));
        } else if (fa.f_hi == 1) {
            prefetch_l2_bytes(in + fa.f_base + tid * fa.f_chunk, g.L * (int64_t)sizeof(C));
        } else if (qint && fa.f_lg == 0 && (l & (fa.f_hi - 1)) == 0) {
            // x pass on a y-position-interleaved intermediate: the first line of a group
            // fetches the group's G L contiguous elements of each chunk
            prefetch_l2_bytes(in + fa.f_base + tid * fa.f_chunk, g.L * fa.f_hi * (int64_t)sizeof(C));
        }
    };
    // asynchronous copies of line l's input into the staging region (PERS)
    auto issue = [&](int64_t l) {
        const LineAddr b = line_addr(g, kind, l, lgi, qint);
        if constexpr (!INV) {
            const C *row = in + rowbase(b);
            C *dst = S + n1 * srow;
            if constexpr (vcont) {
#pragma unroll
                for (int d2 = 0; d2 < 16; d2++) cp_async16(dst + lo0 + DSTEP * d2, row + voff(lo0 + DSTEP * d2));
            } else {
#pragma unroll
                for (int d2 = 0; d2 < 16; d2++) {
                    cp_async8(dst + lo0 + DSTEP * d2, row + voff(lo0 + DSTEP * d2));
                    cp_async8(dst + lo1 + DSTEP * d2, row + voff(lo1 + DSTEP * d2));
                }
            }
        } else {
            const C *ip = in + fofs(b);
            if (fpair) {
                // threads t, t + 1 (t even) need adjacent elements: the even one copies
                // both for kc < 16, the odd one for kc >= 16 (16-byte copies)
                const int half = tid & 1;
                const C *ipp = ip - half;
#pragma unroll
                for (int q = 0; q < 16; q++) {
                    const int kc = 16 * half + q;
                    cp_async16(S + kc * 512 + (tid - half), ipp + fstep * kc);
                }
            } else {
#pragma unroll
                for (int kc = 0; kc < 32; kc++) cp_async8(S + kc * 512 + tid, ip + fstep * kc);
            }
        }
        cp_async_commit();
    };

    int64_t line = blockIdx.x;
    if constexpr (PAIR && !INV && !PERS && VM == 1)   // matched by the wait before the first remote store
        asm volatile("barrier.cluster.arrive.relaxed.aligned;" ::: "memory");
    // prefetch distance: non-persistent, pf_tiles lines (one wave of CTAs); persistent,
    // pf_tiles iterations of the CTA's own walk
    const int64_t pfd = PERS ? prm.pf_tiles * lstep : prm.pf_tiles;
    if (PERS && line < nl) issue(line);
    if (!PERS) prefetch(line + pfd);
    // twiddle tables of this CTA (from the plan's hi/lo table of w_N^m) and the
    // per-thread output twiddle of stage 2, w_N^{d0 ka}
    for (int i = tid; i < KG::NT512 + KG::NT1024; i += KG::NT) {
        int m;
        if (i < KG::NT512) m = 32 * i;
        else {
            const int j = i - KG::NT512, kb = j >> 5, d0 = j & 31;
            m = 16 * ((d0 * kb) & 1023);
        }
        t512[i] = ldtw(twn, m);
    }
    const Wt f1 = ldtw(twn, lane * ka2);

    for (; line < nl; line += lstep) {
        const LineAddr a = line_addr(g, kind, line, lgi, qint);
        if (PERS && pfd > 0) prefetch(line + pfd);
        if constexpr (!INV) {
            // ---- stage 1: two 16-point transforms over d2
            C x0[16], x1[16];
            if constexpr (PERS) {
                cp_async_wait_all();
                const C *src = S + n1 * srow;
                if constexpr (vcont) {
#pragma unroll
                    for (int d2 = 0; d2 < 16; d2++) {
                        const float4 v = *reinterpret_cast<const float4 *>(src + lo0 + DSTEP * d2);
                        x0[d2] = C{v.x, v.y};
                        x1[d2] = C{v.z, v.w};
                    }
                } else {
#pragma unroll
                    for (int d2 = 0; d2 < 16; d2++) {
                        x0[d2] = src[lo0 + DSTEP * d2];
                        x1[d2] = src[lo1 + DSTEP * d2];
                    }
                }
            } else {
                const C *row = in + rowbase(a);
                if constexpr (vcont) {
#pragma unroll
                    for (int d2 = 0; d2 < 16; d2++) {
                        const float4 v = __ldg(reinterpret_cast<const float4 *>(row + voff(lo0 + DSTEP * d2)));
                        x0[d2] = C{v.x, v.y};
                        x1[d2] = C{v.z, v.w};
                    }
                } else if constexpr (PAIR && VM == 1) {
                    // rank rk (= line & 1) loads unit b = rk of both buddy lines; the
                    // partner's element goes to slot d2 * 512 + tid of its shared memory
                    namespace cg = cooperative_groups;
                    const int rk = (int)cg::this_cluster().block_rank();
                    C *peer = cg::this_cluster().map_shared_rank(S, rk ^ 1);
                    const C *prow = row - (line & 1);
                    const int lob = rk ? lo1 : lo0;
                    float4 v[16];
#pragma unroll
                    for (int d2 = 0; d2 < 16; d2++)
                        v[d2] = __ldg(reinterpret_cast<const float4 *>(prow + voff(lob + DSTEP * d2)));
                    asm volatile("barrier.cluster.wait.aligned;" ::: "memory");   // partner running
#pragma unroll
                    for (int d2 = 0; d2 < 16; d2++) {
                        const C e0{v[d2].x, v[d2].y}, e1{v[d2].z, v[d2].w};
                        peer[d2 * 512 + tid] = rk ? e0 : e1;
                        if (rk) x1[d2] = e1;
                        else x0[d2] = e0;
                    }
                    cg::this_cluster().sync();   // both halves delivered
#pragma unroll
                    for (int d2 = 0; d2 < 16; d2++) {
                        if (rk) x0[d2] = S[d2 * 512 + tid];
                        else x1[d2] = S[d2 * 512 + tid];
                    }
                } else {
#pragma unroll
                    for (int d2 = 0; d2 < 16; d2++) {
                        x0[d2] = ldg(row + voff(lo0 + DSTEP * d2));
                        x1[d2] = ldg(row + voff(lo1 + DSTEP * d2));
                    }
                }
            }
            dft<16, DIR, float>(x0);
            dft<16, DIR, float>(x1);
            __syncthreads();   // tables written; staging fully read
#pragma unroll
            for (int ka = 0; ka < 16; ka++) {
                S[KG::s1(ka, d1v0, d0v)] = x0[ka];
                S[KG::s1(ka, d1v1, d0v)] = x1[ka];
            }
            __syncthreads();
            // ---- stage 2: 32-point transforms over d1, unit (d0 = lane, ka = warp)
            C y[32];
#pragma unroll
            for (int d1 = 0; d1 < 32; d1++) {
                const C v = S[KG::s1(ka2, d1, lane)];
                y[d1] = d1 == 0 ? v : twmul<false>(v, t512[d1 * ka2]);
            }
            dft<32, DIR, float>(y);
#pragma unroll
            for (int kb = 0; kb < 32; kb++) {
                const C v = twmul<false>(y[kb], f1);
                y[kb] = kb == 0 ? v : twmul<false>(v, t1024[kb * 32 + lane]);
            }
            __syncthreads();   // exchange 1 fully read
#pragma unroll
            for (int kb = 0; kb < 32; kb++) S[KG::s2(kb, lane, ka2)] = y[kb];
            __syncthreads();
            // ---- stage 3: 32-point transforms over d0, unit k mod 512 = tid
#pragma unroll
            for (int d0 = 0; d0 < 32; d0++) y[d0] = S[KG::s2(kb3, d0, ka3)];
            if (PERS && line + lstep < nl) {
                __syncthreads();   // exchange 2 fully read: the region takes the next line
                issue(line + lstep);
            }
            dft<32, DIR, float>(y);
            C *op = out + fofs(a);
#pragma unroll
            for (int kc = 0; kc < 32; kc++) op[fstep * kc] = scale_c(y[kc]);
        } else {
            // ---- stage A: 32-point inverse transforms over kc, unit k mod 512 = tid
            C y[32];
            if constexpr (PERS) {
                cp_async_wait_all();
                if (fpair) __syncwarp();   // the pair partner copied half of this thread's points
#pragma unroll
                for (int kc = 0; kc < 32; kc++) y[kc] = S[kc * 512 + tid];
            } else {
                const C *ip = in + fofs(a);
#pragma unroll
                for (int kc = 0; kc < 32; kc++) y[kc] = ldg(ip + fstep * kc);
            }
            dft<32, DIR, float>(y);
            __syncthreads();   // tables written; staging fully read
#pragma unroll
            for (int d0 = 0; d0 < 32; d0++) S[KG::s2(kb3, d0, ka3)] = y[d0];
            __syncthreads();
            // ---- stage B: conj(w_N^{d0 (ka + 16 kb)}), 32-point inverse transforms over kb,
            //      conj(w512^{d1 ka}); unit (d0 = lane, ka = warp)
#pragma unroll
            for (int kb = 0; kb < 32; kb++) {
                const C v = twmul<true>(S[KG::s2(kb, lane, ka2)], f1);
                y[kb] = kb == 0 ? v : twmul<true>(v, t1024[kb * 32 + lane]);
            }
            dft<32, DIR, float>(y);
#pragma unroll
            for (int d1 = 1; d1 < 32; d1++) y[d1] = twmul<true>(y[d1], t512[d1 * ka2]);
            __syncthreads();   // exchange 2 fully read
#pragma unroll
            for (int d1 = 0; d1 < 32; d1++) S[KG::s1(ka2, d1, lane)] = y[d1];
            __syncthreads();
            // ---- stage C: 16-point inverse transforms over ka, units (n1, n2_lo = 2 h + b)
            C x0[16], x1[16];
#pragma unroll
            for (int ka = 0; ka < 16; ka++) {
                x0[ka] = S[KG::s1(ka, d1v0, d0v)];
                x1[ka] = S[KG::s1(ka, d1v1, d0v)];
            }
            if (PERS && line + lstep < nl) {
                __syncthreads();   // exchange 1 fully read: the region takes the next line
                issue(line + lstep);
            }
            dft<16, DIR, float>(x0);
            dft<16, DIR, float>(x1);
            C *row = out + rowbase(a);
            if constexpr (vcont) {
#pragma unroll
                for (int d2 = 0; d2 < 16; d2++) {
                    const C u = scale_c(x0[d2]), w = scale_c(x1[d2]);
                    *reinterpret_cast<float4 *>(row + voff(lo0 + DSTEP * d2)) = float4{u.x, u.y, w.x, w.y};
                }
            } else {
#pragma unroll
                for (int d2 = 0; d2 < 16; d2++) {
                    row[voff(lo0 + DSTEP * d2)] = scale_c(x0[d2]);
                    row[voff(lo1 + DSTEP * d2)] = scale_c(x1[d2]);
                }
            }
        }
    }
}

// Non-persistent: one CTA per line, L2 prefetch one wave of CTAs ahead.  PERS: one CTA
// per SM (or fewer when there are fewer lines), L2 prefetch one line of its walk ahead.
template <int LV, int LM, bool INV, bool PERS, int VM, bool PAIR = false>
cudaError_t launch_k3_vm(const LineParams &prm, cudaStream_t st) {
    constexpr size_t smem = K3Geom::SMEM;
    static_assert(smem <= 227 * 1024, "shared memory of one CTA");
    static_assert(!PAIR || (!PERS && !INV && VM == 1), "buddy-line pairs: forward strided one-line passes");
    auto kern = k3_pass_kernel<LV, LM, INV, PERS, VM, PAIR>;
    static int attr_done[64], resident[64];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!attr_done[dev]) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        int per_sm = 0, sms = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, K3Geom::NT, smem);
        if (e != cudaSuccess) return e;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
        if (per_sm <= 0) return cudaErrorInvalidConfiguration;
        resident[dev] = per_sm * sms;
        attr_done[dev] = 1;
    }
    LineParams lp = prm;
    lp.pf_tiles = PERS ? 1 : resident[dev];
    const int64_t grid = PERS ? (prm.nlines < resident[dev] ? prm.nlines : resident[dev]) : prm.nlines;
    if constexpr (PAIR) {
        if ((grid & 1) || prm.lg_inter < 1) return cudaErrorInvalidValue;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)grid);
        cfg.blockDim = dim3(K3Geom::NT);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = 2;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        cudaError_t e = cudaLaunchKernelEx(&cfg, kern, lp);
        if (e != cudaSuccess) return e;
    } else {
        kern<<<(unsigned)grid, K3Geom::NT, smem, st>>>(lp);
    }
    count_launch();
    return cudaGetLastError();
}

// 2D passes of N = 2^14 lines only; the vector side's address form follows from the pass
// kind and the intermediate's interleave.
// PAIR: the forward y pass on a row-interleaved intermediate runs on buddy-line pairs;
// every other pass of the variant runs the one-line kernel.
template <int LV, int LM, bool INV, bool PERS = false, bool PAIR = false>
cudaError_t launch_k3(const LineParams &prm, cudaStream_t st) {
    if (prm.g.n != K3Geom::N || prm.g.logVEC != LV || prm.g.logM != LM || prm.g.dim != 2) return cudaErrorInvalidValue;
    if constexpr (PAIR && !INV && !PERS)
        if (prm.kind == PASS_Y2 && prm.lg_inter > 0 && !prm.inter_q)
            return launch_k3_vm<LV, LM, INV, PERS, 1, true>(prm, st);
    if (prm.kind == PASS_Y2 && prm.lg_inter > 0)
        return prm.inter_q ? launch_k3_vm<LV, LM, INV, PERS, 2>(prm, st) : launch_k3_vm<LV, LM, INV, PERS, 1>(prm, st);
    if (prm.kind != PASS_X2 && prm.kind != PASS_Y2) return cudaErrorInvalidValue;
    return launch_k3_vm<LV, LM, INV, PERS, 0>(prm, st);
}

}  // namespace zm
