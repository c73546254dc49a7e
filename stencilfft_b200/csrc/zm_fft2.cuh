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
//   * each CTA's shared memory holds rows X[t][n1][p] (stride VEC + 2) and columns
//     Y[t][k2][q] (stride M + 1, or one pad per 16 for VEC <= 4) of its slice -- one
//     buffer, two views used at different times.  The padding keeps the warp access
//     patterns of every stage (nearly) free of bank conflicts while every register of a
//     butterfly sits at a compile-time offset from its base;
//   * each sub-transform is at most two register stages of radix <= 16 (Stockham
//     indexing), with the stage twiddles w_VEC, w_M in shared memory and the inter-step
//     twiddle w_N^{n1 k2} read from an [n1][k2]-ordered table, coalesced across lanes;
//   * the vector side (reference real layout / REPACK layout) moves through shared
//     memory as 16-byte vectors, all loads of a thread issued before its stores; the
//     frequency side is read / written straight from registers with lanes along k2.
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

// Shared-memory geometry of one CTA's slice.
template <int LV, int LM, int CL, int TL> struct SliceGeom {
    static constexpr int VEC = 1 << LV, M = 1 << LM;
    static constexpr int ML = M / CL, VL = VEC / CL;
    static constexpr int XR = VEC + 2;                       // padded row
    static constexpr int YP = VEC <= 4 ? 1 : 0;              // pad per 16 in a column
    static constexpr int YR = VEC <= 4 ? M + M / 16 : M + 1; // padded column
    static constexpr int XE = TL * ML * XR, YE = TL * VL * YR;
    static constexpr int ELEMS = XE > YE ? XE : YE;
    static ZM_DEV int X(int t, int n1l, int p) { return (t * ML + n1l) * XR + p; }
    static ZM_DEV int Y(int t, int k2l, int q) { return (t * VL + k2l) * YR + q + (q >> 4) * YP; }
};

template <typename T, int LV, int LM, int CL, int TL, int NT, bool INV>
__global__ void __launch_bounds__(NT, (NT < 1024 ? 1024 / NT : 1)) fused_pass_kernel(const LineParams prm) {
    using SG = SliceGeom<LV, LM, CL, TL>;
    constexpr int VEC = SG::VEC, M = SG::M, N = VEC * M;
    constexpr int ML = SG::ML, VL = SG::VL;
    constexpr int E = TL * N / CL;                    // elements per CTA
    constexpr int EPT = E / NT;
    static_assert(ML >= 1 && VL >= 1 && ML * CL == M && VL * CL == VEC, "cluster split");
    static_assert(EPT * NT == E, "threads must divide the tile");
    constexpr int RA1 = VEC < EPT ? VEC : EPT, RA2 = VEC / RA1;
    constexpr int RC1 = M < EPT ? M : EPT, RC2 = M / RC1;
    static_assert(RA2 <= EPT && RC2 <= EPT, "sub-transform needs more than two register stages");
    static_assert(EPT % RA1 == 0 && EPT % RA2 == 0 && EPT % RC1 == 0 && EPT % RC2 == 0, "radix");
    constexpr int DIR = INV ? 1 : -1;
    using C = cpx<T>;
    using Wt = tw<T>;

    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *S = reinterpret_cast<C *>(smem_raw);
    Wt *stv = reinterpret_cast<Wt *>(smem_raw + sizeof(C) * SG::ELEMS);   // w_VEC^m, m < VEC
    Wt *stm = stv + VEC;                                                    // w_M^m,   m < M
    __shared__ int64_t s_abase[TL], s_fbase[TL];

    int rank = 0;
    if constexpr (CL > 1) rank = (int)cooperative_groups::this_cluster().block_rank();
    const int n1_0 = rank * ML, k2_0 = rank * VL;   // first owned row / column
    const Geom &g = prm.g;
    const int tid = threadIdx.x;
    const int64_t l0 = (int64_t)(blockIdx.x / CL) * TL;
    const C *in = reinterpret_cast<const C *>(prm.in);
    C *out = reinterpret_cast<C *>(prm.out);
    const LineAddr a0 = line_addr(g, prm.kind, l0, prm.lg_inter);
    if (tid < TL) {
        const LineAddr a = line_addr(g, prm.kind, l0 + tid, prm.lg_inter);
        s_abase[tid] = a.a_base;
        s_fbase[tid] = a.f_base;
    }
    {
        const Wt *tv = reinterpret_cast<const Wt *>(prm.twv);
        const Wt *tm = reinterpret_cast<const Wt *>(prm.twm);
        for (int i = tid; i < VEC + M; i += NT) stv[i] = i < VEC ? ldtw(tv, i) : ldtw(tm, i - VEC);
    }
    __syncthreads();
    const int logL = g.logL, logVP = g.logVP;
    const int64_t L = g.L, VP = g.vp;
    const bool scl = prm.apply_scale != 0;
    const T sre = (T)prm.scale_re, sim = (T)prm.scale_im;
    constexpr int VE = 16 / (int)sizeof(C);      // elements per 16-byte vector
    constexpr int VPT = E / VE / NT;             // vectors per thread
    static_assert(VPT * VE * NT == E, "vector copy");

    // frequency side: pointer to (t, k2 global, k1 = k1_0) and the step between k1 and k1 + kstep
    const int flg = a0.f_lg;
    auto fptr = [&](auto *base, int t, int k2, int k1_0) {
        const int64_t c = k2 >> logVP, f = k2 & (VP - 1);
        const int64_t pos = (int64_t)k1_0 * VP + f;
        return base + s_fbase[t] + c * a0.f_chunk + (pos >> flg) * a0.f_hi + (pos & ((1 << flg) - 1));
    };
    // (VP is a multiple of the interleave 2^flg whenever flg > 0)
    const int64_t fstep1 = (((int64_t)RC2 * VP) >> flg) * a0.f_hi;   // k1 += RC2 (column stage 1)
    const int64_t fstep2 = (((int64_t)RC1 * VP) >> flg) * a0.f_hi;   // k1 += RC1 (column stage 2)
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
    auto arow = [&](int t, int n1l) {
        const int r = (n1_0 + n1l) * VEC;
        return s_abase[t] + (int64_t)(r >> logL) * a0.a_chunk + (int64_t)(r & (L - 1)) * apos;
    };
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
    // inter-step twiddles w_N^{(j + s r) k2}, r = 0, 1, ...: FP64 power walk from the
    // table w_N^m (m < 16 VEC), then the stored form (hi/lo split for complex64)
    const double2 *Td = reinterpret_cast<const double2 *>(prm.twd);
    struct Walk {
        double2 w, step;
        ZM_DEV tw<T> next() {
            const tw<T> r = tw_from_d<T>(w);
            w = cmul_d(w, step);
            return r;
        }
    };
    auto walk = [&](int j, int s, int k2) { return Walk{ldd2(Td + j * k2), ldd2(Td + s * k2)}; };
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

    if (!INV) {
        // ---- 1. vector side -> local rows X (16-byte vectors, all loads before stores);
        //         with two row stages the first one reads global memory directly instead
        if constexpr (RA2 == 1) {
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
            int ut[NU], un1[NU], uj[NU];
#pragma unroll
            for (int i = 0; i < NU; i++) {
                const int u = tid + i * NT;
                if constexpr (RA2 == 1) {
                    uj[i] = 0;
                    un1[i] = u % ML;
                    ut[i] = u / ML;
                    const C *row = S + SG::X(ut[i], un1[i], 0);
#pragma unroll
                    for (int r = 0; r < RA1; r++) v[i][r] = row[r];
                } else {
                    rowunit(u, RA2, ut[i], un1[i], uj[i]);
                    const C *row = in + arow(ut[i], un1[i]) + uj[i] * apos;
#pragma unroll
                    for (int r = 0; r < RA1; r++) v[i][r] = ldg(row + RA2 * r * apos);
                }
            }
#pragma unroll
            for (int i = 0; i < NU; i++) dft<RA1, DIR, T>(v[i]);
            if constexpr (RA2 == 1) {
                tile_sync<CL>();   // every CTA has finished reading its rows
#pragma unroll
                for (int i = 0; i < NU; i++)
#pragma unroll
                    for (int r = 0; r < RA1; r++)
                        yowner(r)[SG::Y(ut[i], r % VL, n1_0 + un1[i])] = v[i][r];
            } else {
#pragma unroll
                for (int i = 0; i < NU; i++) {
                    C *row = S + SG::X(ut[i], un1[i], uj[i] * RA1);
#pragma unroll
                    for (int r = 0; r < RA1; r++) row[r] = v[i][r];
                }
                __syncthreads();
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
                    const C *row = S + SG::X(wt[i], wn1[i], wj[i]);
#pragma unroll
                    for (int r = 0; r < RA2; r++) w[i][r] = row[RA1 * r];
                }
#pragma unroll
                for (int i = 0; i < NU2; i++) {
#pragma unroll
                    for (int r = 1; r < RA2; r++) w[i][r] = twmul<false>(w[i][r], stv[wj[i] * r]);
                    dft<RA2, DIR, T>(w[i]);
                }
                tile_sync<CL>();
#pragma unroll
                for (int i = 0; i < NU2; i++)
#pragma unroll
                    for (int r = 0; r < RA2; r++) {
                        const int k2 = wj[i] + RA1 * r;
                        yowner(k2)[SG::Y(wt[i], k2 % VL, n1_0 + wn1[i])] = w[i][r];
                    }
            }
        }
        tile_sync<CL>();
        // ---- 3. w_N^{n1 k2}, M-point column transforms over n1, frequency-side store
        {
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
                const int yb = SG::Y(zt[i], zk[i], 0);
#pragma unroll
                for (int r = 0; r < RC1; r++) {
                    const int q = zj[i] + RC2 * r;
                    z[i][r] = twmul<false>(S[yb + q + (q >> 4) * SG::YP], wk.next());
                }
            }
#pragma unroll
            for (int i = 0; i < NU; i++) dft<RC1, DIR, T>(z[i]);
            if constexpr (RC2 == 1) {
#pragma unroll
                for (int i = 0; i < NU; i++) {
                    C *op = fptr(out, zt[i], k2_0 + zk[i], 0);
#pragma unroll
                    for (int r = 0; r < RC1; r++) op[fstep1 * r] = scale_c(z[i][r]);
                }
            } else {
                __syncthreads();
#pragma unroll
                for (int i = 0; i < NU; i++) {
                    const int yb = SG::Y(zt[i], zk[i], 0);
#pragma unroll
                    for (int r = 0; r < RC1; r++) {
                        const int q = zj[i] * RC1 + r;
                        S[yb + q + (q >> 4) * SG::YP] = z[i][r];
                    }
                }
                __syncthreads();
                constexpr int NU2 = EPT / RC2;
#pragma unroll
                for (int i = 0; i < NU2; i++) {
                    const int u = tid + i * NT;
                    int t, k2l, j2;
                    colunit(u, RC1, t, k2l, j2);
                    const int yb = SG::Y(t, k2l, 0);
                    C y[RC2];
#pragma unroll
                    for (int r = 0; r < RC2; r++) {
                        const int q = j2 + RC1 * r;
                        y[r] = S[yb + q + (q >> 4) * SG::YP];
                    }
#pragma unroll
                    for (int r = 1; r < RC2; r++) y[r] = twmul<false>(y[r], stm[j2 * r]);
                    dft<RC2, DIR, T>(y);
                    C *op = fptr(out, t, k2_0 + k2l, j2);
#pragma unroll
                    for (int r = 0; r < RC2; r++) op[fstep2 * r] = scale_c(y[r]);
                }
            }
        }
    } else {
        // ---- 1. frequency side -> M-point inverse column transforms over k1 (local columns)
        {
            constexpr int NU = EPT / RC1;
            C z[NU][RC1];
            int zt[NU], zk[NU], zj[NU];
#pragma unroll
            for (int i = 0; i < NU; i++) {
                const int u = tid + i * NT;
                colunit(u, RC2, zt[i], zk[i], zj[i]);
                const C *ip = fptr(in, zt[i], k2_0 + zk[i], zj[i]);
#pragma unroll
                for (int r = 0; r < RC1; r++) z[i][r] = ldg(ip + fstep1 * r);
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
                        xowner(r)[SG::X(zt[i], r % ML, k2)] = twmul<true>(z[i][r], wk.next());
                }
            } else {
#pragma unroll
                for (int i = 0; i < NU; i++) {
                    const int yb = SG::Y(zt[i], zk[i], 0);
#pragma unroll
                    for (int r = 0; r < RC1; r++) {
                        const int q = zj[i] * RC1 + r;
                        S[yb + q + (q >> 4) * SG::YP] = z[i][r];
                    }
                }
                __syncthreads();
                constexpr int NU2 = EPT / RC2;
                C y[NU2][RC2];
                int yt[NU2], yk[NU2], yj[NU2];
#pragma unroll
                for (int i = 0; i < NU2; i++) {
                    const int u = tid + i * NT;
                    yk[i] = u % VL;
                    const int rr = u / VL;
                    yj[i] = rr % RC1;
                    yt[i] = rr / RC1;
                    const int yb = SG::Y(yt[i], yk[i], 0);
#pragma unroll
                    for (int r = 0; r < RC2; r++) {
                        const int q = yj[i] + RC1 * r;
                        y[i][r] = S[yb + q + (q >> 4) * SG::YP];
                    }
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
                        xowner(n1)[SG::X(yt[i], n1 % ML, k2)] = twmul<true>(y[i][r], wk.next());
                    }
                }
            }
        }
        tile_sync<CL>();
        // ---- 2. VEC-point inverse row transforms over k2 -> local rows X[t][n1l][n2]
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
                const C *row = S + SG::X(ut[i], un1[i], uj[i]);
#pragma unroll
                for (int r = 0; r < RA1; r++) v[i][r] = row[RA2 * r];
            }
            __syncthreads();
#pragma unroll
            for (int i = 0; i < NU; i++) dft<RA1, DIR, T>(v[i]);
            if constexpr (RA2 == 1) {
#pragma unroll
                for (int i = 0; i < NU; i++) {
                    C *row = S + SG::X(ut[i], un1[i], 0);
#pragma unroll
                    for (int r = 0; r < RA1; r++) row[r] = v[i][r];
                }
            } else {
#pragma unroll
                for (int i = 0; i < NU; i++) {
                    C *row = S + SG::X(ut[i], un1[i], uj[i] * RA1);
#pragma unroll
                    for (int r = 0; r < RA1; r++) row[r] = v[i][r];
                }
                __syncthreads();
                constexpr int NU2 = EPT / RA2;
                C w[NU2][RA2];
                int wt[NU2], wn1[NU2], wj[NU2];
#pragma unroll
                for (int i = 0; i < NU2; i++) {
                    const int u = tid + i * NT;
                    rowunit(u, RA1, wt[i], wn1[i], wj[i]);   // this stage stores to global
                    const C *row = S + SG::X(wt[i], wn1[i], wj[i]);
#pragma unroll
                    for (int r = 0; r < RA2; r++) w[i][r] = row[RA1 * r];
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
        // ---- 3. single row stage: local rows -> vector side (16-byte vectors), scale applied here
        if constexpr (RA2 == 1) {
            __syncthreads();
#pragma unroll
            for (int i = 0; i < VPT; i++) {
                const int e = (tid + i * NT) * VE;
                uint4 v = *reinterpret_cast<const uint4 *>(&S[xidx_of_e(e)]);
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
}

template <typename T, int LV, int LM, int CL, int TL, int NT>
constexpr size_t fused_smem_bytes() {
    return sizeof(cpx<T>) * (size_t)SliceGeom<LV, LM, CL, TL>::ELEMS +
           sizeof(tw<T>) * (((size_t)1 << LV) + ((size_t)1 << LM));
}

template <typename T, int LV, int LM, int CL, int TL, int NT, bool INV>
cudaError_t launch_fused(const LineParams &prm, cudaStream_t st) {
    constexpr size_t smem = fused_smem_bytes<T, LV, LM, CL, TL, NT>();
    auto kern = fused_pass_kernel<T, LV, LM, CL, TL, NT, INV>;
    static int attr_done[64];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && !attr_done[dev]) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        attr_done[dev] = 1;
    }
    const unsigned grid = (unsigned)(prm.nlines / TL) * CL;
    if constexpr (CL == 1) {
        kern<<<grid, NT, smem, st>>>(prm);
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
        cudaError_t e = cudaLaunchKernelEx(&cfg, kern, prm);
        if (e != cudaSuccess) return e;
    }
    count_launch();
    return cudaGetLastError();
}

}  // namespace zm
