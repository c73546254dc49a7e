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
//     slice (one buffer, two views used at different times), XOR-swizzled so the warp
//     access patterns of every stage are (nearly) free of bank conflicts;
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

template <typename T, int LV, int LM, int CL, int TL, int NT, bool INV>
__global__ void __launch_bounds__(NT, (NT < 1024 ? 1024 / NT : 1)) fused_pass_kernel(const LineParams prm) {
    constexpr int VEC = 1 << LV, M = 1 << LM, N = VEC * M;
    constexpr int ML = M / CL, VL = VEC / CL;        // rows / columns owned by one CTA
    constexpr int E = TL * N / CL;                    // elements per CTA
    constexpr int EPT = E / NT;
    static_assert(ML >= 1 && VL >= 1 && ML * CL == M && VL * CL == VEC, "cluster split");
    static_assert(EPT * NT == E, "threads must divide the tile");
    constexpr int RA1 = VEC < EPT ? VEC : EPT, RA2 = VEC / RA1;
    constexpr int RC1 = M < EPT ? M : EPT, RC2 = M / RC1;
    static_assert(RA2 <= EPT && RC2 <= EPT, "sub-transform needs more than two register stages");
    static_assert(EPT % RA1 == 0 && EPT % RA2 == 0 && EPT % RC1 == 0 && EPT % RC2 == 0, "radix");
    constexpr bool C64 = sizeof(T) == 4;
    constexpr int XM = (VEC < 16 ? VEC : 16) - 1;
    constexpr int YM = (M < 16 ? M : 16) - 1;
    constexpr int DIR = INV ? 1 : -1;
    using C = cpx<T>;
    using Wt = tw<T>;

    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *S = reinterpret_cast<C *>(smem_raw);
    Wt *stv = reinterpret_cast<Wt *>(smem_raw + sizeof(C) * E);   // w_VEC^m, m < VEC
    Wt *stm = stv + VEC;                                            // w_M^m,   m < M
    __shared__ int64_t s_abase[TL], s_fbase[TL];

    // local rows X[t][n1l][p] and local columns Y[t][k2l][q]
    auto Xi = [](int t, int n1l, int p) {
        const int s = (C64 ? ((n1l & 7) << 1) : (n1l & 7)) & XM;
        return ((t * ML + n1l) << LV) + (p ^ s);
    };
    auto Yi = [](int t, int k2l, int q) {
        const int s = (C64 ? (k2l & 15) : (k2l & 7)) & YM;
        return ((t * VL + k2l) << LM) + (q ^ s);
    };

    int rank = 0;
    if constexpr (CL > 1) rank = (int)cooperative_groups::this_cluster().block_rank();
    const int n1_0 = rank * ML, k2_0 = rank * VL;   // first owned row / column
    const Geom &g = prm.g;
    const int tid = threadIdx.x;
    const int64_t l0 = (int64_t)(blockIdx.x / CL) * TL;
    const C *in = reinterpret_cast<const C *>(prm.in);
    C *out = reinterpret_cast<C *>(prm.out);
    const Wt *Wg = reinterpret_cast<const Wt *>(prm.W);
    const LineAddr a0 = line_addr(g, prm.kind, l0);
    if (tid < TL) {
        const LineAddr a = line_addr(g, prm.kind, l0 + tid);
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

    // frequency-side element (t, k2 global, k1)
    auto faddr = [&](int t, int k2, int k1) {
        const int64_t c = k2 >> logVP, f = k2 & (VP - 1);
        return s_fbase[t] + c * a0.f_chunk + ((int64_t)k1 * VP + f) * a0.f_pos;
    };
    // vector-side element e of this CTA's rows (row-major over [t][n1l][p]) -> global
    auto aaddr = [&](int e) {
        const int t = e / (ML * VEC), r = (e % (ML * VEC)) + n1_0 * VEC;   // concatenated position
        const int64_t c = r >> logL, pos = r & (L - 1);
        return s_abase[t] + c * a0.a_chunk + pos;
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

    if (!INV) {
        // ---- 1. vector side -> local rows X (16-byte vectors, all loads before stores)
        {
            uint4 buf[VPT];
#pragma unroll
            for (int i = 0; i < VPT; i++) buf[i] = ldg16(in + aaddr((tid + i * NT) * VE));
#pragma unroll
            for (int i = 0; i < VPT; i++) {
                const int e = (tid + i * NT) * VE;
                const int t = e / (ML * VEC), r = e % (ML * VEC);
                *reinterpret_cast<uint4 *>(&S[Xi(t, r >> LV, r & (VEC - 1))]) = buf[i];
            }
        }
        __syncthreads();
        // ---- 2. VEC-point row transforms over n2, results scattered to the column owners
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
#pragma unroll
                for (int r = 0; r < RA1; r++) v[i][r] = S[Xi(ut[i], un1[i], uj[i] + RA2 * r)];
            }
#pragma unroll
            for (int i = 0; i < NU; i++) dft<RA1, DIR, T>(v[i]);
            if constexpr (RA2 == 1) {
                tile_sync<CL>();   // every CTA has finished reading its rows
#pragma unroll
                for (int i = 0; i < NU; i++)
#pragma unroll
                    for (int r = 0; r < RA1; r++)
                        yowner(r)[Yi(ut[i], r % VL, n1_0 + un1[i])] = v[i][r];
            } else {
                __syncthreads();
#pragma unroll
                for (int i = 0; i < NU; i++)
#pragma unroll
                    for (int r = 0; r < RA1; r++) S[Xi(ut[i], un1[i], uj[i] * RA1 + r)] = v[i][r];
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
#pragma unroll
                    for (int r = 0; r < RA2; r++) w[i][r] = S[Xi(wt[i], wn1[i], wj[i] + RA1 * r)];
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
                        yowner(k2)[Yi(wt[i], k2 % VL, n1_0 + wn1[i])] = w[i][r];
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
                zk[i] = u % VL;
                const int rr = u / VL;
                zj[i] = rr % RC2;
                zt[i] = rr / RC2;
                const int k2 = k2_0 + zk[i];
#pragma unroll
                for (int r = 0; r < RC1; r++) {
                    const int n1 = zj[i] + RC2 * r;
                    z[i][r] = twmul<false>(S[Yi(zt[i], zk[i], n1)], ldtw(Wg, n1 * VEC + k2));
                }
            }
#pragma unroll
            for (int i = 0; i < NU; i++) dft<RC1, DIR, T>(z[i]);
            if constexpr (RC2 == 1) {
#pragma unroll
                for (int i = 0; i < NU; i++)
#pragma unroll
                    for (int r = 0; r < RC1; r++) {
                        C o = z[i][r];
                        if (scl) o = {o.x * sre - o.y * sim, o.x * sim + o.y * sre};
                        out[faddr(zt[i], k2_0 + zk[i], r)] = o;
                    }
            } else {
                __syncthreads();
#pragma unroll
                for (int i = 0; i < NU; i++)
#pragma unroll
                    for (int r = 0; r < RC1; r++) S[Yi(zt[i], zk[i], zj[i] * RC1 + r)] = z[i][r];
                __syncthreads();
                constexpr int NU2 = EPT / RC2;
#pragma unroll
                for (int i = 0; i < NU2; i++) {
                    const int u = tid + i * NT;
                    const int k2l = u % VL;
                    const int rr = u / VL;
                    const int j2 = rr % RC1, t = rr / RC1;
                    C y[RC2];
#pragma unroll
                    for (int r = 0; r < RC2; r++) y[r] = S[Yi(t, k2l, j2 + RC1 * r)];
#pragma unroll
                    for (int r = 1; r < RC2; r++) y[r] = twmul<false>(y[r], stm[j2 * r]);
                    dft<RC2, DIR, T>(y);
#pragma unroll
                    for (int r = 0; r < RC2; r++) {
                        C o = y[r];
                        if (scl) o = {o.x * sre - o.y * sim, o.x * sim + o.y * sre};
                        out[faddr(t, k2_0 + k2l, j2 + RC1 * r)] = o;
                    }
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
                zk[i] = u % VL;
                const int rr = u / VL;
                zj[i] = rr % RC2;
                zt[i] = rr / RC2;
#pragma unroll
                for (int r = 0; r < RC1; r++)
                    z[i][r] = ldg(in + faddr(zt[i], k2_0 + zk[i], zj[i] + RC2 * r));
            }
#pragma unroll
            for (int i = 0; i < NU; i++) dft<RC1, DIR, T>(z[i]);
            if constexpr (RC2 == 1) {
                // n1 = r: conj(w_N^{n1 k2}), then to the row owners X[t][n1l][k2]
                tile_sync<CL>();
#pragma unroll
                for (int i = 0; i < NU; i++)
#pragma unroll
                    for (int r = 0; r < RC1; r++) {
                        const int k2 = k2_0 + zk[i];
                        xowner(r)[Xi(zt[i], r % ML, k2)] = twmul<true>(z[i][r], ldtw(Wg, r * VEC + k2));
                    }
            } else {
#pragma unroll
                for (int i = 0; i < NU; i++)
#pragma unroll
                    for (int r = 0; r < RC1; r++) S[Yi(zt[i], zk[i], zj[i] * RC1 + r)] = z[i][r];
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
#pragma unroll
                    for (int r = 0; r < RC2; r++) y[i][r] = S[Yi(yt[i], yk[i], yj[i] + RC1 * r)];
                }
#pragma unroll
                for (int i = 0; i < NU2; i++) {
#pragma unroll
                    for (int r = 1; r < RC2; r++) y[i][r] = twmul<true>(y[i][r], stm[yj[i] * r]);
                    dft<RC2, DIR, T>(y[i]);
                }
                tile_sync<CL>();   // every CTA has finished reading its columns
#pragma unroll
                for (int i = 0; i < NU2; i++)
#pragma unroll
                    for (int r = 0; r < RC2; r++) {
                        const int n1 = yj[i] + RC1 * r, k2 = k2_0 + yk[i];
                        xowner(n1)[Xi(yt[i], n1 % ML, k2)] = twmul<true>(y[i][r], ldtw(Wg, n1 * VEC + k2));
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
#pragma unroll
                for (int r = 0; r < RA1; r++) v[i][r] = S[Xi(ut[i], un1[i], uj[i] + RA2 * r)];
            }
            __syncthreads();
#pragma unroll
            for (int i = 0; i < NU; i++) dft<RA1, DIR, T>(v[i]);
            if constexpr (RA2 == 1) {
#pragma unroll
                for (int i = 0; i < NU; i++)
#pragma unroll
                    for (int r = 0; r < RA1; r++) S[Xi(ut[i], un1[i], r)] = v[i][r];
            } else {
#pragma unroll
                for (int i = 0; i < NU; i++)
#pragma unroll
                    for (int r = 0; r < RA1; r++) S[Xi(ut[i], un1[i], uj[i] * RA1 + r)] = v[i][r];
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
#pragma unroll
                    for (int r = 0; r < RA2; r++) w[i][r] = S[Xi(wt[i], wn1[i], wj[i] + RA1 * r)];
                }
                __syncthreads();
#pragma unroll
                for (int i = 0; i < NU2; i++) {
#pragma unroll
                    for (int r = 1; r < RA2; r++) w[i][r] = twmul<true>(w[i][r], stv[wj[i] * r]);
                    dft<RA2, DIR, T>(w[i]);
#pragma unroll
                    for (int r = 0; r < RA2; r++) S[Xi(wt[i], wn1[i], wj[i] + RA1 * r)] = w[i][r];
                }
            }
        }
        __syncthreads();
        // ---- 3. local rows -> vector side (16-byte vectors), scale applied here
        {
#pragma unroll
            for (int i = 0; i < VPT; i++) {
                const int e = (tid + i * NT) * VE;
                const int t = e / (ML * VEC), r = e % (ML * VEC);
                uint4 v = *reinterpret_cast<const uint4 *>(&S[Xi(t, r >> LV, r & (VEC - 1))]);
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
    return sizeof(cpx<T>) * (size_t)TL * ((size_t)1 << (LV + LM)) / CL +
           sizeof(tw<T>) * (((size_t)1 << LV) + ((size_t)1 << LM));
}

template <typename T, int LV, int LM, int CL, int TL, int NT>
cudaError_t launch_fused(const LineParams &prm, bool inv, cudaStream_t st) {
    constexpr size_t smem = fused_smem_bytes<T, LV, LM, CL, TL, NT>();
    auto kern = inv ? fused_pass_kernel<T, LV, LM, CL, TL, NT, true>
                    : fused_pass_kernel<T, LV, LM, CL, TL, NT, false>;
    static int attr_done[64][2];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && !attr_done[dev][inv]) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        attr_done[dev][inv] = 1;
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
