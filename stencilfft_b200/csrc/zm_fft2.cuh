// zm_fft2.cuh -- size-specialised fused axis pass (the fast path of zm_fft.cu).
//
// Same computation as line_fft_kernel (see zm_fft.cu for how one pass replaces the
// reference's FFT1a / pack / All-to-All / unpack+twiddle / FFT1b / repack stages), with
// the sizes VEC = 2^LV and M = 2^LM fixed at compile time so every index, stride and
// radix is a constant:
//   * the CTA holds TL lines as two views of one shared-memory buffer: rows X[t][n1][p]
//     (the VEC-point transforms) and columns Y[t][k2][q] (the M-point transforms), each
//     XOR-swizzled so the warp access patterns of every stage are (nearly) free of bank
//     conflicts;
//   * each sub-transform is at most two register stages of radix <= 16 (Stockham
//     indexing), with the stage twiddles w_VEC, w_M in shared memory and the inter-step
//     twiddle w_N^{n1 k2} read from an [n1][k2]-ordered table, coalesced across lanes;
//   * the vector side (reference real layout / REPACK layout) moves through shared
//     memory as 16-byte vectors, all loads of a thread issued before its stores; the
//     frequency side is read / written straight from registers with lanes along k2.
#pragma once

#include "zm_common.cuh"

namespace zm {

template <typename T> ZM_DEV uint4 ldg16(const cpx<T> *p) {
    return __ldg(reinterpret_cast<const uint4 *>(p));
}

template <typename T, int LV, int LM, int TL, int NT, bool INV>
__global__ void __launch_bounds__(NT, (NT < 1024 ? 1024 / NT : 1)) fused_pass_kernel(const LineParams prm) {
    constexpr int VEC = 1 << LV, M = 1 << LM, N = VEC * M, E = TL * N;
    constexpr int EPT = E / NT;
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

    // rows: X[t][n1][p]; columns: Y[t][k2][q] (same storage, used at different times)
    auto Xi = [](int t, int n1, int p) {
        const int s = (C64 ? ((n1 & 7) << 1) : (n1 & 7)) & XM;
        return ((t * M + n1) << LV) + (p ^ s);
    };
    auto Yi = [](int t, int k2, int q) {
        const int s = (C64 ? (k2 & 15) : (k2 & 7)) & YM;
        return ((t * VEC + k2) << LM) + (q ^ s);
    };

    const Geom &g = prm.g;
    const int tid = threadIdx.x;
    const int64_t l0 = (int64_t)blockIdx.x * TL;
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

    auto fstore_addr = [&](int t, int k2, int k1) {
        const int64_t c = k2 >> logVP, f = k2 & (VP - 1);
        return s_fbase[t] + c * a0.f_chunk + ((int64_t)k1 * VP + f) * a0.f_pos;
    };

    if (!INV) {
        // ---- 1. vector side -> rows X (16-byte vectors, all loads before stores)
        {
            uint4 buf[VPT];
#pragma unroll
            for (int i = 0; i < VPT; i++) {
                const int e = (tid + i * NT) * VE;
                const int t = e >> (LV + LM), r = e & (N - 1);
                const int64_t c = r >> logL, pos = r & (L - 1);
                buf[i] = ldg16(in + s_abase[t] + c * a0.a_chunk + pos);
            }
#pragma unroll
            for (int i = 0; i < VPT; i++) {
                const int e = (tid + i * NT) * VE;
                const int t = e >> (LV + LM), r = e & (N - 1);
                *reinterpret_cast<uint4 *>(&S[Xi(t, r >> LV, r & (VEC - 1))]) = buf[i];
            }
        }
        __syncthreads();
        // ---- 2. VEC-point row transforms over n2 -> columns Y[t][k2][n1]
        {
            constexpr int NU = EPT / RA1;
            C v[NU][RA1];
            int ut[NU], un1[NU], uj[NU];
#pragma unroll
            for (int i = 0; i < NU; i++) {
                const int u = tid + i * NT;
                uj[i] = u & (RA2 - 1);
                const int rr = u / RA2;
                un1[i] = rr & (M - 1);
                ut[i] = rr >> LM;
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
                    for (int r = 0; r < RA1; r++) S[Yi(ut[i], r, un1[i])] = v[i][r];
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
                    wn1[i] = rr & (M - 1);
                    wt[i] = rr >> LM;
#pragma unroll
                    for (int r = 0; r < RA2; r++) w[i][r] = S[Xi(wt[i], wn1[i], wj[i] + RA1 * r)];
                }
                __syncthreads();
#pragma unroll
                for (int i = 0; i < NU2; i++) {
#pragma unroll
                    for (int r = 1; r < RA2; r++) w[i][r] = twmul<false>(w[i][r], stv[wj[i] * r]);
                    dft<RA2, DIR, T>(w[i]);
#pragma unroll
                    for (int r = 0; r < RA2; r++) S[Yi(wt[i], wj[i] + RA1 * r, wn1[i])] = w[i][r];
                }
            }
        }
        __syncthreads();
        // ---- 3. w_N^{n1 k2}, M-point column transforms over n1, frequency-side store
        {
            constexpr int NU = EPT / RC1;
            C z[NU][RC1];
            int zt[NU], zk[NU], zj[NU];
#pragma unroll
            for (int i = 0; i < NU; i++) {
                const int u = tid + i * NT;
                zk[i] = u & (VEC - 1);
                const int rr = u >> LV;
                zj[i] = rr % RC2;
                zt[i] = rr / RC2;
#pragma unroll
                for (int r = 0; r < RC1; r++) {
                    const int n1 = zj[i] + RC2 * r;
                    z[i][r] = twmul<false>(S[Yi(zt[i], zk[i], n1)], ldtw(Wg, n1 * VEC + zk[i]));
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
                        out[fstore_addr(zt[i], zk[i], r)] = o;
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
                    const int k2 = u & (VEC - 1);
                    const int rr = u >> LV;
                    const int j2 = rr % RC1, t = rr / RC1;
                    C y[RC2];
#pragma unroll
                    for (int r = 0; r < RC2; r++) y[r] = S[Yi(t, k2, j2 + RC1 * r)];
#pragma unroll
                    for (int r = 1; r < RC2; r++) y[r] = twmul<false>(y[r], stm[j2 * r]);
                    dft<RC2, DIR, T>(y);
#pragma unroll
                    for (int r = 0; r < RC2; r++) {
                        C o = y[r];
                        if (scl) o = {o.x * sre - o.y * sim, o.x * sim + o.y * sre};
                        out[fstore_addr(t, k2, j2 + RC1 * r)] = o;
                    }
                }
            }
        }
    } else {
        // ---- 1. frequency side -> M-point inverse column transforms over k1
        {
            constexpr int NU = EPT / RC1;
            C z[NU][RC1];
            int zt[NU], zk[NU], zj[NU];
#pragma unroll
            for (int i = 0; i < NU; i++) {
                const int u = tid + i * NT;
                zk[i] = u & (VEC - 1);
                const int rr = u >> LV;
                zj[i] = rr % RC2;
                zt[i] = rr / RC2;
#pragma unroll
                for (int r = 0; r < RC1; r++) z[i][r] = ldg(in + fstore_addr(zt[i], zk[i], zj[i] + RC2 * r));
            }
#pragma unroll
            for (int i = 0; i < NU; i++) dft<RC1, DIR, T>(z[i]);
            if constexpr (RC2 == 1) {
                // n1 = r: conj(w_N^{n1 k2}), then rows X[t][n1][k2]
#pragma unroll
                for (int i = 0; i < NU; i++)
#pragma unroll
                    for (int r = 0; r < RC1; r++)
                        S[Xi(zt[i], r, zk[i])] = twmul<true>(z[i][r], ldtw(Wg, r * VEC + zk[i]));
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
                    yk[i] = u & (VEC - 1);
                    const int rr = u >> LV;
                    yj[i] = rr % RC1;
                    yt[i] = rr / RC1;
#pragma unroll
                    for (int r = 0; r < RC2; r++) y[i][r] = S[Yi(yt[i], yk[i], yj[i] + RC1 * r)];
                }
                __syncthreads();
#pragma unroll
                for (int i = 0; i < NU2; i++) {
#pragma unroll
                    for (int r = 1; r < RC2; r++) y[i][r] = twmul<true>(y[i][r], stm[yj[i] * r]);
                    dft<RC2, DIR, T>(y[i]);
#pragma unroll
                    for (int r = 0; r < RC2; r++) {
                        const int n1 = yj[i] + RC1 * r;
                        S[Xi(yt[i], n1, yk[i])] = twmul<true>(y[i][r], ldtw(Wg, n1 * VEC + yk[i]));
                    }
                }
            }
        }
        __syncthreads();
        // ---- 2. VEC-point inverse row transforms over k2 -> rows X[t][n1][n2]
        {
            constexpr int NU = EPT / RA1;
            C v[NU][RA1];
            int ut[NU], un1[NU], uj[NU];
#pragma unroll
            for (int i = 0; i < NU; i++) {
                const int u = tid + i * NT;
                uj[i] = u & (RA2 - 1);
                const int rr = u / RA2;
                un1[i] = rr & (M - 1);
                ut[i] = rr >> LM;
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
                    wn1[i] = rr & (M - 1);
                    wt[i] = rr >> LM;
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
        // ---- 3. rows -> vector side (16-byte vectors), scale applied here
        {
#pragma unroll
            for (int i = 0; i < VPT; i++) {
                const int e = (tid + i * NT) * VE;
                const int t = e >> (LV + LM), r = e & (N - 1);
                const int64_t c = r >> logL, pos = r & (L - 1);
                uint4 v = *reinterpret_cast<const uint4 *>(&S[Xi(t, r >> LV, r & (VEC - 1))]);
                if (scl) {
                    C *cv = reinterpret_cast<C *>(&v);
#pragma unroll
                    for (int q = 0; q < VE; q++) {
                        const C o = cv[q];
                        cv[q] = {sre * o.x - sim * o.y, sre * o.y + sim * o.x};
                    }
                }
                *reinterpret_cast<uint4 *>(out + s_abase[t] + c * a0.a_chunk + pos) = v;
            }
        }
    }
}

template <typename T, int LV, int LM, int TL, int NT>
constexpr size_t fused_smem_bytes() {
    return sizeof(cpx<T>) * (size_t)TL * ((size_t)1 << (LV + LM)) +
           sizeof(tw<T>) * (((size_t)1 << LV) + ((size_t)1 << LM));
}

template <typename T, int LV, int LM, int TL, int NT>
cudaError_t launch_fused(const LineParams &prm, bool inv, cudaStream_t st) {
    constexpr size_t smem = fused_smem_bytes<T, LV, LM, TL, NT>();
    auto kern = inv ? fused_pass_kernel<T, LV, LM, TL, NT, true> : fused_pass_kernel<T, LV, LM, TL, NT, false>;
    static int attr_done[64][2];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && !attr_done[dev][inv]) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        attr_done[dev][inv] = 1;
    }
    const unsigned grid = (unsigned)(prm.nlines / TL);
    kern<<<grid, NT, smem, st>>>(prm);
    count_launch();
    return cudaGetLastError();
}

}  // namespace zm
