// zm_fft.cu -- fused axis-pass kernels of the interleaved block-cyclic FFT.
//
// The reference runs one axis of its 2D/3D transform as six stages with a
// host-staged MPI All-to-All in the middle (zmodel/transforms/fft.cu:207-269):
//   FFT1a   VEC-point cuFFT over every packed vector           (plan0)
//   PACK    split each vector into P pieces of VP = VEC/P       (pack_forward_fft)
//   COMMS   MPI_Alltoall over the row / column communicator
//   UNPACK  gather into rows, times w_N^{n1 k2}                 (unpack_forward_fft)
//   FFT1b   M-point cuFFT at stride VP, one host call per row   (plan1)
//   REPACK  local transpose + vector re-packing                 (repack_transpose)
// Here every virtual rank lives in the same HBM, so one CTA takes T whole
// global lines (the N = VEC * M points one axis of the field has, spread over
// the P ranks of a row/column communicator), runs the same Cooley-Tukey split
// N = VEC * M on them in shared memory -- VEC-point transforms over n2, the
// twiddle w_N^{n1 k2}, M-point transforms over n1 -- and writes each frequency
// (k1, k2) straight to where the reference's REPACK (or final FFT1b) would put
// it.  The All-to-All becomes the address arithmetic of that store, so each
// axis pass reads and writes the field exactly once (2F bytes).
//
// Sub-transforms are Stockham radix-R stages (R = 2..16) done in place in
// shared memory: every thread loads its R-point butterflies into registers,
// the block synchronises, then every thread stores its results.
#include "zm_common.cuh"
#include "zm_internal.h"
#include "zm_lines.cuh"

namespace zm {

// ------------------------------------------------------------ Stockham stage
// One radix-R stage over all sub-transforms of length n held in shared memory.
//   COLM = false: sub-transform (t, n1) is the contiguous row s[t*N + n1*VEC + i]
//   COLM = true:  sub-transform (t, k2) is the column s[t*N + i*VEC + k2]
// DIR = -1 forward, +1 inverse.  PRETW multiplies the loaded inputs by the
// inter-step twiddle w_N^{n1 k2} (forward, COLM) or its conjugate (inverse, rows).
template <int R, int EPT, bool COLM, int DIR, bool PRETW, typename T>
ZM_DEV void stockham_stage(cpx<T> *s, const Geom &g, int n, int logn, int Ns, int nthr, int tid,
                           const tw<T> *twN) {
    constexpr int NB = EPT / R;
    constexpr bool CONJ = DIR > 0;
    cpx<T> v[NB][R];
    int base[NB], jv[NB];
    const int nR = n / R;
    const int logR = (R == 2) ? 1 : (R == 4) ? 2 : (R == 8) ? 3 : 4;
    const int lognR = logn - logR;
    const int str = COLM ? (int)g.vec : 1;
#pragma unroll
    for (int u = 0; u < NB; u++) {
        const int sig = tid + u * nthr;
        int j, bb, tagn;  // tagn: the sub-transform's n1 (rows) or k2 (columns)
        if (!COLM) {
            j = sig & (nR - 1);
            const int b = sig >> lognR;              // b = t*M + n1
            bb = b << g.logVEC;
            tagn = b & (int)(g.m - 1);
        } else {
            const int k2 = sig & (int)(g.vec - 1);
            const int rest = sig >> g.logVEC;
            j = rest & (nR - 1);
            const int t = rest >> lognR;
            bb = (t << g.logN) + k2;
            tagn = k2;
        }
        base[u] = bb;
        jv[u] = j;
#pragma unroll
        for (int r = 0; r < R; r++) {
            const int i = j + r * nR;
            cpx<T> x = s[bb + i * str];
            if (PRETW) x = twmul<CONJ>(x, ldtw(twN, (int64_t)i * tagn));
            v[u][r] = x;
        }
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < NB; u++) {
        const int j = jv[u];
        const int k = j & (Ns - 1);
        if (Ns > 1) {
            // w_{Ns R}^{k r} = w_N^{k r N / (Ns R)}
            const int sh = g.logN - logn + (logn - __ffs(Ns * R) + 1);
#pragma unroll
            for (int r = 1; r < R; r++)
                v[u][r] = twmul<CONJ>(v[u][r], ldtw(twN, ((int64_t)k * r) << sh));
        }
        dft<R, DIR, T>(v[u]);
        const int idxD = (j - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; r++) s[base[u] + (idxD + r * Ns) * str] = v[u][r];
    }
    __syncthreads();
}

template <int EPT, bool COLM, int DIR, typename T>
ZM_DEV void run_subfft(cpx<T> *s, const Geom &g, int n, int logn, const int *rad, int nst,
                       bool pretw, int nthr, int tid, const tw<T> *twN) {
    int Ns = 1;
    for (int st = 0; st < nst; st++) {
        const int R = rad[st];
        const bool pre = pretw && st == 0;
#define ZM_STAGE(RR)                                                                               \
    if (pre) stockham_stage<RR, EPT, COLM, DIR, true, T>(s, g, n, logn, Ns, nthr, tid, twN);      \
    else stockham_stage<RR, EPT, COLM, DIR, false, T>(s, g, n, logn, Ns, nthr, tid, twN);
        if (R == 2) { ZM_STAGE(2) }
        else if (R == 4) { ZM_STAGE(4) }
        else if (R == 8) { ZM_STAGE(8) }
        else {
            if constexpr (EPT >= 16) { ZM_STAGE(16) }
        }
#undef ZM_STAGE
        Ns *= R;
    }
}

// ------------------------------------------------------------------ kernel
template <typename T, int EPT, bool INV>
__global__ void __launch_bounds__(1024) line_fft_kernel(const LineParams prm) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpx<T> *s = reinterpret_cast<cpx<T> *>(smem_raw);
    __shared__ int64_t s_abase[64], s_fbase[64];
    const Geom &g = prm.g;
    const int nthr = blockDim.x, tid = threadIdx.x;
    const int TL = prm.T;
    const int logT = __ffs(TL) - 1;
    const int64_t l0 = (int64_t)blockIdx.x * TL;
    const int64_t N = g.n, L = g.L;
    const cpx<T> *in = reinterpret_cast<const cpx<T> *>(prm.in);
    cpx<T> *out = reinterpret_cast<cpx<T> *>(prm.out);
    const tw<T> *twN = reinterpret_cast<const tw<T> *>(prm.twN);

    const LineAddr a0 = line_addr(g, prm.kind, l0);
    for (int t = tid; t < TL; t += nthr) {
        const LineAddr a = line_addr(g, prm.kind, l0 + t);
        s_abase[t] = a.a_base;
        s_fbase[t] = a.f_base;
    }
    __syncthreads();
    const int tot = TL << g.logN;
    const bool f_contig = a0.f_pos == 1;

    // ---------------------------------------------------------------- load
    if (!INV) {
        // vector side: line t, chunk c, position pos -> s[t][c*L + pos] = s[t][n1*VEC + n2]
        for (int e = tid; e < tot; e += nthr) {
            const int t = e >> g.logN;
            const int r = e & (int)(N - 1);
            const int c = r >> g.logL, pos = r & (int)(L - 1);
            s[e] = ldg(in + s_abase[t] + c * a0.a_chunk + pos);
        }
    } else {
        // frequency side: (t, c, pos = k1*VP + f) -> s[t][k1*VEC + c*VP + f]
        for (int e = tid; e < tot; e += nthr) {
            int t, c, pos;
            if (f_contig) {
                t = e >> g.logN;
                const int r = e & (int)(N - 1);
                c = r >> g.logL; pos = r & (int)(L - 1);
            } else {
                t = e & (TL - 1);
                const int cp = e >> logT;
                c = cp >> g.logL; pos = cp & (int)(L - 1);
            }
            const int k1 = pos >> g.logVP, f = pos & (int)(g.vp - 1);
            const int si = (t << g.logN) + (k1 << g.logVEC) + (c << g.logVP) + f;
            s[si] = ldg(in + s_fbase[t] + c * a0.f_chunk + pos * a0.f_pos);
        }
    }
    __syncthreads();

    // ------------------------------------------------------------- compute
    if (!prm.permute_only) {
        if (!INV) {
            run_subfft<EPT, false, -1, T>(s, g, (int)g.vec, g.logVEC, prm.rad_vec, prm.nst_vec, false,
                                          nthr, tid, twN);
            run_subfft<EPT, true, -1, T>(s, g, (int)g.m, g.logM, prm.rad_m, prm.nst_m, true, nthr,
                                         tid, twN);
        } else {
            run_subfft<EPT, true, 1, T>(s, g, (int)g.m, g.logM, prm.rad_m, prm.nst_m, false, nthr,
                                        tid, twN);
            run_subfft<EPT, false, 1, T>(s, g, (int)g.vec, g.logVEC, prm.rad_vec, prm.nst_vec, true,
                                         nthr, tid, twN);
        }
    }

    // --------------------------------------------------------------- store
    const bool scl = prm.apply_scale && !prm.permute_only;
    const T sr = (T)prm.scale_re, si_ = (T)prm.scale_im;
    if (!INV) {
        for (int e = tid; e < tot; e += nthr) {
            int t, c, pos;
            if (f_contig) {
                t = e >> g.logN;
                const int r = e & (int)(N - 1);
                c = r >> g.logL; pos = r & (int)(L - 1);
            } else {
                t = e & (TL - 1);
                const int cp = e >> logT;
                c = cp >> g.logL; pos = cp & (int)(L - 1);
            }
            const int k1 = pos >> g.logVP, f = pos & (int)(g.vp - 1);
            cpx<T> v = s[(t << g.logN) + (k1 << g.logVEC) + (c << g.logVP) + f];
            if (scl) v = {v.x * sr - v.y * si_, v.x * si_ + v.y * sr};
            out[s_fbase[t] + c * a0.f_chunk + pos * a0.f_pos] = v;
        }
    } else {
        for (int e = tid; e < tot; e += nthr) {
            const int t = e >> g.logN;
            const int r = e & (int)(N - 1);
            const int c = r >> g.logL, pos = r & (int)(L - 1);
            cpx<T> v = s[e];
            if (scl) v = {sr * v.x - si_ * v.y, sr * v.y + si_ * v.x};
            out[s_abase[t] + c * a0.a_chunk + pos] = v;
        }
    }
}

// ------------------------------------------------------------------ launch
template <typename T, int EPT, bool INV>
static cudaError_t launch_typed(const LineParams &prm, int threads, size_t smem, cudaStream_t st) {
    auto kern = line_fft_kernel<T, EPT, INV>;
    static bool attr_done[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && !attr_done[dev]) {
        // the opt-in limit covers static + dynamic shared memory
        cudaFuncAttributes fa;
        cudaError_t e = cudaFuncGetAttributes(&fa, kern);
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 max_dyn_smem() - (int)fa.sharedSizeBytes);
        if (e != cudaSuccess) return e;
        attr_done[dev] = true;
    }
    const unsigned grid = (unsigned)(prm.nlines / prm.T);
    kern<<<grid, threads, smem, st>>>(prm);
    count_launch();
    return cudaGetLastError();
}

int ept_for(int dtype) { return dtype == 0 ? 8 : 16; }

cudaError_t launch_line_pass(const LineParams &prm, int dtype, bool inv, cudaStream_t st) {
    if (!prm.permute_only && prm.twd) {
        bool handled = false;
        cudaError_t e;
        if (dtype == 0) e = inv ? launch_fused_c128_inv(prm, st, &handled) : launch_fused_c128_fwd(prm, st, &handled);
        else e = inv ? launch_fused_c64_inv(prm, st, &handled) : launch_fused_c64_fwd(prm, st, &handled);
        if (handled) return e;
    }
    // the runtime-sized kernel reads and writes only the plain REPACK intermediate
    if (prm.lg_inter != 0) return cudaErrorInvalidValue;
    const int ept = ept_for(dtype);
    const int threads = (int)((prm.T * prm.g.n) / ept);
    const size_t smem = (size_t)prm.T * prm.g.n * (dtype == 0 ? 16 : 8);
    if (dtype == 0) {
        return inv ? launch_typed<double, 8, true>(prm, threads, smem, st)
                   : launch_typed<double, 8, false>(prm, threads, smem, st);
    }
    return inv ? launch_typed<float, 16, true>(prm, threads, smem, st)
               : launch_typed<float, 16, false>(prm, threads, smem, st);
}

}  // namespace zm
