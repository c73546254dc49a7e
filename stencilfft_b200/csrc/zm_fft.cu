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
// shared memory (zm_tile.cuh): every thread loads its R-point butterflies into
// registers, the block synchronises, then every thread stores its results.
#include "zm_common.cuh"
#include "zm_internal.h"
#include "zm_tile.cuh"

namespace zm {

// ------------------------------------------------------------------ kernel
template <typename T, int EPT, bool INV>
__global__ void __launch_bounds__(1024) line_fft_kernel(const LineParams prm) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpx<T> *s = reinterpret_cast<cpx<T> *>(smem_raw);
    __shared__ int64_t s_abase[64], s_fbase[64];
    const Geom &g = prm.g;
    const int nthr = blockDim.x, tid = threadIdx.x;
    const cpx<T> *in = reinterpret_cast<const cpx<T> *>(prm.in);
    cpx<T> *out = reinterpret_cast<cpx<T> *>(prm.out);
    const tw<T> *twN = reinterpret_cast<const tw<T> *>(prm.twN);
    const Tile c = tile_begin(g, prm.kind, (int64_t)blockIdx.x * prm.T, prm.T, s_abase, s_fbase, nthr, tid);
    __syncthreads();
    if (!INV) tile_load_vec<EPT>(c, g, s, in, nthr, tid);
    else tile_load_freq<EPT>(c, g, s, in, nthr, tid);
    __syncthreads();
    if (!prm.permute_only)
        tile_transform<T, EPT, INV>(s, g, prm.rad_vec, prm.nst_vec, prm.rad_m, prm.nst_m, nthr, tid, twN);
    const bool scl = prm.apply_scale && !prm.permute_only;
    const T sr = (T)prm.scale_re, si = (T)prm.scale_im;
    if (!INV) tile_store_freq<EPT>(c, g, s, out, scl, sr, si, nthr, tid);
    else tile_store_vec<EPT>(c, g, s, out, scl, sr, si, nthr, tid);
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
    if (prm.lg_inter != 0 || prm.inter_q) return cudaErrorInvalidValue;
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
