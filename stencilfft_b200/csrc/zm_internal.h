// zm_internal.h -- host-side declarations shared by the translation units of libzmodel_b200.
#pragma once

#include <cuda_runtime.h>

#include "zm_plan.h"

namespace zm {

// launch bookkeeping
void count_launch();
// radix schedule (remainder radix first, then rmax stages) of a power-of-two length
int radix_schedule(int64_t n, int rmax, int *rad);
int max_dyn_smem();
// record `code` with a formatted message as the calling thread's last error; returns code
int report_error(int code, const char *fmt, ...);

// zm_fft.cu
int ept_for(int dtype);
cudaError_t launch_line_pass(const LineParams &prm, int dtype, bool inv, cudaStream_t st);

// zm_fft2_<dtype>_<dir>.cu (generated by gen_fused.py): size-specialised fused passes.
// `handled` is false when (log2 VEC, log2 M, variant) has no specialisation;
// fused_variants_* gives the number of tile-shape variants (0 = none).
cudaError_t launch_fused_c64_fwd(const LineParams &prm, cudaStream_t st, bool *handled);
cudaError_t launch_fused_c64_inv(const LineParams &prm, cudaStream_t st, bool *handled);
cudaError_t launch_fused_c128_fwd(const LineParams &prm, cudaStream_t st, bool *handled);
cudaError_t launch_fused_c128_inv(const LineParams &prm, cudaStream_t st, bool *handled);
int fused_variants_c64(int logvec, int logm);
int fused_variants_c128(int logvec, int logm);
// log2 of the widest row interleave of the 2D intermediate variant `variant` of (VEC, M)
// supports (0 = none).
int fused_interleave_lg_c64(int logvec, int logm, int variant);
int fused_interleave_lg_c128(int logvec, int logm, int variant);
// 1 and the (x variant, y variant, log2 interleave, y-position interleave flag) of the
// out-of-place 2D forward configuration of (VEC, M), when there is one.
int fused_fwd_oop_c64(int logvec, int logm, int *vx, int *vy, int *lg, int *qint);
int fused_fwd_oop_c128(int logvec, int logm, int *vx, int *vy, int *lg, int *qint);
// the same for the out-of-place 2D inverse (y pass in -> work, x pass work -> out)
int fused_inv_oop_c64(int logvec, int logm, int *vx, int *vy, int *lg, int *qint);
int fused_inv_oop_c128(int logvec, int logm, int *vx, int *vy, int *lg, int *qint);

// zm_stencil.cu
enum StencilOp : int { ST_LAPLACE = 0, ST_DX = 1, ST_DY = 2, ST_ALL = 3 };
// ST_ALL (2D): Laplacian (coef) into out, dx / dy (coef2 = delta) into out2 / out3
cudaError_t launch_stencil(const zm_plan_s *p, int op, bool real_field, const void *in, void *out,
                           double coef, cudaStream_t st, void *out2 = nullptr, void *out3 = nullptr,
                           double coef2 = 1.0);

// zm_layout.cu
cudaError_t launch_convert(const zm_plan_s *p, bool reciprocal, bool to_natural, const void *in,
                           void *out, cudaStream_t st);
cudaError_t launch_spectral(const zm_plan_s *p, void *data, int op, double a, cudaStream_t st);
cudaError_t launch_fill(const zm_plan_s *p, void *data, int kind, uint64_t seed, cudaStream_t st);
cudaError_t launch_fill_modes(const zm_plan_s *p, void *data, int nmodes, const int64_t *modes,
                              const double *amps, double noise, uint64_t seed, cudaStream_t st);

}  // namespace zm
