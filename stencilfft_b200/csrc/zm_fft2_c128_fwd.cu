// zm_fft2_c128_fwd.cu -- generated by gen_fused.py: size-specialised fused axis passes,
// c128, forward direction (kernel template in zm_fft2.cuh).
#include "zm_internal.h"
#include "zm_lines.cuh"
#include "zm_fft2.cuh"
#include "zm_fft3.cuh"

namespace zm {

cudaError_t launch_fused_c128_fwd(const LineParams &prm, cudaStream_t st, bool *handled) {
    *handled = true;
    switch ((prm.g.logVEC << 16) | (prm.g.logM << 8) | prm.variant) {
    case (4 << 16) | (4 << 8) | 0: return launch_fused<double, 4, 4, 1, 16, 256, false, false>(prm, st);
    case (4 << 16) | (5 << 8) | 0: return launch_fused<double, 4, 5, 1, 8, 256, false, false>(prm, st);
    case (4 << 16) | (6 << 8) | 0: return launch_fused<double, 4, 6, 1, 4, 256, false, false>(prm, st);
    case (2 << 16) | (7 << 8) | 0: return launch_fused<double, 2, 7, 1, 8, 256, false, false>(prm, st);
    case (2 << 16) | (7 << 8) | 1: return launch_fused<double, 2, 7, 1, 4, 128, false, false>(prm, st);
    case (2 << 16) | (7 << 8) | 2: return launch_fused<double, 2, 7, 1, 16, 512, false, false>(prm, st);
    case (5 << 16) | (6 << 8) | 0: return launch_fused<double, 5, 6, 1, 2, 256, false, false>(prm, st);
    case (5 << 16) | (7 << 8) | 0: return launch_fused<double, 5, 7, 1, 1, 256, false, false>(prm, st);
    case (5 << 16) | (7 << 8) | 1: return launch_fused<double, 5, 7, 2, 2, 256, false, false>(prm, st);
    case (4 << 16) | (8 << 8) | 0: return launch_fused<double, 4, 8, 1, 1, 256, false, false>(prm, st);
    case (4 << 16) | (8 << 8) | 1: return launch_fused<double, 4, 8, 2, 2, 256, false, false>(prm, st);
    case (5 << 16) | (8 << 8) | 0: return launch_fused<double, 5, 8, 1, 1, 512, false, false>(prm, st);
    case (5 << 16) | (8 << 8) | 1: return launch_fused<double, 5, 8, 2, 1, 256, false, false>(prm, st);
    case (6 << 16) | (7 << 8) | 0: return launch_fused<double, 6, 7, 2, 1, 256, false, false>(prm, st);
    case (6 << 16) | (7 << 8) | 1: return launch_fused<double, 6, 7, 1, 1, 512, false, false>(prm, st);
    case (6 << 16) | (8 << 8) | 0: return launch_fused<double, 6, 8, 2, 1, 512, false, false>(prm, st);
    case (6 << 16) | (8 << 8) | 1: return launch_fused<double, 6, 8, 4, 1, 256, false, false>(prm, st);
    case (6 << 16) | (8 << 8) | 2: return launch_fused<double, 6, 8, 4, 2, 512, false, false>(prm, st);
    case (6 << 16) | (8 << 8) | 3: return launch_fused<double, 6, 8, 2, 1, 512, false, false, true>(prm, st);
    case (6 << 16) | (8 << 8) | 4: return launch_fused<double, 6, 8, 4, 2, 512, false, false, true>(prm, st);
    default: break;
    }
    *handled = false;
    return cudaSuccess;
}

int fused_variants_c128(int logvec, int logm) {
    switch ((logvec << 8) | logm) {
    case (4 << 8) | 4: return 1;
    case (4 << 8) | 5: return 1;
    case (4 << 8) | 6: return 1;
    case (2 << 8) | 7: return 3;
    case (5 << 8) | 6: return 1;
    case (5 << 8) | 7: return 2;
    case (4 << 8) | 8: return 2;
    case (5 << 8) | 8: return 2;
    case (6 << 8) | 7: return 2;
    case (6 << 8) | 8: return 5;
    default: return 0;
    }
}

int fused_interleave_lg_c128(int logvec, int logm, int variant) {
    switch ((logvec << 16) | (logm << 8) | variant) {
    case (5 << 16) | (6 << 8) | 0: return 1;
    case (5 << 16) | (7 << 8) | 1: return 1;
    case (6 << 16) | (8 << 8) | 2: return 1;
    case (6 << 16) | (8 << 8) | 4: return 1;
    default: return 0;
    }
}

int fused_fwd_oop_c128(int logvec, int logm, int *vx, int *vy, int *lg, int *qint) {
    switch ((logvec << 8) | logm) {
    case (6 << 8) | 8: *vx = 0; *vy = 3; *lg = 4; *qint = 0; return 1;
    default: return 0;
    }
}

int fused_inv_oop_c128(int logvec, int logm, int *vx, int *vy, int *lg, int *qint) {
    switch ((logvec << 8) | logm) {
    case (6 << 8) | 8: *vx = 3; *vy = 3; *lg = 0; *qint = 0; return 1;
    default: return 0;
    }
}

}  // namespace zm
