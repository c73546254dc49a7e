// zm_fft2_c64_fwd.cu -- generated by gen_fused.py: size-specialised fused axis passes,
// c64, forward direction (kernel template in zm_fft2.cuh).
#include "zm_internal.h"
#include "zm_lines.cuh"
#include "zm_fft2.cuh"
#include "zm_fft3.cuh"

namespace zm {

cudaError_t launch_fused_c64_fwd(const LineParams &prm, cudaStream_t st, bool *handled) {
    *handled = true;
    switch ((prm.g.logVEC << 16) | (prm.g.logM << 8) | prm.variant) {
    case (4 << 16) | (4 << 8) | 0: return launch_fused<float, 4, 4, 1, 32, 512, false, false>(prm, st);
    case (4 << 16) | (5 << 8) | 0: return launch_fused<float, 4, 5, 1, 16, 512, false, false>(prm, st);
    case (4 << 16) | (6 << 8) | 0: return launch_fused<float, 4, 6, 1, 8, 512, false, false>(prm, st);
    case (4 << 16) | (6 << 8) | 1: return launch_fused<float, 4, 6, 1, 4, 256, false, false>(prm, st);
    case (2 << 16) | (7 << 8) | 0: return launch_fused<float, 2, 7, 1, 8, 256, false, false>(prm, st);
    case (2 << 16) | (7 << 8) | 1: return launch_fused<float, 2, 7, 1, 16, 512, false, false>(prm, st);
    case (2 << 16) | (7 << 8) | 2: return launch_fused<float, 2, 7, 1, 32, 1024, false, false>(prm, st);
    case (2 << 16) | (7 << 8) | 3: return launch_fused<float, 2, 7, 1, 4, 128, false, false>(prm, st);
    case (5 << 16) | (6 << 8) | 0: return launch_fused<float, 5, 6, 1, 4, 512, false, false>(prm, st);
    case (5 << 16) | (7 << 8) | 0: return launch_fused<float, 5, 7, 1, 2, 512, false, false>(prm, st);
    case (5 << 16) | (7 << 8) | 1: return launch_fused<float, 5, 7, 2, 2, 256, false, false>(prm, st);
    case (5 << 16) | (7 << 8) | 2: return launch_fused<float, 5, 7, 2, 4, 512, false, false>(prm, st);
    case (5 << 16) | (7 << 8) | 3: return launch_fused<float, 5, 7, 1, 1, 256, false, false>(prm, st);
    case (5 << 16) | (7 << 8) | 4: return launch_fused<float, 5, 7, 1, 4, 1024, false, false>(prm, st);
    case (4 << 16) | (8 << 8) | 0: return launch_fused<float, 4, 8, 1, 2, 512, false, false>(prm, st);
    case (4 << 16) | (8 << 8) | 1: return launch_fused<float, 4, 8, 2, 4, 512, false, false>(prm, st);
    case (4 << 16) | (8 << 8) | 2: return launch_fused<float, 4, 8, 1, 1, 256, false, false>(prm, st);
    case (4 << 16) | (8 << 8) | 3: return launch_fused<float, 4, 8, 1, 4, 1024, false, false>(prm, st);
    case (5 << 16) | (8 << 8) | 0: return launch_fused<float, 5, 8, 2, 2, 512, false, false>(prm, st);
    case (5 << 16) | (8 << 8) | 1: return launch_fused<float, 5, 8, 1, 1, 512, false, false>(prm, st);
    case (5 << 16) | (8 << 8) | 2: return launch_fused<float, 5, 8, 2, 1, 256, false, false>(prm, st);
    case (5 << 16) | (8 << 8) | 3: return launch_fused<float, 5, 8, 4, 4, 512, false, false>(prm, st);
    case (5 << 16) | (8 << 8) | 4: return launch_fused<float, 5, 8, 2, 4, 1024, false, false>(prm, st);
    case (5 << 16) | (8 << 8) | 5: return launch_fused<float, 5, 8, 1, 2, 1024, false, false>(prm, st);
    case (6 << 16) | (7 << 8) | 0: return launch_fused<float, 6, 7, 2, 2, 512, false, false>(prm, st);
    case (6 << 16) | (7 << 8) | 1: return launch_fused<float, 6, 7, 1, 1, 512, false, false>(prm, st);
    case (6 << 16) | (7 << 8) | 2: return launch_fused<float, 6, 7, 1, 2, 1024, false, false>(prm, st);
    case (6 << 16) | (8 << 8) | 0: return launch_fused<float, 6, 8, 4, 2, 512, false, false>(prm, st);
    case (6 << 16) | (8 << 8) | 1: return launch_fused<float, 6, 8, 2, 1, 512, false, false>(prm, st);
    case (6 << 16) | (8 << 8) | 2: return launch_fused<float, 6, 8, 1, 1, 1024, false, false>(prm, st);
    case (6 << 16) | (8 << 8) | 3: return launch_fused<float, 6, 8, 8, 4, 512, false, false>(prm, st);
    case (6 << 16) | (8 << 8) | 4: return launch_fused<float, 6, 8, 4, 4, 1024, false, false>(prm, st);
    case (6 << 16) | (8 << 8) | 5: return launch_fused<float, 6, 8, 4, 2, 512, false, true>(prm, st);
    case (6 << 16) | (8 << 8) | 6: return launch_k3<6, 8, false, false, false>(prm, st);
    case (6 << 16) | (8 << 8) | 7: return launch_k3<6, 8, false, true, false>(prm, st);
    case (6 << 16) | (8 << 8) | 8: return launch_k3<6, 8, false, false, true>(prm, st);
    default: break;
    }
    *handled = false;
    return cudaSuccess;
}

int fused_variants_c64(int logvec, int logm) {
    switch ((logvec << 8) | logm) {
    case (4 << 8) | 4: return 1;
    case (4 << 8) | 5: return 1;
    case (4 << 8) | 6: return 2;
    case (2 << 8) | 7: return 4;
    case (5 << 8) | 6: return 1;
    case (5 << 8) | 7: return 5;
    case (4 << 8) | 8: return 4;
    case (5 << 8) | 8: return 6;
    case (6 << 8) | 7: return 3;
    case (6 << 8) | 8: return 9;
    default: return 0;
    }
}

int fused_interleave_lg_c64(int logvec, int logm, int variant) {
    switch ((logvec << 16) | (logm << 8) | variant) {
    case (5 << 16) | (6 << 8) | 0: return 2;
    case (5 << 16) | (7 << 8) | 0: return 1;
    case (5 << 16) | (7 << 8) | 1: return 1;
    case (5 << 16) | (7 << 8) | 2: return 2;
    case (5 << 16) | (7 << 8) | 4: return 2;
    case (5 << 16) | (8 << 8) | 0: return 1;
    case (5 << 16) | (8 << 8) | 3: return 2;
    case (5 << 16) | (8 << 8) | 4: return 2;
    case (5 << 16) | (8 << 8) | 5: return 1;
    case (6 << 16) | (7 << 8) | 0: return 1;
    case (6 << 16) | (7 << 8) | 2: return 1;
    case (6 << 16) | (8 << 8) | 0: return 1;
    case (6 << 16) | (8 << 8) | 3: return 2;
    case (6 << 16) | (8 << 8) | 4: return 2;
    case (6 << 16) | (8 << 8) | 5: return 1;
    default: return 0;
    }
}

int fused_fwd_oop_c64(int logvec, int logm, int *vx, int *vy, int *lg, int *qint) {
    switch ((logvec << 8) | logm) {
    case (6 << 8) | 8: *vx = 7; *vy = 8; *lg = 3; *qint = 0; return 1;
    case (5 << 8) | 8: *vx = 5; *vy = 5; *lg = 1; *qint = 0; return 1;
    case (6 << 8) | 7: *vx = 2; *vy = 2; *lg = 1; *qint = 0; return 1;
    default: return 0;
    }
}

int fused_inv_oop_c64(int logvec, int logm, int *vx, int *vy, int *lg, int *qint) {
    switch ((logvec << 8) | logm) {
    case (6 << 8) | 8: *vx = 7; *vy = 7; *lg = 2; *qint = 1; return 1;
    default: return 0;
    }
}

}  // namespace zm
