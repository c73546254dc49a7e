// zm_fft2_c128_inv.cu -- generated by gen_fused.py: size-specialised fused axis passes,
// c128, inverse direction (kernel template in zm_fft2.cuh).
#include "zm_internal.h"
#include "zm_lines.cuh"
#include "zm_fft2.cuh"
#include "zm_fft3.cuh"

namespace zm {

cudaError_t launch_fused_c128_inv(const LineParams &prm, cudaStream_t st, bool *handled) {
    *handled = true;
    switch ((prm.g.logVEC << 16) | (prm.g.logM << 8) | prm.variant) {
    case (4 << 16) | (4 << 8) | 0: return launch_fused<double, 4, 4, 1, 16, 256, true, false>(prm, st);
    case (4 << 16) | (5 << 8) | 0: return launch_fused<double, 4, 5, 1, 8, 256, true, false>(prm, st);
    case (4 << 16) | (6 << 8) | 0: return launch_fused<double, 4, 6, 1, 4, 256, true, false>(prm, st);
    case (2 << 16) | (7 << 8) | 0: return launch_fused<double, 2, 7, 1, 8, 256, true, false>(prm, st);
    case (2 << 16) | (7 << 8) | 1: return launch_fused<double, 2, 7, 1, 4, 128, true, false>(prm, st);
    case (2 << 16) | (7 << 8) | 2: return launch_fused<double, 2, 7, 1, 16, 512, true, false>(prm, st);
    case (5 << 16) | (6 << 8) | 0: return launch_fused<double, 5, 6, 1, 2, 256, true, false>(prm, st);
    case (5 << 16) | (7 << 8) | 0: return launch_fused<double, 5, 7, 1, 1, 256, true, false>(prm, st);
    case (5 << 16) | (7 << 8) | 1: return launch_fused<double, 5, 7, 2, 2, 256, true, false>(prm, st);
    case (4 << 16) | (8 << 8) | 0: return launch_fused<double, 4, 8, 1, 1, 256, true, false>(prm, st);
    case (4 << 16) | (8 << 8) | 1: return launch_fused<double, 4, 8, 2, 2, 256, true, false>(prm, st);
    case (5 << 16) | (8 << 8) | 0: return launch_fused<double, 5, 8, 1, 1, 512, true, false>(prm, st);
    case (5 << 16) | (8 << 8) | 1: return launch_fused<double, 5, 8, 2, 1, 256, true, false>(prm, st);
    case (6 << 16) | (7 << 8) | 0: return launch_fused<double, 6, 7, 2, 1, 256, true, false>(prm, st);
    case (6 << 16) | (7 << 8) | 1: return launch_fused<double, 6, 7, 1, 1, 512, true, false>(prm, st);
    case (6 << 16) | (8 << 8) | 0: return launch_fused<double, 6, 8, 2, 1, 512, true, false>(prm, st);
    case (6 << 16) | (8 << 8) | 1: return launch_fused<double, 6, 8, 4, 1, 256, true, false>(prm, st);
    case (6 << 16) | (8 << 8) | 2: return launch_fused<double, 6, 8, 4, 2, 512, true, false>(prm, st);
    case (6 << 16) | (8 << 8) | 3: return launch_fused<double, 6, 8, 2, 1, 512, true, false, true>(prm, st);
    case (6 << 16) | (8 << 8) | 4: return launch_fused<double, 6, 8, 4, 2, 512, true, false, true>(prm, st);
    default: break;
    }
    *handled = false;
    return cudaSuccess;
}

}  // namespace zm
