// zm_fft2_c64_inv.cu -- generated by gen_fused.py: size-specialised fused axis passes,
// c64, inverse direction (kernel template in zm_fft2.cuh).
#include "zm_internal.h"
#include "zm_lines.cuh"
#include "zm_fft2.cuh"
#include "zm_fft3.cuh"

namespace zm {

cudaError_t launch_fused_c64_inv(const LineParams &prm, cudaStream_t st, bool *handled) {
    *handled = true;
    switch ((prm.g.logVEC << 16) | (prm.g.logM << 8) | prm.variant) {
    case (4 << 16) | (4 << 8) | 0: return launch_fused<float, 4, 4, 1, 32, 512, true, false>(prm, st);
    case (4 << 16) | (5 << 8) | 0: return launch_fused<float, 4, 5, 1, 16, 512, true, false>(prm, st);
    case (4 << 16) | (6 << 8) | 0: return launch_fused<float, 4, 6, 1, 8, 512, true, false>(prm, st);
    case (4 << 16) | (6 << 8) | 1: return launch_fused<float, 4, 6, 1, 4, 256, true, false>(prm, st);
    case (2 << 16) | (7 << 8) | 0: return launch_fused<float, 2, 7, 1, 8, 256, true, false>(prm, st);
    case (2 << 16) | (7 << 8) | 1: return launch_fused<float, 2, 7, 1, 16, 512, true, false>(prm, st);
    case (2 << 16) | (7 << 8) | 2: return launch_fused<float, 2, 7, 1, 32, 1024, true, false>(prm, st);
    case (2 << 16) | (7 << 8) | 3: return launch_fused<float, 2, 7, 1, 4, 128, true, false>(prm, st);
    case (5 << 16) | (6 << 8) | 0: return launch_fused<float, 5, 6, 1, 4, 512, true, false>(prm, st);
    case (5 << 16) | (7 << 8) | 0: return launch_fused<float, 5, 7, 1, 2, 512, true, false>(prm, st);
    case (5 << 16) | (7 << 8) | 1: return launch_fused<float, 5, 7, 2, 2, 256, true, false>(prm, st);
    case (5 << 16) | (7 << 8) | 2: return launch_fused<float, 5, 7, 2, 4, 512, true, false>(prm, st);
    case (5 << 16) | (7 << 8) | 3: return launch_fused<float, 5, 7, 1, 1, 256, true, false>(prm, st);
    case (5 << 16) | (7 << 8) | 4: return launch_fused<float, 5, 7, 1, 4, 1024, true, false>(prm, st);
    case (4 << 16) | (8 << 8) | 0: return launch_fused<float, 4, 8, 1, 2, 512, true, false>(prm, st);
    case (4 << 16) | (8 << 8) | 1: return launch_fused<float, 4, 8, 2, 4, 512, true, false>(prm, st);
    case (4 << 16) | (8 << 8) | 2: return launch_fused<float, 4, 8, 1, 1, 256, true, false>(prm, st);
    case (4 << 16) | (8 << 8) | 3: return launch_fused<float, 4, 8, 1, 4, 1024, true, false>(prm, st);
    case (5 << 16) | (8 << 8) | 0: return launch_fused<float, 5, 8, 2, 2, 512, true, false>(prm, st);
    case (5 << 16) | (8 << 8) | 1: return launch_fused<float, 5, 8, 1, 1, 512, true, false>(prm, st);
    case (5 << 16) | (8 << 8) | 2: return launch_fused<float, 5, 8, 2, 1, 256, true, false>(prm, st);
    case (5 << 16) | (8 << 8) | 3: return launch_fused<float, 5, 8, 4, 4, 512, true, false>(prm, st);
    case (5 << 16) | (8 << 8) | 4: return launch_fused<float, 5, 8, 2, 4, 1024, true, false>(prm, st);
    case (5 << 16) | (8 << 8) | 5: return launch_fused<float, 5, 8, 1, 2, 1024, true, false>(prm, st);
    case (6 << 16) | (7 << 8) | 0: return launch_fused<float, 6, 7, 2, 2, 512, true, false>(prm, st);
    case (6 << 16) | (7 << 8) | 1: return launch_fused<float, 6, 7, 1, 1, 512, true, false>(prm, st);
    case (6 << 16) | (7 << 8) | 2: return launch_fused<float, 6, 7, 1, 2, 1024, true, false>(prm, st);
    case (6 << 16) | (8 << 8) | 0: return launch_fused<float, 6, 8, 4, 2, 512, true, false>(prm, st);
    case (6 << 16) | (8 << 8) | 1: return launch_fused<float, 6, 8, 2, 1, 512, true, false>(prm, st);
    case (6 << 16) | (8 << 8) | 2: return launch_fused<float, 6, 8, 1, 1, 1024, true, false>(prm, st);
    case (6 << 16) | (8 << 8) | 3: return launch_fused<float, 6, 8, 8, 4, 512, true, false>(prm, st);
    case (6 << 16) | (8 << 8) | 4: return launch_fused<float, 6, 8, 4, 4, 1024, true, false>(prm, st);
    case (6 << 16) | (8 << 8) | 5: return launch_fused<float, 6, 8, 4, 2, 512, true, true>(prm, st);
    case (6 << 16) | (8 << 8) | 6: return launch_k3<6, 8, true, false, false>(prm, st);
    case (6 << 16) | (8 << 8) | 7: return launch_k3<6, 8, true, true, false>(prm, st);
    case (6 << 16) | (8 << 8) | 8: return launch_k3<6, 8, true, false, true>(prm, st);
    default: break;
    }
    *handled = false;
    return cudaSuccess;
}

}  // namespace zm
