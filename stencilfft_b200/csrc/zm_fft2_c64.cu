// zm_fft2_c64.cu -- size-specialised fused axis passes, float (complex64).
// Each (log2 VEC, log2 M) pair below runs zm_fft2.cuh's fused_pass_kernel; other sizes
// fall back to the runtime-sized kernel of zm_fft.cu.
#include "zm_internal.h"
#include "zm_lines.cuh"
#include "zm_fft2.cuh"

namespace zm {

cudaError_t launch_fused_c64(const LineParams &prm, bool inv, cudaStream_t st, bool *handled) {
    *handled = true;
    switch ((prm.g.logVEC << 8) | prm.g.logM) {
    case (4 << 8) | 4: return launch_fused<float, 4, 4, 32, 512>(prm, inv, st);
    case (4 << 8) | 5: return launch_fused<float, 4, 5, 16, 512>(prm, inv, st);
    case (4 << 8) | 6: return launch_fused<float, 4, 6, 8, 512>(prm, inv, st);
    case (2 << 8) | 7: return launch_fused<float, 2, 7, 16, 512>(prm, inv, st);
    case (5 << 8) | 7: return launch_fused<float, 5, 7, 2, 512>(prm, inv, st);
    case (5 << 8) | 6: return launch_fused<float, 5, 6, 4, 512>(prm, inv, st);
    case (4 << 8) | 8: return launch_fused<float, 4, 8, 2, 512>(prm, inv, st);
    case (5 << 8) | 8: return launch_fused<float, 5, 8, 1, 512>(prm, inv, st);
    case (6 << 8) | 8: return launch_fused<float, 6, 8, 1, 1024>(prm, inv, st);
    default: break;
    }
    *handled = false;
    return cudaSuccess;
}

int fused_lines_c64(int logvec, int logm) {
    switch ((logvec << 8) | logm) {
    case (4 << 8) | 4: return 32;
    case (4 << 8) | 5: return 16;
    case (4 << 8) | 6: return 8;
    case (2 << 8) | 7: return 16;
    case (5 << 8) | 7: return 2;
    case (5 << 8) | 6: return 4;
    case (4 << 8) | 8: return 2;
    case (5 << 8) | 8: return 1;
    case (6 << 8) | 8: return 1;
    default: return 0;
    }
}

}  // namespace zm
