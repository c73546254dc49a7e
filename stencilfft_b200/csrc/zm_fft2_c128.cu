// zm_fft2_c128.cu -- size-specialised fused axis passes, double (complex128).
// Each (log2 VEC, log2 M) pair below runs zm_fft2.cuh's fused_pass_kernel; other sizes
// fall back to the runtime-sized kernel of zm_fft.cu.
#include "zm_internal.h"
#include "zm_lines.cuh"
#include "zm_fft2.cuh"

namespace zm {

cudaError_t launch_fused_c128(const LineParams &prm, bool inv, cudaStream_t st, bool *handled) {
    *handled = true;
    switch ((prm.g.logVEC << 8) | prm.g.logM) {
    case (4 << 8) | 4: return launch_fused<double, 4, 4, 16, 256>(prm, inv, st);
    case (4 << 8) | 5: return launch_fused<double, 4, 5, 8, 256>(prm, inv, st);
    case (4 << 8) | 6: return launch_fused<double, 4, 6, 4, 256>(prm, inv, st);
    case (2 << 8) | 7: return launch_fused<double, 2, 7, 8, 256>(prm, inv, st);
    case (5 << 8) | 7: return launch_fused<double, 5, 7, 1, 256>(prm, inv, st);
    case (5 << 8) | 6: return launch_fused<double, 5, 6, 2, 256>(prm, inv, st);
    case (4 << 8) | 8: return launch_fused<double, 4, 8, 1, 256>(prm, inv, st);
    case (5 << 8) | 8: return launch_fused<double, 5, 8, 1, 512>(prm, inv, st);
    default: break;
    }
    *handled = false;
    return cudaSuccess;
}

int fused_lines_c128(int logvec, int logm) {
    switch ((logvec << 8) | logm) {
    case (4 << 8) | 4: return 16;
    case (4 << 8) | 5: return 8;
    case (4 << 8) | 6: return 4;
    case (2 << 8) | 7: return 8;
    case (5 << 8) | 7: return 1;
    case (5 << 8) | 6: return 2;
    case (4 << 8) | 8: return 1;
    case (5 << 8) | 8: return 1;
    default: return 0;
    }
}

}  // namespace zm
