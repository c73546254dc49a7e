// zm_plan.h -- plan object and kernel parameter blocks of libzmodel_b200 (host + device).
#pragma once

#include <stddef.h>
#include <stdint.h>

namespace zm {

// Which axis pass of a transform a line kernel runs.  Every pass reads each
// global line (N points along one axis) from P contiguous rank chunks of L
// points and writes it to the layout of the next stage of the reference
// pipeline:
//   X2  2D x pass: real layout -> layout after REPACK (fft.cu:207-269)
//   Y2  2D y pass: layout after REPACK -> reciprocal layout (fft.cu:271-328)
//   X3  3D x pass: real layout -> layout after REPACK_XY (fft3d.cu:246-298)
//   Y3  3D y pass: after REPACK_XY -> after REPACK_YZ (fft3d.cu:300-352)
//   Z3  3D z pass: after REPACK_YZ -> reciprocal layout (fft3d.cu:354-401)
enum PassKind : int { PASS_X2 = 0, PASS_Y2 = 1, PASS_X3 = 2, PASS_Y3 = 3, PASS_Z3 = 4 };

struct Geom {
    int64_t n, b, p, L, vec, vp, m;
    int logN, logB, logP, logL, logVEC, logVP, logM;
    int dim;
};

// Parameters of one launch of the fused line kernel.
struct LineParams {
    Geom g;
    int kind;          // PassKind
    int T;             // lines per CTA (consecutive lines)
    int64_t nlines;    // lines in this pass
    const void *in;
    void *out;
    const void *twN;   // w_N^m, m < N, forward sign (tw<double> or tw<float>)
    const void *twv;   // w_VEC^m, m < VEC
    const void *twm;   // w_M^m, m < M
    const void *twd;   // w_N^m, m < N, in FP64 (double2) for every dtype
    double scale_re, scale_im;
    int apply_scale;   // multiply the stored values by scale
    int variant;       // tile-shape variant of the size-specialised kernel (0 = default)
    int permute_only;  // skip all arithmetic (reference do_compute=false)
    int lg_inter;      // 2D: log2 of the row interleave of the x -> y intermediate (0 = plain REPACK layout)
    int inter_q;       // 2D, lg_inter > 0: interleave groups of 2^lg_inter y positions instead of
                       // x-frequency rows (three-stage passes only)
    int *err;          // device word set to 1 when a bounded wait inside a kernel gives up
    int64_t pf_tiles;  // size-specialised passes: L2 prefetch distance in tiles (0 = none)
    // radix schedules of the two sub-transforms (first stage first)
    int nst_vec, nst_m;
    int rad_vec[8], rad_m[8];
};

}  // namespace zm

struct zm_plan_s {
    zm::Geom g;
    int dtype;        // zm_dtype
    unsigned flags;
    int64_t ranks, rank_elems, total;
    size_t elem_bytes;
    int device;
    void *twN;        // device twiddle table (N entries)
    void *twv;        // w_VEC^m (VEC entries)
    void *twm;        // w_M^m (M entries)
    void *twd;        // w_N^m in FP64 (N entries; the same table as twN for complex128)
    int T[3];         // lines per CTA for the passes (x, y, z)
    int max_radix;
    int variant;      // tile-shape variant of the size-specialised kernel
    int nvariants;    // variants available for (VEC, M, dtype); 0 = runtime-sized kernel only
    int *dev_err;     // device error word (bounded waits that gave up), inside the tables allocation
    void *own_work;   // ZM_FLAG_OWN_WORKSPACE: one field, used by transforms called with work = NULL
};
