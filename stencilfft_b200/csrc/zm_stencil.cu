// zm_stencil.cu -- periodic stencils on the interleaved real-space layout.
//
// The reference packs halo rows / vectors on every rank (pack_laplace,
// laplace.cu:172-191), swaps them with host-staged MPI_Sendrecv
// (communicate_laplace, laplace.cu:194-256) and then runs a one-element-per-
// thread kernel that picks each neighbour from its own array or a receive
// buffer (laplace.cu:73-169).  With every virtual rank in one HBM the halo is
// simply the neighbouring rank's array: each thread maps its elements to global
// (row, column[, depth]) coordinates, steps one (two) points along the axis
// with periodic wrap, and maps back to (rank, local row, packed column) with the
// block-cyclic maps of zmodel/utils.h:166-214.  The neighbours are accumulated
// in the reference's order (above, below, left, right[, front, back], then the
// centre term), so the 2D Laplacian and dx / dy are bit-identical to it in FP64.
//
// The unit of work is one 16-byte vector of the field (two complex64, one
// complex128, four float or two double values): one per thread in stencil_kernel,
// four rows of a B-row block per thread in stencil_rows_kernel (2D, FP32) and two or
// four vectors of one line per thread in stencil3d_lines_kernel (3D Laplacian, long
// lines).  The elements of a vector share a row and a packed vector j, so every
// neighbour along y or z is again one aligned 16-byte vector; along x it is one too
// except where the step crosses into the left / right rank at the periodic wrap
// (utils.h:122-128: the shift by one element at cid = 0 / P-1), which is read element
// by element.
#include "zm_common.cuh"
#include "zm_internal.h"

namespace zm {

// global row/column/depth coordinate of a local (block-cyclic) index, and back
ZM_DEV int l2g(int li, int id, const Geom &g) {   // utils.h:168
    return ((li >> g.logB) << (g.logB + g.logP)) + (id << g.logB) + (li & ((int)g.b - 1));
}
ZM_DEV void g2l(int gi, const Geom &g, int &id, int &li) {  // utils.h:178-180
    id = (gi >> g.logB) & ((int)g.p - 1);
    li = ((gi >> (g.logB + g.logP)) << g.logB) + (gi & ((int)g.b - 1));
}
// packed column position <-> global column (utils.h:122-128 then 169)
ZM_DEV int pos2gc(int pos, int cid, const Geom &g) {
    const int j = pos >> g.logVEC, jj = pos & ((int)g.vec - 1);
    return (jj << (g.logB + g.logP)) + (cid << g.logB) + j;
}
ZM_DEV void gc2pos(int gc, const Geom &g, int &cid, int &pos) {
    cid = (gc >> g.logB) & ((int)g.p - 1);
    pos = ((gc & ((int)g.b - 1)) << g.logVEC) + (gc >> (g.logB + g.logP));
}

template <typename V> struct ops;
template <> struct ops<double> {
    static ZM_DEV double add(double a, double b) { return __dadd_rn(a, b); }
    static ZM_DEV double sub(double a, double b) { return __dsub_rn(a, b); }
    static ZM_DEV double mul(double a, double b) { return __dmul_rn(a, b); }
    static ZM_DEV double fmaop(double a, double b, double c) { return fma(a, b, c); }
    static ZM_DEV double div(double a, double b) { return __ddiv_rn(a, b); }
};
template <> struct ops<float> {
    static ZM_DEV float add(float a, float b) { return __fadd_rn(a, b); }
    static ZM_DEV float sub(float a, float b) { return __fsub_rn(a, b); }
    static ZM_DEV float mul(float a, float b) { return __fmul_rn(a, b); }
    static ZM_DEV float fmaop(float a, float b, float c) { return fmaf(a, b, c); }
    static ZM_DEV float div(float a, float b) { return __fdiv_rn(a, b); }
};

// 16 bytes of scalars
template <typename S> struct vec16 {
    static constexpr int n = 16 / (int)sizeof(S);
    S v[n];
};

// S = scalar type; NC = scalars per element (2 complex, 1 real).  One thread = one
// 16-byte vector = K = 16 / (NC * sizeof(S)) consecutive elements.
// OP = ST_ALL (2D): the Laplacian (coef) into `out`, dx and dy (coef2 = delta) into
// `out2` / `out3` from one read of the neighbourhood; each result is computed exactly as
// by its own kernel.
// dx / dy divide by 12 delta.  FP64 divides, as the reference does (dx.cu:79), so the
// results are bit-identical to it; FP32 (no reference counterpart) multiplies by
// rden = 1 / (12 delta), computed in FP64 and rounded once, at most one ulp from the
// quotient and a fraction of the cost of a correctly rounded FP32 division.
template <typename S> ZM_DEV S div_den(S x, S den, S rden);
template <> ZM_DEV double div_den<double>(double x, double den, double) { return __ddiv_rn(x, den); }
template <> ZM_DEV float div_den<float>(float x, float, float rden) { return __fmul_rn(x, rden); }

template <typename S, int NC, int OP, int DIM>
__global__ void __launch_bounds__(256) stencil_kernel(const S *__restrict__ in, S *__restrict__ out,
                                                      S *__restrict__ out2, S *__restrict__ out3,
                                                      const Geom g, int64_t nvec, S coef, S coef2, S rden) {
    using O = ops<S>;
    using V = vec16<S>;
    constexpr int K = V::n / NC;                 // elements per vector
    const int64_t vi = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (vi >= nvec) return;
    const int64_t e = vi * K;                    // first element
    const int L = (int)g.L;
    const int N = (int)g.n;
    int rank, lr, ld = 0, did = 0;
    if (DIM == 2) {
        rank = (int)(e >> (2 * g.logL));
        lr = (int)(e >> g.logL) & (L - 1);
    } else {
        rank = (int)(e >> (3 * g.logL));
        ld = (int)(e >> (2 * g.logL)) & (L - 1);
        lr = (int)(e >> g.logL) & (L - 1);
    }
    const int pos = (int)(e & (L - 1));
    const int P = (int)g.p;
    const int cid = rank & (P - 1);
    const int rid = DIM == 2 ? rank >> g.logP : (rank >> g.logP) & (P - 1);
    if (DIM == 3) did = rank >> (2 * g.logP);
    const int gr = l2g(lr, rid, g);
    const int gd = DIM == 3 ? l2g(ld, did, g) : 0;
    auto rank_of = [&](int d_, int r_, int c_) { return DIM == 2 ? r_ * P + c_ : (d_ * P + r_) * P + c_; };
    auto addr = [&](int rk, int ld_, int lr_, int pos_) -> int64_t {
        return DIM == 2 ? ((int64_t)rk << (2 * g.logL)) + (int64_t)lr_ * L + pos_
                        : ((int64_t)rk << (3 * g.logL)) + ((int64_t)ld_ * L + lr_) * L + pos_;
    };
    // neighbour vectors along y (rows) and z (depth): same packed position
    auto vrow = [&](int d) {
        int id, li;
        g2l((gr + d + N) & (N - 1), g, id, li);
        return __ldg(reinterpret_cast<const uint4 *>(in + addr(rank_of(did, id, cid), ld, li, pos) * NC));
    };
    auto vdep = [&](int d) {
        int id, li;
        g2l((gd + d + N) & (N - 1), g, id, li);
        return __ldg(reinterpret_cast<const uint4 *>(in + addr(rank_of(id, rid, cid), li, lr, pos) * NC));
    };
    // neighbour along x (columns) at column offset d of the K elements
    auto vcol = [&](int d) {
        V r;
        const int j = pos >> g.logVEC;
        if (j + d >= 0 && j + d < (int)g.b && (K == 1 || (int)g.vec % K == 0)) {
            // same rank and same jj: the neighbour vector is d packed vectors away
            *reinterpret_cast<uint4 *>(&r) = __ldg(reinterpret_cast<const uint4 *>(
                in + (e + (int64_t)d * (int64_t)g.vec) * NC));
            return r;
        }
        const int gc0 = pos2gc(pos, cid, g);
        int id0, p0;
        gc2pos((gc0 + d + N) & (N - 1), g, id0, p0);
        const int64_t a0 = addr(rank_of(did, rid, id0), ld, lr, p0);
        bool contiguous = true;
        if (K > 1) {
            const int gcl = pos2gc(pos + K - 1, cid, g);
            int idl, pl;
            gc2pos((gcl + d + N) & (N - 1), g, idl, pl);
            // one aligned 16-byte load only if the K neighbours are consecutive and start on
            // a K-element boundary (the cid = 0 wrap shifts them by one element)
            contiguous = idl == id0 && pl == p0 + K - 1 && (p0 & (K - 1)) == 0;
        }
        if (contiguous) {
            *reinterpret_cast<uint4 *>(&r) = __ldg(reinterpret_cast<const uint4 *>(in + a0 * NC));
        } else {
#pragma unroll
            for (int k = 0; k < K; k++) {
                int idk, pk;
                gc2pos((pos2gc(pos + k, cid, g) + d + N) & (N - 1), g, idk, pk);
                const int64_t ak = addr(rank_of(did, rid, idk), ld, lr, pk);
#pragma unroll
                for (int q = 0; q < NC; q++) r.v[k * NC + q] = __ldg(in + ak * NC + q);
            }
        }
        return r;
    };
    auto as = [](uint4 u) {
        V r;
        *reinterpret_cast<uint4 *>(&r) = u;
        return r;
    };
    V res;
    if (OP == ST_ALL) {
        const V up = as(vrow(-1)), dn = as(vrow(1)), lf = vcol(-1), rt = vcol(1);
        const V up2 = as(vrow(-2)), dn2 = as(vrow(2)), lf2 = vcol(-2), rt2 = vcol(2);
        const V c = as(__ldg(reinterpret_cast<const uint4 *>(in + e * NC)));
        V rx, ry;
        const S den = O::mul((S)12, coef2);
#pragma unroll
        for (int i = 0; i < V::n; i++) {
            S s = O::add((S)0, up.v[i]);
            s = O::add(s, dn.v[i]);
            s = O::add(s, lf.v[i]);
            s = O::add(s, rt.v[i]);
            s = O::fmaop((S)(-4), c.v[i], s);
            res.v[i] = O::mul(s, coef);
            S x = O::add((S)0, O::mul(lf.v[i], (S)-8));
            x = O::add(x, lf2.v[i]);
            x = O::add(x, O::mul(rt.v[i], (S)8));
            x = O::sub(x, rt2.v[i]);
            rx.v[i] = div_den(x, den, rden);
            S y = O::add((S)0, O::mul(up.v[i], (S)-8));
            y = O::add(y, up2.v[i]);
            y = O::add(y, O::mul(dn.v[i], (S)8));
            y = O::sub(y, dn2.v[i]);
            ry.v[i] = div_den(y, den, rden);
        }
        *reinterpret_cast<uint4 *>(out2 + e * NC) = *reinterpret_cast<const uint4 *>(&rx);
        *reinterpret_cast<uint4 *>(out3 + e * NC) = *reinterpret_cast<const uint4 *>(&ry);
    } else if (OP == ST_LAPLACE) {
        // laplace.cu:91-168 / laplace3d.cu:98-224 accumulation order
        const V up = as(vrow(-1)), dn = as(vrow(1)), lf = vcol(-1), rt = vcol(1);
        const V c = as(__ldg(reinterpret_cast<const uint4 *>(in + e * NC)));
        V fr, bk;
        if (DIM == 3) {
            fr = as(vdep(-1));
            bk = as(vdep(1));
        }
#pragma unroll
        for (int i = 0; i < V::n; i++) {
            S s = O::add((S)0, up.v[i]);      // scratch = {0,0}; scratch += above
            s = O::add(s, dn.v[i]);
            s = O::add(s, lf.v[i]);
            s = O::add(s, rt.v[i]);
            if (DIM == 3) {
                s = O::add(s, fr.v[i]);
                s = O::add(s, bk.v[i]);
            }
            s = O::fmaop((S)(-2 * DIM), c.v[i], s);
            res.v[i] = O::mul(s, coef);       // coef = 1/h^2 (1 reproduces the reference)
        }
    } else {
        // dx.cu:26-79 / dy.cu:34-100: ((-8 f[-1] + f[-2]) + 8 f[+1]) - f[+2], then / (12 delta)
        V m1, m2, p1, p2;
        if (OP == ST_DX) {
            m1 = vcol(-1); m2 = vcol(-2); p1 = vcol(1); p2 = vcol(2);
        } else {
            m1 = as(vrow(-1)); m2 = as(vrow(-2)); p1 = as(vrow(1)); p2 = as(vrow(2));
        }
        const S den = O::mul((S)12, coef);    // coef = delta
#pragma unroll
        for (int i = 0; i < V::n; i++) {
            S s = O::add((S)0, O::mul(m1.v[i], (S)-8));
            s = O::add(s, m2.v[i]);
            s = O::add(s, O::mul(p1.v[i], (S)8));
            s = O::sub(s, p2.v[i]);
            res.v[i] = div_den(s, den, rden);
        }
    }
    *reinterpret_cast<uint4 *>(out + e * NC) = *reinterpret_cast<const uint4 *>(&res);
}

// 2D stencils (OP as in stencil_kernel), RY consecutive local rows of one B-row block per
// thread (the same packed position): the 16-byte vectors of the rows the stencil needs
// (lr0 - 2 .. lr0 + RY + 1 for dy and the three in one launch, lr0 - 1 .. lr0 + RY for the
// Laplacian, none beyond the centre rows for dx) are loaded once and shared by the RY
// outputs, and the index arithmetic is done once per thread.  Rows outside the block
// (above a block's first row group, below its last) go through the block-cyclic maps as
// in stencil_kernel; every output is computed by the same expressions, in the same order.
template <typename S, int NC, int OP, int RY>
__global__ void __launch_bounds__(256) stencil_rows_kernel(const S *__restrict__ in, S *__restrict__ out,
                                                           S *__restrict__ out2, S *__restrict__ out3,
                                                           const Geom g, int64_t nthreads, S coef, S coef2,
                                                           S rden) {
    using O = ops<S>;
    using V = vec16<S>;
    constexpr int K = V::n / NC;                 // elements per vector
    const int64_t vi = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (vi >= nthreads) return;
    const int L = (int)g.L, N = (int)g.n, P = (int)g.p;
    const int vrow_n = L / K;                    // vectors per row
    const int vpos = (int)(vi % vrow_n);
    const int64_t rest = vi / vrow_n;
    const int rg = (int)(rest % (L / RY));
    const int rank = (int)(rest / (L / RY));
    const int lr0 = rg * RY, pos = vpos * K;
    const int64_t e0 = ((int64_t)rank << (2 * g.logL)) + (int64_t)lr0 * L + pos;
    const int cid = rank & (P - 1), rid = rank >> g.logP;
    const int gr0 = l2g(lr0, rid, g);
    const int lrb0 = lr0 & ((int)g.b - 1);
    auto ld16 = [&](int64_t el) {
        V r;
        *reinterpret_cast<uint4 *>(&r) = __ldg(reinterpret_cast<const uint4 *>(in + el * NC));
        return r;
    };
    // row lr0 + d (d in [-2, RY + 1]) at the same packed position
    auto rowv = [&](int d) {
        if (lrb0 + d >= 0 && lrb0 + d < (int)g.b) return ld16(e0 + (int64_t)d * L);
        int id, li;
        g2l((gr0 + d + N) & (N - 1), g, id, li);
        return ld16(((int64_t)(id * P + cid) << (2 * g.logL)) + (int64_t)li * L + pos);
    };
    // neighbour along x at column offset d of row lr (element e of its first point)
    const int j = pos >> g.logVEC;
    auto colv = [&](int64_t e, int lr, int d) {
        if (j + d >= 0 && j + d < (int)g.b && (K == 1 || (int)g.vec % K == 0))
            return ld16(e + (int64_t)d * (int64_t)g.vec);
        V r;
        const int gc0 = pos2gc(pos, cid, g);
        int id0, p0;
        gc2pos((gc0 + d + N) & (N - 1), g, id0, p0);
        const int64_t a0 = ((int64_t)(rid * P + id0) << (2 * g.logL)) + (int64_t)lr * L + p0;
        bool contiguous = true;
        if (K > 1) {
            const int gcl = pos2gc(pos + K - 1, cid, g);
            int idl, pl;
            gc2pos((gcl + d + N) & (N - 1), g, idl, pl);
            contiguous = idl == id0 && pl == p0 + K - 1 && (p0 & (K - 1)) == 0;
        }
        if (contiguous) return ld16(a0);
#pragma unroll
        for (int k = 0; k < K; k++) {
            int idk, pk;
            gc2pos((pos2gc(pos + k, cid, g) + d + N) & (N - 1), g, idk, pk);
            const int64_t ak = ((int64_t)(rid * P + idk) << (2 * g.logL)) + (int64_t)lr * L + pk;
#pragma unroll
            for (int q = 0; q < NC; q++) r.v[k * NC + q] = __ldg(in + ak * NC + q);
        }
        return r;
    };
    // rows lr0 + d for d in [-H, RY + H), H = the stencil's reach along y
    constexpr int H = OP == ST_LAPLACE ? 1 : (OP == ST_DX ? 0 : 2);
    V ys[RY + 2 * H];
#pragma unroll
    for (int d = -H; d < RY + H; d++) ys[d + H] = rowv(d);
    if constexpr (OP != ST_ALL) {
        const S den = O::mul((S)12, coef);    // dx / dy: coef = delta
#pragma unroll
        for (int r = 0; r < RY; r++) {
            const int64_t e = e0 + (int64_t)r * L;
            V res;
            if constexpr (OP == ST_LAPLACE) {
                // laplace.cu:91-168 accumulation order
                const V lf = colv(e, lr0 + r, -1), rt = colv(e, lr0 + r, 1);
                const V &up = ys[r], &dn = ys[r + 2], &c = ys[r + 1];
#pragma unroll
                for (int i = 0; i < V::n; i++) {
                    S s = O::add((S)0, up.v[i]);
                    s = O::add(s, dn.v[i]);
                    s = O::add(s, lf.v[i]);
                    s = O::add(s, rt.v[i]);
                    s = O::fmaop((S)(-4), c.v[i], s);
                    res.v[i] = O::mul(s, coef);
                }
            } else {
                // dx.cu:26-79 / dy.cu:34-100: ((-8 f[-1] + f[-2]) + 8 f[+1]) - f[+2], / (12 delta)
                V m1, m2, p1, p2;
                if constexpr (OP == ST_DX) {
                    m1 = colv(e, lr0 + r, -1); m2 = colv(e, lr0 + r, -2);
                    p1 = colv(e, lr0 + r, 1); p2 = colv(e, lr0 + r, 2);
                } else {
                    m1 = ys[r + 1]; m2 = ys[r]; p1 = ys[r + 3]; p2 = ys[r + 4];
                }
#pragma unroll
                for (int i = 0; i < V::n; i++) {
                    S s = O::add((S)0, O::mul(m1.v[i], (S)-8));
                    s = O::add(s, m2.v[i]);
                    s = O::add(s, O::mul(p1.v[i], (S)8));
                    s = O::sub(s, p2.v[i]);
                    res.v[i] = div_den(s, den, rden);
                }
            }
            *reinterpret_cast<uint4 *>(out + e * NC) = *reinterpret_cast<const uint4 *>(&res);
        }
        return;
    }
    const S den = O::mul((S)12, coef2);
#pragma unroll
    for (int r = 0; r < RY; r++) {
        const int64_t e = e0 + (int64_t)r * L;
        const V lf = colv(e, lr0 + r, -1), rt = colv(e, lr0 + r, 1);
        const V lf2 = colv(e, lr0 + r, -2), rt2 = colv(e, lr0 + r, 2);
        const V &up = ys[r + 1], &dn = ys[r + 3], &up2 = ys[r], &dn2 = ys[r + 4], &c = ys[r + 2];
        V res, rx, ry;
#pragma unroll
        for (int i = 0; i < V::n; i++) {
            S s = O::add((S)0, up.v[i]);
            s = O::add(s, dn.v[i]);
            s = O::add(s, lf.v[i]);
            s = O::add(s, rt.v[i]);
            s = O::fmaop((S)(-4), c.v[i], s);
            res.v[i] = O::mul(s, coef);
            S x = O::add((S)0, O::mul(lf.v[i], (S)-8));
            x = O::add(x, lf2.v[i]);
            x = O::add(x, O::mul(rt.v[i], (S)8));
            x = O::sub(x, rt2.v[i]);
            rx.v[i] = div_den(x, den, rden);
            S y = O::add((S)0, O::mul(up.v[i], (S)-8));
            y = O::add(y, up2.v[i]);
            y = O::add(y, O::mul(dn.v[i], (S)8));
            y = O::sub(y, dn2.v[i]);
            ry.v[i] = div_den(y, den, rden);
        }
        *reinterpret_cast<uint4 *>(out + e * NC) = *reinterpret_cast<const uint4 *>(&res);
        *reinterpret_cast<uint4 *>(out2 + e * NC) = *reinterpret_cast<const uint4 *>(&rx);
        *reinterpret_cast<uint4 *>(out3 + e * NC) = *reinterpret_cast<const uint4 *>(&ry);
    }
}

// 3D Laplacian (laplace3d.cu:98-224 accumulation order) with RX vectors of one line per
// thread.  A warp takes 32 * RX consecutive 16-byte vectors of one (rank, depth, row) line
// (lane t: vectors t, t + 32, ..., so every load instruction of the warp stays one
// contiguous 512-byte run), and the four neighbour lines along y and z (block-cyclic
// maps with the periodic wrap) are located once per thread for its RX vectors instead of
// once per vector: the integer index work, not DRAM, bounds the one-vector kernel
// (stencil_kernel<..., 3>).  Each output is computed by the same expressions in the same
// order as there.
template <typename S, int NC, int RX>
__global__ void __launch_bounds__(256) stencil3d_lines_kernel(const S *__restrict__ in, S *__restrict__ out,
                                                              const Geom g, int64_t nseg, S coef) {
    using O = ops<S>;
    using V = vec16<S>;
    constexpr int K = V::n / NC;                 // elements per vector
    const int64_t seg = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (seg >= nseg) return;
    const int lane = (int)(threadIdx.x & 31);
    const int L = (int)g.L, N = (int)g.n, P = (int)g.p;
    const int segs_line = L / (K * 32 * RX);     // warps per line
    // Line order.  Complex128 (RX = 4): global order -- global depth, global row, then the
    // P ranks that share that global row -- so that a line's y and z neighbours (at a
    // block edge they sit in another rank's array, far away in memory) are read close in
    // time to when they are the centre line (N = 512: 1.126 -> 1.034 ms).  Complex64
    // (RX = 2): rank order, which measured faster for it (0.617 against 0.643 ms).
    constexpr bool GORDER = RX == 4;
    const int64_t gline = seg / segs_line;       // GORDER: (gd * N + gr) * P + cid
    const int v0 = (int)(seg - gline * segs_line) * 32 * RX + lane;
    int cid, rid, lr, did, ld, gr, gd;
    if constexpr (GORDER) {
        cid = (int)gline & (P - 1);
        gr = (int)(gline >> g.logP) & (N - 1);
        gd = (int)(gline >> (g.logP + g.logN));
        g2l(gr, g, rid, lr);
        g2l(gd, g, did, ld);
    } else {                                     // (rank * L + ld) * L + lr
        lr = (int)gline & (L - 1);
        ld = (int)(gline >> g.logL) & (L - 1);
        const int rk = (int)(gline >> (2 * g.logL));
        cid = rk & (P - 1);
        rid = (rk >> g.logP) & (P - 1);
        did = rk >> (2 * g.logP);
        gr = l2g(lr, rid, g);
        gd = l2g(ld, did, g);
    }
    const int rank = (did * P + rid) * P + cid;
    const int64_t line = ((((int64_t)rank << g.logL) + ld) << g.logL) + lr;   // (rank * L + ld) * L + lr
    // first element of the neighbour lines
    auto yline = [&](int d) {
        int id, li;
        g2l((gr + d + N) & (N - 1), g, id, li);
        const int rk = (did * P + id) * P + cid;
        return (((((int64_t)rk << g.logL) + ld) << g.logL) + li) << g.logL;
    };
    auto zline = [&](int d) {
        int id, li;
        g2l((gd + d + N) & (N - 1), g, id, li);
        const int rk = (id * P + rid) * P + cid;
        return (((((int64_t)rk << g.logL) + li) << g.logL) + lr) << g.logL;
    };
    const int64_t ec = line << g.logL, eu = yline(-1), ed = yline(1), ef = zline(-1), eb = zline(1);
    auto ld16 = [&](int64_t el) {
        V r;
        *reinterpret_cast<uint4 *>(&r) = __ldg(reinterpret_cast<const uint4 *>(in + el * NC));
        return r;
    };
    // neighbour along x (d = -1 / +1) of the vector at packed position pos (VEC a multiple
    // of K, checked by the host).  Inside a B-column block it is the vector VEC positions
    // away.  Across the block edge it is column B - 1 / 0 of the rank to the left / right
    // at the same cycle jj, except past the end of a block cycle (cid = 0 / P - 1): there
    // the rank is P - 1 ranks away and the cycle moves by one, so the K neighbours are
    // shifted by one element (utils.h:122-128) and read one by one.
    const int64_t l3 = (int64_t)1 << (3 * g.logL);
    auto colv = [&](int pos, int d) {
        const int j = pos >> g.logVEC;
        if (d < 0 ? j > 0 : j < (int)g.b - 1) return ld16(ec + pos + (int64_t)d * (int64_t)g.vec);
        const bool wrap = d < 0 ? cid == 0 : cid == P - 1;
        const int64_t e1 = ec + (wrap ? (int64_t)(-d * (P - 1)) : (int64_t)d) * l3 +
                           (d < 0 ? ((int)g.b - 1) << g.logVEC : 0);
        const int jj = pos & ((int)g.vec - 1);
        if (!wrap) return ld16(e1 + jj);
        V r;
#pragma unroll
        for (int k = 0; k < K; k++) {
            const int64_t ak = e1 + ((jj + k + d) & ((int)g.vec - 1));
#pragma unroll
            for (int q = 0; q < NC; q++) r.v[k * NC + q] = __ldg(in + ak * NC + q);
        }
        return r;
    };
#pragma unroll
    for (int x = 0; x < RX; x++) {
        const int pos = (v0 + 32 * x) * K;
        const V up = ld16(eu + pos), dn = ld16(ed + pos), lf = colv(pos, -1), rt = colv(pos, 1);
        const V fr = ld16(ef + pos), bk = ld16(eb + pos), c = ld16(ec + pos);
        V res;
#pragma unroll
        for (int i = 0; i < V::n; i++) {
            S s = O::add((S)0, up.v[i]);
            s = O::add(s, dn.v[i]);
            s = O::add(s, lf.v[i]);
            s = O::add(s, rt.v[i]);
            s = O::add(s, fr.v[i]);
            s = O::add(s, bk.v[i]);
            s = O::fmaop((S)(-6), c.v[i], s);
            res.v[i] = O::mul(s, coef);
        }
        *reinterpret_cast<uint4 *>(out + (ec + pos) * NC) = *reinterpret_cast<const uint4 *>(&res);
    }
}

template <typename S, int NC>
static cudaError_t launch_s(const zm_plan_s *p, int op, const void *in, void *out, void *out2, void *out3,
                            double coef, double coef2, cudaStream_t st) {
    constexpr int K = 16 / (int)sizeof(S) / NC;
    if (p->g.L % K) return cudaErrorInvalidValue;
    const int64_t nvec = p->total / K;
    const int threads = 256;
    const unsigned grid = (unsigned)((nvec + threads - 1) / threads);
    const S *i = reinterpret_cast<const S *>(in);
    S *o = reinterpret_cast<S *>(out), *o2 = reinterpret_cast<S *>(out2), *o3 = reinterpret_cast<S *>(out3);
    const S c = (S)coef, c2 = (S)coef2;
    // 1 / (12 delta) for the FP32 derivatives (delta = coef for dx / dy, coef2 for ST_ALL)
    const double dl = op == ST_ALL ? coef2 : coef;
    const S rd = (S)(1.0 / (12.0 * dl));
    if (p->g.dim == 2) {
        if (sizeof(S) == 4 && p->g.b % 4 == 0) {
            // four rows of a B-row block per thread (FP32; the FP64 form stays one row
            // per thread: its four-row form was slower, 4.20 -> 4.34 ms at N = 16384 for
            // the three stencils in one launch)
            const int64_t nt = nvec / 4;
            const unsigned g4 = (unsigned)((nt + threads - 1) / threads);
            if (op == ST_LAPLACE)
                stencil_rows_kernel<S, NC, ST_LAPLACE, 4><<<g4, threads, 0, st>>>(i, o, o2, o3, p->g, nt, c, c2, rd);
            else if (op == ST_DX)
                stencil_rows_kernel<S, NC, ST_DX, 4><<<g4, threads, 0, st>>>(i, o, o2, o3, p->g, nt, c, c2, rd);
            else if (op == ST_DY)
                stencil_rows_kernel<S, NC, ST_DY, 4><<<g4, threads, 0, st>>>(i, o, o2, o3, p->g, nt, c, c2, rd);
            else
                stencil_rows_kernel<S, NC, ST_ALL, 4><<<g4, threads, 0, st>>>(i, o, o2, o3, p->g, nt, c, c2, rd);
        } else if (op == ST_LAPLACE)
            stencil_kernel<S, NC, ST_LAPLACE, 2><<<grid, threads, 0, st>>>(i, o, o2, o3, p->g, nvec, c, c2, rd);
        else if (op == ST_DX)
            stencil_kernel<S, NC, ST_DX, 2><<<grid, threads, 0, st>>>(i, o, o2, o3, p->g, nvec, c, c2, rd);
        else if (op == ST_DY)
            stencil_kernel<S, NC, ST_DY, 2><<<grid, threads, 0, st>>>(i, o, o2, o3, p->g, nvec, c, c2, rd);
        else
            stencil_kernel<S, NC, ST_ALL, 2><<<grid, threads, 0, st>>>(i, o, o2, o3, p->g, nvec, c, c2, rd);
    } else {
        if (op != ST_LAPLACE) return cudaErrorInvalidValue;
        // vectors of one line per thread: 4 for one complex128 per vector, else 2
        constexpr int RX = K == 1 ? 4 : 2;
        const int64_t vline = p->g.L / K;       // vectors per line
        if (vline % (32 * RX) == 0 && p->g.vec % K == 0) {
            const int64_t nseg = nvec / (32 * RX);
            const unsigned gs = (unsigned)((nseg * 32 + threads - 1) / threads);
            stencil3d_lines_kernel<S, NC, RX><<<gs, threads, 0, st>>>(i, o, p->g, nseg, c);
        } else {
            stencil_kernel<S, NC, ST_LAPLACE, 3><<<grid, threads, 0, st>>>(i, o, o2, o3, p->g, nvec, c, c2, rd);
        }
    }
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_stencil(const zm_plan_s *p, int op, bool real_field, const void *in, void *out,
                           double coef, cudaStream_t st, void *out2, void *out3, double coef2) {
    if (p->dtype == 0) {
        return real_field ? launch_s<double, 1>(p, op, in, out, out2, out3, coef, coef2, st)
                          : launch_s<double, 2>(p, op, in, out, out2, out3, coef, coef2, st);
    }
    return real_field ? launch_s<float, 1>(p, op, in, out, out2, out3, coef, coef2, st)
                      : launch_s<float, 2>(p, op, in, out, out2, out3, coef, coef2, st);
}

}  // namespace zm
