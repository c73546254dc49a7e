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
ZM_DEV void stencil_rows_body(const S *__restrict__ in, S *__restrict__ out, S *__restrict__ out2,
                              S *__restrict__ out3, const Geom &g, int64_t nthreads, S coef, S coef2, S rden) {
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
                if constexpr (sizeof(S) == 4) {   // two scalars per FP32x2 instruction, same order
                    using F2 = cpx<float>;
                    auto pr = [](const V &v, int i) { return F2{v.v[2 * i], v.v[2 * i + 1]}; };
#pragma unroll
                    for (int i = 0; i < V::n / 2; i++) {
                        F2 t = cadd(F2{0.f, 0.f}, pr(up, i));
                        t = cadd(t, pr(dn, i));
                        t = cadd(t, pr(lf, i));
                        t = cadd(t, pr(rt, i));
                        t = cfma2(F2{-4.f, -4.f}, pr(c, i), t);
                        t = cmul2(t, F2{coef, coef});
                        res.v[2 * i] = t.x;
                        res.v[2 * i + 1] = t.y;
                    }
                } else {
#pragma unroll
                    for (int i = 0; i < V::n; i++) {
                        S s = O::add((S)0, up.v[i]);
                        s = O::add(s, dn.v[i]);
                        s = O::add(s, lf.v[i]);
                        s = O::add(s, rt.v[i]);
                        s = O::fmaop((S)(-4), c.v[i], s);
                        res.v[i] = O::mul(s, coef);
                    }
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
                if constexpr (sizeof(S) == 4) {   // two scalars per FP32x2 instruction, same order
                    using F2 = cpx<float>;
                    auto pr = [](const V &v, int i) { return F2{v.v[2 * i], v.v[2 * i + 1]}; };
#pragma unroll
                    for (int i = 0; i < V::n / 2; i++) {
                        F2 t = cadd(F2{0.f, 0.f}, cmul2(pr(m1, i), F2{-8.f, -8.f}));
                        t = cadd(t, pr(m2, i));
                        t = cadd(t, cmul2(pr(p1, i), F2{8.f, 8.f}));
                        t = csub(t, pr(p2, i));
                        t = cmul2(t, F2{rden, rden});
                        res.v[2 * i] = t.x;
                        res.v[2 * i + 1] = t.y;
                    }
                } else {
#pragma unroll
                    for (int i = 0; i < V::n; i++) {
                        S s = O::add((S)0, O::mul(m1.v[i], (S)-8));
                        s = O::add(s, m2.v[i]);
                        s = O::add(s, O::mul(p1.v[i], (S)8));
                        s = O::sub(s, p2.v[i]);
                        res.v[i] = div_den(s, den, rden);
                    }
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
        if constexpr (sizeof(S) == 4) {
            // FP32: the same operations in the same order on two scalars at a time, one
            // FP32x2 instruction each
            using F2 = cpx<float>;
            auto pr = [](const V &v, int i) { return F2{v.v[2 * i], v.v[2 * i + 1]}; };
            const F2 z{0.f, 0.f}, m8{-8.f, -8.f}, p8{8.f, 8.f}, m4{-4.f, -4.f}, cf{coef, coef}, rd{rden, rden};
#pragma unroll
            for (int i = 0; i < V::n / 2; i++) {
                F2 t = cadd(z, pr(up, i));
                t = cadd(t, pr(dn, i));
                t = cadd(t, pr(lf, i));
                t = cadd(t, pr(rt, i));
                t = cfma2(m4, pr(c, i), t);
                t = cmul2(t, cf);
                res.v[2 * i] = t.x;
                res.v[2 * i + 1] = t.y;
                F2 x = cadd(z, cmul2(pr(lf, i), m8));
                x = cadd(x, pr(lf2, i));
                x = cadd(x, cmul2(pr(rt, i), p8));
                x = csub(x, pr(rt2, i));
                x = cmul2(x, rd);
                rx.v[2 * i] = x.x;
                rx.v[2 * i + 1] = x.y;
                F2 y = cadd(z, cmul2(pr(up, i), m8));
                y = cadd(y, pr(up2, i));
                y = cadd(y, cmul2(pr(dn, i), p8));
                y = csub(y, pr(dn2, i));
                y = cmul2(y, rd);
                ry.v[2 * i] = y.x;
                ry.v[2 * i + 1] = y.y;
            }
        } else {
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
        }
        *reinterpret_cast<uint4 *>(out + e * NC) = *reinterpret_cast<const uint4 *>(&res);
        *reinterpret_cast<uint4 *>(out2 + e * NC) = *reinterpret_cast<const uint4 *>(&rx);
        *reinterpret_cast<uint4 *>(out3 + e * NC) = *reinterpret_cast<const uint4 *>(&ry);
    }
}

// The kernels: the default register allocation (four rows per thread, FP32), and one
// row per thread in FP64 held to 51 registers, five CTAs per SM (the FP64 kernel waits on
// its loads: 56 registers and four CTAs per SM left the three stencils at 4.01 ms at
// N = 16384 c128, five take 3.72 ms)
template <typename S, int NC, int OP, int RY>
__global__ void __launch_bounds__(256) stencil_rows_kernel(const S *__restrict__ in, S *__restrict__ out,
                                                           S *__restrict__ out2, S *__restrict__ out3,
                                                           const Geom g, int64_t nthreads, S coef, S coef2,
                                                           S rden) {
    stencil_rows_body<S, NC, OP, RY>(in, out, out2, out3, g, nthreads, coef, coef2, rden);
}
template <typename S, int NC, int OP>
__global__ void __launch_bounds__(256, 5) stencil_rows1_kernel(const S *__restrict__ in, S *__restrict__ out,
                                                               S *__restrict__ out2, S *__restrict__ out3,
                                                               const Geom g, int64_t nthreads, S coef, S coef2,
                                                               S rden) {
    stencil_rows_body<S, NC, OP, 1>(in, out, out2, out3, g, nthreads, coef, coef2, rden);
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

// ------------------------------------------------ 3D Laplacian on shared-memory plane tiles
// mbarrier helpers (bulk copies into shared memory complete on an mbarrier)
ZM_DEV unsigned st_smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
ZM_DEV void st_mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(st_smem_u32(bar)), "r"(count) : "memory");
}
ZM_DEV void st_mbar_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(st_smem_u32(bar)), "r"(bytes)
                 : "memory");
}
ZM_DEV bool st_mbar_try_wait(uint64_t *bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(st_smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
ZM_DEV unsigned long long st_gtimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
ZM_DEV void st_bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     st_smem_u32(dst)),
                 "l"((unsigned long long)__cvta_generic_to_global(src)), "r"(bytes), "r"(st_smem_u32(bar))
                 : "memory");
}
constexpr unsigned long long kPlaneWaitNs = 1000000000ull;   // 1 s per bounded wait
constexpr int kMarchSlots = 4;                                // plane tiles in flight + in use

ZM_DEV void st_cp_async(void *dst, const void *src, int bytes) {   // 8 or 16 bytes, aligned
    if (bytes == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(st_smem_u32(dst)),
                     "l"((unsigned long long)__cvta_generic_to_global(src))
                     : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(st_smem_u32(dst)),
                     "l"((unsigned long long)__cvta_generic_to_global(src))
                     : "memory");
}
ZM_DEV void st_cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> ZM_DEV void st_cp_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// One CTA owns a tile of TY local rows (TY | B, so the rows are globally consecutive) of
// one rank column (rid, cid) and walks a chunk of global depths gd, upwards in even chunks
// and downwards in odd ones, so that two neighbouring chunks read their shared boundary
// planes at about the same time (the second read comes from L2).  Every step brings the
// next plane's tile -- its TY rows (one contiguous run of the rank's array) and the y
// neighbours of its first and last rows (the same or the neighbouring rank) -- into a
// ring of four shared-memory slots with bulk asynchronous copies (cp.async.bulk, no tensor
// map, no multicast) completing on one mbarrier per slot, and the x neighbours across the
// block edges (the last vector of the left rank's row and the first vector of the right
// rank's, per tile row) with per-thread asynchronous copies (cp.async) into the slot's edge
// area.  The outputs of depth gd then come from the slots of gd - 1, gd, gd + 1 only (at
// the periodic x wrap the edge vector is read shifted by one element, as
// stencil3d_lines_kernel's closed form).  Every plane is read from HBM once, plus two halo
// rows per TY rows, the x edges and two halo planes per chunk; walking global depth makes
// the z neighbours across a block edge simply the next plane of the walk.  Same
// expressions, same order as the other 3D kernels.  A copy that has not landed within two
// bounded waits raises the plan's device error word; the CTA then stops, after its copies
// in flight have landed (bounded).
template <typename S, int TY>
__global__ void __launch_bounds__(256) stencil3d_march_kernel(const cpx<S> *__restrict__ in, cpx<S> *__restrict__ out,
                                                              const Geom g, int zsteps, S coef, int *err) {
    using C = cpx<S>;
    using O = ops<S>;
    constexpr bool PAIRS = sizeof(S) == 4;                   // complex64: two elements per 16 bytes
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ uint64_t s_bar[kMarchSlots];
    const int L = (int)g.L, N = (int)g.n, P = (int)g.p, VEC = (int)g.vec;
    const int tid = threadIdx.x;
    const int logL = g.logL, vsh = g.logVEC, vmask = VEC - 1, bl = (int)g.b - 1;
    // slot: halo row above, TY rows, halo row below; then the edge area [side][row][VEC]
    const int slotE = (TY + 2) * L + 2 * TY * VEC;
    C *slots = reinterpret_cast<C *>(smem_raw);
    // unit of this CTA: (rank column rid * P + cid, depth chunk, row tile), the row tile
    // fastest so that the CTAs of neighbouring tiles (which share halo rows) and of
    // neighbouring chunks (which share halo planes) run at the same time
    const int nchunk = N / zsteps, ntile = L / TY;
    const int tile = blockIdx.x % ntile;
    const int zc = (blockIdx.x / ntile) % nchunk;
    const int col = blockIdx.x / (nchunk * ntile);
    const int rid = col / P, cid = col % P;
    const int lr0 = tile * TY;
    const int gd0 = zc * zsteps;
    const bool down = (zc & 1) != 0;
    int ridU, lrU, ridD, lrD;
    g2l((l2g(lr0, rid, g) - 1 + N) & (N - 1), g, ridU, lrU);
    g2l((l2g(lr0 + TY - 1, rid, g) + 1) & (N - 1), g, ridD, lrD);
    const int64_t l3 = (int64_t)L * L * L;
    // x block edges: the left rank is cid - 1 (cid = 0: P - 1, read shifted by one element),
    // the right rank cid + 1 (cid = P - 1: 0, shifted the other way)
    const int64_t dl = cid == 0 ? (int64_t)(P - 1) * l3 : -l3, dr = cid == P - 1 ? -(int64_t)(P - 1) * l3 : l3;
    const int shl = cid == 0 ? -1 : 0, shr = cid == P - 1 ? 1 : 0;
    auto row_elem = [&](int rk, int ld, int lr) { return ((((((int64_t)rk << logL) + ld) << logL) + lr) << logL); };
    const unsigned row_bytes = (unsigned)(L * sizeof(C));
    // global depth of walk step k (steps 0 and zsteps + 1 are the halo planes)
    auto step_depth = [&](int k) { return down ? gd0 + zsteps - k : gd0 - 1 + k; };
    // step k into slot k mod 4 (its (k / 4)-th use: parity (k / 4) & 1)
    auto issue_bulk = [&](int k) {   // thread 0
        int did, ld;
        g2l((step_depth(k) + N) & (N - 1), g, did, ld);
        const int rk = (did * P + rid) * P + cid;
        const int rkU = (did * P + ridU) * P + cid, rkD = (did * P + ridD) * P + cid;
        C *dst = slots + (size_t)(k % kMarchSlots) * slotE;
        uint64_t *bar = &s_bar[k % kMarchSlots];
        st_mbar_expect_tx(bar, (unsigned)(TY + 2) * row_bytes);
        st_bulk_g2s(dst, in + row_elem(rkU, ld, lrU), row_bytes, bar);
        st_bulk_g2s(dst + L, in + row_elem(rk, ld, lr0), TY * row_bytes, bar);
        st_bulk_g2s(dst + (size_t)(TY + 1) * L, in + row_elem(rkD, ld, lrD), row_bytes, bar);
    };
    // every thread: its share of step k's edge vectors (centre planes only), one group
    auto issue_edges = [&](int k) {
        if (k >= 1 && k <= zsteps) {
            int did, ld;
            g2l((step_depth(k) + N) & (N - 1), g, did, ld);
            const int64_t eb = row_elem((did * P + rid) * P + cid, ld, lr0);
            C *dst = slots + (size_t)(k % kMarchSlots) * slotE + (size_t)(TY + 2) * L;
            for (int q = tid; q < 2 * TY * VEC; q += blockDim.x) {
                const int side = q / (TY * VEC), r = (q / VEC) % TY, jj = q & vmask;
                const int64_t src = eb + ((int64_t)r << logL) + (side ? dr + jj : dl + ((int64_t)bl << vsh) + jj);
                st_cp_async(dst + q, in + src, (int)sizeof(C));
            }
        }
        st_cp_commit();
    };
    auto wait_bounded = [&](int k) {                          // thread 0 only
        uint64_t *bar = &s_bar[k % kMarchSlots];
        const unsigned par = (unsigned)((k / kMarchSlots) & 1);
        if (st_mbar_try_wait(bar, par)) return true;
        const unsigned long long t0 = st_gtimer_ns();
        while (!st_mbar_try_wait(bar, par))
            if (st_gtimer_ns() - t0 > kPlaneWaitNs) return false;
        return true;
    };
    if (tid == 0) {
        for (int i = 0; i < kMarchSlots; i++) st_mbar_init(&s_bar[i], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const int nsteps = zsteps + 2;                            // zsteps >= 16: nsteps > 4
    int issued = 0;                                           // steps issued (uniform count)
    for (; issued < kMarchSlots; issued++) {
        if (tid == 0) issue_bulk(issued);
        issue_edges(issued);
    }
    bool lost = false;                                        // block-uniform
    int waited = 0;                                           // steps whose bulk copies have landed
    auto wait_step = [&](int k) {
        bool ok = true;
        if (tid == 0) {
            ok = wait_bounded(k) || wait_bounded(k);          // two bounded waits, as the FFT passes
            if (!ok && err) atomicExch(err, 1);
        }
        lost = __syncthreads_or(!ok) != 0;
        if (!lost) waited = k + 1;
    };
    wait_step(0);
    if (!lost) wait_step(1);
    const int per_plane = TY * L;
    for (int z = 0; z < zsteps && !lost; z++) {
        // edges of step z + 1: groups issued so far = z + 4, the last two may be pending
        st_cp_wait<2>();
        wait_step(z + 2);                                     // also publishes the edge copies
        if (lost) break;
        const C *p0 = slots + (size_t)(z % kMarchSlots) * slotE;
        const C *pc = slots + (size_t)((z + 1) % kMarchSlots) * slotE;
        const C *p2 = slots + (size_t)((z + 2) % kMarchSlots) * slotE;
        const C *pm = down ? p2 : p0;                         // depth gd - 1
        const C *pp = down ? p0 : p2;                         // depth gd + 1
        const C *eL = pc + (size_t)(TY + 2) * L, *eR = eL + TY * VEC;
        int did, ld;
        g2l(step_depth(z + 1), g, did, ld);
        C *orow = out + row_elem((did * P + rid) * P + cid, ld, lr0);
        auto lap = [&](const C &up, const C &dn, const C &lf, const C &rt, const C &fr, const C &bk, const C &cc) {
            S rx = O::add((S)0, up.x), ry = O::add((S)0, up.y);
            rx = O::add(rx, dn.x);
            ry = O::add(ry, dn.y);
            rx = O::add(rx, lf.x);
            ry = O::add(ry, lf.y);
            rx = O::add(rx, rt.x);
            ry = O::add(ry, rt.y);
            rx = O::add(rx, fr.x);
            ry = O::add(ry, fr.y);
            rx = O::add(rx, bk.x);
            ry = O::add(ry, bk.y);
            rx = O::fmaop((S)(-6), cc.x, rx);
            ry = O::fmaop((S)(-6), cc.y, ry);
            return C{O::mul(rx, coef), O::mul(ry, coef)};
        };
        bool paired = false;
        if constexpr (PAIRS) {
          if (VEC >= 2) {
            paired = true;
            // complex64, two adjacent elements per thread (same row, same vector j): every
            // slot access and the store are 16-byte vectors, except across a block edge;
            // each element's sums run on its (re, im) pair as one FP32x2 instruction (the
            // same operations in the same order per component as lap)
            auto lapv = [&](const C &up, const C &dn, const C &lf, const C &rt, const C &fr, const C &bk,
                            const C &cc) {
                C r = cadd(C{0.f, 0.f}, up);
                r = cadd(r, dn);
                r = cadd(r, lf);
                r = cadd(r, rt);
                r = cadd(r, fr);
                r = cadd(r, bk);
                r = cfma2(C{-6.f, -6.f}, cc, r);
                return cmul2(r, C{coef, coef});
            };
            using C2 = float4;
            auto ld2 = [](const C *p, C &a, C &b) {
                const C2 q = *reinterpret_cast<const C2 *>(p);
                a = C{(S)q.x, (S)q.y};
                b = C{(S)q.z, (S)q.w};
            };
            for (int h = tid; h < per_plane / 2; h += blockDim.x) {
                const int e = 2 * h;
                const int r = e >> logL, pos = e & (L - 1);
                const int c = (r + 1) * L + pos;
                const int j = pos >> vsh, jj = pos & vmask;
                C lf0, lf1, rt0, rt1, up0, up1, dn0, dn1, fr0, fr1, bk0, bk1, c0, c1;
                if (j > 0) {
                    ld2(pc + c - VEC, lf0, lf1);
                } else {
                    lf0 = eL[r * VEC + ((jj + shl) & vmask)];
                    lf1 = eL[r * VEC + ((jj + 1 + shl) & vmask)];
                }
                if (j < bl) {
                    ld2(pc + c + VEC, rt0, rt1);
                } else {
                    rt0 = eR[r * VEC + ((jj + shr) & vmask)];
                    rt1 = eR[r * VEC + ((jj + 1 + shr) & vmask)];
                }
                ld2(pc + c - L, up0, up1);
                ld2(pc + c + L, dn0, dn1);
                ld2(pm + c, fr0, fr1);
                ld2(pp + c, bk0, bk1);
                ld2(pc + c, c0, c1);
                const C o0 = lapv(up0, dn0, lf0, rt0, fr0, bk0, c0), o1 = lapv(up1, dn1, lf1, rt1, fr1, bk1, c1);
                *reinterpret_cast<C2 *>(orow + e) = make_float4((float)o0.x, (float)o0.y, (float)o1.x, (float)o1.y);
            }
          }
        }
        if (!paired) {
            for (int e = tid; e < per_plane; e += blockDim.x) {
                const int r = e >> logL, pos = e & (L - 1);      // tile row, packed position
                const int c = (r + 1) * L + pos;                   // centre's slot element
                const int j = pos >> vsh, jj = pos & vmask;
                const C lf = j > 0 ? pc[c - VEC] : eL[r * VEC + ((jj + shl) & vmask)];
                const C rt = j < bl ? pc[c + VEC] : eR[r * VEC + ((jj + shr) & vmask)];
                orow[e] = lap(pc[c - L], pc[c + L], lf, rt, pm[c], pp[c], pc[c]);
            }
        }
        __syncthreads();                                       // the slot of step z is free
        if (issued < nsteps) {
            if (tid == 0) issue_bulk(issued);
            issue_edges(issued);
            issued++;
        } else {
            st_cp_commit();                                    // keep the group count uniform
        }
    }
    st_cp_wait<0>();
    // after a wait gave up: let the bulk copies still in flight land (bounded) before exiting
    if (lost && tid == 0)
        for (int k = waited; k < issued; k++) wait_bounded(k);
}

// The plane-tile 3D Laplacian where its shape applies (complex fields; tiles of
// TY = min(8 complex64 / 4 complex128, B) rows dividing B and L; the four slots within
// 200 KB of shared memory); cudaErrorNotSupported otherwise, and the caller uses
// stencil3d_lines_kernel.
template <typename S, int TY>
static cudaError_t launch_march_ty(const zm_plan_s *p, const S *in, S *out, S coef, cudaStream_t st) {
    const Geom &g = p->g;
    const size_t smem = (size_t)kMarchSlots * ((TY + 2) * g.L + 2 * TY * g.vec) * sizeof(cpx<S>);
    if (smem > 200 * 1024) return cudaErrorNotSupported;
    auto kern = stencil3d_march_kernel<S, TY>;
    static int attr_done[64];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorNotSupported;
    if (!attr_done[dev]) {
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        if (e != cudaSuccess) return e;
        attr_done[dev] = 1;
    }
    int per_sm = 0, sms = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, smem)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorNotSupported;
    const int64_t cols = g.p * g.p, tiles = g.L / TY;
    // depth chunks: at least four waves of resident CTAs (a short tail), each chunk walking
    // >= 16 depths; its two halo planes are read at the same time by the neighbouring
    // chunk's CTA (next in launch order, walking the other way), mostly from L2
    int64_t chunks = 1;
    while (cols * tiles * chunks < 4 * (int64_t)per_sm * sms && g.n / (chunks * 2) >= 16) chunks *= 2;
    const int zsteps = (int)(g.n / chunks);
    kern<<<(unsigned)(cols * tiles * chunks), 256, smem, st>>>(reinterpret_cast<const cpx<S> *>(in),
                                                               reinterpret_cast<cpx<S> *>(out), g, zsteps, coef,
                                                               p->dev_err);
    return cudaGetLastError();
}
template <typename S>
static cudaError_t launch_march(const zm_plan_s *p, const S *in, S *out, S coef, cudaStream_t st) {
    const Geom &g = p->g;
    const int64_t tymax = sizeof(S) == 4 ? 8 : 4;
    const int64_t ty = g.b < tymax ? g.b : tymax;
    if (g.dim != 3 || g.L % ty || g.b % ty || g.n < 16) return cudaErrorNotSupported;
    if (ty == 8) return launch_march_ty<S, 8>(p, in, out, coef, st);
    if (ty == 4) return launch_march_ty<S, 4>(p, in, out, coef, st);
    if (ty == 2) return launch_march_ty<S, 2>(p, in, out, coef, st);
    return cudaErrorNotSupported;
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
            // four rows of a B-row block per thread (FP32)
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
        } else if (sizeof(S) == 8) {
            // FP64: one row per thread, rows of the same B-row block addressed directly, five
            // CTAs per SM (two rows per thread, 70 registers, were slower: 4.20 -> 4.54 ms at
            // N = 16384 for the three stencils in one launch; four rows 4.34 ms)
            const unsigned g1 = (unsigned)((nvec + threads - 1) / threads);
            if (op == ST_LAPLACE)
                stencil_rows1_kernel<S, NC, ST_LAPLACE><<<g1, threads, 0, st>>>(i, o, o2, o3, p->g, nvec, c, c2, rd);
            else if (op == ST_DX)
                stencil_rows1_kernel<S, NC, ST_DX><<<g1, threads, 0, st>>>(i, o, o2, o3, p->g, nvec, c, c2, rd);
            else if (op == ST_DY)
                stencil_rows1_kernel<S, NC, ST_DY><<<g1, threads, 0, st>>>(i, o, o2, o3, p->g, nvec, c, c2, rd);
            else
                stencil_rows1_kernel<S, NC, ST_ALL><<<g1, threads, 0, st>>>(i, o, o2, o3, p->g, nvec, c, c2, rd);
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
        if (NC == 2) {
            const cudaError_t em = launch_march<S>(p, i, o, c, st);
            if (em == cudaSuccess) count_launch();
            if (em != cudaErrorNotSupported) return em;   // launched (or failed): done
        }
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
