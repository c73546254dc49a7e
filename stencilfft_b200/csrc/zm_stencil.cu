// zm_stencil.cu -- periodic stencils on the interleaved real-space layout.
//
// The reference packs halo rows / vectors on every rank (pack_laplace,
// laplace.cu:172-191), swaps them with host-staged MPI_Sendrecv
// (communicate_laplace, laplace.cu:194-256) and then runs a one-element-per-
// thread kernel that picks each neighbour from its own array or a receive
// buffer (laplace.cu:73-169).  With every virtual rank in one HBM the halo is
// simply the neighbouring rank's array: each thread maps its element to global
// (row, column[, depth]) coordinates, steps one (two) points along the axis
// with periodic wrap, and maps back to (rank, local row, packed column) with the
// block-cyclic maps of zmodel/utils.h:166-214.  The neighbours are accumulated
// in the reference's order (above, below, left, right[, front, back], then the
// centre term), so the 2D Laplacian and dx / dy are bit-identical to it in FP64.
#include "zm_common.cuh"
#include "zm_internal.h"

namespace zm {

struct StencilGeom {
    Geom g;
    int64_t total;   // elements in the field
    int threads_per_elem_shift;
};

// global row/column/depth coordinate of a local (block-cyclic) index, and back
ZM_DEV int64_t l2g(int64_t li, int64_t id, const Geom &g) {   // utils.h:168
    return ((li >> g.logB) << (g.logB + g.logP)) + (id << g.logB) + (li & (g.b - 1));
}
ZM_DEV void g2l(int64_t gi, const Geom &g, int64_t &id, int64_t &li) {  // utils.h:178-180
    id = (gi >> g.logB) & (g.p - 1);
    li = ((gi >> (g.logB + g.logP)) << g.logB) + (gi & (g.b - 1));
}
// packed column position <-> global column (utils.h:122-128 then 169)
ZM_DEV int64_t pos2gc(int64_t pos, int64_t cid, const Geom &g) {
    const int64_t j = pos >> g.logVEC, jj = pos & (g.vec - 1);
    return (jj << (g.logB + g.logP)) + (cid << g.logB) + j;
}
ZM_DEV void gc2pos(int64_t gc, const Geom &g, int64_t &cid, int64_t &pos) {
    cid = (gc >> g.logB) & (g.p - 1);
    pos = ((gc & (g.b - 1)) << g.logVEC) + (gc >> (g.logB + g.logP));
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

// NC = scalar components per element (2 complex, 1 real); S = scalar type.
template <typename S, int NC, int OP, int DIM>
__global__ void __launch_bounds__(256) stencil_kernel(const S *__restrict__ in, S *__restrict__ out,
                                                      const Geom g, int64_t total, S coef) {
    using O = ops<S>;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= total) return;
    const int64_t L = g.L, LL = L * L;
    const int64_t N = g.n;
    int64_t rank, lr, ld = 0, pos, rid, cid, did = 0;
    if (DIM == 2) {
        rank = e >> (2 * g.logL);
        lr = (e >> g.logL) & (L - 1);
        rid = rank >> g.logP;
        cid = rank & (g.p - 1);
    } else {
        rank = e >> (3 * g.logL);
        ld = (e >> (2 * g.logL)) & (L - 1);
        lr = (e >> g.logL) & (L - 1);
        did = rank >> (2 * g.logP);
        rid = (rank >> g.logP) & (g.p - 1);
        cid = rank & (g.p - 1);
    }
    pos = e & (L - 1);
    const int64_t gr = l2g(lr, rid, g);
    const int64_t gc = pos2gc(pos, cid, g);
    const int64_t gd = DIM == 3 ? l2g(ld, did, g) : 0;
    const int64_t P = g.p;
    auto rank_of = [&](int64_t d_, int64_t r_, int64_t c_) {
        return DIM == 2 ? r_ * P + c_ : (d_ * P + r_) * P + c_;
    };
    auto addr = [&](int64_t rk, int64_t ld_, int64_t lr_, int64_t pos_) {
        return DIM == 2 ? (rk << (2 * g.logL)) + lr_ * L + pos_
                        : (rk << (3 * g.logL)) + ld_ * LL + lr_ * L + pos_;
    };
    // neighbour along rows (y) at global row gr + d
    auto nb_row = [&](int64_t d) {
        int64_t id, li;
        g2l((gr + d + N) & (N - 1), g, id, li);
        return addr(rank_of(did, id, cid), ld, li, pos);
    };
    auto nb_col = [&](int64_t d) {
        int64_t id, ps;
        gc2pos((gc + d + N) & (N - 1), g, id, ps);
        return addr(rank_of(did, rid, id), ld, lr, ps);
    };
    auto nb_dep = [&](int64_t d) {
        int64_t id, li;
        g2l((gd + d + N) & (N - 1), g, id, li);
        return addr(rank_of(id, rid, cid), li, lr, pos);
    };
#pragma unroll
    for (int q = 0; q < NC; q++) {
        auto ld_ = [&](int64_t a) { return __ldg(in + a * NC + q); };
        S res;
        if (OP == ST_LAPLACE) {
            // laplace.cu:91-168 / laplace3d.cu:98-224 accumulation order
            S s = O::add((S)0, ld_(nb_row(-1)));   // scratch = {0,0}; scratch += above
            s = O::add(s, ld_(nb_row(1)));
            s = O::add(s, ld_(nb_col(-1)));
            s = O::add(s, ld_(nb_col(1)));
            if (DIM == 3) {
                s = O::add(s, ld_(nb_dep(-1)));
                s = O::add(s, ld_(nb_dep(1)));
            }
            s = O::fmaop((S)(-2 * DIM), ld_(e), s);
            res = O::mul(s, coef);       // coef = 1/h^2 (1 reproduces the reference)
        } else {
            // dx.cu:26-79 / dy.cu:34-100: ((-8 f[-1] + f[-2]) + 8 f[+1]) - f[+2], then / (12 delta)
            auto nb = [&](int64_t d) { return OP == ST_DX ? nb_col(d) : nb_row(d); };
            S s = O::add((S)0, O::mul(ld_(nb(-1)), (S)-8));
            s = O::add(s, ld_(nb(-2)));
            s = O::add(s, O::mul(ld_(nb(1)), (S)8));
            s = O::sub(s, ld_(nb(2)));
            res = O::div(s, O::mul((S)12, coef));   // coef = delta
        }
        out[e * NC + q] = res;
    }
}

template <typename S, int NC>
static cudaError_t launch_s(const zm_plan_s *p, int op, const void *in, void *out, double coef,
                            cudaStream_t st) {
    const int64_t total = p->total;
    const int threads = 256;
    const unsigned grid = (unsigned)((total + threads - 1) / threads);
    const S *i = reinterpret_cast<const S *>(in);
    S *o = reinterpret_cast<S *>(out);
    const S c = (S)coef;
    if (p->g.dim == 2) {
        if (op == ST_LAPLACE) stencil_kernel<S, NC, ST_LAPLACE, 2><<<grid, threads, 0, st>>>(i, o, p->g, total, c);
        else if (op == ST_DX) stencil_kernel<S, NC, ST_DX, 2><<<grid, threads, 0, st>>>(i, o, p->g, total, c);
        else stencil_kernel<S, NC, ST_DY, 2><<<grid, threads, 0, st>>>(i, o, p->g, total, c);
    } else {
        if (op != ST_LAPLACE) return cudaErrorInvalidValue;
        stencil_kernel<S, NC, ST_LAPLACE, 3><<<grid, threads, 0, st>>>(i, o, p->g, total, c);
    }
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_stencil(const zm_plan_s *p, int op, bool real_field, const void *in, void *out,
                           double coef, cudaStream_t st) {
    if (p->dtype == 0) {
        return real_field ? launch_s<double, 1>(p, op, in, out, coef, st)
                          : launch_s<double, 2>(p, op, in, out, coef, st);
    }
    return real_field ? launch_s<float, 1>(p, op, in, out, coef, st)
                      : launch_s<float, 2>(p, op, in, out, coef, st);
}

}  // namespace zm
