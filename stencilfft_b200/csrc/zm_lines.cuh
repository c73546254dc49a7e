// zm_lines.cuh -- where each global line of an axis pass lives in the field buffers.
#pragma once

#include "zm_common.cuh"

namespace zm {

// Addresses of a line on the vector side (A: chunk c, packed position
// pos = j*VEC + n2, n1 = c*B + j) and on the frequency side (F: chunk
// c = k2 / VP, position pos = k1*VP + k2 % VP):
//   A(c, pos) = a_base + c * a_chunk + (pos >> a_lg) * a_hi + (pos & (2^a_lg - 1))
//               (a_lg = 0: a_hi = a_pos, the stride of pos)
//   F(c, pos) = f_base + c * f_chunk + (pos >> f_lg) * f_hi + (pos & (2^f_lg - 1))
// The 2D intermediate between the x and y passes is either exactly the reference's
// layout after REPACK (lg = 0: element (p, q) of a rank at p * L + q, fft.cu:186) or,
// for the size-specialised complex64 passes, the same layout with G = 2^lg consecutive
// x-frequency rows interleaved, (p, q) at (p / G) * G L + q G + p % G, so that both
// passes move whole 32-byte sectors.  The three-stage passes can instead interleave
// groups of G consecutive y positions, (p, q) at (q / G) * G L + p G + q % G (qint): the
// y pass then writes runs of G elements of its line and the x pass reads its line's
// elements G apart -- the mirror image, used by the inverse transform.
struct LineAddr {
    int64_t a_base, a_chunk, a_pos;
    int a_lg;
    int64_t a_hi;
    int64_t f_base, f_chunk, f_pos;   // f_pos: stride of pos when lg = 0
    int64_t f_hi;
    int f_lg;
};

ZM_DEV LineAddr line_addr(const Geom &g, int kind, int64_t l, int lg = 0, bool qint = false) {
    LineAddr a;
    const int64_t L = g.L, P = g.p, LL = L * L, LLL = LL * L;
    a.a_pos = 1;
    a.a_lg = 0;
    a.f_lg = 0;
    switch (kind) {
    case PASS_X2: {  // line = (rid, q), q = packed position of local row lr
        const int64_t rid = l >> g.logL, q = l & (L - 1);
        const int64_t lr = unpack_pos(q, g.vec, g.logVEC, g.logB);
        a.a_base = (rid * P) * LL + lr * L;       // rank (rid, 0), row lr
        a.a_chunk = LL;                            // next cid
        a.f_base = (rid * P) * LL + (q << lg);     // rank (rid, 0), column q (fft.cu:186)
        a.f_chunk = LL;
        a.f_pos = L;
        a.f_lg = lg;
        a.f_hi = L << lg;
        if (qint && lg > 0) {                      // x-frequency rows p at stride G
            const int64_t G = int64_t{1} << lg;
            a.f_base = (rid * P) * LL + (q >> lg) * (L << lg) + (q & (G - 1));
            a.f_lg = 0;
            a.f_hi = G;
        }
    } break;
    case PASS_Y2: {  // line = (cid, p), p = x-frequency position (row after REPACK)
        const int64_t cid = l >> g.logL, p = l & (L - 1);
        const int64_t G = int64_t{1} << lg;
        a.a_base = cid * LL + (p >> lg) * (L << lg) + (p & (G - 1));   // rank (0, cid), row p
        a.a_chunk = P * LL;                        // next rid
        a.a_pos = G;
        a.f_base = cid * LL + p * L;
        a.f_chunk = a.a_chunk;
        a.f_pos = 1;
        a.f_hi = 1;
        if (qint && lg > 0) {                      // runs of G y positions, G L apart
            a.a_base = cid * LL + p * G;
            a.a_pos = 1;
            a.a_lg = lg;
            a.a_hi = L << lg;
        }
    } break;
    case PASS_X3: {  // line = (did, rid, ld, q)
        const int64_t q = l & (L - 1), ld = (l >> g.logL) & (L - 1), dr = l >> (2 * g.logL);
        const int64_t lr = unpack_pos(q, g.vec, g.logVEC, g.logB);
        a.a_base = dr * P * LLL + (ld * L + lr) * L;
        a.a_chunk = LLL;
        a.f_base = dr * P * LLL + ld * LL + q;     // repack_transpose_xy_3d (fft3d.cu:203-209)
        a.f_chunk = LLL;
        a.f_pos = L;
        a.f_hi = L;
    } break;
    case PASS_Y3: {  // line = (did, cid, p, qd), qd = packed position of depth ld
        const int64_t qd = l & (L - 1), p = (l >> g.logL) & (L - 1), dc = l >> (2 * g.logL);
        const int64_t did = dc >> g.logP, cid = dc & (P - 1);
        const int64_t ld = unpack_pos(qd, g.vec, g.logVEC, g.logB);
        const int64_t r0 = did * P * P + cid;     // rank (did, 0, cid)
        a.a_base = r0 * LLL + (ld * L + p) * L;
        a.a_chunk = P * LLL;                       // next rid
        a.f_base = r0 * LLL + p * L + qd;          // repack_transpose_yz_3d (fft3d.cu:214-220)
        a.f_chunk = P * LLL;
        a.f_pos = LL;
        a.f_hi = LL;
    } break;
    default: {       // PASS_Z3: line = (rid, cid, cy, rx)
        const int64_t rc = l >> (2 * g.logL), rest = l & (LL - 1);
        a.a_base = rc * LLL + rest * L;            // rank (0, rid, cid)
        a.a_chunk = P * P * LLL;                   // next did
        a.f_base = a.a_base;
        a.f_chunk = a.a_chunk;
        a.f_pos = 1;
        a.f_hi = 1;
    } break;
    }
    if (a.a_lg == 0) a.a_hi = a.a_pos;
    return a;
}

}  // namespace zm
