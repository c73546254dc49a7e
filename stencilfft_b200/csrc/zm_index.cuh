// zm_index.cuh -- device forms of the reference's index maps (zmodel/utils.h) on the
// interleaved layouts, and the counter-based field generators.
#pragma once

#include "zm_common.cuh"
#include "zm_plan.h"

namespace zm {

// lp / ct of utils.h:232-241 on powers of two
ZM_DEV int64_t d_lp(int64_t i, const Geom &g) { return (i >> g.logVP) + ((i & (g.vp - 1)) << g.logM); }
ZM_DEV int64_t d_ct(int64_t q, const Geom &g) { return ((q & (g.m - 1)) << g.logVEC) + (q >> g.logM); }

ZM_DEV int64_t d_l2g(int64_t li, int64_t id, const Geom &g) {
    return ((li >> g.logB) << (g.logB + g.logP)) + (id << g.logB) + (li & (g.b - 1));
}
ZM_DEV int64_t d_pos2gc(int64_t pos, int64_t cid, const Geom &g) {
    const int64_t j = pos >> g.logVEC, jj = pos & (g.vec - 1);
    return (jj << (g.logB + g.logP)) + (cid << g.logB) + j;
}

struct Coords { int64_t r, l1, l2, pos, did, rid, cid; };

ZM_DEV Coords coords(int64_t e, const Geom &g) {
    Coords c;
    const int64_t L = g.L;
    c.pos = e & (L - 1);
    if (g.dim == 2) {
        c.r = e >> (2 * g.logL);
        c.l2 = (e >> g.logL) & (L - 1);   // local row
        c.l1 = 0;
        c.did = 0;
        c.rid = c.r >> g.logP;
        c.cid = c.r & (g.p - 1);
    } else {
        c.r = e >> (3 * g.logL);
        c.l1 = (e >> (2 * g.logL)) & (L - 1);  // local depth
        c.l2 = (e >> g.logL) & (L - 1);        // local row
        c.did = c.r >> (2 * g.logP);
        c.rid = (c.r >> g.logP) & (g.p - 1);
        c.cid = c.r & (g.p - 1);
    }
    return c;
}

// global linear index held by interleaved element e of the real-space layout
ZM_DEV int64_t real_gidx(int64_t e, const Geom &g) {
    Coords c = coords(e, g);
    const int64_t gc = d_pos2gc(c.pos, c.cid, g);
    const int64_t gr = d_l2g(c.l2, c.rid, g);
    if (g.dim == 2) return (gr << g.logN) + gc;
    const int64_t gd = d_l2g(c.l1, c.did, g);
    return (((gd << g.logN) + gr) << g.logN) + gc;
}

// frequency indices held by element e of the reciprocal layout
ZM_DEV void recip_k(int64_t e, const Geom &g, int64_t &k0, int64_t &k1, int64_t &k2) {
    Coords c = coords(e, g);
    const int64_t L = g.L;
    if (g.dim == 2) {   // (ky, kx): kx from the local row, ky from the local column
        k2 = d_ct(c.cid * L + d_lp(c.l2, g), g);
        k1 = d_ct(c.rid * L + d_lp(c.pos, g), g);
        k0 = 0;
    } else {            // (kd, kr, kc)
        k2 = d_ct(c.cid * L + d_lp(c.l2, g), g);
        k1 = d_ct(c.rid * L + d_lp(c.l1, g), g);
        k0 = d_ct(c.did * L + d_lp(c.pos, g), g);
    }
}
ZM_DEV int64_t recip_gidx(int64_t e, const Geom &g) {
    int64_t k0, k1, k2;
    recip_k(e, g, k0, k1, k2);
    return g.dim == 2 ? (k1 << g.logN) + k2 : (((k0 << g.logN) + k1) << g.logN) + k2;
}

// ---------------------------------------------------------------- generators
// Counter-based: u = splitmix64(seed * 2^40 ^ (2 g + comp)), the same stream the
// oracle draws from, so any subset of a field can be regenerated on the host.
ZM_DEV uint64_t splitmix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
ZM_DEV double u01(uint64_t seed, uint64_t gi, uint64_t comp) {
    return (double)(splitmix64((seed << 40) ^ (2 * gi + comp)) >> 11) * (1.0 / 9007199254740992.0);
}
ZM_DEV double gauss(uint64_t seed, uint64_t gi, int comp) {
    const double u1 = u01(seed, gi, comp), u2 = u01(seed, gi, comp + 2);
    return sqrt(-2.0 * log(1.0 - u1)) * cospi(2.0 * u2);
}

}  // namespace zm
