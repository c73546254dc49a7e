// zm_layout.cu -- layout converters, reciprocal-space pointwise operators and
// seeded field generators on the interleaved layouts.
//
// All of them are element-wise maps driven by the index maps of
// zmodel/utils.h: real_to_global (166-170, 193-198) for the real-space layout
// and reciprocal_to_global (265-268, 298-302) for the transform output.
#include <math.h>

#include "zm_common.cuh"
#include "zm_internal.h"

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

template <typename T, bool RECIP, bool TO_NAT>
__global__ void convert_kernel(const cpx<T> *__restrict__ in, cpx<T> *__restrict__ out, const Geom g,
                               int64_t total) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= total) return;
    const int64_t gi = RECIP ? recip_gidx(e, g) : real_gidx(e, g);
    if (TO_NAT) out[gi] = ldg(in + e);
    else out[e] = ldg(in + gi);
}

template <typename T>
static cudaError_t conv_t(const zm_plan_s *p, bool recip, bool to_nat, const void *in, void *out,
                          cudaStream_t st) {
    const int threads = 256;
    const unsigned grid = (unsigned)((p->total + threads - 1) / threads);
    const cpx<T> *i = reinterpret_cast<const cpx<T> *>(in);
    cpx<T> *o = reinterpret_cast<cpx<T> *>(out);
    if (recip) {
        if (to_nat) convert_kernel<T, true, true><<<grid, threads, 0, st>>>(i, o, p->g, p->total);
        else convert_kernel<T, true, false><<<grid, threads, 0, st>>>(i, o, p->g, p->total);
    } else {
        if (to_nat) convert_kernel<T, false, true><<<grid, threads, 0, st>>>(i, o, p->g, p->total);
        else convert_kernel<T, false, false><<<grid, threads, 0, st>>>(i, o, p->g, p->total);
    }
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_convert(const zm_plan_s *p, bool reciprocal, bool to_natural, const void *in,
                           void *out, cudaStream_t st) {
    return p->dtype == 0 ? conv_t<double>(p, reciprocal, to_natural, in, out, st)
                         : conv_t<float>(p, reciprocal, to_natural, in, out, st);
}

// --------------------------------------------------------- spectral operators
template <typename T>
__global__ void spectral_kernel(cpx<T> *__restrict__ d, const Geom g, int64_t total, int op, double a) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= total) return;
    int64_t k0, k1, k2;
    recip_k(e, g, k0, k1, k2);
    const int64_t half = g.n >> 1;
    const double s0 = (double)(k0 >= half ? k0 - g.n : k0);
    const double s1 = (double)(k1 >= half ? k1 - g.n : k1);
    const double s2 = (double)(k2 >= half ? k2 - g.n : k2);
    const double k2sum = s0 * s0 + s1 * s1 + s2 * s2;
    double f;
    if (op == 0) f = exp(-k2sum / (2.0 * a * a));
    else if (op == 1) f = k2sum == 0.0 ? 0.0 : -1.0 / (a * a * k2sum);
    else f = a;
    cpx<T> v = d[e];
    d[e] = {(T)(v.x * f), (T)(v.y * f)};
}

cudaError_t launch_spectral(const zm_plan_s *p, void *data, int op, double a, cudaStream_t st) {
    const int threads = 256;
    const unsigned grid = (unsigned)((p->total + threads - 1) / threads);
    if (p->dtype == 0)
        spectral_kernel<double><<<grid, threads, 0, st>>>(reinterpret_cast<cpx<double> *>(data), p->g,
                                                          p->total, op, a);
    else
        spectral_kernel<float><<<grid, threads, 0, st>>>(reinterpret_cast<cpx<float> *>(data), p->g,
                                                         p->total, op, a);
    count_launch();
    return cudaGetLastError();
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

template <typename T>
__global__ void fill_kernel(cpx<T> *__restrict__ d, const Geom g, int64_t total, int kind, uint64_t seed) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= total) return;
    const uint64_t gi = (uint64_t)real_gidx(e, g);
    double re, im;
    if (kind == 0) {
        re = u01(seed, gi, 0) * 2.0 - 1.0;
        im = u01(seed, gi, 1) * 2.0 - 1.0;
    } else {
        re = gauss(seed, gi, 0);
        im = gauss(seed, gi, 1);
    }
    d[e] = {(T)re, (T)im};
}

cudaError_t launch_fill(const zm_plan_s *p, void *data, int kind, uint64_t seed, cudaStream_t st) {
    const int threads = 256;
    const unsigned grid = (unsigned)((p->total + threads - 1) / threads);
    if (p->dtype == 0)
        fill_kernel<double><<<grid, threads, 0, st>>>(reinterpret_cast<cpx<double> *>(data), p->g,
                                                      p->total, kind, seed);
    else
        fill_kernel<float><<<grid, threads, 0, st>>>(reinterpret_cast<cpx<float> *>(data), p->g,
                                                     p->total, kind, seed);
    count_launch();
    return cudaGetLastError();
}

constexpr int kMaxModes = 64;
struct ModeSet {
    int n;
    double noise;
    uint64_t seed;
    int64_t kx[kMaxModes], ky[kMaxModes];
    double ar[kMaxModes], ai[kMaxModes];
};

template <typename T>
__global__ void modes_kernel(cpx<T> *__restrict__ d, const Geom g, int64_t total, const ModeSet ms) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= total) return;
    const int64_t gi = real_gidx(e, g);
    const int64_t gr = gi >> g.logN, gc = gi & (g.n - 1);
    double re = 0.0, im = 0.0;
    for (int m = 0; m < ms.n; m++) {
        // exact phase (kx x + ky y) mod N, then one sincospi
        const int64_t ph = (ms.kx[m] * gc + ms.ky[m] * gr) & (g.n - 1);
        double s, c;
        sincospi(2.0 * (double)ph / (double)g.n, &s, &c);
        re += ms.ar[m] * c - ms.ai[m] * s;
        im += ms.ar[m] * s + ms.ai[m] * c;
    }
    if (ms.noise != 0.0) {
        re += ms.noise * gauss(ms.seed, (uint64_t)gi, 0);
        im += ms.noise * gauss(ms.seed, (uint64_t)gi, 1);
    }
    d[e] = {(T)re, (T)im};
}

cudaError_t launch_fill_modes(const zm_plan_s *p, void *data, int nmodes, const int64_t *modes,
                              const double *amps, double noise, uint64_t seed, cudaStream_t st) {
    if (nmodes < 0 || nmodes > kMaxModes || p->g.dim != 2) return cudaErrorInvalidValue;
    ModeSet ms;
    ms.n = nmodes;
    ms.noise = noise;
    ms.seed = seed;
    for (int m = 0; m < nmodes; m++) {
        // reduce to [0, N) so the device phase product stays non-negative
        ms.kx[m] = ((modes[2 * m] % p->g.n) + p->g.n) % p->g.n;
        ms.ky[m] = ((modes[2 * m + 1] % p->g.n) + p->g.n) % p->g.n;
        ms.ar[m] = amps[2 * m];
        ms.ai[m] = amps[2 * m + 1];
    }
    const int threads = 256;
    const unsigned grid = (unsigned)((p->total + threads - 1) / threads);
    if (p->dtype == 0)
        modes_kernel<double><<<grid, threads, 0, st>>>(reinterpret_cast<cpx<double> *>(data), p->g,
                                                       p->total, ms);
    else
        modes_kernel<float><<<grid, threads, 0, st>>>(reinterpret_cast<cpx<float> *>(data), p->g,
                                                      p->total, ms);
    count_launch();
    return cudaGetLastError();
}

}  // namespace zm
