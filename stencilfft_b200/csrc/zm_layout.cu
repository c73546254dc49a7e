// zm_layout.cu -- layout converters, reciprocal-space pointwise operators and
// seeded field generators on the interleaved layouts.
//
// All of them are element-wise maps driven by the index maps of
// zmodel/utils.h: real_to_global (166-170, 193-198) for the real-space layout
// and reciprocal_to_global (265-268, 298-302) for the transform output.
#include <math.h>

#include "zm_common.cuh"
#include "zm_index.cuh"
#include "zm_internal.h"

namespace zm {

// Each thread moves CEPT consecutive interleaved elements e: their CEPT gathers (or
// scatters) on the natural side are all in flight before the first use, and the
// interleaved side moves as 16-byte vectors.  (One element per thread kept one 8-byte
// load in flight and waited on it.)  total is a multiple of CEPT (N^dim, N >= 4).
constexpr int CEPT = 4;
// CEPT consecutive elements at a CEPT-aligned index, as 16-byte vectors
template <typename T> ZM_DEV void ld_run(const cpx<T> *p, cpx<T> *v) {
    constexpr int NV = CEPT * (int)sizeof(cpx<T>) / 16;
#pragma unroll
    for (int q = 0; q < NV; q++)
        reinterpret_cast<uint4 *>(v)[q] = __ldg(reinterpret_cast<const uint4 *>(p) + q);
}
template <typename T> ZM_DEV void st_run(cpx<T> *p, const cpx<T> *v) {
    constexpr int NV = CEPT * (int)sizeof(cpx<T>) / 16;
#pragma unroll
    for (int q = 0; q < NV; q++) reinterpret_cast<uint4 *>(p)[q] = reinterpret_cast<const uint4 *>(v)[q];
}
template <typename T, bool RECIP, bool TO_NAT>
__global__ void __launch_bounds__(256) convert_kernel(const cpx<T> *__restrict__ in, cpx<T> *__restrict__ out,
                                                      const Geom g, int64_t total) {
    const int64_t e0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) * CEPT;
    if (e0 >= total) return;
    int64_t gi[CEPT];
#pragma unroll
    for (int i = 0; i < CEPT; i++) gi[i] = RECIP ? recip_gidx(e0 + i, g) : real_gidx(e0 + i, g);
    cpx<T> v[CEPT];
    if (TO_NAT) {
        ld_run(in + e0, v);
#pragma unroll
        for (int i = 0; i < CEPT; i++) out[gi[i]] = v[i];
    } else {
#pragma unroll
        for (int i = 0; i < CEPT; i++) v[i] = ldg(in + gi[i]);
        st_run(out + e0, v);
    }
}

// Reciprocal layout <-> natural order through shared-memory tiles.  In a rank's
// reciprocal array, TB consecutive local rows l2 inside one run of VP hold TB consecutive
// natural k2 (the contiguous natural axis), and TB consecutive positions inside one run of
// VP hold TB consecutive k1 (2D) / k0 (3D), the natural index's slowest axis
// (reciprocal_to_global, utils.h:265-268, 298-302: k = d_ct(id L + d_lp(i)), and
// d_lp / d_ct step k by one along such a run).  So a TB x TB block of (row, position) is
// the transpose of a natural block made of TB runs of TB contiguous elements.  A CTA
// takes SB = 1024 / TB^2 blocks side by side along the positions (TB rows x SB TB
// positions, 1024 elements): it moves the natural side as runs of TB elements and the
// reciprocal side as runs of SB TB through a padded shared-memory tile.  (The element-wise kernel gathered or scattered one element per
// natural row: 38 % of the copy bandwidth for natural -> reciprocal at N = 8192 c64.)
template <typename T, int TB, bool TO_NAT>
__global__ void __launch_bounds__(256) recip_tile_kernel(const cpx<T> *__restrict__ in, cpx<T> *__restrict__ out,
                                                         const Geom g) {
    constexpr int SB = 1024 / (TB * TB), W = SB * TB;   // blocks per CTA, positions per CTA
    __shared__ cpx<T> tile[SB * TB * (TB + 1)];          // [b][i = position][j = row], padded
    const int64_t L = g.L;
    const int logL = g.logL;
    // CTA -> (rank, l1 (3D), row run, position run of W)
    int64_t c = blockIdx.x;
    const int64_t nsig = L / W, nrho = L / TB;
    const int64_t sig = c % nsig;
    c /= nsig;
    const int64_t rho = c % nrho;
    c /= nrho;
    int64_t l1 = 0, r;
    if (g.dim == 3) {
        l1 = c & (L - 1);
        r = c >> logL;
    } else {
        r = c;
    }
    const int64_t cid = r & (g.p - 1);
    const int64_t rid = g.dim == 2 ? r >> g.logP : (r >> g.logP) & (g.p - 1);
    const int64_t did = g.dim == 2 ? 0 : r >> (2 * g.logP);
    const int64_t p0 = rho * TB, q0 = sig * W;
    const int64_t k2base = d_ct(cid * L + d_lp(p0, g), g);
    const int64_t kmid = g.dim == 3 ? d_ct(rid * L + d_lp(l1, g), g) : 0;
    const int64_t xid = g.dim == 2 ? rid : did;
    const int64_t spos = g.dim == 2 ? g.n : g.n * g.n;       // natural stride of the position axis
    const int64_t rbase = g.dim == 2 ? (((r << logL) + p0) << logL) + q0
                                     : ((((r << logL) + l1) << logL) + p0) * L + q0;
    const int tid = threadIdx.x;
    auto nat_addr = [&](int x) {                              // natural side element x of the CTA
        const int b = x / (TB * TB), i = (x / TB) % TB, j = x % TB;
        const int64_t kpos = d_ct(xid * L + d_lp(q0 + (int64_t)b * TB, g), g) + i;
        return (kpos * spos) + kmid * g.n + k2base + j;
    };
    auto tidx = [](int b, int i, int j) { return (b * TB + i) * (TB + 1) + j; };
    // element x = tid + 256 u of the CTA on both sides: consecutive lanes take consecutive
    // elements of a run, so the shared tile (rows of TB + 1) is read and written without
    // bank conflicts on either side and every warp access covers whole runs
    if (!TO_NAT) {
        cpx<T> v[4];
#pragma unroll
        for (int u = 0; u < 4; u++) v[u] = ldg(in + nat_addr(tid + 256 * u));
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int x = tid + 256 * u;
            tile[tidx(x / (TB * TB), (x / TB) % TB, x % TB)] = v[u];
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int x = tid + 256 * u, jr = x / W, pr = x % W;
            out[rbase + (int64_t)jr * L + pr] = tile[tidx(pr / TB, pr % TB, jr)];
        }
    } else {
        cpx<T> v[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int x = tid + 256 * u, jr = x / W, pr = x % W;
            v[u] = ldg(in + rbase + (int64_t)jr * L + pr);
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int x = tid + 256 * u, jr = x / W, pr = x % W;
            tile[tidx(pr / TB, pr % TB, jr)] = v[u];
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int x = tid + 256 * u;
            out[nat_addr(x)] = tile[tidx(x / (TB * TB), (x / TB) % TB, x % TB)];
        }
    }
}

template <typename T, int TB>
static void recip_tiles(const zm_plan_s *p, bool to_nat, const cpx<T> *i, cpx<T> *o, cudaStream_t st) {
    const int64_t L = p->g.L, W = 1024 / TB;
    const int64_t ctas = (p->g.dim == 2 ? 1 : L) * (p->total / (p->g.dim == 2 ? L * L : L * L * L)) * (L / TB) *
                         (L / W);
    if (to_nat) recip_tile_kernel<T, TB, true><<<(unsigned)ctas, 256, 0, st>>>(i, o, p->g);
    else recip_tile_kernel<T, TB, false><<<(unsigned)ctas, 256, 0, st>>>(i, o, p->g);
}

template <typename T>
static cudaError_t conv_t(const zm_plan_s *p, bool recip, bool to_nat, const void *in, void *out,
                          cudaStream_t st) {
    const int threads = 256;
    const int64_t nthr = p->total / CEPT;
    const unsigned grid = (unsigned)((nthr + threads - 1) / threads);
    const cpx<T> *i = reinterpret_cast<const cpx<T> *>(in);
    cpx<T> *o = reinterpret_cast<cpx<T> *>(out);
    // the tiled reciprocal converter where runs of TB >= 4 exist (TB = min(VP, 32) divides
    // VP) and a rank's rows hold whole CTAs (L a multiple of 1024 / TB)
    const int64_t vp = p->g.vp, tb = vp < 32 ? vp : 32;
    if (recip && tb >= 4 && p->g.L % (1024 / tb) == 0) {
        if (tb == 4) recip_tiles<T, 4>(p, to_nat, i, o, st);
        else if (tb == 8) recip_tiles<T, 8>(p, to_nat, i, o, st);
        else if (tb == 16) recip_tiles<T, 16>(p, to_nat, i, o, st);
        else recip_tiles<T, 32>(p, to_nat, i, o, st);
        count_launch();
        return cudaGetLastError();
    }
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
// Each thread scales CEPT consecutive elements.  The multiplier is computed in the
// working precision: FP64 for complex128; FP32 for complex64, where its relative error
// (a few ulp of FP32) stays far inside the complex64 bar, and the FP64 exp / division
// made the kernel issue bound.
template <typename T>
__global__ void __launch_bounds__(256) spectral_kernel(cpx<T> *__restrict__ d, const Geom g, int64_t total, int op,
                                                       double a) {
    const int64_t e0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) * CEPT;
    if (e0 >= total) return;
    cpx<T> v[CEPT];
    ld_run(d + e0, v);
    const int64_t half = g.n >> 1;
    const T inv2a2 = (T)(1.0 / (2.0 * a * a)), inva2 = (T)(1.0 / (a * a)), ta = (T)a;
    // the CEPT elements are consecutive positions of one row; inside a run of VP positions
    // the position axis' frequency (k1 in 2D, k0 in 3D) steps by one and the others stay
    int64_t k0, k1, k2;
    recip_k(e0, g, k0, k1, k2);
    const bool run = g.vp >= CEPT;
#pragma unroll
    for (int i = 0; i < CEPT; i++) {
        if (i > 0) {
            if (!run) recip_k(e0 + i, g, k0, k1, k2);
            else if (g.dim == 2) k1++;
            else k0++;
        }
        const int64_t s0 = k0 >= half ? k0 - g.n : k0;
        const int64_t s1 = k1 >= half ? k1 - g.n : k1;
        const int64_t s2 = k2 >= half ? k2 - g.n : k2;
        const T k2sum = (T)(s0 * s0 + s1 * s1 + s2 * s2);   // exact in FP64; one rounding in FP32
        T f;
        if (op == 0) f = exp(-k2sum * inv2a2);
        else if (op == 1) f = k2sum == (T)0 ? (T)0 : -inva2 / k2sum;
        else f = ta;
        v[i] = {v[i].x * f, v[i].y * f};
    }
    st_run(d + e0, v);
}

cudaError_t launch_spectral(const zm_plan_s *p, void *data, int op, double a, cudaStream_t st) {
    const int threads = 256;
    const unsigned grid = (unsigned)((p->total / CEPT + threads - 1) / threads);
    if (p->dtype == 0)
        spectral_kernel<double><<<grid, threads, 0, st>>>(reinterpret_cast<cpx<double> *>(data), p->g,
                                                          p->total, op, a);
    else
        spectral_kernel<float><<<grid, threads, 0, st>>>(reinterpret_cast<cpx<float> *>(data), p->g,
                                                         p->total, op, a);
    count_launch();
    return cudaGetLastError();
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
