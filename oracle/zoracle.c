/*
 * zoracle.c -- CPU oracle for the interleaved block-cyclic FFT / stencil path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file restates, in plain C (FP64), the
 * algorithm of StencilFFT's zmodel so that the CUDA product path can be
 * checked against it.  It is never linked into the product library; only the
 * tests, the smoke check and the bench's CPU-baseline leg load it.
 *
 * Every P x P (P^3) process of the reference is held here as a "virtual rank":
 * one contiguous buffer of P^2 (P^3) rank sub-buffers in id order
 * (2D id = rid*P + cid, 3D id = did*P^2 + rid*P + cid; zmodel/transforms/fft.cu:563-566,
 * zmodel/transforms/fft3d.cu:676-679), each rank holding exactly the reference's
 * rank-local L x L (L^3) array.  The MPI All-to-All and halo Sendrecv calls become
 * copies between those sub-buffers.  Each function names the reference lines it
 * follows.  Compile with -ffp-contract=off so FP64 products round like the
 * reference's separate multiply/add.
 *
 * Parity pin: index maps and the ramp fixture are checked bit-exactly against the
 * reference's own utils.h / utils.cu compiled on the host (oracle/_ref), and the
 * transforms against an independent FP64 FFT (numpy pocketfft) through those maps.
 */
#define _GNU_SOURCE
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct { double x, y; } zc;

/* ---------------------------------------------------------------- config */

typedef struct {
    int dim;       /* 2 or 3 */
    int64_t n;     /* N_DIM */
    int64_t b;     /* B_DIM */
    int64_t p;     /* P_DIM */
    int64_t L;     /* LOCAL_DIM = N/P            utils.h:47 */
    int64_t vec;   /* VEC = L/B                  utils.h:60 */
    int64_t vp;    /* VEC/P  (plan1 stride)      fft_host_plans.h:44-48 */
    int64_t m;     /* B*P    (plan1 length)      fft_host_plans.h:43 */
    int64_t ranks; /* P^2 or P^3 */
    int64_t rank_elems; /* L^2 or L^3 */
} cfg_t;

static int mkcfg(int dim, int64_t n, int64_t b, int64_t p, cfg_t *c) {
    if ((dim != 2 && dim != 3) || n <= 0 || b <= 0 || p <= 0) return -1;
    if (n % p) return -1;
    c->dim = dim; c->n = n; c->b = b; c->p = p;
    c->L = n / p;
    if (c->L % b) return -1;
    c->vec = c->L / b;
    if (c->vec % p) return -1;
    c->vp = c->vec / p;
    c->m = b * p;
    c->ranks = dim == 2 ? p * p : p * p * p;
    c->rank_elems = dim == 2 ? c->L * c->L : c->L * c->L * c->L;
    return 0;
}

int zo_check_config(int dim, int64_t n, int64_t b, int64_t p) {
    cfg_t c;
    return mkcfg(dim, n, b, p, &c);
}

/* ---------------------------------------------------------- index maps */

/* utils.h:122-124 */
static inline int64_t p2bc(const cfg_t *c, int64_t pc) { return pc / c->vec + (pc % c->vec) * c->b; }
/* utils.h:126-128 */
static inline int64_t bc2p(const cfg_t *c, int64_t bc) { return (bc % c->b) * c->vec + bc / c->b; }
/* utils.h:232-236 */
static inline int64_t lp(const cfg_t *c, int64_t i) { return i / c->vp + (i % c->vp) * c->m; }
/* utils.h:238-241 */
static inline int64_t ct(const cfg_t *c, int64_t q) { return (q % c->m) * c->vec + q / c->m; }
/* utils.h:243-247 */
static inline int64_t lp_inv(const cfg_t *c, int64_t j) { return (j % c->m) * c->vp + j / c->m; }
/* utils.h:249-252 */
static inline int64_t ct_inv(const cfg_t *c, int64_t k) { return (k % c->vec) * c->m + k / c->vec; }

/* Scalar index-map entry points, same argument order as utils.h. */
int zo_packed_to_block_cyclic(int dim, int64_t n, int64_t b, int64_t p, int64_t pc, int64_t *out) {
    cfg_t c; if (mkcfg(dim, n, b, p, &c)) return -1; *out = p2bc(&c, pc); return 0;
}
int zo_block_cyclic_to_packed(int dim, int64_t n, int64_t b, int64_t p, int64_t bc, int64_t *out) {
    cfg_t c; if (mkcfg(dim, n, b, p, &c)) return -1; *out = bc2p(&c, bc); return 0;
}

/* utils.h:166-170 */
static void real_to_global(const cfg_t *c, int64_t rid, int64_t cid, int64_t lr, int64_t lc,
                           int64_t *gr, int64_t *gc) {
    int64_t bcc = p2bc(c, lc);
    *gr = (lr / c->b) * c->b * c->p + rid * c->b + (lr % c->b);
    *gc = (bcc / c->b) * c->b * c->p + cid * c->b + (bcc % c->b);
}
/* utils.h:177-186 */
static void global_to_real(const cfg_t *c, int64_t gr, int64_t gc, int64_t *rid, int64_t *cid,
                           int64_t *lr, int64_t *lc) {
    *rid = (gr / c->b) % c->p;
    *lr = (gr / (c->b * c->p)) * c->b + (gr % c->b);
    *cid = (gc / c->b) % c->p;
    int64_t bcc = (gc / (c->b * c->p)) * c->b + (gc % c->b);
    *lc = bc2p(c, bcc);
}
/* utils.h:193-198 */
static void real_to_global_3d(const cfg_t *c, int64_t rid, int64_t cid, int64_t did, int64_t ld,
                              int64_t lr, int64_t lc, int64_t *gd, int64_t *gr, int64_t *gc) {
    int64_t bcc = p2bc(c, lc);
    *gd = (ld / c->b) * c->b * c->p + did * c->b + (ld % c->b);
    *gr = (lr / c->b) * c->b * c->p + rid * c->b + (lr % c->b);
    *gc = (bcc / c->b) * c->b * c->p + cid * c->b + (bcc % c->b);
}
/* utils.h:204-214 */
static void global_to_real_3d(const cfg_t *c, int64_t gd, int64_t gr, int64_t gc, int64_t *rid,
                              int64_t *cid, int64_t *did, int64_t *ld, int64_t *lr, int64_t *lc) {
    *did = (gd / c->b) % c->p;
    *ld = (gd / (c->b * c->p)) * c->b + (gd % c->b);
    *rid = (gr / c->b) % c->p;
    *lr = (gr / (c->b * c->p)) * c->b + (gr % c->b);
    *cid = (gc / c->b) % c->p;
    int64_t bcc = (gc / (c->b * c->p)) * c->b + (gc % c->b);
    *lc = bc2p(c, bcc);
}
/* utils.h:265-268 */
static void reciprocal_to_global(const cfg_t *c, int64_t rid, int64_t cid, int64_t lr, int64_t lc,
                                 int64_t *ky, int64_t *kx) {
    *kx = ct(c, cid * c->L + lp(c, lr));
    *ky = ct(c, rid * c->L + lp(c, lc));
}
/* utils.h:274-282 */
static void global_to_reciprocal(const cfg_t *c, int64_t ky, int64_t kx, int64_t *rid, int64_t *cid,
                                 int64_t *lr, int64_t *lc) {
    int64_t px = ct_inv(c, kx);
    *cid = px / c->L;
    *lr = lp_inv(c, px % c->L);
    int64_t py = ct_inv(c, ky);
    *rid = py / c->L;
    *lc = lp_inv(c, py % c->L);
}
/* utils.h:298-302 */
static void reciprocal_to_global_3d(const cfg_t *c, int64_t rid, int64_t cid, int64_t did, int64_t ld,
                                    int64_t lr, int64_t lc, int64_t *kd, int64_t *kr, int64_t *kc) {
    *kc = ct(c, cid * c->L + lp(c, lr));
    *kr = ct(c, rid * c->L + lp(c, ld));
    *kd = ct(c, did * c->L + lp(c, lc));
}
/* utils.h:308-320 */
static void global_to_reciprocal_3d(const cfg_t *c, int64_t kd, int64_t kr, int64_t kc, int64_t *rid,
                                    int64_t *cid, int64_t *did, int64_t *ld, int64_t *lr, int64_t *lc) {
    int64_t pc = ct_inv(c, kc);
    *cid = pc / c->L;
    *lr = lp_inv(c, pc % c->L);
    int64_t pr = ct_inv(c, kr);
    *rid = pr / c->L;
    *ld = lp_inv(c, pr % c->L);
    int64_t pd = ct_inv(c, kd);
    *did = pd / c->L;
    *lc = lp_inv(c, pd % c->L);
}

/* Exported scalar maps (one call = one index), same semantics as utils.h. */
int zo_real_to_global(int64_t n, int64_t b, int64_t p, int64_t rid, int64_t cid, int64_t lr,
                      int64_t lc, int64_t *gr, int64_t *gc) {
    cfg_t c; if (mkcfg(2, n, b, p, &c)) return -1;
    real_to_global(&c, rid, cid, lr, lc, gr, gc); return 0;
}
int zo_global_to_real(int64_t n, int64_t b, int64_t p, int64_t gr, int64_t gc, int64_t *rid,
                      int64_t *cid, int64_t *lr, int64_t *lc) {
    cfg_t c; if (mkcfg(2, n, b, p, &c)) return -1;
    global_to_real(&c, gr, gc, rid, cid, lr, lc); return 0;
}
int zo_reciprocal_to_global(int64_t n, int64_t b, int64_t p, int64_t rid, int64_t cid, int64_t lr,
                            int64_t lc, int64_t *ky, int64_t *kx) {
    cfg_t c; if (mkcfg(2, n, b, p, &c)) return -1;
    reciprocal_to_global(&c, rid, cid, lr, lc, ky, kx); return 0;
}
int zo_global_to_reciprocal(int64_t n, int64_t b, int64_t p, int64_t ky, int64_t kx, int64_t *rid,
                            int64_t *cid, int64_t *lr, int64_t *lc) {
    cfg_t c; if (mkcfg(2, n, b, p, &c)) return -1;
    global_to_reciprocal(&c, ky, kx, rid, cid, lr, lc); return 0;
}
int zo_lp(int64_t n, int64_t b, int64_t p, int64_t i, int64_t *out) {
    cfg_t c; if (mkcfg(2, n, b, p, &c)) return -1; *out = lp(&c, i); return 0;
}
int zo_ct(int64_t n, int64_t b, int64_t p, int64_t i, int64_t *out) {
    cfg_t c; if (mkcfg(2, n, b, p, &c)) return -1; *out = ct(&c, i); return 0;
}
int zo_lp_inv(int64_t n, int64_t b, int64_t p, int64_t i, int64_t *out) {
    cfg_t c; if (mkcfg(2, n, b, p, &c)) return -1; *out = lp_inv(&c, i); return 0;
}
int zo_ct_inv(int64_t n, int64_t b, int64_t p, int64_t i, int64_t *out) {
    cfg_t c; if (mkcfg(2, n, b, p, &c)) return -1; *out = ct_inv(&c, i); return 0;
}

/*
 * Whole-grid maps: for every element of the interleaved buffer (rank-major,
 * then the rank-local array) write the global linear index of the real-space
 * point it holds (gr*N + gc, or (gd*N + gr)*N + gc in 3D) -- real layout --
 * or of the frequency it holds (ky*N + kx, (kd*N + kr)*N + kc) -- reciprocal
 * layout.  These drive the natural <-> interleaved conversions in the tests.
 */
int zo_real_layout_map(int dim, int64_t n, int64_t b, int64_t p, int64_t *gidx) {
    cfg_t c; if (mkcfg(dim, n, b, p, &c)) return -1;
    const int64_t L = c.L;
    #pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < c.ranks; r++) {
        int64_t did = dim == 3 ? r / (c.p * c.p) : 0;
        int64_t rid = dim == 3 ? (r % (c.p * c.p)) / c.p : r / c.p;
        int64_t cid = r % c.p;
        int64_t *o = gidx + r * c.rank_elems;
        if (dim == 2) {
            for (int64_t lr = 0; lr < L; lr++)
                for (int64_t lc = 0; lc < L; lc++) {
                    int64_t gr, gc; real_to_global(&c, rid, cid, lr, lc, &gr, &gc);
                    o[lr * L + lc] = gr * n + gc;
                }
        } else {
            for (int64_t ld = 0; ld < L; ld++)
                for (int64_t lr = 0; lr < L; lr++)
                    for (int64_t lc = 0; lc < L; lc++) {
                        int64_t gd, gr, gc;
                        real_to_global_3d(&c, rid, cid, did, ld, lr, lc, &gd, &gr, &gc);
                        o[(ld * L + lr) * L + lc] = (gd * n + gr) * n + gc;
                    }
        }
    }
    return 0;
}

int zo_reciprocal_layout_map(int dim, int64_t n, int64_t b, int64_t p, int64_t *kidx) {
    cfg_t c; if (mkcfg(dim, n, b, p, &c)) return -1;
    const int64_t L = c.L;
    #pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < c.ranks; r++) {
        int64_t did = dim == 3 ? r / (c.p * c.p) : 0;
        int64_t rid = dim == 3 ? (r % (c.p * c.p)) / c.p : r / c.p;
        int64_t cid = r % c.p;
        int64_t *o = kidx + r * c.rank_elems;
        if (dim == 2) {
            for (int64_t lr = 0; lr < L; lr++)
                for (int64_t lc = 0; lc < L; lc++) {
                    int64_t ky, kx; reciprocal_to_global(&c, rid, cid, lr, lc, &ky, &kx);
                    o[lr * L + lc] = ky * n + kx;
                }
        } else {
            for (int64_t ld = 0; ld < L; ld++)
                for (int64_t lr = 0; lr < L; lr++)
                    for (int64_t lc = 0; lc < L; lc++) {
                        int64_t kd, kr, kc;
                        reciprocal_to_global_3d(&c, rid, cid, did, ld, lr, lc, &kd, &kr, &kc);
                        o[(ld * L + lr) * L + lc] = (kd * n + kr) * n + kc;
                    }
        }
    }
    return 0;
}

/* Inverse whole-grid maps through global_to_real / global_to_reciprocal:
 * for every global linear index, the interleaved-buffer position holding it. */
int zo_real_layout_inverse_map(int dim, int64_t n, int64_t b, int64_t p, int64_t *pos) {
    cfg_t c; if (mkcfg(dim, n, b, p, &c)) return -1;
    const int64_t L = c.L;
    if (dim == 2) {
        #pragma omp parallel for schedule(static)
        for (int64_t gr = 0; gr < n; gr++)
            for (int64_t gc = 0; gc < n; gc++) {
                int64_t rid, cid, lr, lc; global_to_real(&c, gr, gc, &rid, &cid, &lr, &lc);
                pos[gr * n + gc] = (rid * c.p + cid) * c.rank_elems + lr * L + lc;
            }
    } else {
        #pragma omp parallel for schedule(static)
        for (int64_t gd = 0; gd < n; gd++)
            for (int64_t gr = 0; gr < n; gr++)
                for (int64_t gc = 0; gc < n; gc++) {
                    int64_t rid, cid, did, ld, lr, lc;
                    global_to_real_3d(&c, gd, gr, gc, &rid, &cid, &did, &ld, &lr, &lc);
                    pos[(gd * n + gr) * n + gc] =
                        ((did * c.p + rid) * c.p + cid) * c.rank_elems + (ld * L + lr) * L + lc;
                }
    }
    return 0;
}

int zo_reciprocal_layout_inverse_map(int dim, int64_t n, int64_t b, int64_t p, int64_t *pos) {
    cfg_t c; if (mkcfg(dim, n, b, p, &c)) return -1;
    const int64_t L = c.L;
    if (dim == 2) {
        #pragma omp parallel for schedule(static)
        for (int64_t ky = 0; ky < n; ky++)
            for (int64_t kx = 0; kx < n; kx++) {
                int64_t rid, cid, lr, lc; global_to_reciprocal(&c, ky, kx, &rid, &cid, &lr, &lc);
                pos[ky * n + kx] = (rid * c.p + cid) * c.rank_elems + lr * L + lc;
            }
    } else {
        #pragma omp parallel for schedule(static)
        for (int64_t kd = 0; kd < n; kd++)
            for (int64_t kr = 0; kr < n; kr++)
                for (int64_t kc = 0; kc < n; kc++) {
                    int64_t rid, cid, did, ld, lr, lc;
                    global_to_reciprocal_3d(&c, kd, kr, kc, &rid, &cid, &did, &ld, &lr, &lc);
                    pos[(kd * n + kr) * n + kc] =
                        ((did * c.p + rid) * c.p + cid) * c.rank_elems + (ld * L + lr) * L + lc;
                }
    }
    return 0;
}

/* ------------------------------------------------------------- fixtures */

/* utils.h:99-108: packed[i*L + j*VEC + jj] = block_cyclic[i*L + j + jj*B] */
static void vector_pack(const cfg_t *c, const zc *bcy, zc *packed, int64_t rows) {
    for (int64_t i = 0; i < rows; i++)
        for (int64_t j = 0; j < c->b; j++)
            for (int64_t jj = 0; jj < c->vec; jj++)
                packed[i * c->L + j * c->vec + jj] = bcy[i * c->L + j + jj * c->b];
}
/* utils.h:110-119 */
static void vector_unpack(const cfg_t *c, const zc *packed, zc *bcy, int64_t rows) {
    for (int64_t i = 0; i < rows; i++)
        for (int64_t j = 0; j < c->b; j++)
            for (int64_t jj = 0; jj < c->vec; jj++)
                bcy[i * c->L + j + jj * c->b] = packed[i * c->L + j * c->vec + jj];
}

int zo_vector_pack(int dim, int64_t n, int64_t b, int64_t p, const double *bcy, double *packed,
                   int64_t rows) {
    cfg_t c; if (mkcfg(dim, n, b, p, &c)) return -1;
    vector_pack(&c, (const zc *)bcy, (zc *)packed, rows); return 0;
}
int zo_vector_unpack(int dim, int64_t n, int64_t b, int64_t p, const double *packed, double *bcy,
                     int64_t rows) {
    cfg_t c; if (mkcfg(dim, n, b, p, &c)) return -1;
    vector_unpack(&c, (const zc *)packed, (zc *)bcy, rows); return 0;
}

/* utils.cu:9-36 (2D) and utils.cu:43-78 (3D): the deterministic ramp
 * value = global linear index, imag 0, built block-cyclic then vector-packed,
 * for every virtual rank. */
int zo_init_ramp(int dim, int64_t n, int64_t b, int64_t p, double *out) {
    cfg_t c; if (mkcfg(dim, n, b, p, &c)) return -1;
    const int64_t L = c.L, B = c.b, P = c.p, N = c.n, nb = L / B;
    #pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < c.ranks; r++) {
        int64_t did = dim == 3 ? r / (P * P) : 0;
        int64_t rid = dim == 3 ? (r % (P * P)) / P : r / P;
        int64_t cid = r % P;
        zc *bcy = (zc *)malloc(sizeof(zc) * c.rank_elems);
        zc *o = (zc *)out + r * c.rank_elems;
        if (dim == 2) {
            int64_t offset = cid * B + rid * (N * B);
            for (int64_t i = 0; i < nb; i++)
                for (int64_t ii = 0; ii < B; ii++)
                    for (int64_t j = 0; j < nb; j++)
                        for (int64_t jj = 0; jj < B; jj++) {
                            int64_t ai = (i * B * nb * B) + (ii * nb * B) + (j * B) + jj;
                            double v = (double)((i * N * B * P) + (ii * N) + (j * B * P) + jj + offset);
                            bcy[ai].x = v; bcy[ai].y = 0.0;
                        }
            vector_pack(&c, bcy, o, L);
        } else {
            int64_t offset = cid * B + rid * (N * B) + did * (N * N * B);
            for (int64_t i = 0; i < nb; i++)
                for (int64_t ii = 0; ii < B; ii++)
                    for (int64_t j = 0; j < nb; j++)
                        for (int64_t jj = 0; jj < B; jj++)
                            for (int64_t k = 0; k < nb; k++)
                                for (int64_t kk = 0; kk < B; kk++) {
                                    int64_t ai = (i * B * L * L) + (ii * L * L) + (j * B * L) + (jj * L) +
                                                 (k * B) + kk;
                                    double v = (double)((i * N * N * B * P) + (ii * N * N) +
                                                        (j * N * B * P) + (jj * N) + (k * B * P) + kk +
                                                        offset);
                                    bcy[ai].x = v; bcy[ai].y = 0.0;
                                }
            vector_pack(&c, bcy, o, L * L);
        }
        free(bcy);
    }
    return 0;
}

/* Counter-based generator shared with the device generator:
 * u = splitmix64(seed * 2^40 ^ (2*g + comp)); uniform[-1,1) = ((u >> 11) * 2^-53) * 2 - 1.
 * Gaussian = Box-Muller on the uniforms of counter streams comp and comp + 2. */
static inline uint64_t splitmix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static inline double u01(uint64_t seed, uint64_t g, uint64_t comp) {
    uint64_t u = splitmix64((seed << 40) ^ (2 * g + comp));
    return (double)(u >> 11) * (1.0 / 9007199254740992.0);
}
/* natural-order field of `count` complex values, global index g = first + i */
int zo_fill_uniform(uint64_t seed, int64_t first, int64_t count, double *out) {
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < count; i++) {
        uint64_t g = (uint64_t)(first + i);
        out[2 * i] = u01(seed, g, 0) * 2.0 - 1.0;
        out[2 * i + 1] = u01(seed, g, 1) * 2.0 - 1.0;
    }
    return 0;
}
int zo_fill_gaussian(uint64_t seed, int64_t first, int64_t count, double *out) {
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < count; i++) {
        uint64_t g = (uint64_t)(first + i);
        for (int comp = 0; comp < 2; comp++) {
            double u1 = u01(seed, g, comp), u2 = u01(seed, g, comp + 2);
            double r = sqrt(-2.0 * log(1.0 - u1));
            out[2 * i + comp] = r * cos(2.0 * M_PI * u2);
        }
    }
    return 0;
}

/* ------------------------------------------------------ complex helpers */

/* utils.h:91-93 */
static inline zc cmul(zc a, zc b) { zc r = {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; return r; }

/* ------------------------------------------------------ twiddle tables */

/* fft.cu:37-73 (and fft3d.cu:36-68, the same table repeated per depth):
 * tw[lr*L + f_row + f_col*VP] = exp(sign * 2 pi i (f_row + id*VP) * f_col / N)
 * The table is redundant over lr; this restatement keeps one L-row. */
static void init_twiddle_row(const cfg_t *c, int64_t id, int inverse, zc *row) {
    const int64_t stride = c->vp;
    for (int64_t fr = 0; fr < stride; fr++)
        for (int64_t fc = 0; fc < c->L / stride; fc++) {
            double k = (double)(fr + id * stride);
            double l = (double)fc;
            double th = inverse ? 2 * M_PI * k * l / (double)c->n : -2 * M_PI * k * l / (double)c->n;
            row[fr + fc * stride].x = cos(th);
            row[fr + fc * stride].y = sin(th);
        }
}

/* ------------------------------------------------------- 1-D FFT (FP64) */

/* In-place radix-2 decimation-in-time FFT of length n (power of two) over
 * elements x[s*i], i < n.  sign = -1 forward, +1 inverse, unnormalised
 * (cufftExecZ2Z semantics at the reference's call sites, fft.cu:209,257). */
static void fft_pow2(zc *x, int64_t n, int64_t s, int sign, const zc *w /* w[k] = e^{sign 2pi i k / n}, k < n/2 */) {
    if (n <= 1) return;
    for (int64_t i = 1, j = 0; i < n; i++) {
        int64_t bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) { zc t = x[i * s]; x[i * s] = x[j * s]; x[j * s] = t; }
    }
    for (int64_t len = 2; len <= n; len <<= 1) {
        int64_t half = len >> 1, step = n / len;
        for (int64_t i = 0; i < n; i += len)
            for (int64_t k = 0; k < half; k++) {
                zc u = x[(i + k) * s];
                zc v = cmul(x[(i + k + half) * s], w[k * step]);
                x[(i + k) * s].x = u.x + v.x; x[(i + k) * s].y = u.y + v.y;
                x[(i + k + half) * s].x = u.x - v.x; x[(i + k + half) * s].y = u.y - v.y;
            }
    }
    (void)sign;
}

static zc *make_roots(int64_t n, int sign) {
    int64_t h = n / 2 > 0 ? n / 2 : 1;
    zc *w = (zc *)malloc(sizeof(zc) * h);
    for (int64_t k = 0; k < h; k++) {
        long double th = (long double)sign * 2.0L * 3.14159265358979323846264338327950288L *
                         (long double)k / (long double)n;
        w[k].x = (double)cosl(th);
        w[k].y = (double)sinl(th);
    }
    return w;
}

/* plan0 (fft_host_plans.h:25-39): VEC-point transform of each contiguous vector.
 * nvec vectors of the grid buffer `buf`. */
static void fft1a(const cfg_t *c, zc *buf, int64_t nvec, int sign) {
    zc *w = make_roots(c->vec, sign);
    #pragma omp parallel for schedule(static)
    for (int64_t v = 0; v < nvec; v++) fft_pow2(buf + v * c->vec, c->vec, 1, sign, w);
    free(w);
}
/* plan1 (fft_host_plans.h:41-60): for every length-L row, VP interleaved
 * M-point transforms at stride VP (fft.cu:254-258). */
static void fft1b(const cfg_t *c, zc *buf, int64_t nrows, int sign) {
    zc *w = make_roots(c->m, sign);
    #pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < nrows; r++)
        for (int64_t f = 0; f < c->vp; f++) fft_pow2(buf + r * c->L + f, c->m, c->vp, sign, w);
    free(w);
}

/* ------------------------------------------------- permutation kernels */

/* Rank ids of the communicator groups: 2D row_comm = same rid (rank in comm = cid),
 * col_comm = same cid (rank in comm = rid) (fft.cu:561-567); 3D row_comm =
 * same (did,rid), col_comm = same (did,cid), dep_comm = same (rid,cid)
 * (fft3d.cu:685-697).  axis 0 = row, 1 = col, 2 = dep. */
static void rank_coords(const cfg_t *c, int64_t r, int64_t *did, int64_t *rid, int64_t *cid) {
    if (c->dim == 2) { *did = 0; *rid = r / c->p; *cid = r % c->p; }
    else { *did = r / (c->p * c->p); *rid = (r % (c->p * c->p)) / c->p; *cid = r % c->p; }
}
static int64_t rank_id(const cfg_t *c, int64_t did, int64_t rid, int64_t cid) {
    return c->dim == 2 ? rid * c->p + cid : (did * c->p + rid) * c->p + cid;
}
static int64_t comm_index(const cfg_t *c, int64_t r, int axis) {
    int64_t did, rid, cid; rank_coords(c, r, &did, &rid, &cid);
    return axis == 0 ? cid : axis == 1 ? rid : did;
}
static int64_t comm_peer(const cfg_t *c, int64_t r, int axis, int64_t s) {
    int64_t did, rid, cid; rank_coords(c, r, &did, &rid, &cid);
    if (axis == 0) cid = s; else if (axis == 1) rid = s; else did = s;
    return rank_id(c, did, rid, cid);
}

/* MPI_Alltoall over the axis communicator (fft.cu:221-241, 285-305;
 * fft3d.cu:260-270, 314-324, 368-378): chunk s of rank r's send buffer lands
 * in chunk (index of r) of rank s's receive buffer. */
static void alltoall(const cfg_t *c, const zc *send, zc *recv, int axis) {
    const int64_t chunk = c->rank_elems / c->p;
    #pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < c->ranks; r++) {
        int64_t me = comm_index(c, r, axis);
        for (int64_t s = 0; s < c->p; s++) {
            int64_t src = comm_peer(c, r, axis, s);
            memcpy(recv + r * c->rank_elems + s * chunk, send + src * c->rank_elems + me * chunk,
                   sizeof(zc) * chunk);
        }
    }
}

/* pack_forward_fft (fft.cu:138-160) / pack_forward_fft_3d (fft3d.cu:146-169),
 * and when `inverse` the gather of pack_inverse_fft(_3d) with its scale
 * (fft.cu:343-370, fft3d.cu:418-445). */
static void pack_kernel(const cfg_t *c, const zc *in, zc *out, int inverse, int do_compute, zc scale) {
    const int64_t L = c->L, VEC = c->vec, B = c->b, P = c->p;
    const int64_t vec_split = VEC / P, slab_size = (L * L) / P, slab_vec_row = L / P,
                  slab_vec_col = L / vec_split;
    const int64_t depths = c->dim == 3 ? L : 1;
    #pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < c->ranks; r++) {
        const zc *ri = in + r * c->rank_elems;
        zc *ro = out + r * c->rank_elems;
        for (int64_t dep = 0; dep < depths; dep++)
            for (int64_t blk = 0; blk < L * B; blk++) {
                const int64_t row = blk / B, col = blk % B;
                const int64_t nat = row * L + col * VEC + (c->dim == 3 ? dep * L * L : 0);
                const int64_t slab_off = c->dim == 3 ? 0 : 0;
                (void)slab_off;
                const int64_t out_row = (blk / slab_vec_col) % slab_vec_row;
                const int64_t out_col = blk % slab_vec_col;
                for (int64_t vi = 0; vi < VEC; vi++) {
                    const int64_t split = vi / vec_split, iis = vi % vec_split;
                    const int64_t slab_offset = c->dim == 3 ? (split * slab_size * L) + (dep * slab_size)
                                                            : split * slab_size;
                    const int64_t packed = slab_offset + out_row * L + out_col * vec_split + iis;
                    if (!inverse) ro[packed] = ri[nat + vi];
                    else ro[nat + vi] = do_compute ? cmul(scale, ri[packed]) : ri[packed];
                }
            }
    }
}

/* unpack_forward_fft (fft.cu:162-181) / _3d (fft3d.cu:173-198) and, when
 * `inverse`, unpack_inverse_fft (fft.cu:372-391) / _3d (fft3d.cu:449-472).
 * twrow[axis_id] is the L-row of the twiddle table of that rank's id. */
static void unpack_kernel(const cfg_t *c, const zc *in, zc *out, int axis, int inverse, int do_compute) {
    const int64_t L = c->L, P = c->p, ss = L / P, slab_size = (L * L) / P;
    const int64_t depths = c->dim == 3 ? L : 1;
    zc *tw = (zc *)malloc(sizeof(zc) * P * L);
    for (int64_t id = 0; id < P; id++) init_twiddle_row(c, id, inverse, tw + id * L);
    #pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < c->ranks; r++) {
        const zc *ri = in + r * c->rank_elems;
        zc *ro = out + r * c->rank_elems;
        const zc *twr = tw + comm_index(c, r, axis) * L;
        for (int64_t dep = 0; dep < depths; dep++)
            for (int64_t bx = 0; bx < L; bx++)
                for (int64_t tx = 0; tx < L; tx++) {
                    const int64_t irs = bx % ss, ivs = tx % ss, rs = bx / ss, vs = tx / ss;
                    const int64_t row = vs + irs * P, col = rs * ss + ivs;
                    int64_t packed, natural;
                    if (c->dim == 2) { packed = bx * L + tx; natural = row * L + col; }
                    else {
                        packed = rs * slab_size * L + dep * slab_size + irs * L + tx;
                        natural = dep * L * L + row * L + col;
                    }
                    if (!inverse) ro[natural] = do_compute ? cmul(ri[packed], twr[col]) : ri[packed];
                    else ro[packed] = do_compute ? cmul(ri[natural], twr[col]) : ri[natural];
                }
    }
    free(tw);
}

/* repack_transpose (fft.cu:183-187), repack_transpose_xy_3d (fft3d.cu:203-209),
 * repack_transpose_yz_3d (fft3d.cu:214-220) and their inverses
 * (fft.cu:393-397, fft3d.cu:477-494).  kind 0 = 2D / xy, 1 = yz. */
static void repack_kernel(const cfg_t *c, const zc *in, zc *out, int kind, int inverse) {
    const int64_t L = c->L, B = c->b, VEC = c->vec;
    const int64_t depths = c->dim == 3 ? L : 1;
    #pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < c->ranks; r++) {
        const zc *ri = in + r * c->rank_elems;
        zc *ro = out + r * c->rank_elems;
        for (int64_t d = 0; d < depths; d++)
            for (int64_t i = 0; i < L; i++)
                for (int64_t j = 0; j < L; j++) {
                    int64_t src, dst;
                    if (kind == 0) {
                        src = d * L * L + i * L + j;
                        dst = d * L * L + j * L + (i % B) * VEC + (i / B);
                    } else { /* yz: d = depth, i = r, j = c */
                        src = d * L * L + i * L + j;
                        dst = j * L * L + i * L + (d % B) * VEC + (d / B);
                    }
                    if (!inverse) ro[dst] = ri[src];
                    else ro[src] = ri[dst];
                }
    }
}

static void copy_grid(const cfg_t *c, const zc *in, zc *out) {
    memcpy(out, in, sizeof(zc) * c->ranks * c->rank_elems);
}

/* ------------------------------------------------------------ pipelines */

/* One axis pass of forward_fft (fft.cu:207-264, the FFT0..FFT1 block):
 * buf0 -> buf1, buf0 clobbered. */
static void forward_axis(const cfg_t *c, zc *buf0, zc *buf1, int axis, int do_compute) {
    const int64_t rows = c->dim == 2 ? c->L : c->L * c->L;
    const int64_t nvec = c->ranks * rows * c->b;
    zc one = {1.0, 0.0};
    if (do_compute) { copy_grid(c, buf0, buf1); fft1a(c, buf1, nvec, -1); }   /* FFT0 */
    else copy_grid(c, buf0, buf1);
    pack_kernel(c, buf1, buf0, 0, do_compute, one);                            /* PACK0 */
    alltoall(c, buf0, buf1, axis);                                             /* COMMS0 */
    unpack_kernel(c, buf1, buf0, axis, 0, do_compute);                         /* PACK1 */
    copy_grid(c, buf0, buf1);                                                  /* FFT1 */
    if (do_compute) fft1b(c, buf1, c->ranks * rows, -1);
}

/* One axis pass of inverse_fft (fft.cu:420-505 per direction): buf0 -> buf1. */
static void inverse_axis(const cfg_t *c, zc *buf0, zc *buf1, int axis, int do_compute, zc scale) {
    const int64_t rows = c->dim == 2 ? c->L : c->L * c->L;
    const int64_t nvec = c->ranks * rows * c->b;
    copy_grid(c, buf0, buf1);
    if (do_compute) fft1b(c, buf1, c->ranks * rows, +1);                       /* FFT1b^-1 */
    unpack_kernel(c, buf1, buf0, axis, 1, do_compute);                         /* unpack_inverse */
    alltoall(c, buf0, buf1, axis);                                             /* A2A */
    pack_kernel(c, buf1, buf0, 1, do_compute, scale);                          /* pack_inverse */
    copy_grid(c, buf0, buf1);                                                  /* FFT1a^-1 */
    if (do_compute) fft1a(c, buf1, nvec, +1);
}

/* forward_fft (fft.cu:199-339) and forward_fft_3d (fft3d.cu:234-412) over all
 * virtual ranks: `in` (real layout) -> `out` (reciprocal layout).  `in` is
 * not modified (the oracle works on a private copy of buf0). */
int zo_forward_fft(int dim, int64_t n, int64_t b, int64_t p, const double *in, double *out,
                   int do_compute) {
    cfg_t c; if (mkcfg(dim, n, b, p, &c)) return -1;
    const int64_t tot = c.ranks * c.rank_elems;
    zc *buf0 = (zc *)malloc(sizeof(zc) * tot);
    zc *buf1 = (zc *)out;
    if (!buf0) return -2;
    memcpy(buf0, in, sizeof(zc) * tot);
    forward_axis(&c, buf0, buf1, 0, do_compute);                  /* x: FFT0..FFT1, row comm */
    repack_kernel(&c, buf1, buf0, 0, 0);                           /* REPACK / REPACK_XY */
    forward_axis(&c, buf0, buf1, 1, do_compute);                  /* y: FFT2..FFT3, col comm */
    if (dim == 3) {
        repack_kernel(&c, buf1, buf0, 1, 0);                       /* REPACK_YZ */
        forward_axis(&c, buf0, buf1, 2, do_compute);              /* z: FFT4..FFT5, dep comm */
    }
    free(buf0);
    return 0;
}

/* inverse_fft (fft.cu:409-514) and inverse_fft_3d (fft3d.cu:508-633):
 * `in` (reciprocal layout) -> `out` (real layout), scale applied by the last
 * pack_inverse (fft.cu:498). */
int zo_inverse_fft(int dim, int64_t n, int64_t b, int64_t p, const double *in, double *out,
                   double scale_re, double scale_im, int do_compute) {
    cfg_t c; if (mkcfg(dim, n, b, p, &c)) return -1;
    const int64_t tot = c.ranks * c.rank_elems;
    zc *buf0 = (zc *)malloc(sizeof(zc) * tot);
    zc *buf1 = (zc *)out;
    zc one = {1.0, 0.0}, scale = {scale_re, scale_im};
    if (!buf0) return -2;
    memcpy(buf0, in, sizeof(zc) * tot);
    if (dim == 3) {
        inverse_axis(&c, buf0, buf1, 2, do_compute, one);          /* z, dep comm */
        repack_kernel(&c, buf1, buf0, 1, 1);                        /* inverse_repack_transpose_yz_3d */
    }
    inverse_axis(&c, buf0, buf1, 1, do_compute, one);              /* y, col comm */
    repack_kernel(&c, buf1, buf0, 0, 1);                            /* inverse_repack_transpose(_xy_3d) */
    inverse_axis(&c, buf0, buf1, 0, do_compute, scale);            /* x, row comm, scale */
    free(buf0);
    return 0;
}

/* Intermediate state after the first axis pass + repack (stage tag REPACK),
 * used to check the fused first-pass kernel in isolation. */
int zo_forward_first_pass(int dim, int64_t n, int64_t b, int64_t p, const double *in, double *out,
                          int do_compute) {
    cfg_t c; if (mkcfg(dim, n, b, p, &c)) return -1;
    const int64_t tot = c.ranks * c.rank_elems;
    zc *buf0 = (zc *)malloc(sizeof(zc) * tot);
    zc *buf1 = (zc *)malloc(sizeof(zc) * tot);
    if (!buf0 || !buf1) { free(buf0); free(buf1); return -2; }
    memcpy(buf0, in, sizeof(zc) * tot);
    forward_axis(&c, buf0, buf1, 0, do_compute);
    repack_kernel(&c, buf1, (zc *)out, 0, 0);
    free(buf0); free(buf1);
    return 0;
}

/* -------------------------------------------------------------- stencils */

/* laplace (laplace.cu:73-169) after pack_laplace (laplace.cu:172-191) and
 * communicate_laplace (laplace.cu:194-256) for every virtual rank.  The halo
 * a rank receives is its neighbour's send buffer, read in place.  Result has
 * no 1/h^2 factor; out = sum(neighbours) - 4 * centre, accumulated in the
 * reference's order. */
int zo_laplace_2d(int64_t n, int64_t b, int64_t p, const double *in_d, double *out_d) {
    cfg_t c; if (mkcfg(2, n, b, p, &c)) return -1;
    const int64_t L = c.L, B = c.b, P = c.p, VEC = c.vec;
    const zc *in = (const zc *)in_d;
    zc *out = (zc *)out_d;
    const int64_t prow = L * (L / B), pcol = L * VEC;
    zc *s_above = (zc *)malloc(sizeof(zc) * prow * c.ranks), *s_below = (zc *)malloc(sizeof(zc) * prow * c.ranks);
    zc *s_left = (zc *)malloc(sizeof(zc) * pcol * c.ranks), *s_right = (zc *)malloc(sizeof(zc) * pcol * c.ranks);
    for (int64_t r = 0; r < c.ranks; r++) {           /* pack_laplace */
        const zc *ri = in + r * c.rank_elems;
        for (int64_t i = 0; i < L; i++)
            for (int64_t j = 0; j < L; j++) {
                if (i < L / B) {
                    s_above[r * prow + i * L + j] = ri[i * L * B + j];
                    s_below[r * prow + i * L + j] = ri[L * (B - 1) + i * L * B + j];
                }
                if (j < VEC) {
                    s_left[r * pcol + i * VEC + j] = ri[i * L + j];
                    s_right[r * pcol + i * VEC + j] = ri[L - VEC + i * L + j];
                }
            }
    }
    #pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < c.ranks; r++) {
        const int64_t rid = r / P, cid = r % P;
        const int64_t left = (cid - 1 + P) % P, right = (cid + 1) % P, up = (rid - 1 + P) % P,
                      down = (rid + 1) % P;
        /* communicate_laplace: recv_left <- left's send_right, recv_right <- right's send_left,
         * recv_below <- down's send_above, recv_above <- up's send_below */
        const zc *recv_left = s_right + (rid * P + left) * pcol;
        const zc *recv_right = s_left + (rid * P + right) * pcol;
        const zc *recv_below = s_above + (down * P + cid) * prow;
        const zc *recv_above = s_below + (up * P + cid) * prow;
        const zc *di = in + r * c.rank_elems;
        zc *dout = out + r * c.rank_elems;
        for (int64_t blk = 0; blk < L * B; blk++) {
            const int64_t row = blk / B, col = blk % B, my = row * L + col * VEC;
            const int top_of_block = (row % B) == 0, top_block = row == 0, top_p = rid == 0;
            const int bottom_of_block = (row % B) == B - 1, bottom_block = row == L - 1,
                      bottom_p = rid == P - 1;
            const int rightmost_col = col == B - 1, rightmost_p = cid == P - 1;
            const int leftmost_col = col == 0, leftmost_p = cid == 0;
            for (int64_t vi = 0; vi < VEC; vi++) {
                zc s = {0.0, 0.0}, v;
                int64_t off;
                if (top_of_block) {
                    if (top_p) off = top_block ? ((L / B - 1) * L) + col * VEC : ((row / B - 1) * L) + col * VEC;
                    else off = ((row / B) * L) + col * VEC;
                    v = recv_above[off + vi];
                } else v = di[((row - 1) * L) + col * VEC + vi];
                s.x += v.x; s.y += v.y;
                if (bottom_of_block) {
                    if (bottom_p) off = bottom_block ? col * VEC : ((row / B + 1) * L) + col * VEC;
                    else off = ((row / B) * L) + col * VEC;
                    v = recv_below[off + vi];
                } else v = di[((row + 1) * L) + col * VEC + vi];
                s.x += v.x; s.y += v.y;
                if (leftmost_col) {
                    int64_t nvi = leftmost_p ? (vi - 1 + VEC) % VEC : vi;
                    v = recv_left[row * VEC + nvi];
                } else v = di[(row * L) + (col - 1) * VEC + vi];
                s.x += v.x; s.y += v.y;
                if (rightmost_col) {
                    int64_t nvi = rightmost_p ? (vi + 1) % VEC : vi;
                    v = recv_right[row * VEC + nvi];
                } else v = di[(row * L) + (col + 1) * VEC + vi];
                s.x += v.x; s.y += v.y;
                zc cc = di[my + vi];
                s.x -= 4 * cc.x; s.y -= 4 * cc.y;
                dout[my + vi] = s;
            }
        }
    }
    free(s_above); free(s_below); free(s_left); free(s_right);
    return 0;
}

/* laplace_3d (laplace3d.cu:90-225) after pack_laplace_3d (laplace3d.cu:228-262)
 * and communicate_laplace_3d (laplace3d.cu:265-361). */
int zo_laplace_3d(int64_t n, int64_t b, int64_t p, const double *in_d, double *out_d) {
    cfg_t c; if (mkcfg(3, n, b, p, &c)) return -1;
    const int64_t L = c.L, B = c.b, P = c.p, VEC = c.vec, LL = L * L;
    const zc *in = (const zc *)in_d;
    zc *out = (zc *)out_d;
    const int64_t prow = L * (L / B);       /* PACKED_ROW_COMPLEX */
    const int64_t pcol = L * VEC;           /* PACKED_COL_COMPLEX */
    const int64_t face = L * prow;          /* PACKED_FACE_COMPLEX_3D */
    const int64_t R = c.ranks;
    zc *s_above = (zc *)malloc(sizeof(zc) * face * R), *s_below = (zc *)malloc(sizeof(zc) * face * R);
    zc *s_left = (zc *)malloc(sizeof(zc) * face * R), *s_right = (zc *)malloc(sizeof(zc) * face * R);
    zc *s_front = (zc *)malloc(sizeof(zc) * face * R), *s_back = (zc *)malloc(sizeof(zc) * face * R);
    #pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < R; r++) {          /* pack_laplace_3d */
        const zc *ri = in + r * c.rank_elems;
        for (int64_t dep = 0; dep < L; dep++)
            for (int64_t i = 0; i < L; i++)
                for (int64_t j = 0; j < L; j++) {
                    if (i < L / B) {
                        s_above[r * face + dep * prow + i * L + j] = ri[dep * LL + i * L * B + j];
                        s_below[r * face + dep * prow + i * L + j] = ri[dep * LL + L * (B - 1) + i * L * B + j];
                    }
                    if (j < VEC) {
                        s_left[r * face + dep * pcol + i * VEC + j] = ri[dep * LL + i * L + j];
                        s_right[r * face + dep * pcol + i * VEC + j] = ri[dep * LL + L - VEC + i * L + j];
                    }
                    if (dep < L / B) {
                        s_front[r * face + dep * LL + i * L + j] = ri[dep * LL * B + i * L + j];
                        s_back[r * face + dep * LL + i * L + j] = ri[LL * (B - 1) + dep * LL * B + i * L + j];
                    }
                }
    }
    #pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < R; r++) {
        int64_t did, rid, cid; rank_coords(&c, r, &did, &rid, &cid);
        const int64_t left = (cid - 1 + P) % P, right = (cid + 1) % P, up = (rid - 1 + P) % P,
                      down = (rid + 1) % P, front = (did - 1 + P) % P, back = (did + 1) % P;
        const zc *recv_left = s_right + rank_id(&c, did, rid, left) * face;
        const zc *recv_right = s_left + rank_id(&c, did, rid, right) * face;
        const zc *recv_below = s_above + rank_id(&c, did, down, cid) * face;
        const zc *recv_above = s_below + rank_id(&c, did, up, cid) * face;
        const zc *recv_front = s_back + rank_id(&c, front, rid, cid) * face;
        const zc *recv_back = s_front + rank_id(&c, back, rid, cid) * face;
        const zc *di = in + r * c.rank_elems;
        zc *dout = out + r * c.rank_elems;
        for (int64_t dep = 0; dep < L; dep++)
            for (int64_t blk = 0; blk < L * B; blk++) {
                const int64_t row = blk / B, col = blk % B;
                const int64_t my = dep * LL + row * L + col * VEC;
                for (int64_t vi = 0; vi < VEC; vi++) {
                    zc s = {0.0, 0.0}, v;
                    int64_t off;
                    if ((row % B) == 0) {
                        if (rid == 0) off = dep * prow + (row == 0 ? (L / B - 1) * L : (row / B - 1) * L) + col * VEC;
                        else off = dep * prow + (row / B) * L + col * VEC;
                        v = recv_above[off + vi];
                    } else v = di[dep * LL + (row - 1) * L + col * VEC + vi];
                    s.x += v.x; s.y += v.y;
                    if ((row % B) == B - 1) {
                        if (rid == P - 1) off = dep * prow + (row == L - 1 ? 0 : (row / B + 1) * L) + col * VEC;
                        else off = dep * prow + (row / B) * L + col * VEC;
                        v = recv_below[off + vi];
                    } else v = di[dep * LL + (row + 1) * L + col * VEC + vi];
                    s.x += v.x; s.y += v.y;
                    if (col == 0) {
                        int64_t nvi = cid == 0 ? (vi - 1 + VEC) % VEC : vi;
                        v = recv_left[dep * pcol + row * VEC + nvi];
                    } else v = di[dep * LL + row * L + (col - 1) * VEC + vi];
                    s.x += v.x; s.y += v.y;
                    if (col == B - 1) {
                        int64_t nvi = cid == P - 1 ? (vi + 1) % VEC : vi;
                        v = recv_right[dep * pcol + row * VEC + nvi];
                    } else v = di[dep * LL + row * L + (col + 1) * VEC + vi];
                    s.x += v.x; s.y += v.y;
                    if ((dep % B) == 0) {
                        if (did == 0) off = (dep == 0 ? (L / B - 1) * LL : (dep / B - 1) * LL) + row * L + col * VEC;
                        else off = (dep / B) * LL + row * L + col * VEC;
                        v = recv_front[off + vi];
                    } else v = di[(dep - 1) * LL + row * L + col * VEC + vi];
                    s.x += v.x; s.y += v.y;
                    if ((dep % B) == B - 1) {
                        if (did == P - 1) off = (dep == L - 1 ? 0 : (dep / B + 1) * LL) + row * L + col * VEC;
                        else off = (dep / B) * LL + row * L + col * VEC;
                        v = recv_back[off + vi];
                    } else v = di[(dep + 1) * LL + row * L + col * VEC + vi];
                    s.x += v.x; s.y += v.y;
                    zc cc = di[my + vi];
                    s.x -= 6 * cc.x; s.y -= 6 * cc.y;
                    dout[my + vi] = s;
                }
            }
    }
    free(s_above); free(s_below); free(s_left); free(s_right); free(s_front); free(s_back);
    return 0;
}

/* dx (dx.cu:10-82) with the halos init_packed_dx builds (dx.cu:143-161):
 * packed_left0/1 = left rank's last / second-to-last vector, packed_right0/1 =
 * right rank's first / second vector.  `ncomp` = 1 for the reference's real
 * Scalar field, 2 for a complex field (each component independently). */
int zo_dx(int64_t n, int64_t b, int64_t p, const double *in, double *out, double delta, int ncomp) {
    cfg_t c; if (mkcfg(2, n, b, p, &c)) return -1;
    if (c.b < 2) return -1;
    const int64_t L = c.L, B = c.b, P = c.p, VEC = c.vec;
    #pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < c.ranks; r++) {
        const int64_t rid = r / P, cid = r % P;
        const int64_t lr_ = rid * P + (cid - 1 + P) % P, rr_ = rid * P + (cid + 1) % P;
        const double *di = in + r * c.rank_elems * ncomp;
        const double *dl = in + lr_ * c.rank_elems * ncomp, *drr = in + rr_ * c.rank_elems * ncomp;
        double *dout = out + r * c.rank_elems * ncomp;
        const int left_p = cid == 0, right_p = cid == P - 1;
        for (int64_t blk = 0; blk < L * B; blk++) {
            const int64_t row = blk / B, col = blk % B, my = row * L + col * VEC;
            for (int64_t vi = 0; vi < VEC; vi++) {
                const int64_t lvi = left_p ? (vi - 1 + VEC) % VEC : vi;
                const int64_t rvi = right_p ? (vi + 1) % VEC : vi;
                for (int q = 0; q < ncomp; q++) {
                    #define IN(a) di[(a) * ncomp + q]
                    /* packed_left0[row*VEC + x] = left rank in[row*L + L - VEC + x] etc. */
                    #define LEFT0(x) dl[(row * L + L - VEC + (x)) * ncomp + q]
                    #define LEFT1(x) dl[(row * L + L - 2 * VEC + (x)) * ncomp + q]
                    #define RIGHT0(x) drr[(row * L + (x)) * ncomp + q]
                    #define RIGHT1(x) drr[(row * L + VEC + (x)) * ncomp + q]
                    double s = 0.0;
                    if (col == 0) s += LEFT0(lvi) * -8;
                    else s += IN(row * L + (col - 1) * VEC + vi) * -8;
                    if (col == 0) s += LEFT1(lvi);
                    else if (col == 1) s += LEFT0(lvi);
                    else s += IN(row * L + (col - 2) * VEC + vi);
                    if (col == B - 1) s += RIGHT0(rvi) * 8;
                    else s += IN(row * L + (col + 1) * VEC + vi) * 8;
                    if (col == B - 1) s -= RIGHT1(rvi);
                    else if (col == B - 2) s -= RIGHT0(rvi);
                    else s -= IN(row * L + (col + 2) * VEC + vi);
                    s /= (12 * delta);
                    dout[(my + vi) * ncomp + q] = s;
                    #undef IN
                    #undef LEFT0
                    #undef LEFT1
                    #undef RIGHT0
                    #undef RIGHT1
                }
            }
        }
    }
    return 0;
}

/* dy (dy.cu:10-103) with the halos init_packed_dy builds (dy.cu:167-185):
 * packed_above0/1 = above rank's bottom / second-to-bottom row of each block,
 * packed_below0/1 = below rank's top / second row of each block. */
int zo_dy(int64_t n, int64_t b, int64_t p, const double *in, double *out, double delta, int ncomp) {
    cfg_t c; if (mkcfg(2, n, b, p, &c)) return -1;
    if (c.b < 2) return -1;
    const int64_t L = c.L, B = c.b, P = c.p, VEC = c.vec;
    #pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < c.ranks; r++) {
        const int64_t rid = r / P, cid = r % P;
        const int64_t ar = ((rid - 1 + P) % P) * P + cid, br = ((rid + 1) % P) * P + cid;
        const double *di = in + r * c.rank_elems * ncomp;
        const double *da = in + ar * c.rank_elems * ncomp, *db = in + br * c.rank_elems * ncomp;
        double *dout = out + r * c.rank_elems * ncomp;
        const int top_p = rid == 0, bottom_p = rid == P - 1;
        for (int64_t blk = 0; blk < L * B; blk++) {
            const int64_t row = blk / B, col = blk % B;
            for (int64_t t = 0; t < VEC; t++) {
                const int64_t co = col * VEC + t;
                for (int q = 0; q < ncomp; q++) {
                    /* packed rows: i*L + co indexes block i's packed row */
                    #define IN(a) di[(a) * ncomp + q]
                    #define ABOVE0(o) da[(((o) / L) * L * B + L * (B - 1) + co) * ncomp + q]
                    #define ABOVE1(o) da[(((o) / L) * L * B + L * (B - 2) + co) * ncomp + q]
                    #define BELOW0(o) db[(((o) / L) * L * B + co) * ncomp + q]
                    #define BELOW1(o) db[(((o) / L) * L * B + L + co) * ncomp + q]
                    double s = 0.0;
                    int64_t o;
                    const int top0 = (row % B) == 0, top1 = (row % B) == 1;
                    const int bot0 = (row % B) == B - 1, bot1 = (row % B) == B - 2;
                    if (top0) {
                        o = top_p ? (row == 0 ? (L / B - 1) * L : (row / B - 1) * L) : (row / B) * L;
                        s += ABOVE0(o) * -8;
                    } else s += IN((row - 1) * L + co) * -8;
                    if (top0) {
                        o = top_p ? (row == 0 ? (L / B - 1) * L : (row / B - 1) * L) : (row / B) * L;
                        s += ABOVE1(o);
                    } else if (top1) {
                        o = top_p ? (row == 1 ? (L / B - 1) * L : (row / B - 1) * L) : (row / B) * L;
                        s += ABOVE0(o);
                    } else s += IN((row - 2) * L + co);
                    if (bot0) {
                        o = bottom_p ? (row == L - 1 ? 0 : (row / B + 1) * L) : (row / B) * L;
                        s += BELOW0(o) * 8;
                    } else s += IN((row + 1) * L + co) * 8;
                    if (bot0) {
                        o = bottom_p ? (row == L - 1 ? 0 : (row / B + 1) * L) : (row / B) * L;
                        s -= BELOW1(o);
                    } else if (bot1) {
                        o = bottom_p ? (row == L - 2 ? 0 : (row / B + 1) * L) : (row / B) * L;
                        s -= BELOW0(o);
                    } else s -= IN((row + 2) * L + co);
                    s /= (12 * delta);
                    dout[(row * L + co) * ncomp + q] = s;
                    #undef IN
                    #undef ABOVE0
                    #undef ABOVE1
                    #undef BELOW0
                    #undef BELOW1
                }
            }
        }
    }
    return 0;
}

/* Number of host threads the oracle may use (OpenMP). */
int zo_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
void zo_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}
