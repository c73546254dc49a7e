// ref_host_shim.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Exposes the reference's own host-side layout code (zmodel/utils.h index maps,
// vector_pack, and the init_host / init_host_3d ramp fixture of zmodel/utils.cu)
// through a C ABI so the tests can pin the oracle bit-exactly against it.  The
// reference sources are compiled where they lie, one shared object per
// (N_DIM, B_DIM, P_DIM) because the reference fixes them as macros
// (zmodel/utils.h:27-38).  Built by oracle/Makefile into oracle/_ref/.
#include "utils.h"

extern "C" {

void zr_params(int *n, int *b, int *p, int *l, int *vec) {
    *n = N_DIM; *b = B_DIM; *p = P_DIM; *l = LOCAL_DIM; *vec = VEC;
}
int zr_packed_to_block_cyclic(int pc) { return packed_to_block_cyclic(pc); }
int zr_block_cyclic_to_packed(int bc) { return block_cyclic_to_packed(bc); }
int zr_lp(int i) { return lp(i); }
int zr_ct(int i) { return ct(i); }
int zr_lp_inv(int i) { return lp_inv(i); }
int zr_ct_inv(int i) { return ct_inv(i); }

void zr_real_to_global(int rid, int cid, int lr, int lc, int *gr, int *gc) {
    real_to_global(rid, cid, lr, lc, *gr, *gc);
}
void zr_global_to_real(int gr, int gc, int *rid, int *cid, int *lr, int *lc) {
    global_to_real(gr, gc, *rid, *cid, *lr, *lc);
}
void zr_real_to_global_3d(int rid, int cid, int did, int ld, int lr, int lc, int *gd, int *gr, int *gc) {
    real_to_global_3d(rid, cid, did, ld, lr, lc, *gd, *gr, *gc);
}
void zr_global_to_real_3d(int gd, int gr, int gc, int *rid, int *cid, int *did, int *ld, int *lr, int *lc) {
    global_to_real_3d(gd, gr, gc, *rid, *cid, *did, *ld, *lr, *lc);
}
void zr_reciprocal_to_global(int rid, int cid, int lr, int lc, int *ky, int *kx) {
    reciprocal_to_global(rid, cid, lr, lc, *ky, *kx);
}
void zr_global_to_reciprocal(int ky, int kx, int *rid, int *cid, int *lr, int *lc) {
    global_to_reciprocal(ky, kx, *rid, *cid, *lr, *lc);
}
void zr_reciprocal_to_global_3d(int rid, int cid, int did, int ld, int lr, int lc, int *kd, int *kr, int *kc) {
    reciprocal_to_global_3d(rid, cid, did, ld, lr, lc, *kd, *kr, *kc);
}
void zr_global_to_reciprocal_3d(int kd, int kr, int kc, int *rid, int *cid, int *did, int *ld, int *lr, int *lc) {
    global_to_reciprocal_3d(kd, kr, kc, *rid, *cid, *did, *ld, *lr, *lc);
}

// Whole-rank tables in one call (keeps the ctypes round trips out of the test loops).
void zr_real_layout_map(int dim, long long *gidx) {
    const int L = LOCAL_DIM;
    const int ranks = dim == 2 ? P_DIM * P_DIM : P_DIM * P_DIM * P_DIM;
    const long long per = dim == 2 ? (long long)L * L : (long long)L * L * L;
    for (int r = 0; r < ranks; r++) {
        int did = dim == 3 ? r / (P_DIM * P_DIM) : 0;
        int rid = dim == 3 ? (r % (P_DIM * P_DIM)) / P_DIM : r / P_DIM;
        int cid = r % P_DIM;
        long long *o = gidx + r * per;
        if (dim == 2) {
            for (int lr = 0; lr < L; lr++)
                for (int lc = 0; lc < L; lc++) {
                    int gr, gc; real_to_global(rid, cid, lr, lc, gr, gc);
                    o[(long long)lr * L + lc] = (long long)gr * N_DIM + gc;
                }
        } else {
            for (int ld = 0; ld < L; ld++)
                for (int lr = 0; lr < L; lr++)
                    for (int lc = 0; lc < L; lc++) {
                        int gd, gr, gc; real_to_global_3d(rid, cid, did, ld, lr, lc, gd, gr, gc);
                        o[((long long)ld * L + lr) * L + lc] = ((long long)gd * N_DIM + gr) * N_DIM + gc;
                    }
        }
    }
}
void zr_reciprocal_layout_map(int dim, long long *kidx) {
    const int L = LOCAL_DIM;
    const int ranks = dim == 2 ? P_DIM * P_DIM : P_DIM * P_DIM * P_DIM;
    const long long per = dim == 2 ? (long long)L * L : (long long)L * L * L;
    for (int r = 0; r < ranks; r++) {
        int did = dim == 3 ? r / (P_DIM * P_DIM) : 0;
        int rid = dim == 3 ? (r % (P_DIM * P_DIM)) / P_DIM : r / P_DIM;
        int cid = r % P_DIM;
        long long *o = kidx + r * per;
        if (dim == 2) {
            for (int lr = 0; lr < L; lr++)
                for (int lc = 0; lc < L; lc++) {
                    int ky, kx; reciprocal_to_global(rid, cid, lr, lc, ky, kx);
                    o[(long long)lr * L + lc] = (long long)ky * N_DIM + kx;
                }
        } else {
            for (int ld = 0; ld < L; ld++)
                for (int lr = 0; lr < L; lr++)
                    for (int lc = 0; lc < L; lc++) {
                        int kd, kr, kc; reciprocal_to_global_3d(rid, cid, did, ld, lr, lc, kd, kr, kc);
                        o[((long long)ld * L + lr) * L + lc] = ((long long)kd * N_DIM + kr) * N_DIM + kc;
                    }
        }
    }
}

void zr_init_host(int rid, int cid, double *out) { init_host<Complex>(rid, cid, (Complex *)out); }
void zr_init_host_3d(int rid, int cid, int did, double *out) {
    init_host_3d<Complex>(rid, cid, did, (Complex *)out);
}
void zr_init_host_scalar(int rid, int cid, double *out) { init_host<Scalar>(rid, cid, out); }

}  // extern "C"
