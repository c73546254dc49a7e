// zm_common.cuh -- shared device types and helpers of libzmodel_b200.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "zm_plan.h"

#define ZM_DEV __device__ __forceinline__

namespace zm {

// ------------------------------------------------------------------ complex
template <typename R> struct cpx;
template <> struct __align__(16) cpx<double> { double x, y; };
template <> struct __align__(8) cpx<float> { float x, y; };

template <typename R> ZM_DEV cpx<R> cadd(cpx<R> a, cpx<R> b) { return {a.x + b.x, a.y + b.y}; }
template <typename R> ZM_DEV cpx<R> csub(cpx<R> a, cpx<R> b) { return {a.x - b.x, a.y - b.y}; }
// complex64 add / sub as one packed FP32x2 instruction each (sm_100a), same IEEE
// round-to-nearest result per component as the scalar form
template <> ZM_DEV cpx<float> cadd(cpx<float> a, cpx<float> b) {
    unsigned long long A, B, D;
    memcpy(&A, &a, 8);
    memcpy(&B, &b, 8);
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(D) : "l"(A), "l"(B));
    cpx<float> r;
    memcpy(&r, &D, 8);
    return r;
}
template <> ZM_DEV cpx<float> csub(cpx<float> a, cpx<float> b) {
    unsigned long long A, B, D;
    memcpy(&A, &a, 8);
    memcpy(&B, &b, 8);
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(D) : "l"(A), "l"(B));
    cpx<float> r;
    memcpy(&r, &D, 8);
    return r;
}
// per component a * b + c (fused, one rounding) and a * b, one FP32x2 instruction each
ZM_DEV cpx<float> cfma2(cpx<float> a, cpx<float> b, cpx<float> c) {
    unsigned long long A, B, Cc, D;
    memcpy(&A, &a, 8);
    memcpy(&B, &b, 8);
    memcpy(&Cc, &c, 8);
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(D) : "l"(A), "l"(B), "l"(Cc));
    cpx<float> r;
    memcpy(&r, &D, 8);
    return r;
}
ZM_DEV cpx<float> cmul2(cpx<float> a, cpx<float> b) {
    unsigned long long A, B, D;
    memcpy(&A, &a, 8);
    memcpy(&B, &b, 8);
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(D) : "l"(A), "l"(B));
    cpx<float> r;
    memcpy(&r, &D, 8);
    return r;
}

// Twiddle storage: FP64 pair for complex128, split hi/lo FP32 pairs for complex64
// (w = hi + lo with hi = fl32(w), lo = fl32(w - hi), both from an FP64 value).
template <typename R> struct tw;
template <> struct __align__(16) tw<double> { double x, y; };
template <> struct __align__(16) tw<float> { float x, y, lx, ly; };

// a * w (forward sign) or a * conj(w) (CONJ).  complex64 applies the
// compensated product a*hi + a*lo with every partial product fused.
template <bool CONJ> ZM_DEV cpx<double> twmul(cpx<double> a, tw<double> w) {
    const double wy = CONJ ? -w.y : w.y;
    return {fma(a.x, w.x, -a.y * wy), fma(a.x, wy, a.y * w.x)};
}
template <bool CONJ> ZM_DEV cpx<float> twmul(cpx<float> a, tw<float> w) {
    const float wy = CONJ ? -w.y : w.y;
    const float ly = CONJ ? -w.ly : w.ly;
    const float re_lo = fmaf(a.x, w.lx, -a.y * ly);
    const float im_lo = fmaf(a.x, ly, a.y * w.lx);
    return {fmaf(a.x, w.x, fmaf(-a.y, wy, re_lo)), fmaf(a.x, wy, fmaf(a.y, w.x, im_lo))};
}
// FP64 twiddle -> stored form: itself for complex128, the hi/lo FP32 split for complex64.
template <typename R> ZM_DEV tw<R> tw_from_d(double2 w);
template <> ZM_DEV tw<double> tw_from_d<double>(double2 w) { return {w.x, w.y}; }
template <> ZM_DEV tw<float> tw_from_d<float>(double2 w) {
    const float hx = __double2float_rn(w.x), hy = __double2float_rn(w.y);
    return {hx, hy, __double2float_rn(w.x - (double)hx), __double2float_rn(w.y - (double)hy)};
}
ZM_DEV double2 cmul_d(double2 a, double2 b) {
    return {fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x)};
}
ZM_DEV double2 ldd2(const double2 *p) { return __ldg(p); }

template <typename R> ZM_DEV tw<R> ldtw(const tw<R> *t, int64_t i) { return __ldg(t + i); }
template <> ZM_DEV tw<double> ldtw(const tw<double> *t, int64_t i) {
    double2 v = __ldg(reinterpret_cast<const double2 *>(t) + i);
    return {v.x, v.y};
}
template <> ZM_DEV tw<float> ldtw(const tw<float> *t, int64_t i) {
    float4 v = __ldg(reinterpret_cast<const float4 *>(t) + i);
    return {v.x, v.y, v.z, v.w};
}

template <typename R> ZM_DEV cpx<R> ldg(const cpx<R> *p) { return *p; }
template <> ZM_DEV cpx<double> ldg(const cpx<double> *p) {
    double2 v = __ldg(reinterpret_cast<const double2 *>(p));
    return {v.x, v.y};
}
template <> ZM_DEV cpx<float> ldg(const cpx<float> *p) {
    float2 v = __ldg(reinterpret_cast<const float2 *>(p));
    return {v.x, v.y};
}

// ------------------------------------------- per-thread asynchronous copies (cp.async)
ZM_DEV void cp_async8(void *dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
                 "l"((unsigned long long)__cvta_generic_to_global(src))
                 : "memory");
}
ZM_DEV void cp_async16(void *dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
                 "l"((unsigned long long)__cvta_generic_to_global(src))
                 : "memory");
}
ZM_DEV void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
ZM_DEV void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
ZM_DEV void cp_async_wait_one() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }   // all but the newest group

// ------------------------------------------------ tensor memory (TMEM) staging
// 128 lanes x 512 columns of 32 bits per SM.  With the 32x32b shape, warp w reaches the
// 32 lanes 32 (w % 4) .. 32 (w % 4) + 31, lane i of the warp its own lane; an address is
// (lane << 16) | column.  Every access is warp-wide (.sync.aligned).
ZM_DEV void tmem_alloc(uint32_t *s_addr, unsigned ncols) {   // one warp
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"((unsigned)__cvta_generic_to_shared(s_addr)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
ZM_DEV void tmem_dealloc(uint32_t taddr, unsigned ncols) {   // the allocating warp
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
ZM_DEV void tmem_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
ZM_DEV void tmem_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// 16 words of this thread to columns [c, c + 16) of its lane
ZM_DEV void tmem_st16(uint32_t taddr, const uint32_t *w) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16};" ::"r"(taddr),
        "r"(w[0]), "r"(w[1]), "r"(w[2]), "r"(w[3]), "r"(w[4]), "r"(w[5]), "r"(w[6]), "r"(w[7]), "r"(w[8]), "r"(w[9]),
        "r"(w[10]), "r"(w[11]), "r"(w[12]), "r"(w[13]), "r"(w[14]), "r"(w[15])
        : "memory");
}
// waits for this thread's earlier TMEM stores, reads 16 words and waits for the read (in
// one statement, so that no use of w can be scheduled before the data is there)
ZM_DEV void tmem_ld16(uint32_t taddr, uint32_t *w) {
    asm volatile(
        "tcgen05.wait::st.sync.aligned;\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3]), "=r"(w[4]), "=r"(w[5]), "=r"(w[6]), "=r"(w[7]), "=r"(w[8]),
          "=r"(w[9]), "=r"(w[10]), "=r"(w[11]), "=r"(w[12]), "=r"(w[13]), "=r"(w[14]), "=r"(w[15])
        : "r"(taddr)
        : "memory");
}

// ----------------------------------------------------- radix-R DFT codelets
// Constant twiddles w_R^k = exp(DIR * 2 pi i k / R), DIR = -1 forward, +1 inverse.
// cos(2 pi j / 32) for j = 0..8, the first octant of the 32-point circle.
struct k32 {
    static constexpr double c[9] = {1.0,
                                    0.98078528040323044913,    // cos(pi/16)
                                    0.92387953251128675613,    // cos(pi/8)
                                    0.83146961230254523708,    // cos(3pi/16)
                                    0.70710678118654752440,    // cos(pi/4)
                                    0.55557023301960222474,    // cos(5pi/16)
                                    0.38268343236508977173,    // cos(3pi/8)
                                    0.19509032201612826785,    // cos(7pi/16)
                                    0.0};
};

template <int R, int K, int DIR, typename T> ZM_DEV cpx<T> cmul_const(cpx<T> v) {
    constexpr int k = ((K % R) + R) % R;
    constexpr int kc = k * (32 / R);          // position on the 32-point circle (R <= 32)
    static_assert(32 % R == 0, "radix must divide 32");
    if constexpr (kc == 0) {
        return v;
    } else if constexpr (kc == 16) {
        return {-v.x, -v.y};
    } else if constexpr (kc == 8) {            // DIR=-1: -i, DIR=+1: +i
        return DIR < 0 ? cpx<T>{v.y, -v.x} : cpx<T>{-v.y, v.x};
    } else if constexpr (kc == 24) {
        return DIR < 0 ? cpx<T>{-v.y, v.x} : cpx<T>{v.y, -v.x};
    } else {
        // general: (c + DIR*i*s)
        constexpr int q = kc % 16;             // angle in (0, pi) modulo pi
        constexpr double c0 = q <= 8 ? k32::c[q] : -k32::c[16 - q];
        constexpr double s0 = q <= 8 ? k32::c[8 - q] : k32::c[q - 8];
        constexpr double sgn = kc >= 16 ? -1.0 : 1.0;    // add pi
        constexpr double cc = sgn * c0, ss = sgn * s0 * (DIR < 0 ? -1.0 : 1.0);
        const T c = (T)cc, s = (T)ss;
        return {v.x * c - v.y * s, v.x * s + v.y * c};
    }
}

template <int H, int R, int DIR, typename T, int K = 0> struct combine {
    ZM_DEV static void run(cpx<T> *v, const cpx<T> *e, const cpx<T> *o) {
        if constexpr (K < H) {
            cpx<T> t = cmul_const<R, K, DIR>(o[K]);
            v[K] = cadd(e[K], t);
            v[K + H] = csub(e[K], t);
            combine<H, R, DIR, T, K + 1>::run(v, e, o);
        }
    }
};

// In-register DFT of R points, natural order in and out (radix-2 DIT recursion
// with the trivial rotations folded away).
template <int R, int DIR, typename T> ZM_DEV void dft(cpx<T> *v) {
    if constexpr (R == 1) {
        return;
    } else if constexpr (R == 2) {
        cpx<T> a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else {
        constexpr int H = R / 2;
        cpx<T> e[H], o[H];
#pragma unroll
        for (int i = 0; i < H; i++) { e[i] = v[2 * i]; o[i] = v[2 * i + 1]; }
        dft<H, DIR, T>(e);
        dft<H, DIR, T>(o);
        combine<H, R, DIR, T>::run(v, e, o);
    }
}

// --------------------------------------------------------------- utilities
ZM_DEV int64_t pack_pos(int64_t i, int logB, int64_t B, int logVEC) {   // block_cyclic_to_packed
    return ((i & (B - 1)) << logVEC) + (i >> logB);
}
ZM_DEV int64_t unpack_pos(int64_t q, int64_t VEC, int logVEC, int logB) {  // inverse of pack_pos
    return ((q & (VEC - 1)) << logB) + (q >> logVEC);
}

}  // namespace zm
