// zm_tile.cuh -- one tile of an axis pass with runtime sizes: TL consecutive global
// lines held in shared memory, Stockham sub-transforms, and the loads / stores between
// shared memory and the two sides of the pass (see zm_lines.cuh for the addresses).
//
// Shared-memory layout of a tile: line t at s[t * N ...]; rows [n1][n2] on the vector
// side (s[t N + n1 VEC + n2]) and [k1][k2] after the transforms (s[t N + k1 VEC + k2],
// k2 = c VP + f).  Every function assumes nthr * EPT == TL * N (each thread owns EPT
// points of every stage) and leaves synchronisation to the caller where noted.
#pragma once

#include "zm_common.cuh"
#include "zm_lines.cuh"

namespace zm {

// Physical slot of tile element i in shared memory.  SwzNone: the element itself.
// SwzX (tiles with VEC = 4): up to five two-bit fields of i (shift 0 = no field) XORed
// into bits 0-1 (A0, A1), 1-2 (B) and 2-3 (C0, C1), a permutation inside every aligned run
// of 16 elements that is linear over XOR (SwzX::f(a ^ c) = SwzX::f(a) ^ SwzX::f(c)).  The
// shifts per column length M are the ones a bank-conflict model of every shared access of
// a tile found conflict-free for 16-lane half-warps: the row sweeps (lanes on rows 4
// elements apart), each Stockham stage's reads and writes, and both frequency-side
// sweeps (x pass: lines fastest, a stride of N elements; y pass: runs of VP = 2).  The
// earlier two-field form, tuned on the stages alone, left the x pass's frequency sweep
// 2- to 16-way conflicted.
struct SwzNone {
    static constexpr ZM_DEV int f(int i) { return i; }
};
template <int A0, int A1, int B, int C0, int C1> struct SwzX {
    template <int S, int T> static constexpr ZM_DEV int fld(int i) { return S ? ((i >> S) & 3) << T : 0; }
    static constexpr ZM_DEV int f(int i) {
        return i ^ fld<A0, 0>(i) ^ fld<A1, 0>(i) ^ fld<B, 1>(i) ^ fld<C0, 2>(i) ^ fld<C1, 2>(i);
    }
};

// ------------------------------------------------------------ Stockham stage
// One radix-R stage over all sub-transforms of length n held in shared memory.
//   COLM = false: sub-transform (t, n1) is the contiguous row s[t*N + n1*VEC + i]
//   COLM = true:  sub-transform (t, k2) is the column s[t*N + i*VEC + k2]
// DIR = -1 forward, +1 inverse.  PRETW multiplies the loaded inputs by the
// inter-step twiddle w_N^{n1 k2} (forward, COLM) or its conjugate (inverse, rows).
template <int R, int EPT, bool COLM, int DIR, bool PRETW, typename T>
ZM_DEV void stockham_stage(cpx<T> *s, const Geom &g, int n, int logn, int Ns, int nthr, int tid,
                           const tw<T> *twN) {
    constexpr int NB = EPT / R;
    constexpr bool CONJ = DIR > 0;
    cpx<T> v[NB][R];
    int base[NB], jv[NB];
    const int nR = n / R;
    const int logR = (R == 2) ? 1 : (R == 4) ? 2 : (R == 8) ? 3 : 4;
    const int lognR = logn - logR;
    const int str = COLM ? (int)g.vec : 1;
#pragma unroll
    for (int u = 0; u < NB; u++) {
        const int sig = tid + u * nthr;
        int j, bb, tagn;  // tagn: the sub-transform's n1 (rows) or k2 (columns)
        if (!COLM) {
            j = sig & (nR - 1);
            const int b = sig >> lognR;              // b = t*M + n1
            bb = b << g.logVEC;
            tagn = b & (int)(g.m - 1);
        } else {
            const int k2 = sig & (int)(g.vec - 1);
            const int rest = sig >> g.logVEC;
            j = rest & (nR - 1);
            const int t = rest >> lognR;
            bb = (t << g.logN) + k2;
            tagn = k2;
        }
        base[u] = bb;
        jv[u] = j;
#pragma unroll
        for (int r = 0; r < R; r++) {
            const int i = j + r * nR;
            cpx<T> x = s[bb + i * str];
            if (PRETW) x = twmul<CONJ>(x, ldtw(twN, (int64_t)i * tagn));
            v[u][r] = x;
        }
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < NB; u++) {
        const int j = jv[u];
        const int k = j & (Ns - 1);
        if (Ns > 1) {
            // w_{Ns R}^{k r} = w_N^{k r N / (Ns R)}
            const int sh = g.logN - logn + (logn - __ffs(Ns * R) + 1);
#pragma unroll
            for (int r = 1; r < R; r++)
                v[u][r] = twmul<CONJ>(v[u][r], ldtw(twN, ((int64_t)k * r) << sh));
        }
        dft<R, DIR, T>(v[u]);
        const int idxD = (j - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; r++) s[base[u] + (idxD + r * Ns) * str] = v[u][r];
    }
    __syncthreads();
}

template <int EPT, bool COLM, int DIR, typename T>
ZM_DEV void run_subfft(cpx<T> *s, const Geom &g, int n, int logn, const int *rad, int nst,
                       bool pretw, int nthr, int tid, const tw<T> *twN) {
    int Ns = 1;
    for (int st = 0; st < nst; st++) {
        const int R = rad[st];
        const bool pre = pretw && st == 0;
#define ZM_STAGE(RR)                                                                               \
    if (pre) stockham_stage<RR, EPT, COLM, DIR, true, T>(s, g, n, logn, Ns, nthr, tid, twN);      \
    else stockham_stage<RR, EPT, COLM, DIR, false, T>(s, g, n, logn, Ns, nthr, tid, twN);
        if (R == 2) { ZM_STAGE(2) }
        else if (R == 4) { ZM_STAGE(4) }
        else if (R == 8) { ZM_STAGE(8) }
        else {
            if constexpr (EPT >= 16) { ZM_STAGE(16) }
        }
#undef ZM_STAGE
        Ns *= R;
    }
}

// Both sub-transforms of a tile: forward (VEC-point rows, then the twiddled M-point
// columns) or inverse (columns, then the conjugate-twiddled rows).  Synchronised.
template <typename T, int EPT, bool INV>
ZM_DEV void tile_transform(cpx<T> *s, const Geom &g, const int *rad_vec, int nst_vec,
                           const int *rad_m, int nst_m, int nthr, int tid, const tw<T> *twN) {
    if (!INV) {
        run_subfft<EPT, false, -1, T>(s, g, (int)g.vec, g.logVEC, rad_vec, nst_vec, false, nthr, tid, twN);
        run_subfft<EPT, true, -1, T>(s, g, (int)g.m, g.logM, rad_m, nst_m, true, nthr, tid, twN);
    } else {
        run_subfft<EPT, true, 1, T>(s, g, (int)g.m, g.logM, rad_m, nst_m, false, nthr, tid, twN);
        run_subfft<EPT, false, 1, T>(s, g, (int)g.vec, g.logVEC, rad_vec, nst_vec, true, nthr, tid, twN);
    }
}

// ------------------------------------------------ compile-time-sized sub-transforms
// The same Stockham stages as stockham_stage / run_subfft / tile_transform, with the
// tile's VEC = 2^LV and M = 2^LM, the thread count NT and the radix schedule (remainder
// radix first, then radix 2^RL stages, as radix_schedule) fixed at compile time, so the
// per-point index arithmetic folds to constants.  Same shared-memory layout, same
// arithmetic in the same order.
constexpr int ct_log2(int x) { return x <= 1 ? 0 : 1 + ct_log2(x >> 1); }

template <int R, int EPT, bool COLM, int DIR, bool PRETW, typename T, int LV, int LM, int LN, int NS, int NT,
          typename SW = SwzNone>
ZM_DEV void stockham_stage_ct(cpx<T> *s, int tid, const tw<T> *twN) {
    constexpr int NB = EPT / R;
    constexpr bool CONJ = DIR > 0;
    constexpr int n = 1 << LN, VEC = 1 << LV, M = 1 << LM, LOGN = LV + LM;
    constexpr int nR = n / R;
    constexpr int logR = (R == 2) ? 1 : (R == 4) ? 2 : (R == 8) ? 3 : 4;
    constexpr int lognR = LN - logR;
    constexpr int str = COLM ? VEC : 1;
    cpx<T> v[NB][R];
    int base[NB], jv[NB];
#pragma unroll
    for (int u = 0; u < NB; u++) {
        const int sig = tid + u * NT;
        int j, bb, tagn;
        if constexpr (!COLM) {
            j = sig & (nR - 1);
            const int b = sig >> lognR;
            bb = b << LV;
            tagn = b & (M - 1);
        } else {
            const int k2 = sig & (VEC - 1);
            const int rest = sig >> LV;
            j = rest & (nR - 1);
            const int t = rest >> lognR;
            bb = (t << LOGN) + k2;
            tagn = k2;
        }
        base[u] = bb;
        jv[u] = j;
        // bb, j str and r nR str occupy disjoint bits and the slot permutations are linear
        // over XOR: SW::f(bb + i str) = SW::f(bb + j str) ^ SW::f(r nR str), one XOR with a
        // constant per access
        const int fa = SW::f(bb + j * str);
#pragma unroll
        for (int r = 0; r < R; r++) {
            const int i = j + r * nR;
            cpx<T> x = s[fa ^ SW::f(r * nR * str)];
            if constexpr (PRETW) x = twmul<CONJ>(x, ldtw(twN, (int64_t)i * tagn));
            v[u][r] = x;
        }
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < NB; u++) {
        const int j = jv[u];
        const int k = j & (NS - 1);
        if constexpr (NS > 1) {
            constexpr int sh = LOGN - LN + (LN - (ct_log2(NS * R) + 1) + 1);
#pragma unroll
            for (int r = 1; r < R; r++) v[u][r] = twmul<CONJ>(v[u][r], ldtw(twN, ((int64_t)k * r) << sh));
        }
        dft<R, DIR, T>(v[u]);
        const int idxD = (j - k) * R + k;   // (j - k) R and k leave the bits of r NS free
        const int fw = SW::f(base[u] + idxD * str);
#pragma unroll
        for (int r = 0; r < R; r++) s[fw ^ SW::f(r * NS * str)] = v[u][r];
    }
    __syncthreads();
}

template <int LN, int RL> struct radix_sched {
    static constexpr int rem = LN % RL;
    static constexpr int nst = (rem ? 1 : 0) + LN / RL;
    static constexpr int rad(int i) { return (rem && i == 0) ? (1 << rem) : (1 << RL); }
};

template <int ST, int NS, int EPT, bool COLM, int DIR, bool PRE, typename T, int LV, int LM, int LN, int NT, int RL,
          typename SW = SwzNone>
ZM_DEV void run_subfft_ct(cpx<T> *s, int tid, const tw<T> *twN) {
    using SC = radix_sched<LN, RL>;
    if constexpr (ST < SC::nst) {
        constexpr int R = SC::rad(ST);
        stockham_stage_ct<R, EPT, COLM, DIR, PRE && ST == 0, T, LV, LM, LN, NS, NT, SW>(s, tid, twN);
        run_subfft_ct<ST + 1, NS * R, EPT, COLM, DIR, PRE, T, LV, LM, LN, NT, RL, SW>(s, tid, twN);
    }
}

// ROWS = false leaves out the row sub-transform (done by the fused row sweeps below).
template <typename T, int EPT, bool INV, int LV, int LM, int NT, typename SW = SwzNone, bool ROWS = true>
ZM_DEV void tile_transform_ct(cpx<T> *s, int tid, const tw<T> *twN) {
    constexpr int RL = EPT >= 16 ? 4 : 3;   // radix_schedule(n, EPT): largest radix EPT
    if constexpr (!INV) {
        if constexpr (ROWS) run_subfft_ct<0, 1, EPT, false, -1, false, T, LV, LM, LV, NT, RL, SW>(s, tid, twN);
        run_subfft_ct<0, 1, EPT, true, -1, true, T, LV, LM, LM, NT, RL, SW>(s, tid, twN);
    } else {
        run_subfft_ct<0, 1, EPT, true, 1, false, T, LV, LM, LM, NT, RL, SW>(s, tid, twN);
        if constexpr (ROWS) run_subfft_ct<0, 1, EPT, false, 1, true, T, LV, LM, LV, NT, RL, SW>(s, tid, twN);
    }
}

// ------------------------------------------------------------ tile addressing
struct Tile {
    int TL, logT;
    int64_t a_chunk, f_chunk, f_pos;
    bool f_contig;
    const int64_t *abase, *fbase;   // per line, in shared memory
};

// Fills the per-line bases (shared arrays of TL entries) of lines l0 .. l0+TL-1 of pass
// `kind`; the caller synchronises before using the tile.
ZM_DEV Tile tile_begin(const Geom &g, int kind, int64_t l0, int TL, int64_t *abase, int64_t *fbase,
                       int nthr, int tid) {
    const LineAddr a0 = line_addr(g, kind, l0);
    for (int t = tid; t < TL; t += nthr) {
        const LineAddr a = line_addr(g, kind, l0 + t);
        abase[t] = a.a_base;
        fbase[t] = a.f_base;
    }
    Tile c;
    c.TL = TL;
    c.logT = __ffs(TL) - 1;
    c.a_chunk = a0.a_chunk;
    c.f_chunk = a0.f_chunk;
    c.f_pos = a0.f_pos;
    c.f_contig = a0.f_pos == 1;
    c.abase = abase;
    c.fbase = fbase;
    return c;
}

// element e of the frequency-side sweep -> (t, c, pos); lines fastest where the side is
// strided so that consecutive threads touch consecutive lines
ZM_DEV void tile_freq_coords(const Tile &c, const Geom &g, int e, int &t, int &ch, int &pos) {
    if (c.f_contig) {
        t = e >> g.logN;
        const int r = e & (int)(g.n - 1);
        ch = r >> g.logL;
        pos = r & (int)(g.L - 1);
    } else {
        t = e & (c.TL - 1);
        const int cp = e >> c.logT;
        ch = cp >> g.logL;
        pos = cp & (int)(g.L - 1);
    }
}

ZM_DEV int tile_freq_slot(const Geom &g, int t, int ch, int pos) {
    const int k1 = pos >> g.logVP, f = pos & (int)(g.vp - 1);
    return (t << g.logN) + (k1 << g.logVEC) + (ch << g.logVP) + f;
}

// The four sweeps below run exactly EPT elements per thread (e = tid + i * nthr, from
// nthr * EPT == TL * N).  The loads go to registers first, all EPT of them in flight
// before any is written to shared memory: one load at a time per thread leaves far too
// few bytes in flight to cover the DRAM latency.

// vector side -> rows s[t][c*L + pos] = s[t][n1*VEC + n2]
template <int EPT, typename SW = SwzNone, typename T>
ZM_DEV void tile_load_vec(const Tile &c, const Geom &g, cpx<T> *s, const cpx<T> *in, int nthr, int tid) {
    cpx<T> v[EPT];
#pragma unroll
    for (int i = 0; i < EPT; i++) {
        const int e = tid + i * nthr;
        const int t = e >> g.logN;
        const int r = e & (int)(g.n - 1);
        const int ch = r >> g.logL, pos = r & (int)(g.L - 1);
        v[i] = ldg(in + c.abase[t] + ch * c.a_chunk + pos);
    }
#pragma unroll
    for (int i = 0; i < EPT; i++) s[SW::f(tid + i * nthr)] = v[i];
}

// frequency side (t, c, pos = k1*VP + f) -> s[t][k1*VEC + c*VP + f]
template <int EPT, typename SW = SwzNone, typename T>
ZM_DEV void tile_load_freq(const Tile &c, const Geom &g, cpx<T> *s, const cpx<T> *in, int nthr, int tid) {
    cpx<T> v[EPT];
#pragma unroll
    for (int i = 0; i < EPT; i++) {
        int t, ch, pos;
        tile_freq_coords(c, g, tid + i * nthr, t, ch, pos);
        v[i] = ldg(in + c.fbase[t] + ch * c.f_chunk + pos * c.f_pos);
    }
#pragma unroll
    for (int i = 0; i < EPT; i++) {
        int t, ch, pos;
        tile_freq_coords(c, g, tid + i * nthr, t, ch, pos);
        s[SW::f(tile_freq_slot(g, t, ch, pos))] = v[i];
    }
}

template <int EPT, typename SW = SwzNone, typename T>
ZM_DEV void tile_store_freq(const Tile &c, const Geom &g, const cpx<T> *s, cpx<T> *out, bool scl, T sr,
                            T si, int nthr, int tid) {
#pragma unroll
    for (int i = 0; i < EPT; i++) {
        int t, ch, pos;
        tile_freq_coords(c, g, tid + i * nthr, t, ch, pos);
        cpx<T> v = s[SW::f(tile_freq_slot(g, t, ch, pos))];
        if (scl) v = {v.x * sr - v.y * si, v.x * si + v.y * sr};
        out[c.fbase[t] + ch * c.f_chunk + pos * c.f_pos] = v;
    }
}

template <int EPT, typename SW = SwzNone, typename T>
ZM_DEV void tile_store_vec(const Tile &c, const Geom &g, const cpx<T> *s, cpx<T> *out, bool scl, T sr,
                           T si, int nthr, int tid) {
#pragma unroll
    for (int i = 0; i < EPT; i++) {
        const int e = tid + i * nthr;
        const int t = e >> g.logN;
        const int r = e & (int)(g.n - 1);
        const int ch = r >> g.logL, pos = r & (int)(g.L - 1);
        cpx<T> v = s[SW::f(e)];
        if (scl) v = {sr * v.x - si * v.y, sr * v.y + si * v.x};
        out[c.abase[t] + ch * c.a_chunk + pos] = v;
    }
}

// ------------------------------------ complex64 VEC = 4 tiles: row stage fused with the sweep
// With VEC = 4 the row sub-transform is one radix-4 stage over rows of 4 consecutive
// vector-side positions (n1 VEC .. n1 VEC + 3, contiguous when the vector side is, a_pos
// = 1, and 32-byte aligned).  Thread tid takes rows rho = tid + q NT (q < EPT / 4), the
// rows stockham_stage_ct gives it, and the same arithmetic in the same order:
//   forward: two 16-byte loads per row, the radix-4 DFT in registers, the four outputs
//            to their slots (the stage's output order is natural: one stage, NS = 1);
//   inverse: the row's four slots, the conjugate inter-step twiddles w_N^{-n1 k2}
//            (k2 = 0 .. 3), the radix-4 DFT, the optional scale of tile_store_vec, two
//            16-byte stores.
// This drops one shared-memory round trip and its two barriers per tile.
//
// These sweeps, and the frequency-side one below (tile_freq_v4), have every size fixed
// at compile time: M = 2^LM, P = 2^LP and the pass (XP: the 2D x pass, vector side the
// real layout's rows, frequency side a stride of L with the lines fastest; otherwise
// the y pass, both sides runs of L).  Offsets inside one field (N^2 <= 2^24 elements)
// are 32-bit.
template <int LM, int LP, bool XP> struct V4Geom {
    static constexpr int LN = LM + 2, N = 1 << LN, LL = LN - LP, L = 1 << LL, LVP = 2 - LP, VP = 1 << LVP;
    static constexpr int CHUNK = XP ? L * L : (L * L) << LP;   // the next rank of a line (a_chunk, f_chunk)
    static constexpr int FPOS = XP ? L : 1;                    // frequency-side position stride (f_pos)
    static_assert(LP >= 0 && LP <= 2, "VEC = 4 needs P <= 4");
};

template <int EPT, int LM, int LP, bool XP, int NT, typename SW>
ZM_DEV void tile_load_rows_v4(const Tile &c, cpx<float> *s, const cpx<float> *in, int tid) {
    using G = V4Geom<LM, LP, XP>;
    constexpr int RPT = EPT / 4, M = 1 << LM;
    float4 v[RPT][2];
#pragma unroll
    for (int q = 0; q < RPT; q++) {
        const int rho = tid + q * NT;
        const int t = rho >> LM, r = (rho & (M - 1)) << 2;
        const int off = (int)c.abase[t] + (r >> G::LL) * G::CHUNK + (r & (G::L - 1));
        const float4 *p = reinterpret_cast<const float4 *>(in + off);
        v[q][0] = __ldg(p);
        v[q][1] = __ldg(p + 1);
    }
#pragma unroll
    for (int q = 0; q < RPT; q++) {
        cpx<float> x[4] = {{v[q][0].x, v[q][0].y}, {v[q][0].z, v[q][0].w}, {v[q][1].x, v[q][1].y},
                           {v[q][1].z, v[q][1].w}};
        dft<4, -1, float>(x);
        const int f0 = SW::f((tid + q * NT) * 4);   // the slot permutations leave bits 0-1 to k
#pragma unroll
        for (int k = 0; k < 4; k++) s[f0 ^ k] = x[k];
    }
}
template <int EPT, int LM, int LP, bool XP, int NT, typename SW>
ZM_DEV void tile_rows_store_v4(const Tile &c, const cpx<float> *s, cpx<float> *out, bool scl, float sr, float si,
                               const tw<float> *twN, int tid) {
    using G = V4Geom<LM, LP, XP>;
    constexpr int RPT = EPT / 4, M = 1 << LM;
#pragma unroll
    for (int q = 0; q < RPT; q++) {
        const int rho = tid + q * NT;
        const int n1 = rho & (M - 1);
        cpx<float> x[4];
        const int f0 = SW::f(rho * 4);
#pragma unroll
        for (int k = 0; k < 4; k++) x[k] = twmul<true>(s[f0 ^ k], ldtw(twN, (int64_t)k * n1));
        dft<4, 1, float>(x);
        if (scl)
#pragma unroll
            for (int k = 0; k < 4; k++) x[k] = {sr * x[k].x - si * x[k].y, sr * x[k].y + si * x[k].x};
        const int t = rho >> LM, r = n1 << 2;
        const int off = (int)c.abase[t] + (r >> G::LL) * G::CHUNK + (r & (G::L - 1));
        float4 *p = reinterpret_cast<float4 *>(out + off);
        p[0] = make_float4(x[0].x, x[0].y, x[1].x, x[1].y);
        p[1] = make_float4(x[2].x, x[2].y, x[3].x, x[3].y);
    }
}

// Frequency side <-> slots s[t][k1 VEC + c VP + f] (tile_load_freq / tile_store_freq):
// element e = tid + i NT is (line t, chunk c, position pos = k1 VP + f), lines fastest on
// the x pass's strided side.  LOAD: all EPT loads in flight, then the shared-memory writes.
template <int EPT, int LM, int LP, bool XP, int NT, bool LOAD, typename SW>
ZM_DEV void tile_freq_v4(const Tile &c, cpx<float> *s, const cpx<float> *in, cpx<float> *out, int tid) {
    using G = V4Geom<LM, LP, XP>;
    constexpr int TL = NT * EPT >> G::LN, LT = ct_log2(TL);
    auto coords = [&](int i, int &slot, int &off) {
        const int e = tid + i * NT;
        const int t = XP ? (e & (TL - 1)) : (e >> G::LN);
        const int cp = XP ? (e >> LT) : (e & (G::N - 1));
        const int ch = cp >> G::LL, pos = cp & (G::L - 1);
        slot = (t << G::LN) + ((pos >> G::LVP) << 2) + (ch << G::LVP) + (pos & (G::VP - 1));
        off = (int)c.fbase[t] + ch * G::CHUNK + pos * G::FPOS;
    };
    if constexpr (LOAD) {
        cpx<float> v[EPT];
#pragma unroll
        for (int i = 0; i < EPT; i++) {
            int slot, off;
            coords(i, slot, off);
            v[i] = ldg(in + off);
        }
#pragma unroll
        for (int i = 0; i < EPT; i++) {
            int slot, off;
            coords(i, slot, off);
            s[SW::f(slot)] = v[i];
        }
    } else {
#pragma unroll
        for (int i = 0; i < EPT; i++) {
            int slot, off;
            coords(i, slot, off);
            out[off] = s[SW::f(slot)];
        }
    }
}

}  // namespace zm
