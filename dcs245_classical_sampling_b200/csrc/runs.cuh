// Register runs: fused vertex steps over coset tiles with the steps of a run done in registers
// (complex64 tables, FP32 arithmetic).  Kernels and launch templates; the instantiations are
// spread over runs.cu (scalar, local dimension 3, and the C entry point), runs_r4.cu (scalar,
// local dimension 4) and runs_packed.cu (packed FP32x2) so that they compile in parallel.
//
// A group's tile (2^dim entries in shared memory, loaded and stored as in fused.cu) is pushed
// through its steps run by run.  The orbit vectors of a run's steps span a space V of dimension
// R (3 or 4) with a basis b_0..b_{R-1} in which every step acts along fixed local bits: a
// one-vector step along its own bit k (orbits {j, j | 2^k} for local indices j with bit k
// clear), a four-entry shrink along two bits.  Every basis vector has a role coordinate (the
// tile bit of the slot it pivots on) where no other basis vector is one, so with coset
// representatives t0 zero at the role coordinates, local index j of t0 + V is the reference's
// entry c exactly when the step's own bit of j is clear.  A thread loads a coset (2^R entries)
// from shared memory into registers, applies all steps of the run with compile-time register
// indices, and writes it back: shared-memory traffic is one round trip per run, not per step.
// Orbit formulas follow the per-step kernel (reference: source/kernel_opt/inplace_gpu.py:29-58).
//
// Entries of a coset that are inactive at a step (a slot that a later grow activates or an
// earlier shrink removed) are processed like the others: an orbit never mixes active and
// inactive entries (orbit vectors have no inactive coordinate), inactive entries are never
// stored, so the extra values are dead.
#pragma once
#include <string.h>

#include "common.cuh"

namespace dcs_runs {

using namespace dcs;

constexpr int kMaxSteps = 24;
constexpr int kThreads = 256;
constexpr int kThreadLog = 8;

struct RunStep {
    uint64_t beta, cskip;
    uint32_t tbeta, ptab;
    int32_t kind, pidx;
    uint8_t sK, sKa, k1, k2, mix, dead, beff, pad;
};

struct RunDesc {
    uint8_t first, count, nins, pad;
    uint8_t ins[16];
    uint32_t mhi;
    uint16_t off[16];
};

struct RunArgs {
    int32_t count, tile_dim, low_bits, coset_m, ncoset_runs, group, nruns;
    int32_t pair_in, pair_out;
    uint64_t in_mask_first, out_mask_last;
    uint64_t basis[16];
    uint32_t coset_runs[DCS_MAX_RUNS];
    RunStep st[kMaxSteps];
    RunDesc ru[kMaxSteps];
};

__device__ __forceinline__ float2 f2(float x, float y) { return make_float2(x, y); }
__device__ __forceinline__ uint32_t insert0(uint32_t o, int p) {
    return ((o >> p) << (p + 1)) | (o & ((1u << p) - 1u));
}
__device__ __forceinline__ uint32_t spread(uint32_t o, const uint8_t* ins, int n) {
    for (int i = 0; i < n; ++i) o = insert0(o, ins[i]);
    return o;
}
// a with the sign bits flipped by m (bit 31)
__device__ __forceinline__ float2 sflip(float2 a, uint32_t m) {
    return f2(__uint_as_float(__float_as_uint(a.x) ^ m), __uint_as_float(__float_as_uint(a.y) ^ m));
}
// f * x
__device__ __forceinline__ float2 zmul(float2 f, float2 x) {
    return f2(fmaf(f.x, x.x, -f.y * x.y), fmaf(f.x, x.y, f.y * x.x));
}
// acc + f * x
__device__ __forceinline__ float2 zmadd(float2 f, float2 x, float2 acc) {
    return f2(fmaf(f.x, x.x, fmaf(-f.y, x.y, acc.x)), fmaf(f.x, x.y, fmaf(f.y, x.x, acc.y)));
}
__device__ __forceinline__ float2 zadd(float2 a, float2 b) { return f2(a.x + b.x, a.y + b.y); }
// a + g b, g = +-1
__device__ __forceinline__ float2 zaddg(float2 a, float g, float2 b) { return f2(fmaf(g, b.x, a.x), fmaf(g, b.y, a.y)); }

// Step weights of one step for one coset.  The sign of local entry j is (-1)^(m0 + <j, beta>)
// with beta the step's sign functional on the local bits; the bodies are instantiated per
// beta restricted to the bits where the step's representatives vary (template B), so every
// per-orbit sign is a compile-time choice between +-f1 computed once per coset.
struct W {
    float2 f0, f1;
    float gK;
    int y;
    uint32_t m0, ka;  // sign bits: local entry 0, (-1)^sKa
    uint32_t dead;    // local bits of inactive role slots: entries with one of them set are skipped
};
constexpr int cpar(int x) { return x ? ((x & 1) ^ cpar(x >> 1)) : 0; }
constexpr uint32_t kSign = 0x80000000u;

// One-vector kinds along local bit K: orbits {j, j | 2^K}, j with bit K clear; F1p / F1n are
// s f1 for the representatives with <j, B> even / odd, Fap / Fan the same times (-1)^sKa.
template <int KIND, int R, int K, int B, int J = 0>
__device__ __forceinline__ void orb1(float2 (&v)[1 << R], const W& w, float2 F1p, float2 F1n, float2 Fap,
                                     float2 Fan) {
    if constexpr (J < (1 << R)) {
        if (!(J & (1 << K)) && !(J & w.dead)) {
            constexpr int D = J | (1 << K);
            constexpr bool N = cpar(J & B);
            const float2 F1 = N ? F1n : F1p;
            const float2 x = v[J], b = v[D];
            if constexpr (KIND == DCS_KIND_GROW) {
                v[J] = zmul(w.f0, x);
                v[D] = zmul(F1, x);
            } else if constexpr (KIND == DCS_KIND_MIX) {
                // o_c = f0 x + s_c (-1)^sKa f1 b ;  o_d = f0 b + s_c f1 x
                v[J] = zmadd(w.f0, x, zmul(N ? Fan : Fap, b));
                v[D] = zmadd(w.f0, b, zmul(F1, x));
            } else if constexpr (KIND == DCS_KIND_REPLACE) {
                v[J] = zmul(w.f0, zadd(x, b));
                v[D] = zmul(F1, zaddg(x, w.gK, b));
            } else if constexpr (KIND == DCS_KIND_FIXED_SHRINK) {
                v[J] = w.y ? zmul(F1, zaddg(x, w.gK, b)) : zmul(w.f0, zadd(x, b));
            } else {  // DCS_KIND_SHRINK2: f0 (x + b) + s_c f1 (x + gK b)
                v[J] = zmadd(w.f0, zadd(x, b), zmul(F1, zaddg(x, w.gK, b)));
            }
        }
        orb1<KIND, R, K, B, J + 1>(v, w, F1p, F1n, Fap, Fan);
    }
}
template <int KIND, int R, int K, int B>
__device__ __forceinline__ void body1(float2 (&v)[1 << R], const W& w) {
    const float2 F1p = sflip(w.f1, w.m0), F1n = sflip(w.f1, w.m0 ^ kSign);
    float2 Fap = F1p, Fan = F1n;
    if constexpr (KIND == DCS_KIND_MIX) {
        Fap = sflip(F1p, w.ka);
        Fan = sflip(F1n, w.ka);
    }
    orb1<KIND, R, K, B>(v, w, F1p, F1n, Fap, Fan);
}

// One-entry kinds: every local entry; Fp / Fn the factor for <j, B> even / odd.
template <int KIND, int R, int B, int J = 0>
__device__ __forceinline__ void orb0(float2 (&v)[1 << R], const W& w, float2 Fp, float2 Fn) {
    if constexpr (J < (1 << R)) {
        if (!(J & w.dead)) v[J] = zmul(cpar(J & B) ? Fn : Fp, v[J]);
        orb0<KIND, R, B, J + 1>(v, w, Fp, Fn);
    }
}
template <int KIND, int R, int B>
__device__ __forceinline__ void body0(float2 (&v)[1 << R], const W& w) {
    const float2 F1p = sflip(w.f1, w.m0), F1n = sflip(w.f1, w.m0 ^ kSign);
    if constexpr (KIND == DCS_KIND_DIAG) {  // (f0 + s f1) x
        orb0<KIND, R, B>(v, w, zadd(w.f0, F1p), zadd(w.f0, F1n));
    } else {  // DCS_KIND_FIXED: y ? s f1 x : f0 x
        if (w.y) orb0<KIND, R, B>(v, w, F1p, F1n);
        else orb0<KIND, R, 0>(v, w, w.f0, w.f0);
    }
}

// Four-entry shrink along local bits K1 (K's role) and K2 (Ka's role); MIX bit 0: K's local
// mask also has K2, bit 1: Ka's has K1.
//   o_c = f0 (x + b) + s_d f1 (g + gK h) ;  o_{c^Ka} = f0 (g + h) + s_c f1 (x + gK b),
// x = c, b = c^K, g = c^Ka, h = c^Ka^K, s_d = s_c (-1)^sKa.
template <int R, int K1, int K2, int MIX, int B, int J = 0>
__device__ __forceinline__ void orb4(float2 (&v)[1 << R], const W& w, float2 F1p, float2 F1n, float2 Fap,
                                     float2 Fan) {
    if constexpr (J < (1 << R)) {
        if (!(J & ((1 << K1) | (1 << K2))) && !(J & w.dead)) {
            constexpr int MK = (1 << K1) | ((MIX & 1) ? (1 << K2) : 0);
            constexpr int MKA = (1 << K2) | ((MIX & 2) ? (1 << K1) : 0);
            constexpr bool N = cpar(J & B);
            const float2 x = v[J], b = v[J ^ MK], g = v[J ^ MKA], h = v[J ^ MK ^ MKA];
            v[J] = zmadd(w.f0, zadd(x, b), zmul(N ? Fan : Fap, zaddg(g, w.gK, h)));
            v[J ^ MKA] = zmadd(w.f0, zadd(g, h), zmul(N ? F1n : F1p, zaddg(x, w.gK, b)));
        }
        orb4<R, K1, K2, MIX, B, J + 1>(v, w, F1p, F1n, Fap, Fan);
    }
}
template <int R, int K1, int K2, int MIX, int B>
__device__ __forceinline__ void body4(float2 (&v)[1 << R], const W& w) {
    const float2 F1p = sflip(w.f1, w.m0), F1n = sflip(w.f1, w.m0 ^ kSign);
    orb4<R, K1, K2, MIX, B>(v, w, F1p, F1n, sflip(F1p, w.ka), sflip(F1n, w.ka));
}

// Dispatch on the sign functional b (local bits outside the step's own; instantiations with an
// own bit set are never called).
#define DCS_BCASES(CALL)                                                                                   \
    switch (b) {                                                                                          \
        case 0: CALL(0); break;   case 1: CALL(1); break;   case 2: CALL(2); break;   case 3: CALL(3); break;    \
        case 4: CALL(4); break;   case 5: CALL(5); break;   case 6: CALL(6); break;   case 7: CALL(7); break;    \
        case 8: CALL(8); break;   case 9: CALL(9); break;   case 10: CALL(10); break; case 11: CALL(11); break;  \
        case 12: CALL(12); break; case 13: CALL(13); break; case 14: CALL(14); break; default: CALL(15); break; \
    }

template <int KIND, int R, int K>
__device__ __forceinline__ void by_b1(float2 (&v)[1 << R], int b, const W& w) {
#define DCS_CALL1(Bv)                                                                   \
    if constexpr ((Bv) < (1 << R) && !((Bv) & (1 << K))) body1<KIND, R, K, (Bv)>(v, w);
    DCS_BCASES(DCS_CALL1)
#undef DCS_CALL1
}
template <int KIND, int R>
__device__ __forceinline__ void by_b0(float2 (&v)[1 << R], int b, const W& w) {
#define DCS_CALL0(Bv) \
    if constexpr ((Bv) < (1 << R)) body0<KIND, R, (Bv)>(v, w);
    DCS_BCASES(DCS_CALL0)
#undef DCS_CALL0
}
template <int R, int K1, int K2, int MIX>
__device__ __forceinline__ void by_b4(float2 (&v)[1 << R], int b, const W& w) {
#define DCS_CALL4(Bv)                                                                                 \
    if constexpr ((Bv) < (1 << R) && !((Bv) & ((1 << K1) | (1 << K2)))) body4<R, K1, K2, MIX, (Bv)>(v, w);
    DCS_BCASES(DCS_CALL4)
#undef DCS_CALL4
}

template <int KIND, int R>
__device__ __forceinline__ void by_k1(float2 (&v)[1 << R], int k, int b, const W& w) {
    switch (k) {
        case 0: by_b1<KIND, R, 0>(v, b, w); break;
        case 1: by_b1<KIND, R, 1>(v, b, w); break;
        case 2: by_b1<KIND, R, 2>(v, b, w); break;
        default:
            if constexpr (R > 3) by_b1<KIND, R, 3>(v, b, w);
            break;
    }
}

template <int R, int K1, int K2>
__device__ __forceinline__ void by_mix(float2 (&v)[1 << R], int mix, int b, const W& w) {
    if constexpr (K1 != K2 && K1 < R && K2 < R) {
        switch (mix) {
            case 0: by_b4<R, K1, K2, 0>(v, b, w); break;
            case 1: by_b4<R, K1, K2, 1>(v, b, w); break;
            default: by_b4<R, K1, K2, 2>(v, b, w); break;
        }
    }
}
template <int R, int K1>
__device__ __forceinline__ void by_k2(float2 (&v)[1 << R], int k2, int mix, int b, const W& w) {
    switch (k2) {
        case 0: by_mix<R, K1, 0>(v, mix, b, w); break;
        case 1: by_mix<R, K1, 1>(v, mix, b, w); break;
        case 2: by_mix<R, K1, 2>(v, mix, b, w); break;
        default: by_mix<R, K1, 3>(v, mix, b, w); break;
    }
}
template <int R>
__device__ __forceinline__ void shrink4(float2 (&v)[1 << R], int k1, int k2, int mix, int b, const W& w) {
    switch (k1) {
        case 0: by_k2<R, 0>(v, k2, mix, b, w); break;
        case 1: by_k2<R, 1>(v, k2, mix, b, w); break;
        case 2: by_k2<R, 2>(v, k2, mix, b, w); break;
        default: by_k2<R, 3>(v, k2, mix, b, w); break;
    }
}

template <int R>
__device__ __forceinline__ void apply(float2 (&v)[1 << R], const RunStep& st, const W& w) {
    const int b = st.beff;
    switch (st.kind) {
        case DCS_KIND_GROW: by_k1<DCS_KIND_GROW, R>(v, st.k1, b, w); break;
        case DCS_KIND_MIX: by_k1<DCS_KIND_MIX, R>(v, st.k1, b, w); break;
        case DCS_KIND_DIAG: by_b0<DCS_KIND_DIAG, R>(v, b, w); break;
        case DCS_KIND_REPLACE: by_k1<DCS_KIND_REPLACE, R>(v, st.k1, b, w); break;
        case DCS_KIND_FIXED: by_b0<DCS_KIND_FIXED, R>(v, b, w); break;
        case DCS_KIND_FIXED_SHRINK: by_k1<DCS_KIND_FIXED_SHRINK, R>(v, st.k1, b, w); break;
        case DCS_KIND_SHRINK4: shrink4<R>(v, st.k1, st.k2, st.mix, b, w); break;
        default: by_k1<DCS_KIND_SHRINK2, R>(v, st.k1, b, w); break;
    }
}

// One run over every active coset of the tile.  Coset representatives are the tile indices
// zero at ins[] (as in fused.cu, spread(tid) | a masked-increment walk over mhi), handled as
// byte offsets (index << 3).
template <int R>
__device__ __forceinline__ void run_block(unsigned char* __restrict__ shb, int T, const RunArgs& A, const RunDesc& ru,
                                          uint32_t csm, const float4* fw, const int* ovy) {
    const int nb = T >> ru.nins;
    if ((int)threadIdx.x >= nb) return;
    const uint32_t tp = spread(threadIdx.x, ru.ins, ru.nins) << 3;
    const uint32_t mhi3 = ru.mhi << 3;
    const int niter = nb > kThreads ? nb >> kThreadLog : 1;
    uint32_t off[1 << R];
#pragma unroll
    for (int j = 0; j < (1 << R); ++j) off[j] = (uint32_t)ru.off[j] << 3;
    const int s0 = ru.first, s1 = ru.first + ru.count;
    uint32_t tu = 0;
    for (int k = 0; k < niter; ++k) {
        const uint32_t t0 = tp | tu;
        tu = ((tu | ~mhi3) + 1u) & mhi3;
        float2 v[1 << R];
#pragma unroll
        for (int j = 0; j < (1 << R); ++j) v[j] = *reinterpret_cast<const float2*>(shb + (t0 ^ off[j]));
        for (int s = s0; s < s1; ++s) {
            const RunStep& st = A.st[s];
            const float4 f = fw[s];
            W w;
            w.f0 = f2(f.x, f.y);
            w.f1 = f2(f.z, f.w);
            w.gK = st.sK ? -1.f : 1.f;
            w.ka = (uint32_t)(st.sKa & 1) << 31;
            w.y = ovy[s] >> 1;
            w.m0 = (((uint32_t)__popc(t0 & (st.tbeta << 3)) ^ (csm >> s)) & 1u) << 31;
            w.dead = st.dead;
            apply<R>(v, st, w);
        }
#pragma unroll
        for (int j = 0; j < (1 << R); ++j) *reinterpret_cast<float2*>(shb + (t0 ^ off[j])) = v[j];
    }
}

// ---------------------------------------------------------------- packed runs
// Paired tile layout (entries 2i, 2i + 1 as (re, re, im, im) in 16 bytes, as in fused.cu's
// packed kernel): a thread holds the cosets of t0 and t0 | 1 (tile bit 0 outside the run's
// space and zero bits) as the two lanes of float2 values and uses the packed FP32x2
// instructions.  A basis vector with bit 0 set puts local entry j of the two cosets in lanes
// 1 and 0 of the pair at (t0 ^ off_j) & ~1: bit j of `swz` swaps them on load and store.
struct C2 {
    float2 re, im;
};
struct CF {
    float2 r, i, ni;
};
__device__ __forceinline__ CF cf(float2 f) { return CF{f2(f.x, f.x), f2(f.y, f.y), f2(-f.y, -f.y)}; }
__device__ __forceinline__ C2 ldc2(const unsigned char* b, uint32_t off) {
    const float4 q = *reinterpret_cast<const float4*>(b + off);
    return C2{f2(q.x, q.y), f2(q.z, q.w)};
}
__device__ __forceinline__ void stc2(unsigned char* b, uint32_t off, const C2& v) {
    *reinterpret_cast<float4*>(b + off) = make_float4(v.re.x, v.re.y, v.im.x, v.im.y);
}
__device__ __forceinline__ C2 swapl(const C2& v) { return C2{f2(v.re.y, v.re.x), f2(v.im.y, v.im.x)}; }
__device__ __forceinline__ C2 cmul(const CF& f, const C2& v) {
    return C2{__ffma2_rn(f.ni, v.im, __fmul2_rn(f.r, v.re)), __ffma2_rn(f.i, v.re, __fmul2_rn(f.r, v.im))};
}
__device__ __forceinline__ C2 cmadd(const CF& f, const C2& v, const C2& acc) {
    return C2{__ffma2_rn(f.ni, v.im, __ffma2_rn(f.r, v.re, acc.re)),
              __ffma2_rn(f.i, v.re, __ffma2_rn(f.r, v.im, acc.im))};
}
__device__ __forceinline__ C2 smul(float2 s, const C2& v) { return C2{__fmul2_rn(s, v.re), __fmul2_rn(s, v.im)}; }
__device__ __forceinline__ C2 cadd(const C2& a, const C2& b) { return C2{__fadd2_rn(a.re, b.re), __fadd2_rn(a.im, b.im)}; }
__device__ __forceinline__ C2 caddg(const C2& a, float2 g, const C2& b) {
    return C2{__ffma2_rn(g, b.re, a.re), __ffma2_rn(g, b.im, a.im)};
}

// Packed step weights for one coset pair: lane signs S0 of local entry 0 (entry j: S0, or
// -S0 when bit j of ptab is set).
struct PW {
    CF F0, F1, F1a;  // f0, f1, (-1)^sKa f1
    float2 gK, gKa;  // (-1)^sK, (-1)^sKa on both lanes
    float2 S0, NS0;
    uint32_t ptab, dead;
    int y;
};
template <int J>
__device__ __forceinline__ float2 lsign(const PW& w) {
    return ((w.ptab >> J) & 1u) ? w.NS0 : w.S0;
}

// The one-vector kinds (sign identity as in fused.cu: f0 b + S f1 x = S (f0 (S b) + f1 x)).
template <int KIND, int R, int K, int J = 0>
__device__ __forceinline__ void pbody1(C2 (&v)[1 << R], const PW& w) {
    if constexpr (J < (1 << R)) {
        if (!(J & (1 << K)) && !(J & w.dead)) {
            constexpr int D = J | (1 << K);
            const float2 S = lsign<J>(w);
            const C2 x = v[J], b = v[D];
            if constexpr (KIND == DCS_KIND_GROW) {
                v[J] = cmul(w.F0, x);
                v[D] = smul(S, cmul(w.F1, x));
            } else if constexpr (KIND == DCS_KIND_MIX) {
                const C2 bs = smul(S, b);
                v[J] = cmadd(w.F0, x, cmul(w.F1a, bs));
                v[D] = smul(S, cmadd(w.F0, bs, cmul(w.F1, x)));
            } else if constexpr (KIND == DCS_KIND_REPLACE) {
                v[J] = cmul(w.F0, cadd(x, b));
                v[D] = smul(S, cmul(w.F1, caddg(x, w.gK, b)));
            } else if constexpr (KIND == DCS_KIND_FIXED_SHRINK) {
                v[J] = w.y ? smul(S, cmul(w.F1, caddg(x, w.gK, b))) : cmul(w.F0, cadd(x, b));
            } else {  // DCS_KIND_SHRINK2
                v[J] = cmadd(w.F0, cadd(x, b), smul(S, cmul(w.F1, caddg(x, w.gK, b))));
            }
        }
        pbody1<KIND, R, K, J + 1>(v, w);
    }
}

template <int KIND, int R, int J = 0>
__device__ __forceinline__ void pbody0(C2 (&v)[1 << R], const PW& w) {
    if constexpr (J < (1 << R)) {
        if (!(J & w.dead)) {
            const float2 S = lsign<J>(w);
            const C2 x = v[J];
            if constexpr (KIND == DCS_KIND_DIAG) {  // (f0 + S f1) x
                const CF F{__ffma2_rn(S, w.F1.r, w.F0.r), __ffma2_rn(S, w.F1.i, w.F0.i),
                           __ffma2_rn(S, w.F1.ni, w.F0.ni)};
                v[J] = cmul(F, x);
            } else {  // DCS_KIND_FIXED
                v[J] = w.y ? smul(S, cmul(w.F1, x)) : cmul(w.F0, x);
            }
        }
        pbody0<KIND, R, J + 1>(v, w);
    }
}

template <int R, int K1, int K2, int MIX, int J = 0>
__device__ __forceinline__ void pbody4(C2 (&v)[1 << R], const PW& w) {
    if constexpr (J < (1 << R)) {
        if (!(J & ((1 << K1) | (1 << K2))) && !(J & w.dead)) {
            constexpr int MK = (1 << K1) | ((MIX & 1) ? (1 << K2) : 0);
            constexpr int MKA = (1 << K2) | ((MIX & 2) ? (1 << K1) : 0);
            const float2 S = lsign<J>(w);
            const C2 x = v[J], b = v[J ^ MK], g = v[J ^ MKA], h = v[J ^ MK ^ MKA];
            v[J] = cmadd(w.F0, cadd(x, b), smul(__fmul2_rn(S, w.gKa), cmul(w.F1, caddg(g, w.gK, h))));
            v[J ^ MKA] = cmadd(w.F0, cadd(g, h), smul(S, cmul(w.F1, caddg(x, w.gK, b))));
        }
        pbody4<R, K1, K2, MIX, J + 1>(v, w);
    }
}

template <int KIND, int R>
__device__ __forceinline__ void pby_k1(C2 (&v)[1 << R], int k, const PW& w) {
    switch (k) {
        case 0: pbody1<KIND, R, 0>(v, w); break;
        case 1: pbody1<KIND, R, 1>(v, w); break;
        case 2: pbody1<KIND, R, 2>(v, w); break;
        default:
            if constexpr (R > 3) pbody1<KIND, R, 3>(v, w);
            break;
    }
}
template <int R, int K1, int K2>
__device__ __forceinline__ void pby_mix(C2 (&v)[1 << R], int mix, const PW& w) {
    if constexpr (K1 != K2 && K1 < R && K2 < R) {
        switch (mix) {
            case 0: pbody4<R, K1, K2, 0>(v, w); break;
            case 1: pbody4<R, K1, K2, 1>(v, w); break;
            default: pbody4<R, K1, K2, 2>(v, w); break;
        }
    }
}
template <int R, int K1>
__device__ __forceinline__ void pby_k2(C2 (&v)[1 << R], int k2, int mix, const PW& w) {
    switch (k2) {
        case 0: pby_mix<R, K1, 0>(v, mix, w); break;
        case 1: pby_mix<R, K1, 1>(v, mix, w); break;
        case 2: pby_mix<R, K1, 2>(v, mix, w); break;
        default: pby_mix<R, K1, 3>(v, mix, w); break;
    }
}
template <int R>
__device__ __forceinline__ void papply(C2 (&v)[1 << R], const RunStep& st, const PW& w) {
    switch (st.kind) {
        case DCS_KIND_GROW: pby_k1<DCS_KIND_GROW, R>(v, st.k1, w); break;
        case DCS_KIND_MIX: pby_k1<DCS_KIND_MIX, R>(v, st.k1, w); break;
        case DCS_KIND_DIAG: pbody0<DCS_KIND_DIAG, R>(v, w); break;
        case DCS_KIND_REPLACE: pby_k1<DCS_KIND_REPLACE, R>(v, st.k1, w); break;
        case DCS_KIND_FIXED: pbody0<DCS_KIND_FIXED, R>(v, w); break;
        case DCS_KIND_FIXED_SHRINK: pby_k1<DCS_KIND_FIXED_SHRINK, R>(v, st.k1, w); break;
        case DCS_KIND_SHRINK4:
            switch (st.k1) {
                case 0: pby_k2<R, 0>(v, st.k2, st.mix, w); break;
                case 1: pby_k2<R, 1>(v, st.k2, st.mix, w); break;
                case 2: pby_k2<R, 2>(v, st.k2, st.mix, w); break;
                default: pby_k2<R, 3>(v, st.k2, st.mix, w); break;
            }
            break;
        default: pby_k1<DCS_KIND_SHRINK2, R>(v, st.k1, w); break;
    }
}

// One run over every active coset pair (t0, t0 | 1) of the tile.
template <int R, bool SWZ>
__device__ __forceinline__ void run_block_packed(unsigned char* __restrict__ shb, int T, const RunArgs& A,
                                                 const RunDesc& ru, uint32_t csm, const float4* fw, const int* ovy,
                                                 uint32_t swz) {
    const int nb = T >> (ru.nins + 1);
    if ((int)threadIdx.x >= nb) return;
    const uint32_t tp = spread(threadIdx.x << 1, ru.ins, ru.nins) << 3;
    const uint32_t mhi3 = (ru.mhi & (ru.mhi - 1u)) << 3;  // tile bit 0 is the lane bit
    const int niter = nb > kThreads ? nb >> kThreadLog : 1;
    uint32_t off[1 << R];
#pragma unroll
    for (int j = 0; j < (1 << R); ++j) off[j] = ((uint32_t)ru.off[j] & ~1u) << 3;
    const int s0 = ru.first, s1 = ru.first + ru.count;
    uint32_t tu = 0;
    for (int k = 0; k < niter; ++k) {
        const uint32_t t0 = tp | tu;
        tu = ((tu | ~mhi3) + 1u) & mhi3;
        C2 v[1 << R];
#pragma unroll
        for (int j = 0; j < (1 << R); ++j) {
            const C2 q = ldc2(shb, t0 ^ off[j]);
            v[j] = (SWZ && ((swz >> j) & 1u)) ? swapl(q) : q;
        }
        for (int s = s0; s < s1; ++s) {
            const RunStep& st = A.st[s];
            const float4 f = fw[s];
            const float gK = st.sK ? -1.f : 1.f, gKa = st.sKa ? -1.f : 1.f;
            PW w;
            w.F0 = cf(f2(f.x, f.y));
            w.F1 = cf(f2(f.z, f.w));
            w.F1a = cf(f2(gKa * f.z, gKa * f.w));
            w.gK = f2(gK, gK);
            w.gKa = f2(gKa, gKa);
            const uint32_t l0 = (((uint32_t)__popc(t0 & (st.tbeta << 3)) ^ (csm >> s)) & 1u) << 31;
            const uint32_t l1 = l0 ^ ((st.tbeta & 1u) << 31);
            w.S0 = f2(__uint_as_float(0x3f800000u ^ l0), __uint_as_float(0x3f800000u ^ l1));
            w.NS0 = f2(-w.S0.x, -w.S0.y);
            w.ptab = st.ptab;
            w.dead = st.dead;
            w.y = ovy[s] >> 1;
            papply<R>(v, st, w);
        }
#pragma unroll
        for (int j = 0; j < (1 << R); ++j) stc2(shb, t0 ^ off[j], (SWZ && ((swz >> j) & 1u)) ? swapl(v[j]) : v[j]);
    }
}

template <int MINB, int R, bool PK>
__global__ void __launch_bounds__(kThreads, MINB)
k_runs(float2* __restrict__ E, const __grid_constant__ RunArgs A, const dcs_param* __restrict__ params,
       unsigned long long* __restrict__ maxbits, dcs_scale* __restrict__ scale) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int T = 1 << A.tile_dim;
    const int low = A.low_bits;
    const int nhi = 1 << (A.tile_dim - low);
    float2* sh = reinterpret_cast<float2*>(smem);
    uint64_t* hi_tab = reinterpret_cast<uint64_t*>(smem + sizeof(float2) * (size_t)T);
    __shared__ float4 fw[kMaxSteps];
    __shared__ int ovy[kMaxSteps];
    __shared__ uint32_t cs_sh;

    const double m2prev = (double)__uint_as_float((uint32_t)maxbits[A.group]);
    const int e = scale_exponent(m2prev);
    const float sc = (float)ldexp(1.0, -e);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        scale->logscale += (double)e * 0.69314718055994530942;
        scale->exponent_sum += e;
        if (!isfinite(m2prev)) scale->flags |= 1u;
        else if (m2prev == 0.0) scale->flags |= 2u;
    }
    if (threadIdx.x < A.count) {
        const dcs_param p = params[A.st[threadIdx.x].pidx];
        fw[threadIdx.x] = make_float4((float)p.f0r, (float)p.f0i, (float)p.f1r, (float)p.f1i);
        ovy[threadIdx.x] = (p.ov & 1) | ((p.y & 1) << 1);
    }
    for (int h = threadIdx.x; h < nhi; h += blockDim.x) {
        uint64_t a = 0;
        for (int i = 0; i < A.tile_dim - low; ++i)
            if ((h >> i) & 1) a ^= A.basis[i];
        hi_tab[h] = a;
    }
    __syncthreads();

    const uint64_t lowmask = (1ull << low) - 1;
    const uint64_t ntiles = 1ull << A.coset_m;
    const uint64_t in_inactive = ~A.in_mask_first, out_inactive = ~A.out_mask_last;
    float lm = 0.f;
    for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const uint64_t base = deposit(tile, A.coset_runs, A.ncoset_runs);
        // load (entries active before the group)
        if (PK && !A.pair_in) {  // paired layout, entries t and t + 1 copied separately
            for (int t = 2 * threadIdx.x; t < T; t += 2 * kThreads) {
                const uint64_t a = base ^ hi_tab[t >> low] ^ ((uint64_t)t & lowmask);
                const uint64_t a1 = base ^ hi_tab[(t + 1) >> low] ^ ((uint64_t)(t + 1) & lowmask);
                const bool act = !(a & in_inactive), act1 = !(a1 & in_inactive);
                const uint32_t dst = (uint32_t)__cvta_generic_to_shared(&sh[t]);
                const float2* src = act ? E + a : E;
                const float2* src1 = act1 ? E + a1 : E;
                asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst), "l"(src), "r"(act ? 8 : 0)
                             : "memory");
                asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst + 8u), "l"(src1),
                             "r"(act1 ? 8 : 0)
                             : "memory");
            }
        } else if (!PK && A.pair_in && low >= 2) {
            // a lane per 4-entry segment of a row: one address and one activity test per segment,
            // two 16-byte copies (entries 0-1 and 2-3, first one chosen by lane bit 2 so that the
            // eight lanes of a quarter warp hit distinct banks).  Inactive entries are not copied:
            // they are never read by an orbit of an active entry and never stored.
            const uint32_t rot = (threadIdx.x >> 2) & 1u;
            const uint64_t seg_inactive = in_inactive & ~3ull;
            const bool hi_pair_active = !(in_inactive & 2ull);  // slot 1: entries 2-3 of a segment
            for (int q = threadIdx.x; q < (T >> 2); q += kThreads) {
                const int t = q << 2;
                const uint64_t a = base ^ hi_tab[t >> low] ^ ((uint64_t)t & lowmask);
                if (a & seg_inactive) continue;
                const uint32_t dst = (uint32_t)__cvta_generic_to_shared(&sh[t]);
                const float2* src = E + a;
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    const uint32_t cc = c ^ rot;
                    if (cc && !hi_pair_active) continue;
                    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst + 16u * cc), "l"(src + 2 * cc)
                                 : "memory");
                }
            }
        } else if (A.pair_in) {
            for (int t = 2 * threadIdx.x; t < T; t += 2 * kThreads) {
                const uint64_t a = base ^ hi_tab[t >> low] ^ ((uint64_t)t & lowmask);
                const bool act = !(a & in_inactive);
                const uint32_t dst = (uint32_t)__cvta_generic_to_shared(&sh[t]);
                const float2* src = act ? E + a : E;
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(act ? 16 : 0)
                             : "memory");
            }
        } else {
            for (int t = threadIdx.x; t < T; t += kThreads) {
                const uint64_t a = base ^ hi_tab[t >> low] ^ ((uint64_t)t & lowmask);
                const bool act = !(a & in_inactive);
                const uint32_t dst = (uint32_t)__cvta_generic_to_shared(&sh[t]);
                const float2* src = act ? E + a : E;
                asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst), "l"(src), "r"(act ? 8 : 0)
                             : "memory");
            }
        }
        // tile-constant sign parts parity(base & beta) ^ ov, one bit per step
        if (threadIdx.x < 32) {
            const int s = threadIdx.x;
            const int bit = s < A.count ? ((__popcll(base & A.st[s].beta) & 1) ^ (ovy[s] & 1)) : 0;
            const uint32_t m = __ballot_sync(0xffffffffu, bit);
            if (s == 0) cs_sh = m;
        }
        asm volatile("cp.async.wait_all;\n" ::: "memory");
        if constexpr (PK) {  // interleaved -> paired layout, each thread on the pairs it copied
            for (int t = 2 * threadIdx.x; t < T; t += 2 * kThreads) {
                float4* q = reinterpret_cast<float4*>(&sh[t]);
                const float4 v = *q;
                *q = make_float4(v.x, v.z, v.y, v.w);
            }
        }
        __syncthreads();
        const uint32_t csm = cs_sh;
        for (int ri = 0; ri < A.nruns; ++ri) {
            const RunDesc& ru = A.ru[ri];
            if (!(base & A.st[ru.first].cskip)) {
                if constexpr (PK) {
                    uint32_t swz = 0;
#pragma unroll
                    for (int j = 0; j < (1 << R); ++j) swz |= (uint32_t)(ru.off[j] & 1u) << j;
                    if (swz) run_block_packed<R, true>(smem, T, A, ru, csm, fw, ovy, swz);
                    else run_block_packed<R, false>(smem, T, A, ru, csm, fw, ovy, 0u);
                } else {
                    run_block<R>(smem, T, A, ru, csm, fw, ovy);
                }
            }
            __syncthreads();
        }
        // store (entries active after the group) and max
        if constexpr (PK) {
            for (int t = 2 * threadIdx.x; t < T; t += 2 * kThreads) {
                const float4 q = *reinterpret_cast<const float4*>(&sh[t]);  // (re_t, re_t+1, im_t, im_t+1)
                const float2 v0 = f2(q.x * sc, q.z * sc), v1 = f2(q.y * sc, q.w * sc);  // the pass's 2^-e
                const uint64_t a = base ^ hi_tab[t >> low] ^ ((uint64_t)t & lowmask);
                if (A.pair_out) {
                    if (a & out_inactive) continue;
                    lm = fmaxf(lm, fmaxf(v0.x * v0.x + v0.y * v0.y, v1.x * v1.x + v1.y * v1.y));
                    *reinterpret_cast<float4*>(E + a) = make_float4(v0.x, v0.y, v1.x, v1.y);
                } else {
                    const uint64_t a1 = base ^ hi_tab[(t + 1) >> low] ^ ((uint64_t)(t + 1) & lowmask);
                    if (!(a & out_inactive)) {
                        lm = fmaxf(lm, v0.x * v0.x + v0.y * v0.y);
                        E[a] = v0;
                    }
                    if (!(a1 & out_inactive)) {
                        lm = fmaxf(lm, v1.x * v1.x + v1.y * v1.y);
                        E[a1] = v1;
                    }
                }
            }
        } else if (A.pair_out && low >= 2) {  // segments of 4 entries, as the load
            const uint32_t rot = (threadIdx.x >> 2) & 1u;
            const uint64_t seg_inactive = out_inactive & ~3ull;
            const bool hi_pair_active = !(out_inactive & 2ull);
            for (int q = threadIdx.x; q < (T >> 2); q += kThreads) {
                const int t = q << 2;
                const uint64_t a = base ^ hi_tab[t >> low] ^ ((uint64_t)t & lowmask);
                if (a & seg_inactive) continue;
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    const uint32_t cc = c ^ rot;
                    if (cc && !hi_pair_active) continue;
                    const float4 u = *reinterpret_cast<const float4*>(&sh[t + 2 * cc]);
                    const float4 v = make_float4(u.x * sc, u.y * sc, u.z * sc, u.w * sc);  // the pass's 2^-e
                    lm = fmaxf(lm, fmaxf(v.x * v.x + v.y * v.y, v.z * v.z + v.w * v.w));
                    *reinterpret_cast<float4*>(E + a + 2 * cc) = v;
                }
            }
        } else if (A.pair_out) {
            for (int t = 2 * threadIdx.x; t < T; t += 2 * kThreads) {
                const uint64_t a = base ^ hi_tab[t >> low] ^ ((uint64_t)t & lowmask);
                if (a & out_inactive) continue;
                const float4 q = *reinterpret_cast<const float4*>(&sh[t]);
                const float4 v = make_float4(q.x * sc, q.y * sc, q.z * sc, q.w * sc);  // the pass's 2^-e
                lm = fmaxf(lm, fmaxf(v.x * v.x + v.y * v.y, v.z * v.z + v.w * v.w));
                *reinterpret_cast<float4*>(E + a) = v;
            }
        } else {
            for (int t = threadIdx.x; t < T; t += kThreads) {
                const uint64_t a = base ^ hi_tab[t >> low] ^ ((uint64_t)t & lowmask);
                if (a & out_inactive) continue;
                const float2 v = f2(sh[t].x * sc, sh[t].y * sc);
                lm = fmaxf(lm, v.x * v.x + v.y * v.y);
                E[a] = v;
            }
        }
        __syncthreads();
    }
    const unsigned long long bm = block_max_u64(max_bits(lm));
    if (threadIdx.x == 0 && bm) atomicMax(&maxbits[A.group + 1], bm);
}

template <int MINB, int R, bool PK>
int launch(const RunArgs& A, size_t smem, int sms, uint64_t ntiles, cudaStream_t st, void* table,
           const dcs_param* params, uint64_t* maxbits, dcs_scale* scale) {
    static bool attr_set[64] = {false};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        dcs_host::set_error("dcs_fused_runs: no current device");
        return DCS_E_CUDA;
    }
    if (!attr_set[dev]) {
        const cudaError_t e =
            cudaFuncSetAttribute(k_runs<MINB, R, PK>, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
        if (e != cudaSuccess) return dcs_host::check_cuda(e, "k_runs smem attribute");
        attr_set[dev] = true;
    }
    // resident CTAs per SM for this shared-memory size (persistent grid: one wave)
    int per_sm = 0;
    const cudaError_t oe = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_runs<MINB, R, PK>, kThreads, smem);
    if (oe != cudaSuccess) return dcs_host::check_cuda(oe, "k_runs occupancy");
    if (per_sm < 1) per_sm = 1;
    uint64_t g = (uint64_t)sms * per_sm;
    if (g > ntiles) g = ntiles;
    const unsigned grid = (unsigned)g;
    k_runs<MINB, R, PK><<<grid, kThreads, smem, st>>>((float2*)table, A, params, (unsigned long long*)maxbits, scale);
    DCS_CHECK_LAUNCH("k_runs launch");
    return DCS_OK;
}

// Launchers instantiated in the three translation units (mb: CTAs per SM the registers are
// sized for; r: local dimension).
int launch_scalar3(int mb, const RunArgs& A, size_t smem, int sms, uint64_t ntiles, cudaStream_t st, void* table,
                   const dcs_param* params, uint64_t* maxbits, dcs_scale* scale);
int launch_scalar4(int mb, const RunArgs& A, size_t smem, int sms, uint64_t ntiles, cudaStream_t st, void* table,
                   const dcs_param* params, uint64_t* maxbits, dcs_scale* scale);
int launch_packed(int mb, int r, const RunArgs& A, size_t smem, int sms, uint64_t ntiles, cudaStream_t st,
                  void* table, const dcs_param* params, uint64_t* maxbits, dcs_scale* scale);

}  // namespace dcs_runs
