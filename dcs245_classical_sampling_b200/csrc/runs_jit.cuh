// Plan-specialised register runs: the device header of the kernels that jit.py generates per
// fused plan and compiles with NVRTC (sm_100a) at engine setup.
//
// The generated kernel of a group is k_runs (runs.cuh) with every plan quantity a compile-time
// constant: tile shape, basis, coset runs, activity masks, and per run the coset
// representatives' zero bits, the local offsets and, per step, the kind, the local bit(s), the
// sign functional, the dead bits and the partner signs.  What stays at run time is the data of
// the sample: the table, the step weights f0, f1, ov, y, and the renormalisation state.  There
// is no dispatch in the step loop and every shared-memory offset of a coset is an immediate.
//
// Self-contained for NVRTC: no host headers.  The two structs below have the layout of
// dcs_param and dcs_scale in include/dcs245.h (the library checks their sizes).
#pragma once

#ifdef __CUDACC_RTC__
typedef unsigned int uint32_t;
typedef unsigned long long uint64_t;
typedef long long int64_t;
typedef int int32_t;
#else  // the same source built offline with nvcc (register and spill checks)
#include <stdint.h>
#endif

struct jit_param {
    double f0r, f0i, f1r, f1i;
    int32_t ov, y;
};
struct jit_scale {
    double logscale;
    int64_t exponent_sum;
    uint32_t flags, pad;
    double phase;
};

#define JK_GROW 0
#define JK_MIX 1
#define JK_DIAG 2
#define JK_REPLACE 3
#define JK_FIXED 4
#define JK_FIXED_SHRINK 5
#define JK_SHRINK4 6
#define JK_SHRINK2 7

// Entry type of a translation unit: complex64 tables with FP32 arithmetic (default), or
// complex128 tables with FP64 arithmetic when the unit defines DCS_JIT_FP64 (the audit
// recontraction).  One unit holds kernels of one type only.
#ifdef DCS_JIT_FP64
typedef double real_t;
typedef double2 cplx_t;
typedef double4 wts_t;
#else
typedef float real_t;
typedef float2 cplx_t;
typedef float4 wts_t;
#endif

namespace jit {

#ifndef DCS_JIT_THREADS
#define DCS_JIT_THREADS 256
#endif
constexpr int kThreads = DCS_JIT_THREADS;  // threads per CTA of every kernel of the unit
constexpr uint32_t kSign = 0x80000000u;  // sign bit of an FP32 value, or of an FP64 value's high word

__host__ __device__ constexpr int cpar(int x) { return x ? ((x & 1) ^ cpar(x >> 1)) : 0; }

__device__ __forceinline__ float2 f2(float x, float y) { return make_float2(x, y); }
__device__ __forceinline__ double2 f2(double x, double y) { return make_double2(x, y); }
__device__ __forceinline__ float rfma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double rfma(double a, double b, double c) { return fma(a, b, c); }
// sign flip by bit 31 of m
__device__ __forceinline__ float sflip1(float a, uint32_t m) { return __uint_as_float(__float_as_uint(a) ^ m); }
__device__ __forceinline__ double sflip1(double a, uint32_t m) {
    return __hiloint2double(__double2hiint(a) ^ (int)m, __double2loint(a));
}
__device__ __forceinline__ cplx_t sflip(cplx_t a, uint32_t m) { return f2(sflip1(a.x, m), sflip1(a.y, m)); }
// f * x
__device__ __forceinline__ cplx_t zmul(cplx_t f, cplx_t x) {
    return f2(rfma(f.x, x.x, -f.y * x.y), rfma(f.x, x.y, f.y * x.x));
}
// acc + f * x
__device__ __forceinline__ cplx_t zmadd(cplx_t f, cplx_t x, cplx_t acc) {
    return f2(rfma(f.x, x.x, rfma(-f.y, x.y, acc.x)), rfma(f.x, x.y, rfma(f.y, x.x, acc.y)));
}
__device__ __forceinline__ cplx_t zadd(cplx_t a, cplx_t b) { return f2(a.x + b.x, a.y + b.y); }
// a + (-1)^NEG b
template <int NEG>
__device__ __forceinline__ cplx_t zaddg(cplx_t a, cplx_t b) {
    if constexpr (NEG) return f2(a.x - b.x, a.y - b.y);
    else return f2(a.x + b.x, a.y + b.y);
}
// |x|^2 of a stored entry, the running max, and the order-preserving key of a non-negative
// value (maxbits)
__device__ __forceinline__ real_t norm2(cplx_t q) { return q.x * q.x + q.y * q.y; }
__device__ __forceinline__ float rmax(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double rmax(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ unsigned long long max_key(float m) { return (unsigned long long)__float_as_uint(m); }
__device__ __forceinline__ unsigned long long max_key(double m) { return (unsigned long long)__double_as_longlong(m); }

// ---------------------------------------------------------------- orbit bodies
// The weights are unit weights (prologue): f0 = 1 at every free step, and at a fixed step the
// weight its y selects is 1, so no body multiplies by f0.
//
// Local entry j is dead (its address has an inactive slot) when one of the parity masks packed
// in DP (6 bits each, up to five, 0 ends the list) has odd parity with j: the mask of basis
// vectors that have an inactive role coordinate.  When no basis vector touches another's role
// coordinate every mask is one bit, the bits of DEAD.
__host__ __device__ constexpr bool deadp(int j, uint32_t dp) {
    return dp ? (cpar(j & (int)(dp & 63u)) != 0 || deadp(j, dp >> 6)) : false;
}

// One-vector kinds along local bit K: orbits {c, c ^ 2^K}, one per j with bit K clear and not
// dead; c is the entry whose role coordinate is zero: j, or j | 2^K when the other basis vectors
// touching the role (local mask TK) flip it (TK = 0 when no basis vector touches another's role).
// Sign of representative c: (-1)^(m0 + <c, B>), so F1p / F1n = s f1 for <c, B> even / odd.
// SK / SKA: the partner signs (-1)^sK, (-1)^sKa.  Formulas: the per-step kernel's
// (reference: source/kernel_opt/inplace_gpu.py:29-58) with f0 = 1.
template <int KIND, int R, int K, int B, int DEAD, int SK, int SKA, int TK = 0, uint32_t DP = 0, int J = 0>
__device__ __forceinline__ void orb1(cplx_t (&v)[1 << R], cplx_t F1p, cplx_t F1n, cplx_t Fap, cplx_t Fan, int y) {
    if constexpr (J < (1 << R)) {
        if constexpr (!(J & (1 << K)) && !(J & DEAD) && !deadp(J, DP)) {
            constexpr int C = cpar(J & TK) ? (J | (1 << K)) : J;
            constexpr int D = C ^ (1 << K);
            constexpr bool N = cpar(C & B);
            const cplx_t F1 = N ? F1n : F1p;
            const cplx_t x = v[C], b = v[D];
            if constexpr (KIND == JK_GROW) {  // v[C] = x stays
                v[D] = zmul(F1, x);
            } else if constexpr (KIND == JK_MIX) {
                v[C] = zmadd(N ? Fan : Fap, b, x);
                v[D] = zmadd(F1, x, b);
            } else if constexpr (KIND == JK_REPLACE) {
                v[C] = zadd(x, b);
                v[D] = zmul(F1, zaddg<SK>(x, b));
            } else if constexpr (KIND == JK_FIXED_SHRINK) {
                v[C] = y ? zmul(F1, zaddg<SK>(x, b)) : zadd(x, b);
            } else {  // JK_SHRINK2
                v[C] = zmadd(F1, zaddg<SK>(x, b), zadd(x, b));
            }
        }
        orb1<KIND, R, K, B, DEAD, SK, SKA, TK, DP, J + 1>(v, F1p, F1n, Fap, Fan, y);
    }
}
template <int KIND, int R, int K, int B, int DEAD, int SK, int SKA, int TK = 0, uint32_t DP = 0>
__device__ __forceinline__ void body1(cplx_t (&v)[1 << R], wts_t f, int y, uint32_t m0) {
    const cplx_t f1 = f2(f.z, f.w);
    const cplx_t F1p = sflip(f1, m0), F1n = sflip(f1, m0 ^ kSign);
    constexpr uint32_t ka = SKA ? kSign : 0u;
    orb1<KIND, R, K, B, DEAD, SK, SKA, TK, DP>(v, F1p, F1n, sflip(F1p, ka), sflip(F1n, ka), y);
}

// One-entry kinds: every local entry that is not dead.
template <int R, int B, int DEAD, uint32_t DP = 0, int J = 0>
__device__ __forceinline__ void orb0(cplx_t (&v)[1 << R], cplx_t Fp, cplx_t Fn) {
    if constexpr (J < (1 << R)) {
        if constexpr (!(J & DEAD) && !deadp(J, DP)) v[J] = zmul(cpar(J & B) ? Fn : Fp, v[J]);
        orb0<R, B, DEAD, DP, J + 1>(v, Fp, Fn);
    }
}
template <int KIND, int R, int B, int DEAD, uint32_t DP = 0>
__device__ __forceinline__ void body0(cplx_t (&v)[1 << R], wts_t f, int y, uint32_t m0) {
    const cplx_t f1 = f2(f.z, f.w);
    const cplx_t F1p = sflip(f1, m0), F1n = sflip(f1, m0 ^ kSign);
    if constexpr (KIND == JK_DIAG) {  // (1 + s f1) x
        orb0<R, B, DEAD, DP>(v, f2((real_t)1 + F1p.x, F1p.y), f2((real_t)1 + F1n.x, F1n.y));
    } else {  // JK_FIXED: y ? s x : x (the selected weight is 1)
        if (y) orb0<R, B, DEAD, DP>(v, F1p, F1n);
    }
}

// The representative of a four-entry orbit {j ^ a MK ^ b MKA}: the entry whose two role
// coordinates (parities with the local masks ROW1 = 2^K1 | T1, ROW2 = 2^K2 | T2) are zero.
template <int J, int MK, int MKA, int ROW1, int ROW2>
__host__ __device__ constexpr int rep4() {
    int c = J;
    for (int ab = 0; ab < 4; ++ab) {
        const int e = J ^ ((ab & 1) ? MK : 0) ^ ((ab & 2) ? MKA : 0);
        if (!cpar(e & ROW1) && !cpar(e & ROW2)) c = e;
    }
    return c;
}

// Four-entry shrink along local bits K1 (K's role) and K2 (Ka's role); MIX bit 0: K's local
// mask also has K2, bit 1: Ka's has K1; T1 / T2: the other basis vectors touching the roles.
//   o_c = (x + b) + s_d f1 (g + gK h) ;  o_{c^Ka} = (g + h) + s_c f1 (x + gK b).
template <int R, int K1, int K2, int MIX, int B, int DEAD, int SK, int T1 = 0, int T2 = 0, uint32_t DP = 0, int J = 0>
__device__ __forceinline__ void orb4(cplx_t (&v)[1 << R], cplx_t F1p, cplx_t F1n, cplx_t Fap, cplx_t Fan) {
    if constexpr (J < (1 << R)) {
        if constexpr (!(J & ((1 << K1) | (1 << K2))) && !(J & DEAD) && !deadp(J, DP)) {
            constexpr int MK = (1 << K1) | ((MIX & 1) ? (1 << K2) : 0);
            constexpr int MKA = (1 << K2) | ((MIX & 2) ? (1 << K1) : 0);
            constexpr int C = rep4<J, MK, MKA, (1 << K1) | T1, (1 << K2) | T2>();
            constexpr bool N = cpar(C & B);
            const cplx_t x = v[C], b = v[C ^ MK], g = v[C ^ MKA], h = v[C ^ MK ^ MKA];
            v[C] = zmadd(N ? Fan : Fap, zaddg<SK>(g, h), zadd(x, b));
            v[C ^ MKA] = zmadd(N ? F1n : F1p, zaddg<SK>(x, b), zadd(g, h));
        }
        orb4<R, K1, K2, MIX, B, DEAD, SK, T1, T2, DP, J + 1>(v, F1p, F1n, Fap, Fan);
    }
}
template <int R, int K1, int K2, int MIX, int B, int DEAD, int SK, int SKA, int T1 = 0, int T2 = 0, uint32_t DP = 0>
__device__ __forceinline__ void body4(cplx_t (&v)[1 << R], wts_t f, int y, uint32_t m0) {
    const cplx_t f1 = f2(f.z, f.w);
    const cplx_t F1p = sflip(f1, m0), F1n = sflip(f1, m0 ^ kSign);
    constexpr uint32_t ka = SKA ? kSign : 0u;
    orb4<R, K1, K2, MIX, B, DEAD, SK, T1, T2, DP>(v, F1p, F1n, sflip(F1p, ka), sflip(F1n, ka));
}

#ifndef DCS_JIT_FP64
// ---------------------------------------------------------------- packed bodies
// A thread holds the coset pair (t0, t0 | 1) (tile bit 0 outside the run's space): local entry
// j of both cosets is one C2, lane 0 for t0, lane 1 for t0 | 1, and the FP32x2 instructions do
// both.  Lane 1's sign is lane 0's flipped by tile bit 0 of the step's beta (TB0), a constant.
struct C2 {
    float2 re, im;
};
struct CF {  // a complex factor per lane, with its negated imaginary part
    float2 r, i, ni;
};
// The packed bodies are the scalar bodies lane by lane, with the same formulas in the same order:
// f * x is fma(f.re, x.re, (-f.im) x.im) + i fma(f.re, x.im, f.im x.re), and acc + f * x folds acc
// into the inner product first, as zmul and zmadd do (the compiler may still schedule the FP32x2
// instructions so that a result differs from the scalar form in the last unit).
__device__ __forceinline__ C2 c2mul(const CF& f, const C2& v) {
    return C2{__ffma2_rn(f.r, v.re, __fmul2_rn(f.ni, v.im)), __ffma2_rn(f.r, v.im, __fmul2_rn(f.i, v.re))};
}
__device__ __forceinline__ C2 c2madd(const CF& f, const C2& v, const C2& acc) {
    return C2{__ffma2_rn(f.r, v.re, __ffma2_rn(f.ni, v.im, acc.re)),
              __ffma2_rn(f.r, v.im, __ffma2_rn(f.i, v.re, acc.im))};
}
__device__ __forceinline__ C2 c2add(const C2& a, const C2& b) {
    return C2{__fadd2_rn(a.re, b.re), __fadd2_rn(a.im, b.im)};
}
template <int NEG>
__device__ __forceinline__ C2 c2addg(const C2& a, const C2& b) {
    if constexpr (NEG) {  // a - b, rounded once
        const float2 m = f2(-1.f, -1.f);
        return C2{__ffma2_rn(m, b.re, a.re), __ffma2_rn(m, b.im, a.im)};
    } else {
        return c2add(a, b);
    }
}
// factor f with lane signs (bit 31 of m0, m1)
__device__ __forceinline__ CF cf_signed(float2 f, uint32_t m0, uint32_t m1) {
    const float2 a = sflip(f, m0), b = sflip(f, m1);
    return CF{f2(a.x, b.x), f2(a.y, b.y), f2(-a.y, -b.y)};
}

// unit weights (prologue): as orb1 / body1
template <int KIND, int R, int K, int B, int DEAD, int SK, int J = 0>
__device__ __forceinline__ void porb1(C2 (&v)[1 << R], const CF& F1p, const CF& F1n, const CF& Fap, const CF& Fan,
                                      int y) {
    if constexpr (J < (1 << R)) {
        if constexpr (!(J & (1 << K)) && !(J & DEAD)) {
            constexpr int D = J | (1 << K);
            constexpr bool N = cpar(J & B);
            const CF& F1 = N ? F1n : F1p;
            const C2 x = v[J], b = v[D];
            if constexpr (KIND == JK_GROW) {
                v[D] = c2mul(F1, x);
            } else if constexpr (KIND == JK_MIX) {
                v[J] = c2madd(N ? Fan : Fap, b, x);
                v[D] = c2madd(F1, x, b);
            } else if constexpr (KIND == JK_REPLACE) {
                v[J] = c2add(x, b);
                v[D] = c2mul(F1, c2addg<SK>(x, b));
            } else if constexpr (KIND == JK_FIXED_SHRINK) {
                v[J] = y ? c2mul(F1, c2addg<SK>(x, b)) : c2add(x, b);
            } else {  // JK_SHRINK2
                v[J] = c2madd(F1, c2addg<SK>(x, b), c2add(x, b));
            }
        }
        porb1<KIND, R, K, B, DEAD, SK, J + 1>(v, F1p, F1n, Fap, Fan, y);
    }
}
// lane signs of local entry 0: m0 (lane 0) and m0 ^ TB0 (lane 1)
template <int KIND, int R, int K, int B, int DEAD, int SK, int SKA, int TB0>
__device__ __forceinline__ void pbody1(C2 (&v)[1 << R], float4 f, int y, uint32_t m0) {
    const uint32_t m1 = m0 ^ (TB0 ? kSign : 0u);
    const CF F1p = cf_signed(f2(f.z, f.w), m0, m1), F1n = cf_signed(f2(f.z, f.w), m0 ^ kSign, m1 ^ kSign);
    constexpr uint32_t ka = SKA ? kSign : 0u;
    const CF Fap = cf_signed(f2(f.z, f.w), m0 ^ ka, m1 ^ ka), Fan = cf_signed(f2(f.z, f.w), m0 ^ ka ^ kSign, m1 ^ ka ^ kSign);
    porb1<KIND, R, K, B, DEAD, SK>(v, F1p, F1n, Fap, Fan, y);
}

template <int R, int B, int DEAD, int J = 0>
__device__ __forceinline__ void porb0(C2 (&v)[1 << R], const CF& Fp, const CF& Fn) {
    if constexpr (J < (1 << R)) {
        if constexpr (!(J & DEAD)) v[J] = c2mul(cpar(J & B) ? Fn : Fp, v[J]);
        porb0<R, B, DEAD, J + 1>(v, Fp, Fn);
    }
}
// as body0: (1 + s f1) x for the diagonal kind; y ? s x : x for a fixed step
template <int KIND, int R, int B, int DEAD, int TB0>
__device__ __forceinline__ void pbody0(C2 (&v)[1 << R], float4 f, int y, uint32_t m0) {
    const float2 f1 = f2(f.z, f.w);
    const uint32_t m1 = m0 ^ (TB0 ? kSign : 0u);
    if constexpr (KIND == JK_DIAG) {
        const float2 a = sflip(f1, m0), b = sflip(f1, m1), an = sflip(f1, m0 ^ kSign), bn = sflip(f1, m1 ^ kSign);
        const float2 pa = f2(1.f + a.x, a.y), pb = f2(1.f + b.x, b.y);
        const float2 na = f2(1.f + an.x, an.y), nb = f2(1.f + bn.x, bn.y);
        const CF Fp{f2(pa.x, pb.x), f2(pa.y, pb.y), f2(-pa.y, -pb.y)};
        const CF Fn{f2(na.x, nb.x), f2(na.y, nb.y), f2(-na.y, -nb.y)};
        porb0<R, B, DEAD>(v, Fp, Fn);
    } else {  // JK_FIXED
        if (y) porb0<R, B, DEAD>(v, cf_signed(f1, m0, m1), cf_signed(f1, m0 ^ kSign, m1 ^ kSign));
    }
}

// as orb4 / body4
template <int R, int K1, int K2, int MIX, int B, int DEAD, int SK, int J = 0>
__device__ __forceinline__ void porb4(C2 (&v)[1 << R], const CF& F1p, const CF& F1n, const CF& Fap, const CF& Fan) {
    if constexpr (J < (1 << R)) {
        if constexpr (!(J & ((1 << K1) | (1 << K2))) && !(J & DEAD)) {
            constexpr int MK = (1 << K1) | ((MIX & 1) ? (1 << K2) : 0);
            constexpr int MKA = (1 << K2) | ((MIX & 2) ? (1 << K1) : 0);
            constexpr bool N = cpar(J & B);
            const C2 x = v[J], b = v[J ^ MK], g = v[J ^ MKA], h = v[J ^ MK ^ MKA];
            v[J] = c2madd(N ? Fan : Fap, c2addg<SK>(g, h), c2add(x, b));
            v[J ^ MKA] = c2madd(N ? F1n : F1p, c2addg<SK>(x, b), c2add(g, h));
        }
        porb4<R, K1, K2, MIX, B, DEAD, SK, J + 1>(v, F1p, F1n, Fap, Fan);
    }
}
template <int R, int K1, int K2, int MIX, int B, int DEAD, int SK, int SKA, int TB0>
__device__ __forceinline__ void pbody4(C2 (&v)[1 << R], float4 f, int y, uint32_t m0) {
    const uint32_t m1 = m0 ^ (TB0 ? kSign : 0u);
    const CF F1p = cf_signed(f2(f.z, f.w), m0, m1), F1n = cf_signed(f2(f.z, f.w), m0 ^ kSign, m1 ^ kSign);
    constexpr uint32_t ka = SKA ? kSign : 0u;
    const CF Fap = cf_signed(f2(f.z, f.w), m0 ^ ka, m1 ^ ka), Fan = cf_signed(f2(f.z, f.w), m0 ^ ka ^ kSign, m1 ^ ka ^ kSign);
    porb4<R, K1, K2, MIX, B, DEAD, SK>(v, F1p, F1n, Fap, Fan);
}

#endif  // DCS_JIT_FP64

// ---------------------------------------------------------------- group prologue, tiles, epilogue
__device__ __forceinline__ int scale_exponent(double m2) {
    if (!(m2 > 0.0) || !isfinite(m2)) return 0;
    int e;
    frexp(sqrt(m2), &e);
    return e;
}

// Unit weights: a step multiplies every entry it writes by f0 or f1, so its factor c can leave
// the table: c = f0 (at a fixed step, the weight its y selects), the kernel applies (f0, f1) / c,
// whose weight on c's side is exactly 1, and log|c| and arg c go into the item's scale.  The
// scalar bodies then drop every multiplication by f0.  The host keeps f0 != 0 at the free steps
// of items that run these kernels.
__device__ __forceinline__ double2 step_factor(const jit_param& p, bool fixed) {
    return (fixed && (p.y & 1)) ? make_double2(p.f1r, p.f1i) : make_double2(p.f0r, p.f0i);
}
__device__ __forceinline__ wts_t unit_weights(const jit_param& p, bool fixed) {
    wts_t w;
    w.x = fixed && (p.y & 1) ? (real_t)0 : (real_t)1;
    w.y = 0;
    if (fixed) {
        w.z = (p.y & 1) ? (real_t)1 : (real_t)0;
        w.w = 0;
        return w;
    }
    const double n = p.f0r * p.f0r + p.f0i * p.f0i;  // f1 / f0
    w.z = (real_t)((p.f1r * p.f0r + p.f1i * p.f0i) / n);
    w.w = (real_t)((p.f1i * p.f0r - p.f1r * p.f0i) / n);
    return w;
}

// Pass scale 2^-e from the previous pass's max and the group's step factors (block 0 records
// both), the unit step weights into shared memory, and the table of high tile-coordinate
// addresses.  FIXMASK bit i: step FIRST + i is a fixed kind.
// FILL_HI: fill hi_tab (false when the kernel keeps the split tables of fill_hi_split instead).
template <int TD, int LOW, int COUNT, int FIRST, uint32_t FIXMASK, bool FILL_HI = true>
__device__ __forceinline__ real_t prologue(const jit_param* __restrict__ params, const uint64_t* basis,
                                           const unsigned long long* maxbits, int group, jit_scale* scale,
                                           wts_t* fw, int* ovy, uint64_t* hi_tab) {
#ifdef DCS_JIT_FP64
    const double m2prev = __longlong_as_double((long long)maxbits[group]);
#else
    const double m2prev = (double)__uint_as_float((uint32_t)maxbits[group]);
#endif
    const int e = scale_exponent(m2prev);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        double lg = 0.0, ph = 0.0;
        for (int i = 0; i < COUNT; ++i) {
            const double2 c = step_factor(params[FIRST + i], (FIXMASK >> i) & 1u);
            lg += 0.5 * log(c.x * c.x + c.y * c.y);
            ph += atan2(c.y, c.x);
        }
        scale->logscale += (double)e * 0.69314718055994530942 + lg;
        scale->phase += ph;
        scale->exponent_sum += e;
        if (!isfinite(m2prev)) scale->flags |= 1u;
        else if (m2prev == 0.0) scale->flags |= 2u;
    }
    if (threadIdx.x < COUNT) {
        const jit_param p = params[FIRST + threadIdx.x];
        fw[threadIdx.x] = unit_weights(p, (FIXMASK >> threadIdx.x) & 1u);
        ovy[threadIdx.x] = (p.ov & 1) | ((p.y & 1) << 1);
    }
    if constexpr (FILL_HI) {
        for (int h = threadIdx.x; h < (1 << (TD - LOW)); h += kThreads) {
            uint64_t a = 0;
#pragma unroll
            for (int i = 0; i < TD - LOW; ++i)
                if ((h >> i) & 1) a ^= basis[i];
            hi_tab[h] = a;
        }
    }
    __syncthreads();
    return (real_t)ldexp(1.0, -e);
}

// The table of high tile-coordinate addresses split in two (2^A + 2^(NBITS - A) words instead of
// 2^NBITS): addr of high index h = hA[h & (2^A - 1)] ^ hB[h >> A].  Filled before the prologue,
// whose barrier publishes it.
template <int NBITS, int A>
__device__ __forceinline__ void fill_hi_split(const uint64_t* basis, uint64_t* hA, uint64_t* hB) {
    for (int h = threadIdx.x; h < (1 << A) + (1 << (NBITS - A)); h += kThreads) {
        const bool lo = h < (1 << A);
        const int v = lo ? h : h - (1 << A);
        const int o = lo ? 0 : A;
        const int nb = lo ? A : NBITS - A;
        uint64_t a = 0;
        for (int i = 0; i < nb; ++i)
            if ((v >> i) & 1) a ^= basis[o + i];
        if (lo) hA[v] = a; else hB[v] = a;
    }
}

// Asynchronous global -> shared copies (LDGSTS) of the next tile's first-run entries into a
// thread's own staging slots; the thread waits for its own copies only (no barrier needed).
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(uint32_t dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

#ifndef DCS_JIT_FP64
// Tile load: entries active before the group (as runs.cuh: 4-entry segments when slot 0 is
// active and rows have 4 entries or more, else 16-byte pairs or single entries, zero-filled).
template <int T, int LOW, bool PAIR_IN>
__device__ __forceinline__ void load_tile(const float2* __restrict__ E, float2* sh, const uint64_t* hi_tab,
                                          uint64_t base, uint64_t in_inactive) {
    constexpr uint64_t lowmask = (1ull << LOW) - 1;
    if constexpr (PAIR_IN && LOW >= 2) {
        const uint32_t rot = (threadIdx.x >> 2) & 1u;
        const uint64_t seg_inactive = in_inactive & ~3ull;
        const bool hi_pair_active = !(in_inactive & 2ull);
        for (int q = threadIdx.x; q < (T >> 2); q += kThreads) {
            const int t = q << 2;
            const uint64_t a = base ^ hi_tab[t >> LOW] ^ ((uint64_t)t & lowmask);
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
    } else if constexpr (PAIR_IN) {
        for (int t = 2 * threadIdx.x; t < T; t += 2 * kThreads) {
            const uint64_t a = base ^ hi_tab[t >> LOW] ^ ((uint64_t)t & lowmask);
            const bool act = !(a & in_inactive);
            const uint32_t dst = (uint32_t)__cvta_generic_to_shared(&sh[t]);
            const float2* src = act ? E + a : E;
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(act ? 16 : 0)
                         : "memory");
        }
    } else {
        for (int t = threadIdx.x; t < T; t += kThreads) {
            const uint64_t a = base ^ hi_tab[t >> LOW] ^ ((uint64_t)t & lowmask);
            const bool act = !(a & in_inactive);
            const uint32_t dst = (uint32_t)__cvta_generic_to_shared(&sh[t]);
            const float2* src = act ? E + a : E;
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst), "l"(src), "r"(act ? 8 : 0)
                         : "memory");
        }
    }
}

// Tile store of the entries active after the group, scaled by the pass's 2^-e; returns the
// running max |x|^2.
template <int T, int LOW, bool PAIR_OUT>
__device__ __forceinline__ float store_tile(float2* __restrict__ E, const float2* sh, const uint64_t* hi_tab,
                                            uint64_t base, uint64_t out_inactive, float sc, float lm) {
    constexpr uint64_t lowmask = (1ull << LOW) - 1;
    if constexpr (PAIR_OUT && LOW >= 2) {
        const uint32_t rot = (threadIdx.x >> 2) & 1u;
        const uint64_t seg_inactive = out_inactive & ~3ull;
        const bool hi_pair_active = !(out_inactive & 2ull);
        for (int q = threadIdx.x; q < (T >> 2); q += kThreads) {
            const int t = q << 2;
            const uint64_t a = base ^ hi_tab[t >> LOW] ^ ((uint64_t)t & lowmask);
            if (a & seg_inactive) continue;
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const uint32_t cc = c ^ rot;
                if (cc && !hi_pair_active) continue;
                const float4 u = *reinterpret_cast<const float4*>(&sh[t + 2 * cc]);
                const float4 v = make_float4(u.x * sc, u.y * sc, u.z * sc, u.w * sc);
                lm = fmaxf(lm, fmaxf(v.x * v.x + v.y * v.y, v.z * v.z + v.w * v.w));
                *reinterpret_cast<float4*>(E + a + 2 * cc) = v;
            }
        }
    } else if constexpr (PAIR_OUT) {
        for (int t = 2 * threadIdx.x; t < T; t += 2 * kThreads) {
            const uint64_t a = base ^ hi_tab[t >> LOW] ^ ((uint64_t)t & lowmask);
            if (a & out_inactive) continue;
            const float4 q = *reinterpret_cast<const float4*>(&sh[t]);
            const float4 v = make_float4(q.x * sc, q.y * sc, q.z * sc, q.w * sc);
            lm = fmaxf(lm, fmaxf(v.x * v.x + v.y * v.y, v.z * v.z + v.w * v.w));
            *reinterpret_cast<float4*>(E + a) = v;
        }
    } else {
        for (int t = threadIdx.x; t < T; t += kThreads) {
            const uint64_t a = base ^ hi_tab[t >> LOW] ^ ((uint64_t)t & lowmask);
            if (a & out_inactive) continue;
            const float2 v = f2(sh[t].x * sc, sh[t].y * sc);
            lm = fmaxf(lm, v.x * v.x + v.y * v.y);
            E[a] = v;
        }
    }
    return lm;
}

#endif  // DCS_JIT_FP64 (the FP64 units read and write the table directly in the first and last run)

// Tile-constant sign parts parity(base & beta_s) ^ ov_s, one bit per step (warp 0).
template <int COUNT>
__device__ __forceinline__ void sign_bits(const uint64_t* beta, uint64_t base, const int* ovy, uint32_t* cs_sh) {
    if (threadIdx.x < 32) {
        const int s = threadIdx.x;
        const int bit = s < COUNT ? ((__popcll(base & beta[s]) & 1) ^ (ovy[s] & 1)) : 0;
        const uint32_t m = __ballot_sync(0xffffffffu, bit);
        if (s == 0) *cs_sh = m;
    }
}

// The tile's sign bits computed by every warp for itself (kernels with the split barrier between
// tiles share no per-tile word between warps).
template <int COUNT>
__device__ __forceinline__ uint32_t warp_sign_bits(const uint64_t* beta, uint64_t base, const int* ovy) {
    const int s = threadIdx.x & 31;
    const int bit = s < COUNT ? ((__popcll(base & beta[s]) & 1) ^ (ovy[s] & 1)) : 0;
    return __ballot_sync(0xffffffffu, bit);
}

// Split barrier between tiles (shared-memory mbarrier, one arrival per thread per tile): a thread
// arrives once it has read the tile buffer for the last time in a tile, and waits for the
// previous tile's phase only before its first write into the buffer in the next tile, so no
// thread waits at a tile's start.  The wait gives up after kWaitLimit polls and reports it.
#ifndef DCS_JIT_WAIT_LIMIT
#define DCS_JIT_WAIT_LIMIT (1 << 22)
#endif
constexpr int kWaitLimit = DCS_JIT_WAIT_LIMIT;
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(bar);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(a), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(bar);
    asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.shared::cta.b64 st, [%0];\n}\n" ::"r"(a) : "memory");
}
// true once the phase of the given parity has completed; false if kWaitLimit polls did not see it
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(bar);
    for (int i = 0; i < kWaitLimit; ++i) {
        uint32_t done;
        asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                     " selp.u32 %0, 1, 0, p;\n}\n"
                     : "=r"(done)
                     : "r"(a), "r"(parity)
                     : "memory");
        if (done) return true;
    }
    return false;
}
// a wait that gave up: flag 4 in the item's scale, and a NaN block max, so that every consumer of
// the table (the next group's prologue, the block's flags, the draw) sees an invalid result
__device__ __forceinline__ void wait_failed(jit_scale* scale, real_t& lm) {
    atomicOr(&scale->flags, 4u);
    lm = (real_t)__int_as_float(0x7fc00000);
}

__device__ __forceinline__ void block_max(real_t lm, unsigned long long* maxbits, int slot) {
    __shared__ unsigned long long red[32];
    unsigned long long v = max_key(lm);
    for (int off = 16; off > 0; off >>= 1) {
        const unsigned long long o = __shfl_xor_sync(0xffffffffu, v, off);
        v = o > v ? o : v;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (warp == 0) {
        v = lane < (kThreads >> 5) ? red[lane] : 0ull;
        for (int off = 16; off > 0; off >>= 1) {
            const unsigned long long o = __shfl_xor_sync(0xffffffffu, v, off);
            v = o > v ? o : v;
        }
        if (lane == 0 && v) atomicMax(&maxbits[slot], v);
    }
}

__device__ __forceinline__ uint32_t ins0(uint32_t o, int p) { return ((o >> p) << (p + 1)) | (o & ((1u << p) - 1u)); }

}  // namespace jit
