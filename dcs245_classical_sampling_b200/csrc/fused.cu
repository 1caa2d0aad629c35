// Fused vertex steps over coset tiles in shared memory (complex64 tables, FP32 arithmetic).
//
// One launch = one group of consecutive vertex steps (see fused.py for the tile algebra).
// Each CTA loops over tiles (persistent grid): it loads the entries of a tile that are
// active before the group (128-byte rows of 2^low contiguous entries), applies every step of
// the group in shared memory with the same orbit formulas as the per-step kernel
// (reference: source/kernel_opt/inplace_gpu.py:29-58), and stores the entries that are
// active after the group.  The power-of-two renormalisation is applied once per pass (at the
// store; the steps are linear) from the previous pass's max; the pass's own max is reduced per
// CTA and published with one atomicMax.  Tile loads are cp.async copies, zero-filled for
// entries that are inactive before the group.
#include <string.h>

#include "common.cuh"

using namespace dcs;

namespace {

constexpr int kMaxSteps = 24;
constexpr int kThreads = 256;
constexpr int kThreadLog = 8;

struct FusedStep {
    uint64_t beta, cskip;
    uint32_t tK, tKa, tpiv, tbeta;
    int32_t kind, pidx;
    uint8_t sK, sKa, nins, pad;
    uint8_t ins[16];
    uint32_t mhi;
    // pairing with the next step (see dcs_tile_step)
    uint8_t pair, pnins, swapB, swapA;
    uint32_t pmhi, tau1, tau2;
    uint8_t pins[16];
    uint8_t s1e[4], s2e[4];
};

struct FusedArgs {
    int32_t count, tile_dim, low_bits, coset_m, ncoset_runs, group;
    int32_t pair_in, pair_out;  // slot 0 (tile bit 0) active before / after the group
    uint64_t in_mask_first, out_mask_last;
    uint64_t basis[16];
    uint32_t coset_runs[DCS_MAX_RUNS];
    FusedStep st[kMaxSteps];
};

__device__ __forceinline__ float2 f2(float x, float y) { return make_float2(x, y); }

__device__ __forceinline__ uint32_t insert0(uint32_t o, int p) {
    return ((o >> p) << (p + 1)) | (o & ((1u << p) - 1u));
}

// (-1)^s * a by flipping the sign bits
__device__ __forceinline__ float2 negif(float2 a, int s) {
    const uint32_t m = (uint32_t)s << 31;
    return f2(__uint_as_float(__float_as_uint(a.x) ^ m), __uint_as_float(__float_as_uint(a.y) ^ m));
}
// f * x
__device__ __forceinline__ float2 fmul(float2 f, float2 x) {
    return f2(fmaf(f.x, x.x, -f.y * x.y), fmaf(f.x, x.y, f.y * x.x));
}
// acc + f * x
__device__ __forceinline__ float2 fmadd(float2 f, float2 x, float2 acc) {
    return f2(fmaf(f.x, x.x, fmaf(-f.y, x.y, acc.x)), fmaf(f.x, x.y, fmaf(f.y, x.x, acc.y)));
}

// Spread the bits of o over the positions that are not in ins[0..n) (ascending): the inserted
// positions become zero.  A bit injection, so spread(a | b) = spread(a) | spread(b).
__device__ __forceinline__ uint32_t spread(uint32_t o, const uint8_t* ins, int n) {
    for (int i = 0; i < n; ++i) o = insert0(o, ins[i]);
    return o;
}

// One vertex step over every active orbit representative of the tile.  Representatives are the
// tile indices with zero bits at ins[]: the role slots (so the index is the reference's entry c)
// and the tile bits of slots inactive at this step (so every orbit touched is active).  The
// index o = tid + 256 k is spread as spread(tid) | spread(256 k): the first part is fixed per
// thread and step; the second is the same for every thread and walks the tile bits in mhi in
// increasing order with ((v | ~mhi) + 1) & mhi.
// Shared-memory accessors by byte offset (offset = 8 * tile index).  Two tile layouts:
// interleaved (entry t = (re, im) at 8 t) and paired (entries 2j, 2j + 1 as
// (re_2j, re_2j+1, im_2j, im_2j+1) at 16 j, the layout of the packed kernel).
template <bool PL>
__device__ __forceinline__ float2 ldsh(const unsigned char* base, uint32_t off) {
    if constexpr (PL) {
        const unsigned char* p = base + ((off & ~15u) | ((off >> 1) & 4u));
        return f2(*reinterpret_cast<const float*>(p), *reinterpret_cast<const float*>(p + 8));
    } else {
        return *reinterpret_cast<const float2*>(base + off);
    }
}
template <bool PL>
__device__ __forceinline__ void stsh(unsigned char* base, uint32_t off, float2 v) {
    if constexpr (PL) {
        unsigned char* p = base + ((off & ~15u) | ((off >> 1) & 4u));
        *reinterpret_cast<float*>(p) = v.x;
        *reinterpret_cast<float*>(p + 8) = v.y;
    } else {
        *reinterpret_cast<float2*>(base + off) = v;
    }
}

template <int KIND, bool PL = false>
__device__ __forceinline__ void run_step(unsigned char* __restrict__ shb, int T, const FusedStep& st, float2 f0,
                                         float2 f1, int cs, int y) {
    const int nins = st.nins;
    const int nrep = T >> nins;  // a power of two
    if ((int)threadIdx.x >= nrep) return;
    // tile indices are handled as byte offsets (index << 3) throughout
    const uint32_t tbeta3 = st.tbeta << 3;
    const uint32_t tp = spread(threadIdx.x, st.ins, nins) << 3;
    const int hs = (__popc(tp & tbeta3) & 1) ^ cs;
    const uint32_t mhi3 = st.mhi << 3;
    const int niter = nrep > kThreads ? nrep >> kThreadLog : 1;
    // partner-sign factors of this step, (-1)^sK and (-1)^sKa, and f0 +- f1 for the diagonal kinds
    const float gK = st.sK ? -1.f : 1.f, gKa = st.sKa ? -1.f : 1.f;
    const float2 fp = f2(f0.x + f1.x, f0.y + f1.y), fm = f2(f0.x - f1.x, f0.y - f1.y);
    const float2 f1a = f2(gKa * f1.x, gKa * f1.y);  // f1 (-1)^sKa
    const uint32_t tK = st.tK << 3, tKa = st.tKa << 3, tpiv = st.tpiv << 3;
    uint32_t tu = 0;  // spread(256 k) << 3, advanced by a masked increment over mhi << 3
#pragma unroll 4
    for (int k = 0; k < niter; ++k) {
        const uint32_t t = tp | tu;
        const int sc = hs ^ (__popc(tu & tbeta3) & 1);
        tu = ((tu | ~mhi3) + 1u) & mhi3;
        const float2 x = ldsh<PL>(shb, t);
        if constexpr (KIND == DCS_KIND_GROW) {
            stsh<PL>(shb, t, fmul(f0, x));
            stsh<PL>(shb, t ^ tpiv, negif(fmul(f1, x), sc));
        } else if constexpr (KIND == DCS_KIND_MIX) {
            // o0 = f0 x + s_c f1 (-1)^sKa b ;  o1 = f0 b + s_c f1 x
            const uint32_t td = t ^ tKa;
            const float2 b = ldsh<PL>(shb, td);
            stsh<PL>(shb, t, fmadd(f0, x, negif(fmul(f1a, b), sc)));
            stsh<PL>(shb, td, fmadd(f0, b, negif(fmul(f1, x), sc)));
        } else if constexpr (KIND == DCS_KIND_DIAG) {
            stsh<PL>(shb, t, fmul(sc ? fm : fp, x));
        } else if constexpr (KIND == DCS_KIND_REPLACE) {
            // o0 = f0 (x + b) ;  o1 = s_c f1 (x + (-1)^sK b)
            const uint32_t td = t ^ tK;
            const float2 b = ldsh<PL>(shb, td);
            stsh<PL>(shb, t, fmul(f0, f2(x.x + b.x, x.y + b.y)));
            stsh<PL>(shb, td, negif(fmul(f1, f2(fmaf(gK, b.x, x.x), fmaf(gK, b.y, x.y))), sc));
        } else if constexpr (KIND == DCS_KIND_FIXED) {
            stsh<PL>(shb, t, y ? negif(fmul(f1, x), sc) : fmul(f0, x));
        } else if constexpr (KIND == DCS_KIND_FIXED_SHRINK) {
            const uint32_t td = t ^ tK;
            const float2 b = ldsh<PL>(shb, td);
            stsh<PL>(shb, t, y ? negif(fmul(f1, f2(fmaf(gK, b.x, x.x), fmaf(gK, b.y, x.y))), sc)
                           : fmul(f0, f2(x.x + b.x, x.y + b.y)));
        } else if constexpr (KIND == DCS_KIND_SHRINK4) {
            // o0 = f0 (x + b) + s_d f1 (g + (-1)^sK h) ;  o1 = f0 (g + h) + s_c f1 (x + (-1)^sK b)
            const uint32_t t1 = t ^ tK, td = t ^ tKa, td1 = td ^ tK;
            const float2 b = ldsh<PL>(shb, t1), g = ldsh<PL>(shb, td), h = ldsh<PL>(shb, td1);
            const int sd = sc ^ st.sKa;
            stsh<PL>(shb, t, fmadd(f0, f2(x.x + b.x, x.y + b.y),
                               negif(fmul(f1, f2(fmaf(gK, h.x, g.x), fmaf(gK, h.y, g.y))), sd)));
            stsh<PL>(shb, td, fmadd(f0, f2(g.x + h.x, g.y + h.y),
                                negif(fmul(f1, f2(fmaf(gK, b.x, x.x), fmaf(gK, b.y, x.y))), sc)));
        } else {  // DCS_KIND_SHRINK2: f0 (x + b) + s_c f1 (x + (-1)^sK b)
            const uint32_t td = t ^ tK;
            const float2 b = ldsh<PL>(shb, td);
            stsh<PL>(shb, t, fmadd(f0, f2(x.x + b.x, x.y + b.y),
                               negif(fmul(f1, f2(fmaf(gK, b.x, x.x), fmaf(gK, b.y, x.y))), sc)));
        }
    }
}

// ---------------------------------------------------------------- pairs of steps
// Step weights for the pair bodies.
struct StepW {
    float2 f0, f1;
    int y;
};

constexpr bool two_entry(int k) { return k != DCS_KIND_DIAG && k != DCS_KIND_FIXED; }

// One step on a two-entry orbit (c, d) with signs s_c, s_d (reference formulas).
template <int K>
__device__ __forceinline__ void apply2(float2& xc, float2& xd, int sc, int sd, const StepW& w) {
    const float2 f0 = w.f0, f1 = w.f1;
    if constexpr (K == DCS_KIND_GROW) {
        xd = negif(fmul(f1, xc), sc);
        xc = fmul(f0, xc);
    } else if constexpr (K == DCS_KIND_MIX) {
        const float2 oc = fmadd(f0, xc, negif(fmul(f1, xd), sd));
        xd = fmadd(f0, xd, negif(fmul(f1, xc), sc));
        xc = oc;
    } else if constexpr (K == DCS_KIND_REPLACE) {
        const float2 u = negif(xc, sc), v = negif(xd, sd);
        const float2 oc = fmul(f0, f2(xc.x + xd.x, xc.y + xd.y));
        xd = fmul(f1, f2(u.x + v.x, u.y + v.y));
        xc = oc;
    } else if constexpr (K == DCS_KIND_FIXED_SHRINK) {
        if (w.y) {
            const float2 u = negif(xc, sc), v = negif(xd, sd);
            xc = fmul(f1, f2(u.x + v.x, u.y + v.y));
        } else {
            xc = fmul(f0, f2(xc.x + xd.x, xc.y + xd.y));
        }
    } else {  // DCS_KIND_SHRINK2: f0 (x + b) + f1 (s_c x + s_d b)
        const float2 u = negif(xc, sc), v = negif(xd, sd);
        xc = fmadd(f1, f2(u.x + v.x, u.y + v.y), fmul(f0, f2(xc.x + xd.x, xc.y + xd.y)));
    }
}

// One step on a one-entry orbit with sign s.
template <int K>
__device__ __forceinline__ void apply1(float2& x, int s, const StepW& w) {
    if constexpr (K == DCS_KIND_DIAG) {
        x = fmadd(w.f0, x, negif(fmul(w.f1, x), s));
    } else {  // DCS_KIND_FIXED
        x = w.y ? negif(fmul(w.f1, x), s) : fmul(w.f0, x);
    }
}

// Two consecutive steps per shared-memory round trip.  Super-orbit entries:
// e0 = t, e1 = t ^ tau1, e2 = t ^ tau2, e3 = t ^ tau1 ^ tau2 (e1/e3 absent when step 1 has
// one-entry orbits, e2/e3 when step 2 has).  t is zero at both steps' role coordinates, so e0
// is entry c of both steps; step 1 acts on (e0, e1) and (e2, e3), step 2 on (e0, e2) and (e1, e3),
// with the second pair's roles swapped when the other step's vector has the role bit set.
template <int K1, int K2>
__device__ __forceinline__ void run_pair(unsigned char* __restrict__ shb, int T, const FusedStep& a, const StepW& wa,
                                         int csa, bool doa, const FusedStep& b, const StepW& wb, int csb, bool dob) {
    constexpr bool A2 = two_entry(K1), B2 = two_entry(K2);
    const int nrep = T >> a.pnins;
    if ((int)threadIdx.x >= nrep) return;
    const uint32_t ta3 = a.tbeta << 3, tb3 = b.tbeta << 3;
    const uint32_t tp = spread(threadIdx.x, a.pins, a.pnins) << 3;
    const int hsa = (__popc(tp & ta3) & 1) ^ csa, hsb = (__popc(tp & tb3) & 1) ^ csb;
    const uint32_t mhi3 = a.pmhi << 3, tau1 = a.tau1 << 3, tau2 = a.tau2 << 3;
    const int niter = nrep > kThreads ? nrep >> kThreadLog : 1;
    const int a1 = a.s1e[1], a2 = a.s1e[2], a3 = a.s1e[3], b1 = a.s2e[1], b2 = a.s2e[2], b3 = a.s2e[3];
    const bool swB = a.swapB, swA = a.swapA;
    uint32_t tu = 0;
#pragma unroll 2
    for (int k = 0; k < niter; ++k) {
        const uint32_t t0 = tp | tu;
        const int sa = hsa ^ (__popc(tu & ta3) & 1), sb = hsb ^ (__popc(tu & tb3) & 1);
        tu = ((tu | ~mhi3) + 1u) & mhi3;
        const uint32_t t1 = t0 ^ tau1, t2 = t0 ^ tau2, t3 = t1 ^ tau2;
        float2 e0 = ldsh<false>(shb, t0), e1, e2, e3;
        if constexpr (A2) e1 = ldsh<false>(shb, t1);
        if constexpr (B2) e2 = ldsh<false>(shb, t2);
        if constexpr (A2 && B2) e3 = ldsh<false>(shb, t3);
        if (doa) {
            if constexpr (A2) {
                apply2<K1>(e0, e1, sa, sa ^ a1, wa);
                if constexpr (B2) {
                    if (swB) apply2<K1>(e3, e2, sa ^ a3, sa ^ a2, wa);
                    else apply2<K1>(e2, e3, sa ^ a2, sa ^ a3, wa);
                }
            } else {
                apply1<K1>(e0, sa, wa);
                if constexpr (B2) apply1<K1>(e2, sa ^ a2, wa);
            }
        }
        if (dob) {
            if constexpr (B2) {
                apply2<K2>(e0, e2, sb, sb ^ b2, wb);
                if constexpr (A2) {
                    if (swA) apply2<K2>(e3, e1, sb ^ b3, sb ^ b1, wb);
                    else apply2<K2>(e1, e3, sb ^ b1, sb ^ b3, wb);
                }
            } else {
                apply1<K2>(e0, sb, wb);
                if constexpr (A2) apply1<K2>(e1, sb ^ b1, wb);
            }
        }
        stsh<false>(shb, t0, e0);
        if constexpr (A2) stsh<false>(shb, t1, e1);
        if constexpr (B2) stsh<false>(shb, t2, e2);
        if constexpr (A2 && B2) stsh<false>(shb, t3, e3);
    }
}

template <int K1>
__device__ __forceinline__ void dispatch_pair2(int k2, unsigned char* shb, int T, const FusedStep& a,
                                               const StepW& wa, int csa, bool doa, const FusedStep& b,
                                               const StepW& wb, int csb, bool dob) {
    switch (k2) {
        case DCS_KIND_GROW: run_pair<K1, DCS_KIND_GROW>(shb, T, a, wa, csa, doa, b, wb, csb, dob); break;
        case DCS_KIND_MIX: run_pair<K1, DCS_KIND_MIX>(shb, T, a, wa, csa, doa, b, wb, csb, dob); break;
        case DCS_KIND_DIAG: run_pair<K1, DCS_KIND_DIAG>(shb, T, a, wa, csa, doa, b, wb, csb, dob); break;
        case DCS_KIND_REPLACE: run_pair<K1, DCS_KIND_REPLACE>(shb, T, a, wa, csa, doa, b, wb, csb, dob); break;
        case DCS_KIND_FIXED: run_pair<K1, DCS_KIND_FIXED>(shb, T, a, wa, csa, doa, b, wb, csb, dob); break;
        case DCS_KIND_FIXED_SHRINK:
            run_pair<K1, DCS_KIND_FIXED_SHRINK>(shb, T, a, wa, csa, doa, b, wb, csb, dob);
            break;
        default: run_pair<K1, DCS_KIND_SHRINK2>(shb, T, a, wa, csa, doa, b, wb, csb, dob); break;
    }
}

__device__ __forceinline__ void dispatch_pair(int k1, int k2, unsigned char* shb, int T, const FusedStep& a,
                                              const StepW& wa, int csa, bool doa, const FusedStep& b,
                                              const StepW& wb, int csb, bool dob) {
    switch (k1) {
        case DCS_KIND_GROW: dispatch_pair2<DCS_KIND_GROW>(k2, shb, T, a, wa, csa, doa, b, wb, csb, dob); break;
        case DCS_KIND_MIX: dispatch_pair2<DCS_KIND_MIX>(k2, shb, T, a, wa, csa, doa, b, wb, csb, dob); break;
        case DCS_KIND_DIAG: dispatch_pair2<DCS_KIND_DIAG>(k2, shb, T, a, wa, csa, doa, b, wb, csb, dob); break;
        case DCS_KIND_REPLACE: dispatch_pair2<DCS_KIND_REPLACE>(k2, shb, T, a, wa, csa, doa, b, wb, csb, dob); break;
        case DCS_KIND_FIXED: dispatch_pair2<DCS_KIND_FIXED>(k2, shb, T, a, wa, csa, doa, b, wb, csb, dob); break;
        case DCS_KIND_FIXED_SHRINK:
            dispatch_pair2<DCS_KIND_FIXED_SHRINK>(k2, shb, T, a, wa, csa, doa, b, wb, csb, dob);
            break;
        default: dispatch_pair2<DCS_KIND_SHRINK2>(k2, shb, T, a, wa, csa, doa, b, wb, csb, dob); break;
    }
}

// ---------------------------------------------------------------- packed orbit pairs
// Paired tile layout: a thread takes the representatives t and t + 1 (tile bit 0 free at the
// step) together, one per lane of a float2, and does the arithmetic of both with the packed
// FP32x2 instructions.  Lane 1's sign is lane 0's flipped by tile bit 0 of beta.  A partner
// vector v with bit 0 set lands the partners of t and t + 1 in lanes 1 and 0 of the pair at
// (t ^ v) & ~1: the lanes are swapped on load and back on store.
struct C2 {
    float2 re, im;  // lanes: entry t, entry t + 1
};
// a complex factor on both lanes, with its negated imaginary part
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
template <bool SW>
__device__ __forceinline__ C2 lanes(const C2& v) {
    if constexpr (SW) return C2{f2(v.re.y, v.re.x), f2(v.im.y, v.im.x)};
    else return v;
}
// f v
__device__ __forceinline__ C2 cmul(const CF& f, const C2& v) {
    return C2{__ffma2_rn(f.ni, v.im, __fmul2_rn(f.r, v.re)), __ffma2_rn(f.i, v.re, __fmul2_rn(f.r, v.im))};
}
// acc + f v
__device__ __forceinline__ C2 cmadd(const CF& f, const C2& v, const C2& acc) {
    return C2{__ffma2_rn(f.ni, v.im, __ffma2_rn(f.r, v.re, acc.re)),
              __ffma2_rn(f.i, v.re, __ffma2_rn(f.r, v.im, acc.im))};
}
// lane signs s v (s = +-1 per lane)
__device__ __forceinline__ C2 smul(float2 s, const C2& v) { return C2{__fmul2_rn(s, v.re), __fmul2_rn(s, v.im)}; }
__device__ __forceinline__ C2 cadd(const C2& a, const C2& b) { return C2{__fadd2_rn(a.re, b.re), __fadd2_rn(a.im, b.im)}; }
// a + g b, g = +-1 on both lanes
__device__ __forceinline__ C2 caddg(const C2& a, float2 g, const C2& b) {
    return C2{__ffma2_rn(g, b.re, a.re), __ffma2_rn(g, b.im, a.im)};
}

// Step weights of the packed bodies.
struct PW {
    CF F0, F1, F1a;   // f0, f1, (-1)^sKa f1
    float2 gK, gKa;   // (-1)^sK, (-1)^sKa on both lanes
    int y;
};

// One vertex step over the active representative pairs of the tile (bit 0 of the tile index
// is free at the step).  The sign identities used: with S the lane signs of the entries c,
// f0 b + S f1 x = S (f0 (S b) + f1 x), so one lane-sign product on each side of the formula
// replaces a per-lane factor.
template <int KIND, bool SW1, bool SW2>
__device__ __forceinline__ void run_packed(unsigned char* __restrict__ shb, int T, const FusedStep& st, const PW& w,
                                           int cs) {
    const int nins = st.nins;
    const int nrep = T >> (nins + 1);  // representative pairs (t, t + 1), a power of two
    if ((int)threadIdx.x >= nrep) return;
    const uint32_t tbeta3 = st.tbeta << 3;
    const uint32_t tp = spread(threadIdx.x << 1, st.ins, nins) << 3;
    // lane-0 sign as the bit pattern of +-1.0f; lane 1 differs by tile bit 0 of beta
    const uint32_t h0 = (((uint32_t)(__popc(tp & tbeta3) ^ cs) & 1u) << 31) ^ 0x3f800000u;
    const uint32_t d0 = (st.tbeta & 1u) << 31;
    const uint32_t mhi = st.mhi & (st.mhi - 1u);  // the free tile bits past the threads, bit 0 excluded
    const uint32_t mhi3 = mhi << 3;
    const int niter = nrep > kThreads ? nrep >> kThreadLog : 1;
    const uint32_t tK = (st.tK & ~1u) << 3, tKa = (st.tKa & ~1u) << 3, tpiv = (st.tpiv & ~1u) << 3;
    uint32_t tu = 0;
#pragma unroll 4
    for (int k = 0; k < niter; ++k) {
        const uint32_t t = tp | tu;
        const uint32_t sb = ((uint32_t)__popc(tu & tbeta3) << 31) ^ h0;
        const float2 S = f2(__uint_as_float(sb), __uint_as_float(sb ^ d0));
        tu = ((tu | ~mhi3) + 1u) & mhi3;
        const C2 x = ldc2(shb, t);
        if constexpr (KIND == DCS_KIND_GROW) {
            stc2(shb, t, cmul(w.F0, x));
            stc2(shb, t ^ tpiv, smul(S, cmul(w.F1, x)));
        } else if constexpr (KIND == DCS_KIND_MIX) {
            // o0 = f0 x + S f1a b ;  o1 = f0 b + S f1 x = S (f0 (S b) + f1 x)
            const uint32_t td = t ^ tKa;
            const C2 bs = smul(S, lanes<SW1>(ldc2(shb, td)));
            stc2(shb, t, cmadd(w.F0, x, cmul(w.F1a, bs)));
            stc2(shb, td, lanes<SW1>(smul(S, cmadd(w.F0, bs, cmul(w.F1, x)))));
        } else if constexpr (KIND == DCS_KIND_DIAG) {
            // (f0 + S f1) x: lane factor f0 + f1 or f0 - f1
            const CF F{__ffma2_rn(S, w.F1.r, w.F0.r), __ffma2_rn(S, w.F1.i, w.F0.i), __ffma2_rn(S, w.F1.ni, w.F0.ni)};
            stc2(shb, t, cmul(F, x));
        } else if constexpr (KIND == DCS_KIND_REPLACE) {
            // o0 = f0 (x + b) ;  o1 = S f1 (x + gK b)
            const uint32_t td = t ^ tK;
            const C2 b = lanes<SW1>(ldc2(shb, td));
            stc2(shb, t, cmul(w.F0, cadd(x, b)));
            stc2(shb, td, lanes<SW1>(smul(S, cmul(w.F1, caddg(x, w.gK, b)))));
        } else if constexpr (KIND == DCS_KIND_FIXED) {
            stc2(shb, t, w.y ? smul(S, cmul(w.F1, x)) : cmul(w.F0, x));
        } else if constexpr (KIND == DCS_KIND_FIXED_SHRINK) {
            const C2 b = lanes<SW1>(ldc2(shb, t ^ tK));
            stc2(shb, t, w.y ? smul(S, cmul(w.F1, caddg(x, w.gK, b))) : cmul(w.F0, cadd(x, b)));
        } else if constexpr (KIND == DCS_KIND_SHRINK4) {
            // o0 = f0 (x + b) + S gKa f1 (g + gK h) ;  o1 = f0 (g + h) + S f1 (x + gK b)
            constexpr bool SWH = SW1 != SW2;
            const uint32_t td = t ^ tKa;
            const C2 b = lanes<SW1>(ldc2(shb, t ^ tK)), g = lanes<SW2>(ldc2(shb, td));
            const C2 h = lanes<SWH>(ldc2(shb, td ^ tK));
            const float2 Sd = __fmul2_rn(S, w.gKa);
            stc2(shb, t, cmadd(w.F0, cadd(x, b), smul(Sd, cmul(w.F1, caddg(g, w.gK, h)))));
            stc2(shb, td, lanes<SW2>(cmadd(w.F0, cadd(g, h), smul(S, cmul(w.F1, caddg(x, w.gK, b))))));
        } else {  // DCS_KIND_SHRINK2: f0 (x + b) + S f1 (x + gK b)
            const C2 b = lanes<SW1>(ldc2(shb, t ^ tK));
            stc2(shb, t, cmadd(w.F0, cadd(x, b), smul(S, cmul(w.F1, caddg(x, w.gK, b)))));
        }
    }
}

// Packed step if tile bit 0 is free at the step; false means "use the one-entry path".
__device__ __forceinline__ bool dispatch_packed(unsigned char* shb, int T, int tile_dim, const FusedStep& st,
                                                const PW& w, int cs) {
    if (st.nins >= tile_dim || (st.nins && st.ins[0] == 0)) return false;
    const bool k1 = st.tK & 1u, ka1 = st.tKa & 1u;
    switch (st.kind) {
        case DCS_KIND_GROW:
            if (st.tpiv & 1u) return false;
            run_packed<DCS_KIND_GROW, false, false>(shb, T, st, w, cs);
            break;
        case DCS_KIND_MIX:
            if (ka1) run_packed<DCS_KIND_MIX, true, false>(shb, T, st, w, cs);
            else run_packed<DCS_KIND_MIX, false, false>(shb, T, st, w, cs);
            break;
        case DCS_KIND_DIAG: run_packed<DCS_KIND_DIAG, false, false>(shb, T, st, w, cs); break;
        case DCS_KIND_REPLACE:
            if (k1) run_packed<DCS_KIND_REPLACE, true, false>(shb, T, st, w, cs);
            else run_packed<DCS_KIND_REPLACE, false, false>(shb, T, st, w, cs);
            break;
        case DCS_KIND_FIXED: run_packed<DCS_KIND_FIXED, false, false>(shb, T, st, w, cs); break;
        case DCS_KIND_FIXED_SHRINK:
            if (k1) run_packed<DCS_KIND_FIXED_SHRINK, true, false>(shb, T, st, w, cs);
            else run_packed<DCS_KIND_FIXED_SHRINK, false, false>(shb, T, st, w, cs);
            break;
        case DCS_KIND_SHRINK4:
            if (k1) {
                if (ka1) run_packed<DCS_KIND_SHRINK4, true, true>(shb, T, st, w, cs);
                else run_packed<DCS_KIND_SHRINK4, true, false>(shb, T, st, w, cs);
            } else {
                if (ka1) run_packed<DCS_KIND_SHRINK4, false, true>(shb, T, st, w, cs);
                else run_packed<DCS_KIND_SHRINK4, false, false>(shb, T, st, w, cs);
            }
            break;
        default:
            if (k1) run_packed<DCS_KIND_SHRINK2, true, false>(shb, T, st, w, cs);
            else run_packed<DCS_KIND_SHRINK2, false, false>(shb, T, st, w, cs);
            break;
    }
    return true;
}

template <int MINB, bool PACKED>
__global__ void __launch_bounds__(kThreads, MINB)
k_fused(float2* __restrict__ E, const __grid_constant__ FusedArgs A, const dcs_param* __restrict__ params,
        unsigned long long* __restrict__ maxbits, dcs_scale* __restrict__ scale) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int T = 1 << A.tile_dim;
    const int low = A.low_bits;
    const int nhi = 1 << (A.tile_dim - low);
    float2* sh = reinterpret_cast<float2*>(smem);
    uint64_t* hi_tab = reinterpret_cast<uint64_t*>(smem + sizeof(float2) * (size_t)T);
    __shared__ float4 fw[kMaxSteps];
    __shared__ int ovy[kMaxSteps];

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
        // load (only entries active before the group; the rest are written before being read):
        // asynchronous copies, zero-filled for inactive entries, all in flight at once.  When
        // slot 0 is active before the group, entries t and t+1 (t even) share their activity
        // and sit in one aligned 16-byte pair: one copy moves both.
        if (PACKED || A.pair_in) {
            for (int t = 2 * threadIdx.x; t < T; t += 2 * kThreads) {
                const uint64_t a = base ^ hi_tab[t >> low] ^ ((uint64_t)t & lowmask);
                const bool act = !(a & in_inactive);
                const uint32_t dst = (uint32_t)__cvta_generic_to_shared(&sh[t]);
                if (A.pair_in) {
                    const float2* src = act ? E + a : E;
                    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src),
                                 "r"(act ? 16 : 0)
                                 : "memory");
                } else {  // packed layout, entries t and t + 1 separately (different rows or activity)
                    const uint64_t a1 = base ^ hi_tab[(t + 1) >> low] ^ ((uint64_t)(t + 1) & lowmask);
                    const bool act1 = !(a1 & in_inactive);
                    const float2* src = act ? E + a : E;
                    const float2* src1 = act1 ? E + a1 : E;
                    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst), "l"(src),
                                 "r"(act ? 8 : 0)
                                 : "memory");
                    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst + 8u), "l"(src1),
                                 "r"(act1 ? 8 : 0)
                                 : "memory");
                }
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
        asm volatile("cp.async.wait_all;\n" ::: "memory");
        if constexpr (PACKED) {
            // interleaved -> paired layout, each thread on the 16-byte pairs it copied itself
            for (int t = 2 * threadIdx.x; t < T; t += 2 * kThreads) {
                float4* q = reinterpret_cast<float4*>(&sh[t]);
                const float4 v = *q;
                *q = make_float4(v.x, v.z, v.y, v.w);
            }
        }
        __syncthreads();
        for (int s = 0; s < A.count;) {
            const FusedStep& st = A.st[s];
            const float4 w = fw[s];
            const float2 f0 = f2(w.x, w.y), f1 = f2(w.z, w.w);
            const int y = ovy[s] >> 1;
            // tile-constant part of the sign: parity(base & beta) ^ ov
            const int cs = (__popcll(base & st.beta) & 1) ^ (ovy[s] & 1);
            if constexpr (!PACKED) {
                if (st.pair && s + 1 < A.count) {
                    const FusedStep& st2 = A.st[s + 1];
                    const float4 w2 = fw[s + 1];
                    const StepW wa{f0, f1, y}, wb{f2(w2.x, w2.y), f2(w2.z, w2.w), ovy[s + 1] >> 1};
                    const int cs2 = (__popcll(base & st2.beta) & 1) ^ (ovy[s + 1] & 1);
                    dispatch_pair(st.kind, st2.kind, smem, T, st, wa, cs, !(base & st.cskip), st2, wb, cs2,
                                  !(base & st2.cskip));
                    __syncthreads();
                    s += 2;
                    continue;
                }
            }
            if (!(base & st.cskip)) {
                bool done = false;
                if constexpr (PACKED) {
                    const float gK = st.sK ? -1.f : 1.f, gKa = st.sKa ? -1.f : 1.f;
                    const PW pw{cf(f0), cf(f1), cf(f2(gKa * f1.x, gKa * f1.y)), f2(gK, gK), f2(gKa, gKa), y};
                    done = dispatch_packed(smem, T, A.tile_dim, st, pw, cs);
                }
                if (!done) switch (st.kind) {
                    case DCS_KIND_GROW: run_step<DCS_KIND_GROW, PACKED>(smem, T, st, f0, f1, cs, y); break;
                    case DCS_KIND_MIX: run_step<DCS_KIND_MIX, PACKED>(smem, T, st, f0, f1, cs, y); break;
                    case DCS_KIND_DIAG: run_step<DCS_KIND_DIAG, PACKED>(smem, T, st, f0, f1, cs, y); break;
                    case DCS_KIND_REPLACE: run_step<DCS_KIND_REPLACE, PACKED>(smem, T, st, f0, f1, cs, y); break;
                    case DCS_KIND_FIXED: run_step<DCS_KIND_FIXED, PACKED>(smem, T, st, f0, f1, cs, y); break;
                    case DCS_KIND_FIXED_SHRINK:
                        run_step<DCS_KIND_FIXED_SHRINK, PACKED>(smem, T, st, f0, f1, cs, y);
                        break;
                    case DCS_KIND_SHRINK4: run_step<DCS_KIND_SHRINK4, PACKED>(smem, T, st, f0, f1, cs, y); break;
                    default: run_step<DCS_KIND_SHRINK2, PACKED>(smem, T, st, f0, f1, cs, y); break;
                }
            }
            __syncthreads();
            ++s;
        }
        // store (only entries active after the group) and max; pairs when slot 0 is active after
        if constexpr (PACKED) {
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
                const float2 v = f2(sh[t].x * sc, sh[t].y * sc);  // the pass's 2^-e (exact; the steps are linear)
                lm = fmaxf(lm, v.x * v.x + v.y * v.y);
                E[a] = v;
            }
        }
        __syncthreads();
    }
    const unsigned long long bm = block_max_u64(max_bits(lm));
    if (threadIdx.x == 0 && bm) atomicMax(&maxbits[A.group + 1], bm);
}

}  // namespace

extern "C" int dcs_fused_groups(void* table, const dcs_step* steps, int nsteps, const dcs_group* groups, int ngroups,
                                const dcs_tile_step* tile_steps, const dcs_param* params, int g0, int ng,
                                uint64_t* maxbits, dcs_scale* scale, void* stream) {
    if (!table || !steps || !groups || !tile_steps || !params || !maxbits || !scale || g0 < 0 || ng < 0 ||
        g0 + ng > ngroups) {
        dcs_host::set_error("dcs_fused_groups: invalid arguments");
        return DCS_E_ARG;
    }
    const int sms = dcs_host::sm_count();
    if (sms <= 0) return DCS_E_CUDA;
    cudaStream_t st = (cudaStream_t)stream;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        dcs_host::set_error("dcs_fused_groups: no current device");
        return DCS_E_CUDA;
    }
    static int max_smem_set[64] = {0};
    for (int gi = g0; gi < g0 + ng; ++gi) {
        const dcs_group& g = groups[gi];
        if (g.count < 1 || g.count > kMaxSteps || g.first < 0 || g.first + g.count > nsteps || g.tile_dim < 0 ||
            g.tile_dim > 14 || g.low_bits < 0 || g.low_bits > g.tile_dim || g.tile_dim - g.low_bits > 16 ||
            g.ncoset_runs < 0 || g.ncoset_runs > DCS_MAX_RUNS || g.coset_m < 0 || g.coset_m > DCS_MAX_SLOTS) {
            dcs_host::set_error("dcs_fused_groups: malformed group %d", gi);
            return DCS_E_ARG;
        }
        // variant bit 0: two CTAs per SM (more registers); bit 1: paired layout with packed
        // FP32x2 arithmetic (tiles of at least two entries)
        const bool packed = (g.variant & 2) && g.tile_dim >= 1;
        FusedArgs A;
        memset(&A, 0, sizeof(A));
        A.count = g.count;
        A.tile_dim = g.tile_dim;
        A.low_bits = g.low_bits;
        A.coset_m = g.coset_m;
        A.ncoset_runs = g.ncoset_runs;
        A.group = gi;
        A.in_mask_first = steps[g.first].in_mask;
        A.out_mask_last = g.out_mask;
        A.pair_in = g.low_bits >= 1 && (A.in_mask_first & 1ull);
        A.pair_out = g.low_bits >= 1 && (A.out_mask_last & 1ull);
        for (int i = 0; i < 16; ++i) A.basis[i] = g.basis[i];
        for (int r = 0; r < DCS_MAX_RUNS; ++r) A.coset_runs[r] = g.coset_runs[r];
        for (int s = 0; s < g.count; ++s) {
            const dcs_step& d = steps[g.first + s];
            const dcs_tile_step& ts = tile_steps[g.step_tile_off + s];
            FusedStep& f = A.st[s];
            f.beta = d.beta;
            f.cskip = ts.cskip;
            f.tK = ts.tK; f.tKa = ts.tKa; f.tpiv = ts.tpiv; f.tbeta = ts.tbeta;
            f.sK = ts.sK; f.sKa = ts.sKa; f.nins = ts.nins; f.mhi = ts.mhi;
            f.pair = !packed && ts.pair && s + 1 < g.count && d.kind != DCS_KIND_SHRINK4 &&
                     steps[g.first + s + 1].kind != DCS_KIND_SHRINK4;
            f.pnins = ts.pnins; f.swapB = ts.swapB; f.swapA = ts.swapA;
            f.pmhi = ts.pmhi; f.tau1 = ts.tau1; f.tau2 = ts.tau2;
            for (int i = 0; i < 4; ++i) { f.s1e[i] = ts.s1e[i]; f.s2e[i] = ts.s2e[i]; }
            f.kind = d.kind;
            f.pidx = g.first + s;
            bool bad = f.nins > 16 || f.nins > g.tile_dim || (f.tK | f.tKa | f.tpiv | f.tbeta) >> g.tile_dim;
            for (int i = 0; i < f.nins && !bad; ++i) {
                f.ins[i] = ts.ins[i];
                bad = ts.ins[i] >= g.tile_dim || (i && ts.ins[i] <= ts.ins[i - 1]);
            }
            if (f.pair) {
                bad = bad || f.pnins > 16 || f.pnins > g.tile_dim || (f.tau1 | f.tau2) >> g.tile_dim;
                for (int i = 0; i < f.pnins && !bad; ++i) {
                    f.pins[i] = ts.pins[i];
                    bad = ts.pins[i] >= g.tile_dim || (i && ts.pins[i] <= ts.pins[i - 1]);
                }
            }
            if (bad) {
                dcs_host::set_error("dcs_fused_groups: malformed tile step %d", g.first + s);
                return DCS_E_ARG;
            }
        }
        const size_t smem = sizeof(float2) * ((size_t)1 << g.tile_dim) +
                            sizeof(uint64_t) * ((size_t)1 << (g.tile_dim - g.low_bits));
        if (!max_smem_set[dev]) {
            const int lim = 160 * 1024;
            cudaError_t e = cudaFuncSetAttribute(k_fused<3, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(k_fused<2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(k_fused<3, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(k_fused<2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
            if (e != cudaSuccess) return dcs_host::check_cuda(e, "k_fused smem attribute");
            max_smem_set[dev] = 1;
        }
        const uint64_t ntiles = 1ull << g.coset_m;
        const bool two = g.variant & 1;
        // resident CTAs per SM for this shared-memory size (persistent grid: one wave)
        int per_sm = 0;
        cudaError_t oe;
        if (packed)
            oe = two ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fused<2, true>, kThreads, smem)
                     : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fused<3, true>, kThreads, smem);
        else
            oe = two ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fused<2, false>, kThreads, smem)
                     : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fused<3, false>, kThreads, smem);
        if (oe != cudaSuccess) return dcs_host::check_cuda(oe, "k_fused occupancy");
        if (per_sm < 1) per_sm = 1;
        uint64_t grid = (uint64_t)sms * per_sm;
        if (grid > ntiles) grid = ntiles;
        // at least 3 CTAs per SM (register cap 85) or 2 CTAs per SM (more registers)
        float2* E = (float2*)table;
        unsigned long long* mb = (unsigned long long*)maxbits;
        if (packed) {
            if (two) k_fused<2, true><<<(unsigned)grid, kThreads, smem, st>>>(E, A, params, mb, scale);
            else k_fused<3, true><<<(unsigned)grid, kThreads, smem, st>>>(E, A, params, mb, scale);
        } else {
            if (two) k_fused<2, false><<<(unsigned)grid, kThreads, smem, st>>>(E, A, params, mb, scale);
            else k_fused<3, false><<<(unsigned)grid, kThreads, smem, st>>>(E, A, params, mb, scale);
        }
        DCS_CHECK_LAUNCH("k_fused launch");
    }
    return DCS_OK;
}
