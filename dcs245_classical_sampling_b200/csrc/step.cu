// One vertex step of the preserved-coordinate plan, in place on one table (sm_100a).
//
// Semantics follow the reference executor kernel `inplace_step`
// (source/kernel_opt/inplace_gpu.py:20-63): every orbit of 1, 2 or 4 table entries is read
// completely before any of its entries is written, orbits are disjoint, so one buffer suffices.
// Differences by design:
//   * the scale 2^-e is derived on the device from the previous step's max (no host sync);
//   * complex64 tables are computed in FP32 (complex128 tables, and the binary16 tables of
//     the half-storage tier, in FP64);
//   * each thread keeps ORB orbits in flight (all loads issued before any arithmetic) so
//     that enough bytes are outstanding to cover HBM latency;
//   * the block max is reduced in shared memory and published with one atomicMax per CTA.
#include <stdarg.h>
#include <stdio.h>

#include <string>

#include "common.cuh"

using namespace dcs;

namespace {

template <class S, int KIND, int ORB, class M = S>
__global__ void __launch_bounds__(256)
k_step(M* __restrict__ table, uint64_t table_stride, const __grid_constant__ dcs_step st, int s,
       const dcs_param* __restrict__ params, uint64_t param_stride,
       unsigned long long* __restrict__ maxbits, uint64_t maxbits_stride, dcs_scale* __restrict__ scale) {
    using R = typename Store<S>::R;
    using IO = Mem<S, M>;
    using Q = typename IO::Q;
    constexpr int NT = 256;  // threads per block (the launch uses exactly this)
    constexpr int LU = ORB == 8 ? 3 : (ORB == 4 ? 2 : 1);
    static_assert((1 << LU) == ORB, "ORB is a power of two");
    const int item = blockIdx.y;
    M* E = table + (uint64_t)item * table_stride;
    const dcs_param p = params[(uint64_t)item * param_stride + s];
    unsigned long long* mb = maxbits + (uint64_t)item * maxbits_stride;
    const double m2prev = (double)bits_to_m2<R>(mb[s]);
    const int e = scale_exponent(m2prev);
    const R sc = (R)ldexp(1.0, -e);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        dcs_scale* sp = scale + item;
        sp->logscale += (double)e * 0.69314718055994530942;  // ln 2, as the reference's e*log(2.)
        sp->exponent_sum += e;
        if (!isfinite(m2prev)) sp->flags |= 1u;
        else if (m2prev == 0.0) sp->flags |= 2u;
    }
    // the power-of-two scale is folded into the weights: (f * 2^-e) * v == (f * v) * 2^-e exactly
    // (outside the subnormal range), and the scaled weights drop two multiplies per output
    const S f0 = cscale(Store<S>::make((R)p.f0r, (R)p.f0i), sc);
    const S f1 = cscale(Store<S>::make((R)p.f1r, (R)p.f1i), sc);
    const int y = p.y;
    const uint64_t norbits = 1ull << st.m;
    const bool ident = st.nruns == 0 || (st.nruns == 1 && st.runs[0] == ((uint32_t)st.m << 16));
    const uint64_t beta = st.beta, K = st.K, Ka = st.Ka, pbit = st.pivot_bit;
    // Orbit x = base | u << 8 | t (t = thread, u = orbit slot of the thread, base a multiple of
    // NT * ORB).  The deposit into the table's slots is OR-linear over those disjoint bit
    // fields and the sign parity(c & beta) is XOR-linear, so both are split into a per-thread
    // part, ORB compile-time combinations of the deposits of bits 8.. 8+LU-1, and one full
    // deposit per iteration.
    auto dep = [&](uint64_t x) { return ident ? x : deposit(x, st.runs, st.nruns); };
    auto par = [&](uint64_t c) { return (int)(__popcll(c & beta) & 1); };
    const uint64_t dt = dep(threadIdx.x);
    uint64_t du[LU];
    int pu = 0;  // bit u = parity of deposit(u << 8) & beta
#pragma unroll
    for (int b = 0; b < LU; ++b) du[b] = dep(1ull << (8 + b));
#pragma unroll
    for (int u = 0; u < ORB; ++u) {
        uint64_t d = 0;
#pragma unroll
        for (int b = 0; b < LU; ++b)
            if (u >> b & 1) d |= du[b];
        pu |= par(d) << u;
    }
    const int st_ov = p.ov ^ par(dt);           // sign of c = parity(base) ^ bit u of pu ^ st_ov
    const int pK = par(K), pKa = par(Ka);       // sign(c ^ K) = sign(c) ^ pK, likewise for Ka
    Q lm = 0;
    constexpr uint64_t chunk = (uint64_t)NT * ORB;
    for (uint64_t base = (uint64_t)blockIdx.x * chunk; base < norbits; base += (uint64_t)gridDim.x * chunk) {
        const uint64_t cb = dep(base) | dt;
        const int sb = par(dep(base)) ^ st_ov;
        uint64_t c[ORB];
        M ra[ORB], rb[ORB], rg[ORB], rh[ORB];  // raw entries: converted to S only when combined
        bool ok[ORB];
#pragma unroll
        for (int u = 0; u < ORB; ++u) {
            const uint64_t x = base + threadIdx.x + (uint64_t)u * NT;
            ok[u] = x < norbits;
            uint64_t cu = cb;
#pragma unroll
            for (int b = 0; b < LU; ++b)
                if (u >> b & 1) cu |= du[b];
            c[u] = cu;
            if (ok[u]) {
                ra[u] = E[cu];
                if constexpr (KIND == DCS_KIND_MIX) rb[u] = E[cu ^ Ka];
                if constexpr (KIND == DCS_KIND_REPLACE || KIND == DCS_KIND_FIXED_SHRINK ||
                              KIND == DCS_KIND_SHRINK2 || KIND == DCS_KIND_SHRINK4)
                    rb[u] = E[cu ^ K];
                if constexpr (KIND == DCS_KIND_SHRINK4) {
                    rg[u] = E[cu ^ Ka];
                    rh[u] = E[cu ^ Ka ^ K];
                }
            }
        }
#pragma unroll
        for (int u = 0; u < ORB; ++u) {
            if (!ok[u]) continue;
            const uint64_t cc = c[u];
            const int sgn = sb ^ (pu >> u & 1);  // 1: entry cc carries the sign -1
            S a, b, g, h;
            a = IO::ld(ra[u]);
            if constexpr (KIND != DCS_KIND_GROW && KIND != DCS_KIND_DIAG && KIND != DCS_KIND_FIXED) b = IO::ld(rb[u]);
            if constexpr (KIND == DCS_KIND_SHRINK4) {
                g = IO::ld(rg[u]);
                h = IO::ld(rh[u]);
            }
            S o0, o1;
            if constexpr (KIND == DCS_KIND_GROW) {
                o0 = cmul(f0, a);
                o1 = cmul(f1, cneg_if(a, sgn));
                const Q m0 = IO::st(E, cc, o0), m1 = IO::st(E, cc | pbit, o1);
                lm = fmax(lm, fmax(m0, m1));
            } else if constexpr (KIND == DCS_KIND_MIX) {
                const uint64_t d = cc ^ Ka;
                o0 = cadd(cmul(f0, a), cmul(f1, cneg_if(b, sgn ^ pKa)));
                o1 = cadd(cmul(f0, b), cmul(f1, cneg_if(a, sgn)));
                const Q m0 = IO::st(E, cc, o0), m1 = IO::st(E, d, o1);
                lm = fmax(lm, fmax(m0, m1));
            } else if constexpr (KIND == DCS_KIND_DIAG) {
                o0 = cmul(cadd(f0, cneg_if(f1, sgn)), a);
                lm = fmax(lm, IO::st(E, cc, o0));
            } else if constexpr (KIND == DCS_KIND_REPLACE) {
                const uint64_t d = cc ^ K;
                o0 = cmul(f0, cadd(a, b));
                o1 = cmul(f1, cadd(cneg_if(a, sgn), cneg_if(b, sgn ^ pK)));
                const Q m0 = IO::st(E, cc, o0), m1 = IO::st(E, d, o1);
                lm = fmax(lm, fmax(m0, m1));
            } else if constexpr (KIND == DCS_KIND_FIXED) {
                o0 = cmul(y ? cneg_if(f1, sgn) : f0, a);
                lm = fmax(lm, IO::st(E, cc, o0));
            } else if constexpr (KIND == DCS_KIND_FIXED_SHRINK) {
                o0 = y ? cmul(f1, cadd(cneg_if(a, sgn), cneg_if(b, sgn ^ pK))) : cmul(f0, cadd(a, b));
                lm = fmax(lm, IO::st(E, cc, o0));
            } else if constexpr (KIND == DCS_KIND_SHRINK4) {
                const uint64_t d = cc ^ Ka;
                const int sd = sgn ^ pKa;
                o0 = cadd(cmul(f0, cadd(a, b)), cmul(f1, cadd(cneg_if(g, sd), cneg_if(h, sd ^ pK))));
                o1 = cadd(cmul(f0, cadd(g, h)), cmul(f1, cadd(cneg_if(a, sgn), cneg_if(b, sgn ^ pK))));
                const Q m0 = IO::st(E, cc, o0), m1 = IO::st(E, d, o1);
                lm = fmax(lm, fmax(m0, m1));
            } else {  // DCS_KIND_SHRINK2
                o0 = cadd(cmul(cadd(f0, cneg_if(f1, sgn)), a), cmul(cadd(f0, cneg_if(f1, sgn ^ pK)), b));
                lm = fmax(lm, IO::st(E, cc, o0));
            }
        }
    }
    const unsigned long long bm = block_max_u64(max_bits((R)lm));
    if (threadIdx.x == 0 && bm) atomicMax(&mb[s + 1], bm);
}

// Reference-compatible kernel: byte address tables, runtime kind, host scale, FP64 arithmetic
// for both storage types (as inplace_gpu.py:13-18 does).
template <class S>
__global__ void __launch_bounds__(256)
k_ref_step(S* __restrict__ E, uint64_t norbits, const uint64_t* __restrict__ T, int nb, int identity,
           int kind, uint64_t K, uint64_t Ka, int pivot, uint64_t beta, int ov, double f0r, double f0i,
           double f1r, double f1i, int fixed_y, double scale, unsigned long long* dmax) {
    using R = typename Store<S>::R;
    const double2 f0 = make_double2(f0r, f0i), f1 = make_double2(f1r, f1i);
    double lm = 0;
    auto rd = [&](uint64_t c) { S v = E[c]; return make_double2((double)v.x, (double)v.y); };
    auto wr = [&](uint64_t c, double2 x) {
        const R r = (R)(x.x * scale), i = (R)(x.y * scale);
        E[c] = Store<S>::make(r, i);
        lm = fmax(lm, (double)(r * r + i * i));
    };
    const uint64_t stride = (uint64_t)blockDim.x * gridDim.x;
    for (uint64_t x = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; x < norbits; x += stride) {
        uint64_t c = identity ? x : 0;
        if (!identity)
            for (int b = 0; b < nb; ++b) c ^= T[256 * b + ((x >> (8 * b)) & 255ull)];
        const double2 a = rd(c);
        if (kind == 0) {
            wr(c, cmul(f0, a));
            wr(c | (1ull << pivot), cmul(f1, cneg_if(a, neg_sign(c, beta, ov))));
        } else if (kind == 1) {
            const uint64_t d = c ^ Ka;
            const double2 b = rd(d);
            const double2 o0 = cadd(cmul(f0, a), cmul(f1, cneg_if(b, neg_sign(d, beta, ov))));
            const double2 o1 = cadd(cmul(f0, b), cmul(f1, cneg_if(a, neg_sign(c, beta, ov))));
            wr(c, o0); wr(d, o1);
        } else if (kind == 2) {
            wr(c, cmul(cadd(f0, cneg_if(f1, neg_sign(c, beta, ov))), a));
        } else if (kind == 3) {
            const uint64_t d = c ^ K;
            const double2 b = rd(d);
            const double2 o0 = cmul(f0, cadd(a, b));
            const double2 o1 = cmul(f1, cadd(cneg_if(a, neg_sign(c, beta, ov)), cneg_if(b, neg_sign(d, beta, ov))));
            wr(c, o0); wr(d, o1);
        } else if (kind == 4) {
            wr(c, cmul(fixed_y ? cneg_if(f1, neg_sign(c, beta, ov)) : f0, a));
        } else if (kind == 5) {
            const uint64_t d = c ^ K;
            const double2 b = rd(d);
            wr(c, fixed_y ? cmul(f1, cadd(cneg_if(a, neg_sign(c, beta, ov)), cneg_if(b, neg_sign(d, beta, ov))))
                          : cmul(f0, cadd(a, b)));
        } else if (kind == 6) {
            const uint64_t c1 = c ^ K, d = c ^ Ka, d1 = d ^ K;
            const double2 b = rd(c1), e = rd(d), g = rd(d1);
            const double2 o0 = cadd(cmul(f0, cadd(a, b)), cmul(f1, cadd(cneg_if(e, neg_sign(d, beta, ov)), cneg_if(g, neg_sign(d1, beta, ov)))));
            const double2 o1 = cadd(cmul(f0, cadd(e, g)), cmul(f1, cadd(cneg_if(a, neg_sign(c, beta, ov)), cneg_if(b, neg_sign(c1, beta, ov)))));
            wr(c, o0); wr(d, o1);
        } else {
            const uint64_t d = c ^ K;
            const double2 b = rd(d);
            wr(c, cadd(cmul(cadd(f0, cneg_if(f1, neg_sign(c, beta, ov))), a),
                       cmul(cadd(f0, cneg_if(f1, neg_sign(d, beta, ov))), b)));
        }
    }
    const unsigned long long bm = sizeof(R) == 4 ? max_bits((float)lm) : max_bits(lm);
    const unsigned long long red = block_max_u64(bm);
    if (threadIdx.x == 0 && red) atomicMax(dmax, red);
}

constexpr int kThreads = 256;

template <class S, int KIND, class M = S>
int launch_kind(M* table, uint64_t table_stride, const dcs_step& st, int s, const dcs_param* params,
                uint64_t param_stride, unsigned long long* maxbits, uint64_t mstride, dcs_scale* scale,
                int nitems, cudaStream_t stream) {
    // orbits in flight per thread: 64 B of loads for MIX-like kinds at every entry size
    constexpr int ORB = sizeof(M) == 16 ? 2 : (sizeof(M) == 8 ? 4 : 8);
    const uint64_t norbits = 1ull << st.m;
    const uint64_t per_block = (uint64_t)kThreads * ORB;
    uint64_t blocks = (norbits + per_block - 1) / per_block;
    const uint64_t cap = (uint64_t)dcs_host::sm_count() * 8;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    dim3 grid((unsigned)blocks, (unsigned)nitems);
    k_step<S, KIND, ORB, M><<<grid, kThreads, 0, stream>>>(table, table_stride, st, s, params, param_stride,
                                                           maxbits, mstride, scale);
    DCS_CHECK_LAUNCH("k_step launch");
    return DCS_OK;
}

template <class S, class M = S>
int launch_step(M* table, uint64_t table_stride, const dcs_step& st, int s, const dcs_param* params,
                uint64_t param_stride, unsigned long long* maxbits, uint64_t mstride, dcs_scale* scale,
                int nitems, cudaStream_t stream) {
    switch (st.kind) {
#define DCS_CASE(K) \
    case K: return launch_kind<S, K, M>(table, table_stride, st, s, params, param_stride, maxbits, mstride, scale, nitems, stream);
        DCS_CASE(DCS_KIND_GROW)
        DCS_CASE(DCS_KIND_MIX)
        DCS_CASE(DCS_KIND_DIAG)
        DCS_CASE(DCS_KIND_REPLACE)
        DCS_CASE(DCS_KIND_FIXED)
        DCS_CASE(DCS_KIND_FIXED_SHRINK)
        DCS_CASE(DCS_KIND_SHRINK4)
        DCS_CASE(DCS_KIND_SHRINK2)
#undef DCS_CASE
    }
    dcs_host::set_error("step %d: unknown orbit kind %d", s, st.kind);
    return DCS_E_ARG;
}

int validate_step(const dcs_step& st, int s) {
    if (st.kind < 0 || st.kind > 7) { dcs_host::set_error("step %d: kind %d out of range", s, st.kind); return DCS_E_ARG; }
    if (st.m < 0 || st.m > DCS_MAX_SLOTS) { dcs_host::set_error("step %d: m=%d out of range", s, st.m); return DCS_E_ARG; }
    if (st.nruns < 0 || st.nruns > DCS_MAX_RUNS) { dcs_host::set_error("step %d: nruns=%d out of range", s, st.nruns); return DCS_E_ARG; }
    int total = 0;
    for (int r = 0; r < st.nruns; ++r) {
        const uint32_t w = st.runs[r];
        const int src = w & 255, dst = (w >> 8) & 255, len = (w >> 16) & 255;
        if (src != total || len < 1 || dst + len > DCS_MAX_SLOTS) {
            dcs_host::set_error("step %d: malformed deposit run %d", s, r);
            return DCS_E_ARG;
        }
        total += len;
    }
    if (total != st.m) { dcs_host::set_error("step %d: deposit runs cover %d bits, m=%d", s, total, st.m); return DCS_E_ARG; }
    return DCS_OK;
}

}  // namespace

extern "C" int dcs_inplace_step(int dtype, void* E, uint64_t norbits, const uint64_t* T, int nb, int identity_map,
                                int kind, uint64_t K, uint64_t Ka, int pivot, uint64_t beta, int ov, double f0r,
                                double f0i, double f1r, double f1i, int fixed_y, double scale, void* dmax, int grid,
                                void* stream) {
    if (!E || !dmax || (!identity_map && (!T || nb < 1 || nb > 8)) || kind < 0 || kind > 7 ||
        (kind == 0 && (pivot < 0 || pivot > 63))) {
        dcs_host::set_error("dcs_inplace_step: invalid arguments");
        return DCS_E_ARG;
    }
    if (norbits == 0) return DCS_OK;
    int sm = dcs_host::sm_count();
    if (sm <= 0) return DCS_E_CUDA;
    uint64_t g = grid > 0 ? (uint64_t)grid : (uint64_t)sm * 32;
    const uint64_t need = (norbits + 255) / 256;
    if (g > need) g = need;
    cudaStream_t st = (cudaStream_t)stream;
    if (dtype == DCS_C64)
        k_ref_step<float2><<<(unsigned)g, 256, 0, st>>>((float2*)E, norbits, T, nb, identity_map, kind, K, Ka, pivot,
                                                        beta, ov, f0r, f0i, f1r, f1i, fixed_y, scale,
                                                        (unsigned long long*)dmax);
    else if (dtype == DCS_C128)
        k_ref_step<double2><<<(unsigned)g, 256, 0, st>>>((double2*)E, norbits, T, nb, identity_map, kind, K, Ka, pivot,
                                                         beta, ov, f0r, f0i, f1r, f1i, fixed_y, scale,
                                                         (unsigned long long*)dmax);
    else {
        dcs_host::set_error("dcs_inplace_step: unknown dtype %d", dtype);
        return DCS_E_ARG;
    }
    DCS_CHECK_LAUNCH("k_ref_step launch");
    return DCS_OK;
}

extern "C" int dcs_slice_steps_batched(int dtype, void* table, uint64_t table_stride, const dcs_step* steps,
                                       const dcs_param* params, uint64_t param_stride, int nsteps, int first,
                                       int count, uint64_t* maxbits, dcs_scale* scale, int nitems, void* stream) {
    if (!table || !steps || !params || !maxbits || !scale || nitems < 1 || nitems > 65535 || first < 0 ||
        count < 0 || first + count > nsteps) {
        dcs_host::set_error("dcs_slice_steps: invalid arguments (first=%d count=%d nsteps=%d nitems=%d)", first,
                            count, nsteps, nitems);
        return DCS_E_ARG;
    }
    cudaStream_t st = (cudaStream_t)stream;
    for (int s = first; s < first + count; ++s) {
        int rc = validate_step(steps[s], s);
        if (rc) return rc;
        if (dtype == DCS_C64)
            rc = launch_step<float2>((float2*)table, table_stride, steps[s], s, params, param_stride,
                                     (unsigned long long*)maxbits, (uint64_t)nsteps + 1, scale, nitems, st);
        else if (dtype == DCS_C128)
            rc = launch_step<double2>((double2*)table, table_stride, steps[s], s, params, param_stride,
                                      (unsigned long long*)maxbits, (uint64_t)nsteps + 1, scale, nitems, st);
        else if (dtype == DCS_H16)
            rc = launch_step<double2, ushort2>((ushort2*)table, table_stride, steps[s], s, params, param_stride,
                                              (unsigned long long*)maxbits, (uint64_t)nsteps + 1, scale, nitems, st);
        else {
            dcs_host::set_error("dcs_slice_steps: unknown dtype %d", dtype);
            return DCS_E_ARG;
        }
        if (rc) return rc;
    }
    return DCS_OK;
}

extern "C" int dcs_slice_steps(int dtype, void* table, const dcs_step* steps, const dcs_param* params, int nsteps,
                               int first, int count, uint64_t* maxbits, dcs_scale* scale, void* stream) {
    return dcs_slice_steps_batched(dtype, table, 0, steps, params, 0, nsteps, first, count, maxbits, scale, 1,
                                   stream);
}
