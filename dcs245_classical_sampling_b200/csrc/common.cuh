// Shared device helpers for the conditional-block kernels (sm_100a).
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "dcs245.h"

namespace dcs {

// ---------------------------------------------------------------- complex arithmetic
template <class S> struct Store;
template <> struct Store<float2> {
    using R = float;
    static __device__ __forceinline__ float2 make(float r, float i) { return make_float2(r, i); }
};
template <> struct Store<double2> {
    using R = double;
    static __device__ __forceinline__ double2 make(double r, double i) { return make_double2(r, i); }
};

template <class S> __device__ __forceinline__ S cmul(S a, S b) {
    return Store<S>::make(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <class S> __device__ __forceinline__ S cadd(S a, S b) { return Store<S>::make(a.x + b.x, a.y + b.y); }
// multiply by (-1)^neg
template <class S> __device__ __forceinline__ S cneg_if(S a, int neg) {
    return neg ? Store<S>::make(-a.x, -a.y) : a;
}
template <class S> __device__ __forceinline__ S cscale(S a, typename Store<S>::R s) {
    return Store<S>::make(a.x * s, a.y * s);
}

// Table entries in memory type M, arithmetic in S: M == S for complex64 / complex128 tables;
// M = ushort2 (two IEEE binary16 components, 4 bytes) with S = double2 for the half-storage
// tier, which keeps the reference's FP64 arithmetic and rounds only on the store
// (source/kernel_opt/inplace_half_gpu.py:22-26): FP64 -> FP32 -> binary16, each to nearest even.
// st() writes an entry and returns |stored value|^2 for the renormalisation max; for binary16
// that is the max of the rounded values, summed in FP32 as the reference does.
template <class S, class M> struct Mem;
template <class S> struct Mem<S, S> {
    using Q = typename Store<S>::R;  // type of the running max
    static __device__ __forceinline__ S ld(const S& m) { return m; }
    static __device__ __forceinline__ Q st(S* E, uint64_t c, S v) {
        E[c] = v;
        return v.x * v.x + v.y * v.y;
    }
};
template <> struct Mem<double2, ushort2> {
    using Q = float;  // |v|^2 of a binary16 pair is exact in FP32 up to the final rounding
    static __device__ __forceinline__ double2 ld(const ushort2& m) {
        const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&m));
        return make_double2((double)f.x, (double)f.y);
    }
    static __device__ __forceinline__ float st(ushort2* E, uint64_t c, double2 v) {
        const __half2 h = __floats2half2_rn(__double2float_rn(v.x), __double2float_rn(v.y));
        E[c] = *reinterpret_cast<const ushort2*>(&h);
        const float2 r = __half22float2(h);
        return r.x * r.x + r.y * r.y;
    }
};
// an entry of any table type as FP64 (re, im)
__device__ __forceinline__ double2 entry_f64(const float2& v) { return make_double2((double)v.x, (double)v.y); }
__device__ __forceinline__ double2 entry_f64(const double2& v) { return v; }
__device__ __forceinline__ double2 entry_f64(const ushort2& v) {
    return make_double2((double)__half2float(__ushort_as_half(v.x)), (double)__half2float(__ushort_as_half(v.y)));
}

// parity(c & beta) ^ ov : 1 means the sign is -1
__device__ __forceinline__ int neg_sign(uint64_t c, uint64_t beta, int ov) {
    return (__popcll(c & beta) & 1) ^ ov;
}

// deposit the low bits of x into slot runs (src | dst << 8 | len << 16)
__device__ __forceinline__ uint64_t deposit(uint64_t x, const uint32_t* runs, int nruns) {
    uint64_t c = 0;
    for (int r = 0; r < nruns; ++r) {
        const uint32_t w = runs[r];
        const int src = w & 255, dst = (w >> 8) & 255, len = (w >> 16) & 255;
        c |= ((x >> src) & ((len >= 64) ? ~0ull : ((1ull << len) - 1))) << dst;
    }
    return c;
}

// bit pattern of |x|^2 for atomicMax (non-negative floats order like unsigned ints; NaN and
// +inf patterns compare above every finite value)
__device__ __forceinline__ unsigned long long max_bits(float m2) { return (unsigned long long)__float_as_uint(m2); }
__device__ __forceinline__ unsigned long long max_bits(double m2) { return (unsigned long long)__double_as_longlong(m2); }

template <class R> __device__ __forceinline__ R bits_to_m2(unsigned long long b);
template <> __device__ __forceinline__ float bits_to_m2<float>(unsigned long long b) { return __uint_as_float((uint32_t)b); }
template <> __device__ __forceinline__ double bits_to_m2<double>(unsigned long long b) { return __longlong_as_double((long long)b); }

// exponent e of frexp(sqrt(m2)) (0 for m2 == 0 or nonfinite), computed as the reference's
// host loop does: maximum = sqrt(m2) in FP64, e = frexp(maximum)[1]
__device__ __forceinline__ int scale_exponent(double m2) {
    if (!(m2 > 0.0) || !isfinite(m2)) return 0;
    int e;
    frexp(sqrt(m2), &e);
    return e;
}

// block-wide max of an unsigned 64-bit value; result valid in thread 0
__device__ __forceinline__ unsigned long long block_max_u64(unsigned long long v) {
    __shared__ unsigned long long red[32];
    for (int off = 16; off > 0; off >>= 1) {
        unsigned long long o = __shfl_xor_sync(0xffffffffu, v, off);
        v = o > v ? o : v;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (warp == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        v = lane < nw ? red[lane] : 0ull;
        for (int off = 16; off > 0; off >>= 1) {
            unsigned long long o = __shfl_xor_sync(0xffffffffu, v, off);
            v = o > v ? o : v;
        }
    }
    return v;
}

}  // namespace dcs

// error plumbing shared by the ABI translation units
namespace dcs_host {
void set_error(const char* fmt, ...);
int check_cuda(cudaError_t e, const char* what);
int sm_count();
}  // namespace dcs_host

#define DCS_CHECK_LAUNCH(what)                                                      \
    do {                                                                            \
        cudaError_t _e = cudaGetLastError();                                        \
        if (_e != cudaSuccess) return dcs_host::check_cuda(_e, what);               \
    } while (0)
