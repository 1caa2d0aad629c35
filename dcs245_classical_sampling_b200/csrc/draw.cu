// FP64 inverse-CDF draw of the free bits from a complex128 block (sm_100a).
//
// Reference: `draw_checked`, source/sampling/sampling_protocol.py:44-88.  The reference
// computes weights w = re*re + im*im (two roundings, no FMA), the SEQUENTIAL cumulative sum
// S_i, divides by S_n, forces the last value to 1 and takes searchsorted(u, side='right'),
// i.e. the first i with u < S_i/S_n.  It cross-checks the chosen bin with math.fsum.
//
// Device method:
//   1. weights with the same two-rounding formula (__dmul_rn/__dadd_rn), plus double-double
//      (error-free TwoSum, Knuth; Dekker) partial sums per chunk;
//   2. exclusive double-double scan of the chunk sums -> total T (accurate to ~2^-104);
//   3. the chunk and element with P_{i-1} <= u*T < P_i (P = accurate prefix sums);
//   4. certification: a sequential FP64 sum of non-negative terms satisfies
//      |S_i - P_i| <= gamma_{i} P_i (Higham, Accuracy and Stability, Sec. 4.2), so if u lies
//      outside the error intervals of both bin edges, numpy's index is the same index.
//      Otherwise the block is flagged as a tie and an exact sequential FP64 pass (the same
//      operation order as numpy's cumsum) decides — on the device, without host sync.  On
//      request (DCS_DRAW_SEQUENTIAL) that pass runs for every block, so that the reported CDF
//      values are numpy's bit for bit (the production record rows derive a grid count from them);
//   5. the 53-bit grid total-variation diagnostic of the reference.
#include <cuda.h>
#include <string.h>

#include <mutex>

#include "common.cuh"

namespace {

struct dd { double hi, lo; };

__device__ __forceinline__ dd two_sum(double a, double b) {
    const double s = __dadd_rn(a, b);
    const double bb = __dsub_rn(s, a);
    const double err = __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb));
    return {s, err};
}
__device__ __forceinline__ dd fast_two_sum(double a, double b) {
    const double s = __dadd_rn(a, b);
    return {s, __dsub_rn(b, __dsub_rn(s, a))};
}
__device__ __forceinline__ dd dd_add(dd a, double b) {
    dd s = two_sum(a.hi, b);
    return fast_two_sum(s.hi, __dadd_rn(s.lo, a.lo));
}
__device__ __forceinline__ dd dd_add(dd a, dd b) {
    dd s = two_sum(a.hi, b.hi);
    return fast_two_sum(s.hi, __dadd_rn(s.lo, __dadd_rn(a.lo, b.lo)));
}
__device__ __forceinline__ dd dd_mul(dd a, double b) {  // Dekker product with FMA error term
    const double p = __dmul_rn(a.hi, b);
    const double e = fma(a.hi, b, -p);
    return fast_two_sum(p, __dadd_rn(e, __dmul_rn(a.lo, b)));
}
__device__ __forceinline__ double dd_div(dd a, dd b) {  // a / b to ~1 ulp
    if (b.hi == 0.0) return 0.0;
    const double q = a.hi / b.hi;
    const dd qb = dd_mul(b, q);
    const dd r = dd_add(a, dd{-qb.hi, -qb.lo});
    return q + r.hi / b.hi;
}
__device__ __forceinline__ bool dd_lt(dd a, dd b) { return a.hi < b.hi || (a.hi == b.hi && a.lo < b.lo); }

constexpr int kChunkLog = 11;
constexpr int kChunk = 1 << kChunkLog;
constexpr int kThreads = 256;
constexpr int kPer = kChunk / kThreads;

struct BlockState {  // per block scratch (device)
    dd total;
    double total_plain;
    int64_t chunk;
    int32_t status;
    int32_t nonfinite;
};

// sequential pass: one checkpoint (the running FP64 sum before the group) per 32 elements
constexpr int kSeqLog = 5;
__host__ __device__ constexpr size_t seq_groups(size_t n) { return (n + 31) >> kSeqLog; }

// layout of the scratch area
struct Layout {
    size_t w, chunk_sum, state, tv_part, sq_part, ckpt, bytes;
};
__host__ __device__ constexpr Layout layout(int k, int nblocks) {
    const size_t n = (size_t)1 << k;
    const size_t nch = n >= (size_t)kChunk ? n / kChunk : 1;
    Layout L{};
    L.w = 0;
    L.chunk_sum = L.w + n * nblocks * sizeof(double);
    L.state = L.chunk_sum + nch * nblocks * sizeof(dd);
    L.tv_part = L.state + nblocks * sizeof(BlockState);
    L.sq_part = L.tv_part + nch * nblocks * sizeof(double);
    L.ckpt = L.sq_part + nch * nblocks * sizeof(double);
    L.bytes = L.ckpt + seq_groups(n) * nblocks * sizeof(double);
    L.bytes = (L.bytes + 255) & ~(size_t)255;
    return L;
}

__device__ __forceinline__ dd block_sum_dd(dd v) {
    __shared__ dd red[kThreads / 32];
    for (int off = 16; off > 0; off >>= 1) {
        dd o{__shfl_xor_sync(0xffffffffu, v.hi, off), __shfl_xor_sync(0xffffffffu, v.lo, off)};
        v = dd_add(v, o);
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        dd s = red[0];
        for (int w = 1; w < kThreads / 32; ++w) s = dd_add(s, red[w]);
        red[0] = s;
    }
    __syncthreads();
    dd r = red[0];
    __syncthreads();
    return r;
}

// 1. weights + per-chunk double-double sums
__global__ void __launch_bounds__(kThreads)
k_weights(const double2* __restrict__ blocks, int k, double* __restrict__ w, dd* __restrict__ chunk_sum,
          BlockState* __restrict__ state) {
    const int b = blockIdx.y;
    const uint64_t n = 1ull << k;
    const uint64_t start = (uint64_t)blockIdx.x * kChunk;
    const double2* v = blocks + ((uint64_t)b << k);
    double* wb = w + ((uint64_t)b << k);
    dd acc{0.0, 0.0};
    int bad = 0;
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
        const uint64_t i = start + threadIdx.x + (uint64_t)j * kThreads;
        if (i < n) {
            const double2 a = v[i];
            bad |= !isfinite(a.x) || !isfinite(a.y);
            const double wi = __dadd_rn(__dmul_rn(a.x, a.x), __dmul_rn(a.y, a.y));
            wb[i] = wi;
            acc = dd_add(acc, wi);
        }
    }
    const dd s = block_sum_dd(acc);
    const int anybad = __syncthreads_or(bad);
    if (threadIdx.x == 0) {
        chunk_sum[(uint64_t)b * gridDim.x + blockIdx.x] = s;
        if (anybad) atomicOr(&state[b].nonfinite, 1);
    }
}

// 2. chunk scan (sequential over <= 2^k/2048 chunks) + chunk search, one thread per block
__global__ void k_scan_locate(dd* __restrict__ chunk_sum, int nch, const double* __restrict__ uniforms,
                              BlockState* __restrict__ state, dcs_draw_result* __restrict__ res) {
    const int b = blockIdx.x;
    dd* cs = chunk_sum + (uint64_t)b * nch;
    dd run{0.0, 0.0};
    for (int c = 0; c < nch; ++c) {  // exclusive scan in place
        const dd s = cs[c];
        cs[c] = run;
        run = dd_add(run, s);
    }
    BlockState& st = state[b];
    st.total = run;
    const double u = uniforms[b];
    dcs_draw_result& r = res[b];
    memset(&r, 0, sizeof(r));
    r.uniform = u;
    r.index = -1;
    if (st.nonfinite || !(u >= 0.0 && u < 1.0)) { r.status = DCS_E_ARG; st.status = DCS_E_ARG; return; }
    if (!(run.hi > 0.0) || !isfinite(run.hi)) { r.status = DCS_E_CDF; st.status = DCS_E_CDF; return; }
    const dd target = dd_mul(run, u);
    // last chunk whose exclusive start is <= target
    int lo = 0, hi = nch - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (dd_lt(target, cs[mid])) hi = mid - 1; else lo = mid;
    }
    st.chunk = lo;
    st.status = 0;
}

// 3. element search inside the chunk + certification (one CTA per block)
__global__ void __launch_bounds__(kThreads)
k_locate_elem(const double* __restrict__ w, int k, const dd* __restrict__ chunk_sum, int nch,
              BlockState* __restrict__ state, dcs_draw_result* __restrict__ res) {
    const int b = blockIdx.x;
    BlockState& st = state[b];
    if (st.status) return;
    const uint64_t n = 1ull << k;
    const int64_t c = st.chunk;
    const uint64_t start = (uint64_t)c * kChunk;
    const double* wb = w + ((uint64_t)b << k);
    const dd off = chunk_sum[(uint64_t)b * nch + c];
    const dd T = st.total;
    const double u = res[b].uniform;
    const dd target = dd_mul(T, u);
    // thread t owns kPer consecutive elements
    __shared__ dd pre[kThreads];
    double loc[kPer];
    dd acc{0.0, 0.0};
    for (int j = 0; j < kPer; ++j) {
        const uint64_t i = start + (uint64_t)threadIdx.x * kPer + j;
        loc[j] = i < n ? wb[i] : 0.0;
        acc = dd_add(acc, loc[j]);
    }
    pre[threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {  // exclusive scan of the 256 thread sums
        dd run = off;
        for (int t = 0; t < kThreads; ++t) {
            const dd s = pre[t];
            pre[t] = run;
            run = dd_add(run, s);
        }
    }
    __syncthreads();
    // each thread scans its own elements; the first i with P_i > target wins
    dd run = pre[threadIdx.x];
    int64_t found = -1;
    dd p_before{0, 0}, p_at{0, 0};
    for (int j = 0; j < kPer; ++j) {
        const uint64_t i = start + (uint64_t)threadIdx.x * kPer + j;
        if (i >= n) break;
        const dd nxt = dd_add(run, loc[j]);
        if (dd_lt(target, nxt) && loc[j] > 0.0) {
            found = (int64_t)i;
            p_before = run;
            p_at = nxt;
            break;
        }
        run = nxt;
    }
    __shared__ unsigned long long best;
    if (threadIdx.x == 0) best = ~0ull;
    __syncthreads();
    if (found >= 0) atomicMin(&best, (unsigned long long)found);
    __syncthreads();
    if (found >= 0 && (unsigned long long)found == best) {
        dcs_draw_result& r = res[b];
        // math.fsum rounds each sum to double before the division (sampling_protocol.py:67-69);
        // a normalised double-double's high word is that rounding
        const double lo = __ddiv_rn(p_before.hi, T.hi), hi = __ddiv_rn(p_at.hi, T.hi);
        const double wi = loc[found - (int64_t)start - (int64_t)threadIdx.x * kPer];
        r.index = found;
        r.selected_weight = wi;
        r.total_exact = T.hi;
        r.total_cdf = r.total_exact;
        r.cdf_lower_exact = lo;
        r.cdf_upper_exact = hi;
        r.cdf_lower = found ? lo : 0.0;
        r.cdf_upper = ((uint64_t)found == n - 1) ? 1.0 : hi;
        // certification against numpy's sequential cumsum (bound on each side + 4 ulp slack)
        const double eps = 1.1102230246251565e-16;  // 2^-53
        const double rel = ((double)found + (double)n + 8.0) * eps;
        const bool low_ok = found == 0 || lo * (1.0 + rel) <= u;
        const bool high_ok = ((uint64_t)found == n - 1) || hi * (1.0 - rel) > u;
        r.tie = !(low_ok && high_ok);
        r.status = 0;
    }
    if (threadIdx.x == 0 && best == ~0ull) {
        // u*T beyond every accurate prefix (possible only within rounding of T): sequential path decides
        res[b].tie = 1;
        res[b].total_exact = T.hi;
    }
}

// 4. exact sequential FP64 CDF (numpy's operation order), one warp per block: for blocks
//    flagged as ties, or for every block when `force`.  Every lane runs the same dependent
//    chain S <- S + w_i (the 32 weights of a group are loaded by the 32 lanes and broadcast by
//    shuffles, the next 128 prefetched), so the chain is numpy's cumsum exactly.  Pass 1 gives
//    S_n and a checkpoint before every 32-element group; the selected group is the last one
//    whose starting value satisfies fl(start / S_n) <= u (fl(x / S_n) is non-decreasing in x),
//    and pass 2 replays that group only.  The compensated interval of the selected index is
//    checked against u as the reference's independent check does (sampling_protocol.py:67-72).
__global__ void __launch_bounds__(32)
k_sequential(const double* __restrict__ w, int k, const dd* __restrict__ chunk_sum, int nch,
             BlockState* __restrict__ state, dcs_draw_result* __restrict__ res, double* __restrict__ ckpt,
             int force) {
    const int b = blockIdx.x;
    const int lane = threadIdx.x;
    dcs_draw_result& r = res[b];
    if (state[b].status || !(r.tie || force)) return;
    const uint64_t n = 1ull << k;
    const uint64_t ng = seq_groups(n);
    const double* wb = w + ((uint64_t)b << k);
    double* ck = ckpt + (uint64_t)b * ng;
    // pass 1: S_n with checkpoints, four groups (128 weights) per iteration, the next four in flight
    double S = 0.0;
    double cur[4], nxt[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const uint64_t i = (uint64_t)q * 32 + lane;
        cur[q] = i < n ? wb[i] : 0.0;
    }
    for (uint64_t g0 = 0; g0 < ng; g0 += 4) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const uint64_t i = (g0 + 4 + q) * 32 + lane;
            nxt[q] = i < n ? wb[i] : 0.0;
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if (g0 + q < ng) {
                if (lane == 0) ck[g0 + q] = S;
                const uint64_t base = (g0 + q) * 32;
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const double v = __shfl_sync(0xffffffffu, cur[q], j);
                    if (base + j < n) S = __dadd_rn(S, v);
                }
            }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) cur[q] = nxt[q];
    }
    if (lane != 0) return;  // lane 0 wrote the checkpoints and finishes alone
    if (!(S > 0.0) || !isfinite(S)) {
        r.status = DCS_E_CDF;
        return;
    }
    const double u = r.uniform;
    // last group whose starting value's quotient is <= u (group 0 starts at 0)
    uint64_t lo = 0, hi = ng - 1;
    while (lo < hi) {
        const uint64_t mid = (lo + hi + 1) >> 1;
        if (__ddiv_rn(ck[mid], S) <= u) lo = mid; else hi = mid - 1;
    }
    // pass 2: replay the group; the last element's value is forced to 1 (numpy: cumulative[-1] = 1)
    double run = ck[lo], prev = __ddiv_rn(run, S);
    uint64_t idx = n - 1;
    double upper = 1.0;
    for (uint64_t i = lo * 32; i < n && i < (lo + 1) * 32; ++i) {
        run = __dadd_rn(run, wb[i]);
        const double ci = (i == n - 1) ? 1.0 : __ddiv_rn(run, S);
        if (u < ci) { idx = i; upper = ci; break; }
        prev = ci;
    }
    // compensated prefix before idx: the scan's chunk prefix plus the chunk's elements before idx
    const uint64_t c0 = idx / kChunk;
    dd pre = chunk_sum[(uint64_t)b * nch + c0];
    for (uint64_t i = c0 * kChunk; i < idx; ++i) pre = dd_add(pre, wb[i]);
    const dd at = dd_add(pre, wb[idx]);
    const dd T = state[b].total;
    r.cdf_lower = idx ? prev : 0.0;
    r.cdf_upper = upper;
    r.cdf_lower_exact = __ddiv_rn(pre.hi, T.hi);
    r.cdf_upper_exact = __ddiv_rn(at.hi, T.hi);
    r.index = (int64_t)idx;
    r.total_cdf = S;
    r.total_exact = T.hi;
    r.selected_weight = wb[idx];
    if (!(wb[idx] > 0.0)) r.status = DCS_E_CDF;
    // the reference's independent check of the interval (a disagreement is an error, never a resample)
    else if (!(r.cdf_lower_exact <= u && u < r.cdf_upper_exact)) r.status = DCS_E_CDF;
}

// 5. 53-bit grid TV and the sum of squared weights, per chunk partial sums (deterministic final
//    sums in k_tv_final)
__global__ void __launch_bounds__(kThreads)
k_tv(const double* __restrict__ w, int k, const dd* __restrict__ chunk_sum, int nch,
     const BlockState* __restrict__ state, const dcs_draw_result* __restrict__ res, double* __restrict__ part,
     double* __restrict__ sq_part) {
    const int b = blockIdx.y;
    const int c = blockIdx.x;
    const uint64_t n = 1ull << k;
    if (state[b].status) return;
    const dd T = state[b].total;
    const double mass = res[b].total_exact;
    const uint64_t start = (uint64_t)c * kChunk;
    const double* wb = w + ((uint64_t)b << k);
    __shared__ dd pre[kThreads];
    double loc[kPer];
    dd acc{0.0, 0.0};
    for (int j = 0; j < kPer; ++j) {
        const uint64_t i = start + (uint64_t)threadIdx.x * kPer + j;
        loc[j] = i < n ? wb[i] : 0.0;
        acc = dd_add(acc, loc[j]);
    }
    pre[threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        dd run = chunk_sum[(uint64_t)b * nch + c];
        for (int t = 0; t < kThreads; ++t) {
            const dd s = pre[t];
            pre[t] = run;
            run = dd_add(run, s);
        }
    }
    __syncthreads();
    dd run = pre[threadIdx.x];
    const double two53 = 9007199254740992.0;
    double prev_end = ceil(dd_div(run, T) * two53);
    if (start + (uint64_t)threadIdx.x * kPer == 0) prev_end = 0.0;
    double s = 0.0, q = 0.0;
    for (int j = 0; j < kPer; ++j) {
        const uint64_t i = start + (uint64_t)threadIdx.x * kPer + j;
        if (i >= n) break;
        run = dd_add(run, loc[j]);
        const double ci = (i == n - 1) ? 1.0 : dd_div(run, T);
        const double end = ceil(ci * two53);
        s += fabs((end - prev_end) / two53 - loc[j] / mass);
        const double p = loc[j] / mass;
        q = fma(p, p, q);
        prev_end = end;
    }
    const dd tot = block_sum_dd(dd{s, 0.0});
    const dd sq = block_sum_dd(dd{q, 0.0});
    if (threadIdx.x == 0) {
        part[(uint64_t)b * nch + c] = tot.hi + tot.lo;
        sq_part[(uint64_t)b * nch + c] = sq.hi + sq.lo;
    }
}

__global__ void k_tv_final(const double* __restrict__ part, const double* __restrict__ sq_part, int nch,
                           const BlockState* __restrict__ state, dcs_draw_result* __restrict__ res, int nblocks) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nblocks) return;
    if (state[b].status) { res[b].status = state[b].status; return; }
    double s = 0.0, q = 0.0;
    for (int c = 0; c < nch; ++c) {
        s += part[(uint64_t)b * nch + c];
        q += sq_part[(uint64_t)b * nch + c];
    }
    res[b].tv53 = 0.5 * s;
    res[b].weight_l2 = q;
}

// ---------------------------------------------------------------- audit overlap
__global__ void __launch_bounds__(kThreads)
k_overlap(const double2* __restrict__ ref, const double2* __restrict__ ap, uint64_t len, dd* __restrict__ part) {
    dd rr{0, 0}, aa{0, 0}, re{0, 0}, im{0, 0};
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (uint64_t)gridDim.x * blockDim.x) {
        const double2 r = ref[i], a = ap[i];
        rr = dd_add(rr, r.x * r.x + r.y * r.y);
        aa = dd_add(aa, a.x * a.x + a.y * a.y);
        re = dd_add(re, r.x * a.x + r.y * a.y);   // <ref, ap> = sum conj(ref) * ap
        im = dd_add(im, r.x * a.y - r.y * a.x);
    }
    rr = block_sum_dd(rr);
    aa = block_sum_dd(aa);
    re = block_sum_dd(re);
    im = block_sum_dd(im);
    if (threadIdx.x == 0) {
        part[4 * blockIdx.x + 0] = rr;
        part[4 * blockIdx.x + 1] = aa;
        part[4 * blockIdx.x + 2] = re;
        part[4 * blockIdx.x + 3] = im;
    }
}

__global__ void k_overlap_final(const dd* __restrict__ part, int nparts, double* __restrict__ out) {
    const int q = threadIdx.x;
    if (q >= 4) return;
    dd s{0, 0};
    for (int p = 0; p < nparts; ++p) s = dd_add(s, part[4 * p + q]);
    out[q] = s.hi + s.lo;
}

}  // namespace

extern "C" size_t dcs_draw_scratch_bytes(int k, int nblocks) {
    if (k < 0 || k > 30 || nblocks < 1) return 0;
    return layout(k, nblocks).bytes;
}

namespace {
// the draw kernels on a scratch area laid out by layout(k, nblocks)
int enqueue_draw(const double* blocks, int k, int nblocks, const double* uniforms, unsigned flags, void* scratch,
                 dcs_draw_result* results, cudaStream_t s) {
    const Layout L = layout(k, nblocks);
    char* base = (char*)scratch;
    double* w = (double*)(base + L.w);
    dd* cs = (dd*)(base + L.chunk_sum);
    BlockState* st = (BlockState*)(base + L.state);
    double* part = (double*)(base + L.tv_part);
    double* sq = (double*)(base + L.sq_part);
    double* ck = (double*)(base + L.ckpt);
    const uint64_t n = 1ull << k;
    const int nch = (int)(n >= (uint64_t)kChunk ? n / kChunk : 1);
    // the scratch keeps the previous call's contents: the per-block state must start at zero
    cudaError_t e = cudaMemsetAsync(st, 0, nblocks * sizeof(BlockState), s);
    if (e != cudaSuccess) return dcs_host::check_cuda(e, "dcs_draw memset");
    k_weights<<<dim3(nch, nblocks), kThreads, 0, s>>>((const double2*)blocks, k, w, cs, st);
    DCS_CHECK_LAUNCH("k_weights");
    k_scan_locate<<<nblocks, 1, 0, s>>>(cs, nch, uniforms, st, results);
    DCS_CHECK_LAUNCH("k_scan_locate");
    k_locate_elem<<<nblocks, kThreads, 0, s>>>(w, k, cs, nch, st, results);
    DCS_CHECK_LAUNCH("k_locate_elem");
    k_sequential<<<nblocks, 32, 0, s>>>(w, k, cs, nch, st, results, ck, (flags & DCS_DRAW_SEQUENTIAL) ? 1 : 0);
    DCS_CHECK_LAUNCH("k_sequential");
    k_tv<<<dim3(nch, nblocks), kThreads, 0, s>>>(w, k, cs, nch, st, results, part, sq);
    DCS_CHECK_LAUNCH("k_tv");
    k_tv_final<<<(nblocks + 31) / 32, 32, 0, s>>>(part, sq, nch, st, results, nblocks);
    DCS_CHECK_LAUNCH("k_tv_final");
    return DCS_OK;
}
}  // namespace

extern "C" int dcs_draw_ex(const double* blocks, int k, int nblocks, const double* uniforms, unsigned flags,
                           void* scratch, dcs_draw_result* results, void* stream) {
    if (!blocks || !uniforms || !scratch || !results || k < 0 || k > 30 || nblocks < 1 || nblocks > 65535 ||
        (flags & ~(unsigned)DCS_DRAW_SEQUENTIAL)) {
        dcs_host::set_error("dcs_draw: invalid arguments");
        return DCS_E_ARG;
    }
    return enqueue_draw(blocks, k, nblocks, uniforms, flags, scratch, results, (cudaStream_t)stream);
}

extern "C" int dcs_draw(const double* blocks, int k, int nblocks, const double* uniforms, void* scratch,
                        dcs_draw_result* results, void* stream) {
    return dcs_draw_ex(blocks, k, nblocks, uniforms, 0u, scratch, results, stream);
}

extern "C" int dcs_overlap(const double* ref, const double* ap, uint64_t len, double* out, void* scratch,
                           void* stream) {
    if (!ref || !ap || !out || !scratch || len == 0) {
        dcs_host::set_error("dcs_overlap: invalid arguments");
        return DCS_E_ARG;
    }
    const int parts = 256;
    cudaStream_t s = (cudaStream_t)stream;
    k_overlap<<<parts, kThreads, 0, s>>>((const double2*)ref, (const double2*)ap, len, (dd*)scratch);
    DCS_CHECK_LAUNCH("k_overlap");
    k_overlap_final<<<1, 32, 0, s>>>((const dd*)scratch, parts, out);
    DCS_CHECK_LAUNCH("k_overlap_final");
    return DCS_OK;
}

// ---------------------------------------------------------------- draw without allocation
//
// For callers that cannot allocate device memory at the point where they draw: code that runs
// while a CUDA stream is being captured (cudaMalloc cannot be captured), host runtimes that
// hand the library only the buffers they own and forbid allocation in their sampling loop, and
// latency-sensitive loops where an allocation would synchronise the device.  The scratch lives
// in a file-scope device array of fixed size, so this entry point allocates nothing.
//
// Limit: one block of up to 2^20 amplitudes per call (DCS_DRAW_STATIC_MAX_K); every GPU that
// loads the library holds the array (about 8.4 MiB) until the process exits.
namespace {
constexpr size_t kStaticDrawBytes = layout(DCS_DRAW_STATIC_MAX_K, 1).bytes;
static __device__ __align__(256) unsigned char g_draw_scratch[kStaticDrawBytes];

// The device address of g_draw_scratch, looked up once per device with that device current,
// and the context it was looked up in: a new context on the device (after cudaDeviceReset, or
// a context torn down and created again) loads the module elsewhere, so the lookup is redone.
std::mutex g_static_mutex;
void* g_static_ptr[64] = {nullptr};
void* g_static_ctx[64] = {nullptr};
typedef CUresult (*ctx_get_current_fn)(CUcontext*);

int current_context(void** ctx) {
    static ctx_get_current_fn fn = nullptr;
    if (!fn) {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        const cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q);
        if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !f) {
            dcs_host::set_error("dcs_draw_static: cuCtxGetCurrent is not available");
            return DCS_E_CUDA;
        }
        fn = (ctx_get_current_fn)f;
    }
    CUcontext c = nullptr;
    if (fn(&c) != CUDA_SUCCESS) {
        dcs_host::set_error("dcs_draw_static: cuCtxGetCurrent failed");
        return DCS_E_CUDA;
    }
    *ctx = (void*)c;
    return DCS_OK;
}
}  // namespace

extern "C" int dcs_draw_static(const double* blocks, int k, const double* uniform, dcs_draw_result* result,
                               void* stream) {
    if (!blocks || !uniform || !result || k < 0 || k > 30) {
        dcs_host::set_error("dcs_draw_static: invalid arguments");
        return DCS_E_ARG;
    }
    const Layout L = layout(k, 1);
    if (k > DCS_DRAW_STATIC_MAX_K || L.bytes > kStaticDrawBytes) {
        dcs_host::set_error("dcs_draw_static: block of 2^%d amplitudes exceeds the static maximum of 2^%d", k,
                            DCS_DRAW_STATIC_MAX_K);
        return DCS_E_ARG;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return dcs_host::check_cuda(e, "dcs_draw_static: cudaGetDevice");
    if (dev < 0 || dev >= 64) {
        dcs_host::set_error("dcs_draw_static: device index %d out of range", dev);
        return DCS_E_ARG;
    }
    void* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_static_mutex);
        void* ctx = nullptr;
        const int rc = current_context(&ctx);
        if (rc != DCS_OK) return rc;
        if (!g_static_ptr[dev] || g_static_ctx[dev] != ctx) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_draw_scratch);
            if (e != cudaSuccess) return dcs_host::check_cuda(e, "dcs_draw_static: cudaGetSymbolAddress");
            g_static_ptr[dev] = p;
            g_static_ctx[dev] = ctx;
        }
        scratch = g_static_ptr[dev];
    }
    return enqueue_draw(blocks, k, 1, uniform, 0u, scratch, result, (cudaStream_t)stream);
}
