// Gather-form vertex step on two tables (sm_100a): the executor of the reference's
// ConditionalBlockGPU (source/dcs_rankwidth/gpu_kernel.py:58-103, scan_step_scaled, driven by
// source/sampling/conditional_block_gpu.py:92-126).  It is not the production path (the in-place
// executor is), but keeps the reference's second engine available on the B200.
//
// Per output c' of 2^r_out: p0 = XOR over the bytes of c' of the step's byte table (the right
// inverse L applied to c'), then the sum over the kernel combinations p = p0 ^ combo of
// E[p & mask_in] times f_v(y) with sign (-1)^(y * (parity(c & beta) ^ ov)), y = bit r_in of p for a
// free step, else the fixed value.  Sums are FP64 for both storages (as the reference's kernel),
// written scaled by 2^-e.  Differences by design: e is derived on the device from the previous
// step's max (no host sync); the byte tables and combinations of the step sit in shared memory;
// several work items (slices) per launch (blockIdx.y).
#include "common.cuh"

using namespace dcs;

namespace {

constexpr int kThreads = 256;
constexpr int kMaxTableWords = 8 * 256;  // up to 64-bit outputs
constexpr int kMaxCombos = 64;

template <class S>
__global__ void __launch_bounds__(kThreads)
k_gather(const S* __restrict__ Ein, S* __restrict__ Eout, uint64_t stride, const __grid_constant__ dcs_gather_step st,
         const uint64_t* __restrict__ words, int s, const dcs_param* __restrict__ params, uint64_t param_stride,
         unsigned long long* __restrict__ maxbits, uint64_t maxbits_stride, dcs_scale* __restrict__ scale) {
    using R = typename Store<S>::R;
    __shared__ uint64_t T[kMaxTableWords];
    __shared__ uint64_t C[kMaxCombos];
    const int item = blockIdx.y;
    const S* E = Ein + (uint64_t)item * stride;
    S* out = Eout + (uint64_t)item * stride;
    const dcs_param p = params[(uint64_t)item * param_stride + s];
    unsigned long long* mb = maxbits + (uint64_t)item * maxbits_stride;
    const double m2prev = (double)bits_to_m2<R>(mb[s]);
    const int e = scale_exponent(m2prev);
    const double sc = ldexp(1.0, -e);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        dcs_scale* sp = scale + item;
        sp->logscale += (double)e * 0.69314718055994530942;
        sp->exponent_sum += e;
        if (!isfinite(m2prev)) sp->flags |= 1u;
        else if (m2prev == 0.0) sp->flags |= 2u;
    }
    for (int i = threadIdx.x; i < st.nbytes * 256; i += kThreads) T[i] = words[st.table_off + i];
    for (int i = threadIdx.x; i < st.ncombos; i += kThreads) C[i] = words[st.combo_off + i];
    __syncthreads();
    const uint64_t mask = st.r_in >= 64 ? ~0ull : ((1ull << st.r_in) - 1ull);
    const uint64_t n_out = 1ull << st.r_out;
    const uint64_t beta = st.beta;
    const int ov = p.ov & 1, y_fixed = p.y & 1;
    // the two weights with their sign applied, as FP64
    const double w0r = p.f0r, w0i = p.f0i, w1r = p.f1r, w1i = p.f1i;
    R lm = 0;
    for (uint64_t cp = (uint64_t)blockIdx.x * kThreads + threadIdx.x; cp < n_out; cp += (uint64_t)gridDim.x * kThreads) {
        uint64_t p0 = 0;
        for (int b = 0; b < st.nbytes; ++b) p0 ^= T[b * 256 + (int)((cp >> (8 * b)) & 255)];
        double ar = 0.0, ai = 0.0;
        for (int k = 0; k < st.ncombos; ++k) {
            const uint64_t q = p0 ^ C[k];
            const uint64_t c = q & mask;
            const int par = neg_sign(c, beta, ov);
            const int y = st.free_ ? (int)((q >> st.r_in) & 1ull) : y_fixed;
            double wr = y ? w1r : w0r, wi = y ? w1i : w0i;
            if (y & par) {
                wr = -wr;
                wi = -wi;
            }
            const double2 v = entry_f64(E[c]);
            ar += v.x * wr - v.y * wi;
            ai += v.x * wi + v.y * wr;
        }
        const S o = Store<S>::make((R)(ar * sc), (R)(ai * sc));
        out[cp] = o;
        lm = fmax(lm, o.x * o.x + o.y * o.y);
    }
    const unsigned long long mx = block_max_u64(max_bits(lm));
    if (threadIdx.x == 0 && mx) atomicMax(&mb[s + 1], mx);
}

template <class S>
int run_steps(void* a, void* b, uint64_t stride, const dcs_gather_step* steps, const uint64_t* words,
              const dcs_param* params, uint64_t param_stride, int s0, int count, unsigned long long* maxbits,
              uint64_t maxbits_stride, dcs_scale* scale, int n_items, cudaStream_t stream) {
    const int sms = dcs_host::sm_count();
    S* bufs[2] = {(S*)a, (S*)b};
    for (int s = s0; s < s0 + count; ++s) {
        const dcs_gather_step& st = steps[s];
        if (st.nbytes < 1 || st.nbytes > 8 || st.ncombos < 1 || st.ncombos > kMaxCombos || st.r_out > 62 ||
            st.r_in > 62) {
            dcs_host::set_error("dcs_gather_steps: step %d outside the kernel's limits", s);
            return DCS_E_ARG;
        }
        const uint64_t n_out = 1ull << st.r_out;
        const uint64_t want = (n_out + kThreads - 1) / kThreads;
        const unsigned grid = (unsigned)(want < (uint64_t)sms * 8 ? want : (uint64_t)sms * 8);
        const int k = s - s0;
        k_gather<S><<<dim3(grid, n_items), kThreads, 0, stream>>>(bufs[k & 1], bufs[(k & 1) ^ 1], stride, st, words, s,
                                                                 params, param_stride, maxbits, maxbits_stride,
                                                                 scale);
        DCS_CHECK_LAUNCH("k_gather");
    }
    return DCS_OK;
}

}  // namespace

extern "C" int dcs_gather_steps(int dtype, void* table_a, void* table_b, uint64_t stride, const dcs_gather_step* steps,
                                const uint64_t* words, const dcs_param* params, uint64_t param_stride, int s0,
                                int count, unsigned long long* maxbits, uint64_t maxbits_stride, dcs_scale* scale,
                                int n_items, void* stream) {
    if (!table_a || !table_b || !steps || !words || !params || !maxbits || !scale || s0 < 0 || count < 0 ||
        n_items < 1 || n_items > 65535 || (dtype != DCS_C64 && dtype != DCS_C128)) {
        dcs_host::set_error("dcs_gather_steps: invalid arguments");
        return DCS_E_ARG;
    }
    if (dtype == DCS_C64)
        return run_steps<float2>(table_a, table_b, stride, steps, words, params, param_stride, s0, count, maxbits,
                                 maxbits_stride, scale, n_items, (cudaStream_t)stream);
    return run_steps<double2>(table_a, table_b, stride, steps, words, params, param_stride, s0, count, maxbits,
                              maxbits_stride, scale, n_items, (cudaStream_t)stream);
}
