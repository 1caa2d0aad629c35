// Device-side request generation for the serving loop (sm_100a).
//
// 1. k_philox_prefixes: Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers:
//    as easy as 1, 2, 3", SC 2011) with counter (request id, sample index, 0, 0) and a 64-bit
//    key: the 128 output bits give the closed prefix bits (up to 64, bit i -> i-th closed
//    qubit) and a 53-bit uniform in [0, 1).
// 2. k_build_items: the reference's per-slice bookkeeping (sampling/conditional_block_gpu.py
//    :136-157, kernel_opt/inplace_gpu.py:111-114) from the prefix bits, on the device: per
//    (sample, slice) item the weights f0, f1 of every step (row x_q of U_q for data vertices,
//    the precomputed W U_q for references, f1 negated where a slice flips the vertex), the fixed
//    values y (|f0| <= 1e-12), the offset bits ov (XOR of the later-neighbour masks of fixed
//    vertices with y = 1) and the scatter xor of the terminal offset and the free-vertex flips.
#include "common.cuh"

namespace {

__host__ __device__ inline void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)M0 * c[0], p1 = (uint64_t)M1 * c[2];
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
        k0 += W0; k1 += W1;
    }
}

__global__ void k_philox_prefixes(const uint32_t* __restrict__ req, const uint32_t* __restrict__ idx, int count,
                                  uint32_t key0, uint32_t key1, const int32_t* __restrict__ closed, int nclosed,
                                  uint64_t* __restrict__ xbits, double* __restrict__ uniforms) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    uint32_t c[4] = {req[i], idx[i], 0u, 0u};
    philox4x32_10(c, key0, key1);
    const uint64_t r = ((uint64_t)c[1] << 32) | c[0];
    uint64_t x = 0;
    for (int j = 0; j < nclosed; ++j) x |= ((r >> j) & 1ull) << closed[j];
    xbits[i] = x;
    const uint64_t u = (((uint64_t)c[3] << 32) | c[2]) >> 11;
    uniforms[i] = (double)u * (1.0 / 9007199254740992.0);  // exact: u < 2^53
}

// One CTA per item (sample s, slice l); threads over steps.  Static tables (device):
//   fsel[j]  : 8 doubles = (f for x bit 0: re, im, re, im), (f for x bit 1: ...)
//   xq[j]    : data qubit selecting the row, -1 for references
//   fixidx[j]: index of the step among the fixed steps, -1 if free
//   flip[l * nsteps + j]  : 1 if slice l flips the vertex of step j
//   F[a * fwords + w]     : bit j of the later-neighbour mask of fixed step a, inside the steps
//   tail[a]               : terminal-offset xor contribution of fixed step a
//   coef[2l], coef[2l+1]  : slice coefficient (x independent for reference-vertex slices)
//   freeflip[l]           : free-vertex flips of slice l
struct BuildArgs {
    const double* fsel;
    const int32_t* xq;
    const int32_t* fixidx;
    const uint8_t* flip;
    const uint32_t* F;
    const uint64_t* tail;
    const double* coef;
    const uint64_t* freeflip;
    int nsteps, nfixed, fwords, nslices;
};

__global__ void __launch_bounds__(256)
k_build_items(const __grid_constant__ BuildArgs B, const uint64_t* __restrict__ xbits, int nsamples,
              dcs_param* __restrict__ params, double* __restrict__ coefs, uint64_t* __restrict__ xors) {
    extern __shared__ uint32_t yfix[];  // nfixed flags
    const int item = blockIdx.x;
    const int s = item / B.nslices, l = item % B.nslices;
    if (s >= nsamples) return;
    const uint64_t x = xbits[s];
    dcs_param* P = params + (uint64_t)item * B.nsteps;
    for (int j = threadIdx.x; j < B.nsteps; j += blockDim.x) {
        const int q = B.xq[j];
        const int b = q >= 0 ? (int)((x >> q) & 1ull) : 0;
        const double* f = B.fsel + 8 * j + 4 * b;
        const double sgn = B.flip[(uint64_t)l * B.nsteps + j] ? -1.0 : 1.0;
        dcs_param p;
        p.f0r = f[0]; p.f0i = f[1];
        p.f1r = f[2] * sgn; p.f1i = f[3] * sgn;
        p.ov = 0;
        p.y = 0;
        const int a = B.fixidx[j];
        if (a >= 0) {
            const double m = sqrt(f[0] * f[0] + f[1] * f[1]);
            p.y = (m > 1e-12) ? 0 : 1;
            yfix[a] = (uint32_t)p.y;
        }
        P[j] = p;
    }
    __syncthreads();
    for (int j = threadIdx.x; j < B.nsteps; j += blockDim.x) {
        uint32_t ov = 0;
        for (int a = 0; a < B.nfixed; ++a) ov ^= yfix[a] & (B.F[(uint64_t)a * B.fwords + (j >> 5)] >> (j & 31));
        P[j].ov = (int32_t)(ov & 1u);
    }
    if (threadIdx.x == 0) {
        uint64_t xo = B.freeflip[l];
        for (int a = 0; a < B.nfixed; ++a)
            if (yfix[a]) xo ^= B.tail[a];
        xors[item] = xo;
        coefs[2 * item] = B.coef[2 * l];
        coefs[2 * item + 1] = B.coef[2 * l + 1];
    }
}

}  // namespace

extern "C" int dcs_philox_prefixes(const uint32_t* req, const uint32_t* idx, int count, uint64_t key,
                                   const int32_t* closed, int nclosed, uint64_t* xbits, double* uniforms,
                                   void* stream) {
    if (count < 0 || nclosed < 0 || nclosed > 64 || (count && (!req || !idx || !xbits || !uniforms)) ||
        (nclosed && !closed)) {
        dcs_host::set_error("dcs_philox_prefixes: invalid arguments");
        return DCS_E_ARG;
    }
    if (!count) return DCS_OK;
    k_philox_prefixes<<<(count + 127) / 128, 128, 0, (cudaStream_t)stream>>>(
        req, idx, count, (uint32_t)key, (uint32_t)(key >> 32), closed, nclosed, xbits, uniforms);
    DCS_CHECK_LAUNCH("k_philox_prefixes");
    return DCS_OK;
}

extern "C" void dcs_philox4x32_10_host(uint32_t ctr[4], uint32_t key0, uint32_t key1) {
    philox4x32_10(ctr, key0, key1);
}

extern "C" int dcs_build_items(const double* fsel, const int32_t* xq, const int32_t* fixidx, const uint8_t* flip,
                               const uint32_t* F, const uint64_t* tail, const double* coef, const uint64_t* freeflip,
                               int nsteps, int nfixed, int nslices, const uint64_t* xbits, int nsamples,
                               dcs_param* params, double* coefs, uint64_t* xors, void* stream) {
    if (nsteps < 1 || nfixed < 0 || nfixed > 4096 || nslices < 1 || nsamples < 0 || !fsel || !xq || !fixidx ||
        !flip || (nfixed && (!F || !tail)) || !coef || !freeflip || (nsamples && (!xbits || !params || !coefs ||
        !xors))) {
        dcs_host::set_error("dcs_build_items: invalid arguments");
        return DCS_E_ARG;
    }
    if (!nsamples) return DCS_OK;
    BuildArgs B{fsel, xq, fixidx, flip, F, tail, coef, freeflip, nsteps, nfixed, (nsteps + 31) / 32, nslices};
    const uint64_t items = (uint64_t)nsamples * nslices;
    if (items > 0x7fffffffull) {
        dcs_host::set_error("dcs_build_items: too many items");
        return DCS_E_ARG;
    }
    k_build_items<<<(unsigned)items, 256, sizeof(uint32_t) * (nfixed > 0 ? nfixed : 1), (cudaStream_t)stream>>>(
        B, xbits, nsamples, params, coefs, xors);
    DCS_CHECK_LAUNCH("k_build_items");
    return DCS_OK;
}
