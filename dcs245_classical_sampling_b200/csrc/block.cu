// Block assembly: terminal gather + syndrome scatter + coherent slice sum, then the
// Walsh-Hadamard / open-edge phase / U_open tail (sm_100a).
//
// Reference: source/kernel_opt/inplace_gpu.py:124 (terminal gather),
// source/sampling/conditional_block_gpu.py:155-158 (scatter-add, coefficient
// coef * exp(logscale - (N_full - n + k)/2 ln 2)), :159-171 (tail).
//
// The scatter `total[synd(i) ^ xor] += env(i) * coef` is evaluated as a gather over the
// output index t: i = L(t ^ xor) when t ^ xor lies in the image of the syndrome map
// (parity checks H), with L a left inverse.  Every output entry is owned by one thread and
// the slices of one block are summed in slice order, so the sum is deterministic.
#include <string.h>

#include "common.cuh"

using namespace dcs;

namespace {

struct TermMap {
    uint32_t runs[DCS_MAX_RUNS];  // deposit of i into the terminal slots
    uint32_t linv[32];            // i_j = parity(s & linv[j])
    uint32_t check[32];           // s in image iff parity(s & check[r]) == 0 for all r
    int nruns, tr, nchecks, k;
};

template <class S>
__global__ void __launch_bounds__(256)
k_accumulate(const S* __restrict__ table, uint64_t table_stride, const __grid_constant__ TermMap tm,
             const uint64_t* __restrict__ xors, const double* __restrict__ coefs, const int32_t* __restrict__ item_begin,
             double log_shift, dcs_scale* __restrict__ scale, const unsigned long long* __restrict__ maxbits_final,
             uint64_t mstride, double2* __restrict__ total) {
    // grid.y = output block; items item_begin[b] .. item_begin[b+1]-1 belong to block b
    const int blk = blockIdx.y;
    const int i0 = item_begin[blk], i1 = item_begin[blk + 1];
    double2* out = total + ((uint64_t)blk << tm.k);
    const uint64_t n = 1ull << tm.k;
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (uint64_t)gridDim.x * blockDim.x) {
        double2 acc = out[t];
        for (int it = i0; it < i1; ++it) {
            const dcs_scale sc = scale[it];
            const unsigned long long mf = maxbits_final[(uint64_t)it * mstride];
            if (sc.flags & 3u) continue;  // zero table (skipped slice) or nonfinite (reported)
            if (mf == 0) continue;        // the last step produced an all-zero table
            const uint32_t sv = (uint32_t)(t ^ xors[it]);
            bool in = true;
            for (int r = 0; r < tm.nchecks; ++r) in &= !(__popc(sv & tm.check[r]) & 1);
            if (!in) continue;
            uint32_t i = 0;
            for (int j = 0; j < tm.tr; ++j) i |= (uint32_t)(__popc(sv & tm.linv[j]) & 1) << j;
            const uint64_t c = deposit(i, tm.runs, tm.nruns);
            const double2 v = entry_f64(table[(uint64_t)it * table_stride + c]);
            const double m = exp(sc.logscale - log_shift);
            double cr = coefs[2 * it] * m, ci = coefs[2 * it + 1] * m;
            if (sc.phase != 0.0) {  // step factors divided out by the plan-specialised kernels
                double sp, cp;
                sincos(sc.phase, &sp, &cp);
                const double r = cr * cp - ci * sp;
                ci = cr * sp + ci * cp;
                cr = r;
            }
            const double vr = v.x, vi = v.y;
            acc.x += vr * cr - vi * ci;
            acc.y += vr * ci + vi * cr;
        }
        out[t] = acc;
    }
}

// flags for nonfinite final maxima (the reference checks every step's max, including the last)
__global__ void k_final_flags(const unsigned long long* __restrict__ maxbits_final, uint64_t mstride, int is64,
                              dcs_scale* __restrict__ scale, int nitems) {
    const int it = blockIdx.x * blockDim.x + threadIdx.x;
    if (it >= nitems) return;
    const unsigned long long b = maxbits_final[(uint64_t)it * mstride];
    const double m2 = is64 ? __longlong_as_double((long long)b) : (double)__uint_as_float((uint32_t)b);
    if (!isfinite(m2)) scale[it].flags |= 1u;
}

// ---------------------------------------------------------------- tail
struct TailParams {
    double u[32][8];     // per physical bit: 2x2 complex row-major (re, im)
    uint32_t adj_hi[32]; // open-edge adjacency, b > a
    int k;
};

// Apply per-bit 2x2 transforms over the tile bits [tb_lo, tb_hi) of tiles made of
// physical bits [0, a) (contiguous) and [b_lo, b_hi).  mode 0: Walsh-Hadamard;
// mode 1: multiply by the open-edge phase on load, then U_open.
__global__ void __launch_bounds__(512)
k_tail(double2* __restrict__ total, const __grid_constant__ TailParams tp, int a, int b_lo, int b_hi, int tb_lo,
       int tb_hi, int mode) {
    extern __shared__ double2 sh[];
    const int k = tp.k;
    const int tile_log = a + (b_hi - b_lo);
    const int tsize = 1 << tile_log;
    const uint64_t nblk_elems = 1ull << k;
    const uint64_t ntiles_per_block = nblk_elems >> tile_log;
    const uint64_t blk = blockIdx.x / ntiles_per_block;
    const uint64_t g = blockIdx.x % ntiles_per_block;
    double2* v = total + (blk << k);
    // complement bits: [a, b_lo) then [b_hi, k)
    const int mid = b_lo - a;
    const uint64_t g_lo = g & ((1ull << mid) - 1), g_hi = g >> mid;
    const uint64_t gbase = (g_lo << a) | (g_hi << b_hi);
    auto addr = [&](int t) -> uint64_t {
        const uint64_t lo = (uint64_t)t & ((1ull << a) - 1);
        const uint64_t hi = (uint64_t)t >> a;
        return gbase | lo | (hi << b_lo);
    };
    for (int t = threadIdx.x; t < tsize; t += blockDim.x) {
        const uint64_t ad = addr(t);
        double2 x = v[ad];
        if (mode == 1) {
            int par = 0;
            for (int q = 0; q < k; ++q)
                if ((ad >> q) & 1) par ^= __popc((uint32_t)ad & tp.adj_hi[q]) & 1;
            if (par) { x.x = -x.x; x.y = -x.y; }
        }
        sh[t] = x;
    }
    __syncthreads();
    for (int j = tb_lo; j < tb_hi; ++j) {
        const int q = j < a ? j : b_lo + (j - a);  // physical bit
        const int half = tsize >> 1;
        const double* m = tp.u[q];
        for (int h = threadIdx.x; h < half; h += blockDim.x) {
            const int lo_part = h & ((1 << j) - 1);
            const int t0 = ((h >> j) << (j + 1)) | lo_part;
            const int t1 = t0 | (1 << j);
            const double2 x0 = sh[t0], x1 = sh[t1];
            double2 y0, y1;
            if (mode == 0) {
                y0 = make_double2(x0.x + x1.x, x0.y + x1.y);
                y1 = make_double2(x0.x - x1.x, x0.y - x1.y);
            } else {
                y0 = make_double2(m[0] * x0.x - m[1] * x0.y + m[2] * x1.x - m[3] * x1.y,
                                  m[0] * x0.y + m[1] * x0.x + m[2] * x1.y + m[3] * x1.x);
                y1 = make_double2(m[4] * x0.x - m[5] * x0.y + m[6] * x1.x - m[7] * x1.y,
                                  m[4] * x0.y + m[5] * x0.x + m[6] * x1.y + m[7] * x1.x);
            }
            sh[t0] = y0;
            sh[t1] = y1;
        }
        __syncthreads();
    }
    for (int t = threadIdx.x; t < tsize; t += blockDim.x) v[addr(t)] = sh[t];
}

constexpr int kTailLog = 12;  // 4096 complex128 = 64 KiB of shared memory per tile

int tail_pass(double2* total, const TailParams& tp, int a, int b_lo, int b_hi, int tb_lo, int tb_hi, int mode,
              int nblocks, cudaStream_t st) {
    const int tile_log = a + (b_hi - b_lo);
    const uint64_t tiles = (uint64_t)nblocks << (tp.k - tile_log);
    if (tiles > 0x7fffffffull) {
        dcs_host::set_error("dcs_block_tail: too many tiles");
        return DCS_E_ARG;
    }
    const int threads = tile_log >= 10 ? 512 : (1 << (tile_log > 5 ? tile_log - 1 : 5));
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        dcs_host::set_error("dcs_block_tail: no current device");
        return DCS_E_CUDA;
    }
    static int attr_set[64] = {0};
    if (!attr_set[dev]) {
        cudaError_t e = cudaFuncSetAttribute(k_tail, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)(sizeof(double2) << kTailLog));
        if (e != cudaSuccess) return dcs_host::check_cuda(e, "k_tail smem attribute");
        attr_set[dev] = 1;
    }
    k_tail<<<(unsigned)tiles, threads, sizeof(double2) << tile_log, st>>>(total, tp, a, b_lo, b_hi, tb_lo, tb_hi,
                                                                         mode);
    DCS_CHECK_LAUNCH("k_tail launch");
    return DCS_OK;
}

}  // namespace

static int build_termmap(TermMap& tm, int tr, const uint32_t* runs, int nruns, const uint64_t* tbasis_host, int k) {
    if (tr < 0 || tr > 31 || k < 0 || k > 31 || tr > k || nruns < 0 || nruns > DCS_MAX_RUNS) {
        dcs_host::set_error("dcs_accumulate: tr=%d k=%d nruns=%d out of range", tr, k, nruns);
        return DCS_E_ARG;
    }
    memset(&tm, 0, sizeof(tm));
    tm.tr = tr; tm.k = k; tm.nruns = nruns;
    for (int r = 0; r < nruns; ++r) tm.runs[r] = runs[r];
    // Gauss-Jordan on the tr basis vectors (k bits each): rows = basis, track combinations.
    uint32_t row[32], comb[32];
    int piv[32];
    for (int j = 0; j < tr; ++j) {
        if (tbasis_host[j] >> k) { dcs_host::set_error("dcs_accumulate: basis vector wider than k"); return DCS_E_ARG; }
        row[j] = (uint32_t)tbasis_host[j];
        comb[j] = 1u << j;
    }
    for (int j = 0; j < tr; ++j) {
        if (!row[j]) { dcs_host::set_error("dcs_accumulate: dependent terminal basis"); return DCS_E_ARG; }
        piv[j] = 31 - __builtin_clz(row[j]);
        for (int o = 0; o < tr; ++o)
            if (o != j && ((row[o] >> piv[j]) & 1)) { row[o] ^= row[j]; comb[o] ^= comb[j]; }
    }
    // now row[j] has a 1 at piv[j] and 0 at every other pivot; s = sum_j i_j basis_j means
    // reduced coordinates: s in image iff s == XOR_{j: s_piv[j]} row[j]; then i = XOR comb[j].
    // i_bit = parity(s & linv[bit]) with linv[bit] = {piv[j] : comb[j] has bit}
    for (int bit = 0; bit < tr; ++bit) {
        uint32_t m = 0;
        for (int j = 0; j < tr; ++j)
            if ((comb[j] >> bit) & 1) m |= 1u << piv[j];
        tm.linv[bit] = m;
    }
    // parity checks: for every non-pivot bit q, s_q == XOR_j s_piv[j] * row[j]_q
    uint32_t pivmask = 0;
    for (int j = 0; j < tr; ++j) pivmask |= 1u << piv[j];
    int nc = 0;
    for (int q = 0; q < k; ++q) {
        if ((pivmask >> q) & 1) continue;
        uint32_t m = 1u << q;
        for (int j = 0; j < tr; ++j)
            if ((row[j] >> q) & 1) m |= 1u << piv[j];
        tm.check[nc++] = m;
    }
    tm.nchecks = nc;
    return DCS_OK;
}

extern "C" int dcs_accumulate_batched(int dtype, const void* table, uint64_t table_stride, int tr,
                                      const uint32_t* terminal_runs, int nruns, const uint64_t* tbasis,
                                      const uint64_t* xors, const double* coefs, const int32_t* item_begin,
                                      int nblocks, double log_shift, dcs_scale* scale, const uint64_t* maxbits_final,
                                      uint64_t mstride, double* total, int k, int nitems, void* stream) {
    if (!table || !xors || !coefs || !item_begin || !scale || !maxbits_final || !total || nblocks < 1 ||
        nblocks > 65535 || nitems < 0) {
        dcs_host::set_error("dcs_accumulate: invalid arguments");
        return DCS_E_ARG;
    }
    TermMap tm;
    int rc = build_termmap(tm, tr, terminal_runs, nruns, tbasis, k);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    if (nitems > 0) {
        k_final_flags<<<(nitems + 127) / 128, 128, 0, st>>>((const unsigned long long*)maxbits_final, mstride,
                                                            dtype == DCS_C128, scale, nitems);
        DCS_CHECK_LAUNCH("k_final_flags launch");
    }
    const uint64_t n = 1ull << k;
    uint64_t bx = (n + 255) / 256;
    const uint64_t cap = (uint64_t)dcs_host::sm_count() * 8;
    if (bx > cap) bx = cap;
    dim3 grid((unsigned)bx, (unsigned)nblocks);
    if (dtype == DCS_C64)
        k_accumulate<float2><<<grid, 256, 0, st>>>((const float2*)table, table_stride, tm, xors, coefs, item_begin,
                                                   log_shift, scale, (const unsigned long long*)maxbits_final, mstride,
                                                   (double2*)total);
    else if (dtype == DCS_C128)
        k_accumulate<double2><<<grid, 256, 0, st>>>((const double2*)table, table_stride, tm, xors, coefs, item_begin,
                                                    log_shift, scale, (const unsigned long long*)maxbits_final,
                                                    mstride, (double2*)total);
    else if (dtype == DCS_H16)
        k_accumulate<ushort2><<<grid, 256, 0, st>>>((const ushort2*)table, table_stride, tm, xors, coefs, item_begin,
                                                    log_shift, scale, (const unsigned long long*)maxbits_final,
                                                    mstride, (double2*)total);
    else {
        dcs_host::set_error("dcs_accumulate: unknown dtype %d", dtype);
        return DCS_E_ARG;
    }
    DCS_CHECK_LAUNCH("k_accumulate launch");
    return DCS_OK;
}

extern "C" int dcs_block_tail(double* total, int k, const uint32_t* adj_hi, const double* u_open, int nblocks,
                              void* stream) {
    if (!total || k < 0 || k > 30 || nblocks < 1 || (k > 0 && (!adj_hi || !u_open))) {
        dcs_host::set_error("dcs_block_tail: invalid arguments");
        return DCS_E_ARG;
    }
    if (k == 0) return DCS_OK;
    TailParams tp;
    memset(&tp, 0, sizeof(tp));
    tp.k = k;
    for (int q = 0; q < k; ++q) {
        tp.adj_hi[q] = adj_hi[q];
        for (int e = 0; e < 8; ++e) tp.u[q][e] = u_open[8 * q + e];
    }
    cudaStream_t st = (cudaStream_t)stream;
    double2* v = (double2*)total;
    int rc;
    if (k <= kTailLog) {
        // one tile per block: all bits at once
        if ((rc = tail_pass(v, tp, k, k, k, 0, k, 0, nblocks, st))) return rc;
        if ((rc = tail_pass(v, tp, k, k, k, 0, k, 1, nblocks, st))) return rc;
        return DCS_OK;
    }
    // low tile: bits [0, L); high tile: 3 contiguous low bits + bits [L, k)
    const int L = kTailLog - 3 > k - 3 ? k - 3 : kTailLog;
    const int hb = k - L;  // high bits
    if (hb + 3 > kTailLog) {
        dcs_host::set_error("dcs_block_tail: k=%d too large for the two-pass tail", k);
        return DCS_E_ARG;
    }
    if ((rc = tail_pass(v, tp, L, L, L, 0, L, 0, nblocks, st))) return rc;
    if ((rc = tail_pass(v, tp, 3, L, k, 3, 3 + hb, 0, nblocks, st))) return rc;
    if ((rc = tail_pass(v, tp, L, L, L, 0, L, 1, nblocks, st))) return rc;
    // second U pass must not re-apply the phase: mode 2 == U without phase
    if ((rc = tail_pass(v, tp, 3, L, k, 3, 3 + hb, 2, nblocks, st))) return rc;
    return DCS_OK;
}
