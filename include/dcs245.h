/*
 * dcs245.h — C ABI of the B200 conditional-block contraction and free-bit sampler.
 *
 * Plain C: pointers, sizes and POD structs only.  Every entry point returns 0
 * on success or a negative DCS_E_* code; dcs_last_error() gives the message of
 * the last failure on the calling thread.  No C++ exception crosses the ABI.
 * All device pointers are CUDA global-memory pointers of the current device;
 * `stream` is a cudaStream_t (NULL = legacy default stream).  All work is
 * enqueued asynchronously on `stream` unless stated otherwise.
 *
 * Reference interfaces replaced (paths inside the reference project):
 *   dcs_inplace_step      kernel `inplace_step` + its launch,
 *                         source/kernel_opt/inplace_gpu.py:20-63 and :117-119
 *   dcs_slice_steps       the per-step host loop `prefix_inplace`,
 *                         source/kernel_opt/inplace_gpu.py:107-124
 *                         (renormalisation kept on the device, no host sync)
 *   dcs_fused_groups      same loop, several steps per pass over the table
 *   dcs_accumulate        terminal gather + syndrome scatter + coherent slice sum,
 *                         source/kernel_opt/inplace_gpu.py:124 and
 *                         source/sampling/conditional_block_gpu.py:155-158
 *   dcs_block_tail        Walsh-Hadamard, open-edge phase and U_open passes,
 *                         source/sampling/conditional_block_gpu.py:159-171
 *   dcs_draw              FP64 CDF draw `draw_checked`,
 *                         source/sampling/sampling_protocol.py:44-88
 */
#ifndef DCS245_H
#define DCS245_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* the library is built with hidden visibility; everything declared here is exported */
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#define DCS_ABI_VERSION 1

/* error codes */
#define DCS_OK 0
#define DCS_E_ARG -1      /* invalid argument (size, kind, alignment, range) */
#define DCS_E_CUDA -2     /* a CUDA runtime call failed */
#define DCS_E_NONFINITE -3 /* nonfinite table (reference: ArithmeticError) */
#define DCS_E_CDF -4      /* zero / nonfinite block or invalid outcome (reference: ArithmeticError) */

/* storage types of the in-place table */
#define DCS_C64 0  /* float2: complex64 storage, FP32 arithmetic */
#define DCS_C128 1 /* double2: complex128 storage, FP64 arithmetic */
/* two IEEE binary16 components per entry (4 bytes), FP64 arithmetic, each output rounded
 * FP64 -> FP32 -> binary16 to nearest even; max bits are FP64 bits of the rounded |v|^2:
 * the half-storage tier of the reference (source/kernel_opt/inplace_half_gpu.py), an approximate
 * variant; the per-step executors and the terminal gather take it, the fused executors do not */
#define DCS_H16 2

/* orbit kinds (same numbering as the reference kernel's `kind`) */
#define DCS_KIND_GROW 0
#define DCS_KIND_MIX 1
#define DCS_KIND_DIAG 2
#define DCS_KIND_REPLACE 3
#define DCS_KIND_FIXED 4
#define DCS_KIND_FIXED_SHRINK 5
#define DCS_KIND_SHRINK4 6
#define DCS_KIND_SHRINK2 7

#define DCS_MAX_RUNS 28
#define DCS_MAX_SLOTS 40

/* One vertex step of the preserved-coordinate plan (static per plan; HOST memory: the
 * library passes it to the kernel by value, so a captured CUDA graph keeps it).
 * Orbit representatives are enumerated by depositing x in [0, 2^m) into the slots of
 * enum_mask; the deposit is stored as runs: run r copies `len` bits of x starting at bit
 * `src` to bits starting at `dst` (packed src | dst << 8 | len << 16). */
typedef struct dcs_step {
    uint64_t K;        /* kernel vector (slot mask) */
    uint64_t Ka;       /* Pauli shift (slot mask) */
    uint64_t beta;     /* sign mask: parity(c & beta) */
    uint64_t pivot_bit;/* grow: 1 << pivot; else 0 */
    uint64_t in_mask;  /* active_in slots */
    uint64_t out_mask; /* active_out slots */
    int32_t kind;      /* DCS_KIND_* */
    int32_t m;         /* log2 of the number of orbits */
    int32_t nruns;
    int32_t free_;     /* vertex is free (not structurally fixed) */
    uint32_t runs[DCS_MAX_RUNS];
} dcs_step;

/* Per-(slice, step) contraction weights and offset bits (built on the host per block). */
typedef struct dcs_param {
    double f0r, f0i, f1r, f1i; /* f_v = (f0, f1) */
    int32_t ov;                /* offset bit of this position */
    int32_t y;                 /* fixed value (fixed kinds only) */
} dcs_param;

/* Device-resident renormalisation state of one work item (one slice of one prefix).
 * maxbits[s] holds the bit pattern of max|x|^2 written by step s-1 (float bits in the low
 * 32 bits for DCS_C64, double bits for DCS_C128); maxbits[0] must be the pattern of 1.0.
 * Step s scales its writes by 2^-e with e = frexp(sqrt(maxbits[s]))'s exponent and adds
 * e*ln2 to logscale (sequential FP64 sum, as the reference's host loop does). */
typedef struct dcs_scale {
    double logscale;
    int64_t exponent_sum;
    uint32_t flags; /* bit 0: a nonfinite maximum was seen; bit 1: the table became zero */
    uint32_t pad;
    double phase;   /* radians: the argument of the step factors the plan-specialised kernels divide
                       out of the weights (the table is e^{logscale + i phase} times its entries) */
} dcs_scale;

/* One fused pass: steps [first, first+count) applied to every coset tile of `tile_dim`
 * dimensions.  Tile element t has address base ^ tile_addr(t); the tile basis vectors are
 * in basis[0..tile_dim) (low `low_bits` of them are the unit vectors 1,2,4,..), and the
 * coset bases are the deposit of x in [0, 2^coset_m) into coset_runs. */
typedef struct dcs_group {
    int32_t first, count;
    int32_t tile_dim, low_bits;
    int32_t coset_m, ncoset_runs;
    int32_t step_tile_off; /* index into the per-step tile-mask table */
    int32_t variant;       /* kernel variant bits: 1 = 2 CTAs per SM (else 3); 2 = paired tile layout with
                              packed FP32x2 arithmetic; 4 = register runs (dcs_fused_runs); 8 = runs of
                              local dimension 4 (else 3) */
    uint64_t out_mask;     /* active_out after the last step (for the max) */
    uint64_t basis[16];    /* tile basis (slot masks) */
    uint32_t coset_runs[DCS_MAX_RUNS];
} dcs_group;

/* Per-step tile-coordinate data used by the fused kernel (one per step of each group).
 * Orbit representatives of step s are the tile indices with zero bits at ins[0..nins)
 * (ascending): the role slots of the step (the zero pivots of the reference's entry c) and the
 * slots of the group universe that are inactive at the step and lie on tile bits.  Inactive
 * slots that are coset bits are in cskip: a tile whose base has one of them set skips the step.
 * Signs: parity(a & beta) = parity(base & beta) ^ parity(t & tbeta); the partner t ^ tK
 * (t ^ tKa) flips it by sK (sKa). */
typedef struct dcs_tile_step {
    uint64_t cskip;         /* inactive coset slots */
    uint32_t tK, tKa, tpiv; /* tile-coordinate masks of K, Ka, grow pivot */
    uint32_t tbeta;         /* sign functional in tile coordinates */
    uint8_t sK, sKa;        /* parity(tK & tbeta), parity(tKa & tbeta) */
    uint8_t nins;           /* number of inserted zero bits (<= 16) */
    uint8_t rb1, rb2;       /* physical role slots (for checking) */
    /* register runs (group variant bit 4): local bit of the step's orbit vector (shrink4: of K's
     * reduced vector) and of Ka's reduced vector; rmix bit 0: K = local rk1 + rk2, bit 1: Ka =
     * local rk1 + rk2 */
    uint8_t rk1, rk2, rmix;
    uint8_t ins[16];        /* inserted tile bits, ascending */
    uint32_t mhi;           /* tile bits receiving representative-index bits 8 and up (256 threads) */
    /* pairing with the next step (one shared-memory round trip for both): super-orbit
     * {t, t^tau1, t^tau2, t^tau1^tau2} with t zero at pins[]; step 1 acts along tau1, step 2 along
     * tau2; swapB / swapA: the entry with zero role slot in pair (t^tau2, t^tau1^tau2) for step 1 /
     * (t^tau1, t^tau1^tau2) for step 2 is the second one; s1e / s2e: sign parity of the offsets
     * (0, tau1, tau2, tau1^tau2) under step 1's / step 2's tile functional. */
    uint8_t pair;           /* 1: this step and the next run as a pair */
    uint8_t pnins, swapB, swapA;
    uint32_t pmhi;
    uint32_t tau1, tau2;
    uint8_t pins[16];
    uint8_t s1e[4], s2e[4];
    uint16_t ptab;          /* register runs: bit j = parity(local offset j & tbeta) */
    uint8_t run_len;        /* register runs: steps in the run that starts here (0 inside a run) */
    uint8_t rdead;          /* register runs: local bits whose role slot is inactive at this step (entries
                               with such a bit set are skipped) */
} dcs_tile_step;

/* A register run: consecutive steps of a group whose orbit vectors span a space V of dimension
 * r (3 or 4) with one role coordinate per basis vector, and no basis vector touching another's
 * role coordinate.  The tile splits into cosets t0 + V with t0 zero at ins[] (the role
 * coordinates and the coordinates inactive through the run); a thread holds one coset in
 * registers (entry j at tile index t0 ^ off[j]) and applies every step of the run to it. */
typedef struct dcs_tile_run {
    uint8_t nins;           /* zero bits of the coset representatives t0, ascending in ins[] */
    uint8_t count;          /* steps in the run */
    uint8_t r;              /* local dimension */
    uint8_t pad;
    uint8_t ins[16];
    uint32_t mhi;           /* tile bits receiving representative-index bits 8 and up (256 threads) */
    uint16_t off[16];       /* tile offsets of the 2^r local entries */
} dcs_tile_run;

/* One step of the gather form of the plan (the reference's ConditionalBlockGPU, the plan of
 * source/dcs_rankwidth/scan_plan.py:58-105): output c' of 2^r_out sums, over the ncombos kernel
 * combinations q = L c' ^ combo, E[q mod 2^r_in] times f(y) with y = bit r_in of q (free step)
 * or the fixed value.  L c' is read byte by byte from an nbytes x 256 table. */
typedef struct dcs_gather_step {
    uint64_t beta;          /* sign functional on the input coordinates */
    uint64_t table_off;     /* offset (64-bit words) of the step's byte table in `words` */
    uint64_t combo_off;     /* offset (64-bit words) of its kernel combinations in `words` */
    int32_t r_in, r_out;    /* input and output ranks */
    int32_t nbytes;         /* bytes of c' read through the table: ceil(r_out / 8), at least 1 */
    int32_t ncombos;        /* 2^(kernel dimension), at most 64 */
    int32_t free_;          /* 1: y is bit r_in of q; 0: y is the step's fixed value */
    int32_t pad;
} dcs_gather_step;

/* Result of one draw (device-side struct; the host copies it back). */
typedef struct dcs_draw_result {
    int64_t index;             /* A_index */
    int32_t tie;               /* 1: the parallel CDF could not certify the index; the exact
                                  sequential CDF was used */
    int32_t status;            /* 0 ok, else DCS_E_CDF */
    double total_cdf;          /* last value of the FP64 CDF before normalisation */
    double total_exact;        /* compensated total (math.fsum equivalent) */
    double selected_weight;    /* weights[index] */
    double cdf_lower, cdf_upper;           /* normalised CDF at index-1 and index */
    double cdf_lower_exact, cdf_upper_exact;/* compensated prefix / total */
    double uniform;
    double tv53;               /* 53-bit grid TV against the normalised weights */
    double weight_l2;          /* sum of the squared normalised weights (sum p_i^2) */
} dcs_draw_result;

int dcs_abi_version(void);
const char *dcs_last_error(void);
/* Number of SMs of the current device (for grid sizing); negative on error. */
int dcs_sm_count(void);
/* sizeof of the ABI structs, so that bindings can check their layouts:
 * 0 dcs_step, 1 dcs_param, 2 dcs_scale, 3 dcs_group, 4 dcs_tile_step, 5 dcs_draw_result,
 * 6 dcs_tile_run, 7 dcs_gather_step. */
size_t dcs_struct_size(int which);

/* Host planner (no device work): the GF(2) cut rank of every proper prefix of a vertex order on
 * the induced subgraph, ranks[i-1] = rank A[order[0..i-1], order[i..m-1]] for i = 1..m-1.
 * adj: n x n symmetric 0/1 bytes, row-major; order: m distinct vertices.  Replaces
 * prefix_ranks_matrix (source/dcs_rankwidth/parity_slicing.py:35-54), the cost of every trial in
 * choose_parity_slices (:62-105). */
int dcs_prefix_cut_ranks(const uint8_t *adj, int n, const int32_t *order, int m, int32_t *ranks);

/* Reference-compatible single step (kernel `inplace_step`, inplace_gpu.py:20-63): the same
 * arguments in the same order, with the address table T (nb x 256 uint64, device) and a
 * host-chosen scale.  `dmax` receives atomicMax of the float/double bits of |x|^2 and must be
 * zeroed by the caller (the reference does d_max.fill(0)).  grid <= 0 picks SMs*32. */
int dcs_inplace_step(int dtype, void *E, uint64_t norbits, const uint64_t *T, int nb, int identity_map,
                     int kind, uint64_t K, uint64_t Ka, int pivot, uint64_t beta, int ov,
                     double f0r, double f0i, double f1r, double f1i, int fixed_y, double scale,
                     void *dmax, int grid, void *stream);

/* Steps [first, first+count) of one work item with device-resident renormalisation.
 * table: 2^maxslots entries (device); steps: the plan (host array of nsteps); params: one
 * dcs_param per step (device); maxbits: nsteps+1 words (device, maxbits[first] valid on
 * entry); scale: device.  No host synchronisation. */
int dcs_slice_steps(int dtype, void *table, const dcs_step *steps, const dcs_param *params, int nsteps,
                    int first, int count, uint64_t *maxbits, dcs_scale *scale, void *stream);

/* Batched variant: `nitems` independent work items that share the plan (one launch per step
 * covers every item).  Item i uses table + i*table_stride entries, params + i*param_stride,
 * maxbits + i*(nsteps+1) and scale + i. */
int dcs_slice_steps_batched(int dtype, void *table, uint64_t table_stride, const dcs_step *steps,
                            const dcs_param *params, uint64_t param_stride, int nsteps, int first, int count,
                            uint64_t *maxbits, dcs_scale *scale, int nitems, void *stream);

/* Gather-form steps [s0, s0 + count) on two tables of nitems work items each (item i at
 * i * stride entries): step s0 reads table_a and writes table_b, the next reads table_b, and so on,
 * so the result is in table_b for odd count.  Replaces the host loop of the reference's
 * ConditionalBlockGPU._prefix (sampling/conditional_block_gpu.py:92-126) and its kernel
 * scan_step_scaled (dcs_rankwidth/gpu_kernel.py:58-103): FP64 sums, writes scaled by 2^-e with e
 * from maxbits[s] (the previous step's max |x|^2, IEEE bits of the storage precision; maxbits[s0]
 * = bits of 1.0 before the first step), max |x|^2 into maxbits[s + 1], e ln 2 into scale->logscale,
 * no host synchronisation.  dtype DCS_C64 or DCS_C128; steps: host array; words, params,
 * maxbits (maxbits_stride words per item), scale: device. */
int dcs_gather_steps(int dtype, void *table_a, void *table_b, uint64_t stride, const dcs_gather_step *steps,
                     const uint64_t *words, const dcs_param *params, uint64_t param_stride, int s0, int count,
                     unsigned long long *maxbits, uint64_t maxbits_stride, dcs_scale *scale, int nitems,
                     void *stream);

/* Fused passes over coset tiles (complex64 tables): groups [g0, g0+ng) of a fused plan.
 * steps, groups and tile_steps are host arrays; params, maxbits (ngroups+1 words) and scale
 * are device memory.  Renormalisation is per pass. */
int dcs_fused_groups(void *table, const dcs_step *steps, int nsteps, const dcs_group *groups, int ngroups,
                     const dcs_tile_step *tile_steps, const dcs_param *params, int g0, int ng,
                     uint64_t *maxbits, dcs_scale *scale, void *stream);

/* The same passes, with register runs for the groups whose variant has bit 4: tile_runs[i] is
 * the run that starts at step i (tile_steps[i].run_len > 0); other groups run as in
 * dcs_fused_groups. */
int dcs_fused_runs(void *table, const dcs_step *steps, int nsteps, const dcs_group *groups, int ngroups,
                   const dcs_tile_step *tile_steps, const dcs_tile_run *tile_runs, const dcs_param *params,
                   int g0, int ng, uint64_t *maxbits, dcs_scale *scale, void *stream);

/* Plan-specialised group kernels (no reference counterpart: the reference's kernels are fixed
 * sources compiled once).  A fused plan with register runs is turned into one CUDA kernel per
 * group with every plan quantity a constant (generator: jit.py, device header: runs_jit.cuh).
 * dcs_jit_compile compiles CUDA source for sm_100a with NVRTC into a cubin image (release with
 * dcs_jit_free); `log` receives the compiler log.  dcs_jit_load loads an image through the
 * runtime library API.  dcs_jit_kernel looks up a kernel, allows it `smem` bytes of dynamic
 * shared memory and returns its resident blocks per SM at `threads` per block.  dcs_jit_launch
 * runs it with `threads` per block (the count the source was generated for) on (table, params,
 * maxbits, scale), as dcs_fused_runs runs one group. */
int dcs_jit_compile(const char *source, const char *name, const char *header_source, const char *header_name,
                    int lineinfo, void **image, size_t *image_size, char *log, size_t log_capacity);
void dcs_jit_free(void *image);
int dcs_jit_load(const void *image, void **library);
int dcs_jit_unload(void *library);
int dcs_jit_kernel(void *library, const char *name, size_t smem, int threads, void **kernel, int *blocks_per_sm);
int dcs_jit_launch(void *kernel, unsigned grid, int threads, size_t smem, void *table, const dcs_param *params,
                   uint64_t *maxbits, dcs_scale *scale, void *stream);

/* Terminal gather + syndrome scatter + coherent slice accumulation into complex128 blocks.
 * For output block b, items item_begin[b] .. item_begin[b+1]-1 (slices, in slice order) add
 *   total_b[synd(i) ^ xors[it]] += env_it(i) * (coefs[2it] + i coefs[2it+1]) * exp(logscale_it - log_shift)
 *                                  * exp(i phase_it)
 * with env_it(i) = table[it*table_stride + deposit(i, terminal_runs)], synd(i) = XOR of
 * tbasis[j] (host array, tr entries of k bits) over the bits j of i, i in [0, 2^tr).
 * Items whose scale flags report a zero or nonfinite table, or whose final maximum
 * (maxbits_final[it*mstride]) is zero, add nothing.  xors, coefs, item_begin, scale,
 * maxbits_final and total are device memory; total holds nblocks * 2^k complex128. */
int dcs_accumulate_batched(int dtype, const void *table, uint64_t table_stride, int tr,
                           const uint32_t *terminal_runs, int nruns, const uint64_t *tbasis,
                           const uint64_t *xors, const double *coefs, const int32_t *item_begin, int nblocks,
                           double log_shift, dcs_scale *scale, const uint64_t *maxbits_final, uint64_t mstride,
                           double *total, int k, int nitems, void *stream);

/* Block tail for nblocks consecutive blocks of 2^k complex128: Walsh-Hadamard over k bits,
 * multiply by (-1)^(sum over open edges of y_a y_b) (adj_hi[a] = mask of b > a adjacent to a),
 * then apply u_open[q] (2x2 complex, row-major re/im interleaved: 8 doubles per bit) on bit q.
 * adj_hi and u_open are host arrays. */
int dcs_block_tail(double *total, int k, const uint32_t *adj_hi, const double *u_open, int nblocks, void *stream);

/* FP64 draw from `nblocks` blocks of 2^k complex128 amplitudes with one uniform each
 * (uniforms: device).  scratch: dcs_draw_scratch_bytes(k, nblocks) bytes of device memory.
 * results: nblocks dcs_draw_result (device); status DCS_E_ARG = nonfinite block or uniform
 * outside [0,1) (reference: ValueError), DCS_E_CDF = zero block / invalid outcome
 * (reference: ArithmeticError). */
size_t dcs_draw_scratch_bytes(int k, int nblocks);
int dcs_draw(const double *blocks, int k, int nblocks, const double *uniforms, void *scratch,
             dcs_draw_result *results, void *stream);
/* dcs_draw with flags.  DCS_DRAW_SEQUENTIAL: run the exact sequential FP64 CDF pass (numpy's
 * cumsum order, otherwise run only for ties) for every block, so that cdf_lower, cdf_upper and
 * total_cdf are numpy's values bit for bit (the reference's record rows derive
 * actual_53bit_conditional_probability from them, production/worker.py:116).  In every mode a
 * selected index whose compensated interval does not contain u gives DCS_E_CDF (reference:
 * sampling_protocol.py:67-72). */
#define DCS_DRAW_SEQUENTIAL 1u
int dcs_draw_ex(const double *blocks, int k, int nblocks, const double *uniforms, unsigned flags, void *scratch,
                dcs_draw_result *results, void *stream);

/* Draw that allocates nothing (no counterpart in the reference; this library's addition).
 * For callers that cannot allocate device memory where they sample: code running while a
 * stream is captured, host runtimes that lend the library only their own buffers, loops where
 * an allocation would synchronise the device.  Same computation and result as dcs_draw for
 * one block, with the scratch in a fixed device array inside the library (about 8.4 MiB per
 * GPU that loads the library, held until the process exits).  Limit: one block of at most
 * 2^DCS_DRAW_STATIC_MAX_K amplitudes per call; larger blocks are rejected with DCS_E_ARG.
 * The first call on each device looks the array up (cudaGetSymbolAddress) with that device
 * current; make that first call before any stream capture.  A new context on the device (after
 * cudaDeviceReset) is noticed and the lookup redone on the next call.  All calls share the array:
 * calls that overlap on the GPU (other streams, other threads) race and must be serialised
 * by the caller.  blocks, uniform (1 double) and result are device memory. */
#define DCS_DRAW_STATIC_MAX_K 20
int dcs_draw_static(const double *blocks, int k, const double *uniform, dcs_draw_result *result, void *stream);

/* Serving: prefixes and uniforms from Philox4x32-10 on the device (no reference counterpart:
 * the reference draws them on the host with NumPy PCG64, sampling_protocol.py:14-41).
 * Sample i uses counter (req[i], idx[i], 0, 0) and key (low, high 32 bits of `key`); output
 * words 0-1 give the closed bits (bit j -> qubit closed[j], nclosed <= 64) as a qubit mask in
 * xbits[i], words 2-3 give uniforms[i] = (w3:w2 >> 11) * 2^-53.  All pointers device. */
int dcs_philox_prefixes(const uint32_t *req, const uint32_t *idx, int count, uint64_t key, const int32_t *closed,
                        int nclosed, uint64_t *xbits, double *uniforms, void *stream);
/* The same Philox4x32-10 bijection on the host (ctr is updated in place), for checking. */
void dcs_philox4x32_10_host(uint32_t ctr[4], uint32_t key0, uint32_t key1);

/* Serving: per-(sample, slice) contraction parameters built on the device from prefix bits —
 * the reference's host bookkeeping (conditional_block_gpu.py:136-157, inplace_gpu.py:111-114).
 * Static per-circuit tables (device): fsel (8 doubles per step: f for x bit 0, f for x bit 1),
 * xq (data qubit selecting the row, -1 for references), fixidx (index among fixed steps or -1),
 * flip (nslices x nsteps bytes), F (nfixed x ceil(nsteps/32) words: later-neighbour masks of
 * fixed steps), tail (nfixed terminal-offset xors), coef (2 doubles per slice), freeflip (per
 * slice).  Output item i = sample * nslices + slice: params[i * nsteps + j], coefs[2i..2i+1],
 * xors[i]. */
int dcs_build_items(const double *fsel, const int32_t *xq, const int32_t *fixidx, const uint8_t *flip,
                    const uint32_t *F, const uint64_t *tail, const double *coef, const uint64_t *freeflip,
                    int nsteps, int nfixed, int nslices, const uint64_t *xbits, int nsamples, dcs_param *params,
                    double *coefs, uint64_t *xors, void *stream);

/* Audit sums of two complex128 vectors (compensated FP64): out[0] = <ref,ref>,
 * out[1] = <ap,ap>, out[2] + i out[3] = <ref,ap> = sum conj(ref) ap.  scratch: 16 KiB of
 * device memory; out: 4 doubles of device memory.  Reference quantity:
 * source/review/full_vector_audit_certificate.py:30-36. */
int dcs_overlap(const double *ref, const double *ap, uint64_t len, double *out, void *scratch, void *stream);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif
#endif /* DCS245_H */
