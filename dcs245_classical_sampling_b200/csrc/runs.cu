// Register runs: the C entry point and the scalar kernels of local dimension 3 (the kernels
// and their algebra are in runs.cuh).
#include "runs.cuh"

namespace dcs_runs {
int launch_scalar3(int mb, const RunArgs& A, size_t smem, int sms, uint64_t ntiles, cudaStream_t st, void* table,
                   const dcs_param* params, uint64_t* maxbits, dcs_scale* scale) {
    return mb == 2 ? launch<2, 3, false>(A, smem, sms, ntiles, st, table, params, maxbits, scale)
                   : launch<3, 3, false>(A, smem, sms, ntiles, st, table, params, maxbits, scale);
}
}  // namespace dcs_runs

using namespace dcs_runs;

extern "C" int dcs_fused_runs(void* table, const dcs_step* steps, int nsteps, const dcs_group* groups, int ngroups,
                              const dcs_tile_step* tile_steps, const dcs_tile_run* tile_runs,
                              const dcs_param* params, int g0, int ng, uint64_t* maxbits, dcs_scale* scale,
                              void* stream) {
    if (!table || !steps || !groups || !tile_steps || !tile_runs || !params || !maxbits || !scale || g0 < 0 ||
        ng < 0 || g0 + ng > ngroups) {
        dcs_host::set_error("dcs_fused_runs: invalid arguments");
        return DCS_E_ARG;
    }
    const int sms = dcs_host::sm_count();
    if (sms <= 0) return DCS_E_CUDA;
    cudaStream_t st = (cudaStream_t)stream;
    for (int gi = g0; gi < g0 + ng; ++gi) {
        const dcs_group& g = groups[gi];
        if (!(g.variant & 4)) {  // a group without register runs: the one-step-per-round-trip kernel
            const int rc = dcs_fused_groups(table, steps, nsteps, groups, ngroups, tile_steps, params, gi, 1,
                                            maxbits, scale, stream);
            if (rc != DCS_OK) return rc;
            continue;
        }
        const int R = (g.variant & 8) ? 4 : 3;
        if (g.count < 1 || g.count > kMaxSteps || g.first < 0 || g.first + g.count > nsteps || g.tile_dim < R ||
            g.tile_dim > 14 || g.low_bits < 0 || g.low_bits > g.tile_dim || g.tile_dim - g.low_bits > 16 ||
            g.ncoset_runs < 0 || g.ncoset_runs > DCS_MAX_RUNS || g.coset_m < 0 || g.coset_m > DCS_MAX_SLOTS) {
            dcs_host::set_error("dcs_fused_runs: malformed group %d", gi);
            return DCS_E_ARG;
        }
        RunArgs A;
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
        const uint32_t T = 1u << g.tile_dim;
        int s = 0;
        while (s < g.count) {
            const dcs_tile_step& ts = tile_steps[g.step_tile_off + s];
            const dcs_tile_run& tr = tile_runs[g.step_tile_off + s];
            const int n = ts.run_len;
            bool bad = n < 1 || s + n > g.count || tr.count != n || tr.r != R || tr.nins > 16 ||
                       tr.nins > g.tile_dim || (tr.mhi >> g.tile_dim) != 0;
            for (int i = 0; i < tr.nins && !bad; ++i)
                bad = tr.ins[i] >= g.tile_dim || (i && tr.ins[i] <= tr.ins[i - 1]);
            for (int j = 0; j < (1 << R) && !bad; ++j) bad = tr.off[j] >= T;
            if (bad) {
                dcs_host::set_error("dcs_fused_runs: malformed run at step %d", g.first + s);
                return DCS_E_ARG;
            }
            RunDesc& d = A.ru[A.nruns++];
            d.first = (uint8_t)s;
            d.count = (uint8_t)n;
            d.nins = tr.nins;
            for (int i = 0; i < 16; ++i) d.ins[i] = tr.ins[i];
            d.mhi = tr.mhi;
            for (int j = 0; j < 16; ++j) d.off[j] = tr.off[j];
            for (int i = s; i < s + n; ++i) {
                const dcs_step& ds = steps[g.first + i];
                const dcs_tile_step& t = tile_steps[g.step_tile_off + i];
                RunStep& f = A.st[i];
                f.beta = ds.beta;
                f.cskip = t.cskip;
                f.tbeta = t.tbeta;
                f.ptab = t.ptab;
                f.kind = ds.kind;
                f.pidx = g.first + i;
                f.sK = t.sK;
                f.sKa = t.sKa;
                f.k1 = t.rk1;
                f.k2 = t.rk2;
                f.mix = t.rmix;
                f.dead = t.rdead;
                // local sign functional: bit k = parity(off[2^k] & tbeta) = bit 2^k of ptab, without
                // the bits where the step's representatives are fixed (its own local bits)
                uint32_t bl = 0;
                for (int k = 0; k < R; ++k) bl |= ((uint32_t)(t.ptab >> (1 << k)) & 1u) << k;
                uint32_t own = 0;
                if (ds.kind != DCS_KIND_DIAG && ds.kind != DCS_KIND_FIXED) own |= 1u << f.k1;
                if (ds.kind == DCS_KIND_SHRINK4) own |= 1u << f.k2;
                f.beff = (uint8_t)(bl & ~own);
                const bool two = ds.kind == DCS_KIND_SHRINK4;
                if (i > s && t.run_len != 0) bad = true;
                if (ds.kind < 0 || ds.kind > 7 || f.k1 >= R || (two && (f.k2 >= R || f.k2 == f.k1 || f.mix > 2)) ||
                    (t.tbeta >> g.tile_dim) != 0)
                    bad = true;
            }
            if (bad) {
                dcs_host::set_error("dcs_fused_runs: malformed run step in group %d", gi);
                return DCS_E_ARG;
            }
            s += n;
        }
        const size_t smem = sizeof(float2) * (size_t)T + sizeof(uint64_t) * ((size_t)1 << (g.tile_dim - g.low_bits));
        const uint64_t ntiles = 1ull << g.coset_m;
        const bool two_cta = g.variant & 1;
        // packed (variant bit 1): every run needs tile bit 0 free (the lane bit) and a coset pair
        bool pk = (g.variant & 2) != 0;
        for (int r = 0; r < A.nruns && pk; ++r) pk = A.ru[r].nins < g.tile_dim && (A.ru[r].nins == 0 || A.ru[r].ins[0]);
        const int mb = two_cta ? 2 : 3;
        int rc;
        if (pk) rc = launch_packed(R == 4 ? 2 : mb, R, A, smem, sms, ntiles, st, table, params, maxbits, scale);
        else if (R == 4) rc = launch_scalar4(mb, A, smem, sms, ntiles, st, table, params, maxbits, scale);
        else rc = launch_scalar3(mb, A, smem, sms, ntiles, st, table, params, maxbits, scale);
        if (rc != DCS_OK) return rc;
    }
    return DCS_OK;
}
