// Register runs: scalar kernels of local dimension 4.
#include "runs.cuh"

namespace dcs_runs {
int launch_scalar4(int mb, const RunArgs& A, size_t smem, int sms, uint64_t ntiles, cudaStream_t st, void* table,
                   const dcs_param* params, uint64_t* maxbits, dcs_scale* scale) {
    return mb == 2 ? launch<2, 4, false>(A, smem, sms, ntiles, st, table, params, maxbits, scale)
                   : launch<3, 4, false>(A, smem, sms, ntiles, st, table, params, maxbits, scale);
}
}  // namespace dcs_runs
