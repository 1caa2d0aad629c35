// Register runs: packed FP32x2 kernels (paired tile layout); local dimension 4 only with the
// register budget of two CTAs per SM (three spill).
#include "runs.cuh"

namespace dcs_runs {
int launch_packed(int mb, int r, const RunArgs& A, size_t smem, int sms, uint64_t ntiles, cudaStream_t st,
                  void* table, const dcs_param* params, uint64_t* maxbits, dcs_scale* scale) {
    if (r == 4) return launch<2, 4, true>(A, smem, sms, ntiles, st, table, params, maxbits, scale);
    return mb == 2 ? launch<2, 3, true>(A, smem, sms, ntiles, st, table, params, maxbits, scale)
                   : launch<3, 3, true>(A, smem, sms, ntiles, st, table, params, maxbits, scale);
}
}  // namespace dcs_runs
