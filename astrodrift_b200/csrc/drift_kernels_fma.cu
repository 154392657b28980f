// Integration kernels with multiply-add contraction (compiled -fmad=true).
#define DRIFT_EXACT_ARITH 0
#define DRIFT_PRECISION_NS fma_mode
#include "drift_kernels.cuh"

namespace drift {
cudaError_t launch_fma(const KernelArgs &a, int method, int grid, int block,
                       cudaStream_t stream)
{
    return fma_mode::launch_impl(a, method, grid, block, stream);
}
int max_threads_fma() { return fma_mode::max_threads_impl(); }
cudaError_t force_fma(const drift_potential &p, int64_t n, const double *xyz, double *acc,
                      const BulgeTable &bt, int grid, cudaStream_t stream)
{
    return fma_mode::force_impl(p, n, xyz, acc, bt, grid, stream);
}
cudaError_t occupancy_fma(int method, int kind, int block, bool tape, int *blocks_per_sm)
{
    return fma_mode::occupancy_impl(method, kind, block, tape, blocks_per_sm);
}
}  // namespace drift
