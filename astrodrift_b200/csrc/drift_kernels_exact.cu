// Integration kernels without multiply-add contraction (compiled -fmad=false):
// the stage arithmetic rounds exactly as the reference's Rust code does.
#define DRIFT_EXACT_ARITH 1
#define DRIFT_PRECISION_NS exact
#include "drift_kernels.cuh"

namespace drift {
cudaError_t launch_exact(const KernelArgs &a, int method, int grid, int block,
                         cudaStream_t stream)
{
    return exact::launch_impl(a, method, grid, block, stream);
}
cudaError_t force_exact(const drift_potential &p, int64_t n, const double *xyz, double *acc,
                        const BulgeTable &bt, int grid, cudaStream_t stream)
{
    return exact::force_impl(p, n, xyz, acc, bt, grid, stream);
}
int max_threads_exact() { return exact::max_threads_impl(); }
cudaError_t build_order(const KernelArgs &a, int method, uint8_t *keys, unsigned *counts,
                        uint32_t *order, int sm_count, cudaStream_t stream)
{
    return exact::build_order_impl(a, method, keys, counts, order, sm_count, stream);
}
cudaError_t occupancy_exact(int method, int kind, int block, bool tape, int *blocks_per_sm)
{
    return exact::occupancy_impl(method, kind, block, tape, blocks_per_sm);
}
}  // namespace drift
