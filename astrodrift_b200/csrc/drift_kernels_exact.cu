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
cudaError_t model_force_exact(const drift_force_model &m, const BulgeTable &bt, double t, int64_t n,
                              const double *xyz, double *acc, int grid, cudaStream_t stream)
{
    exact::model_force_kernel<<<grid, 256, 0, stream>>>(m, bt, t, n, xyz, acc);
    return cudaGetLastError();
}
cudaError_t origin_table_exact(const drift_force_model &source_model, const BulgeTable &bt,
                               int64_t n_sources, int64_t nt, double t0, double dt,
                               const double *trajectory, double *origins, cudaStream_t stream)
{
    const int64_t work = (nt - 1) * n_sources;
    const int grid = (int)std::min<int64_t>((work + 255) / 256, 4096);
    exact::origin_table_kernel<<<grid, 256, 0, stream>>>(source_model, bt, n_sources, nt, t0, dt,
                                                         trajectory, origins);
    return cudaGetLastError();
}
int max_threads_exact() { return exact::max_threads_impl(); }
cudaError_t build_order(const KernelArgs &a, int method, uint8_t *keys, unsigned *counts,
                        uint32_t *order, int sm_count, cudaStream_t stream)
{
    return exact::build_order_impl(a, method, keys, counts, order, sm_count, stream);
}
cudaError_t build_order_chunked(const KernelArgs &a, int method, uint8_t *keys, unsigned *counts,
                                unsigned *split, unsigned *chunk_counts, uint32_t *order, int64_t chunk_len,
                                int nchunks, int64_t lanes, int sm_count, cudaStream_t stream)
{
    return exact::build_order_chunked_impl(a, method, keys, counts, split, chunk_counts, order, chunk_len, nchunks,
                                           lanes, sm_count, stream);
}
cudaError_t occupancy_exact(int method, int kind, int block, bool tape, int *blocks_per_sm)
{
    return exact::occupancy_impl(method, kind, block, tape, blocks_per_sm);
}
}  // namespace drift
