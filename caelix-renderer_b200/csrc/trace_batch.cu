// Dispatch over the register-cap variants of the batched persistent trace kernel
// (variants/trace_batch_kernel.cu, compiled once per variant).
#include "trace.cuh"

namespace cx {

int trace_batch_blocks_per_sm_b4();
int trace_batch_blocks_per_sm_b6();
int trace_batch_blocks_per_sm_b8();
cudaError_t trace_batch_launch_b4(const BatchLaunch& launch, uint32_t grid, cudaStream_t stream);
cudaError_t trace_batch_launch_b6(const BatchLaunch& launch, uint32_t grid, cudaStream_t stream);
cudaError_t trace_batch_launch_b8(const BatchLaunch& launch, uint32_t grid, cudaStream_t stream);

bool trace_batch_variant_ok(uint32_t min_blocks)
{
    return min_blocks == 4 || min_blocks == 6 || min_blocks == 8;
}

int trace_batch_blocks_per_sm(uint32_t min_blocks)
{
    switch (min_blocks) {
    case 4: return trace_batch_blocks_per_sm_b4();
    case 6: return trace_batch_blocks_per_sm_b6();
    case 8: return trace_batch_blocks_per_sm_b8();
    default: return 0;
    }
}

cudaError_t trace_batch_launch(const BatchLaunch& launch, uint32_t min_blocks, uint32_t grid, cudaStream_t stream)
{
    if (grid == 0 || launch.item_count == 0) return cudaSuccess;
    if (launch.view_count == 0 || launch.view_count > kMaxBatchViews ||
        (launch.block_width != 8 && launch.block_width != 16 && launch.block_width != 32) || launch.refill_min == 0 ||
        launch.refill_min > 32)
        return cudaErrorInvalidValue;
    switch (min_blocks) {
    case 4: return trace_batch_launch_b4(launch, grid, stream);
    case 6: return trace_batch_launch_b6(launch, grid, stream);
    case 8: return trace_batch_launch_b8(launch, grid, stream);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace cx
