// stage_f32.cu -- the stage kernels instantiated for float storage (FP32 path);
// built with contraction and approximate single-precision division.
#include "sac_stage.cuh"
#include "sac_stage2d.cuh"

namespace sacgpu {
template void launch_face<float>(const Stage2Args&, int, cudaStream_t);
template void launch_nu<float>(const Stage2Args&, cudaStream_t);
template void launch_update<float>(const Stage2Args&, cudaStream_t);
template void launch_cross<float>(const Stage2Args&, cudaStream_t);
template void launch_batch_face<float>(const BatchStageArgs&, double, cudaStream_t);
template void launch_batch_nu<float>(const BatchStageArgs&, cudaStream_t);
template void launch_batch_update<float>(const BatchStageArgs&, dim3, cudaStream_t);
template void launch_batch_courant<float>(const BatchStageArgs&, double, cudaStream_t);
template void launch_batch_ctot<float>(const BatchStageArgs&, cudaStream_t);
template cudaError_t launch_batch_stage2d<float>(const BatchStageArgs&, int, cudaStream_t);
}  // namespace sacgpu
