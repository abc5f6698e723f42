// stage_f64.cu -- the stage kernels instantiated for double storage; built with
// --fmad=false and IEEE division so that every expression rounds as the reference.
#include "sac_stage.cuh"
#include "sac_stage2d.cuh"

namespace sacgpu {
template void launch_face<double>(const Stage2Args&, int, cudaStream_t);
template void launch_nu<double>(const Stage2Args&, cudaStream_t);
template void launch_update<double>(const Stage2Args&, cudaStream_t);
template void launch_cross<double>(const Stage2Args&, cudaStream_t);
template void launch_batch_face<double>(const BatchStageArgs&, double, cudaStream_t);
template void launch_batch_nu<double>(const BatchStageArgs&, cudaStream_t);
template void launch_batch_update<double>(const BatchStageArgs&, dim3, cudaStream_t);
template void launch_batch_courant<double>(const BatchStageArgs&, double, cudaStream_t);
template void launch_batch_ctot<double>(const BatchStageArgs&, cudaStream_t);
template cudaError_t launch_batch_stage2d<double>(const BatchStageArgs&, int, cudaStream_t);
}  // namespace sacgpu
