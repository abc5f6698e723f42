// stage_f32.cu -- the stage kernels instantiated for float storage (FP32 path);
// built with contraction and approximate single-precision division.
#include "sac_stage.cuh"

namespace sacgpu {
template void launch_face<float>(const Geom&, const void*, const double*, void*, void*, unsigned long long*, double,
                               int, cudaStream_t);
template void launch_nu<float>(const Geom&, const void*, const void*, void*, const unsigned long long*, cudaStream_t);
template void launch_update<float>(const Stage2Args&, cudaStream_t);
}  // namespace sacgpu
