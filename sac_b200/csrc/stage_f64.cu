// stage_f64.cu -- the stage kernels instantiated for double storage; built with
// --fmad=false and IEEE division so that every expression rounds as the reference.
#include "sac_stage.cuh"

namespace sacgpu {
template void launch_face<double>(const Geom&, const void*, const double*, void*, void*, unsigned long long*, double,
                               int, cudaStream_t);
template void launch_nu<double>(const Geom&, const void*, const void*, void*, const unsigned long long*, cudaStream_t);
template void launch_update<double>(const Stage2Args&, cudaStream_t);
}  // namespace sacgpu
