// fno_host.h -- host-side declarations shared by the FNO translation units.
#pragma once
#include <cuda_runtime.h>

#include <string>

#include "fno_gemm.cuh"

namespace fno {

void set_error(const std::string& m);
// 0 ok, 1 bad argument, 3 CUDA error (message via set_error)
int gemm(const GemmDesc& d, cudaStream_t st);

}  // namespace fno
