// stage_joint.cu -- the kernels of a batched RK4 step over two batches at once,
// one of FP64 instances and one of FP32-perturbation instances (sac_batch_join).
//
// Each kernel walks one tile list made of the FP64 batch's tiles followed by the
// FP32 batch's, and runs the per-tile body of its storage type: a CTA may take an
// FP64 tile and then an FP32 one, so both precisions share one persistent launch
// and its tail.  Built with the FP64 stage's flags (no contraction, IEEE division
// and square root), so the FP64 instances round exactly as in a batch of their
// own; the FP32 instances compute with the same rules, which is more exact than
// the FP32 stage unit's contraction.
#include "sac_stage.cuh"
#include "sac_stage2d.cuh"

namespace sacgpu {

namespace {

template <int NDIM, int NDIR>
__global__ void __launch_bounds__(256) kj_courant(const __grid_constant__ JointStageArgs j, double gamma) {
  __shared__ double sh[32];
  const int n0 = j.b[0].ntiles, n = n0 + j.b[1].ntiles;
  for (int t = blockIdx.x; t < n; t += gridDim.x) {
    if (t < n0)
      courant_tile<NDIM, NDIR, double>(j.b[0], t, gamma, sh);
    else
      courant_tile<NDIM, NDIR, float>(j.b[1], t - n0, gamma, sh);
  }
}

template <int NDIM, int NDIR>
__global__ void __launch_bounds__(256) kj_ctot(const __grid_constant__ JointStageArgs j, double gamma) {
  __shared__ double sh[32];
  const int n0 = j.b[0].ntiles, n = n0 + j.b[1].ntiles;
  for (int t = blockIdx.x; t < n; t += gridDim.x) {
    if (t < n0)
      ctot_tile<NDIM, NDIR, double>(j.b[0], t, gamma, sh);
    else
      ctot_tile<NDIM, NDIR, float>(j.b[1], t - n0, gamma, sh);
  }
}

// the tile memory is sized for the FP64 box; an FP32 tile uses its first half
template <int NDIR, int TX, int TY>
__global__ void __launch_bounds__(TX * TY) kj_stage2d(const __grid_constant__ JointStageArgs j) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ double shred[32];
  const int n0 = j.b[0].ntiles, n = n0 + j.b[1].ntiles;
  for (int t = blockIdx.x; t < n; t += gridDim.x) {
    if (t < n0)
      stage2d_tile<NDIR, double, TX, TY>(j.b[0], t, smraw, shred);
    else
      stage2d_tile<NDIR, float, TX, TY>(j.b[1], t - n0, smraw, shred);
  }
}

__global__ void __launch_bounds__(256) kj_bound(const __grid_constant__ JointBoundArgs j, int nvar) {
  __shared__ BcArgs a;
  const int n0 = j.n[0], n = n0 + j.n[1];
  for (int t = blockIdx.x; t < n; t += gridDim.x) {
    if (t < n0)
      bound_chunk<double>(j.proto[0], j.inst[0], j.chunks[0], t, nvar, j.dyn[0], a);
    else
      bound_chunk<float>(j.proto[1], j.inst[1], j.chunks[1], t - n0, nvar, j.dyn[1], a);
  }
}

JointStageArgs with_fields(const JointStageArgs& j0) {
  JointStageArgs j = j0;
  fill_field_ptrs(j.b[0].a, sizeof(double));
  fill_field_ptrs(j.b[1].a, sizeof(float));
  return j;
}

}  // namespace

void launch_joint_courant(const JointStageArgs& j0, double gamma, cudaStream_t st) {
  const JointStageArgs j = with_fields(j0);
  const int n = j.b[0].ntiles + j.b[1].ntiles;
  if (!n) return;
  dispatch_nd(j.b[0].a.g, [&](auto ND, auto NR) {
    kj_courant<decltype(ND)::value, decltype(NR)::value><<<persistent_grid(n, 8), dim3(32, 8, 1), 0, st>>>(j, gamma);
  });
}

void launch_joint_ctot(const JointStageArgs& j0, cudaStream_t st) {
  const JointStageArgs j = with_fields(j0);
  const int n = j.b[0].ntiles + j.b[1].ntiles;
  if (!n) return;
  dispatch_nd(j.b[0].a.g, [&](auto ND, auto NR) {
    kj_ctot<decltype(ND)::value, decltype(NR)::value><<<persistent_grid(n, 8), dim3(32, 8, 1), 0, st>>>(
        j, j.b[0].a.gamma);
  });
}

cudaError_t launch_joint_stage2d(const JointStageArgs& j0, int shape, cudaStream_t st) {
  const JointStageArgs j = with_fields(j0);
  const int n = j.b[0].ntiles + j.b[1].ntiles;
  if (!n) return cudaSuccess;
  auto go = [&](auto NRC, auto SH) -> cudaError_t {
    constexpr int NDIR = decltype(NRC)::value, I = decltype(SH)::value;
    constexpr int TX = stage2d_tx(I), TY = stage2d_ty(I);
    constexpr int smem = stage2d_smem<NDIR, double, TX, TY>();
    static_assert(stage2d_smem<NDIR, float, TX, TY>() <= smem, "the FP32 box fits in the FP64 one");
    auto* k = kj_stage2d<NDIR, TX, TY>;
    static int per_sm = 0;  // per instantiation: the resident CTAs the tile memory allows
    if (!per_sm) {
      cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
      if (e != cudaSuccess) return e;
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, TX * TY, smem);
      if (e != cudaSuccess) return e;
      if (per_sm < 1) per_sm = 1;
    }
    k<<<persistent_grid(n, per_sm), TX * TY, smem, st>>>(j);
    return cudaGetLastError();
  };
  auto by_shape = [&](auto NRC) -> cudaError_t {
    if (shape == 1) return go(NRC, std::integral_constant<int, 1>{});
    return go(NRC, std::integral_constant<int, 0>{});
  };
  if (j.b[0].a.g.ndim != 2 || j.b[1].a.g.ndim != 2 || j.b[0].a.g.ndir != j.b[1].a.g.ndir) return cudaErrorInvalidValue;
  if (j.b[0].a.g.ndir == 3) return by_shape(std::integral_constant<int, 3>{});
  return by_shape(std::integral_constant<int, 2>{});
}

void launch_joint_bound(const JointBoundArgs& j, int nvar, cudaStream_t st) {
  const int n = j.n[0] + j.n[1];
  if (!n) return;
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const unsigned grid = (unsigned)std::min<long>(n, (long)nsm * 8);
  kj_bound<<<grid, 256, 0, st>>>(j, nvar);
}

}  // namespace sacgpu
