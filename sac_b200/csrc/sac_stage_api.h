// sac_stage_api.h -- host-visible interface of the stage kernels (sac_stage.cuh).
// The kernels are instantiated per storage type in their own translation units:
// stage_f64.cu (no contraction, IEEE division) and stage_f32.cu.
#pragma once
#include <cuda_runtime.h>

#include <type_traits>

#include "sac_kernels.cuh"

namespace sacgpu {

template <int NDIM>
struct Pairs {
  // setnu pairs: rho(k), e173(k), v_l(k) (all l), b_l(k) (l != k)
  static constexpr int NR = 2 * NDIM + NDIM * NDIM + NDIM * (NDIM - 1);
  static __host__ __device__ constexpr int rho(int k) { return k; }
  static __host__ __device__ constexpr int e(int k) { return NDIM + k; }
  static __host__ __device__ constexpr int v(int l, int k) { return 2 * NDIM + l * NDIM + k; }
  static __host__ __device__ constexpr int b(int l, int k) {
    return 2 * NDIM + NDIM * NDIM + l * (NDIM - 1) + (k < l ? k : k - 1);
  }
};

inline int nr_pairs(int ndim) { return 2 * ndim + ndim * ndim + ndim * (ndim - 1); }

// addsource_visc's cross-derivative pairs (l != k): the centred half-sums of the
// momentum terms (v_l along k) and of the field terms (b_l along k), stored per
// cell by k_cross for the single-grid update
template <int NDIM>
struct Cross {
  static constexpr int N = 2 * NDIM * (NDIM - 1);
  static __host__ __device__ constexpr int m(int l, int k) { return l * (NDIM - 1) + (k < l ? k : k - 1); }
  static __host__ __device__ constexpr int b(int l, int k) { return NDIM * (NDIM - 1) + m(l, k); }
};

inline int n_cross(int ndim) { return 2 * ndim * (ndim - 1); }

struct Stage2Args {
  Geom g;
  long sP, sB, sI, sX;  // field strides of the four families
  const void* wct;   // S[np][N]   stage input, advanced variables
  const double* bgv; // double[nb][N] eb, rhob, bg1..
  const void* base;  // S[np][N]   may alias out
  void* out;         // S[np][N]
  void* aux1;        // S[np][N]   RK4 accumulator
  const void* aux2;  // S[np][N]   w2 for the stage-3 epilogue
  const void* D;     // S[ndir+3][N] rho+rhob, v.., e173, p'_tot
  const void* F;     // S[ndim*np][N] fluxes, F[d*np+iw]
  const void* R;     // S[NR][N]   setnu face quotients
  const void* X;     // S[n_cross][N] cross-derivative half-sums (single grid), or nullptr
  const double* dx;  // double[ndim][N]
  const double* drv; // driver profiles [2][N] or nullptr
  const unsigned long long* ctot;
  unsigned long long* maxnu;
  double qdt, qdt2, gamma, tdep;
  double grav[3];
  double drvA;
  int dmin, dmax;
  unsigned iwmask;
  int zero1[3][2];
  int grav_on, visc_on, driver, epi;
  int divb_on;            // Powell div B source (divbfix, ndim > 1)
  int res_on;             // resistive source with the constant eta below
  int res_compact;        // ... in the compact form addsource_res1 (compactres)
  double eta;
  // per-field base pointers (filled by fill_field_ptrs), so that a load is one
  // pointer from parameter space plus the cell offset
  const void* fF[3][8];   // F[d][iw]
  const void* fQ[21];     // setnu face quotients per pair
  const void* fW[8];      // wct per advanced variable
  const void* fD[6];      // rho+rhob, v.., e173, p'_tot
  const double* fBG[5];   // eb, rhob, bg..
  const double* fDX[3];   // dx per dimension
  const void* fX[12];     // cross-derivative half-sums per pair
};

// Fill the per-field pointers of a from its block pointers and family strides
// (np, ndir, ndim from a.g; a.sP..a.sX default to g.ncell when zero).
inline void fill_field_ptrs(Stage2Args& a, size_t es) {
  const Geom& g = a.g;
  if (!a.sP) a.sP = g.ncell;
  if (!a.sB) a.sB = g.ncell;
  if (!a.sI) a.sI = g.ncell;
  if (!a.sX) a.sX = g.ncell;
  auto off = [&](const void* base, long k, long s) {
    return base ? (const void*)((const char*)base + (size_t)k * s * es) : nullptr;
  };
  for (int d = 0; d < 3; ++d)
    for (int iw = 0; iw < 8; ++iw)
      a.fF[d][iw] = (d < g.ndim && iw < g.np) ? off(a.F, (long)d * g.np + iw, a.sI) : nullptr;
  for (int i = 0; i < 21; ++i) a.fQ[i] = (i < nr_pairs(g.ndim)) ? off(a.R, i, a.sI) : nullptr;
  for (int iw = 0; iw < 8; ++iw) a.fW[iw] = (iw < g.np) ? off(a.wct, iw, a.sP) : nullptr;
  for (int i = 0; i < 6; ++i) a.fD[i] = (i < g.ndir + 3) ? off(a.D, i, a.sI) : nullptr;
  for (int i = 0; i < 5; ++i) a.fBG[i] = (i < g.nw - g.np) ? a.bgv + (size_t)i * a.sB : nullptr;
  for (int d = 0; d < 3; ++d) a.fDX[d] = (d < g.ndim) ? a.dx + (size_t)d * a.sX : nullptr;
  for (int i = 0; i < 12; ++i) a.fX[i] = (i < n_cross(g.ndim)) ? off(a.X, i, a.sI) : nullptr;
}

struct BatchStageArgs {
  Stage2Args a;            // pointers/strides of the whole batch (geometry per instance)
  const InstInfo* inst;
  InstDyn* dyn;
  const Tile* tiles;
  int ntiles;
  int stage;               // RK4 stage 0..3: qdt = dt/2, dt/2, dt, dt/6
};

template <typename S>
void launch_face(const Stage2Args& a, int do_ctot, cudaStream_t st);
template <typename S>
void launch_nu(const Stage2Args& a, cudaStream_t st);
template <typename S>
void launch_update(const Stage2Args& a, cudaStream_t st);
template <typename S>
void launch_cross(const Stage2Args& a, cudaStream_t st);

template <typename S>
void launch_batch_face(const BatchStageArgs& b, double gamma, cudaStream_t st);
template <typename S>
void launch_batch_nu(const BatchStageArgs& b, cudaStream_t st);
template <typename S>
void launch_batch_update(const BatchStageArgs& b, dim3 blk, cudaStream_t st);
template <typename S>
void launch_batch_courant(const BatchStageArgs& b, double gamma, cudaStream_t st);

// the fused 2D stage (sac_stage2d.cuh): c_tot of the stage input, then one kernel
// per tile for face, setnu and update; shape indexes the tile shapes
template <typename S>
void launch_batch_ctot(const BatchStageArgs& b, cudaStream_t st);
template <typename S>
cudaError_t launch_batch_stage2d(const BatchStageArgs& b, int shape, cudaStream_t st);
constexpr int kStage2dShapeCount = 2;
inline int stage2d_shape_tx(int i) { return i == 0 ? 32 : 16; }
inline int stage2d_shape_ty(int i) { return i == 0 ? 8 : 8; }
extern template void launch_batch_ctot<double>(const BatchStageArgs&, cudaStream_t);
extern template void launch_batch_ctot<float>(const BatchStageArgs&, cudaStream_t);
extern template cudaError_t launch_batch_stage2d<double>(const BatchStageArgs&, int, cudaStream_t);
extern template cudaError_t launch_batch_stage2d<float>(const BatchStageArgs&, int, cudaStream_t);

// two batches stepped together (stage_joint.cu): b[0] holds FP64 instances, b[1]
// FP32 ones; each kernel walks b[0]'s tiles, then b[1]'s
struct JointStageArgs {
  BatchStageArgs b[2];
};
struct JointBoundArgs {
  BcArgs proto[2];
  const InstInfo* inst[2];
  const GhostChunk* chunks[2];
  int n[2];
  const InstDyn* dyn[2];
};
void launch_joint_courant(const JointStageArgs& j, double gamma, cudaStream_t st);
void launch_joint_ctot(const JointStageArgs& j, cudaStream_t st);
cudaError_t launch_joint_stage2d(const JointStageArgs& j, int shape, cudaStream_t st);
void launch_joint_bound(const JointBoundArgs& j, int nvar, cudaStream_t st);

extern template void launch_batch_face<double>(const BatchStageArgs&, double, cudaStream_t);
extern template void launch_batch_face<float>(const BatchStageArgs&, double, cudaStream_t);
extern template void launch_batch_nu<double>(const BatchStageArgs&, cudaStream_t);
extern template void launch_batch_nu<float>(const BatchStageArgs&, cudaStream_t);
extern template void launch_batch_update<double>(const BatchStageArgs&, dim3, cudaStream_t);
extern template void launch_batch_update<float>(const BatchStageArgs&, dim3, cudaStream_t);
extern template void launch_batch_courant<double>(const BatchStageArgs&, double, cudaStream_t);
extern template void launch_batch_courant<float>(const BatchStageArgs&, double, cudaStream_t);
extern template void launch_face<double>(const Stage2Args&, int, cudaStream_t);
extern template void launch_face<float>(const Stage2Args&, int, cudaStream_t);
extern template void launch_nu<double>(const Stage2Args&, cudaStream_t);
extern template void launch_nu<float>(const Stage2Args&, cudaStream_t);
extern template void launch_update<double>(const Stage2Args&, cudaStream_t);
extern template void launch_update<float>(const Stage2Args&, cudaStream_t);
extern template void launch_cross<double>(const Stage2Args&, cudaStream_t);
extern template void launch_cross<float>(const Stage2Args&, cudaStream_t);

}  // namespace sacgpu
