// sac_batch.cu -- many independent 1D/2D grids advanced together (libsacgpu.so).
//
// Thousands of uneven problems share one set of arrays: every instance owns a
// contiguous full grid (ghosts included) in each field block of the advanced
// state, the background and the cell widths; the per-stage intermediates (D, F,
// R) are sized for one group of instances and reused group by group.  Each pass
// of the stage is one persistent launch whose CTAs walk a tile list built once
// on the host; per-instance dt, c_tot and max nu live in a device table, so a
// whole RK4 step (getdt_courant, getdt_visc, four stages with their boundary
// fills) needs no host round trip and is captured in one CUDA graph.  The tile
// shape of the update pass is chosen by timing the candidates on the actual batch.
//
// Each instance follows exactly the single-grid path (sac_gpu.cu): the same cell
// bodies, the same ghost resolve, the same dt rules of src/vac.t:61-70.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "sac_gpu.h"
#include "sac_grid.h"
#include "sac_kernels.cuh"
#include "sac_stage_api.h"

using namespace sacgpu;

namespace {
constexpr double kBig = 1.0e99, kSmallD = 1.0e-99;

struct Group {
  int i0 = 0, i1 = 0;  // instances [i0, i1)
  long cells = 0;      // cells of the intermediates this group needs
  InstInfo* d_inst = nullptr;  // instance table with group-local intermediate offsets
  Tile *d_face = nullptr, *d_nu = nullptr, *d_upd = nullptr;
  int n_face = 0, n_nu = 0, n_upd = 0;
  GhostChunk* d_gh = nullptr;
  int n_gh = 0;
};
}  // namespace

struct sac_batch {
  sac_params par{};
  std::string err;
  int dev = 0, prec = SAC_PREC_FP64;
  size_t es = 8;
  cudaStream_t stream = nullptr;
  int ndim = 0, ndir = 0, nw = 0, np = 0, ninst = 0;
  std::vector<InstInfo> h_inst;  // global offsets, I offsets unused
  long totP = 0, totX = 0;
  void* P[4] = {nullptr, nullptr, nullptr, nullptr};
  double* BG = nullptr;
  double* dx = nullptr;
  double* drv = nullptr;  // driver profiles [2][totX] (users strat and tube)
  double* stg = nullptr;
  InstDyn* d_dyn = nullptr;
  InstInfo* d_inst = nullptr;  // global table (courant pass, boundaries)
  Tile* d_cour = nullptr;
  int n_cour = 0;
  long* d_meshoff = nullptr;  // per instance: first mesh cell in the packed mesh order
  long mesh_total = 0;
  GhostChunk* d_gh_all = nullptr;
  int n_gh_all = 0;
  std::vector<Group> groups;
  long maxI = 0;
  void *D = nullptr, *F = nullptr, *R = nullptr;
  int8_t* d_type = nullptr;
  int* d_fixed = nullptr;
  double* d_fixB = nullptr;
  int pairshift[3][2] = {};
  int zero1[3][2] = {};
  dim3 upd_blk = dim3(32, 8, 1);
  // the stage as one fused kernel per tile (2D, default sources; sac_stage2d.cuh)
  // instead of the face / setnu / update passes, with its tile shape
  bool fused = false;
  int fused_shape = 0;
  Tile* d_fused = nullptr;
  int n_fused = 0;
  double tune_three_ms = 0, tune_fused_ms = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  // sac_batch_join: the lead (FP64) steps its partner (FP32) in the same launches;
  // while joined the partner's work runs on the lead's stream (own_stream kept)
  sac_batch* partner = nullptr;
  sac_batch* lead = nullptr;
  cudaStream_t own_stream = nullptr;
  // the lead's join form: 0 = joint kernels (one launch per kernel over both
  // batches), 1 = the two batches' own kernels on two branches of the graph;
  // sac_batch_join times one stage in each and keeps the faster
  int join_form = 0;
  double join_ms[2] = {0.0, 0.0};
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  bool grid_set = false, bc_set = false, state_set = false, bc_init = false;
  std::vector<double> mindx2, dtgrav;
};

namespace {

sac_status bfail(sac_batch* b, sac_status st, const std::string& m) {
  if (b) b->err = m;
  return st;
}

#define BK(call)                                                                         \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return bfail(b, SAC_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

bool visc_on_b(const sac_batch* b) {
  if (b->par.user == SAC_USR_SLOG) return true;
  if (b->par.user == SAC_USR_NONE) return false;
  return std::fabs(b->par.nu) > kSmallD;
}
bool grav_mod(int u) { return u == SAC_USR_SLOG || u == SAC_USR_GRAVVISC || u == SAC_USR_STRAT || u == SAC_USR_TUBE; }

// the fused stage covers 2D instances with the default sources (gravity,
// hyperdiffusion, the Gaussian drivers); Powell's and the resistive terms take the
// three passes
bool fused_ok(const sac_batch* b) {
  const bool divb = b->par.sourceunsplit && b->par.divbfix && b->ndim > 1;
  const bool res = b->par.sourceunsplit && std::fabs(b->par.eta) > kSmallD;
  return b->ndim == 2 && !divb && !res;
}

template <typename T>
sac_status upload_vec(sac_batch* b, T** dptr, const std::vector<T>& v) {
  if (*dptr) cudaFree(*dptr), *dptr = nullptr;
  if (v.empty()) return SAC_OK;
  BK(cudaMalloc(dptr, sizeof(T) * v.size()));
  BK(cudaMemcpy(*dptr, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
  return SAC_OK;
}

// tiles of shape (tx,ty,tz) covering coordinates lo..hi of every instance in [i0,i1)
std::vector<Tile> make_tiles(const std::vector<InstInfo>& in, int i0, int i1, int mode, dim3 t) {
  std::vector<Tile> out;
  for (int i = i0; i < i1; ++i) {
    const Geom& g = in[i].g;
    int lo[3], hi[3];
    for (int d = 0; d < 3; ++d) {
      if (d >= g.ndim) {
        lo[d] = hi[d] = 0;
      } else if (mode == 0) {  // whole grid
        lo[d] = 0;
        hi[d] = g.n[d] - 1;
      } else if (mode == 1) {  // setnu faces
        lo[d] = g.lo[d] - 1;
        hi[d] = g.hi[d];
      } else {  // mesh
        lo[d] = g.lo[d];
        hi[d] = g.hi[d];
      }
    }
    for (int z = lo[2]; z <= hi[2]; z += (int)t.z)
      for (int y = lo[1]; y <= hi[1]; y += (int)t.y)
        for (int x = lo[0]; x <= hi[0]; x += (int)t.x) out.push_back(Tile{i, {x, y, z}});
  }
  return out;
}

std::vector<GhostChunk> make_ghosts(const std::vector<InstInfo>& in, int i0, int i1) {
  std::vector<GhostChunk> out;
  for (int i = i0; i < i1; ++i) {
    long ns[3];
    ghost_slabs(in[i].g, ns);
    const long tot = ns[0] + ns[1] + ns[2];
    for (long s = 0; s < tot; s += 256) out.push_back(GhostChunk{i, (int)s});
  }
  return out;
}

// the instance tables a per-instance kernel covers: a batch's own, or a joined
// pair's (the lead's instances first)
struct DynPair {
  InstDyn* d[2];
  int n[2];
  __device__ __forceinline__ InstDyn* at(int i) const {
    return i < n[0] ? d[0] + i : (i < n[0] + n[1] ? d[1] + (i - n[0]) : nullptr);
  }
  int total() const { return n[0] + n[1]; }
};

__global__ void kb_zero(DynPair dp, int what) {
  InstDyn* D = dp.at(blockIdx.x * blockDim.x + threadIdx.x);
  if (!D) return;
  if (what == 0) {
    D->ctot[0] = D->ctot[1] = D->ctot[2] = 0ull;
  } else {
    D->courant = 0ull;
  }
}

// the dt block of program vac per instance (src/vac.t:61-70): getdt_courant,
// getdt_res (src/vacphys.mhdres.t:5-45), getdt_visc (src/vacusr.viscosity.t:509-542),
// getdt_grav (fixed at itmin)
__global__ void kb_dt(DynPair dp, int ndim, double courantpar, double dtpar, int visc, int grav, int cantgrow,
                      double eta, double dtdiffpar) {
  InstDyn* Dp = dp.at(blockIdx.x * blockDim.x + threadIdx.x);
  if (!Dp) return;
  InstDyn& D = *Dp;
  double dt;
  if (dtpar > 0.0) {
    dt = dtpar;
  } else {
    dt = kBig;
    const double cm = __longlong_as_double((long long)D.courant);
    if (!(cm == cm) || isinf(cm)) D.bad = 1;
    if (courantpar > 0.0 && cm > kSmallD) dt = fmin(dt, courantpar / cm);
    if (eta > 0.0) {
      // dtdiffpar*minval(dx(ixM,1:ndim))**2/eta; min over dimensions of the min of
      // dx^2 is that square, rounding being monotonic.  dtdiffpar is the parameter
      // until getdt_visc has overwritten it with 0.25 at an earlier step.
      double m2 = kBig;
      for (int d = 0; d < ndim; ++d) m2 = fmin(m2, D.mindx2[d]);
      dt = fmin(dt, (D.visc_dt_seen ? 0.25 : dtdiffpar) * m2 / eta);
    }
    if (grav && visc) {
      const double mv = __longlong_as_double((long long)D.maxnu);
      if (!(mv == mv)) D.bad = 1;
      for (int d = 0; d < ndim; ++d) dt = fmin(dt, 0.25 / ((mv + 0.0) / D.mindx2[d]));
      D.maxnu = 0ull;
      D.visc_dt_seen = 1;
    }
    if (grav) dt = fmin(dt, D.dtgrav);
    if (cantgrow && D.it > 0) dt = fmin(dt, D.dt);  // dtcantgrow, src/vac.t:68
  }
  if (D.tmax > 0.0) dt = D.t >= D.tmax ? 0.0 : fmin(dt, D.tmax - D.t + kSmallD);  // tmaxexact, src/vac.t:82
  D.dt = dt;
}

__global__ void kb_time(DynPair dp) {
  InstDyn* D = dp.at(blockIdx.x * blockDim.x + threadIdx.x);
  if (!D) return;
  if (D->dt == 0.0) return;  // finished at tmax
  D->t += D->dt;
  D->it += 1;
}

template <typename D>
__device__ __forceinline__ D to_t(double v) { return (D)v; }
template <>
__device__ __forceinline__ __nv_bfloat16 to_t<__nv_bfloat16>(double v) { return __float2bfloat16((float)v); }
__device__ __forceinline__ double to_d(double v) { return v; }
__device__ __forceinline__ double to_d(float v) { return (double)v; }
__device__ __forceinline__ double to_d(__nv_bfloat16 v) { return (double)__bfloat162float(v); }

// packed mesh order: instance i owns np*mesh_i consecutive values, variable-major,
// x1 fastest, ghosts excluded.  dir 0: state -> packed (gather), 1: packed -> state.
template <typename S, typename D>
__global__ void __launch_bounds__(256) kb_pack(const InstInfo* __restrict__ inst, const Tile* __restrict__ tiles,
                                               int ntiles, const long* __restrict__ meshoff, S* P0, long sP, D* pk,
                                               int np, int dir) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Tile tl = tiles[t];
    const Geom& g = inst[tl.inst].g;
    const int p0 = tl.p[0] + threadIdx.x, p1 = tl.p[1] + threadIdx.y;
    if (p0 > g.hi[0] || p1 > g.hi[1]) continue;
    const long nm0 = g.hi[0] - g.lo[0] + 1, nm = nm0 * (g.hi[1] - g.lo[1] + 1);
    const long q = (p1 - g.lo[1]) * nm0 + (p0 - g.lo[0]);
    const long c = inst[tl.inst].o.P + p0 + g.st[1] * p1;
    D* dst = pk + meshoff[tl.inst] * np + q;
    for (int iw = 0; iw < np; ++iw) {
      if (dir == 0)
        dst[(long)iw * nm] = to_t<D>(to_d(P0[(long)iw * sP + c]));
      else
        P0[(long)iw * sP + c] = (S)to_d(dst[(long)iw * nm]);
    }
  }
}

BcArgs bc_proto(sac_batch* b, void* A) {
  BcArgs a{};
  a.A = A;
  a.bgA = b->BG;
  a.type = b->d_type;
  a.fixed = b->d_fixed;
  a.fixB = b->d_fixB;
  std::memcpy(a.pairshift, b->pairshift, sizeof(a.pairshift));
  a.sA = b->totP;
  a.sB = b->totP;
  return a;
}

template <typename S>
void launch_bound_b(sac_batch* b, BcArgs a, int nvar, const GhostChunk* chunks, int n, const InstDyn* dyn) {
  if (!n) return;
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, b->dev);
  const unsigned grid = (unsigned)std::min<long>(n, (long)nsm * 8);
  kb_bound<S><<<grid, 256, 0, b->stream>>>(a, b->d_inst, chunks, n, nvar, dyn);
}

Stage2Args stage_base(sac_batch* b) {
  Stage2Args a{};
  a.g = b->h_inst[0].g;  // ndim, ndir, np, nw (geometry itself comes per instance)
  a.sP = b->totP;
  a.sB = b->totP;
  a.sI = b->maxI;
  a.sX = b->totX;
  a.bgv = b->BG;
  a.D = b->D;
  a.F = b->F;
  a.R = b->R;
  a.dx = b->dx;
  a.gamma = b->par.gamma;
  for (int d = 0; d < 3; ++d) a.grav[d] = (d < b->ndim) ? b->par.grav[d] : 0.0;
  a.dmin = 0;
  a.dmax = b->ndim - 1;
  a.iwmask = (1u << b->np) - 1u;
  for (int d = 0; d < 3; ++d)
    for (int s = 0; s < 2; ++s) a.zero1[d][s] = b->zero1[d][s];
  a.grav_on = (b->par.sourceunsplit && grav_mod(b->par.user)) ? 1 : 0;
  a.visc_on = (b->par.sourceunsplit && visc_on_b(b)) ? 1 : 0;
  a.divb_on = (b->par.sourceunsplit && b->par.divbfix && b->ndim > 1) ? 1 : 0;  // src/vacphys.mhd0.t:255
  a.res_on = (b->par.sourceunsplit && std::fabs(b->par.eta) > kSmallD) ? 1 : 0;
  a.eta = b->par.eta;
  a.driver = DRV_NONE;
  if (b->par.sourceunsplit && b->drv)
    a.driver = b->par.user == SAC_USR_STRAT ? DRV_STRAT : DRV_TUBE;  // amplitude and omega per instance
  a.drv = b->drv;
  return a;
}

BcArgs stage_bc(sac_batch* b, int s);
BatchStageArgs stage_args(sac_batch* b, int s, const Tile* tiles, int n);

// one fused RK stage s of batch b on b->stream: c_tot of the stage input, the
// fused kernel, the boundary fill (with the RK4 combinations of stages 3 and 4)
template <typename S>
void enqueue_fused_stage(sac_batch* b, int s, bool visc) {
  BatchStageArgs sa = stage_args(b, s, b->d_cour, b->n_cour);
  if (visc) launch_batch_ctot<S>(sa, b->stream);
  sa.tiles = b->d_fused;
  sa.ntiles = b->n_fused;
  launch_batch_stage2d<S>(sa, b->fused_shape, b->stream);
  launch_bound_b<S>(b, stage_bc(b, s), b->np, b->d_gh_all, b->n_gh_all, b->d_dyn);
}

// one RK4 step of every instance, src/vac.t:439-455 (enqueued on b->stream)
template <typename S>
void enqueue_step(sac_batch* b) {
  const int nb = (b->ninst + 255) / 256;
  const int ngrav = grav_mod(b->par.user) ? 1 : 0;
  const DynPair dp{{b->d_dyn, nullptr}, {b->ninst, 0}};
  kb_zero<<<nb, 256, 0, b->stream>>>(dp, 1);
  BatchStageArgs cb{};
  cb.a = stage_base(b);
  cb.a.wct = b->P[0];
  cb.inst = b->d_inst;
  cb.dyn = b->d_dyn;
  cb.tiles = b->d_cour;
  cb.ntiles = b->n_cour;
  launch_batch_courant<S>(cb, b->par.gamma, b->stream);
  kb_dt<<<nb, 256, 0, b->stream>>>(dp, b->ndim, b->par.courantpar, b->par.dtpar, visc_on_b(b) ? 1 : 0, ngrav,
                                   b->par.dtcantgrow ? 1 : 0, b->par.eta, b->par.dtdiffpar);
  void *w = b->P[0], *w1 = b->P[1], *w2 = b->P[2], *w3 = b->P[3];
  const void* wct[4] = {w, w1, w2, w3};
  void* out[4] = {w1, w2, w3, w};
  const int epi[4] = {EPI_PLAIN, EPI_PLAIN, EPI_RK4_S3, EPI_RK4_S4};
  const bool visc = visc_on_b(b);
  for (int s = 0; s < 4; ++s) {
    kb_zero<<<nb, 256, 0, b->stream>>>(dp, 0);
    if (b->fused) {
      enqueue_fused_stage<S>(b, s, visc);
      continue;
    }
    for (Group& gr : b->groups) {
      BatchStageArgs sa{};
      sa.a = stage_base(b);
      sa.a.wct = wct[s];
      sa.a.base = w;
      sa.a.out = out[s];
      sa.a.aux1 = w1;
      sa.a.aux2 = w2;
      sa.a.epi = epi[s];
      sa.inst = gr.d_inst;
      sa.dyn = b->d_dyn;
      sa.stage = s;
      sa.tiles = gr.d_face;
      sa.ntiles = gr.n_face;
      launch_batch_face<S>(sa, b->par.gamma, b->stream);
      if (visc) {
        sa.tiles = gr.d_nu;
        sa.ntiles = gr.n_nu;
        launch_batch_nu<S>(sa, b->stream);
      }
      sa.tiles = gr.d_upd;
      sa.ntiles = gr.n_upd;
      launch_batch_update<S>(sa, b->upd_blk, b->stream);
      BcArgs ba = bc_proto(b, out[s]);
      if (epi[s] == EPI_RK4_S3) {
        ba.mode = 1;
        ba.aux1 = w1;
        ba.aux2 = w2;
        ba.basep = w;
      } else if (epi[s] == EPI_RK4_S4) {
        ba.mode = 2;
        ba.aux1 = w1;
      }
      launch_bound_b<S>(b, ba, b->np, gr.d_gh, gr.n_gh, b->d_dyn);
    }
  }
  kb_time<<<nb, 256, 0, b->stream>>>(dp);
}

// the boundary-fill arguments of stage s (the RK4 combinations of stages 3 and 4
// are fused into the fill, as in the stage's update)
BcArgs stage_bc(sac_batch* b, int s) {
  void* out[4] = {b->P[1], b->P[2], b->P[3], b->P[0]};
  BcArgs ba = bc_proto(b, out[s]);
  if (s == 2) {
    ba.mode = 1;
    ba.aux1 = b->P[1];
    ba.aux2 = b->P[2];
    ba.basep = b->P[0];
  } else if (s == 3) {
    ba.mode = 2;
    ba.aux1 = b->P[1];
  }
  return ba;
}

// the fused-stage arguments of stage s over tile list (tiles, n)
BatchStageArgs stage_args(sac_batch* b, int s, const Tile* tiles, int n) {
  void *w = b->P[0], *w1 = b->P[1], *w2 = b->P[2], *w3 = b->P[3];
  const void* wct[4] = {w, w1, w2, w3};
  void* out[4] = {w1, w2, w3, w};
  const int epi[4] = {EPI_PLAIN, EPI_PLAIN, EPI_RK4_S3, EPI_RK4_S4};
  BatchStageArgs sa{};
  sa.a = stage_base(b);
  sa.a.wct = wct[s];
  sa.a.base = w;
  sa.a.out = out[s];
  sa.a.aux1 = w1;
  sa.a.aux2 = w2;
  sa.a.epi = epi[s];
  sa.inst = b->d_inst;
  sa.dyn = b->d_dyn;
  sa.stage = s;
  sa.tiles = tiles;
  sa.ntiles = n;
  return sa;
}

// stage s of a joined pair in joint kernels (c_tot when with_ctot, the fused
// stage, the boundary fill), on the lead's stream
void enqueue_joint_stage(sac_batch* b, sac_batch* p, int s, bool with_ctot) {
  cudaStream_t st = b->stream;
  if (with_ctot) {
    JointStageArgs jt{};
    jt.b[0] = stage_args(b, s, b->d_cour, b->n_cour);
    jt.b[1] = stage_args(p, s, p->d_cour, p->n_cour);
    launch_joint_ctot(jt, st);
  }
  JointStageArgs js{};
  js.b[0] = stage_args(b, s, b->d_fused, b->n_fused);
  js.b[1] = stage_args(p, s, p->d_fused, p->n_fused);
  launch_joint_stage2d(js, b->fused_shape, st);
  JointBoundArgs jb{};
  sac_batch* both[2] = {b, p};
  for (int k = 0; k < 2; ++k) {
    jb.proto[k] = stage_bc(both[k], s);
    jb.inst[k] = both[k]->d_inst;
    jb.chunks[k] = both[k]->d_gh_all;
    jb.n[k] = both[k]->n_gh_all;
    jb.dyn[k] = both[k]->d_dyn;
  }
  launch_joint_bound(jb, b->np, st);
}

// one RK4 step of the instances of a joined pair, every kernel covering both
// batches: b holds the FP64 instances, p the FP32 ones (same parameters, both 2D
// on the fused stage); the steps and their order are those of enqueue_step
void enqueue_joint(sac_batch* b, sac_batch* p) {
  const DynPair dp{{b->d_dyn, p->d_dyn}, {b->ninst, p->ninst}};
  const int nb = (dp.total() + 255) / 256;
  const int ngrav = grav_mod(b->par.user) ? 1 : 0;
  cudaStream_t st = b->stream;
  kb_zero<<<nb, 256, 0, st>>>(dp, 1);
  JointStageArgs jc{};
  jc.b[0] = stage_args(b, 0, b->d_cour, b->n_cour);
  jc.b[1] = stage_args(p, 0, p->d_cour, p->n_cour);
  launch_joint_courant(jc, b->par.gamma, st);
  kb_dt<<<nb, 256, 0, st>>>(dp, b->ndim, b->par.courantpar, b->par.dtpar, visc_on_b(b) ? 1 : 0, ngrav,
                            b->par.dtcantgrow ? 1 : 0, b->par.eta, b->par.dtdiffpar);
  const bool visc = visc_on_b(b);
  for (int s = 0; s < 4; ++s) {
    kb_zero<<<nb, 256, 0, st>>>(dp, 0);
    enqueue_joint_stage(b, p, s, visc);
  }
  kb_time<<<nb, 256, 0, st>>>(dp);
}

// one RK4 step of a joined pair as two branches of the graph: the partner's own
// kernels on its own stream beside the lead's (both forked from and joined back
// to the lead's stream)
void enqueue_forked(sac_batch* b, sac_batch* p) {
  cudaEventRecord(b->ev_fork, b->stream);
  cudaStreamWaitEvent(p->own_stream, b->ev_fork, 0);
  p->stream = p->own_stream;
  enqueue_step<float>(p);
  p->stream = b->stream;
  cudaEventRecord(b->ev_join, p->own_stream);
  enqueue_step<double>(b);
  cudaStreamWaitEvent(b->stream, b->ev_join, 0);
}

void drop_exec(sac_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec), b->exec = nullptr;
  if (b->graph) cudaGraphDestroy(b->graph), b->graph = nullptr;
}

// a batch's graph, and the joint graph that also reads its arrays
void drop_graph(sac_batch* b) {
  drop_exec(b);
  if (b->lead) drop_exec(b->lead);
}

sac_status build_graph(sac_batch* b) {
  drop_graph(b);
  BK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  if (b->partner && b->join_form == 1)
    enqueue_forked(b, b->partner);
  else if (b->partner)
    enqueue_joint(b, b->partner);
  else if (b->prec == SAC_PREC_FP32)
    enqueue_step<float>(b);
  else
    enqueue_step<double>(b);
  BK(cudaStreamEndCapture(b->stream, &b->graph));
  BK(cudaGraphInstantiate(&b->exec, b->graph, 0));
  return SAC_OK;
}

sac_status build_lists(sac_batch* b) {
  // a global mesh tile list (courant) and ghost list (boundaries)
  std::vector<Tile> cour = make_tiles(b->h_inst, 0, b->ninst, 2, dim3(32, 8, 1));
  std::vector<GhostChunk> gh = make_ghosts(b->h_inst, 0, b->ninst);
  sac_status st;
  if ((st = upload_vec(b, &b->d_cour, cour)) != SAC_OK) return st;
  if ((st = upload_vec(b, &b->d_gh_all, gh)) != SAC_OK) return st;
  b->n_cour = (int)cour.size();
  b->n_gh_all = (int)gh.size();
  if (fused_ok(b)) {
    const dim3 ft((unsigned)stage2d_shape_tx(b->fused_shape), (unsigned)stage2d_shape_ty(b->fused_shape), 1);
    std::vector<Tile> fu = make_tiles(b->h_inst, 0, b->ninst, 2, ft);
    if ((st = upload_vec(b, &b->d_fused, fu)) != SAC_OK) return st;
    b->n_fused = (int)fu.size();
  }
  for (Group& gr : b->groups) {
    std::vector<Tile> f = make_tiles(b->h_inst, gr.i0, gr.i1, 0, dim3(32, 8, 1));
    std::vector<Tile> n = make_tiles(b->h_inst, gr.i0, gr.i1, 1, dim3(32, 8, 1));
    std::vector<Tile> u = make_tiles(b->h_inst, gr.i0, gr.i1, 2, b->upd_blk);
    std::vector<GhostChunk> g = make_ghosts(b->h_inst, gr.i0, gr.i1);
    if ((st = upload_vec(b, &gr.d_face, f)) != SAC_OK) return st;
    if ((st = upload_vec(b, &gr.d_nu, n)) != SAC_OK) return st;
    if ((st = upload_vec(b, &gr.d_upd, u)) != SAC_OK) return st;
    if ((st = upload_vec(b, &gr.d_gh, g)) != SAC_OK) return st;
    gr.n_face = (int)f.size();
    gr.n_nu = (int)n.size();
    gr.n_upd = (int)u.size();
    gr.n_gh = (int)g.size();
  }
  return SAC_OK;
}

// the parameters two joined batches share: all but the precision
bool same_family(const sac_batch* a, const sac_batch* b) {
  const sac_params &x = a->par, &y = b->par;
  if (a->ndim != b->ndim || a->ndir != b->ndir || a->dev != b->dev) return false;
  if (x.gamma != y.gamma || x.eta != y.eta || x.nu != y.nu || x.courantpar != y.courantpar || x.dtpar != y.dtpar ||
      x.dtdiffpar != y.dtdiffpar || x.dtcantgrow != y.dtcantgrow || x.sourceunsplit != y.sourceunsplit ||
      x.divbfix != y.divbfix || x.user != y.user || x.alias_nu_grav3 != y.alias_nu_grav3)
    return false;
  for (int d = 0; d < 3; ++d)
    if (x.grav[d] != y.grav[d]) return false;
  for (int i = 0; i < 16; ++i)
    if (x.userpar[i] != y.userpar[i]) return false;
  return std::strcmp(x.typeadvance, y.typeadvance) == 0;
}

// ms of one RK stage of a joined pair in form f (stage 0: it reads w and writes
// the scratch w1 only), on the lead's stream, after one untimed run
double join_stage_ms(sac_batch* b, sac_batch* p, int f, cudaEvent_t e0, cudaEvent_t e1) {
  const bool visc = visc_on_b(b);
  auto zero = [](sac_batch* x, InstDyn* d2, int n2) {
    const DynPair dp{{x->d_dyn, d2}, {x->ninst, n2}};
    kb_zero<<<(dp.total() + 255) / 256, 256, 0, x->stream>>>(dp, 0);
  };
  auto run = [&]() {
    if (f == 0) {
      zero(b, p->d_dyn, p->ninst);
      enqueue_joint_stage(b, p, 0, visc);
      return;
    }
    cudaEventRecord(b->ev_fork, b->stream);
    cudaStreamWaitEvent(p->own_stream, b->ev_fork, 0);
    p->stream = p->own_stream;
    zero(p, nullptr, 0);
    enqueue_fused_stage<float>(p, 0, visc);
    p->stream = b->stream;
    cudaEventRecord(b->ev_join, p->own_stream);
    zero(b, nullptr, 0);
    enqueue_fused_stage<double>(b, 0, visc);
    cudaStreamWaitEvent(b->stream, b->ev_join, 0);
  };
  run();
  cudaEventRecord(e0, b->stream);
  for (int r = 0; r < 3; ++r) run();
  cudaEventRecord(e1, b->stream);
  cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  return ms / 3;
}

// ends a join (lead: the FP64 batch); the partner gets its own stream back
void unjoin(sac_batch* lead) {
  sac_batch* p = lead->partner;
  if (!p) return;
  cudaSetDevice(lead->dev);
  cudaStreamSynchronize(lead->stream);
  drop_exec(lead);
  if (lead->ev_fork) cudaEventDestroy(lead->ev_fork), lead->ev_fork = nullptr;
  if (lead->ev_join) cudaEventDestroy(lead->ev_join), lead->ev_join = nullptr;
  p->stream = p->own_stream;
  p->own_stream = nullptr;
  p->lead = nullptr;
  lead->partner = nullptr;
}

bool joined(const sac_batch* b) { return b->lead || b->partner; }

// frees the device arrays; the group ranges stay (they depend on the sizes only)
void free_all(sac_batch* b) {
  drop_graph(b);
  for (auto& p : b->P)
    if (p) cudaFree(p), p = nullptr;
  auto fr = [](auto*& p) {
    if (p) cudaFree((void*)p);
    p = nullptr;
  };
  fr(b->BG), fr(b->dx), fr(b->drv), fr(b->stg), fr(b->d_dyn), fr(b->d_inst), fr(b->d_cour), fr(b->d_gh_all), fr(b->d_meshoff);
  fr(b->d_fused);
  fr(b->D), fr(b->F), fr(b->R), fr(b->d_type), fr(b->d_fixed), fr(b->d_fixB);
  for (Group& gr : b->groups) fr(gr.d_inst), fr(gr.d_face), fr(gr.d_nu), fr(gr.d_upd), fr(gr.d_gh);
}

}  // namespace

extern "C" {

sac_status sac_batch_create(const sac_params* p, int ndim, int ndir, int ninst, const int* nx, long group_cells,
                            sac_batch** out) {
  if (!p || !nx || !out || ninst < 1) return SAC_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return SAC_ERR_NODEVICE;
  if (ndim < 1 || ndim > 2 || ndir < ndim || ndir > 3) return SAC_ERR_UNSUPPORTED;
  if (std::string(p->typeadvance) != "fourstep") return SAC_ERR_UNSUPPORTED;
  if (p->precision != SAC_PREC_FP64 && p->precision != SAC_PREC_FP32) return SAC_ERR_UNSUPPORTED;
  if (p->user == SAC_USR_SLOG || (p->user == SAC_USR_TUBE && ndim < 2)) return SAC_ERR_UNSUPPORTED;
  if (p->eta < 0.0) return SAC_ERR_UNSUPPORTED;  // a user specialeta; eta > 0 is built
  if (p->smallfix) return SAC_ERR_UNSUPPORTED;    // keeppositive runs on single-grid contexts only
  if (p->compactres) return SAC_ERR_UNSUPPORTED;  // so does the compact resistive form
  sac_batch* b = new sac_batch();
  b->par = *p;
  b->dev = p->device;
  b->prec = p->precision;
  b->es = b->prec == SAC_PREC_FP32 ? 4 : 8;
  b->ndim = ndim;
  b->ndir = ndir;
  b->nw = 3 * ndir + 4;
  b->np = 2 * ndir + 2;
  b->ninst = ninst;
  if (cudaSetDevice(b->dev) != cudaSuccess || cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking)) {
    delete b;
    return SAC_ERR_CUDA;
  }
  // instance geometry and offsets
  long off = 0;
  b->h_inst.resize(ninst);
  for (int i = 0; i < ninst; ++i) {
    Geom& g = b->h_inst[i].g;
    g.ndim = ndim;
    g.ndir = ndir;
    g.nw = b->nw;
    g.np = b->np;
    for (int d = 0; d < 3; ++d) {
      g.n[d] = d < ndim ? nx[i * ndim + d] + 4 : 1;
      g.lo[d] = d < ndim ? 2 : 0;
      g.hi[d] = d < ndim ? nx[i * ndim + d] + 1 : 0;
      if (d < ndim && nx[i * ndim + d] < 6) {
        sac_batch_destroy(b);
        return SAC_ERR_ARG;
      }
    }
    g.st[0] = 1;
    g.st[1] = g.n[0];
    g.st[2] = (long)g.n[0] * g.n[1];
    g.ncell = (long)g.n[0] * g.n[1] * g.n[2];
    if (g.ncell > 2147483647L) {  // cell indices inside one instance are 32-bit
      sac_batch_destroy(b);
      return SAC_ERR_UNSUPPORTED;
    }
    b->h_inst[i].o = Offs{off, off, 0, off};
    off += g.ncell;
  }
  b->totP = b->totX = off;
  // groups: consecutive instances with at most group_cells cells of intermediates
  const long cap = group_cells > 0 ? group_cells : (1L << 26);
  Group cur;
  cur.i0 = 0;
  for (int i = 0; i < ninst; ++i) {
    const long n = b->h_inst[i].g.ncell;
    if (cur.cells > 0 && cur.cells + n > cap) {
      cur.i1 = i;
      b->groups.push_back(cur);
      cur = Group();
      cur.i0 = i;
    }
    cur.cells += n;
  }
  cur.i1 = ninst;
  b->groups.push_back(cur);
  for (const Group& gr : b->groups) b->maxI = std::max(b->maxI, gr.cells);
  *out = b;
  return SAC_OK;
}

void sac_batch_destroy(sac_batch* b) {
  if (!b) return;
  if (b->partner) unjoin(b);
  if (b->lead) unjoin(b->lead);
  cudaSetDevice(b->dev);
  if (b->stream) cudaStreamSynchronize(b->stream);
  free_all(b);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

const char* sac_batch_last_error(const sac_batch* b) { return b ? b->err.c_str() : "null batch"; }

// x: the instances' full-grid coordinate blocks x(ixG^T,ndim) one after another
sac_status sac_batch_set_grid(sac_batch* b, const double* x) {
  if (!b || !x) return SAC_ERR_ARG;
  if (joined(b)) return bfail(b, SAC_ERR_STATE, "sac_batch_unjoin first");
  BK(cudaSetDevice(b->dev));
  const int ndim = b->ndim;
  std::vector<double> hdx((size_t)ndim * b->totX);
  const bool gauss = b->par.user == SAC_USR_STRAT || b->par.user == SAC_USR_TUBE;
  std::vector<double> hdrv(gauss ? (size_t)2 * b->totX : 0), prof;
  b->mindx2.assign((size_t)b->ninst * 3, 0.0);
  b->dtgrav.assign(b->ninst, kBig);
  long xoff = 0;
  for (int i = 0; i < b->ninst; ++i) {
    const Geom& g = b->h_inst[i].g;
    std::vector<double> hx1, hdx1;
    gridsetup1(g.n, g.lo, g.hi, ndim, g.ncell, x + xoff, false, hx1, hdx1);
    xoff += (long)ndim * g.ncell;
    if (gauss) {
      prof.assign((size_t)2 * g.ncell, 0.0);
      gauss_driver_profiles(b->par.user, ndim, g.ncell, hx1.data(), b->par.userpar, prof.data());
      for (int k = 0; k < 2; ++k)
        std::copy(prof.begin() + (long)k * g.ncell, prof.begin() + (long)(k + 1) * g.ncell,
                  hdrv.begin() + (long)k * b->totX + b->h_inst[i].o.X);
    }
    double mindx_all = kBig;
    for (int d = 0; d < ndim; ++d) {
      double m2 = kBig;
      for (long c = 0; c < g.ncell; ++c) {
        hdx[(size_t)d * b->totX + b->h_inst[i].o.X + c] = hdx1[(size_t)d * g.ncell + c];
        const int p0 = (int)(c % g.n[0]), p1 = (int)((c / g.n[0]) % g.n[1]);
        if (p0 < g.lo[0] || p0 > g.hi[0] || p1 < g.lo[1] || p1 > g.hi[1]) continue;
        const double v = hdx1[(size_t)d * g.ncell + c];
        m2 = std::min(m2, v * v);
        mindx_all = std::min(mindx_all, v);
      }
      b->mindx2[i * 3 + d] = m2;
    }
    for (int d = 0; d < ndim; ++d)
      if (std::fabs(b->par.grav[d]) > 0.0)
        b->dtgrav[i] = std::min(b->dtgrav[i], 1.0 / std::sqrt(std::fabs(b->par.grav[d]) / mindx_all));
  }
  free_all(b);
  b->grid_set = b->bc_set = b->state_set = b->bc_init = false;
  const size_t es = b->es;
  for (auto& p : b->P) {
    BK(cudaMalloc(&p, es * b->np * b->totP));
    BK(cudaMemset(p, 0, es * b->np * b->totP));  // scratch stages of finished instances stay finite
  }
  BK(cudaMalloc(&b->BG, sizeof(double) * (b->nw - b->np) * b->totP));
  BK(cudaMalloc(&b->dx, sizeof(double) * ndim * b->totX));
  BK(cudaMemcpy(b->dx, hdx.data(), sizeof(double) * hdx.size(), cudaMemcpyHostToDevice));
  if (gauss) {
    BK(cudaMalloc(&b->drv, sizeof(double) * hdrv.size()));
    BK(cudaMemcpy(b->drv, hdrv.data(), sizeof(double) * hdrv.size(), cudaMemcpyHostToDevice));
  }
  BK(cudaMalloc(&b->D, es * (b->ndir + 3) * b->maxI));
  BK(cudaMalloc(&b->F, es * (size_t)ndim * b->np * b->maxI));
  BK(cudaMalloc(&b->R, es * (size_t)nr_pairs(ndim) * b->maxI));
  BK(cudaMemset(b->R, 0, es * (size_t)nr_pairs(ndim) * b->maxI));
  if (b->prec == SAC_PREC_FP32) BK(cudaMalloc(&b->stg, sizeof(double) * b->np * b->totP));
  // instance tables: global and per group (group-local intermediate offsets)
  sac_status st;
  if ((st = upload_vec(b, &b->d_inst, b->h_inst)) != SAC_OK) return st;
  for (Group& gr : b->groups) {
    std::vector<InstInfo> t = b->h_inst;
    long ioff = 0;
    for (int i = gr.i0; i < gr.i1; ++i) {
      t[i].o.I = ioff;
      ioff += t[i].g.ncell;
    }
    if ((st = upload_vec(b, &gr.d_inst, t)) != SAC_OK) return st;
  }
  std::vector<long> moff(b->ninst + 1, 0);
  for (int i = 0; i < b->ninst; ++i) {
    const Geom& g = b->h_inst[i].g;
    long nm = 1;
    for (int d = 0; d < ndim; ++d) nm *= g.hi[d] - g.lo[d] + 1;
    moff[i + 1] = moff[i] + nm;
  }
  b->mesh_total = moff[b->ninst];
  if ((st = upload_vec(b, &b->d_meshoff, moff)) != SAC_OK) return st;
  std::vector<InstDyn> dyn(b->ninst);
  for (int i = 0; i < b->ninst; ++i) {
    std::memset(&dyn[i], 0, sizeof(InstDyn));
    for (int d = 0; d < 3; ++d) dyn[i].mindx2[d] = b->mindx2[i * 3 + d];
    dyn[i].dtgrav = b->dtgrav[i];
    dyn[i].drvA = b->par.userpar[0];
    dyn[i].omega = b->par.userpar[1];
  }
  if ((st = upload_vec(b, &b->d_dyn, dyn)) != SAC_OK) return st;
  if ((st = build_lists(b)) != SAC_OK) return st;
  b->grid_set = true;
  return SAC_OK;
}

// one typeB(nw,2*ndim) shared by every instance; types that store ghost values
// (fixed, fixed1, grad1) are not available in the batch
sac_status sac_batch_set_boundaries(sac_batch* b, const char* typeB) {
  if (!b || !typeB) return SAC_ERR_ARG;
  if (joined(b)) return bfail(b, SAC_ERR_STATE, "sac_batch_unjoin first");
  if (!b->grid_set) return bfail(b, SAC_ERR_STATE, "sac_batch_set_grid first");
  BK(cudaSetDevice(b->dev));
  const int nB = 2 * b->ndim;
  std::vector<int8_t> ty((size_t)b->nw * nB);
  std::vector<int> fx((size_t)b->nw * nB, 0);
  std::vector<std::string> t((size_t)b->nw * nB);
  for (int iB = 0; iB < nB; ++iB)
    for (int iw = 0; iw < b->nw; ++iw) {
      std::string s(typeB + SAC_LENTYPE * ((long)iw + (long)b->nw * iB), SAC_LENTYPE);
      while (!s.empty() && (s.back() == ' ' || s.back() == '\0')) s.pop_back();
      int8_t code;
      if (s == "cont") code = BT_CONT;
      else if (s == "cont1") code = BT_CONT1;
      else if (s == "periodic") code = BT_PERIODIC;
      else if (s == "symm") code = BT_SYMM;
      else if (s == "symm0") code = BT_SYMM0;
      else if (s == "asymm") code = BT_ASYMM;
      else if (s == "contCD4") code = BT_CONTCD4;
      else return bfail(b, SAC_ERR_UNSUPPORTED, "boundary type '" + s + "' is not available in the batch");
      ty[iw * nB + iB] = code;
      t[iw + (long)b->nw * iB] = s;
    }
  for (int iB = 0; iB < nB; ++iB)
    if (t[(long)b->nw * iB] == "periodic" && t[(long)b->nw * (iB ^ 1)] != "periodic")
      return bfail(b, SAC_ERR_ARG, "Error in BoundSetup: No periodic pair");
  for (int d = 0; d < b->ndim; ++d)
    for (int s = 0; s < 2; ++s) {
      const std::string& t1 = t[(long)b->nw * (2 * d + s)];
      b->zero1[d][s] = (t1 != "periodic" && t1 != "mpi") ? 1 : 0;
    }
  // periodic source offsets are per instance (mesh size): kb_bound reads them
  // from the geometry, so pairshift here only flags the use
  sac_status st;
  if ((st = upload_vec(b, &b->d_type, ty)) != SAC_OK) return st;
  if ((st = upload_vec(b, &b->d_fixed, fx)) != SAC_OK) return st;
  if (!b->d_fixB) BK(cudaMalloc(&b->d_fixB, sizeof(double)));
  b->bc_set = true;
  return SAC_OK;
}

// w: the full-grid state blocks w(ixG^T,nw) of instances i0..i0+n-1, one after another
sac_status sac_batch_upload_range(sac_batch* b, int i0, int n, const double* w) {
  if (!b || !w || i0 < 0 || n < 0 || i0 + n > (b ? b->ninst : 0)) return SAC_ERR_ARG;
  if (!b->grid_set) return bfail(b, SAC_ERR_STATE, "sac_batch_set_grid first");
  if (!n) return SAC_OK;
  BK(cudaSetDevice(b->dev));
  const int nb = b->nw - b->np;
  long woff = 0;
  double* dst64 = b->prec == SAC_PREC_FP32 ? b->stg : (double*)b->P[0];
  for (int i = i0; i < i0 + n; ++i) {
    const long nc = b->h_inst[i].g.ncell, o = b->h_inst[i].o.P;
    for (int iw = 0; iw < b->np; ++iw)
      BK(cudaMemcpyAsync(dst64 + (long)iw * b->totP + o, w + woff + (long)iw * nc, sizeof(double) * nc,
                         cudaMemcpyHostToDevice, b->stream));
    for (int k = 0; k < nb; ++k)
      BK(cudaMemcpyAsync(b->BG + (long)k * b->totP + o, w + woff + (long)(b->np + k) * nc, sizeof(double) * nc,
                         cudaMemcpyHostToDevice, b->stream));
    woff += (long)b->nw * nc;
  }
  if (b->prec == SAC_PREC_FP32) {
    const long o0 = b->h_inst[i0].o.P, span = woff / b->nw;
    for (int iw = 0; iw < b->np; ++iw)
      k_convert<float, double><<<592, 256, 0, b->stream>>>((float*)b->P[0] + (long)iw * b->totP + o0,
                                                           b->stg + (long)iw * b->totP + o0, span);
    BK(cudaGetLastError());
  }
  BK(cudaStreamSynchronize(b->stream));
  b->state_set = true;
  return SAC_OK;
}

sac_status sac_batch_download_range(sac_batch* b, int i0, int n, double* w) {
  if (!b || !w || i0 < 0 || n < 0 || i0 + n > (b ? b->ninst : 0)) return SAC_ERR_ARG;
  if (!b->state_set) return bfail(b, SAC_ERR_STATE, "no state on the device");
  if (!n) return SAC_OK;
  BK(cudaSetDevice(b->dev));
  const int nb = b->nw - b->np;
  const double* src64 = (const double*)b->P[0];
  const long o0 = b->h_inst[i0].o.P;
  const long span = b->h_inst[i0 + n - 1].o.P + b->h_inst[i0 + n - 1].g.ncell - o0;
  if (b->prec == SAC_PREC_FP32) {
    for (int iw = 0; iw < b->np; ++iw)
      k_convert<double, float><<<592, 256, 0, b->stream>>>(b->stg + (long)iw * b->totP + o0,
                                                           (const float*)b->P[0] + (long)iw * b->totP + o0, span);
    BK(cudaGetLastError());
    src64 = b->stg;
  }
  long woff = 0;
  for (int i = i0; i < i0 + n; ++i) {
    const long nc = b->h_inst[i].g.ncell, o = b->h_inst[i].o.P;
    for (int iw = 0; iw < b->np; ++iw)
      BK(cudaMemcpyAsync(w + woff + (long)iw * nc, src64 + (long)iw * b->totP + o, sizeof(double) * nc,
                         cudaMemcpyDeviceToHost, b->stream));
    for (int k = 0; k < nb; ++k)
      BK(cudaMemcpyAsync(w + woff + (long)(b->np + k) * nc, b->BG + (long)k * b->totP + o, sizeof(double) * nc,
                         cudaMemcpyDeviceToHost, b->stream));
    woff += (long)b->nw * nc;
  }
  BK(cudaStreamSynchronize(b->stream));
  return SAC_OK;
}

sac_status sac_batch_upload(sac_batch* b, const double* w) {
  return b ? sac_batch_upload_range(b, 0, b->ninst, w) : SAC_ERR_ARG;
}

sac_status sac_batch_download(sac_batch* b, double* w) {
  return b ? sac_batch_download_range(b, 0, b->ninst, w) : SAC_ERR_ARG;
}

// getboundary(t,1,nw,1,ndim,w) on every instance
sac_status sac_batch_getboundary(sac_batch* b) {
  if (!b) return SAC_ERR_ARG;
  if (!b->state_set || !b->bc_set) return bfail(b, SAC_ERR_STATE, "state and boundaries must be set");
  BK(cudaSetDevice(b->dev));
  BcArgs a = bc_proto(b, b->P[0]);
  a.init = 1;
  if (b->prec == SAC_PREC_FP32)
    launch_bound_b<float>(b, a, b->nw, b->d_gh_all, b->n_gh_all, nullptr);
  else
    launch_bound_b<double>(b, a, b->nw, b->d_gh_all, b->n_gh_all, nullptr);
  BK(cudaGetLastError());
  BK(cudaStreamSynchronize(b->stream));
  b->bc_init = true;
  return SAC_OK;
}

// advance every instance by nsteps RK4 steps with its own dt (graph replays)
sac_status sac_batch_advance(sac_batch* b, int nsteps) {
  if (!b || nsteps < 0) return SAC_ERR_ARG;
  if (!b->bc_init) return bfail(b, SAC_ERR_STATE, "call sac_batch_getboundary first");
  if (b->lead) return bfail(b, SAC_ERR_STATE, "joined: sac_batch_advance on the FP64 batch advances this one");
  BK(cudaSetDevice(b->dev));
  if (!b->exec) {
    sac_status st = build_graph(b);
    if (st != SAC_OK) return st;
  }
  for (int k = 0; k < nsteps; ++k) BK(cudaGraphLaunch(b->exec, b->stream));
  BK(cudaGetLastError());
  return SAC_OK;
}

// per-instance t, last dt and step count (synchronises); returns
// SAC_ERR_NONFINITE when any instance met a NaN/Inf in its dt reductions
sac_status sac_batch_state(sac_batch* b, double* t, double* dt, int* it) {
  if (!b) return SAC_ERR_ARG;
  BK(cudaSetDevice(b->dev));
  std::vector<InstDyn> dyn(b->ninst);
  BK(cudaMemcpyAsync(dyn.data(), b->d_dyn, sizeof(InstDyn) * b->ninst, cudaMemcpyDeviceToHost, b->stream));
  BK(cudaStreamSynchronize(b->stream));
  int bad = 0;
  for (int i = 0; i < b->ninst; ++i) {
    if (t) t[i] = dyn[i].t;
    if (dt) dt[i] = dyn[i].dt;
    if (it) it[i] = dyn[i].it;
    bad |= dyn[i].bad;
  }
  return bad ? bfail(b, SAC_ERR_NONFINITE, "non-finite wave speed or viscosity in an instance") : SAC_OK;
}

sac_status sac_batch_synchronize(sac_batch* b) {
  if (!b) return SAC_ERR_ARG;
  BK(cudaSetDevice(b->dev));
  BK(cudaStreamSynchronize(b->stream));
  return SAC_OK;
}

void* sac_batch_get_stream(const sac_batch* b) { return b ? (void*)b->stream : nullptr; }

// Autotuner: time the update pass of stage 1 for each candidate tile shape on
// the actual batch, keep the fastest, rebuild the tile lists and the graph.
// tile_out[2] receives the chosen shape, ms_out the time per update pass.
sac_status sac_batch_tune(sac_batch* b, int* tile_out, double* ms_out) {
  if (!b) return SAC_ERR_ARG;
  if (joined(b)) return bfail(b, SAC_ERR_STATE, "tune each batch before sac_batch_join");
  if (!b->bc_init) return bfail(b, SAC_ERR_STATE, "call sac_batch_getboundary first");
  BK(cudaSetDevice(b->dev));
  const dim3 cands[] = {dim3(32, 4, 1), dim3(32, 8, 1), dim3(64, 4, 1), dim3(16, 16, 1), dim3(128, 2, 1),
                        dim3(256, 1, 1)};
  // the update pass skips instances with dt = 0 (finished, or before the first
  // step): time it with a tiny nonzero dt and restore the table afterwards
  std::vector<InstDyn> saved(b->ninst), tmp;
  BK(cudaMemcpy(saved.data(), b->d_dyn, sizeof(InstDyn) * b->ninst, cudaMemcpyDeviceToHost));
  tmp = saved;
  for (auto& d : tmp)
    if (d.dt == 0.0) d.dt = 1e-300;
  BK(cudaMemcpy(b->d_dyn, tmp.data(), sizeof(InstDyn) * b->ninst, cudaMemcpyHostToDevice));
  cudaEvent_t e0, e1;
  BK(cudaEventCreate(&e0));
  BK(cudaEventCreate(&e1));
  double best = 1e300;
  dim3 bestb = b->upd_blk;
  for (const dim3& blk : cands) {
    if (b->ndim == 1 && blk.y != 1) continue;
    b->upd_blk = blk;
    sac_status st = build_lists(b);
    if (st != SAC_OK) return st;
    auto run = [&]() {
      for (Group& gr : b->groups) {
        BatchStageArgs sa{};
        sa.a = stage_base(b);
        sa.a.wct = b->P[0];
        sa.a.base = b->P[0];
        sa.a.out = b->P[1];
        sa.a.epi = EPI_PLAIN;
        sa.inst = gr.d_inst;
        sa.dyn = b->d_dyn;
        sa.stage = 0;
        sa.tiles = gr.d_upd;
        sa.ntiles = gr.n_upd;
        if (b->prec == SAC_PREC_FP32)
          launch_batch_update<float>(sa, blk, b->stream);
        else
          launch_batch_update<double>(sa, blk, b->stream);
      }
    };
    run();  // warm-up
    BK(cudaEventRecord(e0, b->stream));
    for (int r = 0; r < 3; ++r) run();
    BK(cudaEventRecord(e1, b->stream));
    BK(cudaEventSynchronize(e1));
    float ms = 0;
    BK(cudaEventElapsedTime(&ms, e0, e1));
    if (ms / 3 < best) {
      best = ms / 3;
      bestb = blk;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  // the timing runs wrote w1 (scratch) and the running max nu: restore the table
  BK(cudaMemcpy(b->d_dyn, saved.data(), sizeof(InstDyn) * b->ninst, cudaMemcpyHostToDevice));
  b->upd_blk = bestb;
  b->fused = false;
  sac_status st = build_lists(b);
  if (st != SAC_OK) return st;
  // the whole stage: the three passes with the chosen update tile against the
  // fused kernel in each of its tile shapes (2D, default sources)
  if (fused_ok(b) && visc_on_b(b)) {
    BK(cudaMemcpy(b->d_dyn, tmp.data(), sizeof(InstDyn) * b->ninst, cudaMemcpyHostToDevice));
    BK(cudaEventCreate(&e0));
    BK(cudaEventCreate(&e1));
    auto stage_ms = [&](auto&& run) -> double {
      run();
      cudaEventRecord(e0, b->stream);
      for (int r = 0; r < 3; ++r) run();
      cudaEventRecord(e1, b->stream);
      cudaEventSynchronize(e1);
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      return ms / 3;
    };
    auto proto = [&]() {
      BatchStageArgs sa{};
      sa.a = stage_base(b);
      sa.a.wct = b->P[0];
      sa.a.base = b->P[0];
      sa.a.out = b->P[1];
      sa.a.epi = EPI_PLAIN;
      sa.dyn = b->d_dyn;
      sa.stage = 0;
      return sa;
    };
    double three = stage_ms([&]() {
      for (Group& gr : b->groups) {
        BatchStageArgs sa = proto();
        sa.inst = gr.d_inst;
        sa.tiles = gr.d_face;
        sa.ntiles = gr.n_face;
        if (b->prec == SAC_PREC_FP32) launch_batch_face<float>(sa, b->par.gamma, b->stream);
        else launch_batch_face<double>(sa, b->par.gamma, b->stream);
        sa.tiles = gr.d_nu;
        sa.ntiles = gr.n_nu;
        if (b->prec == SAC_PREC_FP32) launch_batch_nu<float>(sa, b->stream);
        else launch_batch_nu<double>(sa, b->stream);
        sa.tiles = gr.d_upd;
        sa.ntiles = gr.n_upd;
        if (b->prec == SAC_PREC_FP32) launch_batch_update<float>(sa, b->upd_blk, b->stream);
        else launch_batch_update<double>(sa, b->upd_blk, b->stream);
      }
    });
    double bestf = 1e300;
    int bests = 0;
    for (int sh = 0; sh < kStage2dShapeCount; ++sh) {
      b->fused_shape = sh;
      if ((st = build_lists(b)) != SAC_OK) return st;
      const double ms = stage_ms([&]() {
        BatchStageArgs sa = proto();
        sa.inst = b->d_inst;
        sa.tiles = b->d_cour;
        sa.ntiles = b->n_cour;
        if (b->prec == SAC_PREC_FP32) launch_batch_ctot<float>(sa, b->stream);
        else launch_batch_ctot<double>(sa, b->stream);
        sa.tiles = b->d_fused;
        sa.ntiles = b->n_fused;
        if (b->prec == SAC_PREC_FP32) launch_batch_stage2d<float>(sa, sh, b->stream);
        else launch_batch_stage2d<double>(sa, sh, b->stream);
      });
      if (ms < bestf) {
        bestf = ms;
        bests = sh;
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    BK(cudaGetLastError());
    BK(cudaMemcpy(b->d_dyn, saved.data(), sizeof(InstDyn) * b->ninst, cudaMemcpyHostToDevice));
    b->fused_shape = bests;
    b->fused = bestf < three;
    b->tune_three_ms = three;
    b->tune_fused_ms = bestf;
    if ((st = build_lists(b)) != SAC_OK) return st;
  }
  drop_graph(b);
  if (tile_out) {
    tile_out[0] = (int)bestb.x;
    tile_out[1] = (int)bestb.y;
  }
  if (ms_out) *ms_out = best;
  return SAC_OK;
}

// stage form: fused != 0 runs each stage as the fused per-tile kernel in tile
// shape `shape` (2D instances with the default sources only), 0 as the face /
// setnu / update passes
sac_status sac_batch_set_stage(sac_batch* b, int fused, int shape) {
  if (!b) return SAC_ERR_ARG;
  if (joined(b)) return bfail(b, SAC_ERR_STATE, "joined batches keep the fused stage; sac_batch_unjoin first");
  if (fused && !fused_ok(b))
    return bfail(b, SAC_ERR_UNSUPPORTED, "the fused stage covers 2D instances without Powell's or the resistive term");
  if (shape < 0 || shape >= kStage2dShapeCount) return bfail(b, SAC_ERR_ARG, "no such tile shape");
  BK(cudaSetDevice(b->dev));
  b->fused = fused != 0;
  b->fused_shape = shape;
  if (b->grid_set) {
    sac_status st = build_lists(b);
    if (st != SAC_OK) return st;
  }
  drop_graph(b);
  return SAC_OK;
}

// the stage form in use: fused (0/1), its tile shape, and the tuner's timings of
// one stage (three passes, fused; 0 before sac_batch_tune)
sac_status sac_batch_join(sac_batch* lead, sac_batch* partner) {
  if (!lead || !partner || lead == partner) return SAC_ERR_ARG;
  if (joined(lead) || joined(partner)) return bfail(lead, SAC_ERR_STATE, "a batch is joined already");
  if (lead->prec != SAC_PREC_FP64 || partner->prec != SAC_PREC_FP32)
    return bfail(lead, SAC_ERR_ARG, "the lead holds FP64 instances and the partner FP32 ones");
  if (!same_family(lead, partner))
    return bfail(lead, SAC_ERR_ARG, "joined batches need the same parameters, ndim, ndir and device");
  if (!fused_ok(lead))
    return bfail(lead, SAC_ERR_UNSUPPORTED,
                 "joined batches run the fused stage: 2D instances without Powell's or the resistive term");
  if (!lead->bc_init || !partner->bc_init)
    return bfail(lead, SAC_ERR_STATE, "call sac_batch_getboundary on both batches first");
  sac_batch* b = lead;  // BK reports on the lead
  BK(cudaSetDevice(lead->dev));
  BK(cudaStreamSynchronize(lead->stream));
  BK(cudaStreamSynchronize(partner->stream));
  const int shape = lead->fused_shape;
  for (sac_batch* x : {lead, partner}) {
    if (!x->fused || x->fused_shape != shape) {
      x->fused = true;
      x->fused_shape = shape;
      sac_status st = build_lists(x);
      if (st != SAC_OK) return bfail(lead, st, x->err);
    }
    drop_exec(x);
  }
  BK(cudaEventCreateWithFlags(&lead->ev_fork, cudaEventDisableTiming));
  BK(cudaEventCreateWithFlags(&lead->ev_join, cudaEventDisableTiming));
  partner->own_stream = partner->stream;
  partner->stream = lead->stream;
  partner->lead = lead;
  lead->partner = partner;
  // time one stage in both forms and keep the faster.  The stage kernels skip
  // instances with dt = 0 (before the first step): time them with a tiny
  // nonzero dt, then restore both instance tables (c_tot and max nu included)
  std::vector<InstDyn> save[2], tmp[2];
  sac_batch* both[2] = {lead, partner};
  for (int k = 0; k < 2; ++k) {
    save[k].resize(both[k]->ninst);
    BK(cudaMemcpy(save[k].data(), both[k]->d_dyn, sizeof(InstDyn) * both[k]->ninst, cudaMemcpyDeviceToHost));
    tmp[k] = save[k];
    for (auto& d : tmp[k])
      if (d.dt == 0.0) d.dt = 1e-300;
    BK(cudaMemcpy(both[k]->d_dyn, tmp[k].data(), sizeof(InstDyn) * both[k]->ninst, cudaMemcpyHostToDevice));
  }
  cudaEvent_t e0, e1;
  BK(cudaEventCreate(&e0));
  BK(cudaEventCreate(&e1));
  for (int f = 0; f < 2; ++f) lead->join_ms[f] = join_stage_ms(lead, partner, f, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  BK(cudaGetLastError());
  for (int k = 0; k < 2; ++k)
    BK(cudaMemcpy(both[k]->d_dyn, save[k].data(), sizeof(InstDyn) * both[k]->ninst, cudaMemcpyHostToDevice));
  lead->join_form = lead->join_ms[1] < lead->join_ms[0] ? 1 : 0;
  return SAC_OK;
}

sac_status sac_batch_set_join_form(sac_batch* lead, int form) {
  if (!lead || form < 0 || form > 1) return SAC_ERR_ARG;
  if (!lead->partner) return bfail(lead, SAC_ERR_STATE, "not the lead of a joined pair");
  lead->join_form = form;
  drop_exec(lead);
  return SAC_OK;
}

sac_status sac_batch_get_join(const sac_batch* lead, int* form, double* ms_joint, double* ms_forked) {
  if (!lead) return SAC_ERR_ARG;
  if (form) *form = lead->partner ? lead->join_form : -1;
  if (ms_joint) *ms_joint = lead->join_ms[0];
  if (ms_forked) *ms_forked = lead->join_ms[1];
  return SAC_OK;
}

sac_status sac_batch_unjoin(sac_batch* lead) {
  if (!lead) return SAC_ERR_ARG;
  if (lead->lead) return bfail(lead, SAC_ERR_STATE, "sac_batch_unjoin takes the FP64 batch of the pair");
  unjoin(lead);
  return SAC_OK;
}

sac_status sac_batch_get_stage(const sac_batch* b, int* fused, int* shape, double* ms_three, double* ms_fused) {
  if (!b) return SAC_ERR_ARG;
  if (fused) *fused = b->fused ? 1 : 0;
  if (shape) *shape = b->fused_shape;
  if (ms_three) *ms_three = b->tune_three_ms;
  if (ms_fused) *ms_fused = b->tune_fused_ms;
  return SAC_OK;
}


// per-instance driver amplitude A and angular frequency omega (tdep = sin(omega t));
// either array may be NULL to keep the current values
sac_status sac_batch_set_driver(sac_batch* b, const double* A, const double* omega) {
  if (!b) return SAC_ERR_ARG;
  if (!b->grid_set) return bfail(b, SAC_ERR_STATE, "sac_batch_set_grid first");
  BK(cudaSetDevice(b->dev));
  std::vector<InstDyn> dyn(b->ninst);
  BK(cudaMemcpyAsync(dyn.data(), b->d_dyn, sizeof(InstDyn) * b->ninst, cudaMemcpyDeviceToHost, b->stream));
  BK(cudaStreamSynchronize(b->stream));
  for (int i = 0; i < b->ninst; ++i) {
    if (A) dyn[i].drvA = A[i];
    if (omega) dyn[i].omega = omega[i];
  }
  BK(cudaMemcpyAsync(b->d_dyn, dyn.data(), sizeof(InstDyn) * b->ninst, cudaMemcpyHostToDevice, b->stream));
  BK(cudaStreamSynchronize(b->stream));
  return SAC_OK;
}

// per-instance time t and step count it (either may be NULL to keep them); a
// step counter of 0 makes the next step the first one (no dtcantgrow bound)
sac_status sac_batch_set_time(sac_batch* b, const double* t, const int* it) {
  if (!b) return SAC_ERR_ARG;
  if (!b->grid_set) return bfail(b, SAC_ERR_STATE, "sac_batch_set_grid first");
  BK(cudaSetDevice(b->dev));
  std::vector<InstDyn> dyn(b->ninst);
  BK(cudaMemcpyAsync(dyn.data(), b->d_dyn, sizeof(InstDyn) * b->ninst, cudaMemcpyDeviceToHost, b->stream));
  BK(cudaStreamSynchronize(b->stream));
  for (int i = 0; i < b->ninst; ++i) {
    if (t) dyn[i].t = t[i];
    if (it) dyn[i].it = it[i];
  }
  BK(cudaMemcpyAsync(b->d_dyn, dyn.data(), sizeof(InstDyn) * b->ninst, cudaMemcpyHostToDevice, b->stream));
  BK(cudaStreamSynchronize(b->stream));
  return SAC_OK;
}

// per-instance end time (tmaxexact): dt is clipped so that the instance lands on
// tmax exactly, after which it takes dt = 0 steps that leave it untouched; a
// value <= 0 removes the limit
sac_status sac_batch_set_tmax(sac_batch* b, const double* tmax) {
  if (!b || !tmax) return SAC_ERR_ARG;
  if (!b->grid_set) return bfail(b, SAC_ERR_STATE, "sac_batch_set_grid first");
  BK(cudaSetDevice(b->dev));
  std::vector<InstDyn> dyn(b->ninst);
  BK(cudaMemcpyAsync(dyn.data(), b->d_dyn, sizeof(InstDyn) * b->ninst, cudaMemcpyDeviceToHost, b->stream));
  BK(cudaStreamSynchronize(b->stream));
  for (int i = 0; i < b->ninst; ++i) dyn[i].tmax = tmax[i];
  BK(cudaMemcpyAsync(b->d_dyn, dyn.data(), sizeof(InstDyn) * b->ninst, cudaMemcpyHostToDevice, b->stream));
  BK(cudaStreamSynchronize(b->stream));
  return SAC_OK;
}

long sac_batch_mesh_cells(const sac_batch* b) { return b ? b->mesh_total : 0; }

static sac_status pack(sac_batch* b, void* dev, int dtype, int dir) {
  if (!b || !dev || dtype < 0 || dtype > 2) return SAC_ERR_ARG;
  if (!b->state_set) return bfail(b, SAC_ERR_STATE, "no state on the device");
  BK(cudaSetDevice(b->dev));
  const unsigned grid = (unsigned)std::min<long>(b->n_cour, 148L * 8);
  auto go = [&](auto S0) {
    using S = decltype(S0);
    S* P0 = (S*)b->P[0];
    if (dtype == SAC_PACK_F32)
      kb_pack<S, float><<<grid, dim3(32, 8), 0, b->stream>>>(b->d_inst, b->d_cour, b->n_cour, b->d_meshoff, P0,
                                                               b->totP, (float*)dev, b->np, dir);
    else if (dtype == SAC_PACK_BF16)
      kb_pack<S, __nv_bfloat16><<<grid, dim3(32, 8), 0, b->stream>>>(
          b->d_inst, b->d_cour, b->n_cour, b->d_meshoff, P0, b->totP, (__nv_bfloat16*)dev, b->np, dir);
    else
      kb_pack<S, double><<<grid, dim3(32, 8), 0, b->stream>>>(b->d_inst, b->d_cour, b->n_cour, b->d_meshoff, P0,
                                                                b->totP, (double*)dev, b->np, dir);
  };
  if (b->prec == SAC_PREC_FP32)
    go(0.0f);
  else
    go(0.0);
  BK(cudaGetLastError());
  return SAC_OK;
}

// the advanced variables on the mesh of every instance to / from a packed
// device buffer (asynchronous on the batch stream)
sac_status sac_batch_gather(sac_batch* b, void* dev, int dtype) { return pack(b, dev, dtype, 0); }
sac_status sac_batch_scatter(sac_batch* b, const void* dev, int dtype) { return pack(b, (void*)dev, dtype, 1); }

}  // extern "C"
