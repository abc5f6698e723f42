// sac_gpu.cu -- libsacgpu.so: the C-ABI of include/sac_gpu.h on sm_100a.
//
// Device state per context; S is the storage type of the advanced variables
// (double, or float for SAC_PREC_FP32):
//   P[4]  advanced blocks (rho, m1.., e, b1..) of w, w1, w2, w3, np*ncell of S
//         each, Fortran layout w(ix1,ix2,ix3,iw) restricted to those variables;
//   BG    the static background block (eb, rhob, bg1..), FP64, shared by all four;
//   D, F, R  per-stage intermediates of S: derived cell fields, fluxes along each
//         dimension, setnu face ratios (sac_stage.cuh);
//   x, dx, 1/dx  grid coordinates and widths (gridsetup1), FP64;
//   fixB  compact ghost slabs of 'fixed'/'fixed1'/'grad1' regions, FP64.
// One RK4 step (typeadvance='fourstep', src/vac.t:439-455) is four
// (k_face, k_nu, k_update, k_bound) sequences; the w1 accumulation and the final
// w+w1 are fused into the k_update stores and the boundary pass.
#include <cuda_runtime.h>

#include <algorithm>
#include <type_traits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "sac_gpu.h"
#include "sac_kernels.cuh"
#include "sac_stage_api.h"
#include "sac_grid.h"

using namespace sacgpu;

namespace {
constexpr double bigdouble = 1.0e99, smalldouble = 1.0e-99;
}

struct sac_ctx {
  sac_params par{};
  std::string err;
  int dev = 0;
  cudaStream_t stream = nullptr;
  Geom g{};
  bool grid_set = false, bc_set = false, state_set = false, bc_init_done = false;
  int fullgridini = 0;
  int prec = SAC_PREC_FP64;
  size_t es = sizeof(double);  // bytes per stored advanced value
  void* P[4] = {nullptr, nullptr, nullptr, nullptr};
  double* BG = nullptr;
  void* D = nullptr;
  void* F = nullptr;
  void* R = nullptr;
  void* X = nullptr;  // cross-derivative half-sums (k_cross), allocated with hyperdiffusion
  double* x = nullptr;
  double* dx = nullptr;
  double* drv = nullptr;
  double* stg = nullptr;  // FP64 staging block for FP32 upload/download
  double drvA = 0.0;
  unsigned long long* red = nullptr;  // 0..2 ctot, 3 maxnu, 4 courant, 5 divb max, 6 divb sq (as double)
  unsigned long long* kp = nullptr;   // keeppositive's words (smallfix only), see k_keeppos_scan
  int it_now = 0;                     // the step number last passed to sac_getdt or sac_advect
  double* fixB = nullptr;
  long fixoff[6] = {0, 0, 0, 0, 0, 0}, slab[6] = {0, 0, 0, 0, 0, 0};
  int8_t* d_type = nullptr;
  int* d_fixed = nullptr;
  std::vector<int8_t> h_type;
  std::vector<int> h_fixed;
  int pairshift[3][2] = {{0, 0}, {0, 0}, {0, 0}};
  int zero1[3][2] = {{0, 0}, {0, 0}, {0, 0}};
  // user boundary regions (&boundlist ixB^LIM): filled one region per launch, in order
  struct Region {
    int lo[3], hi[3];
    int d, up;
    long shift, cells, fixoff;
    bool anyfix;
  };
  bool regions = false;
  int nB = 0;
  std::vector<Region> reg;
  // host-side grid reductions
  double mindx2[3] = {0, 0, 0};  // min over the mesh of dx*dx per dimension
  double mindx_all = 0;          // min over the mesh and all dimensions of dx
  std::vector<double> h_dx;      // for diagnostics
  double dtold = 0, dtgrav = bigdouble;
  int itmin = 0;
  bool itmin_set = false;
  long kernel_launches = 0;
  cudaStream_t own_stream = nullptr;
  // event profiling
  bool prof = false;
  struct Rec {
    int kind;
    cudaEvent_t a, b;
  };
  std::vector<Rec> recs;
  std::vector<cudaEvent_t> pool;
  double prof_ms[SAC_K_COUNT] = {};
  long prof_n[SAC_K_COUNT] = {};
};

namespace {

sac_status fail(sac_ctx* c, sac_status st, const std::string& msg) {
  if (c) c->err = msg;
  return st;
}

#define CK(call)                                                                        \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess)                                                              \
      return fail(c, SAC_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

int np_of(int ndir) { return 2 * ndir + 2; }

cudaEvent_t ev_get(sac_ctx* c) {
  if (!c->pool.empty()) {
    cudaEvent_t e = c->pool.back();
    c->pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}

// Bracket one launch with events when profiling is on.
struct Prof {
  sac_ctx* c;
  int kind;
  cudaEvent_t a = nullptr;
  Prof(sac_ctx* c_, int k) : c(c_), kind(k) {
    c->kernel_launches++;
    if (c->prof) {
      a = ev_get(c);
      cudaEventRecord(a, c->stream);
    }
  }
  ~Prof() {
    if (a) {
      cudaEvent_t b = ev_get(c);
      cudaEventRecord(b, c->stream);
      c->recs.push_back({kind, a, b});
    }
  }
};

void prof_collect(sac_ctx* c) {
  if (c->recs.empty()) return;
  cudaStreamSynchronize(c->stream);
  for (auto& r : c->recs) {
    float ms = 0;
    cudaEventElapsedTime(&ms, r.a, r.b);
    c->prof_ms[r.kind] += ms;
    c->prof_n[r.kind] += 1;
    c->pool.push_back(r.a);
    c->pool.push_back(r.b);
  }
  c->recs.clear();
}

int8_t btype(const std::string& t, bool* ok) {
  *ok = true;
  if (t == "cont") return BT_CONT;
  if (t == "fixed") return BT_FIXED;
  if (t == "cont1") return BT_CONT1;
  if (t == "fixed1") return BT_FIXED1;
  if (t == "grad1") return BT_GRAD1;
  if (t == "periodic") return BT_PERIODIC;
  if (t == "symm") return BT_SYMM;
  if (t == "symm0") return BT_SYMM0;
  if (t == "asymm") return BT_ASYMM;
  if (t == "contCD4") return BT_CONTCD4;
  if (t == "zero") return BT_ZERO;
  *ok = false;
  return BT_CONT;
}

bool visc_on(const sac_ctx* c) {
  if (c->par.user == SAC_USR_SLOG) return true;  // eqpar(nu_)=1.0d0 each call, src/vacusr.f:1280
  if (c->par.user == SAC_USR_NONE) return false;
  return std::fabs(c->par.nu) > smalldouble;
}
bool grav_module(int u) {
  return u == SAC_USR_SLOG || u == SAC_USR_GRAVVISC || u == SAC_USR_STRAT || u == SAC_USR_TUBE;
}

void release(sac_ctx* c) {
  for (auto& p : c->P)
    if (p) cudaFree(p), p = nullptr;
  for (void* p : {(void*)c->BG, c->D, c->F, c->R, c->X, (void*)c->x, (void*)c->dx, (void*)c->drv,
                  (void*)c->stg, (void*)c->red, (void*)c->kp, (void*)c->fixB, (void*)c->d_type,
                  (void*)c->d_fixed})
    if (p) cudaFree(p);
  c->BG = c->x = c->dx = c->drv = c->stg = c->fixB = nullptr;
  c->D = c->F = c->R = c->X = nullptr;
  c->red = c->kp = nullptr;
  c->d_type = nullptr;
  c->d_fixed = nullptr;
}

// --------------------------------------------------------------------------
// launch helpers
// --------------------------------------------------------------------------
BcArgs bc_args(sac_ctx* c, void* A) {
  BcArgs b{};
  b.g = c->g;
  b.A = A;
  b.bgA = c->BG;
  b.type = c->d_type;
  b.fixed = c->d_fixed;
  b.fixB = c->fixB;
  for (int i = 0; i < 6; ++i) {
    b.fixoff[i] = c->fixoff[i];
    b.slab[i] = c->slab[i];
  }
  std::memcpy(b.pairshift, c->pairshift, sizeof(b.pairshift));
  b.fullgridini = c->fullgridini;
  b.sA = b.sB = c->g.ncell;
  b.oA = b.oB = 0;
  return b;
}

RegionArgs region_args(sac_ctx* c, void* A, int iB) {
  const sac_ctx::Region& r = c->reg[iB];
  RegionArgs a{};
  a.g = c->g;
  a.A = A;
  a.bgA = c->BG;
  a.type = c->d_type;
  a.fixed = c->d_fixed;
  a.fixB = r.anyfix ? c->fixB + r.fixoff : nullptr;
  for (int e = 0; e < 3; ++e) {
    a.lo[e] = r.lo[e];
    a.hi[e] = r.hi[e];
  }
  a.shift = r.shift;
  a.cells = r.cells;
  a.d = r.d;
  a.up = r.up;
  a.iB = iB;
  a.nB = c->nB;
  a.fullgridini = c->fullgridini;
  return a;
}

template <typename S>
void launch_bound(sac_ctx* c, const BcArgs& b, int nvar) {
  const Geom& g = c->g;
  if (c->regions) {  // user regions: one pass per region, in the reference's order
    // every variable, background included: a 'zero' variable of any kind converts
    // the whole grid to primitive variables and back around its copy
    const int nv = g.nw;
    auto zero_pass = [&](auto ND) {
      constexpr int NDIR = decltype(ND)::value;
      const unsigned nb = (unsigned)std::min<long>((g.ncell + 255) / 256, 148L * 16);
      Prof pr(c, SAC_K_BOUND);
      k_primitive<NDIR, S><<<nb, 256, 0, c->stream>>>(g, (S*)b.A, c->BG, c->par.gamma);
      return nb;
    };
    auto conserve_pass = [&](auto ND, unsigned nb) {
      constexpr int NDIR = decltype(ND)::value;
      Prof pr(c, SAC_K_BOUND);
      k_conserve<NDIR, S><<<nb, 256, 0, c->stream>>>(g, (S*)b.A, c->BG, c->par.gamma);
    };
    for (int iB = 0; iB < c->nB; ++iB) {
      const RegionArgs a = region_args(c, b.A, iB);
      const unsigned rb = (unsigned)((a.cells + 255) / 256);
      int iw = 0;
      while (iw < nv) {
        int z = iw;  // the next 'zero' variable of this region
        while (z < nv && c->h_type[z * c->nB + iB] != BT_ZERO) ++z;
        if (z > iw) {
          Prof pr(c, SAC_K_BOUND);
          k_bound_region<S><<<rb, 256, 0, c->stream>>>(a, iw, z);
        }
        if (z >= nv) break;
        auto around = [&](auto ND) {
          const unsigned nb = zero_pass(ND);
          {
            Prof pr(c, SAC_K_BOUND);
            k_bound_region<S><<<rb, 256, 0, c->stream>>>(a, z, z + 1);
          }
          conserve_pass(ND, nb);
        };
        if (g.ndir == 1)
          around(std::integral_constant<int, 1>{});
        else if (g.ndir == 2)
          around(std::integral_constant<int, 2>{});
        else
          around(std::integral_constant<int, 3>{});
        iw = z + 1;
      }
    }
    (void)nvar;
    return;
  }
  long ns[3];
  ghost_slabs(g, ns);
  const long tot = ns[0] + ns[1] + ns[2];
  if (tot == 0) return;
  const int bs = 256;
  Prof pr(c, SAC_K_BOUND);
  k_bound<S><<<(unsigned)((tot + bs - 1) / bs), bs, 0, c->stream>>>(b, ns[0], ns[1], ns[2], nvar);
}

sac_status keeppositive(sac_ctx* c, void* A);

// advect1 (src/vac.t:490-549): out = base + qdt R(wct), then getboundary(out)
template <typename S>
sac_status advect1_t(sac_ctx* c, const std::string& method, double qdt, int dmin, int dmax, double qt,
                     const void* wct, const void* base, void* out, unsigned mask, int epi, void* aux1,
                     const void* aux2) {
  const Geom& g = c->g;
  if (method == "cd4" || method == "source") {
    const bool flux = (method == "cd4");
    const int u = c->par.user;
    const bool visc = c->par.sourceunsplit && visc_on(c);
    CK(cudaMemsetAsync(c->red, 0, 3 * sizeof(unsigned long long), c->stream));
    Stage2Args a{};
    a.g = g;
    a.wct = wct;
    a.bgv = c->BG;
    a.base = base;
    a.out = out;
    a.aux1 = aux1;
    a.aux2 = aux2;
    a.D = c->D;
    a.F = c->F;
    a.R = c->R;
    a.X = c->X;
    a.dx = c->dx;
    a.drv = c->drv;
    a.ctot = c->red;
    a.maxnu = c->red + 3;
    a.qdt = qdt;
    // sources inside centdiff4 carry qdt*(idimmax-idimmin+1)/ndim, src/vaccd.t:73-75;
    // advect1 'source' passes qdt unchanged
    a.qdt2 = flux ? qdt * ((double)(dmax - dmin) + 1.0) / (double)g.ndim : qdt;
    a.gamma = c->par.gamma;
    for (int d = 0; d < 3; ++d) a.grav[d] = (d < g.ndim) ? c->par.grav[d] : 0.0;
    if (c->par.alias_nu_grav3 && g.ndim == 3) a.grav[2] = 1.0;
    a.dmin = flux ? dmin : 1;
    a.dmax = flux ? dmax : 0;
    a.iwmask = mask;
    for (int d = 0; d < 3; ++d)
      for (int s2 = 0; s2 < 2; ++s2) a.zero1[d][s2] = c->zero1[d][s2];
    a.grav_on = (c->par.sourceunsplit && grav_module(u)) ? 1 : 0;
    a.visc_on = visc ? 1 : 0;
    // addsource (src/vacphys.mhd0.t:225-258): resistivity when |eta| > smalldouble,
    // Powell's term when divbfix is set, compiled out of 1D builds ({^NOONED}, :255)
    a.res_on = (c->par.sourceunsplit && std::fabs(c->par.eta) > smalldouble) ? 1 : 0;
    a.res_compact = c->par.compactres ? 1 : 0;
    a.eta = c->par.eta;
    a.divb_on = (c->par.sourceunsplit && c->par.divbfix && g.ndim > 1) ? 1 : 0;
    a.driver = DRV_NONE;
    if (c->par.sourceunsplit && c->drv) {
      if (u == SAC_USR_SLOG && g.ndim == 3) {
        a.driver = DRV_SLOG;  // tdep=SIN(qt*2*pi/s_period), src/vacusr.f:1321
        a.tdep = std::sin(qt * 2.0 * (double)3.1415926535897932384626433832795f / 240.0);
      } else if (u == SAC_USR_STRAT || u == SAC_USR_TUBE) {
        a.driver = (u == SAC_USR_STRAT) ? DRV_STRAT : DRV_TUBE;
        a.tdep = std::sin(c->par.userpar[1] * qt);
      }
      a.drvA = c->drvA;
    }
    a.epi = epi;
    {
      Prof pr(c, SAC_K_PREP);
      launch_face<S>(a, visc ? 1 : 0, c->stream);
    }
    if (visc) {
      Prof pr(c, SAC_K_NU);
      launch_nu<S>(a, c->stream);
      if (c->X) launch_cross<S>(a, c->stream);
    }
    {
      Prof pr(c, SAC_K_STAGE);
      launch_update<S>(a, c->stream);
    }
  } else if (base != out) {
    CK(cudaMemcpyAsync(out, base, c->es * g.np * g.ncell, cudaMemcpyDeviceToDevice, c->stream));
  }
  if ((c->par.smallfix || c->regions) && epi != EPI_PLAIN)
    return fail(c, SAC_ERR_STATE, "smallfix and user boundary regions need the unfused Runge-Kutta stages");
  if (c->par.smallfix) {  // getboundary's keeppositive, src/vacgrid.t:220
    sac_status st = keeppositive(c, out);
    if (st != SAC_OK) return st;
  }
  BcArgs b = bc_args(c, out);
  if (epi == EPI_RK4_S3) {
    b.mode = 1;
    b.aux1 = aux1;
    b.aux2 = aux2;
    b.basep = base;
  } else if (epi == EPI_RK4_S4) {
    b.mode = 2;
    b.aux1 = aux1;
  }
  launch_bound<S>(c, b, g.np);
  CK(cudaGetLastError());
  return SAC_OK;
}

sac_status advect1(sac_ctx* c, const std::string& method, double qdt, int dmin, int dmax, double qt, const void* wct,
                   const void* base, void* out, unsigned mask, int epi = EPI_PLAIN, void* aux1 = nullptr,
                   const void* aux2 = nullptr) {
  if (c->prec == SAC_PREC_FP32)
    return advect1_t<float>(c, method, qdt, dmin, dmax, qt, wct, base, out, mask, epi, aux1, aux2);
  return advect1_t<double>(c, method, qdt, dmin, dmax, qt, wct, base, out, mask, epi, aux1, aux2);
}

template <typename S>
__global__ void k_lin_threestep_a(S* w2, const S* w, const S* w1, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    w2[i] = S(3 * 0.25) * w[i] + S(0.25) * w1[i];
}
template <typename S>
__global__ void k_lin_threestep_b(S* w, const S* w2, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    w[i] = w[i] / S(3) + w2[i] * S(2.0 / 3);
}

// The two whole-grid combinations of 'fourstep' (src/vac.t:450,454), for runs
// whose fills change the mesh (keeppositive), so that they cannot be folded into
// the stage stores: w1 = (w1 + 2 w2 + w3 - 4 w)/3, and w = w + w1.
template <typename S>
__global__ void k_rk4_acc(S* w1, const S* w2, const S* w3, const S* w, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    w1[i] = (w1[i] + S(2) * w2[i] + w3[i] - S(4) * w[i]) / S(3);
}
template <typename S>
__global__ void k_rk4_final(S* w, const S* w1, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    w[i] = w[i] + w1[i];
}

// ---------------------------------------------------------------------------
// keeppositive (src/vacphys.t.mhd:8-49) on the mesh of one advanced array, run at
// the start of every boundary fill when smallfix is set (src/vacgrid.t:220).
// kp[0]: a mesh pressure fell below max(0,smallp) in this fill; kp[1]: the
// order key of this fill's minimum pressure; kp[2]: nerror(toosmallp_);
// kp[3], kp[4]: step number and minimum-pressure key of the first error.
// ---------------------------------------------------------------------------
// a 64-bit key whose unsigned order is the order of the doubles (no NaN)
__device__ __forceinline__ unsigned long long order_key(double v) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(v);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
double order_key_value(unsigned long long k) {
  const unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
  double v;
  std::memcpy(&v, &b, sizeof(v));
  return v;
}

// getpthermal (src/vacphys0.t.mhd:163-183) of one cell from its loaded fields
template <int NDIR>
__device__ __forceinline__ double thermal_pressure(const double* m, const double* b, const double* bg, double rho,
                                                   double rhob, double e, double gamma) {
  double m2 = m[0] * m[0], b2 = b[0] * b[0], bb = b[0] * bg[0];
#pragma unroll
  for (int C = 1; C < NDIR; ++C) {
    m2 = m2 + m[C] * m[C];
    b2 = b2 + b[C] * b[C];
    bb = bb + b[C] * bg[C];
  }
  double q = 0.5 * m2 / (rho + rhob);
  q = q + 0.5 * b2 + bb;
  return (gamma - 1.0) * (e - q);
}

struct KeepPar {
  double gamma, smallp, smallrho, vacuumrho;
};

// Pass 1: the vacuum state where rho'+rhob < smallrho (:21-26), then the thermal
// pressure against max(0,smallp) (:29-32); one OR and one minimum per block.
template <int NDIR, typename S>
__global__ void __launch_bounds__(256) k_keeppos_scan(const __grid_constant__ Geom g, S* __restrict__ wp,
                                                      const double* __restrict__ bgv, const KeepPar k,
                                                      unsigned long long* kp) {
  __shared__ unsigned long long sh[8];
  const long N = g.ncell;
  constexpr int E = NDIR + 1;
  const double pfloor = fmax(0.0, k.smallp);
  bool low = false;
  unsigned long long kmin = ~0ull;
  // 32-bit decode: sac_set_grid keeps the grid's cell offsets below 2^31
  const unsigned nm0 = g.hi[0] - g.lo[0] + 1, nm1 = g.hi[1] - g.lo[1] + 1, nm2 = g.hi[2] - g.lo[2] + 1;
  const unsigned tot = nm0 * nm1 * nm2;
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += gridDim.x * blockDim.x) {
    const unsigned q = t / nm0;
    const long c = (g.lo[0] + (long)(t - q * nm0)) + g.st[1] * (g.lo[1] + (long)(q % nm1)) +
                   g.st[2] * (g.lo[2] + (long)(q / nm1));
    const double rhob = bgv[N + c], eb = bgv[c];
    double rho = (double)wp[c], e = (double)wp[E * N + c];
    double m[NDIR], b[NDIR], bg[NDIR];
#pragma unroll
    for (int C = 0; C < NDIR; ++C) {
      m[C] = (double)wp[(1 + C) * N + c];
      b[C] = (double)wp[(E + 1 + C) * N + c];
      bg[C] = bgv[(2 + C) * N + c];
    }
    if (rho + rhob < k.smallrho) {
      double b2 = b[0] * b[0];
#pragma unroll
      for (int C = 1; C < NDIR; ++C) b2 = b2 + b[C] * b[C];
#pragma unroll
      for (int C = 0; C < NDIR; ++C) {
        m[C] = 0.0;
        wp[(1 + C) * N + c] = S(0);
      }
      const S rs = (S)(k.vacuumrho - rhob), es = (S)(k.smallp / (k.gamma - 1.0) + 0.5 * b2 - eb);
      wp[c] = rs;
      wp[E * N + c] = es;
      rho = (double)rs;  // the stored values, which the pressure below reads
      e = (double)es;
    }
    const double p = thermal_pressure<NDIR>(m, b, bg, rho, rhob, e, k.gamma);
    low = low || (p < pfloor);
    if (p == p) kmin = min(kmin, order_key(p));
  }
  low = __syncthreads_or(low) != 0;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) kmin = min(kmin, __shfl_xor_sync(0xffffffffu, kmin, o));
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = kmin;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 1; i < (int)(blockDim.x >> 5); ++i) kmin = min(kmin, sh[i]);
    atomicMin(kp + 1, kmin);
    if (low) atomicOr(kp, 1ull);
  }
}

// Pass 2 (smallp > 0, after an error in this fill): e' rebuilt from max(p,smallp)
// over the whole mesh, the kinetic term over rho' alone as the reference writes
// it (:43-45).  p is recomputed from the same stored fields as pass 1 read.
template <int NDIR, typename S>
__global__ void __launch_bounds__(256) k_keeppos_energy(const __grid_constant__ Geom g, S* __restrict__ wp,
                                                        const double* __restrict__ bgv, const KeepPar k,
                                                        const unsigned long long* kp) {
  if (kp[0] == 0) return;
  const long N = g.ncell;
  constexpr int E = NDIR + 1;
  const unsigned nm0 = g.hi[0] - g.lo[0] + 1, nm1 = g.hi[1] - g.lo[1] + 1, nm2 = g.hi[2] - g.lo[2] + 1;
  const unsigned tot = nm0 * nm1 * nm2;
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += gridDim.x * blockDim.x) {
    const unsigned q = t / nm0;
    const long c = (g.lo[0] + (long)(t - q * nm0)) + g.st[1] * (g.lo[1] + (long)(q % nm1)) +
                   g.st[2] * (g.lo[2] + (long)(q / nm1));
    const double rhob = bgv[N + c], eb = bgv[c];
    const double rho = (double)wp[c], e = (double)wp[E * N + c];
    double m[NDIR], b[NDIR], bg[NDIR];
#pragma unroll
    for (int C = 0; C < NDIR; ++C) {
      m[C] = (double)wp[(1 + C) * N + c];
      b[C] = (double)wp[(E + 1 + C) * N + c];
      bg[C] = bgv[(2 + C) * N + c];
    }
    const double p = thermal_pressure<NDIR>(m, b, bg, rho, rhob, e, k.gamma);
    double m2 = m[0] * m[0], b2 = b[0] * b[0];
#pragma unroll
    for (int C = 1; C < NDIR; ++C) {
      m2 = m2 + m[C] * m[C];
      b2 = b2 + b[C] * b[C];
    }
    wp[E * N + c] = (S)(fmax(p, k.smallp) / (k.gamma - 1.0) + 0.5 * (m2 / rho + b2) - eb);
  }
}

// Pass 3 (one thread): count the error, keep the first one's step and minimum,
// and reset the per-fill words for the next fill.
__global__ void k_keeppos_close(unsigned long long* kp, int it) {
  if (kp[0]) {
    kp[2] += 1;
    if (kp[2] == 1) {
      kp[3] = (unsigned long long)(long long)it;
      kp[4] = kp[1];
    }
  }
  kp[0] = 0;
  kp[1] = ~0ull;
}

// keeppositive on the mesh of the advanced array A, at the start of a fill
sac_status keeppositive(sac_ctx* c, void* A) {
  if (!c->par.smallfix) return SAC_OK;
  if (!c->kp) return fail(c, SAC_ERR_STATE, "smallfix: no error words (sac_set_grid allocates them)");
  const Geom& g = c->g;
  const KeepPar k{c->par.gamma, c->par.smallp, c->par.smallrho, c->par.vacuumrho};
  const long nm = (long)(g.hi[0] - g.lo[0] + 1) * (g.hi[1] - g.lo[1] + 1) * (g.hi[2] - g.lo[2] + 1);
  const int bs = 256;  // k_keeppos_scan reduces over exactly 8 warps
  const unsigned nb = (unsigned)std::min<long>((nm + bs - 1) / bs, 148L * 8);
  const bool energy = c->par.smallp > 0.0;
  auto launch = [&](auto S0, auto ND) {
    using S = decltype(S0);
    constexpr int NDIR = decltype(ND)::value;
    {
      Prof pr(c, SAC_K_OTHER);
      k_keeppos_scan<NDIR, S><<<nb, bs, 0, c->stream>>>(g, (S*)A, c->BG, k, c->kp);
    }
    if (energy) {
      Prof pr(c, SAC_K_OTHER);
      k_keeppos_energy<NDIR, S><<<nb, bs, 0, c->stream>>>(g, (S*)A, c->BG, k, c->kp);
    }
  };
  auto by_ndir = [&](auto S0) {
    switch (g.ndir) {
      case 1: launch(S0, std::integral_constant<int, 1>{}); break;
      case 2: launch(S0, std::integral_constant<int, 2>{}); break;
      default: launch(S0, std::integral_constant<int, 3>{}); break;
    }
  };
  if (c->prec == SAC_PREC_FP32)
    by_ndir(0.0f);
  else
    by_ndir(0.0);
  {
    Prof pr(c, SAC_K_OTHER);
    k_keeppos_close<<<1, 1, 0, c->stream>>>(c->kp, c->it_now);
  }
  CK(cudaGetLastError());
  return SAC_OK;
}

// ---------------------------------------------------------------------------
// getdt_courant with file-scope scratch (sac_getdt_static): a two-pass,
// deterministic block reduction.  Pass 1 writes one partial maximum per block
// of kStaticCellsPerBlock mesh cells; pass 2 reduces the partials into the
// slot after them.  Every slot read is written earlier in the same call, so
// nothing has to start at zero.
// ---------------------------------------------------------------------------
constexpr int kStaticPartials = 8192;
constexpr long kStaticCellsPerBlock = 256L * 16;
constexpr long kStaticMaxCells = kStaticPartials * kStaticCellsPerBlock;  // 33,554,432 mesh cells
static_assert(kStaticMaxCells == SAC_STATIC_MAX_CELLS, "the header states the limit");
__device__ __align__(256) double g_courant_scratch[kStaticPartials + 1];  // partials, then the result

// block max of non-negative values, NaN-sticky; valid in thread 0
__device__ __forceinline__ double block_max_value(double v, double* sh) {
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const bool anynan = __syncthreads_or(v != v);
  v = (v != v) ? 0.0 : v;
  v = warp_max(v);
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double m = 0.0;
  if (tid < 32) {
    m = (tid < (int)(blockDim.x + 31) / 32) ? sh[tid] : 0.0;
    m = warp_max(m);
  }
  return anynan ? __longlong_as_double(0x7ff8000000000000ll) : m;
}

template <int NDIR, typename S>
__global__ void __launch_bounds__(256) k_courant_partial(Geom g, const S* __restrict__ wp,
                                                         const double* __restrict__ bgv,
                                                         const double* __restrict__ dx, double* part,
                                                         double gamma) {
  __shared__ double sh[32];
  const long nm0 = g.hi[0] - g.lo[0] + 1, nm1 = g.hi[1] - g.lo[1] + 1, nm2 = g.hi[2] - g.lo[2] + 1;
  const long tot = nm0 * nm1 * nm2;
  const long t0 = blockIdx.x * kStaticCellsPerBlock;
  const long t1 = t0 + kStaticCellsPerBlock < tot ? t0 + kStaticCellsPerBlock : tot;
  double best = 0.0;
  for (long t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
    const int i0 = g.lo[0] + (int)(t % nm0);
    const int i1 = g.lo[1] + (int)((t / nm0) % nm1);
    const int i2 = g.lo[2] + (int)(t / (nm0 * nm1));
    best = max_sticky(best, courant_cell<NDIR, S>(g, wp, bgv, dx, i0, i1, i2, gamma));
  }
  best = block_max_value(best, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = best;
}

__global__ void __launch_bounds__(1024) k_courant_final(double* part, int n) {
  __shared__ double sh[32];
  double best = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) best = max_sticky(best, part[i]);
  best = block_max_value(best, sh);
  if (threadIdx.x == 0) part[kStaticPartials] = best;
}

// device address of g_courant_scratch per device ordinal, looked up once.  The
// address belongs to the module loaded in the device's primary context; it stays
// valid as long as that context lives (no cudaDeviceReset while the library is
// loaded), which the header states as a condition of sac_getdt_static.
std::mutex g_static_mu;
double* g_static_addr[64] = {};

sac_status static_scratch(sac_ctx* c, double** out) {
  std::lock_guard<std::mutex> lk(g_static_mu);
  if (c->dev < 0 || c->dev >= 64) return fail(c, SAC_ERR_ARG, "device ordinal out of range");
  if (!g_static_addr[c->dev]) {
    void* p = nullptr;
    CK(cudaSetDevice(c->dev));
    CK(cudaGetSymbolAddress(&p, g_courant_scratch));
    g_static_addr[c->dev] = (double*)p;
  }
  *out = g_static_addr[c->dev];
  return SAC_OK;
}

// max over the mesh of cmax/dx into *cm, scratch in g_courant_scratch
sac_status courant_max_static(sac_ctx* c, double* cm) {
  const Geom& g = c->g;
  const long nm = (long)(g.hi[0] - g.lo[0] + 1) * (g.hi[1] - g.lo[1] + 1) * (g.hi[2] - g.lo[2] + 1);
  if (nm > kStaticMaxCells)
    return fail(c, SAC_ERR_UNSUPPORTED,
                "sac_getdt_static: the mesh has " + std::to_string(nm) + " cells, more than the " +
                    std::to_string(kStaticMaxCells) + " its static scratch covers; use sac_getdt");
  double* part = nullptr;
  sac_status st = static_scratch(c, &part);
  if (st != SAC_OK) return st;
  const int nb = (int)((nm + kStaticCellsPerBlock - 1) / kStaticCellsPerBlock);
  auto launch = [&](auto S0) {
    using S = decltype(S0);
    const S* wp = (const S*)c->P[0];
    switch (g.ndir) {
      case 1: k_courant_partial<1, S><<<nb, 256, 0, c->stream>>>(g, wp, c->BG, c->dx, part, c->par.gamma); break;
      case 2: k_courant_partial<2, S><<<nb, 256, 0, c->stream>>>(g, wp, c->BG, c->dx, part, c->par.gamma); break;
      default: k_courant_partial<3, S><<<nb, 256, 0, c->stream>>>(g, wp, c->BG, c->dx, part, c->par.gamma); break;
    }
  };
  {
    Prof pr(c, SAC_K_COURANT);
    if (c->prec == SAC_PREC_FP32)
      launch(0.0f);
    else
      launch(0.0);
  }
  {
    Prof pr(c, SAC_K_COURANT);
    k_courant_final<<<1, 1024, 0, c->stream>>>(part, nb);
  }
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(cm, part + kStaticPartials, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return SAC_OK;
}

}  // namespace

// ==========================================================================
// C-ABI
// ==========================================================================
extern "C" {

void sac_default_params(sac_params* p) {
  std::memset(p, 0, sizeof(*p));
  p->gamma = 5.0 / 3.0;
  p->courantpar = 0.8;  // par/DEFAULT:66
  p->dtpar = -1.0;
  p->dtdiffpar = 0.5;
  std::strcpy(p->typeadvance, "twostep");  // par/DEFAULT:31
  std::strcpy(p->typepred, "nul");
  p->sourceunsplit = 1;  // par/DEFAULT:44
  p->user = SAC_USR_NONE;
  p->precision = SAC_PREC_FP64;
  p->smallp = p->smallrho = p->vacuumrho = -1.0;  // src/vacio.t:99-101; smallfix F, par/DEFAULT:54
}

sac_status sac_create(const sac_params* p, sac_ctx** out) {
  if (!p || !out) return SAC_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return SAC_ERR_NODEVICE;
  if (p->device < 0 || p->device >= ndev) return SAC_ERR_ARG;
  if (p->precision != SAC_PREC_FP64 && p->precision != SAC_PREC_FP32) return SAC_ERR_UNSUPPORTED;
  sac_ctx* c = new sac_ctx();
  c->par = *p;
  c->prec = p->precision;
  c->es = (c->prec == SAC_PREC_FP32) ? sizeof(float) : sizeof(double);
  c->dev = p->device;
  if (cudaSetDevice(c->dev) != cudaSuccess || cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return SAC_ERR_CUDA;
  }
  c->own_stream = c->stream;
  *out = c;
  return SAC_OK;
}

void sac_destroy(sac_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->dev);
  if (c->stream) cudaStreamSynchronize(c->stream);
  release(c);
  for (auto& r : c->recs) {
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  for (auto e : c->pool) cudaEventDestroy(e);
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
  delete c;
}

const char* sac_last_error(const sac_ctx* c) { return c ? c->err.c_str() : "null context"; }

sac_status sac_synchronize(sac_ctx* c) {
  if (!c) return SAC_ERR_ARG;
  CK(cudaSetDevice(c->dev));
  CK(cudaStreamSynchronize(c->stream));
  return SAC_OK;
}

sac_status sac_set_grid(sac_ctx* c, int ndim, int ndir, const int ixGhi[3], const int ixM[6], const double* x,
                        int fullgridini) {
  if (!c || !ixGhi || !ixM || !x) return SAC_ERR_ARG;
  if (ndim < 1 || ndim > 3 || ndir < ndim || ndir > 3) return fail(c, SAC_ERR_ARG, "bad ndim/ndir");
  CK(cudaSetDevice(c->dev));
  release(c);
  Geom& g = c->g;
  g.ndim = ndim;
  g.ndir = ndir;
  g.nw = 3 * ndir + 4;
  g.np = np_of(ndir);
  for (int d = 0; d < 3; ++d) {
    g.n[d] = (d < ndim) ? ixGhi[d] : 1;
    g.lo[d] = (d < ndim) ? ixM[d] - 1 : 0;
    g.hi[d] = (d < ndim) ? ixM[3 + d] - 1 : 0;
    if (d < ndim && (g.lo[d] != 2 || g.hi[d] != g.n[d] - 3 || g.hi[d] < g.lo[d] + 5))
      return fail(c, SAC_ERR_ARG, "mesh must be ixG shrunk by dixB=2 and hold at least 6 cells per dimension");
  }
  g.st[0] = 1;
  g.st[1] = g.n[0];
  g.st[2] = (long)g.n[0] * g.n[1];
  g.ncell = (long)g.n[0] * g.n[1] * g.n[2];
  c->fullgridini = fullgridini ? 1 : 0;
  const long N = g.ncell;
  // gridsetup1 (src/vacgrid.t:585-629): extrapolate x into the ghosts, dx = (x(+1)-x(-1))/2
  std::vector<double> hx, hdx;
  gridsetup1(g.n, g.lo, g.hi, ndim, N, x, c->fullgridini != 0, hx, hdx);
  auto gid = [&](int i, int j, int k) { return i + g.st[1] * j + g.st[2] * k; };
  c->mindx_all = bigdouble;
  for (int d = 0; d < ndim; ++d) {
    double m2 = bigdouble;
    for (int k = g.lo[2]; k <= g.hi[2]; ++k)
      for (int j = g.lo[1]; j <= g.hi[1]; ++j)
        for (int i = g.lo[0]; i <= g.hi[0]; ++i) {
          const double v = hdx[d * N + gid(i, j, k)];
          m2 = std::min(m2, v * v);
          c->mindx_all = std::min(c->mindx_all, v);
        }
    c->mindx2[d] = m2;
  }
  c->h_dx = hdx;
  // cell offsets inside one block of np (or ndir+3) fields are 32-bit
  if ((long)std::max(g.np, ndir + 3) * N > 2147483647L)
    return fail(c, SAC_ERR_UNSUPPORTED, "grid too large for 32-bit in-block indexing");
  // driver spatial profiles (time independent), evaluated with the host libm as the
  // oracle does: Slog vortex (src/vacusr.f:1324-1370) or the Gaussian velocity drivers
  std::vector<double> hdrv;
  const int u = c->par.user;
  if ((u == SAC_USR_SLOG && ndim == 3) || u == SAC_USR_STRAT || (u == SAC_USR_TUBE && ndim >= 2)) {
    hdrv.assign((size_t)2 * N, 0.0);
    const double* up = c->par.userpar;
    for (long q = 0; q < N; ++q) {
      const double x1 = hx[q], x2 = ndim > 1 ? hx[N + q] : 0.0, x3 = ndim > 2 ? hx[2 * N + q] : 0.0;
      if (u == SAC_USR_SLOG) {
        const double xc1 = (double)0.1f * 1.0e6, xc2 = 1.0e6, xc3 = 1.0e6, B = (double)0.05f;
        const double dz = 0.05e6, dxx = 0.5e6, dyy = 0.5e6;
        const double xx = x2 - xc2, yy = x3 - xc3, zz = x1 - xc1;
        const double exz = std::exp(-(zz * zz) / (dz * dz)), exx = std::exp(-(xx * xx) / (dxx * dxx)),
                     exy = std::exp(-(yy * yy) / (dyy * dyy));
        const double exyz = exx * exy * exz;
        const double th = std::atan2(yy, xx), ph = std::atan2(1.0, B);
        const double ux = std::cos(th + ph), uy = std::sin(th + ph);
        hdrv[q] = (ux / std::sqrt(ux * ux + uy * uy)) * exyz;
        hdrv[N + q] = (uy / std::sqrt(ux * ux + uy * uy)) * exyz;
        c->drvA = 10.0;
      } else {
        c->drvA = up[0];
      }
    }
    if (u == SAC_USR_STRAT || u == SAC_USR_TUBE) gauss_driver_profiles(u, ndim, N, hx.data(), up, hdrv.data());
  }
  const size_t bp = c->es * g.np * N;
  for (auto& p : c->P) CK(cudaMalloc(&p, bp));
  CK(cudaMalloc(&c->BG, sizeof(double) * (g.nw - g.np) * N));
  CK(cudaMalloc(&c->D, c->es * (ndir + 3) * N));
  CK(cudaMalloc(&c->F, c->es * (size_t)ndim * g.np * N));
  CK(cudaMalloc(&c->R, c->es * (size_t)nr_pairs(ndim) * N));
  if (visc_on(c) && ndim > 1 && c->prec == SAC_PREC_FP64)  // the FP64 update reads them (k_cross)
    CK(cudaMalloc(&c->X, c->es * (size_t)n_cross(ndim) * N));
  CK(cudaMalloc(&c->x, sizeof(double) * ndim * N));
  CK(cudaMalloc(&c->dx, sizeof(double) * ndim * N));
  if (!hdrv.empty()) CK(cudaMalloc(&c->drv, sizeof(double) * 2 * N));
  if (c->prec == SAC_PREC_FP32) CK(cudaMalloc(&c->stg, sizeof(double) * g.np * N));
  CK(cudaMalloc(&c->red, 8 * sizeof(unsigned long long)));
  CK(cudaMemsetAsync(c->red, 0, 8 * sizeof(unsigned long long), c->stream));
  if (c->par.smallfix) {
    static const unsigned long long kp0[5] = {0, ~0ull, 0, 0, ~0ull};
    CK(cudaMalloc(&c->kp, sizeof(kp0)));
    CK(cudaMemcpyAsync(c->kp, kp0, sizeof(kp0), cudaMemcpyHostToDevice, c->stream));
  }
  CK(cudaMemsetAsync(c->R, 0, c->es * (size_t)nr_pairs(ndim) * N, c->stream));
  CK(cudaMemcpyAsync(c->x, hx.data(), sizeof(double) * ndim * N, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->dx, hdx.data(), sizeof(double) * ndim * N, cudaMemcpyHostToDevice, c->stream));
  if (!hdrv.empty())
    CK(cudaMemcpyAsync(c->drv, hdrv.data(), sizeof(double) * 2 * N, cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->grid_set = true;
  c->bc_set = false;
  c->state_set = false;
  c->bc_init_done = false;
  c->itmin_set = false;
  return SAC_OK;
}

sac_status sac_set_boundaries(sac_ctx* c, int nB, const char* typeB, const int* ixB, const int* idimB,
                              const int* upperB, const int* ipairB) {
  if (!c || !typeB) return SAC_ERR_ARG;
  if (!c->grid_set) return fail(c, SAC_ERR_STATE, "sac_set_grid first");
  const Geom& g = c->g;
  const bool user = ixB != nullptr;
  if (user && (!idimB || !upperB)) return fail(c, SAC_ERR_ARG, "user boundary regions need ixB, idimB and upperB");
  if (nB < 1 || nB > SAC_NHIB) return fail(c, SAC_ERR_ARG, "nB must be 1..nhiB (10)");
  if (!user && nB != 2 * g.ndim) return fail(c, SAC_ERR_ARG, "the default boundary regions are 2*ndim");
  CK(cudaSetDevice(c->dev));
  // the regions, 0-based and inclusive: the default ones (boundsetup, src/vacgrid.t:53-70)
  // or the user's, which must lie inside the grid (:71-99)
  std::vector<sac_ctx::Region> reg((size_t)nB);
  bool is_default = true;
  for (int iB = 0; iB < nB; ++iB) {
    sac_ctx::Region& r = reg[iB];
    r = sac_ctx::Region{};
    const int dd = iB / 2;
    int dlo[3], dhi[3];  // the default region iB (when iB < 2*ndim)
    for (int e = 0; e < 3; ++e) {
      dlo[e] = 0;
      dhi[e] = e < g.ndim ? g.n[e] - 1 : 0;
    }
    if (dd < g.ndim) {
      if (iB % 2) {
        dlo[dd] = g.hi[dd] + 1;
      } else {
        dhi[dd] = g.lo[dd] - 1;
      }
    }
    if (user) {
      r.d = idimB[iB] - 1;
      r.up = upperB[iB] ? 1 : 0;
      if (r.d < 0 || r.d >= g.ndim) return fail(c, SAC_ERR_ARG, "Error in BoundSetup: idimB out of range");
      for (int e = 0; e < 3; ++e) {
        r.lo[e] = e < g.ndim ? ixB[e + g.ndim * iB] - 1 : 0;
        r.hi[e] = e < g.ndim ? ixB[g.ndim * nB + e + g.ndim * iB] - 1 : 0;
        if (e < g.ndim && (r.lo[e] < 0 || r.hi[e] > g.n[e] - 1 || r.lo[e] > r.hi[e]))
          return fail(c, SAC_ERR_ARG, "Error in BoundSetup: Boundary region is outside grid (iB=" +
                                          std::to_string(iB + 1) + ")");
      }
      if (r.up ? r.lo[r.d] <= g.hi[r.d] : r.hi[r.d] >= g.lo[r.d])
        return fail(c, SAC_ERR_UNSUPPORTED, "boundary region " + std::to_string(iB + 1) +
                                                " reaches into the mesh along idimB; regions must lie in the ghost layers");
    } else {
      r.d = dd;
      r.up = iB % 2;
      for (int e = 0; e < 3; ++e) {
        r.lo[e] = dlo[e];
        r.hi[e] = dhi[e];
      }
    }
    bool same = iB < 2 * g.ndim && r.d == dd && r.up == iB % 2;
    for (int e = 0; e < 3 && same; ++e) same = r.lo[e] == dlo[e] && r.hi[e] == dhi[e];
    is_default = is_default && same;
    r.cells = 1;
    for (int e = 0; e < 3; ++e) r.cells *= (long)(r.hi[e] - r.lo[e] + 1);
  }
  is_default = is_default && nB == 2 * g.ndim;
  // gradient4, gradient1 and setnu read the boundary of dimension idim from the regions
  // 2*idim-1 (lower) and 2*idim (upper) (src/vacgrid.t:690-709, src/vacusr.viscosity.t:378-400)
  if (nB < 2 * g.ndim) return fail(c, SAC_ERR_UNSUPPORTED, "fewer regions than 2*ndim");
  for (int iB = 0; iB < 2 * g.ndim; ++iB)
    if (reg[iB].d != iB / 2 || reg[iB].up != iB % 2)
      return fail(c, SAC_ERR_UNSUPPORTED,
                  "regions 2*idim-1 and 2*idim must be the lower and upper boundaries of dimension idim");
  c->h_type.assign((size_t)g.nw * nB, 0);
  c->h_fixed.assign((size_t)g.nw * nB, 0);
  std::vector<std::string> t((size_t)g.nw * nB);
  for (int iB = 0; iB < nB; ++iB)
    for (int iw = 0; iw < g.nw; ++iw) {
      std::string s(typeB + SAC_LENTYPE * ((long)iw + (long)g.nw * iB), SAC_LENTYPE);
      while (!s.empty() && (s.back() == ' ' || s.back() == '\0')) s.pop_back();
      bool ok;
      c->h_type[iw * nB + iB] = btype(s, &ok);
      if (!ok) return fail(c, SAC_ERR_UNSUPPORTED, "boundary type '" + s + "' is not implemented");
      t[iw + (long)g.nw * iB] = s;
    }
  // periodic pairing (src/vacgrid.t:103-120): direction, orientation and extent
  int pair[SAC_NHIB];
  for (int iB = 0; iB < nB; ++iB) pair[iB] = ipairB ? ipairB[iB] - 1 : -1;
  auto same_extent = [&](int iB, int jB) {
    for (int e = 0; e < g.ndim; ++e)
      if (reg[iB].hi[e] - reg[iB].lo[e] != reg[jB].hi[e] - reg[jB].lo[e]) return false;
    return true;
  };
  for (int iB = 0; iB < nB; ++iB)
    if (t[(long)g.nw * iB] == "periodic" && pair[iB] < 0) {
      for (int jB = iB + 1; jB < nB; ++jB)
        if (t[(long)g.nw * jB] == "periodic" && pair[jB] < 0 && reg[jB].d == reg[iB].d &&
            reg[jB].up != reg[iB].up && same_extent(iB, jB)) {
          pair[iB] = jB;
          pair[jB] = iB;
        }
      if (pair[iB] < 0) return fail(c, SAC_ERR_ARG, "Error in BoundSetup: No periodic pair");
    }
  for (int iB = 0; iB < nB; ++iB) {
    if (pair[iB] < 0 || pair[iB] >= nB) continue;
    // source of region iB: its pair moved by dixB along idim (src/vacgrid.t:236-246)
    const sac_ctx::Region& q = reg[pair[iB]];
    long sh = 0;
    for (int e = 0; e < g.ndim; ++e) {
      int se = q.lo[e] - reg[iB].lo[e];
      if (e == reg[iB].d) se += reg[iB].up ? 2 : -2;
      sh += (long)se * g.st[e];
    }
    reg[iB].shift = sh;
  }
  for (int d = 0; d < g.ndim; ++d) {
    const int nm = g.hi[d] - g.lo[d] + 1;
    c->pairshift[d][0] = nm;   // lower ghosts copy ixMmax-1..ixMmax
    c->pairshift[d][1] = -nm;  // upper ghosts copy ixMmin..ixMmin+1
    for (int s = 0; s < 2; ++s) {
      const std::string& t1 = t[(long)g.nw * (2 * d + s)];  // typeB(1,iB)
      c->zero1[d][s] = (t1 != "periodic" && t1 != "mpi") ? 1 : 0;
    }
  }
  // 'zero' converts the whole grid around its copy, which the one-pass resolver
  // cannot express: it takes the region-by-region fill
  bool any_zero = false;
  for (int8_t ty : c->h_type) any_zero = any_zero || ty == BT_ZERO;
  const bool region_mode = !is_default || any_zero;
  // fixB slabs for every region that holds a fixed-type variable: the default
  // regions' slabs are the dixB layers times the full grid across (k_bound), a user
  // region's slab is its own cells
  long off = 0;
  for (int iB = 0; iB < nB; ++iB) {
    long sl;
    if (!region_mode) {
      const int d = iB / 2;
      sl = 2;  // dixB layers
      for (int e = 0; e < g.ndim; ++e)
        if (e != d) sl *= g.n[e];
      if (iB < 6) c->slab[iB] = sl;
    } else {
      sl = reg[iB].cells;
    }
    if (iB < 6) c->fixoff[iB] = off;
    reg[iB].fixoff = off;
    bool any = false;
    for (int iw = 0; iw < g.nw; ++iw) {
      int8_t ty = c->h_type[iw * nB + iB];
      any = any || ty == BT_FIXED || ty == BT_FIXED1 || ty == BT_GRAD1;
    }
    reg[iB].anyfix = any;
    if (any) off += sl * g.nw;
  }
  c->nB = nB;
  c->reg = reg;
  c->regions = region_mode;
  if (c->fixB) cudaFree(c->fixB), c->fixB = nullptr;
  if (c->d_type) cudaFree(c->d_type), c->d_type = nullptr;
  if (c->d_fixed) cudaFree(c->d_fixed), c->d_fixed = nullptr;
  CK(cudaMalloc(&c->fixB, sizeof(double) * std::max(off, 1L)));
  CK(cudaMalloc(&c->d_type, c->h_type.size()));
  CK(cudaMalloc(&c->d_fixed, sizeof(int) * c->h_fixed.size()));
  CK(cudaMemcpy(c->d_type, c->h_type.data(), c->h_type.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_fixed, c->h_fixed.data(), sizeof(int) * c->h_fixed.size(), cudaMemcpyHostToDevice));
  c->bc_set = true;
  c->bc_init_done = false;
  return SAC_OK;
}

sac_status sac_upload(sac_ctx* c, const double* w) {
  if (!c || !w) return SAC_ERR_ARG;
  if (!c->grid_set) return fail(c, SAC_ERR_STATE, "sac_set_grid first");
  CK(cudaSetDevice(c->dev));
  const Geom& g = c->g;
  const long N = g.ncell;
  if (c->prec == SAC_PREC_FP32) {
    CK(cudaMemcpyAsync(c->stg, w, sizeof(double) * g.np * N, cudaMemcpyHostToDevice, c->stream));
    Prof pr(c, SAC_K_OTHER);
    k_convert<float, double><<<592, 256, 0, c->stream>>>((float*)c->P[0], c->stg, (long)g.np * N);
  } else {
    CK(cudaMemcpyAsync(c->P[0], w, sizeof(double) * g.np * N, cudaMemcpyHostToDevice, c->stream));
  }
  CK(cudaMemcpyAsync(c->BG, w + (long)g.np * N, sizeof(double) * (g.nw - g.np) * N, cudaMemcpyHostToDevice,
                     c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->state_set = true;
  return SAC_OK;
}

sac_status sac_download(sac_ctx* c, double* w) {
  if (!c || !w) return SAC_ERR_ARG;
  if (!c->state_set) return fail(c, SAC_ERR_STATE, "no state on the device");
  CK(cudaSetDevice(c->dev));
  const Geom& g = c->g;
  const long N = g.ncell;
  if (c->prec == SAC_PREC_FP32) {
    {
      Prof pr(c, SAC_K_OTHER);
      k_convert<double, float><<<592, 256, 0, c->stream>>>(c->stg, (const float*)c->P[0], (long)g.np * N);
    }
    CK(cudaMemcpyAsync(w, c->stg, sizeof(double) * g.np * N, cudaMemcpyDeviceToHost, c->stream));
  } else {
    CK(cudaMemcpyAsync(w, c->P[0], sizeof(double) * g.np * N, cudaMemcpyDeviceToHost, c->stream));
  }
  CK(cudaMemcpyAsync(w + (long)g.np * N, c->BG, sizeof(double) * (g.nw - g.np) * N, cudaMemcpyDeviceToHost,
                     c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return SAC_OK;
}

// getboundary(t,1,nw,1,ndim,w) on the resident state; the first call captures fixB.
sac_status sac_getboundary(sac_ctx* c, double t) {
  (void)t;
  if (!c) return SAC_ERR_ARG;
  if (!c->state_set || !c->bc_set) return fail(c, SAC_ERR_STATE, "state and boundaries must be set");
  CK(cudaSetDevice(c->dev));
  const Geom& g = c->g;
  sac_status st = keeppositive(c, c->P[0]);  // src/vacgrid.t:220
  if (st != SAC_OK) return st;
  BcArgs b = bc_args(c, c->P[0]);
  b.init = c->bc_init_done ? 0 : 1;
  if (c->prec == SAC_PREC_FP32)
    launch_bound<float>(c, b, g.nw);
  else
    launch_bound<double>(c, b, g.nw);
  if (!c->bc_init_done) {
    const int nB = c->nB;
    for (int iB = 0; iB < nB; ++iB)
      for (int iw = 0; iw < g.nw; ++iw) {
        const int8_t ty = c->h_type[iw * nB + iB];
        if ((ty == BT_FIXED || ty == BT_FIXED1 || ty == BT_GRAD1) && !c->h_fixed[iw * nB + iB]) {
          const int bs = 256;
          Prof pr(c, SAC_K_OTHER);
          if (c->regions) {
            RegionArgs a = region_args(c, c->P[0], iB);
            const unsigned nb = (unsigned)((a.cells + bs - 1) / bs);
            if (c->prec == SAC_PREC_FP32)
              k_fixcapture_region<float><<<nb, bs, 0, c->stream>>>(a, c->fixB + c->reg[iB].fixoff, iw,
                                                                   ty == BT_GRAD1 ? 1 : 0);
            else
              k_fixcapture_region<double><<<nb, bs, 0, c->stream>>>(a, c->fixB + c->reg[iB].fixoff, iw,
                                                                    ty == BT_GRAD1 ? 1 : 0);
            c->h_fixed[iw * nB + iB] = 1;
            continue;
          }
          const unsigned nb = (unsigned)((c->slab[iB] + bs - 1) / bs);
          if (c->prec == SAC_PREC_FP32)
            k_fixcapture<float><<<nb, bs, 0, c->stream>>>(g, (const float*)c->P[0], c->BG, c->fixB, c->fixoff[iB],
                                                          c->slab[iB], iw, iB / 2, iB % 2, ty == BT_GRAD1 ? 1 : 0);
          else
            k_fixcapture<double><<<nb, bs, 0, c->stream>>>(g, (const double*)c->P[0], c->BG, c->fixB,
                                                           c->fixoff[iB], c->slab[iB], iw, iB / 2, iB % 2,
                                                           ty == BT_GRAD1 ? 1 : 0);
          c->h_fixed[iw * nB + iB] = 1;
        }
      }
    CK(cudaMemcpyAsync(c->d_fixed, c->h_fixed.data(), sizeof(int) * c->h_fixed.size(), cudaMemcpyHostToDevice,
                       c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->bc_init_done = true;
  }
  CK(cudaGetLastError());
  return SAC_OK;
}

// the dt block of program vac, src/vac.t:61-70
static sac_status getdt_impl(sac_ctx* c, double* dt, int it, bool static_scratch_courant) {
  if (!c || !dt) return SAC_ERR_ARG;
  if (!c->state_set || !c->bc_set) return fail(c, SAC_ERR_STATE, "state and boundaries must be set");
  CK(cudaSetDevice(c->dev));
  if (!c->itmin_set) {
    c->itmin = it;
    c->itmin_set = true;
  }
  c->it_now = it;
  const Geom& g = c->g;
  double d;
  if (c->par.dtpar > 0.0) {
    d = c->par.dtpar;
  } else {
    d = bigdouble;
    if (c->par.courantpar > 0.0 && static_scratch_courant) {  // getdt_courant, src/vac.t:641-699
      double courantmax = 0.0;
      sac_status st = courant_max_static(c, &courantmax);
      if (st != SAC_OK) return st;
      if (!(courantmax == courantmax) || std::isinf(courantmax))
        return fail(c, SAC_ERR_NONFINITE, "non-finite wave speed in getdt_courant");
      if (courantmax > smalldouble) d = std::min(d, c->par.courantpar / courantmax);
    } else if (c->par.courantpar > 0.0) {  // getdt_courant, src/vac.t:641-699
      CK(cudaMemsetAsync(c->red + 4, 0, sizeof(unsigned long long), c->stream));
      const long nm = (long)(g.hi[0] - g.lo[0] + 1) * (g.hi[1] - g.lo[1] + 1) * (g.hi[2] - g.lo[2] + 1);
      const int bs = 256;
      const unsigned nb = (unsigned)std::min<long>((nm + bs - 1) / bs, 148L * 16);
      {
      Prof pr(c, SAC_K_COURANT);
      auto launch = [&](auto S0) {
        using S = decltype(S0);
        const S* wp = (const S*)c->P[0];
        switch (g.ndir) {
          case 1: k_courant<1, S><<<nb, bs, 0, c->stream>>>(g, wp, c->BG, c->dx, c->red + 4, c->par.gamma); break;
          case 2: k_courant<2, S><<<nb, bs, 0, c->stream>>>(g, wp, c->BG, c->dx, c->red + 4, c->par.gamma); break;
          default: k_courant<3, S><<<nb, bs, 0, c->stream>>>(g, wp, c->BG, c->dx, c->red + 4, c->par.gamma); break;
        }
      };
      if (c->prec == SAC_PREC_FP32)
        launch(0.0f);
      else
        launch(0.0);
      }
      unsigned long long bits = 0;
      CK(cudaMemcpyAsync(&bits, c->red + 4, sizeof(bits), cudaMemcpyDeviceToHost, c->stream));
      CK(cudaStreamSynchronize(c->stream));
      double courantmax;
      std::memcpy(&courantmax, &bits, sizeof(double));
      if (!(courantmax == courantmax) || std::isinf(courantmax))
        return fail(c, SAC_ERR_NONFINITE, "non-finite wave speed in getdt_courant");
      if (courantmax > smalldouble) d = std::min(d, c->par.courantpar / courantmax);
    }
    if (c->par.eta < 0.0) return fail(c, SAC_ERR_UNSUPPORTED, "eta < 0 needs a user specialeta");
    // getdt_res, src/vacphys.mhdres.t:5-45: dtdiffpar*minval(dx(ixM,1:ndim))**2/eta,
    // with dtdiffpar as getdt_visc may have overwritten it at an earlier call
    if (c->par.eta > 0.0) d = std::min(d, c->par.dtdiffpar * (c->mindx_all * c->mindx_all) / c->par.eta);
    const int u = c->par.user;
    if (grav_module(u)) {  // getdt_special of the Slog/gravity user files
      if (visc_on(c)) {    // getdt_visc, src/vacusr.viscosity.t:509-542
        unsigned long long bits = 0;
        CK(cudaMemcpyAsync(&bits, c->red + 3, sizeof(bits), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        double maxviscoef;
        std::memcpy(&maxviscoef, &bits, sizeof(double));
        if (!(maxviscoef == maxviscoef)) return fail(c, SAC_ERR_NONFINITE, "non-finite hyperdiffusion coefficient");
        c->par.dtdiffpar = 0.25;
        for (int dd = 0; dd < g.ndim; ++dd) {
          const double m = (maxviscoef + 0.0) / c->mindx2[dd];  // = max over the mesh of (maxviscoef/dx^2)
          d = std::min(d, c->par.dtdiffpar / m);
        }
        CK(cudaMemsetAsync(c->red + 3, 0, sizeof(unsigned long long), c->stream));
      }
      // getdt_grav, src/vacusr.gravity.t:97-138 (evaluated at it==itmin only)
      if (it == c->itmin) {
        c->dtgrav = bigdouble;
        for (int dd = 0; dd < g.ndim; ++dd)
          if (std::fabs(c->par.grav[dd]) > 0.0)
            c->dtgrav = std::min(c->dtgrav, 1.0 / std::sqrt(std::fabs(c->par.grav[dd]) / c->mindx_all));
      }
      d = std::min(d, c->dtgrav);
    }
    if (c->par.dtcantgrow && it > c->itmin) d = std::min(d, c->dtold);
    c->dtold = d;
  }
  *dt = d;
  return SAC_OK;
}

sac_status sac_getdt(sac_ctx* c, double* dt, int it) { return getdt_impl(c, dt, it, false); }

sac_status sac_getdt_static(sac_ctx* c, double* dt, int it) { return getdt_impl(c, dt, it, true); }

sac_status sac_advect(sac_ctx* c, const char* method, const int* iws, int idimmin, int idimmax, double dt, double t,
                      int it) {
  if (!c || !method) return SAC_ERR_ARG;
  if (!c->state_set || !c->bc_set) return fail(c, SAC_ERR_STATE, "state and boundaries must be set");
  if (!c->bc_init_done) return fail(c, SAC_ERR_STATE, "call sac_getboundary once before the first advect");
  CK(cudaSetDevice(c->dev));
  const Geom& g = c->g;
  std::string m(method);
  while (!m.empty() && (m.back() == ' ' || m.back() == '\0')) m.pop_back();
  if (m != "cd4" && m != "source" && m != "nul") return fail(c, SAC_ERR_UNSUPPORTED, "method " + m);
  if (idimmin < 1 || idimmax > g.ndim || idimmin > idimmax) return fail(c, SAC_ERR_ARG, "idim range");
  if (c->par.eta < -smalldouble) return fail(c, SAC_ERR_UNSUPPORTED, "eta < 0 needs a user specialeta");
  unsigned mask = 0;
  if (iws) {
    const int n = iws[g.nw];
    for (int i = 0; i < n; ++i) {
      const int iw = iws[i] - 1;
      if (iw < 0 || iw >= g.nw) return fail(c, SAC_ERR_ARG, "iws entry out of range");
      if (iw < g.np) mask |= 1u << iw;
    }
  } else {
    mask = (1u << g.np) - 1u;
  }
  c->it_now = it;
  const int dmin = idimmin - 1, dmax = idimmax - 1;
  void *w = c->P[0], *w1 = c->P[1], *w2 = c->P[2], *w3 = c->P[3];
  const size_t bytes = c->es * g.np * g.ncell;
  const std::string ta(c->par.typeadvance);
  sac_status st = SAC_OK;
#define RUN(x)                    \
  do {                            \
    st = (x);                     \
    if (st != SAC_OK) return st;  \
  } while (0)
  if (ta == "fourstep" && (c->par.smallfix || c->regions)) {
    // keeppositive changes the mesh of w3 and of w at their fills, before the
    // combinations read them, and user regions fill region by region: the
    // combinations run as passes of their own, as src/vac.t:450,454 write them
    const long n = (long)g.np * g.ncell;
    RUN(advect1(c, m, dt / 2, dmin, dmax, t, w, w, w1, mask));
    RUN(advect1(c, m, dt / 2, dmin, dmax, t, w1, w, w2, mask));
    RUN(advect1(c, m, dt, dmin, dmax, t, w2, w, w3, mask));
    {
      Prof pr(c, SAC_K_OTHER);
      if (c->prec == SAC_PREC_FP32)
        k_rk4_acc<float><<<592, 256, 0, c->stream>>>((float*)w1, (const float*)w2, (const float*)w3,
                                                     (const float*)w, n);
      else
        k_rk4_acc<double><<<592, 256, 0, c->stream>>>((double*)w1, (const double*)w2, (const double*)w3,
                                                      (const double*)w, n);
    }
    RUN(advect1(c, m, dt / 6, dmin, dmax, t, w3, w, w, mask));
    {
      Prof pr(c, SAC_K_OTHER);
      if (c->prec == SAC_PREC_FP32)
        k_rk4_final<float><<<592, 256, 0, c->stream>>>((float*)w, (const float*)w1, n);
      else
        k_rk4_final<double><<<592, 256, 0, c->stream>>>((double*)w, (const double*)w1, n);
    }
  } else if (ta == "fourstep") {
    RUN(advect1(c, m, dt / 2, dmin, dmax, t, w, w, w1, mask));
    RUN(advect1(c, m, dt / 2, dmin, dmax, t, w1, w, w2, mask));
    RUN(advect1(c, m, dt, dmin, dmax, t, w2, w, w3, mask, EPI_RK4_S3, w1, w2));
    RUN(advect1(c, m, dt / 6, dmin, dmax, t, w3, w, w, mask, EPI_RK4_S4, w1));
  } else if (ta == "onestep") {
    CK(cudaMemcpyAsync(w1, w, bytes, cudaMemcpyDeviceToDevice, c->stream));
    RUN(advect1(c, m, dt, dmin, dmax, t, w1, w, w, mask));
  } else if (ta == "twostep") {
    const std::string pred(c->par.typepred);
    CK(cudaMemcpyAsync(w1, w, bytes, cudaMemcpyDeviceToDevice, c->stream));
    RUN(advect1(c, pred, dt / 2, dmin, dmax, t, w, w1, w1, mask));
    RUN(advect1(c, m, dt, dmin, dmax, t, w1, w, w, mask));
  } else if (ta == "threestep") {
    const long n = (long)g.np * g.ncell;
    CK(cudaMemcpyAsync(w1, w, bytes, cudaMemcpyDeviceToDevice, c->stream));
    RUN(advect1(c, m, dt, dmin, dmax, t, w, w1, w1, mask));
    {
      Prof pr(c, SAC_K_OTHER);
      if (c->prec == SAC_PREC_FP32)
        k_lin_threestep_a<float><<<592, 256, 0, c->stream>>>((float*)w2, (const float*)w, (const float*)w1, n);
      else
        k_lin_threestep_a<double><<<592, 256, 0, c->stream>>>((double*)w2, (const double*)w, (const double*)w1, n);
    }
    RUN(advect1(c, m, dt / 4, dmin, dmax, t + dt / 4, w1, w2, w2, mask));
    {
      Prof pr(c, SAC_K_OTHER);
      if (c->prec == SAC_PREC_FP32)
        k_lin_threestep_b<float><<<592, 256, 0, c->stream>>>((float*)w, (const float*)w2, n);
      else
        k_lin_threestep_b<double><<<592, 256, 0, c->stream>>>((double*)w, (const double*)w2, n);
    }
    RUN(advect1(c, m, dt * 2.0 / 3, dmin, dmax, t + dt / 3, w2, w, w, mask));
  } else if (ta == "sterck") {
    const double c012 = (double)0.12f;  // default-real literal in src/vac.t:459
    CK(cudaMemcpyAsync(w1, w, bytes, cudaMemcpyDeviceToDevice, c->stream));
    RUN(advect1(c, m, dt * c012, dmin, dmax, t, w, w1, w1, mask));
    CK(cudaMemcpyAsync(w2, w, bytes, cudaMemcpyDeviceToDevice, c->stream));
    RUN(advect1(c, m, dt / 4, dmin, dmax, t, w1, w2, w2, mask));
    CK(cudaMemcpyAsync(w1, w, bytes, cudaMemcpyDeviceToDevice, c->stream));
    RUN(advect1(c, m, dt / 2, dmin, dmax, t, w2, w1, w1, mask));
    RUN(advect1(c, m, dt, dmin, dmax, t, w1, w, w, mask));
  } else if (ta == "jameson") {
    CK(cudaMemcpyAsync(w1, w, bytes, cudaMemcpyDeviceToDevice, c->stream));
    RUN(advect1(c, m, dt / 4, dmin, dmax, t, w, w1, w1, mask));
    CK(cudaMemcpyAsync(w2, w, bytes, cudaMemcpyDeviceToDevice, c->stream));
    RUN(advect1(c, m, dt / 3, dmin, dmax, t, w1, w2, w2, mask));
    CK(cudaMemcpyAsync(w1, w, bytes, cudaMemcpyDeviceToDevice, c->stream));
    RUN(advect1(c, m, dt / 2, dmin, dmax, t, w2, w1, w1, mask));
    RUN(advect1(c, m, dt, dmin, dmax, t, w1, w, w, mask));
  } else {
    return fail(c, SAC_ERR_UNSUPPORTED, "typeadvance=" + ta);
  }
#undef RUN
  CK(cudaGetLastError());
  return SAC_OK;
}

sac_status sac_diag(sac_ctx* c, sac_diag_out* out) {
  if (!c || !out) return SAC_ERR_ARG;
  if (!c->state_set) return fail(c, SAC_ERR_STATE, "no state on the device");
  CK(cudaSetDevice(c->dev));
  const Geom& g = c->g;
  const long N = g.ncell;
  std::vector<double> w((size_t)g.nw * N);
  sac_status st = sac_download(c, w.data());
  if (st != SAC_OK) return st;
  std::memset(out, 0, sizeof(*out));
  auto dxv = [&](int d, long cc) { return c->h_dx[(size_t)d * N + cc]; };
  double volume = 0;
  std::vector<double> dvol(N, 1.0);
  for (long cc = 0; cc < N; ++cc) {
    double v = 1.0;
    for (int d = 0; d < g.ndim; ++d) v = v * dxv(d, cc);
    dvol[cc] = v;
  }
  auto mesh = [&](auto f) {
    for (int k = g.lo[2]; k <= g.hi[2]; ++k)
      for (int j = g.lo[1]; j <= g.hi[1]; ++j)
        for (int i = g.lo[0]; i <= g.hi[0]; ++i) f(i, j, k, i + g.st[1] * j + g.st[2] * k);
  };
  mesh([&](int, int, int, long cc) { volume += dvol[cc]; });
  for (int iw = 0; iw < g.nw && iw < SAC_NWMAX; ++iw) {
    double s = 0;
    mesh([&](int, int, int, long cc) { s += dvol[cc] * w[(size_t)iw * N + cc]; });
    out->wmean[iw] = s / volume;
  }
  double s2 = 0, mx = 0;
  long n = 0;
  int nonfinite = 0;
  mesh([&](int i, int j, int k, long cc) {
    int p[3] = {i, j, k};
    double divb = 0;
    for (int d = 0; d < g.ndim; ++d) {
      if (p[d] <= g.lo[d] + 1 || p[d] >= g.hi[d] - 1) continue;  // gradient4 edge zeroing
      const long s = g.st[d];
      auto B = [&](long q) { return w[(size_t)(g.ndir + 2 + d) * N + q] + w[(size_t)(g.np + 2 + d) * N + q]; };
      divb = divb + -(B(cc + 2 * s) - 8.0 * (B(cc + s) - B(cc - s)) - B(cc - 2 * s)) / dxv(d, cc) / 12.0;
    }
    s2 += divb * divb;
    mx = std::max(mx, std::fabs(divb));
    ++n;
    for (int iw = 0; iw < g.nw; ++iw)
      if (!std::isfinite(w[(size_t)iw * N + cc])) nonfinite = 1;
  });
  out->divb_l2 = std::sqrt(s2 / (double)n);
  out->divb_linf = mx;
  unsigned long long bits[8];
  CK(cudaMemcpy(bits, c->red, sizeof(bits), cudaMemcpyDeviceToHost));
  std::memcpy(&out->maxviscoef, &bits[3], sizeof(double));
  for (int d = 0; d < 3; ++d) std::memcpy(&out->ctot[d], &bits[d], sizeof(double));
  out->nonfinite = nonfinite;
  if (c->kp) {
    unsigned long long kp[5];
    CK(cudaMemcpy(kp, c->kp, sizeof(kp), cudaMemcpyDeviceToHost));
    out->nerror_toosmallp = (int)kp[2];
    out->toosmallp_it = (int)(long long)kp[3];
    out->toosmallp_min = kp[2] ? order_key_value(kp[4]) : 0.0;
  }
  return SAC_OK;
}

// Number of kernels this library launched on the context (benchmark accounting).
long sac_kernel_launches(const sac_ctx* c) { return c ? c->kernel_launches : 0; }

sac_status sac_set_stream(sac_ctx* c, void* stream) {
  if (!c) return SAC_ERR_ARG;
  CK(cudaSetDevice(c->dev));
  CK(cudaStreamSynchronize(c->stream));
  prof_collect(c);
  c->stream = stream ? (cudaStream_t)stream : c->own_stream;
  return SAC_OK;
}

void* sac_get_stream(const sac_ctx* c) { return c ? (void*)c->stream : nullptr; }

sac_status sac_profile(sac_ctx* c, int enable) {
  if (!c) return SAC_ERR_ARG;
  CK(cudaSetDevice(c->dev));
  prof_collect(c);
  c->prof = enable != 0;
  return SAC_OK;
}

sac_status sac_profile_read(sac_ctx* c, int kernel, double* total_ms, long* launches, int reset) {
  if (!c || kernel < 0 || kernel >= SAC_K_COUNT) return SAC_ERR_ARG;
  CK(cudaSetDevice(c->dev));
  prof_collect(c);
  if (total_ms) *total_ms = c->prof_ms[kernel];
  if (launches) *launches = c->prof_n[kernel];
  if (reset) {
    c->prof_ms[kernel] = 0;
    c->prof_n[kernel] = 0;
  }
  return SAC_OK;
}

}  // extern "C"
