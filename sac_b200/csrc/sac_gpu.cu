// sac_gpu.cu -- libsacgpu.so: the C-ABI of include/sac_gpu.h on sm_100a.
//
// Device state per context (all FP64 in this path):
//   P[4]  perturbed blocks (rho, m1.., e, b1..) of w, w1, w2, w3, np*ncell each,
//         Fortran layout w(ix1,ix2,ix3,iw) restricted to the advanced variables;
//   BG    the static background block (eb, rhob, bg1..), shared by all four;
//   D     derived per-cell fields of the current stage input (k_prep);
//   x, dx grid coordinates and cell widths (gridsetup1);
//   fixB  compact ghost slabs of 'fixed'/'fixed1'/'grad1' regions.
// One RK4 step (typeadvance='fourstep', src/vac.t:439-455) is four (prep, stage,
// boundary) triples; the w1 accumulation and the final w+w1 are fused into the
// stage stores and the boundary pass.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "sac_gpu.h"
#include "sac_kernels.cuh"

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
  double* P[4] = {nullptr, nullptr, nullptr, nullptr};
  double* BG = nullptr;
  double* D = nullptr;
  double* x = nullptr;
  double* dx = nullptr;
  unsigned long long* red = nullptr;  // 0..2 ctot, 3 maxnu, 4 courant, 5 divb max, 6 divb sq (as double)
  double* fixB = nullptr;
  long fixoff[6] = {0, 0, 0, 0, 0, 0}, slab[6] = {0, 0, 0, 0, 0, 0};
  int8_t* d_type = nullptr;
  int* d_fixed = nullptr;
  std::vector<int8_t> h_type;
  std::vector<int> h_fixed;
  int pairshift[3][2] = {{0, 0}, {0, 0}, {0, 0}};
  int zero1[3][2] = {{0, 0}, {0, 0}, {0, 0}};
  // host-side grid reductions
  double mindx2[3] = {0, 0, 0};  // min over the mesh of dx*dx per dimension
  double mindx_all = 0;          // min over the mesh and all dimensions of dx
  std::vector<double> h_dx;      // for diagnostics
  double dtold = 0, dtgrav = bigdouble;
  int itmin = 0;
  bool itmin_set = false;
  long kernel_launches = 0;
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
  for (void* p : {(void*)c->BG, (void*)c->D, (void*)c->x, (void*)c->dx, (void*)c->red, (void*)c->fixB,
                  (void*)c->d_type, (void*)c->d_fixed})
    if (p) cudaFree(p);
  c->BG = c->D = c->x = c->dx = c->fixB = nullptr;
  c->red = nullptr;
  c->d_type = nullptr;
  c->d_fixed = nullptr;
}

// --------------------------------------------------------------------------
// launch helpers
// --------------------------------------------------------------------------
template <int NDIR>
void launch_prep_t(sac_ctx* c, const double* wp) {
  const long N = c->g.ncell;
  const int bs = 256;
  k_prep<NDIR><<<(unsigned)((N + bs - 1) / bs), bs, 0, c->stream>>>(c->g, wp, c->BG, c->D, c->red, c->par.gamma,
                                                                    c->g.ndim);
}

void launch_prep(sac_ctx* c, const double* wp) {
  switch (c->g.ndir) {
    case 1: launch_prep_t<1>(c, wp); break;
    case 2: launch_prep_t<2>(c, wp); break;
    default: launch_prep_t<3>(c, wp); break;
  }
  c->kernel_launches++;
}

template <int NDIM, int NDIR>
void launch_stage_t(sac_ctx* c, const StageArgs& a) {
  dim3 blk, grd;
  const int n0 = a.g.hi[0] - a.g.lo[0] + 1, n1 = a.g.hi[1] - a.g.lo[1] + 1, n2 = a.g.hi[2] - a.g.lo[2] + 1;
  if (NDIM == 1)
    blk = dim3(128, 1, 1);
  else if (NDIM == 2)
    blk = dim3(32, 4, 1);
  else
    blk = dim3(32, 2, 2);
  grd = dim3((n0 + blk.x - 1) / blk.x, (n1 + blk.y - 1) / blk.y, (n2 + blk.z - 1) / blk.z);
  k_stage<NDIM, NDIR><<<grd, blk, 0, c->stream>>>(a);
}

void launch_stage(sac_ctx* c, const StageArgs& a) {
  const int nd = c->g.ndim, nr = c->g.ndir;
  if (nd == 1 && nr == 1) launch_stage_t<1, 1>(c, a);
  else if (nd == 1 && nr == 2) launch_stage_t<1, 2>(c, a);
  else if (nd == 1 && nr == 3) launch_stage_t<1, 3>(c, a);
  else if (nd == 2 && nr == 2) launch_stage_t<2, 2>(c, a);
  else if (nd == 2 && nr == 3) launch_stage_t<2, 3>(c, a);
  else launch_stage_t<3, 3>(c, a);
  c->kernel_launches++;
}

BcArgs bc_args(sac_ctx* c, double* A) {
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
  return b;
}

void launch_bound(sac_ctx* c, const BcArgs& b, int nvar) {
  const Geom& g = c->g;
  long ns[3] = {0, 0, 0};
  for (int d = 0; d < g.ndim; ++d) {
    long n = 2L * g.lo[d];
    for (int e = 0; e < g.ndim; ++e) {
      if (e < d) n *= g.n[e];
      if (e > d) n *= (g.hi[e] - g.lo[e] + 1);
    }
    ns[d] = n;
  }
  const long tot = ns[0] + ns[1] + ns[2];
  if (tot == 0) return;
  const int bs = 256;
  k_bound<<<(unsigned)((tot + bs - 1) / bs), bs, 0, c->stream>>>(b, ns[0], ns[1], ns[2], nvar);
  c->kernel_launches++;
}

StageArgs stage_args(sac_ctx* c, double qdt, int dmin, int dmax, bool flux_on, double qt, const double* wct,
                     const double* base, double* out, unsigned mask) {
  StageArgs a{};
  a.g = c->g;
  a.wct_p = wct;
  a.bgv = c->BG;
  a.base = base;
  a.out = out;
  a.D = c->D;
  a.dx = c->dx;
  a.x = c->x;
  a.ctot = c->red;
  a.maxnu = c->red + 3;
  a.qdt = qdt;
  // sources in centdiff4 carry qdt*(idimmax-idimmin+1)/ndim, src/vaccd.t:73-75;
  // advect1 'source' passes qdt unchanged
  a.qdt2 = flux_on ? qdt * ((double)(dmax - dmin) + 1.0) / (double)c->g.ndim : qdt;
  a.gamma = c->par.gamma;
  a.t = qt;
  for (int d = 0; d < 3; ++d) a.grav[d] = (d < c->g.ndim) ? c->par.grav[d] : 0.0;
  if (c->par.alias_nu_grav3 && c->g.ndim == 3) a.grav[2] = 1.0;
  std::memcpy(a.up, c->par.userpar, sizeof(a.up));
  a.dmin = flux_on ? dmin : 1;
  a.dmax = flux_on ? dmax : 0;
  a.iwmask = mask;
  for (int d = 0; d < 3; ++d)
    for (int s = 0; s < 2; ++s) {
      a.zero4[d][s] = (d < c->g.ndim) ? 1 : 0;  // single device: no 'mpi' boundaries
      a.mirror[d][s] = (d < c->g.ndim) ? 1 : 0;
      a.zero1[d][s] = c->zero1[d][s];
    }
  const int u = c->par.user;
  a.grav_on = (c->par.sourceunsplit && grav_module(u)) ? 1 : 0;
  a.visc_on = (c->par.sourceunsplit && visc_on(c)) ? 1 : 0;
  a.driver = DRV_NONE;
  if (c->par.sourceunsplit) {
    if (u == SAC_USR_SLOG) a.driver = DRV_SLOG;
    if (u == SAC_USR_STRAT) a.driver = DRV_STRAT;
    if (u == SAC_USR_TUBE) a.driver = DRV_TUBE;
  }
  a.epi = EPI_PLAIN;
  return a;
}

// advect1 (src/vac.t:490-549): out = base + qdt R(wct) then getboundary(out)
sac_status advect1(sac_ctx* c, const std::string& method, double qdt, int dmin, int dmax, double qt,
                   const double* wct, const double* base, double* out, unsigned mask, int epi = EPI_PLAIN,
                   double* aux1 = nullptr, const double* aux2 = nullptr) {
  if (method == "cd4" || method == "source") {
    const bool flux = (method == "cd4");
    CK(cudaMemsetAsync(c->red, 0, 3 * sizeof(unsigned long long), c->stream));
    launch_prep(c, wct);
    StageArgs a = stage_args(c, qdt, dmin, dmax, flux, qt, wct, base, out, mask);
    a.epi = epi;
    a.aux1 = aux1;
    a.aux2 = aux2;
    launch_stage(c, a);
  } else if (base != out) {
    CK(cudaMemcpyAsync(out, base, sizeof(double) * c->g.np * c->g.ncell, cudaMemcpyDeviceToDevice, c->stream));
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
  launch_bound(c, b, c->g.np);
  CK(cudaGetLastError());
  return SAC_OK;
}

__global__ void k_lin_threestep_a(double* w2, const double* w, const double* w1, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    w2[i] = 3 * 0.25 * w[i] + 0.25 * w1[i];
}
__global__ void k_lin_threestep_b(double* w, const double* w2, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    w[i] = w[i] / 3 + w2[i] * (2.0 / 3);
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
}

sac_status sac_create(const sac_params* p, sac_ctx** out) {
  if (!p || !out) return SAC_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return SAC_ERR_NODEVICE;
  if (p->device < 0 || p->device >= ndev) return SAC_ERR_ARG;
  if (p->precision != SAC_PREC_FP64) return SAC_ERR_UNSUPPORTED;
  sac_ctx* c = new sac_ctx();
  c->par = *p;
  c->dev = p->device;
  if (cudaSetDevice(c->dev) != cudaSuccess || cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return SAC_ERR_CUDA;
  }
  *out = c;
  return SAC_OK;
}

void sac_destroy(sac_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->dev);
  if (c->stream) cudaStreamSynchronize(c->stream);
  release(c);
  if (c->stream) cudaStreamDestroy(c->stream);
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
  // gridsetup1 (src/vacgrid.t:585-629): extrapolate x into the ghosts and one layer
  // beyond, then dx = (x(+1)-x(-1))/2.
  int qn[3], qo[3];
  for (int d = 0; d < 3; ++d) {
    qn[d] = (d < ndim) ? g.n[d] + 2 : 1;
    qo[d] = (d < ndim) ? 1 : 0;
  }
  const long qc = (long)qn[0] * qn[1] * qn[2];
  std::vector<double> qx((size_t)ndim * qc, 0.0);
  auto qid = [&](int i, int j, int k) { return (i + qo[0]) + (long)qn[0] * ((j + qo[1]) + (long)qn[1] * (k + qo[2])); };
  auto gid = [&](int i, int j, int k) { return i + g.st[1] * j + g.st[2] * k; };
  for (int jd = 0; jd < ndim; ++jd)
    for (int k = 0; k < g.n[2]; ++k)
      for (int j = 0; j < g.n[1]; ++j)
        for (int i = 0; i < g.n[0]; ++i) qx[jd * qc + qid(i, j, k)] = x[jd * N + gid(i, j, k)];
  for (int d = 0; d < ndim; ++d) {
    int lo3[3], hi3[3];
    for (int e = 0; e < 3; ++e) {
      lo3[e] = (e < ndim) ? -1 : 0;
      hi3[e] = (e < ndim) ? g.n[e] : 0;
    }
    for (int side = 0; side < 2; ++side) {
      int a, b, ixe, ixf;
      if (side == 0) {
        b = g.n[d];
        a = c->fullgridini ? g.n[d] : g.hi[d] + 1;
        ixe = a - 1;
        ixf = ixe - 1;
      } else {
        a = -1;
        b = c->fullgridini ? -1 : g.lo[d] - 1;
        ixe = b + 1;
        ixf = ixe + 1;
      }
      for (int jd = 0; jd < ndim; ++jd)
        for (int q = a; q <= b; ++q) {
          int l2[3] = {lo3[0], lo3[1], lo3[2]}, h2[3] = {hi3[0], hi3[1], hi3[2]};
          l2[d] = h2[d] = q;
          for (int k = l2[2]; k <= h2[2]; ++k)
            for (int j = l2[1]; j <= h2[1]; ++j)
              for (int i = l2[0]; i <= h2[0]; ++i) {
                int ie[3] = {i, j, k}, iff[3] = {i, j, k};
                ie[d] = ixe;
                iff[d] = ixf;
                const int n = std::abs(ixe - q);
                qx[jd * qc + qid(i, j, k)] = (double)(1 + n) * qx[jd * qc + qid(ie[0], ie[1], ie[2])] -
                                             (double)n * qx[jd * qc + qid(iff[0], iff[1], iff[2])];
              }
        }
    }
  }
  std::vector<double> hx((size_t)ndim * N), hdx((size_t)ndim * N);
  for (int jd = 0; jd < ndim; ++jd)
    for (int k = 0; k < g.n[2]; ++k)
      for (int j = 0; j < g.n[1]; ++j)
        for (int i = 0; i < g.n[0]; ++i) hx[jd * N + gid(i, j, k)] = qx[jd * qc + qid(i, j, k)];
  for (int d = 0; d < ndim; ++d)
    for (int k = 0; k < g.n[2]; ++k)
      for (int j = 0; j < g.n[1]; ++j)
        for (int i = 0; i < g.n[0]; ++i) {
          int p[3] = {i, j, k}, m[3] = {i, j, k};
          p[d] += 1;
          m[d] -= 1;
          hdx[d * N + gid(i, j, k)] = 0.5 * (qx[d * qc + qid(p[0], p[1], p[2])] - qx[d * qc + qid(m[0], m[1], m[2])]);
        }
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
  const size_t bp = sizeof(double) * g.np * N;
  for (auto& p : c->P) CK(cudaMalloc(&p, bp));
  CK(cudaMalloc(&c->BG, sizeof(double) * (g.nw - g.np) * N));
  CK(cudaMalloc(&c->D, sizeof(double) * (ndir + 3) * N));
  CK(cudaMalloc(&c->x, sizeof(double) * ndim * N));
  CK(cudaMalloc(&c->dx, sizeof(double) * ndim * N));
  CK(cudaMalloc(&c->red, 8 * sizeof(unsigned long long)));
  CK(cudaMemsetAsync(c->red, 0, 8 * sizeof(unsigned long long), c->stream));
  CK(cudaMemcpyAsync(c->x, hx.data(), sizeof(double) * ndim * N, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->dx, hdx.data(), sizeof(double) * ndim * N, cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->grid_set = true;
  c->bc_set = false;
  c->state_set = false;
  c->bc_init_done = false;
  c->itmin_set = false;
  return SAC_OK;
}

sac_status sac_set_boundaries(sac_ctx* c, int nB, const char* typeB, const int* ipairB) {
  if (!c || !typeB) return SAC_ERR_ARG;
  if (!c->grid_set) return fail(c, SAC_ERR_STATE, "sac_set_grid first");
  const Geom& g = c->g;
  if (nB != 2 * g.ndim) return fail(c, SAC_ERR_UNSUPPORTED, "only the default 2*ndim boundary regions are implemented");
  CK(cudaSetDevice(c->dev));
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
  // periodic pairing (src/vacgrid.t:109-120) and source offsets
  int pair[6] = {-1, -1, -1, -1, -1, -1};
  for (int iB = 0; iB < nB; ++iB) pair[iB] = ipairB ? ipairB[iB] - 1 : -1;
  for (int iB = 0; iB < nB; ++iB)
    if (t[(long)g.nw * iB] == "periodic" && pair[iB] < 0) {
      for (int jB = iB + 1; jB < nB; ++jB)
        if (t[(long)g.nw * jB] == "periodic" && pair[jB] < 0 && jB / 2 == iB / 2 && (jB % 2) != (iB % 2)) {
          pair[iB] = jB;
          pair[jB] = iB;
        }
      if (pair[iB] < 0) return fail(c, SAC_ERR_ARG, "Error in BoundSetup: No periodic pair");
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
  // fixB slabs for every region that holds a fixed-type variable
  long off = 0;
  for (int iB = 0; iB < nB; ++iB) {
    const int d = iB / 2;
    long sl = 2;  // dixB layers
    for (int e = 0; e < g.ndim; ++e)
      if (e != d) sl *= g.n[e];
    c->slab[iB] = sl;
    c->fixoff[iB] = off;
    bool any = false;
    for (int iw = 0; iw < g.nw; ++iw) {
      int8_t ty = c->h_type[iw * nB + iB];
      any = any || ty == BT_FIXED || ty == BT_FIXED1 || ty == BT_GRAD1;
    }
    if (any) off += sl * g.nw;
  }
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
  CK(cudaMemcpyAsync(c->P[0], w, sizeof(double) * g.np * N, cudaMemcpyHostToDevice, c->stream));
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
  CK(cudaMemcpyAsync(w, c->P[0], sizeof(double) * g.np * N, cudaMemcpyDeviceToHost, c->stream));
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
  BcArgs b = bc_args(c, c->P[0]);
  b.init = c->bc_init_done ? 0 : 1;
  launch_bound(c, b, g.nw);
  if (!c->bc_init_done) {
    const int nB = 2 * g.ndim;
    for (int iB = 0; iB < nB; ++iB)
      for (int iw = 0; iw < g.nw; ++iw) {
        const int8_t ty = c->h_type[iw * nB + iB];
        if ((ty == BT_FIXED || ty == BT_FIXED1 || ty == BT_GRAD1) && !c->h_fixed[iw * nB + iB]) {
          const int bs = 256;
          k_fixcapture<<<(unsigned)((c->slab[iB] + bs - 1) / bs), bs, 0, c->stream>>>(
              g, c->P[0], c->BG, c->fixB, c->fixoff[iB], c->slab[iB], iw, iB / 2, iB % 2, ty == BT_GRAD1 ? 1 : 0);
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
sac_status sac_getdt(sac_ctx* c, double* dt, int it) {
  if (!c || !dt) return SAC_ERR_ARG;
  if (!c->state_set || !c->bc_set) return fail(c, SAC_ERR_STATE, "state and boundaries must be set");
  CK(cudaSetDevice(c->dev));
  if (!c->itmin_set) {
    c->itmin = it;
    c->itmin_set = true;
  }
  const Geom& g = c->g;
  double d;
  if (c->par.dtpar > 0.0) {
    d = c->par.dtpar;
  } else {
    d = bigdouble;
    if (c->par.courantpar > 0.0) {  // getdt_courant, src/vac.t:641-699
      CK(cudaMemsetAsync(c->red + 4, 0, sizeof(unsigned long long), c->stream));
      const long nm = (long)(g.hi[0] - g.lo[0] + 1) * (g.hi[1] - g.lo[1] + 1) * (g.hi[2] - g.lo[2] + 1);
      const int bs = 256;
      const unsigned nb = (unsigned)std::min<long>((nm + bs - 1) / bs, 148L * 16);
      switch (g.ndir) {
        case 1: k_courant<1><<<nb, bs, 0, c->stream>>>(g, c->P[0], c->BG, c->dx, c->red + 4, c->par.gamma); break;
        case 2: k_courant<2><<<nb, bs, 0, c->stream>>>(g, c->P[0], c->BG, c->dx, c->red + 4, c->par.gamma); break;
        default: k_courant<3><<<nb, bs, 0, c->stream>>>(g, c->P[0], c->BG, c->dx, c->red + 4, c->par.gamma); break;
      }
      c->kernel_launches++;
      unsigned long long bits = 0;
      CK(cudaMemcpyAsync(&bits, c->red + 4, sizeof(bits), cudaMemcpyDeviceToHost, c->stream));
      CK(cudaStreamSynchronize(c->stream));
      double courantmax;
      std::memcpy(&courantmax, &bits, sizeof(double));
      if (!(courantmax == courantmax) || std::isinf(courantmax))
        return fail(c, SAC_ERR_NONFINITE, "non-finite wave speed in getdt_courant");
      if (courantmax > smalldouble) d = std::min(d, c->par.courantpar / courantmax);
    }
    if (c->par.eta != 0.0) return fail(c, SAC_ERR_UNSUPPORTED, "Resistive MHD module is OFF (eta must be 0)");
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

sac_status sac_advect(sac_ctx* c, const char* method, const int* iws, int idimmin, int idimmax, double dt, double t,
                      int it) {
  (void)it;
  if (!c || !method) return SAC_ERR_ARG;
  if (!c->state_set || !c->bc_set) return fail(c, SAC_ERR_STATE, "state and boundaries must be set");
  if (!c->bc_init_done) return fail(c, SAC_ERR_STATE, "call sac_getboundary once before the first advect");
  CK(cudaSetDevice(c->dev));
  const Geom& g = c->g;
  std::string m(method);
  while (!m.empty() && (m.back() == ' ' || m.back() == '\0')) m.pop_back();
  if (m != "cd4" && m != "source" && m != "nul") return fail(c, SAC_ERR_UNSUPPORTED, "method " + m);
  if (idimmin < 1 || idimmax > g.ndim || idimmin > idimmax) return fail(c, SAC_ERR_ARG, "idim range");
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
  const int dmin = idimmin - 1, dmax = idimmax - 1;
  double *w = c->P[0], *w1 = c->P[1], *w2 = c->P[2], *w3 = c->P[3];
  const size_t bytes = sizeof(double) * g.np * g.ncell;
  const std::string ta(c->par.typeadvance);
  sac_status st = SAC_OK;
#define RUN(x)                    \
  do {                            \
    st = (x);                     \
    if (st != SAC_OK) return st;  \
  } while (0)
  if (ta == "fourstep") {
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
    k_lin_threestep_a<<<592, 256, 0, c->stream>>>(w2, w, w1, n);
    RUN(advect1(c, m, dt / 4, dmin, dmax, t + dt / 4, w1, w2, w2, mask));
    k_lin_threestep_b<<<592, 256, 0, c->stream>>>(w, w2, n);
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
  return SAC_OK;
}

// Number of kernels this library launched on the context (benchmark accounting).
long sac_kernel_launches(const sac_ctx* c) { return c ? c->kernel_launches : 0; }

}  // extern "C"
