// sac_kernels.cuh -- sm_100a kernels of the perturbation-MHD stage.
//
// One thread owns one mesh cell and computes its complete stage update
//     out = base + qdt * R(wCT)
// in registers, adding the terms in the order the reference adds them to w:
//   flux divergence per dimension and variable, e-equation background work
//     (centdiff4, src/vaccd.t:35-70),
//   gravity (addsource_grav, src/vacusr.gravity.t:24-81),
//   hyperdiffusion (addsource_visc + setnu, src/vacusr.viscosity.t:2-455),
//   the user driver (specialsource, src/vacusr.f:1255-1382),
// with optional Runge-Kutta epilogues fused into the store.  Neighbour data are
// read through the read-only data cache; per-cell quantities that need a
// division (v = m/rho, the "173" energy, p'_tot, rho+rhob) come precomputed by
// k_prep, which also produces the per-dimension c_tot maxima setnu needs.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace sacgpu {

constexpr double kSmall = 1.0e-99;  // smalldouble, src/vacdef.t:50
constexpr int kMaxDim = 3;

// Boundary codes (typeB strings of src/vacgrid.t:257-470)
enum BType : int8_t {
  BT_CONT = 0, BT_FIXED, BT_CONT1, BT_FIXED1, BT_GRAD1, BT_PERIODIC, BT_SYMM, BT_SYMM0, BT_ASYMM,
  BT_CONTCD4
};

// Driver codes
enum Drv : int { DRV_NONE = 0, DRV_SLOG = 1, DRV_STRAT = 2, DRV_TUBE = 3 };

// Run-Kutta epilogues fused into the stage store
enum Epi : int {
  EPI_PLAIN = 0,   // out = acc
  EPI_RK4_S3 = 1,  // out = acc; aux1 = (aux1 + 2*aux2 + acc - 4*base)/3   (src/vac.t:450)
  EPI_RK4_S4 = 2   // out = acc + aux1                                      (src/vac.t:454)
};

struct Geom {
  int ndim, ndir, nw, np;
  int n[3];        // grid extents incl. ghosts
  int lo[3], hi[3];  // mesh bounds (0-based, inclusive)
  long st[3];      // strides
  long ncell;
};

// Per-stage arguments (passed by value).
struct StageArgs {
  Geom g;
  const double* __restrict__ wct_p;  // perturbed vars of wCT, np*ncell
  const double* __restrict__ bgv;    // background vars (eb, rhob, bg1..), (nw-np)*ncell
  const double* base;                // perturbed vars of the base state (may alias out)
  double* out;                       // perturbed vars of the result
  double* aux1;                      // RK4 accumulator (EPI_RK4_*)
  const double* aux2;                // w2 for EPI_RK4_S3
  const double* __restrict__ D;      // derived: rt, v1..v_ndir, e173, ptot (ndir+3)*ncell
  const double* __restrict__ dx;     // ndim*ncell
  const double* __restrict__ x;      // ndim*ncell
  const unsigned long long* ctot;    // [3] bits of c_tot per dimension
  unsigned long long* maxnu;         // running max of nu (bits)
  double qdt, qdt2, gamma, t;
  double grav[3];
  double up[16];
  int dmin, dmax;
  unsigned iwmask;     // perturbed variables that receive fluxes/gravity
  int zero4[3][2];     // gradient4 edge zeroing (boundary not 'mpi')
  int zero1[3][2];     // gradient1* edge zeroing (typeB(1,iB) neither periodic nor mpi)
  int mirror[3][2];    // setnu third-layer mirror (boundary not 'mpi')
  int grav_on, visc_on, driver, epi;
};

__device__ __forceinline__ void atomic_max_nonneg(unsigned long long* a, double v) {
  // non-negative doubles order like their bit patterns; NaN maps above +Inf
  unsigned long long b = __double_as_longlong(v);
  if (v != v) b = 0x7ff8000000000000ull;
  atomicMax(a, b);
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// block-wide max of non-negative values -> one atomic per block.  NaN is
// propagated (it maps above +Inf in the bit order used by atomic_max_nonneg).
__device__ __forceinline__ void block_max_to(unsigned long long* dst, double v, double* sh) {
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nthr = blockDim.x * blockDim.y * blockDim.z;
  const int lane = tid & 31, wid = tid >> 5;
  const bool nan = (v != v);
  const bool anynan = __syncthreads_or(nan);
  v = nan ? 0.0 : v;
  v = warp_max(v);
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  if (tid < 32) {
    double m = (tid < (nthr + 31) / 32) ? sh[tid] : 0.0;
    m = warp_max(m);
    if (tid == 0) atomic_max_nonneg(dst, anynan ? __longlong_as_double(0x7ff8000000000000ll) : m);
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// k_prep: derived per-cell fields over the whole grid and c_tot maxima on the mesh
// ---------------------------------------------------------------------------
template <int NDIR>
__global__ void k_prep(Geom g, const double* __restrict__ wp, const double* __restrict__ bgv,
                       double* __restrict__ D, unsigned long long* ctot, double gamma, int ndim) {
  __shared__ double sh[32];
  const long c = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const long N = g.ncell;
  double cm[3] = {0.0, 0.0, 0.0};
  if (c < N) {
    constexpr int E = NDIR + 1;
    const double rho = wp[c];
    const double rhob = bgv[1 * N + c];
    const double eb = bgv[c];
    const double rt = rho + rhob;
    double m[NDIR], b[NDIR], bg[NDIR];
#pragma unroll
    for (int C = 0; C < NDIR; ++C) {
      m[C] = wp[(1 + C) * N + c];
      b[C] = wp[(E + 1 + C) * N + c];
      bg[C] = bgv[(2 + C) * N + c];
    }
    const double e = wp[E * N + c];
    D[c] = rt;
#pragma unroll
    for (int C = 0; C < NDIR; ++C) D[(1 + C) * N + c] = m[C] / rt;
    // q of setnu for iw=173: e - (b^2 + m^2/rho)/2, src/vacusr.viscosity.t:301
    double b2 = 0.0, m2 = 0.0, bb = 0.0, bgs = 0.0, Bt2 = 0.0;
#pragma unroll
    for (int C = 0; C < NDIR; ++C) b2 = b2 + b[C] * b[C];
#pragma unroll
    for (int C = 0; C < NDIR; ++C) m2 = m2 + m[C] * m[C];
    D[(NDIR + 1) * N + c] = e - 0.5 * (b2 + m2 / rt);
    // getptotal, src/vacphys0.t.mhd:199-201
#pragma unroll
    for (int C = 0; C < NDIR; ++C) bb = bb + b[C] * bg[C];
    const double pp = (gamma - 2.0) * (bb + 0.5 * b2);
    D[(NDIR + 2) * N + c] = (gamma - 1.0) * (e - 0.5 * m2 / rt) - pp;
    // c_tot candidates (getcmax over ixM), src/vacphys0.t.mhd:95-106
    int p0 = (int)(c % g.n[0]);
    int p1 = (int)((c / g.n[0]) % g.n[1]);
    int p2 = (int)(c / ((long)g.n[0] * g.n[1]));
    bool mesh = p0 >= g.lo[0] && p0 <= g.hi[0] && p1 >= g.lo[1] && p1 <= g.hi[1] && p2 >= g.lo[2] &&
                p2 <= g.hi[2];
    if (mesh) {
      // getpthermal then getcsound2
      double q = 0.5 * m2 / rt;
      q = q + 0.5 * b2 + bb;
      const double p = (gamma - 1.0) * (e - q);
#pragma unroll
      for (int C = 0; C < NDIR; ++C) bgs = bgs + bg[C] * bg[C];
      const double cs2 = gamma * (p + (gamma - 1.0) * (eb - 0.5 * bgs)) / rt;
#pragma unroll
      for (int C = 0; C < NDIR; ++C) {
        double B = b[C] + bg[C];
        Bt2 = Bt2 + B * B;
      }
      const double cf2 = Bt2 / rt + cs2;
      for (int d = 0; d < ndim; ++d) {
        const double Bd = b[d] + bg[d];
        cm[d] = sqrt(0.5 * (cf2 + sqrt(cf2 * cf2 - 4.0 * cs2 * (Bd * Bd) / rt))) + fabs(m[d] / rt);
      }
    }
  }
  for (int d = 0; d < ndim; ++d) {
    block_max_to(&ctot[d], cm[d], sh);
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// k_courant: max over the mesh and dimensions of cmax/dx (getdt_courant)
// ---------------------------------------------------------------------------
template <int NDIR>
__global__ void k_courant(Geom g, const double* __restrict__ wp, const double* __restrict__ bgv,
                          const double* __restrict__ dx, unsigned long long* out, double gamma) {
  __shared__ double sh[32];
  const long N = g.ncell;
  double best = 0.0;
  const long nm0 = g.hi[0] - g.lo[0] + 1, nm1 = g.hi[1] - g.lo[1] + 1, nm2 = g.hi[2] - g.lo[2] + 1;
  const long tot = nm0 * nm1 * nm2;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < tot; t += (long)gridDim.x * blockDim.x) {
    const int i0 = g.lo[0] + (int)(t % nm0);
    const int i1 = g.lo[1] + (int)((t / nm0) % nm1);
    const int i2 = g.lo[2] + (int)(t / (nm0 * nm1));
    const long c = i0 + g.st[1] * i1 + g.st[2] * i2;
    constexpr int E = NDIR + 1;
    const double rho = wp[c], rhob = bgv[N + c], eb = bgv[c];
    const double rt = rho + rhob;
    double m2 = 0, b2 = 0, bb = 0, bgs = 0, Bt2 = 0;
#pragma unroll
    for (int C = 0; C < NDIR; ++C) m2 = m2 + wp[(1 + C) * N + c] * wp[(1 + C) * N + c];
#pragma unroll
    for (int C = 0; C < NDIR; ++C) b2 = b2 + wp[(E + 1 + C) * N + c] * wp[(E + 1 + C) * N + c];
#pragma unroll
    for (int C = 0; C < NDIR; ++C) bb = bb + wp[(E + 1 + C) * N + c] * bgv[(2 + C) * N + c];
    double q = 0.5 * m2 / rt;
    q = q + 0.5 * b2 + bb;
    const double p = (gamma - 1.0) * (wp[E * N + c] - q);
#pragma unroll
    for (int C = 0; C < NDIR; ++C) bgs = bgs + bgv[(2 + C) * N + c] * bgv[(2 + C) * N + c];
    const double cs2 = gamma * (p + (gamma - 1.0) * (eb - 0.5 * bgs)) / rt;
#pragma unroll
    for (int C = 0; C < NDIR; ++C) {
      double B = wp[(E + 1 + C) * N + c] + bgv[(2 + C) * N + c];
      Bt2 = Bt2 + B * B;
    }
    const double cf2 = Bt2 / rt + cs2;
    for (int d = 0; d < g.ndim; ++d) {
      const double Bd = wp[(E + 1 + d) * N + c] + bgv[(2 + d) * N + c];
      double cmax = sqrt(0.5 * (cf2 + sqrt(cf2 * cf2 - 4.0 * cs2 * (Bd * Bd) / rt))) +
                    fabs(wp[(1 + d) * N + c] / rt);
      double r = cmax / dx[d * N + c];
      best = (r != r) ? r : fmax(best, r);
      if (r != r) break;
    }
  }
  block_max_to(out, best, sh);
}

// ---------------------------------------------------------------------------
// the stage kernel
// ---------------------------------------------------------------------------
template <int NDIR>
struct Var {
  static constexpr int RHO = 0, M0 = 0, E = NDIR + 1, B0 = NDIR + 1, NP = 2 * NDIR + 2;
  // background block: eb, rhob, bg1..
  static constexpr int EB = 0, RHOB = 1, BG0 = 1;
};

// flux of every perturbed variable along d at cell j (getflux + transport,
// src/vacphys.mhd0.t:147-222, src/vaccd.t:43-46), evaluated in the reference's
// operation order.
template <int NDIR>
__device__ __forceinline__ void flux_all(const StageArgs& a, int d, long j, double* F) {
  using Vr = Var<NDIR>;
  const long N = a.g.ncell;
  const double* wp = a.wct_p;
  const double* bgv = a.bgv;
  const double rho = __ldg(wp + j);
  const double rhob = __ldg(bgv + N + j);
  const double rt = rho + rhob;
  const double eb = __ldg(bgv + j);
  const double ptot = __ldg(a.D + (NDIR + 2) * N + j);
  double m[NDIR], b[NDIR], bg[NDIR], v[NDIR];
#pragma unroll
  for (int C = 0; C < NDIR; ++C) {
    m[C] = __ldg(wp + (1 + C) * N + j);
    b[C] = __ldg(wp + (Vr::B0 + 1 + C) * N + j);
    bg[C] = __ldg(bgv + (2 + C) * N + j);
    v[C] = __ldg(a.D + (1 + C) * N + j);
  }
  const double e = __ldg(wp + Vr::E * N + j);
  double md = 0, bd = 0, bgd = 0, vd = 0;
#pragma unroll
  for (int C = 0; C < NDIR; ++C)
    if (C == d) {
      md = m[C];
      bd = b[C];
      bgd = bg[C];
      vd = v[C];
    }
  // rho
  F[0] = rhob * md / rt + vd * rho;
  // momenta
#pragma unroll
  for (int C = 0; C < NDIR; ++C) {
    double f;
    if (C == d)
      f = (ptot + 0.0) - (b[C] * bgd + bd * bg[C]) - b[C] * bd;
    else
      f = -(b[C] * bgd + bd * bg[C]) - b[C] * bd;
    F[1 + C] = f + vd * m[C];
  }
  // energy
  {
    double s1 = 0, s2 = 0;
#pragma unroll
    for (int C = 0; C < NDIR; ++C) s1 = s1 + bg[C] * m[C];
#pragma unroll
    for (int C = 0; C < NDIR; ++C) s2 = s2 + b[C] * m[C];
    double f = (md * (ptot + 0.0) - bd * s1 - bgd * s2) / rt + eb * md / rt - bd * s2 / rt;
    F[Vr::E] = f + vd * e;
  }
  // induction
#pragma unroll
  for (int C = 0; C < NDIR; ++C) {
    if (C == d)
      F[Vr::B0 + 1 + C] = 0.0;
    else
      F[Vr::B0 + 1 + C] = -(v[C] * (bd + bgd)) + vd * bg[C] + vd * b[C];
  }
}

// setnu's left/right coefficients at cell j along k for one q field
// (src/vacusr.viscosity.t:372-450).  pos is j's coordinate along k.
struct NuPair {
  double l, r;
};

__device__ __forceinline__ NuPair nu_pair(const double* __restrict__ q, long j, long s, int pos, int lo,
                                          int hi, bool /*mlo*/, bool /*mhi*/, double pre, double dxk) {
  double qq[7];
#pragma unroll
  for (int a = -3; a <= 3; ++a) {
    // the third layer beyond the two ghost layers does not exist in the array;
    // setnu mirrors it about the first/last mesh cell at every boundary that is not
    // 'mpi' (always the case on one device), so the window never leaves the grid
    int p = pos + a;
    if (p <= lo - 3) p = lo + 3;
    if (p >= hi + 3) p = hi - 3;
    qq[a + 3] = __ldg(q + j + (long)(p - pos) * s);
  }
  // d1R(a) = |q(a+1)-q(a)|, a=-3..2 ; d3R(a) = |3(q(a+1)-q(a)) - (q(a+2)-q(a-1))|, a=-2..1
  double d1[6], d3[4];
#pragma unroll
  for (int a = 0; a < 6; ++a) d1[a] = fabs(qq[a + 1] - qq[a]);
#pragma unroll
  for (int a = 0; a < 4; ++a) d3[a] = fabs(3.0 * (qq[a + 2] - qq[a + 1]) - (qq[a + 3] - qq[a]));
  // indices: d1[a+3] = d1R(a), d3[a+2] = d3R(a)
  const double md3R = fmax(fmax(d3[1], d3[2]), d3[3]);
  const double md1R = fmax(fmax(fmax(fmax(d1[1], d1[2]), d1[3]), d1[4]), d1[5]);
  const double md3L = fmax(fmax(d3[0], d3[1]), d3[2]);
  const double md1L = fmax(fmax(fmax(fmax(d1[0], d1[1]), d1[2]), d1[3]), d1[4]);
  NuPair n;
  n.r = (md1R > 0.0) ? pre * md3R / md1R * dxk : 0.0;
  n.l = (md1L > 0.0) ? pre * md3L / md1L * dxk : 0.0;
  return n;
}

template <int NDIM, int NDIR>
__global__ void __launch_bounds__(128) k_stage(const StageArgs a) {
  using Vr = Var<NDIR>;
  constexpr int NP = Vr::NP;
  __shared__ double sh[32];
  const Geom& g = a.g;
  const long N = g.ncell;
  int pos[3];
  pos[0] = g.lo[0] + blockIdx.x * blockDim.x + threadIdx.x;
  pos[1] = g.lo[1] + blockIdx.y * blockDim.y + threadIdx.y;
  pos[2] = g.lo[2] + blockIdx.z * blockDim.z + threadIdx.z;
  const bool active = pos[0] <= g.hi[0] && pos[1] <= g.hi[1] && pos[2] <= g.hi[2];
  double numax = 0.0;
  if (active) {
    const long c = pos[0] + g.st[1] * pos[1] + g.st[2] * pos[2];
    double acc[NP];
#pragma unroll
    for (int iw = 0; iw < NP; ++iw) acc[iw] = a.base[iw * N + c];
    const double* D = a.D;
    const double* wp = a.wct_p;
    const double* bgv = a.bgv;

    // --- centdiff4: flux divergence and e background work -------------------
    for (int d = a.dmin; d <= a.dmax; ++d) {
      const long s = g.st[d];
      const double dxd = __ldg(a.dx + d * N + c);
      const bool z = (a.zero4[d][0] && pos[d] <= g.lo[d] + 1) || (a.zero4[d][1] && pos[d] >= g.hi[d] - 1);
      if (!z) {
        double Fp2[NP], Fp1[NP], Fm1[NP], Fm2[NP];
        flux_all<NDIR>(a, d, c + 2 * s, Fp2);
        flux_all<NDIR>(a, d, c + s, Fp1);
        flux_all<NDIR>(a, d, c - s, Fm1);
        flux_all<NDIR>(a, d, c - 2 * s, Fm2);
#pragma unroll
        for (int iw = 0; iw < NP; ++iw) {
          if (!((a.iwmask >> iw) & 1u)) continue;
          const double g4 = -(Fp2[iw] - 8.0 * (Fp1[iw] - Fm1[iw]) - Fm2[iw]) / dxd / 12.0;
          acc[iw] = acc[iw] - a.qdt * g4;
        }
      }
      if ((a.iwmask >> Vr::E) & 1u) {
        const double* vd = D + (1 + d) * N;
        // -qdt * d_d(v_d) * ptotal_bg
        if (!z) {
          const double g4 = -(__ldg(vd + c + 2 * s) - 8.0 * (__ldg(vd + c + s) - __ldg(vd + c - s)) -
                              __ldg(vd + c - 2 * s)) / dxd / 12.0;
          double bgs = 0.0;
#pragma unroll
          for (int C = 0; C < NDIR; ++C) bgs = bgs + __ldg(bgv + (2 + C) * N + c) * __ldg(bgv + (2 + C) * N + c);
          const double fb = (a.gamma - 1.0) * __ldg(bgv + c) - 0.5 * (a.gamma - 2.0) * bgs;
          acc[Vr::E] = acc[Vr::E] - a.qdt * g4 * fb;
        }
        for (int di = a.dmin; di <= a.dmax; ++di) {
          const long si = g.st[di];
          const bool zi = (a.zero4[di][0] && pos[di] <= g.lo[di] + 1) ||
                          (a.zero4[di][1] && pos[di] >= g.hi[di] - 1);
          if (zi) continue;
          const double dxi = __ldg(a.dx + di * N + c);
          const double g4 = -(__ldg(vd + c + 2 * si) - 8.0 * (__ldg(vd + c + si) - __ldg(vd + c - si)) -
                              __ldg(vd + c - 2 * si)) / dxi / 12.0;
          acc[Vr::E] = acc[Vr::E] + a.qdt * __ldg(bgv + (2 + di) * N + c) * __ldg(bgv + (2 + d) * N + c) * g4;
        }
      }
    }

    const double qdt = a.qdt2;
    // --- gravity --------------------------------------------------------------
    if (a.grav_on) {
      const double rho = __ldg(wp + c);
#pragma unroll
      for (int d = 0; d < NDIM; ++d)
        if (((a.iwmask >> (1 + d)) & 1u) && fabs(a.grav[d]) > kSmall)
          acc[1 + d] = acc[1 + d] + qdt * a.grav[d] * rho;
      if ((a.iwmask >> Vr::E) & 1u) {
        const double rt = __ldg(D + c);
#pragma unroll
        for (int d = 0; d < NDIM; ++d)
          if (fabs(a.grav[d]) > kSmall)
            acc[Vr::E] = acc[Vr::E] + qdt * a.grav[d] * rho * __ldg(wp + (1 + d) * N + c) / rt;
      }
    }

    // --- hyperdiffusion --------------------------------------------------------
    if (a.visc_on) {
      const double* rtf = D;
      auto inmesh = [&](int d, int p) { return p >= g.lo[d] && p <= g.hi[d]; };
      auto z1 = [&](int d, int p) {  // gradient1 zero rule at coordinate p along d
        return (a.zero1[d][0] && (p == g.lo[d] - 1 || p == g.lo[d])) ||
               (a.zero1[d][1] && (p == g.hi[d] + 1 || p == g.hi[d]));
      };
      double ct[NDIM];
#pragma unroll
      for (int k = 0; k < NDIM; ++k) ct[k] = __longlong_as_double((long long)a.ctot[k]);

      // density and the "173" energy, :45-64
#pragma unroll
      for (int pass = 0; pass < 2; ++pass) {
        const double* q = (pass == 0) ? wp : (D + (NDIR + 1) * N);
        const int tgt = (pass == 0) ? 0 : Vr::E;
#pragma unroll
        for (int k = 0; k < NDIM; ++k) {
          const long s = g.st[k];
          const double dxk = __ldg(a.dx + k * N + c);
          NuPair nu = nu_pair(q, c, s, pos[k], g.lo[k], g.hi[k], a.mirror[k][0], a.mirror[k][1], ct[k] * 0.04, dxk);
          numax = fmax(numax, fmax(nu.r, nu.l));
          const bool zz = z1(k, pos[k]);
          const double qc = __ldg(q + c);
          const double gL = zz ? 0.0 : (qc - __ldg(q + c - s)) / dxk;
          const double gR = zz ? 0.0 : (__ldg(q + c + s) - qc) / dxk;
          const double tL = (nu.l + 0.0) * gL, tR = (nu.r + 0.0) * gR;
          acc[tgt] = acc[tgt] + (tR - tL) / dxk * qdt;
        }
      }
      // momentum, :69-133
#pragma unroll
      for (int k = 0; k < NDIM; ++k) {
        const long sk = g.st[k];
        const double dxk = __ldg(a.dx + k * N + c);
        const double rC = __ldg(rtf + c);
        const double rL = (rC + __ldg(rtf + c - sk)) / 2.0;
        const double rR = (__ldg(rtf + c + sk) + rC) / 2.0;
        const bool zk = z1(k, pos[k]);
#pragma unroll
        for (int l = 0; l < NDIM; ++l) {
          const double* q = D + (1 + l) * N;  // v_l
          NuPair nu = nu_pair(q, c, sk, pos[k], g.lo[k], g.hi[k], a.mirror[k][0], a.mirror[k][1], ct[k] * 0.4, dxk);
          numax = fmax(numax, fmax(nu.r, nu.l));
          const double qc = __ldg(q + c);
          const double gL = zk ? 0.0 : (qc - __ldg(q + c - sk)) / dxk;
          const double gR = zk ? 0.0 : (__ldg(q + c + sk) - qc) / dxk;
          const double tL = (nu.l + 0.0) * gL, tR = (nu.r + 0.0) * gR;
          const double* ml = wp + (1 + l) * N;
          const double mc = __ldg(ml + c);
          const double VL = (mc + __ldg(ml + c - sk)) / 2.0;
          const double VR = (__ldg(ml + c + sk) + mc) / 2.0;
          const double t2m = (rR * tR - rL * tL) / dxk / 2.0;
          const double t2e = (VR * tR - VL * tL) / dxk / 2.0;
          // ii1=0: i=k, ii0=l
          acc[1 + l] = acc[1 + l] + t2m * qdt;
          acc[Vr::E] = acc[Vr::E] + t2e * qdt;
          if (l == k) {
            // ii1=1 with l==k takes the same branch again
            acc[1 + l] = acc[1 + l] + t2m * qdt;
            acc[Vr::E] = acc[Vr::E] + t2e * qdt;
          } else {
            // ii1=1: i=l, ii0=k: d_l( rho * d_k v_l * (nuL+nuR)/4 ) and d_l( m_k * ... )
            const long sl = g.st[l];
            double Tm[2], Te[2];
#pragma unroll
            for (int sgn = 0; sgn < 2; ++sgn) {
              const long j = sgn ? c + sl : c - sl;
              const int pl = pos[l] + (sgn ? 1 : -1);
              double H = 0.0;
              if (inmesh(l, pl)) {
                const double dxkj = __ldg(a.dx + k * N + j);
                NuPair nj = nu_pair(q, j, sk, pos[k], g.lo[k], g.hi[k], a.mirror[k][0], a.mirror[k][1],
                                    ct[k] * 0.4, dxkj);
                const double gC = zk ? 0.0 : (__ldg(q + j + sk) - __ldg(q + j - sk)) / dxkj / 2.0;
                H = gC * (nj.l + nj.r + 2.0 * 0.0) / 2.0 / 2.0;
              }
              Tm[sgn] = __ldg(rtf + j) * H;
              Te[sgn] = __ldg(wp + (1 + k) * N + j) * H;
            }
            const bool zl = z1(l, pos[l]);
            const double dxl = __ldg(a.dx + l * N + c);
            const double tCm = zl ? 0.0 : (Tm[1] - Tm[0]) / dxl / 2.0;
            const double tCe = zl ? 0.0 : (Te[1] - Te[0]) / dxl / 2.0;
            acc[1 + k] = acc[1 + k] + tCm * qdt;
            acc[Vr::E] = acc[Vr::E] + tCe * qdt;
          }
        }
      }
      // magnetic field, :139-215
#pragma unroll
      for (int k = 0; k < NDIM; ++k)
#pragma unroll
        for (int l = 0; l < NDIM; ++l) {
          if (k == l) continue;
          const long sk = g.st[k], sl = g.st[l];
          const double dxk = __ldg(a.dx + k * N + c);
          const double* q = wp + (Vr::B0 + 1 + l) * N;  // b_l
          NuPair nu = nu_pair(q, c, sk, pos[k], g.lo[k], g.hi[k], a.mirror[k][0], a.mirror[k][1], ct[k] * 0.04, dxk);
          numax = fmax(numax, fmax(nu.r, nu.l));
          const bool zk = z1(k, pos[k]);
          // ii1=0: ii0=k, m=l, sB=-1, j=k  (m /= k branch)
          {
            double K[2], Ke[2];
#pragma unroll
            for (int sgn = 0; sgn < 2; ++sgn) {
              const long j = sgn ? c + sl : c - sl;
              const int pl = pos[l] + (sgn ? 1 : -1);
              double Kv = 0.0;
              if (inmesh(l, pl)) {
                const double dxkj = __ldg(a.dx + k * N + j);
                NuPair nj = nu_pair(q, j, sk, pos[k], g.lo[k], g.hi[k], a.mirror[k][0], a.mirror[k][1],
                                    ct[k] * 0.04, dxkj);
                const double gC = zk ? 0.0 : (__ldg(q + j + sk) - __ldg(q + j - sk)) / dxkj / 2.0;
                Kv = gC * (nj.l + nj.r) / 2.0;
              }
              K[sgn] = Kv;
              Ke[sgn] = Kv * __ldg(wp + (Vr::B0 + 1 + k) * N + j);
            }
            const bool zl = z1(l, pos[l]);
            const double dxl = __ldg(a.dx + l * N + c);
            const double tC = zl ? 0.0 : (K[1] - K[0]) / dxl / 2.0;
            const double tCe = zl ? 0.0 : (Ke[1] - Ke[0]) / dxl / 2.0;
            acc[Vr::B0 + 1 + k] = acc[Vr::B0 + 1 + k] + -1.0 * tC * qdt;
            acc[Vr::E] = acc[Vr::E] + -1.0 * tCe * qdt;
          }
          // ii1=1: ii0=l, m=k, sB=+1, j=l  (m == k branch)
          {
            const double qc = __ldg(q + c);
            const double qm = __ldg(q + c - sk), qp = __ldg(q + c + sk);
            const double BL = (qc + qm) / 2.0, BR = (qp + qc) / 2.0;
            const double gL = zk ? 0.0 : (qc - qm) / dxk;
            const double gR = zk ? 0.0 : (qp - qc) / dxk;
            const double tL = nu.l * gL, tR = nu.r * gR;
            acc[Vr::B0 + 1 + l] = acc[Vr::B0 + 1 + l] + 1.0 * (tR - tL) / dxk * qdt;
            acc[Vr::E] = acc[Vr::E] + 1.0 * (tR * BR - tL * BL) / dxk * qdt;
          }
        }
    }

    // --- user driver -------------------------------------------------------------
    if (a.driver != DRV_NONE) {
      const double rt_new = acc[0] + __ldg(bgv + N + c);
      if (a.driver == DRV_SLOG && NDIM == 3 && NDIR == 3) {
        const double pi_ref = (double)3.1415926535897932384626433832795f;
        const double xc1 = (double)0.1f * 1.0e6, xc2 = 1.0e6, xc3 = 1.0e6;
        const double dz = 0.05e6, dxx = 0.5e6, dyy = 0.5e6, AA = 10.0, B = (double)0.05f;
        const double tdep = sin(a.t * 2.0 * pi_ref / 240.0);
        const double xx = a.x[N + c] - xc2, yy = a.x[2 * N + c] - xc3, zz = a.x[c] - xc1;
        const double ex = exp(-(xx * xx) / (dxx * dxx)), ey = exp(-(yy * yy) / (dyy * dyy)),
                     ez = exp(-(zz * zz) / (dz * dz));
        const double exp_xyz = ex * ey * ez;
        const double th = atan2(yy, xx), ph = atan2(1.0, B);
        const double ux = cos(th + ph), uy = sin(th + ph);
        const double vvx = (ux / sqrt(ux * ux + uy * uy)) * exp_xyz * tdep * AA;
        const double vvy = (uy / sqrt(ux * ux + uy * uy)) * exp_xyz * tdep * AA;
        acc[2] = acc[2] + rt_new * vvx * qdt;
        acc[3] = acc[3] + rt_new * vvy * qdt;
        acc[Vr::E] = acc[Vr::E] + rt_new * (vvx * vvx + vvy * vvy + 0.0 * 0.0) * qdt / 2.0;
      } else if (a.driver == DRV_STRAT) {
        const double tdep = sin(a.up[1] * a.t);
        const double xx = (NDIM > 1) ? a.x[N + c] - a.up[2] : 0.0;
        const double yy = (NDIM > 2) ? a.x[2 * N + c] - a.up[3] : 0.0;
        const double zz = a.x[c] - a.up[5];
        const double v = a.up[0] * tdep * exp(-(xx * xx + yy * yy) / (a.up[4] * a.up[4])) *
                         exp(-(zz * zz) / (a.up[6] * a.up[6]));
        acc[1] = acc[1] + rt_new * v * qdt;
        acc[Vr::E] = acc[Vr::E] + rt_new * (v * v) * qdt / 2.0;
      } else if (a.driver == DRV_TUBE && NDIM >= 2) {
        const double tdep = sin(a.up[1] * a.t);
        const double zz = a.x[c] - a.up[2], xx = a.x[N + c] - a.up[4];
        const double v = a.up[0] * tdep * exp(-(zz * zz) / (a.up[3] * a.up[3])) *
                         exp(-(xx * xx) / (a.up[5] * a.up[5]));
        acc[2] = acc[2] + rt_new * v * qdt;
        acc[Vr::E] = acc[Vr::E] + rt_new * (v * v) * qdt / 2.0;
      }
    }

    // --- store with the Runge-Kutta epilogue ------------------------------------
    if (a.epi == EPI_PLAIN) {
#pragma unroll
      for (int iw = 0; iw < NP; ++iw) a.out[iw * N + c] = acc[iw];
    } else if (a.epi == EPI_RK4_S3) {
#pragma unroll
      for (int iw = 0; iw < NP; ++iw) {
        a.out[iw * N + c] = acc[iw];
        const double w1 = a.aux1[iw * N + c];
        a.aux1[iw * N + c] = (w1 + 2.0 * a.aux2[iw * N + c] + acc[iw] - 4.0 * a.base[iw * N + c]) / 3.0;
      }
    } else {
#pragma unroll
      for (int iw = 0; iw < NP; ++iw) a.out[iw * N + c] = acc[iw] + a.aux1[iw * N + c];
    }
  }
  if (a.visc_on) block_max_to(a.maxnu, numax, sh);
}

// ---------------------------------------------------------------------------
// boundaries: every ghost cell resolved in one pass (getboundary, src/vacgrid.t:195-512)
// ---------------------------------------------------------------------------
// The reference fills boundary regions iB=1..nB in order; a ghost cell's final
// value is written by the region of its highest ghost dimension d, from cells that
// differ only along d and were completed by the lower dimensions.  Resolving that
// chain per cell reproduces the sequential result in one parallel pass.
//
// fixB of region iB is stored compactly: the dixB ghost layers along idimB(iB)
// times the full grid in the other dimensions, one block per variable.
struct BcArgs {
  Geom g;
  double* A;                        // perturbed block of the target array (np vars)
  double* bgA;                      // background block (nw-np vars)
  const int8_t* __restrict__ type;  // [iw*nB + iB]
  const int* __restrict__ fixed;    // [iw*nB + iB] 1 once fixB holds values
  const double* __restrict__ fixB;  // compact slabs, region iB at fixoff[iB]
  long fixoff[6];
  long slab[6];                     // cells per variable in region iB
  int pairshift[3][2];              // periodic source offset along d for lower/upper ghosts
  int init;                         // first call: fixed acts as cont, or keeps the values read (fullgridini)
  int fullgridini;
  int mode;                         // 0 plain, 1 RK4 stage-3 epilogue, 2 RK4 final combination
  double* aux1;                     // w1 (mode 1: written; mode 2: read)
  const double* aux2;               // w2 (mode 1)
  const double* basep;              // w (mode 1)
};

__device__ __forceinline__ long fix_index(const Geom& g, int d, bool up, const int p[3]) {
  int q[3] = {p[0], p[1], p[2]};
  int ext[3];
  for (int e = 0; e < 3; ++e) ext[e] = (e < g.ndim) ? g.n[e] : 1;
  ext[d] = g.lo[d];
  q[d] = up ? p[d] - (g.hi[d] + 1) : p[d];
  return q[0] + (long)ext[0] * (q[1] + (long)ext[1] * q[2]);
}

__device__ __forceinline__ double bc_read(const BcArgs& a, int iw, long c) {
  const int np = a.g.np;
  return iw < np ? a.A[(long)iw * a.g.ncell + c] : a.bgA[(long)(iw - np) * a.g.ncell + c];
}

// Value of variable iw at cell p (mesh or ghost).  fixed_leaf/leaf report a chain
// that ended in a stored fixB value (needed by the RK4 final combination).
template <int DEPTH>
__device__ double bc_resolve(const BcArgs& a, int iw, const int p[3], bool& fixed_leaf, long& leaf) {
  const long c = p[0] + a.g.st[1] * p[1] + a.g.st[2] * p[2];
  int d = -1;
  for (int e = 0; e < a.g.ndim; ++e)
    if (p[e] < a.g.lo[e] || p[e] > a.g.hi[e]) d = e;
  if constexpr (DEPTH == 0) {
    return bc_read(a, iw, c);
  } else {
    if (d < 0) return bc_read(a, iw, c);
    const bool up = p[d] > a.g.hi[d];
    const int iB = 2 * d + (up ? 1 : 0);
    const int nB = 2 * a.g.ndim;
    const int t = a.type[iw * nB + iB];
    const int edge = up ? a.g.hi[d] : a.g.lo[d];
    auto at = [&](int q) {
      int r[3] = {p[0], p[1], p[2]};
      r[d] = q;
      return bc_resolve<DEPTH - 1>(a, iw, r, fixed_leaf, leaf);
    };
    const bool isfixed = a.fixed[iw * nB + iB] != 0;
    auto fbv = [&]() { return a.fixB[a.fixoff[iB] + (long)iw * a.slab[iB] + fix_index(a.g, d, up, p)]; };
    switch (t) {
      case BT_CONT:
        return at(edge);
      case BT_FIXED:
        if (isfixed) {
          fixed_leaf = true;
          leaf = c;
          return fbv();
        }
        if (a.init && a.fullgridini) return bc_read(a, iw, c);
        return at(edge);
      case BT_PERIODIC:
        return at(p[d] + a.pairshift[d][up ? 1 : 0]);
      case BT_SYMM:
      case BT_SYMM0:
        return at(up ? 2 * a.g.hi[d] + 1 - p[d] : 2 * a.g.lo[d] - 1 - p[d]);
      case BT_ASYMM:
        return -at(up ? 2 * a.g.hi[d] + 1 - p[d] : 2 * a.g.lo[d] - 1 - p[d]);
      case BT_CONTCD4: {  // reflection about the edge cell, src/vacgrid.t:261-293
        const int n = up ? p[d] - a.g.hi[d] : a.g.lo[d] - p[d];
        return at(up ? a.g.hi[d] - n : a.g.lo[d] + n);
      }
      default: {  // cont1, fixed1, grad1, src/vacgrid.t:373-409
        if (isfixed) {
          if (t == BT_GRAD1) return fbv() + at(edge);
          fixed_leaf = true;
          leaf = c;
          return fbv();
        }
        if (t != BT_CONT1 && a.init && a.fullgridini) return bc_read(a, iw, c);
        const int f = up ? edge - 1 : edge + 1;
        const int n = abs(p[d] - edge);
        const double ve = at(edge), vf = at(f);
        return (double)(n + 1) * ve - (double)n * vf;
      }
    }
  }
}

// Ghost cells enumerated slab by slab: slab d holds the cells whose highest ghost
// dimension is d (all coordinates for dims < d, mesh coordinates for dims > d).
__global__ void k_bound(BcArgs a, long nslab0, long nslab1, long nslab2, int nvar) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const long tot = nslab0 + nslab1 + nslab2;
  if (t >= tot) return;
  const Geom& g = a.g;
  int d;
  long r;
  if (t < nslab0) {
    d = 0;
    r = t;
  } else if (t < nslab0 + nslab1) {
    d = 1;
    r = t - nslab0;
  } else {
    d = 2;
    r = t - nslab0 - nslab1;
  }
  int ext[3], off[3];
  for (int e = 0; e < 3; ++e) {
    if (e >= g.ndim) {
      ext[e] = 1;
      off[e] = 0;
    } else if (e < d) {
      ext[e] = g.n[e];
      off[e] = 0;
    } else if (e > d) {
      ext[e] = g.hi[e] - g.lo[e] + 1;
      off[e] = g.lo[e];
    } else {
      ext[e] = 2 * g.lo[e];  // dixB lower + dixB upper layers
      off[e] = 0;
    }
  }
  int p[3];
  p[0] = (int)(r % ext[0]);
  p[1] = (int)((r / ext[0]) % ext[1]);
  p[2] = (int)(r / ((long)ext[0] * ext[1]));
  for (int e = 0; e < 3; ++e) p[e] += off[e];
  if (p[d] >= g.lo[d]) p[d] = g.hi[d] + 1 + (p[d] - g.lo[d]);  // upper layers
  const long c = p[0] + g.st[1] * p[1] + g.st[2] * p[2];
  for (int iw = 0; iw < nvar; ++iw) {
    bool fl = false;
    long leaf = 0;
    double v = bc_resolve<3>(a, iw, p, fl, leaf);
    const bool pert = iw < g.np;
    if (a.mode == 2 && pert && fl) v = v + a.aux1[(long)iw * g.ncell + leaf];
    if (pert)
      a.A[(long)iw * g.ncell + c] = v;
    else
      a.bgA[(long)(iw - g.np) * g.ncell + c] = v;
    if (a.mode == 1 && pert) {
      const long o = (long)iw * g.ncell + c;
      a.aux1[o] = (a.aux1[o] + 2.0 * a.aux2[o] + v - 4.0 * a.basep[o]) / 3.0;
    }
  }
}

// Store fixB of region (d,up) for variable iw after the first fill
// (src/vacgrid.t:476-507); grad1 stores the difference to the edge value.
__global__ void k_fixcapture(Geom g, const double* __restrict__ A, const double* __restrict__ bgA, double* fixB,
                             long off, long slab, int iw, int d, int up, int grad) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= slab) return;
  int ext[3];
  for (int e = 0; e < 3; ++e) ext[e] = (e < g.ndim) ? g.n[e] : 1;
  ext[d] = g.lo[d];
  int p[3];
  p[0] = (int)(t % ext[0]);
  p[1] = (int)((t / ext[0]) % ext[1]);
  p[2] = (int)(t / ((long)ext[0] * ext[1]));
  if (up) p[d] += g.hi[d] + 1;
  const long c = p[0] + g.st[1] * p[1] + g.st[2] * p[2];
  auto rd = [&](long cc) { return iw < g.np ? A[(long)iw * g.ncell + cc] : bgA[(long)(iw - g.np) * g.ncell + cc]; };
  double v = rd(c);
  if (grad) {
    const int edge = up ? g.hi[d] : g.lo[d];
    v = v - rd(c + (long)(edge - p[d]) * g.st[d]);
  }
  fixB[off + (long)iw * slab + t] = v;
}

// elementwise helpers over whole perturbed blocks
__global__ void k_copy(double* __restrict__ dst, const double* __restrict__ src, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) dst[i] = src[i];
}

// getdivb (4th order), per-cell |div B| and its square, for diagnostics
template <int NDIR>
__global__ void k_divb(Geom g, const double* __restrict__ wp, const double* __restrict__ bgv,
                       const double* __restrict__ dx, double* out_sq, unsigned long long* out_max,
                       int z00, int z01, int z10, int z11, int z20, int z21) {
  __shared__ double sh[32];
  const long N = g.ncell;
  const long nm0 = g.hi[0] - g.lo[0] + 1, nm1 = g.hi[1] - g.lo[1] + 1, nm2 = g.hi[2] - g.lo[2] + 1;
  const long tot = nm0 * nm1 * nm2;
  const int zz[3][2] = {{z00, z01}, {z10, z11}, {z20, z21}};
  double best = 0.0, sq = 0.0;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < tot; t += (long)gridDim.x * blockDim.x) {
    int p[3];
    p[0] = g.lo[0] + (int)(t % nm0);
    p[1] = g.lo[1] + (int)((t / nm0) % nm1);
    p[2] = g.lo[2] + (int)(t / (nm0 * nm1));
    const long c = p[0] + g.st[1] * p[1] + g.st[2] * p[2];
    double divb = 0.0;
    for (int d = 0; d < g.ndim; ++d) {
      const bool z = (zz[d][0] && p[d] <= g.lo[d] + 1) || (zz[d][1] && p[d] >= g.hi[d] - 1);
      if (z) continue;
      const long s = g.st[d];
      const double* b = wp + (NDIR + 2 + d) * N;
      const double* bg = bgv + (2 + d) * N;
      auto B = [&](long j) { return b[j] + bg[j]; };
      divb = divb + -(B(c + 2 * s) - 8.0 * (B(c + s) - B(c - s)) - B(c - 2 * s)) / dx[d * N + c] / 12.0;
    }
    best = fmax(best, fabs(divb));
    sq += divb * divb;
  }
  // sum of squares: one double atomic per thread block
  double v = sq;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out_sq, v);
  block_max_to(out_max, best, sh);
}

}  // namespace sacgpu
