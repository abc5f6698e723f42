// sac_oracle.cpp -- CPU FP64 restatement of the SAC/VAC perturbation-MHD hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity checker and the timed CPU
// baseline; the product (libsacgpu.so) never links or calls it.  It restates,
// array pass by array pass, the reference routines cited beside each function
// (paths relative to the drewleonard42/SAC project root).  The reference cannot
// be compiled here (it is Fortran; no Fortran compiler exists on these machines),
// so its outputs cannot be produced: parity of this restatement is unpinned by
// reference outputs.  It is pinned instead by the reference's own initial-data
// scripts (inipar/*.py, run to make tests/golden fixtures), by numpy
// transcriptions of the Fortran array statements of centdiff4, addsource_visc
// with setnu, the gravity, Powell and resistive sources, the first getdt,
// getboundary, keeppositive and, composed from them, a whole RK4 step, each
// equal to this file's result bit for bit (tests/test_oracle_centdiff.py,
// tests/test_oracle_visc.py, tests/test_oracle_sources.py,
// tests/test_oracle_boundaries.py, tests/test_oracle_keeppositive.py,
// tests/test_oracle_rk4.py), by physics invariants
// (tests/test_oracle_physics.py) and by the independently written per-cell CUDA
// path agreeing with it to 1e-12 (tests/test_gpu_*.py).
//
// Indexing: 0-based, w[iw*ncell + i1 + n1*(i2 + n2*i3)], i.e. the reference's
// Fortran layout w(ix1,ix2,ix3,iw) with x1 fastest.  Dimension d = idim-1.
// Arithmetic follows the Fortran expressions' evaluation order (left to right,
// parenthesised as written) so that results agree to rounding; build with
// -O2 -ffp-contract=off -fno-fast-math.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "sac_gpu.h"

namespace {

constexpr double smalldouble = 1.0e-99, bigdouble = 1.0e99;  // src/vacdef.t:50
// src/vacdef.t:49 declares pi with a default-real (single precision) literal, so
// the stored DOUBLE PRECISION value is the float 3.1415927 widened.
const double pi_ref = (double)3.1415926535897932384626433832795f;

struct Rg {
  int lo[3], hi[3];
};

struct Oracle {
  sac_params par{};
  int ndim = 0, ndir = 0, nw = 0, dixB = 2;
  int nG[3] = {1, 1, 1};
  long ncell = 0;
  long st[3] = {0, 0, 0};  // strides per dimension
  Rg ixG{}, ixM{};
  bool fullgridini = false;
  // variable indices, src/vacpar.t.mhd:9-13
  int rho_ = 0, m0_ = 0, e_ = 0, b0_ = 0, eb_ = 0, rhob_ = 0, bg0_ = 0;
  std::vector<double> x, dx, dvolume;
  double volume = 0;
  // boundaries, src/vacdef.t:107-111
  int nB = 0;
  std::vector<std::string> typeB;  // typeB[iw + nw*iB]
  int idimB[SAC_NHIB]{}, ipairB[SAC_NHIB]{};
  bool upperB[SAC_NHIB]{};
  Rg ixB[SAC_NHIB]{};
  std::vector<double> fixB[SAC_NHIB];
  std::vector<char> fixedB;
  bool bc_initialized = false;  // the SAVEd 'initialized' of getboundary
  bool grid_set = false, bc_set = false, state_set = false;
  // state and the reference's RK scratch arrays
  std::vector<double> w, w1, w2, w3;
  // globals touched on the path
  double maxviscoef = 0;  // src/vacdef.t:176
  double dtgrav = bigdouble;
  double dtold = 0;
  double ctot_last[3] = {0, 0, 0};
  int itmin = 0;
  bool itmin_set = false;
  int it_now = 0;  // the step number last passed to getdt or advect
  // nerror(toosmallp_) and what the first keeppositive error reports, src/vacphys.t.mhd:34-41
  int nerror_toosmallp = 0, toosmallp_it = 0;
  double toosmallp_min = 0;
  std::string err;

  long id(int i, int j, int k) const { return i + (long)nG[0] * (j + (long)nG[1] * k); }
  double* V(std::vector<double>& a, int iw) { return a.data() + (long)iw * ncell; }
  const double* V(const std::vector<double>& a, int iw) const { return a.data() + (long)iw * ncell; }
  int coord(long c, int d) const {
    if (d == 0) return (int)(c % nG[0]);
    if (d == 1) return (int)((c / nG[0]) % nG[1]);
    return (int)(c / ((long)nG[0] * nG[1]));
  }
  bool isM(long c) const {
    for (int d = 0; d < ndim; ++d) {
      int q = coord(c, d);
      if (q < ixM.lo[d] || q > ixM.hi[d]) return false;
    }
    return true;
  }
  const std::string& tB(int iw, int iB) const { return typeB[iw + (long)nw * iB]; }
};

template <class F>
void forR(const Oracle& o, const Rg& r, F f) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = r.lo[2]; k <= r.hi[2]; ++k)
    for (int j = r.lo[1]; j <= r.hi[1]; ++j)
      for (int i = r.lo[0]; i <= r.hi[0]; ++i) f(o.id(i, j, k));
}

Rg grow(const Oracle& o, Rg r, int n) {  // ix^L^LADDn in the used dims
  for (int d = 0; d < o.ndim; ++d) {
    r.lo[d] -= n;
    r.hi[d] += n;
  }
  return r;
}
Rg grow1(Rg r, int d, int n) {  // ix^L^LADDn*kr(idim,^D)
  r.lo[d] -= n;
  r.hi[d] += n;
  return r;
}

// ---------------------------------------------------------------------------
// physics, src/vacphys0.t.mhd and src/vacphys.mhd0.t
// ---------------------------------------------------------------------------
using Arr = std::vector<double>;

// getv, src/vacphys0.t.mhd:55-73
void getv(const Oracle& o, const Arr& w, const Rg& ix, int d, Arr& v) {
  const double *m = o.V(w, o.m0_ + 1 + d), *r = o.V(w, o.rho_), *rb = o.V(w, o.rhob_);
  forR(o, ix, [&](long c) { v[c] = m[c] / (r[c] + rb[c]); });
}

// getptotal, src/vacphys0.t.mhd:186-205
void getptotal(const Oracle& o, const Arr& w, const Rg& ix, Arr& p) {
  const double g = o.par.gamma;
  forR(o, ix, [&](long c) {
    double bb = 0, b2 = 0, m2 = 0;
    for (int C = 1; C <= o.ndir; ++C) bb += o.V(w, o.b0_ + C)[c] * o.V(w, o.bg0_ + C)[c];
    for (int C = 1; C <= o.ndir; ++C) b2 += o.V(w, o.b0_ + C)[c] * o.V(w, o.b0_ + C)[c];
    for (int C = 1; C <= o.ndir; ++C) m2 += o.V(w, o.m0_ + C)[c] * o.V(w, o.m0_ + C)[c];
    double pp = (g - 2.0) * (bb + 0.5 * b2);
    p[c] = (g - 1.0) * (o.V(w, o.e_)[c] - 0.5 * m2 / (o.V(w, o.rho_)[c] + o.V(w, o.rhob_)[c])) - pp;
  });
}

// getptotal_bg, src/vacphys0.t.mhd:208-224
void getptotal_bg(const Oracle& o, const Arr& w, const Rg& ix, Arr& p) {
  const double g = o.par.gamma;
  forR(o, ix, [&](long c) {
    double s = 0;
    for (int C = 1; C <= o.ndir; ++C) s += o.V(w, o.bg0_ + C)[c] * o.V(w, o.bg0_ + C)[c];
    p[c] = (g - 1.0) * o.V(w, o.eb_)[c] - 0.5 * (g - 2.0) * s;
  });
}

// getpthermal, src/vacphys0.t.mhd:163-183
void getpthermal(const Oracle& o, const Arr& w, const Rg& ix, Arr& p) {
  const double g = o.par.gamma;
  forR(o, ix, [&](long c) {
    double m2 = 0, b2 = 0, bb = 0;
    for (int C = 1; C <= o.ndir; ++C) m2 += o.V(w, o.m0_ + C)[c] * o.V(w, o.m0_ + C)[c];
    double q = 0.5 * m2 / (o.V(w, o.rho_)[c] + o.V(w, o.rhob_)[c]);
    for (int C = 1; C <= o.ndir; ++C) b2 += o.V(w, o.b0_ + C)[c] * o.V(w, o.b0_ + C)[c];
    for (int C = 1; C <= o.ndir; ++C) bb += o.V(w, o.b0_ + C)[c] * o.V(w, o.bg0_ + C)[c];
    q = q + 0.5 * b2 + bb;
    p[c] = (g - 1.0) * (o.V(w, o.e_)[c] - q);
  });
}

// getcsound2, src/vacphys0.t.mhd:137-160
void getcsound2(const Oracle& o, const Arr& w, const Rg& ix, Arr& cs2) {
  getpthermal(o, w, ix, cs2);
  const double g = o.par.gamma;
  forR(o, ix, [&](long c) {
    double s = 0;
    for (int C = 1; C <= o.ndir; ++C) s += o.V(w, o.bg0_ + C)[c] * o.V(w, o.bg0_ + C)[c];
    cs2[c] = g * (cs2[c] + (g - 1.0) * (o.V(w, o.eb_)[c] - 0.5 * s)) /
             (o.V(w, o.rho_)[c] + o.V(w, o.rhob_)[c]);
  });
}

// getcmax, src/vacphys0.t.mhd:77-112.  The direction-independent part (csound2,
// cfast2) is recomputed when new_cmax is set, as in the reference.
struct CmaxCache {
  Arr cs2, cf2;
};
void getcmax(const Oracle& o, bool& new_cmax, const Arr& w, const Rg& ix, int d, Arr& cmax,
             CmaxCache& cc) {
  if (cc.cs2.size() != (size_t)o.ncell) {
    cc.cs2.assign(o.ncell, 0.0);
    cc.cf2.assign(o.ncell, 0.0);
  }
  if (new_cmax) {
    new_cmax = false;
    getcsound2(o, w, ix, cc.cs2);
    forR(o, ix, [&](long c) {
      double s = 0;
      for (int C = 1; C <= o.ndir; ++C) {
        double B = o.V(w, o.b0_ + C)[c] + o.V(w, o.bg0_ + C)[c];
        s += B * B;
      }
      cc.cf2[c] = s / (o.V(w, o.rho_)[c] + o.V(w, o.rhob_)[c]) + cc.cs2[c];
    });
  }
  forR(o, ix, [&](long c) {
    double rt = o.V(w, o.rho_)[c] + o.V(w, o.rhob_)[c];
    double Bd = o.V(w, o.b0_ + 1 + d)[c] + o.V(w, o.bg0_ + 1 + d)[c];
    double cf2 = cc.cf2[c];
    cmax[c] = std::sqrt(0.5 * (cf2 + std::sqrt(cf2 * cf2 - 4.0 * cc.cs2[c] * (Bd * Bd) / rt))) +
              std::fabs(o.V(w, o.m0_ + 1 + d)[c] / rt);
  });
}

// getflux, src/vacphys.mhd0.t:147-222.  iw is 0-based; returns 'transport'.
bool getflux(const Oracle& o, const Arr& w, const Rg& ix, int iw, int d, Arr& f, Arr& fbuf) {
  const int D = d + 1;
  const double *rho = o.V(w, o.rho_), *rhob = o.V(w, o.rhob_);
  const double *md = o.V(w, o.m0_ + D), *bd = o.V(w, o.b0_ + D), *bgd = o.V(w, o.bg0_ + D);
  if (iw == o.rho_) {
    forR(o, ix, [&](long c) { f[c] = rhob[c] * md[c] / (rho[c] + rhob[c]); });
    return true;
  }
  if (iw > o.m0_ && iw <= o.m0_ + o.ndir) {
    const int C = iw - o.m0_;
    const double *bC = o.V(w, o.b0_ + C), *bgC = o.V(w, o.bg0_ + C);
    if (D == C) {
      getptotal(o, w, ix, f);
      // getptotal_bg is called and its result zeroed (fb=0.d0, :174-175)
      forR(o, ix, [&](long c) {
        f[c] = (f[c] + 0.0) - (bC[c] * bgd[c] + bd[c] * bgC[c]) - bC[c] * bd[c];
      });
    } else {
      forR(o, ix, [&](long c) { f[c] = -(bC[c] * bgd[c] + bd[c] * bgC[c]) - bC[c] * bd[c]; });
    }
    return true;
  }
  if (iw == o.e_) {
    getptotal(o, w, ix, f);
    const double* eb = o.V(w, o.eb_);
    forR(o, ix, [&](long c) {
      double s1 = 0, s2 = 0;
      for (int C = 1; C <= o.ndir; ++C) s1 += o.V(w, o.bg0_ + C)[c] * o.V(w, o.m0_ + C)[c];
      for (int C = 1; C <= o.ndir; ++C) s2 += o.V(w, o.b0_ + C)[c] * o.V(w, o.m0_ + C)[c];
      double rt = rho[c] + rhob[c];
      f[c] = (md[c] * (f[c] + 0.0) - bd[c] * s1 - bgd[c] * s2) / rt + eb[c] * md[c] / rt -
             bd[c] * s2 / rt;
    });
    return true;
  }
  if (iw > o.b0_ && iw <= o.b0_ + o.ndir) {
    const int C = iw - o.b0_;
    if (D == C) {
      forR(o, ix, [&](long c) { f[c] = 0.0; });
      return false;
    }
    const double *mC = o.V(w, o.m0_ + C), *bgC = o.V(w, o.bg0_ + C);
    forR(o, ix, [&](long c) {
      double rt = rho[c] + rhob[c];
      f[c] = -(mC[c] / rt * (bd[c] + bgd[c])) + md[c] / rt * bgC[c];
    });
    return true;
  }
  (void)fbuf;
  return false;
}

// ---------------------------------------------------------------------------
// finite differences
// ---------------------------------------------------------------------------
// gradient4, src/vacgrid.t:665-712: zero the two edge layers at every boundary
// that is not 'mpi' (all boundaries on one device).
void gradient4(const Oracle& o, const Arr& q, const Rg& ix, int d, Arr& g) {
  const long s = o.st[d];
  const double* dxd = o.dx.data() + (long)d * o.ncell;
  forR(o, ix, [&](long c) {
    g[c] = -(q[c + 2 * s] - 8.0 * (q[c + s] - q[c - s]) - q[c - 2 * s]) / dxd[c] / 12.0;
  });
  for (int k = 0; k < 2; ++k) {
    int iB = 2 * d + k;
    if (o.tB(0, iB) == "mpi") continue;
    Rg p = ix;
    if (o.upperB[iB]) {
      for (int q2 = ix.hi[d] - 1; q2 <= ix.hi[d]; ++q2) {
        p.lo[d] = p.hi[d] = q2;
        forR(o, p, [&](long c) { g[c] = 0.0; });
      }
    } else {
      for (int q2 = ix.lo[d]; q2 <= ix.lo[d] + 1; ++q2) {
        p.lo[d] = p.hi[d] = q2;
        forR(o, p, [&](long c) { g[c] = 0.0; });
      }
    }
  }
}

// gradient1 / gradient1L / gradient1R, src/vacusr.viscosity.t:547-675: two-point
// differences, the two edge layers of ix zeroed at boundaries that are neither
// 'periodic' nor 'mpi' (checked on typeB(1,iB)).
enum GKind { G_C, G_L, G_R };
void gradient1x(const Oracle& o, GKind kind, const Arr& q, const Rg& ix, int d, Arr& g) {
  const long s = o.st[d];
  const double* dxd = o.dx.data() + (long)d * o.ncell;
  if (kind == G_C)
    forR(o, ix, [&](long c) { g[c] = (q[c + s] - q[c - s]) / dxd[c] / 2.0; });
  else if (kind == G_L)
    forR(o, ix, [&](long c) { g[c] = (q[c] - q[c - s]) / dxd[c]; });
  else
    forR(o, ix, [&](long c) { g[c] = (q[c + s] - q[c]) / dxd[c]; });
  for (int k = 0; k < 2; ++k) {
    int iB = 2 * d + k;
    if (o.tB(0, iB) == "periodic" || o.tB(0, iB) == "mpi") continue;
    Rg p = ix;
    int a = o.upperB[iB] ? ix.hi[d] - 1 : ix.lo[d];
    for (int q2 = a; q2 <= a + 1; ++q2) {
      p.lo[d] = p.hi[d] = q2;
      forR(o, p, [&](long c) { g[c] = 0.0; });
    }
  }
}

// ---------------------------------------------------------------------------
// hyperdiffusion, src/vacusr.viscosity.t
// ---------------------------------------------------------------------------
const int IW173 = 173;  // the reference's tag for e - b^2/2 - m^2/(2 rho)

// setnu, src/vacusr.viscosity.t:224-455, for ix = ixM.  nuR/nuL are written on the
// mesh only and are zero elsewhere (the reference leaves them undefined there).
void setnu(Oracle& o, const Arr& w, int iw, int d, Arr& nuR, Arr& nuL, CmaxCache& cc, Arr& cmax,
           Arr& tmp_nu) {
  bool new_cmax = true;
  getcmax(o, new_cmax, w, o.ixM, d, cmax, cc);
  double c_tot = 0;
  {
    double m = -bigdouble;
    for (int k = o.ixM.lo[2]; k <= o.ixM.hi[2]; ++k)
      for (int j = o.ixM.lo[1]; j <= o.ixM.hi[1]; ++j)
        for (int i = o.ixM.lo[0]; i <= o.ixM.hi[0]; ++i) m = std::max(m, cmax[o.id(i, j, k)]);
    c_tot = m;
  }
  o.ctot_last[d] = c_tot;
  double c_hyp = 0.4;
  if (iw > o.b0_ && iw <= o.b0_ + o.ndim) c_hyp = 0.04;
  if (iw == o.rho_) c_hyp = 0.04;
  if (iw == IW173) c_hyp = 0.04;

  if (iw != IW173) {
    const double* q = o.V(w, iw);
    forR(o, o.ixG, [&](long c) { tmp_nu[c] = q[c]; });
    if (iw > o.m0_ && iw <= o.m0_ + o.ndim) {
      const double *r = o.V(w, o.rho_), *rb = o.V(w, o.rhob_);
      forR(o, o.ixG, [&](long c) { tmp_nu[c] = q[c] / (r[c] + rb[c]); });
    }
  } else {
    forR(o, o.ixG, [&](long c) {
      double b2 = 0, m2 = 0;
      for (int C = 1; C <= o.ndir; ++C) b2 += o.V(w, o.b0_ + C)[c] * o.V(w, o.b0_ + C)[c];
      for (int C = 1; C <= o.ndir; ++C) m2 += o.V(w, o.m0_ + C)[c] * o.V(w, o.m0_ + C)[c];
      tmp_nu[c] = o.V(w, o.e_)[c] -
                  0.5 * (b2 + m2 / (o.V(w, o.rho_)[c] + o.V(w, o.rhob_)[c]));
    });
  }
  const int iwc = (iw == IW173) ? o.e_ : iw;
  // third ghost layer: tmp_nuI(ixFlo-1)=tmp_nuI(ixFlo+5) and
  // tmp_nuI(ixFhi+1)=tmp_nuI(ixFhi-5), i.e. q(ixMmin-3)=q(ixMmin+3) and
  // q(ixMmax+3)=q(ixMmax-3) at every non-'mpi' boundary (:378-400)
  const bool mirror_lo = o.tB(iwc, 2 * d) != "mpi";
  const bool mirror_hi = o.tB(iwc, 2 * d + 1) != "mpi";
  const int lo = o.ixM.lo[d], hi = o.ixM.hi[d];
  const long s = o.st[d];
  const double* dxd = o.dx.data() + (long)d * o.ncell;
  const double pre = c_tot * c_hyp;
  double mv = o.maxviscoef;
#pragma omp parallel for collapse(2) schedule(static) reduction(max : mv)
  for (int k = o.ixM.lo[2]; k <= o.ixM.hi[2]; ++k)
    for (int j = o.ixM.lo[1]; j <= o.ixM.hi[1]; ++j)
      for (int i = o.ixM.lo[0]; i <= o.ixM.hi[0]; ++i) {
        const long c = o.id(i, j, k);
        const int pos = o.coord(c, d);
        auto q = [&](int a) -> double {  // tmp_nu at offset a along d, third layer mirrored
          int p = pos + a;
          if (p == lo - 3 && mirror_lo) p = lo + 3;
          if (p == hi + 3 && mirror_hi) p = hi - 3;
          return tmp_nu[c + (long)(p - pos) * s];
        };
        auto d3R = [&](int a) { return std::fabs(3.0 * (q(a + 1) - q(a)) - (q(a + 2) - q(a - 1))); };
        auto d1R = [&](int a) { return std::fabs(q(a + 1) - q(a)); };
        auto d3L = [&](int a) { return std::fabs(3.0 * (q(a) - q(a - 1)) - (q(a + 1) - q(a - 2))); };
        auto d1L = [&](int a) { return std::fabs(q(a) - q(a - 1)); };
        double md3R = std::max(std::max(d3R(-1), d3R(0)), d3R(1));
        double md1R = std::max(std::max(std::max(std::max(d1R(-2), d1R(-1)), d1R(0)), d1R(1)), d1R(2));
        double md3L = std::max(std::max(d3L(-1), d3L(0)), d3L(1));
        double md1L = std::max(std::max(std::max(std::max(d1L(-2), d1L(-1)), d1L(0)), d1L(1)), d1L(2));
        double nr = (md1R > 0.0) ? pre * md3R / md1R * dxd[c] : 0.0;
        double nl = (md1L > 0.0) ? pre * md3L / md1L * dxd[c] : 0.0;
        nuR[c] = nr;
        nuL[c] = nl;
        mv = std::max(mv, std::max(nr, nl));
      }
  o.maxviscoef = mv;
}

struct ViscWork {
  Arr tmp, tmp2, tmpL, tmpR, tmpC, nuL, nuR, rhoL, rhoR, rhoC, VL, VR, BL, BR, cmax, tmp_nu, prod;
  CmaxCache cc;
  void init(long n) {
    for (Arr* a : {&tmp, &tmp2, &tmpL, &tmpR, &tmpC, &nuL, &nuR, &rhoL, &rhoR, &rhoC, &VL, &VR,
                   &BL, &BR, &cmax, &tmp_nu, &prod})
      if ((long)a->size() != n) a->assign(n, 0.0);
  }
};

// addsource_visc, src/vacusr.viscosity.t:2-221, with ixO=ixM (the reference's
// ensurebound(2,...) never widens it) and ix=ixM+-1.  Updates wnew on the mesh;
// the ghost layers, which the reference fills with values that getboundary then
// overwrites, are left untouched.
void addsource_visc(Oracle& o, double qdt, const Arr& w, Arr& wnew, ViscWork& vw) {
  vw.init(o.ncell);
  const Rg ixM = o.ixM;
  const Rg ix = grow(o, ixM, 1);
  auto zero = [&](Arr& a) { std::fill(a.begin(), a.end(), 0.0); };
  auto dxp = [&](int d) { return o.dx.data() + (long)d * o.ncell; };
  // setnushk (:460-504): the shock-viscosity body is commented out, nushk = 0.

  // density, :45-53
  for (int d = 0; d < o.ndim; ++d) {
    forR(o, o.ixG, [&](long c) { vw.tmp[c] = o.V(w, o.rho_)[c]; });
    setnu(o, w, o.rho_, d, vw.nuR, vw.nuL, vw.cc, vw.cmax, vw.tmp_nu);
    gradient1x(o, G_L, vw.tmp, ix, d, vw.tmp2);
    forR(o, ixM, [&](long c) { vw.tmpL[c] = (vw.nuL[c] + 0.0) * vw.tmp2[c]; });
    gradient1x(o, G_R, vw.tmp, ix, d, vw.tmp2);
    forR(o, ixM, [&](long c) { vw.tmpR[c] = (vw.nuR[c] + 0.0) * vw.tmp2[c]; });
    double* wr = o.V(wnew, o.rho_);
    const double* dd = dxp(d);
    forR(o, ixM, [&](long c) { wr[c] = wr[c] + (vw.tmpR[c] - vw.tmpL[c]) / dd[c] * qdt; });
  }
  // energy with q = e - b^2/2 - m^2/(2 rho), :56-64
  for (int d = 0; d < o.ndim; ++d) {
    forR(o, o.ixG, [&](long c) {
      double b2 = 0, m2 = 0;
      for (int C = 1; C <= o.ndir; ++C) b2 += o.V(w, o.b0_ + C)[c] * o.V(w, o.b0_ + C)[c];
      for (int C = 1; C <= o.ndir; ++C) m2 += o.V(w, o.m0_ + C)[c] * o.V(w, o.m0_ + C)[c];
      vw.tmp[c] = o.V(w, o.e_)[c] - 0.5 * (b2 + m2 / (o.V(w, o.rho_)[c] + o.V(w, o.rhob_)[c]));
    });
    setnu(o, w, IW173, d, vw.nuR, vw.nuL, vw.cc, vw.cmax, vw.tmp_nu);
    gradient1x(o, G_L, vw.tmp, ix, d, vw.tmp2);
    forR(o, ixM, [&](long c) { vw.tmpL[c] = (vw.nuL[c] + 0.0) * vw.tmp2[c]; });
    gradient1x(o, G_R, vw.tmp, ix, d, vw.tmp2);
    forR(o, ixM, [&](long c) { vw.tmpR[c] = (vw.nuR[c] + 0.0) * vw.tmp2[c]; });
    double* we = o.V(wnew, o.e_);
    const double* dd = dxp(d);
    forR(o, ixM, [&](long c) { we[c] = we[c] + (vw.tmpR[c] - vw.tmpL[c]) / dd[c] * qdt; });
  }
  // momentum, :69-133
  forR(o, o.ixG, [&](long c) { vw.rhoC[c] = o.V(w, o.rho_)[c] + o.V(w, o.rhob_)[c]; });
  for (int k = 0; k < o.ndim; ++k) {
    const long sk = o.st[k];
    forR(o, ix, [&](long c) {
      vw.rhoL[c] = (vw.rhoC[c] + vw.rhoC[c - sk]) / 2.0;
      vw.rhoR[c] = (vw.rhoC[c + sk] + vw.rhoC[c]) / 2.0;
    });
    for (int l = 0; l < o.ndim; ++l) {
      setnu(o, w, o.m0_ + 1 + l, k, vw.nuR, vw.nuL, vw.cc, vw.cmax, vw.tmp_nu);
      forR(o, o.ixG, [&](long c) { vw.tmp[c] = o.V(w, o.m0_ + 1 + l)[c] / vw.rhoC[c]; });
      for (int ii1 = 0; ii1 <= 1; ++ii1) {
        int i_, ii0;
        if (ii1 == 0) {
          i_ = k;
          ii0 = l;
        } else {
          i_ = l;
          ii0 = k;
        }
        if (i_ == k) {
          const double* mi = o.V(w, o.m0_ + 1 + ii0);
          forR(o, ix, [&](long c) {
            vw.VL[c] = (mi[c] + mi[c - sk]) / 2.0;
            vw.VR[c] = (mi[c + sk] + mi[c]) / 2.0;
          });
          gradient1x(o, G_L, vw.tmp, ix, k, vw.tmp2);
          forR(o, ixM, [&](long c) { vw.tmpL[c] = (vw.nuL[c] + 0.0) * vw.tmp2[c]; });
          gradient1x(o, G_R, vw.tmp, ix, k, vw.tmp2);
          forR(o, ixM, [&](long c) { vw.tmpR[c] = (vw.nuR[c] + 0.0) * vw.tmp2[c]; });
          const double* dd = dxp(k);
          double* wm = o.V(wnew, o.m0_ + 1 + ii0);
          double* we = o.V(wnew, o.e_);
          forR(o, ixM, [&](long c) {
            double t2 = (vw.rhoR[c] * vw.tmpR[c] - vw.rhoL[c] * vw.tmpL[c]) / dd[c] / 2.0;
            wm[c] = wm[c] + t2 * qdt;
            t2 = (vw.VR[c] * vw.tmpR[c] - vw.VL[c] * vw.tmpL[c]) / dd[c] / 2.0;
            we[c] = we[c] + t2 * qdt;
          });
        }
        if (i_ != k) {
          zero(vw.tmp2);
          gradient1x(o, G_C, vw.tmp, ix, k, vw.tmp2);
          // nu (and nushk) vanish outside the mesh
          forR(o, o.ixG, [&](long c) {
            vw.tmp2[c] = vw.tmp2[c] * (vw.nuL[c] + vw.nuR[c] + 2.0 * 0.0) / 2.0 / 2.0;
          });
          Arr& T = vw.tmpC;
          Arr& prod = vw.prod;  // the reference's tmp=rhoC*tmp2; tmp=v_l is kept apart
          forR(o, o.ixG, [&](long c) { prod[c] = vw.rhoC[c] * vw.tmp2[c]; });
          gradient1x(o, G_C, prod, ix, i_, T);
          double* wm = o.V(wnew, o.m0_ + 1 + ii0);
          forR(o, ixM, [&](long c) { wm[c] = wm[c] + T[c] * qdt; });
          const double* mi = o.V(w, o.m0_ + 1 + ii0);
          forR(o, o.ixG, [&](long c) { prod[c] = mi[c] * vw.tmp2[c]; });
          gradient1x(o, G_C, prod, ix, i_, T);
          double* we = o.V(wnew, o.e_);
          forR(o, ixM, [&](long c) { we[c] = we[c] + T[c] * qdt; });
          // the reference leaves tmp = m_ii0*tmp2 here; it is reassigned to v_l
          // only at the next l, and ii1=1 is the last use for this l.
        }
      }
    }
  }
  // magnetic field, :139-215
  for (int k = 0; k < o.ndim; ++k)
    for (int l = 0; l < o.ndim; ++l) {
      if (k == l) continue;
      setnu(o, w, o.b0_ + 1 + l, k, vw.nuR, vw.nuL, vw.cc, vw.cmax, vw.tmp_nu);
      for (int ii1 = 0; ii1 <= 1; ++ii1) {
        int ii0, m, j_;
        double sB;
        if (ii1 == 0) {
          ii0 = k;
          m = l;
          sB = -1.0;
          j_ = k;
        } else {
          ii0 = l;
          m = k;
          sB = 1.0;
          j_ = l;
        }
        const double* bl = o.V(w, o.b0_ + 1 + l);
        const double* bj = o.V(w, o.b0_ + 1 + j_);
        if (m == k) {
          const long sm = o.st[m];
          forR(o, ix, [&](long c) {
            vw.BL[c] = (bj[c] + bj[c - sm]) / 2.0;
            vw.BR[c] = (bj[c + sm] + bj[c]) / 2.0;
          });
          forR(o, o.ixG, [&](long c) { vw.tmp[c] = bl[c]; });
          gradient1x(o, G_L, vw.tmp, ix, k, vw.tmp2);
          forR(o, ixM, [&](long c) { vw.tmpL[c] = vw.nuL[c] * vw.tmp2[c]; });
          gradient1x(o, G_R, vw.tmp, ix, k, vw.tmp2);
          forR(o, ixM, [&](long c) { vw.tmpR[c] = vw.nuR[c] * vw.tmp2[c]; });
          const double* dd = dxp(k);
          double* wb = o.V(wnew, o.b0_ + 1 + ii0);
          double* we = o.V(wnew, o.e_);
          forR(o, ixM, [&](long c) {
            wb[c] = wb[c] + sB * (vw.tmpR[c] - vw.tmpL[c]) / dd[c] * qdt;
            we[c] = we[c] + sB * (vw.tmpR[c] * vw.BR[c] - vw.tmpL[c] * vw.BL[c]) / dd[c] * qdt;
          });
        }
        if (m != k) {
          forR(o, o.ixG, [&](long c) { vw.tmp[c] = bl[c]; });
          zero(vw.tmp2);
          gradient1x(o, G_C, vw.tmp, ix, k, vw.tmp2);
          forR(o, o.ixG, [&](long c) { vw.tmp2[c] = vw.tmp2[c] * (vw.nuL[c] + vw.nuR[c]) / 2.0; });
          gradient1x(o, G_C, vw.tmp2, ix, m, vw.tmpC);
          double* wb = o.V(wnew, o.b0_ + 1 + ii0);
          forR(o, ixM, [&](long c) { wb[c] = wb[c] + sB * vw.tmpC[c] * qdt; });
          forR(o, o.ixG, [&](long c) { vw.tmp2[c] = vw.tmp2[c] * bj[c]; });
          gradient1x(o, G_C, vw.tmp2, ix, m, vw.tmpC);
          double* we = o.V(wnew, o.e_);
          forR(o, ixM, [&](long c) { we[c] = we[c] + sB * vw.tmpC[c] * qdt; });
        }
      }
    }
}

// addsource_grav, src/vacusr.gravity.t:24-81
void addsource_grav(Oracle& o, double qdt, const std::vector<int>& iws, const Arr& w, Arr& wnew,
                    const double g[3]) {
  const double *rho = o.V(w, o.rho_), *rhob = o.V(w, o.rhob_);
  for (int iw : iws) {
    if (iw > o.m0_ && iw <= o.m0_ + o.ndim) {
      int d = iw - o.m0_ - 1;
      if (std::fabs(g[d]) > smalldouble) {
        double* wm = o.V(wnew, iw);
        forR(o, o.ixM, [&](long c) { wm[c] = wm[c] + qdt * g[d] * rho[c]; });
      }
    } else if (iw == o.e_) {
      for (int d = 0; d < o.ndim; ++d)
        if (std::fabs(g[d]) > smalldouble) {
          double* we = o.V(wnew, o.e_);
          const double* md = o.V(w, o.m0_ + 1 + d);
          forR(o, o.ixM, [&](long c) {
            we[c] = we[c] + qdt * g[d] * rho[c] * md[c] / (rho[c] + rhob[c]);
          });
        }
    }
  }
}

// ---------------------------------------------------------------------------
// user modules (specialsource), drivers
// ---------------------------------------------------------------------------
void effective_gravity(const Oracle& o, double g[3]) {
  for (int d = 0; d < 3; ++d) g[d] = (d < o.ndim) ? o.par.grav[d] : 0.0;
  // Slog's specialsource sets eqpar(nu_)=1 every call; with nu_=grav3_=6 in 3D
  // (src/vacusrpar.f:4-5) that forces g3=1.
  if (o.par.alias_nu_grav3 && o.ndim == 3) g[2] = 1.0;
}
bool visc_on(const Oracle& o) {
  if (o.par.user == SAC_USR_SLOG) return true;  // eqpar(nu_)=1.0d0, src/vacusr.f:1280
  return std::fabs(o.par.nu) > smalldouble;
}
bool grav_in_module(int user) {
  return user == SAC_USR_SLOG || user == SAC_USR_GRAVVISC || user == SAC_USR_STRAT ||
         user == SAC_USR_TUBE;
}

// Slog Gaussian vortex driver, src/vacusr.f:1294-1377 (3D, x1 vertical).  Several
// constants are default-real (single precision) literals in the reference and
// are reproduced as such.
void driver_slog(Oracle& o, double qdt, double qt, Arr& w) {
  const double xc1 = (double)0.1f * 1.0e6, xc2 = 1.0 * 1.0e6, xc3 = 1.0 * 1.0e6;
  const double delta_z = 0.05e6, delta_x = 0.5e6, delta_y = 0.5e6;
  const double AA = 10.0, B = (double)0.05f, s_period = 240.0;
  const double tdep = std::sin(qt * 2.0 * pi_ref / s_period);
  const double *x1 = o.x.data(), *x2 = o.x.data() + o.ncell, *x3 = o.x.data() + 2 * o.ncell;
  double *m2 = o.V(w, o.m0_ + 2), *m3 = o.V(w, o.m0_ + 3), *e = o.V(w, o.e_);
  const double *r = o.V(w, o.rho_), *rb = o.V(w, o.rhob_);
  forR(o, o.ixM, [&](long c) {
    double xx = x2[c] - xc2, yy = x3[c] - xc3, zz = x1[c] - xc1;
    double exp_z = std::exp(-(zz * zz) / (delta_z * delta_z));
    double exp_x = std::exp(-(xx * xx) / (delta_x * delta_x));
    double exp_y = std::exp(-(yy * yy) / (delta_y * delta_y));
    double exp_xyz = exp_x * exp_y * exp_z;
    double theta = std::atan2(yy, xx), phi = std::atan2(1.0, B);
    double ux = std::cos(theta + phi), uy = std::sin(theta + phi);
    double vvx = (ux / std::sqrt(ux * ux + uy * uy)) * exp_xyz * tdep * AA;
    double vvy = (uy / std::sqrt(ux * ux + uy * uy)) * exp_xyz * tdep * AA;
    double vvz = 0.0;
    m2[c] = m2[c] + (r[c] + rb[c]) * vvx * qdt;
    m3[c] = m3[c] + (r[c] + rb[c]) * vvy * qdt;
    e[c] = e[c] + (r[c] + rb[c]) * (vvx * vvx + vvy * vvy + vvz * vvz) * qdt / 2.0;
  });
}

// Velocity drivers of the stratified and flux-tube workloads, written in the
// Slog style (w_m += (rho+rhob)*v*qdt, e += (rho+rhob)*v^2/2*qdt, evaluated at qt).
void driver_gauss(Oracle& o, double qdt, double qt, Arr& w) {
  const double* up = o.par.userpar;
  const double A = up[0], om = up[1];
  const double tdep = std::sin(om * qt);
  double *r = o.V(w, o.rho_), *rb = o.V(w, o.rhob_), *e = o.V(w, o.e_);
  const double* x1 = o.x.data();
  if (o.par.user == SAC_USR_STRAT) {
    const double *x2 = o.x.data() + o.ncell, *x3 = o.x.data() + 2 * o.ncell;
    double* m1 = o.V(w, o.m0_ + 1);
    forR(o, o.ixM, [&](long c) {
      double xx = x2[c] - up[2], yy = (o.ndim > 2) ? x3[c] - up[3] : 0.0, zz = x1[c] - up[5];
      double v = A * tdep * std::exp(-(xx * xx + yy * yy) / (up[4] * up[4])) *
                 std::exp(-(zz * zz) / (up[6] * up[6]));
      m1[c] = m1[c] + (r[c] + rb[c]) * v * qdt;
      e[c] = e[c] + (r[c] + rb[c]) * (v * v) * qdt / 2.0;
    });
  } else {  // SAC_USR_TUBE
    const double* x2 = o.x.data() + o.ncell;
    double* m2 = o.V(w, o.m0_ + 2);
    forR(o, o.ixM, [&](long c) {
      double zz = x1[c] - up[2], xx = x2[c] - up[4];
      double v = A * tdep * std::exp(-(zz * zz) / (up[3] * up[3])) *
                 std::exp(-(xx * xx) / (up[5] * up[5]));
      m2[c] = m2[c] + (r[c] + rb[c]) * v * qdt;
      e[c] = e[c] + (r[c] + rb[c]) * (v * v) * qdt / 2.0;
    });
  }
}

struct Work {
  ViscWork vw;
  Arr v, f, fb, tmp, fbuf;
  void init(long n) {
    for (Arr* a : {&v, &f, &fb, &tmp, &fbuf})
      if ((long)a->size() != n) a->assign(n, 0.0);
  }
};

// specialsource: the user module, src/vacusr.f:1255-1382, sac/src/vacusr.t.stuart:46-72
void specialsource(Oracle& o, double qdt, const std::vector<int>& iws, double qtC, const Arr& wCT,
                   double qt, Arr& w, Work& wk) {
  (void)qtC;
  const int u = o.par.user;
  if (u == SAC_USR_NONE) return;
  double g[3];
  effective_gravity(o, g);
  if (grav_in_module(u)) addsource_grav(o, qdt, iws, wCT, w, g);
  if (visc_on(o)) addsource_visc(o, qdt, wCT, w, wk.vw);
  if (u == SAC_USR_SLOG && o.ndim == 3) driver_slog(o, qdt, qt, w);
  if (u == SAC_USR_STRAT || u == SAC_USR_TUBE) driver_gauss(o, qdt, qt, w);
}

// addsource_divb, src/vacphys.mhd0.t:263-297.  ensurebound(1,...) keeps ixO=ixM
// and ixI=ixG (the mesh has two ghost layers), so no boundary refill.  getdivb
// (:106-144) sums gradient4 of b+bg over every dimension; gradient4 zeroes the
// two edge layers, so the layer of b+bg it reads beyond ixO+1 never reaches the
// result and computing b+bg on the whole grid is equivalent.
void addsource_divb(Oracle& o, double qdt, const std::vector<int>& iws, const Arr& w, Arr& wnew, Work& wk) {
  wk.init(o.ncell);
  Arr &tmp = wk.f, &g = wk.tmp, &divb = wk.fb;
  forR(o, o.ixM, [&](long c) { divb[c] = 0.0; });
  for (int d = 0; d < o.ndim; ++d) {
    const double *b = o.V(w, o.b0_ + 1 + d), *bg = o.V(w, o.bg0_ + 1 + d);
    forR(o, o.ixG, [&](long c) { tmp[c] = b[c] + bg[c]; });
    gradient4(o, tmp, o.ixM, d, g);
    forR(o, o.ixM, [&](long c) { divb[c] = divb[c] + g[c]; });
  }
  forR(o, o.ixM, [&](long c) { divb[c] = qdt * divb[c]; });
  const double *r = o.V(w, o.rho_), *rb = o.V(w, o.rhob_);
  for (int iw : iws) {
    double* wn = o.V(wnew, iw);
    if (iw > o.m0_ && iw <= o.m0_ + o.ndir) {
      const int C = iw - o.m0_;
      const double *b = o.V(w, o.b0_ + C), *bg = o.V(w, o.bg0_ + C);
      forR(o, o.ixM, [&](long c) { wn[c] = wn[c] - (b[c] + bg[c]) * divb[c]; });
    } else if (iw > o.b0_ && iw <= o.b0_ + o.ndir) {
      const double* m = o.V(w, o.m0_ + (iw - o.b0_));
      forR(o, o.ixM, [&](long c) { wn[c] = wn[c] - m[c] / (r[c] + rb[c]) * divb[c]; });
    } else if (iw == o.e_) {
      forR(o, o.ixM, [&](long c) {
        double s = o.V(w, o.m0_ + 1)[c] * (o.V(w, o.b0_ + 1)[c] + o.V(w, o.bg0_ + 1)[c]);
        for (int C = 2; C <= o.ndir; ++C)
          s = s + o.V(w, o.m0_ + C)[c] * (o.V(w, o.b0_ + C)[c] + o.V(w, o.bg0_ + C)[c]);
        wn[c] = wn[c] - s / (r[c] + rb[c]) * divb[c];
      });
    }
  }
}

// Levi-Civita symbol lvc(i,j,k) of 0-based indices (src/vacdef.t:91)
int lvc(int i, int j, int k) {
  if (i == j || j == k || i == k) return 0;
  return ((i + 1) % 3 == j) ? 1 : -1;
}

// gradient of the resistive module, src/vacphys.mhdres.t:304-317: note the sign,
// -(q(+1)-q(-1))/dx/2; it enters every resistive term twice, or squared
void gradient_res(const Oracle& o, const Arr& q, const Rg& ix, int d, Arr& g) {
  const long s = o.st[d];
  const double* dxd = o.dx.data() + (long)d * o.ncell;
  forR(o, ix, [&](long c) { g[c] = -(q[c + s] - q[c - s]) / dxd[c] / 2.0; });
}

// getcurrent, src/vacphys.mhdres.t:48-95: J_i = sum eps_ijk gradient_j(b_k+bg_k)
// on ix for i >= idirmin0 = 7-2*ndir (1-based); returns idirmin (0-based, 3 when
// no component exists)
int getcurrent(const Oracle& o, const Arr& w, const Rg& ix, Arr J[3], Arr& tmp, Arr& g) {
  const int k0 = 6 - 2 * o.ndir;
  int idirmin = 3;
  for (int i = std::max(k0, 0); i < 3; ++i) forR(o, ix, [&](long c) { J[i][c] = 0.0; });
  for (int i = std::max(k0, 0); i < 3; ++i)
    for (int j = 0; j < o.ndim; ++j)
      for (int k = 0; k < o.ndir; ++k) {
        const int l = lvc(i, j, k);
        if (l == 0) continue;
        const double *b = o.V(w, o.b0_ + 1 + k), *bg = o.V(w, o.bg0_ + 1 + k);
        forR(o, grow(o, ix, 1), [&](long c) { tmp[c] = b[c] + bg[c]; });
        gradient_res(o, tmp, ix, j, g);
        if (l == 1)
          forR(o, ix, [&](long c) { J[i][c] = J[i][c] + g[c]; });
        else
          forR(o, ix, [&](long c) { J[i][c] = J[i][c] - g[c]; });
        idirmin = std::min(idirmin, i);
      }
  return idirmin;
}

// addsource_res2, src/vacphys.mhdres.t:231-301, for a constant eta =
// eqpar(eta_) > 0 (eta < 0 needs a user specialeta and is rejected).
// ensurebound(2,...) keeps ixO=ixM, and ix=ixM+1.
void addsource_res2(Oracle& o, double qdt, const std::vector<int>& iws, const Arr& w, Arr& wnew, Work& wk) {
  wk.init(o.ncell);
  const long n = o.ncell;
  Arr J[3];
  for (Arr& a : J) a.assign(n, 0.0);
  const Rg ixO = o.ixM, ix = grow(o, ixO, 1);
  const int idirmin = getcurrent(o, w, ix, J, wk.f, wk.tmp);
  const double eta = o.par.eta;
  Arr &tmp = wk.f, &tmp2 = wk.tmp;
  for (int iw : iws) {
    if (iw > o.b0_ && iw <= o.b0_ + o.ndir) {
      const int i = iw - o.b0_ - 1;
      double* wn = o.V(wnew, iw);
      for (int j = 0; j < o.ndim; ++j)
        for (int k = idirmin; k < 3; ++k) {
          const int l = lvc(i, j, k);
          if (l == 0) continue;
          forR(o, ix, [&](long c) { tmp[c] = J[k][c] * eta * qdt; });
          gradient_res(o, tmp, ixO, j, tmp2);
          if (l == 1)
            forR(o, ixO, [&](long c) { wn[c] = wn[c] - tmp2[c]; });
          else
            forR(o, ixO, [&](long c) { wn[c] = wn[c] + tmp2[c]; });
        }
    } else if (iw == o.e_) {
      double* wn = o.V(wnew, iw);
      for (int i = 0; i < o.ndim; ++i)
        for (int j = 0; j < o.ndir; ++j)
          for (int k = idirmin; k < 3; ++k) {
            const int l = lvc(i, j, k);
            if (l == 0) continue;
            const double *b = o.V(w, o.b0_ + 1 + j), *bg = o.V(w, o.bg0_ + 1 + j);
            forR(o, ix, [&](long c) { tmp[c] = (b[c] + bg[c]) * J[k][c] * eta * qdt; });
            gradient_res(o, tmp, ixO, i, tmp2);
            if (l == 1)
              forR(o, ixO, [&](long c) { wn[c] = wn[c] + tmp2[c]; });
            else
              forR(o, ixO, [&](long c) { wn[c] = wn[c] - tmp2[c]; });
          }
    }
  }
}

// addsource_res1, src/vacphys.mhdres.t:96-220 (compactres=T), for a constant
// eta = eqpar(eta_) > 0: ensurebound(1,...) keeps ixO=ixM, and getcurrent runs on
// ixO.  Per idir: tmp = eta * sum over idim of the 3-point Laplacian of
// B_idir = b_idir + bg_idir, added to b_idir and, times B_idir, to e; then
// eta * J**2 to e.
void addsource_res1(Oracle& o, double qdt, const std::vector<int>& iws, const Arr& w, Arr& wnew, Work& wk) {
  wk.init(o.ncell);
  const long n = o.ncell;
  Arr J[3];
  for (Arr& a : J) a.assign(n, 0.0);
  const Rg ixO = o.ixM;
  const int idirmin = getcurrent(o, w, ixO, J, wk.f, wk.tmp);
  const double eta = o.par.eta;  // eta(ixG^S)=eqpar(eta_), set at it==itmin (:121-122)
  Arr &tmp = wk.f, &tmp2 = wk.tmp;
  for (int idir = 0; idir < o.ndir; ++idir) {
    forR(o, ixO, [&](long c) { tmp[c] = 0.0; });
    const double *b = o.V(w, o.b0_ + 1 + idir), *bg = o.V(w, o.bg0_ + 1 + idir);
    forR(o, o.ixG, [&](long c) { tmp2[c] = b[c] + bg[c]; });
    for (int idim = 0; idim < o.ndim; ++idim) {  // :160-173
      const long s = o.st[idim];
      const double* dx = o.dx.data() + (long)idim * n;
      forR(o, ixO, [&](long c) { tmp[c] = tmp[c] + (tmp2[c + s] - 2 * tmp2[c] + tmp2[c - s]) / (dx[c] * dx[c]); });
    }
    forR(o, ixO, [&](long c) { tmp[c] = tmp[c] * eta; });
    for (int iw : iws) {  // :191-201
      double* wn = o.V(wnew, iw);
      if (iw == o.b0_ + 1 + idir)
        forR(o, ixO, [&](long c) { wn[c] = wn[c] + qdt * tmp[c]; });
      else if (iw == o.e_)
        forR(o, ixO, [&](long c) { wn[c] = wn[c] + qdt * tmp[c] * (b[c] + bg[c]); });
    }
  }
  for (int iw : iws) {  // de/dt += eta*J**2, :205-214
    if (iw != o.e_) continue;
    double* wn = o.V(wnew, iw);
    forR(o, ixO, [&](long c) {
      double s = 0.0;
      for (int i = idirmin; i < 3; ++i) s = s + J[i][c] * J[i][c];
      wn[c] = wn[c] + qdt * eta * s;
    });
  }
}

// addsource2, src/vac.t:552-582: specialsource, then addsource
// (src/vacphys.mhd0.t:225-258): the resistive term when |eta| > smalldouble
// (addsource_res2, or addsource_res1 with compactres), then the Powell term
// when divbfix is set and ndim > 1 ({^NOONED}).
void addsource2(Oracle& o, double qdt, const std::vector<int>& iws, double qtC, const Arr& wCT,
                double qt, Arr& w, Work& wk) {
  specialsource(o, qdt, iws, qtC, wCT, qt, w, wk);
  if (std::fabs(o.par.eta) > smalldouble) {
    if (o.par.compactres)
      addsource_res1(o, qdt, iws, wCT, w, wk);
    else
      addsource_res2(o, qdt, iws, wCT, w, wk);
  }
  if (o.par.divbfix && o.ndim > 1) addsource_divb(o, qdt, iws, wCT, w, wk);
}

// centdiff4, src/vaccd.t:7-78.  The flux divergence is applied on the mesh ixO=ixM.
void centdiff4(Oracle& o, double qdt, const std::vector<int>& iws, int dmin, int dmax, double qtC,
               const Arr& wCT, double qt, Arr& w, Work& wk) {
  wk.init(o.ncell);
  const Rg ixO = o.ixM;
  for (int d = dmin; d <= dmax; ++d) {
    // v is needed on ixO+-2 along d for the fluxes, and along every idir for the
    // background-work term; computing it on the whole grid covers both.
    getv(o, wCT, o.ixG, d, wk.v);
    Rg ix = grow1(ixO, d, 2);
    for (int iw : iws) {
      bool transport = getflux(o, wCT, ix, iw, d, wk.f, wk.fbuf);
      if (transport) {
        const double* q = o.V(wCT, iw);
        forR(o, ix, [&](long c) { wk.f[c] = wk.f[c] + wk.v[c] * q[c]; });
      }
      gradient4(o, wk.f, ixO, d, wk.tmp);
      double* wi = o.V(w, iw);
      forR(o, ixO, [&](long c) { wi[c] = wi[c] - qdt * wk.tmp[c]; });
      if (iw == o.e_) {
        gradient4(o, wk.v, ixO, d, wk.tmp);
        getptotal_bg(o, w, ixO, wk.fb);
        forR(o, ixO, [&](long c) { wi[c] = wi[c] - qdt * wk.tmp[c] * wk.fb[c]; });
        for (int idir = dmin; idir <= dmax; ++idir) {
          gradient4(o, wk.v, ixO, idir, wk.tmp);
          const double *bgi = o.V(w, o.bg0_ + 1 + idir), *bgd = o.V(w, o.bg0_ + 1 + d);
          forR(o, ixO, [&](long c) { wi[c] = wi[c] + qdt * bgi[c] * bgd[c] * wk.tmp[c]; });
        }
      }
    }
  }
  if (o.par.sourceunsplit) {
    double q2 = qdt * ((double)(dmax - dmin) + 1.0) / (double)o.ndim;
    addsource2(o, q2, iws, qtC, wCT, qt, w, wk);
  }
}

// ---------------------------------------------------------------------------
// keeppositive, src/vacphys.t.mhd:8-49, on ixM
// ---------------------------------------------------------------------------
void keeppositive(Oracle& o, Arr& w) {
  const double g = o.par.gamma, smallp = o.par.smallp;
  double *rho = o.V(w, o.rho_), *e = o.V(w, o.e_);
  const double *rhob = o.V(w, o.rhob_), *eb = o.V(w, o.eb_);
  auto sq = [&](int iw0, long c) {  // ^C&w(ix^S,iw0+^C)**2+
    double s = 0;
    for (int C = 1; C <= o.ndir; ++C) s += o.V(w, iw0 + C)[c] * o.V(w, iw0 + C)[c];
    return s;
  };
  // where((rho+rhob) < smallrho): m=0, rho=vacuumrho-rhob, e=smallp/(gamma-1)+b**2/2-eb, :21-26
  forR(o, o.ixM, [&](long c) {
    if (rho[c] + rhob[c] < o.par.smallrho) {
      for (int C = 1; C <= o.ndir; ++C) o.V(w, o.m0_ + C)[c] = 0.0;
      rho[c] = o.par.vacuumrho - rhob[c];
      e[c] = smallp / (g - 1.0) + 0.5 * sq(o.b0_, c) - eb[c];
    }
  });
  Arr tmp(o.ncell, 0.0);
  getpthermal(o, w, o.ixM, tmp);  // :29
  const double floor = std::max(0.0, smallp);
  bool toosmallp = false;
  double mn = bigdouble;
  for (int k = o.ixM.lo[2]; k <= o.ixM.hi[2]; ++k)
    for (int j = o.ixM.lo[1]; j <= o.ixM.hi[1]; ++j)
      for (int i = o.ixM.lo[0]; i <= o.ixM.hi[0]; ++i) {
        const double p = tmp[o.id(i, j, k)];
        if (p < floor) toosmallp = true;  // any(tmp(ix^S)<max(zero,smallp)), :32
        mn = std::min(mn, p);
      }
  if (!toosmallp) return;
  if (++o.nerror_toosmallp == 1) {  // :35-41
    o.toosmallp_it = o.it_now;
    o.toosmallp_min = mn;
  }
  // e = max(p,smallp)/(gamma-1) + (m**2/rho + b**2)/2 - eb over the whole mesh, :43-45;
  // the kinetic term divides by the perturbed density alone, as written there
  if (smallp > 0.0)
    forR(o, o.ixM, [&](long c) {
      e[c] = std::max(tmp[c], smallp) / (g - 1.0) + 0.5 * (sq(o.m0_, c) / rho[c] + sq(o.b0_, c)) - eb[c];
    });
}

// primitive and conserve over the whole grid, src/vacphys0.t.mhd:5-52: p into the
// e slot (getpthermal) and v = m/(rho'+rhob) into the m slots; then back, e from
// p, v and b (e = p/(gamma-1) + (rho'+rhob) v^2/2 + b^2/2 + b.bg) and m = (rho'+rhob) v
void primitive(Oracle& o, Arr& w) {
  Arr p(o.ncell);
  getpthermal(o, w, o.ixG, p);
  forR(o, o.ixG, [&](long c) {
    o.V(w, o.e_)[c] = p[c];
    for (int C = 1; C <= o.ndir; ++C)
      o.V(w, o.m0_ + C)[c] = o.V(w, o.m0_ + C)[c] / (o.V(w, o.rho_)[c] + o.V(w, o.rhob_)[c]);
  });
}
void conserve(Oracle& o, Arr& w) {
  const double g = o.par.gamma;
  forR(o, o.ixG, [&](long c) {
    const double rt = o.V(w, o.rho_)[c] + o.V(w, o.rhob_)[c];
    double v2 = 0, b2 = 0, bb = 0;
    for (int C = 1; C <= o.ndir; ++C) v2 += o.V(w, o.m0_ + C)[c] * o.V(w, o.m0_ + C)[c];
    for (int C = 1; C <= o.ndir; ++C) b2 += o.V(w, o.b0_ + C)[c] * o.V(w, o.b0_ + C)[c];
    for (int C = 1; C <= o.ndir; ++C) bb += o.V(w, o.b0_ + C)[c] * o.V(w, o.bg0_ + C)[c];
    o.V(w, o.e_)[c] = o.V(w, o.e_)[c] / (g - 1.0) + 0.5 * (rt * v2 + b2) + bb;
    for (int C = 1; C <= o.ndir; ++C) o.V(w, o.m0_ + C)[c] = rt * o.V(w, o.m0_ + C)[c];
  });
}

// ---------------------------------------------------------------------------
// boundaries, src/vacgrid.t:9-512
// ---------------------------------------------------------------------------
void getboundary(Oracle& o, Arr& w) {
  if (o.par.smallfix) keeppositive(o, w);  // src/vacgrid.t:220
  for (int iB = 0; iB < o.nB; ++iB) {
    const int d = o.idimB[iB];
    const Rg r = o.ixB[iB];
    const bool up = o.upperB[iB];
    const long s = o.st[d];
    for (int iw = 0; iw < o.nw; ++iw) {
      const std::string& t = o.tB(iw, iB);
      double* a = o.V(w, iw);
      auto plane = [&](int q2) {
        Rg p = r;
        p.lo[d] = p.hi[d] = q2;
        return p;
      };
      if (t == "cont" || t == "fixed") {
        int ixe = up ? r.lo[d] - 1 : r.hi[d] + 1;
        if (o.fixedB[iw + o.nw * iB]) {
          const std::vector<double>& fb = o.fixB[iB];
          forR(o, r, [&](long c) { a[c] = fb[(long)iw * o.ncell + c]; });
        } else if (t == "cont" || !o.fullgridini) {
          for (int q2 = r.lo[d]; q2 <= r.hi[d]; ++q2)
            forR(o, plane(q2), [&](long c) { a[c] = a[c + (long)(ixe - q2) * s]; });
        }
      } else if (t == "cont1" || t == "fixed1" || t == "grad1") {
        int ixe = up ? r.lo[d] - 1 : r.hi[d] + 1;
        int ixf = up ? ixe - 1 : ixe + 1;
        if (o.fixedB[iw + o.nw * iB]) {
          const std::vector<double>& fb = o.fixB[iB];
          if (t == "grad1")
            for (int q2 = r.lo[d]; q2 <= r.hi[d]; ++q2)
              forR(o, plane(q2), [&](long c) {
                a[c] = fb[(long)iw * o.ncell + c] + a[c + (long)(ixe - q2) * s];
              });
          else
            forR(o, r, [&](long c) { a[c] = fb[(long)iw * o.ncell + c]; });
        } else if (t == "cont1" || !o.fullgridini) {
          for (int q2 = r.lo[d]; q2 <= r.hi[d]; ++q2) {
            int n = std::abs(q2 - ixe);
            forR(o, plane(q2), [&](long c) {
              a[c] = (double)(n + 1) * a[c + (long)(ixe - q2) * s] - (double)n * a[c + (long)(ixf - q2) * s];
            });
          }
        }
      } else if (t == "periodic") {
        // w(ix^S) = w(ixpair^S): the pair's region moved by dixB along idim (:236-246)
        const Rg pr = o.ixB[o.ipairB[iB]];
        long shift = 0;
        for (int e = 0; e < o.ndim; ++e) {
          int se = pr.lo[e] - r.lo[e];
          if (e == d) se += up ? o.dixB : -o.dixB;
          shift += (long)se * o.st[e];
        }
        forR(o, r, [&](long c) { a[c] = a[c + shift]; });
      } else if (t == "symm" || t == "symm0" || t == "asymm") {
        int ixe = up ? 2 * r.lo[d] - 1 : 2 * r.hi[d] + 1;
        double sg = (t == "asymm") ? -1.0 : 1.0;
        for (int q2 = r.lo[d]; q2 <= r.hi[d]; ++q2)
          forR(o, plane(q2), [&](long c) { a[c] = sg * a[c + (long)(ixe - q2 - q2) * s]; });
      } else if (t == "contCD4") {
        int q1 = r.lo[d], q2 = r.hi[d];
        int se = up ? r.lo[d] - 2 : r.hi[d] + 3, see = up ? r.lo[d] - 3 : r.hi[d] + 2;
        forR(o, plane(q1), [&](long c) { a[c] = a[c + (long)(se - q1) * s]; });
        forR(o, plane(q2), [&](long c) { a[c] = a[c + (long)(see - q2) * s]; });
      } else if (t == "zero") {  // src/vacgrid.t:295-346: contCD4's copy in primitive variables
        primitive(o, w);
        int q1 = r.lo[d], q2 = r.hi[d];
        int se = up ? r.lo[d] - 2 : r.hi[d] + 3, see = up ? r.lo[d] - 3 : r.hi[d] + 2;
        forR(o, plane(q1), [&](long c) { a[c] = a[c + (long)(se - q1) * s]; });
        forR(o, plane(q2), [&](long c) { a[c] = a[c + (long)(see - q2) * s]; });
        conserve(o, w);
      }
    }
  }
  // fixB capture after the very first fill, :476-507
  if (!o.bc_initialized) {
    o.bc_initialized = true;
    for (int iB = 0; iB < o.nB; ++iB) {
      const int d = o.idimB[iB];
      const Rg r = o.ixB[iB];
      const long s = o.st[d];
      int ixe = o.upperB[iB] ? r.lo[d] - 1 : r.hi[d] + 1;
      for (int iw = 0; iw < o.nw; ++iw) {
        const std::string& t = o.tB(iw, iB);
        if ((t == "fixed" || t == "fixed1" || t == "grad1") && !o.fixedB[iw + o.nw * iB]) {
          o.fixedB[iw + o.nw * iB] = 1;
          if (o.fixB[iB].empty()) o.fixB[iB].assign((size_t)o.nw * o.ncell, 0.0);
          double* fb = o.fixB[iB].data() + (long)iw * o.ncell;
          const double* a = o.V(w, iw);
          for (int q2 = r.lo[d]; q2 <= r.hi[d]; ++q2) {
            Rg p = r;
            p.lo[d] = p.hi[d] = q2;
            if (t == "grad1")
              forR(o, p, [&](long c) { fb[c] = a[c] - a[c + (long)(ixe - q2) * s]; });
            else
              forR(o, p, [&](long c) { fb[c] = a[c]; });
          }
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// time step, src/vac.t:641-699, src/vacusr.viscosity.t:509-542,
// src/vacusr.gravity.t:97-138
// ---------------------------------------------------------------------------
double meshmax(const Oracle& o, const Arr& a) {
  double m = -bigdouble;
  for (int k = o.ixM.lo[2]; k <= o.ixM.hi[2]; ++k)
    for (int j = o.ixM.lo[1]; j <= o.ixM.hi[1]; ++j)
      for (int i = o.ixM.lo[0]; i <= o.ixM.hi[0]; ++i) m = std::max(m, a[o.id(i, j, k)]);
  return m;
}

void getdt_courant(Oracle& o, const Arr& w, double& dt) {
  dt = bigdouble;
  double courantmax = 0.0;
  bool new_cmax = true;
  CmaxCache cc;
  Arr cmax(o.ncell, 0.0), r(o.ncell, 0.0);
  for (int d = 0; d < o.ndim; ++d) {
    getcmax(o, new_cmax, w, o.ixM, d, cmax, cc);
    const double* dd = o.dx.data() + (long)d * o.ncell;
    forR(o, o.ixM, [&](long c) { r[c] = cmax[c] / dd[c]; });
    courantmax = std::max(courantmax, meshmax(o, r));
  }
  if (courantmax > smalldouble) dt = std::min(dt, o.par.courantpar / courantmax);
}

void getdt_visc(Oracle& o, double& dt) {
  double dtdiffpar = 0.25;  // overwritten globally, :530
  o.par.dtdiffpar = dtdiffpar;
  for (int d = 0; d < o.ndim; ++d) {
    const double* dd = o.dx.data() + (long)d * o.ncell;
    double m = -bigdouble;
    for (int k = o.ixM.lo[2]; k <= o.ixM.hi[2]; ++k)
      for (int j = o.ixM.lo[1]; j <= o.ixM.hi[1]; ++j)
        for (int i = o.ixM.lo[0]; i <= o.ixM.hi[0]; ++i) {
          long c = o.id(i, j, k);
          m = std::max(m, (o.maxviscoef + 0.0) / (dd[c] * dd[c]));
        }
    double dtdiff_visc = dtdiffpar / m;  // +Inf while maxviscoef==0
    dt = std::min(dt, dtdiff_visc);
  }
  o.maxviscoef = 0.0;
}

void getdt_grav(Oracle& o, double& dt, int it) {
  if (it == o.itmin) {
    // evaluated before the first specialsource call, i.e. with the file's g
    double g[3] = {o.par.grav[0], o.par.grav[1], o.par.grav[2]};
    o.dtgrav = bigdouble;
    for (int d = 0; d < o.ndim; ++d)
      if (std::fabs(g[d]) > 0.0) {
        double m = -bigdouble;
        for (int jd = 0; jd < o.ndim; ++jd) {
          const double* dd = o.dx.data() + (long)jd * o.ncell;
          for (int k = o.ixM.lo[2]; k <= o.ixM.hi[2]; ++k)
            for (int j = o.ixM.lo[1]; j <= o.ixM.hi[1]; ++j)
              for (int i = o.ixM.lo[0]; i <= o.ixM.hi[0]; ++i)
                m = std::max(m, std::fabs(g[d]) / dd[o.id(i, j, k)]);
        }
        o.dtgrav = std::min(o.dtgrav, 1.0 / std::sqrt(m));
      }
  }
  dt = std::min(dt, o.dtgrav);
}

// ---------------------------------------------------------------------------
// integrator, src/vac.t:364-549
// ---------------------------------------------------------------------------
void advect1(Oracle& o, const std::string& method, double qdt, const std::vector<int>& iws,
             int dmin, int dmax, double qtC, const Arr& wCT, double qt, Arr& w, Work& wk) {
  if (method == "cd4")
    centdiff4(o, qdt, iws, dmin, dmax, qtC, wCT, qt, w, wk);
  else if (method == "source") {
    if (o.par.sourceunsplit) addsource2(o, qdt, iws, qtC, wCT, qt, w, wk);
  }
  getboundary(o, w);
}

template <class F>
void gridop(Oracle& o, F f) {  // over ixG, all variables
  const long n = (long)o.nw * o.ncell;
#pragma omp parallel for schedule(static)
  for (long c = 0; c < n; ++c) f(c);
}

int advect(Oracle& o, const std::string& method, const std::vector<int>& iws, int dmin, int dmax,
           double dt, double t, Work& wk) {
  Arr &w = o.w, &w1 = o.w1, &w2 = o.w2, &w3 = o.w3;
  const long n = (long)o.nw * o.ncell;
  if ((long)w1.size() != n) w1.assign(n, 0.0);
  w1 = w;  // :403
  const std::string ta = o.par.typeadvance;
  if (ta == "onestep") {
    advect1(o, method, dt, iws, dmin, dmax, t, w1, t, w, wk);
  } else if (ta == "twostep") {
    std::string pred = o.par.typepred;
    advect1(o, pred, dt / 2, iws, dmin, dmax, t, w, t, w1, wk);
    advect1(o, method, dt, iws, dmin, dmax, t + dt / 2, w1, t, w, wk);
  } else if (ta == "threestep") {
    if ((long)w2.size() != n) w2.assign(n, 0.0);
    advect1(o, method, dt, iws, dmin, dmax, t, w, t, w1, wk);
    gridop(o, [&](long c) { w2[c] = 3 * 0.25 * w[c] + 0.25 * w1[c]; });
    advect1(o, method, dt / 4, iws, dmin, dmax, t + dt, w1, t + dt / 4, w2, wk);
    gridop(o, [&](long c) { w[c] = w[c] / 3 + w2[c] * (2.0 / 3); });
    advect1(o, method, dt * 2.0 / 3, iws, dmin, dmax, t + dt / 2, w2, t + dt / 3, w, wk);
  } else if (ta == "fourstep") {
    if ((long)w2.size() != n) w2.assign(n, 0.0);
    if ((long)w3.size() != n) w3.assign(n, 0.0);
    advect1(o, method, dt / 2, iws, dmin, dmax, t, w, t, w1, wk);
    w2 = w;
    advect1(o, method, dt / 2, iws, dmin, dmax, t + dt / 2, w1, t, w2, wk);
    w3 = w;
    advect1(o, method, dt, iws, dmin, dmax, t + dt / 2, w2, t, w3, wk);
    gridop(o, [&](long c) { w1[c] = (w1[c] + 2 * w2[c] + w3[c] - 4 * w[c]) / 3; });
    advect1(o, method, dt / 6, iws, dmin, dmax, t + dt, w3, t, w, wk);
    gridop(o, [&](long c) { w[c] = w[c] + w1[c]; });
  } else if (ta == "sterck") {
    if ((long)w2.size() != n) w2.assign(n, 0.0);
    const double c012 = (double)0.12f;  // default-real literal 0.12 in src/vac.t:459
    advect1(o, method, dt * c012, iws, dmin, dmax, t, w, t, w1, wk);
    w2 = w;
    advect1(o, method, dt / 4, iws, dmin, dmax, t + dt * c012, w1, t, w2, wk);
    w1 = w;
    advect1(o, method, dt / 2, iws, dmin, dmax, t + dt / 4, w2, t, w1, wk);
    advect1(o, method, dt, iws, dmin, dmax, t + dt / 2, w1, t, w, wk);
  } else if (ta == "jameson") {
    if ((long)w2.size() != n) w2.assign(n, 0.0);
    advect1(o, method, dt / 4, iws, dmin, dmax, t, w, t, w1, wk);
    w2 = w;
    advect1(o, method, dt / 3, iws, dmin, dmax, t + dt / 4, w1, t, w2, wk);
    w1 = w;
    advect1(o, method, dt / 2, iws, dmin, dmax, t + dt / 3, w2, t, w1, wk);
    advect1(o, method, dt, iws, dmin, dmax, t + dt / 2, w1, t, w, wk);
  } else {
    return SAC_ERR_UNSUPPORTED;
  }
  return SAC_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// C API (same shape as include/sac_gpu.h, prefix oracle_)
// ---------------------------------------------------------------------------
struct oracle_ctx {
  Oracle o;
  Work wk;
};

extern "C" {

void oracle_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

int oracle_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

int oracle_create(const sac_params* p, oracle_ctx** out) {
  if (!p || !out) return SAC_ERR_ARG;
  oracle_ctx* c = new oracle_ctx();
  c->o.par = *p;
  *out = c;
  return SAC_OK;
}

void oracle_destroy(oracle_ctx* c) { delete c; }

const char* oracle_last_error(const oracle_ctx* c) { return c ? c->o.err.c_str() : "null context"; }

// setixGixMix + gridsetup1, src/vacio.t:786-841, src/vacgrid.t:556-661
int oracle_set_grid(oracle_ctx* cx, int ndim, int ndir, const int ixGhi[3], const int ixM[6],
                    const double* x, int fullgridini) {
  Oracle& o = cx->o;
  if (ndim < 1 || ndim > 3 || ndir < ndim || ndir > 3) return SAC_ERR_ARG;
  o.ndim = ndim;
  o.ndir = ndir;
  o.nw = 3 * ndir + 4;
  o.rho_ = 0;
  o.m0_ = 0;
  o.e_ = ndir + 1;
  o.b0_ = o.e_;
  o.eb_ = o.b0_ + ndir + 1;
  o.rhob_ = o.eb_ + 1;
  o.bg0_ = o.rhob_;
  o.fullgridini = fullgridini != 0;
  for (int d = 0; d < 3; ++d) {
    o.nG[d] = (d < ndim) ? ixGhi[d] : 1;
    o.ixG.lo[d] = 0;
    o.ixG.hi[d] = o.nG[d] - 1;
    o.ixM.lo[d] = (d < ndim) ? ixM[d] - 1 : 0;
    o.ixM.hi[d] = (d < ndim) ? ixM[3 + d] - 1 : 0;
    if (d < ndim && (o.ixM.lo[d] != o.dixB || o.ixM.hi[d] != o.nG[d] - 1 - o.dixB))
      return SAC_ERR_ARG;
  }
  o.st[0] = 1;
  o.st[1] = o.nG[0];
  o.st[2] = (long)o.nG[0] * o.nG[1];
  o.ncell = (long)o.nG[0] * o.nG[1] * o.nG[2];
  o.x.assign(x, x + (long)ndim * o.ncell);
  // qx: x with one extra layer beyond ixG in every used dimension
  int qn[3], qoff[3];
  for (int d = 0; d < 3; ++d) {
    qn[d] = (d < ndim) ? o.nG[d] + 2 : 1;
    qoff[d] = (d < ndim) ? 1 : 0;
  }
  const long qcell = (long)qn[0] * qn[1] * qn[2];
  std::vector<double> qx((size_t)ndim * qcell, 0.0);
  auto qid = [&](int i, int j, int k) { return (i + qoff[0]) + (long)qn[0] * ((j + qoff[1]) + (long)qn[1] * (k + qoff[2])); };
  for (int jd = 0; jd < ndim; ++jd)
    for (int k = 0; k < o.nG[2]; ++k)
      for (int j = 0; j < o.nG[1]; ++j)
        for (int i = 0; i < o.nG[0]; ++i) qx[jd * qcell + qid(i, j, k)] = o.x[jd * o.ncell + o.id(i, j, k)];
  for (int d = 0; d < ndim; ++d) {
    int lo[3], hi[3];
    for (int e = 0; e < 3; ++e) {
      lo[e] = (e < ndim) ? -1 : 0;
      hi[e] = (e < ndim) ? o.nG[e] : 0;
    }
    for (int side = 0; side < 2; ++side) {
      int a, b, ixe, ixf;
      if (side == 0) {  // upper layers
        b = o.nG[d];
        a = o.fullgridini ? o.nG[d] : o.ixM.hi[d] + 1;
        ixe = a - 1;
        ixf = ixe - 1;
      } else {  // lower layers
        a = -1;
        b = o.fullgridini ? -1 : o.ixM.lo[d] - 1;
        ixe = b + 1;
        ixf = ixe + 1;
      }
      for (int jd = 0; jd < ndim; ++jd)
        for (int q = a; q <= b; ++q) {
          int l2[3] = {lo[0], lo[1], lo[2]}, h2[3] = {hi[0], hi[1], hi[2]};
          l2[d] = h2[d] = q;
          for (int k = l2[2]; k <= h2[2]; ++k)
            for (int j = l2[1]; j <= h2[1]; ++j)
              for (int i = l2[0]; i <= h2[0]; ++i) {
                int ie[3] = {i, j, k}, iff[3] = {i, j, k};
                ie[d] = ixe;
                iff[d] = ixf;
                int n = std::abs(ixe - q);
                qx[jd * qcell + qid(i, j, k)] = (double)(1 + n) * qx[jd * qcell + qid(ie[0], ie[1], ie[2])] -
                                                (double)n * qx[jd * qcell + qid(iff[0], iff[1], iff[2])];
              }
        }
    }
  }
  for (int jd = 0; jd < ndim; ++jd)
    for (int k = 0; k < o.nG[2]; ++k)
      for (int j = 0; j < o.nG[1]; ++j)
        for (int i = 0; i < o.nG[0]; ++i) o.x[jd * o.ncell + o.id(i, j, k)] = qx[jd * qcell + qid(i, j, k)];
  o.dx.assign((size_t)ndim * o.ncell, 0.0);
  for (int d = 0; d < ndim; ++d)
    for (int k = 0; k < o.nG[2]; ++k)
      for (int j = 0; j < o.nG[1]; ++j)
        for (int i = 0; i < o.nG[0]; ++i) {
          int p[3] = {i, j, k}, m[3] = {i, j, k};
          p[d] += 1;
          m[d] -= 1;
          o.dx[d * o.ncell + o.id(i, j, k)] =
              0.5 * (qx[d * qcell + qid(p[0], p[1], p[2])] - qx[d * qcell + qid(m[0], m[1], m[2])]);
        }
  o.dvolume.assign(o.ncell, 0.0);
  for (long c = 0; c < o.ncell; ++c) {
    double v = 1.0;
    for (int d = 0; d < ndim; ++d) v = v * o.dx[d * o.ncell + c];
    o.dvolume[c] = v;
  }
  o.volume = 0;
  for (int k = o.ixM.lo[2]; k <= o.ixM.hi[2]; ++k)
    for (int j = o.ixM.lo[1]; j <= o.ixM.hi[1]; ++j)
      for (int i = o.ixM.lo[0]; i <= o.ixM.hi[0]; ++i) o.volume += o.dvolume[o.id(i, j, k)];
  o.grid_set = true;
  return SAC_OK;
}

// boundsetup, src/vacgrid.t:9-160: the default regions (ixB == NULL,
// :53-70) or the user's (&boundlist ixB^LIM, idimB, upperB, :71-99), which must
// lie inside the grid; then the periodic pairs (:103-120), matched by direction,
// orientation and extent.  ixB holds ixBmin(1:ndim,1:nB) then ixBmax(1:ndim,1:nB)
// (1-based), idimB 1..ndim, upperB 0/1.
int oracle_set_boundaries(oracle_ctx* cx, int nB, const char* typeB, const int* ixB, const int* idimB,
                          const int* upperB, const int* ipairB) {
  Oracle& o = cx->o;
  if (!o.grid_set) return SAC_ERR_STATE;
  if (nB < 1 || nB > SAC_NHIB) return SAC_ERR_ARG;
  const bool user = ixB != nullptr;
  if (user && (!idimB || !upperB)) return SAC_ERR_ARG;
  if (!user && nB != 2 * o.ndim) return SAC_ERR_ARG;
  o.nB = nB;
  o.typeB.assign((size_t)o.nw * nB, "");
  for (int iB = 0; iB < nB; ++iB)
    for (int iw = 0; iw < o.nw; ++iw) {
      std::string s(typeB + SAC_LENTYPE * ((long)iw + (long)o.nw * iB), SAC_LENTYPE);
      while (!s.empty() && (s.back() == ' ' || s.back() == '\0')) s.pop_back();
      o.typeB[iw + (long)o.nw * iB] = s;
    }
  for (int iB = 0; iB < nB; ++iB) {
    if (user) {
      const int d = idimB[iB] - 1;
      if (d < 0 || d >= o.ndim) {
        o.err = "Error in BoundSetup: idimB out of range";
        return SAC_ERR_ARG;
      }
      o.idimB[iB] = d;
      o.upperB[iB] = upperB[iB] != 0;
      o.ixB[iB] = o.ixG;
      for (int e = 0; e < o.ndim; ++e) {
        o.ixB[iB].lo[e] = ixB[e + o.ndim * iB] - 1;
        o.ixB[iB].hi[e] = ixB[o.ndim * nB + e + o.ndim * iB] - 1;
        if (o.ixB[iB].lo[e] < o.ixG.lo[e] || o.ixB[iB].hi[e] > o.ixG.hi[e]) {
          o.err = "Error in BoundSetup: Boundary region is outside grid";
          return SAC_ERR_ARG;
        }
      }
    } else {
      int d = iB / 2;
      o.idimB[iB] = d;
      o.upperB[iB] = (iB % 2) == 1;
      o.ixB[iB] = o.ixG;
      if (o.upperB[iB]) {
        o.ixB[iB].lo[d] = o.ixM.hi[d] + 1;
        o.ixB[iB].hi[d] = o.ixG.hi[d];
      } else {
        o.ixB[iB].lo[d] = o.ixG.lo[d];
        o.ixB[iB].hi[d] = o.ixM.lo[d] - 1;
      }
    }
    o.ipairB[iB] = ipairB ? ipairB[iB] - 1 : -1;
  }
  auto same_extent = [&](int iB, int jB) {
    for (int e = 0; e < o.ndim; ++e)
      if (o.ixB[iB].hi[e] - o.ixB[iB].lo[e] != o.ixB[jB].hi[e] - o.ixB[jB].lo[e]) return false;
    return true;
  };
  for (int iB = 0; iB < nB; ++iB) {
    if (o.typeB[0 + (long)o.nw * iB] == "periodic" && o.ipairB[iB] < 0) {
      for (int jB = iB + 1; jB < nB; ++jB)
        if (o.typeB[(long)o.nw * jB] == "periodic" && o.ipairB[jB] < 0 && o.idimB[iB] == o.idimB[jB] &&
            o.upperB[iB] != o.upperB[jB] && same_extent(iB, jB)) {
          o.ipairB[iB] = jB;
          o.ipairB[jB] = iB;
        }
      if (o.ipairB[iB] < 0) {
        o.err = "Error in BoundSetup: No periodic pair";
        return SAC_ERR_ARG;
      }
    }
  }
  for (int iB = 0; iB < nB; ++iB)
    for (int iw = 0; iw < o.nw; ++iw) {
      const std::string& t = o.typeB[iw + (long)o.nw * iB];
      if (!(t == "cont" || t == "fixed" || t == "cont1" || t == "fixed1" || t == "grad1" || t == "periodic" ||
            t == "symm" || t == "symm0" || t == "asymm" || t == "contCD4" || t == "zero")) {
        o.err = "boundary type '" + t + "' is not implemented";
        return SAC_ERR_UNSUPPORTED;
      }
    }
  o.fixedB.assign((size_t)o.nw * nB, 0);
  o.bc_initialized = false;
  o.bc_set = true;
  return SAC_OK;
}

int oracle_upload(oracle_ctx* cx, const double* w) {
  Oracle& o = cx->o;
  if (!o.grid_set) return SAC_ERR_STATE;
  o.w.assign(w, w + (long)o.nw * o.ncell);
  o.state_set = true;
  return SAC_OK;
}

int oracle_download(oracle_ctx* cx, double* w) {
  Oracle& o = cx->o;
  if (!o.state_set) return SAC_ERR_STATE;
  std::memcpy(w, o.w.data(), sizeof(double) * o.w.size());
  return SAC_OK;
}

int oracle_getboundary(oracle_ctx* cx, double t) {
  (void)t;
  Oracle& o = cx->o;
  if (!o.state_set || !o.bc_set) return SAC_ERR_STATE;
  getboundary(o, o.w);
  return SAC_OK;
}

// src/vac.t:61-70
int oracle_getdt(oracle_ctx* cx, double* dt, int it) {
  Oracle& o = cx->o;
  if (!o.state_set || !o.bc_set) return SAC_ERR_STATE;
  if (!o.itmin_set) {
    o.itmin = it;
    o.itmin_set = true;
  }
  o.it_now = it;
  double d;
  if (o.par.dtpar > 0.0) {
    d = o.par.dtpar;
  } else {
    d = bigdouble;
    if (o.par.courantpar > 0.0) getdt_courant(o, o.w, d);
    if (o.par.eta < 0.0) {
      o.err = "eta < 0 needs a user specialeta";
      return SAC_ERR_UNSUPPORTED;
    }
    if (o.par.eta > 0.0) {
      // getdt_res, src/vacphys.mhdres.t:5-45: dtdiffpar*minval(dx(ixM,1:ndim))**2/eta,
      // with dtdiffpar as getdt_visc may have overwritten it at an earlier call
      double mn = bigdouble;
      for (int dd = 0; dd < o.ndim; ++dd)
        forR(o, o.ixM, [&](long c) { mn = std::min(mn, o.dx[(long)dd * o.ncell + c]); });
      d = std::min(d, o.par.dtdiffpar * (mn * mn) / o.par.eta);
    }
    const int u = o.par.user;
    if (u == SAC_USR_SLOG || u == SAC_USR_GRAVVISC || u == SAC_USR_STRAT || u == SAC_USR_TUBE) {
      if (visc_on(o)) getdt_visc(o, d);
      getdt_grav(o, d, it);
    }
    if (o.par.dtcantgrow && it > o.itmin) d = std::min(d, o.dtold);
    o.dtold = d;
  }
  *dt = d;
  return SAC_OK;
}

int oracle_advect(oracle_ctx* cx, const char* method, const int* iws, int idimmin, int idimmax, double dt,
                  double t, int it) {
  Oracle& o = cx->o;
  if (!o.state_set || !o.bc_set) return SAC_ERR_STATE;
  o.it_now = it;
  std::vector<int> v;
  if (iws) {
    int n = iws[o.nw];
    for (int i = 0; i < n; ++i) v.push_back(iws[i] - 1);
  } else {
    for (int iw = 0; iw < o.eb_; ++iw) v.push_back(iw);
  }
  std::string m(method);
  while (!m.empty() && m.back() == ' ') m.pop_back();
  if (m != "cd4" && m != "source" && m != "nul") return SAC_ERR_UNSUPPORTED;
  if (idimmin < 1 || idimmax > o.ndim || idimmin > idimmax) return SAC_ERR_ARG;
  if (o.par.eta < -smalldouble) {
    o.err = "eta < 0 needs a user specialeta";
    return SAC_ERR_UNSUPPORTED;
  }
  return advect(o, m, v, idimmin - 1, idimmax - 1, dt, t, cx->wk);
}

int oracle_diag(oracle_ctx* cx, sac_diag_out* out) {
  Oracle& o = cx->o;
  if (!o.state_set) return SAC_ERR_STATE;
  std::memset(out, 0, sizeof(*out));
  for (int iw = 0; iw < o.nw && iw < SAC_NWMAX; ++iw) {
    double s = 0;
    const double* a = o.V(o.w, iw);
    for (int k = o.ixM.lo[2]; k <= o.ixM.hi[2]; ++k)
      for (int j = o.ixM.lo[1]; j <= o.ixM.hi[1]; ++j)
        for (int i = o.ixM.lo[0]; i <= o.ixM.hi[0]; ++i) {
          long c = o.id(i, j, k);
          s += o.dvolume[c] * a[c];
        }
    out->wmean[iw] = s / o.volume;
  }
  // getdivb with the 4th-order stencil, src/vacphys.mhd0.t:106-144
  Arr tmp(o.ncell, 0.0), g(o.ncell, 0.0), divb(o.ncell, 0.0);
  for (int d = 0; d < o.ndim; ++d) {
    forR(o, o.ixG, [&](long c) { tmp[c] = o.V(o.w, o.b0_ + 1 + d)[c] + o.V(o.w, o.bg0_ + 1 + d)[c]; });
    gradient4(o, tmp, o.ixM, d, g);
    forR(o, o.ixM, [&](long c) { divb[c] = divb[c] + g[c]; });
  }
  double s2 = 0, mx = 0;
  long n = 0;
  int nonfinite = 0;
  for (int k = o.ixM.lo[2]; k <= o.ixM.hi[2]; ++k)
    for (int j = o.ixM.lo[1]; j <= o.ixM.hi[1]; ++j)
      for (int i = o.ixM.lo[0]; i <= o.ixM.hi[0]; ++i) {
        long c = o.id(i, j, k);
        s2 += divb[c] * divb[c];
        mx = std::max(mx, std::fabs(divb[c]));
        ++n;
        for (int iw = 0; iw < o.nw; ++iw)
          if (!std::isfinite(o.V(o.w, iw)[c])) nonfinite = 1;
      }
  out->divb_l2 = std::sqrt(s2 / (double)n);
  out->divb_linf = mx;
  out->maxviscoef = o.maxviscoef;
  for (int d = 0; d < 3; ++d) out->ctot[d] = o.ctot_last[d];
  out->nonfinite = nonfinite;
  out->nerror_toosmallp = o.nerror_toosmallp;
  out->toosmallp_it = o.toosmallp_it;
  out->toosmallp_min = o.toosmallp_min;
  return SAC_OK;
}

}  // extern "C"
