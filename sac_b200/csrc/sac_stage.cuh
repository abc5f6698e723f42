// sac_stage.cuh -- the RK stage as three passes that each evaluate a quantity once.
//
//   k_face   per cell: rho+rhob, v=m/(rho+rhob), the "173" energy
//            e-(b^2+m^2/rho)/2, p'_tot (getptotal), the perturbed fluxes of every
//            advanced variable along every dimension (getflux + transport,
//            src/vacphys.mhd0.t:147-222, src/vaccd.t:43-46) and the per-dimension
//            maxima c_tot of getcmax over the mesh (src/vacphys0.t.mhd:77-160).
//   k_nu     per cell and per (field, dimension) pair of setnu: the face quotient
//            Q = (c_tot c_hyp max3 d3R)/max5 d1R (0 where max5 d1R is 0) at the
//            face c+1/2 (src/vacusr.viscosity.t:372-450), so that
//            nu_R(i) = Q(i) dx(i) and nu_L(i) = Q(i-1) dx(i).
//   k_update per mesh cell: flux divergence with gradient4's edge zeroing, the
//            e-equation background work, gravity, the hyperdiffusion terms of
//            addsource_visc, the user driver and the Runge-Kutta epilogue.
//
// S is the storage type of the advanced variables and of D, F and Q.  Every
// expression is written in the reference's evaluation order.  The FP64
// instantiation is compiled without contraction and with IEEE division
// (stage_f64.cu): the reference's hyperdiffusion switch max|d3|/max|d1| is
// scale-free, so rounding noise at a wave front is amplified to order one, and
// only bit-faithful arithmetic keeps the device on the reference's trajectory.
// The FP32 instantiation (stage_f32.cu) may contract and approximate.
#pragma once
#include "sac_kernels.cuh"
#include "sac_stage_api.h"

namespace sacgpu {


template <typename S>
__device__ __forceinline__ S ld(const S* p, int i) {
  return __ldg(p + i);
}
__device__ __forceinline__ double fmaxT(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ float fmaxT(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double fabsT(double a) { return fabs(a); }
__device__ __forceinline__ float fabsT(float a) { return fabsf(a); }

// a load of a stencil field: from global memory through the read-only path, or
// from a shared-memory tile
template <bool TILE, typename S, typename I>
__device__ __forceinline__ S ldt(const S* p, I i) {
  if constexpr (TILE) return p[i];
  else return __ldg(p + i);
}


// ---------------------------------------------------------------------------
// per-cell bodies (one grid, located by the offsets o)
// ---------------------------------------------------------------------------
// the k_face arithmetic of the cell whose fields are read at c: dout(i, v) takes
// the derived field i, fout(d, iw, v) the flux of iw along d for the dimensions in
// the bit mask fdims; mesh tells whether the getcmax maxima apply there
template <int NDIM, int NDIR, typename S, class DOut, class FOut>
__device__ __forceinline__ void face_eval(const Stage2Args& a, const Offs& o, long c, bool mesh, double gamma,
                                          double* cm, unsigned fdims, DOut&& dout, FOut&& fout) {
  constexpr int E = NDIR + 1;
  auto W = [&](int iw) { return (const S*)a.fW[iw] + o.P; };
  auto BG = [&](int i) { return a.fBG[i] + o.B; };
  {
    const double rho = (double)W(0)[c];
    const double eb = BG(0)[c];
    const double rhob = BG(1)[c];
    const double rt = rho + rhob;
    double m[NDIR], b[NDIR], bg[NDIR], v[NDIR];
#pragma unroll
    for (int C = 0; C < NDIR; ++C) {
      m[C] = (double)W(1 + C)[c];
      b[C] = (double)W(E + 1 + C)[c];
      bg[C] = BG(2 + C)[c];
    }
    const double e = (double)W(E)[c];
#pragma unroll
    for (int C = 0; C < NDIR; ++C) v[C] = dvs_rn(m[C], rt);  // getv / tmp_nu for m
    double b2 = 0.0, m2 = 0.0, bb = 0.0;
#pragma unroll
    for (int C = 0; C < NDIR; ++C) {
      b2 = add_rn(b2, mul_rn(b[C], b[C]));
      m2 = add_rn(m2, mul_rn(m[C], m[C]));
      bb = add_rn(bb, mul_rn(b[C], bg[C]));
    }
    dout(0, (S)rt);
#pragma unroll
    for (int C = 0; C < NDIR; ++C) dout(1 + C, (S)v[C]);
    // tmp_nu for iw=173, src/vacusr.viscosity.t:301
    dout(NDIR + 1, (S)sub_rn(e, mul_rn(0.5, add_rn(b2, dvs_rn(m2, rt)))));
    // getptotal, src/vacphys0.t.mhd:199-201
    const double pp = (gamma - 2.0) * (bb + 0.5 * b2);
    const double ptot = (gamma - 1.0) * (e - dvs(0.5 * m2, rt)) - pp;
    dout(NDIR + 2, (S)ptot);
    // fluxes in the storage precision's arithmetic (FP64 for the FP64 path; FP32
    // for the FP32 path, whose pressure/energy recovery above stays FP64)
    using C_ = S;
    C_ mC[NDIR], bC[NDIR], bgC[NDIR], vC[NDIR];
#pragma unroll
    for (int C = 0; C < NDIR; ++C) {
      mC[C] = (C_)m[C];
      bC[C] = (C_)b[C];
      bgC[C] = (C_)bg[C];
      vC[C] = (C_)v[C];
    }
    const C_ rtC = (C_)rt, ptC = (C_)ptot, ebC = (C_)eb, eC = (C_)e, rhoC = (C_)rho, rhobC = (C_)rhob;
    C_ s1 = C_(0), s2 = C_(0);
#pragma unroll
    for (int C = 0; C < NDIR; ++C) s1 = s1 + bgC[C] * mC[C];
#pragma unroll
    for (int C = 0; C < NDIR; ++C) s2 = s2 + bC[C] * mC[C];
#pragma unroll
    for (int d = 0; d < NDIM; ++d) {
      if (!((fdims >> d) & 1u)) continue;
      const C_ vd = vC[d], bd = bC[d], bgd = bgC[d], md = mC[d];
      fout(d, 0, (S)(dvs(rhobC * md, rtC) + vd * rhoC));
#pragma unroll
      for (int C = 0; C < NDIR; ++C) {
        C_ f;
        if (C == d)
          f = (ptC + C_(0)) - (bC[C] * bgd + bd * bgC[C]) - bC[C] * bd;
        else
          f = -(bC[C] * bgd + bd * bgC[C]) - bC[C] * bd;
        fout(d, 1 + C, (S)(f + vd * mC[C]));
      }
      const C_ fe = dvs(md * (ptC + C_(0)) - bd * s1 - bgd * s2, rtC) + dvs(ebC * md, rtC) - dvs(bd * s2, rtC);
      fout(d, E, (S)(fe + vd * eC));
      // b_d has no flux along d (getflux sets transport=.false., src/vacphys.mhd0.t:204-206), and
      // k_update never reads that slot, so it is not written
#pragma unroll
      for (int C = 0; C < NDIR; ++C)
        if (C != d) fout(d, E + 1 + C, (S)(-(vC[C] * (bd + bgd)) + vd * bgC[C] + vd * bC[C]));
    }
    if (mesh) {
        // getpthermal, getcsound2, getcmax: src/vacphys0.t.mhd:95-183
        double q = 0.5 * m2 / rt;
        q = q + 0.5 * b2 + bb;
        const double p = (gamma - 1.0) * (e - q);
        double bgs = 0.0, Bt2 = 0.0;
#pragma unroll
        for (int C = 0; C < NDIR; ++C) bgs = bgs + bg[C] * bg[C];
        const double cs2 = gamma * (p + (gamma - 1.0) * (eb - 0.5 * bgs)) / rt;
#pragma unroll
        for (int C = 0; C < NDIR; ++C) {
          const double B = b[C] + bg[C];
          Bt2 = Bt2 + B * B;
        }
        const double cf2 = Bt2 / rt + cs2;
#pragma unroll
        for (int d = 0; d < NDIM; ++d) {
          const double Bd = b[d] + bg[d];
          cm[d] = sqrt(0.5 * (cf2 + sqrt(cf2 * cf2 - 4.0 * cs2 * (Bd * Bd) / rt))) + fabs(m[d] / rt);
        }
    }
  }
}

// k_face body at local cell c: the derived fields and every flux into D and F
template <int NDIM, int NDIR, typename S>
__device__ __forceinline__ void face_cell(const Stage2Args& a, const Offs& o, int c, bool mesh, double gamma,
                                          double* cm) {
  face_eval<NDIM, NDIR, S>(
      a, o, c, mesh, gamma, cm, (1u << NDIM) - 1u, [&](int i, S v) { ((S*)a.fD[i] + o.I)[c] = v; },
      [&](int d, int iw, S v) { ((S*)a.fF[d][iw] + o.I)[c] = v; });
}

// setnu's face quotient from a window of six values of q along one dimension
// (TILE: q is a shared-memory tile)
template <bool TILE = false, typename S>
__device__ __forceinline__ S face_quotient(const S* __restrict__ q, int c, int s, int pos, int lo, int hi, S pre) {
  // q(c-2..c+3) along s; the layer beyond the two ghosts is the mirror image
  // about the first/last mesh cell (tmp_nuI, src/vacusr.viscosity.t:378-400)
  S a[6];
#pragma unroll
  for (int o = -2; o <= 3; ++o) {
    int p = pos + o;
    if (p <= lo - 3) p = lo + 3;
    if (p >= hi + 3) p = hi - 3;
    a[o + 2] = ldt<TILE>(q, c + (p - pos) * s);
  }
  S d1[5], d3[3];
#pragma unroll
  for (int j = 0; j < 5; ++j) d1[j] = fabsT(a[j + 1] - a[j]);  // d1R(c-2+j), :414
#pragma unroll
  for (int j = 0; j < 3; ++j)  // d3R(c-1+j), :413
    d3[j] = fabsT(sub_rn(mul_rn(S(3), sub_rn(a[j + 2], a[j + 1])), sub_rn(a[j + 3], a[j])));
  const S md3 = fmaxT(fmaxT(d3[0], d3[1]), d3[2]);
  const S md1 = fmaxT(fmaxT(fmaxT(fmaxT(d1[0], d1[1]), d1[2]), d1[3]), d1[4]);
  // zero where the window is flat (md1 == 0): branch before dividing, since 0/0
  // leaves the division's fast path, and a state at rest is flat almost everywhere
  if (!(md1 > S(0))) return S(0);
  return pre * md3 / md1;  // c_tot*c_hyp*md3R/md1R, :424
}

// k_nu body at local cell c with local coordinates p: every setnu pair's face
// quotient at c+1/2 along each dimension
template <int NDIM, int NDIR, typename S>
__device__ __forceinline__ void nu_cell(const Stage2Args& a, const Geom& g, const Offs& o, int c, const int p[3],
                                        const unsigned long long* ctot) {
  using PR = Pairs<NDIM>;
  constexpr int E = NDIR + 1;
#pragma unroll
  for (int k = 0; k < NDIM; ++k) {
    const int s = (int)g.st[k];
    const int pos = p[k], lo = g.lo[k], hi = g.hi[k];
    const double ct = __longlong_as_double((long long)ctot[k]);
    // c_hyp: 0.04 for rho, the "173" energy and b; 0.4 for the momenta (:284-290)
    const S p04 = (S)(ct * 0.04), p4 = (S)(ct * 0.4);
    auto Qw = [&](int ip) { return (S*)a.fQ[ip] + o.I; };
    auto W = [&](int iw) { return (const S*)a.fW[iw] + o.P; };
    auto Df = [&](int i) { return (const S*)a.fD[i] + o.I; };
    Qw(PR::rho(k))[c] = face_quotient(W(0), c, s, pos, lo, hi, p04);
    Qw(PR::e(k))[c] = face_quotient(Df(NDIR + 1), c, s, pos, lo, hi, p04);
#pragma unroll
    for (int l = 0; l < NDIM; ++l) {
      Qw(PR::v(l, k))[c] = face_quotient(Df(1 + l), c, s, pos, lo, hi, p4);
      if (l != k) Qw(PR::b(l, k))[c] = face_quotient(W(E + 1 + l), c, s, pos, lo, hi, p04);
    }
  }
}

// The fused 2D stage's view of one cell for update_cell: the stencil fields in
// shared-memory tiles of row stride st1 (each pointer offset so that [c] is the
// cell), the cell's box index c and its index cg in the instance's global blocks.
template <typename S>
struct TileView {
  const S* W[8];
  const S* D[6];
  const S* F[3][8];
  const S* Q[21];
  int st1, c;
  long cg;
};

// optional source terms of the update, compiled in per instantiation so that the
// default stage carries none of their registers
// OPT_PRE: the cross-derivative half-sums come precomputed from k_cross (the
// single-grid path); without it the update computes them at both neighbours.
// OPT_RES1: the resistive source in the compact form addsource_res1 instead of
// addsource_res2's (OPT_RES); the two are never combined.
// OPT_PART_A / OPT_PART_B: the update in two launches, cut after centdiff4 and
// gravity; part A stores the partial sums in the stage's output array, part B
// continues from them at the same cell, so every addition keeps its order.
enum StageOpt { OPT_DIVB = 1, OPT_RES = 2, OPT_PRE = 4, OPT_RES1 = 8, OPT_PART_A = 16, OPT_PART_B = 32 };

// Levi-Civita symbol of 0-based indices (lvc, src/vacdef.t:91)
__host__ __device__ constexpr int lvc3(int i, int j, int k) {
  return (i == j || j == k || i == k) ? 0 : ((i + 1) % 3 == j ? 1 : -1);
}
// getcurrent's idirmin (0-based): the lowest current component with a term
// eps_ijk d_j B_k, j < ndim, k < ndir (3: none, as for ndir = 1)
__host__ __device__ constexpr int res_idirmin(int ndim, int ndir) {
  int m = 3;
  for (int i = 2; i >= (6 - 2 * ndir > 0 ? 6 - 2 * ndir : 0); --i)
    for (int j = 0; j < ndim; ++j)
      for (int k = 0; k < ndir; ++k)
        if (lvc3(i, j, k) != 0) m = i;
  return m;
}

// k_update body at the mesh cell pos
template <int NDIM, int NDIR, typename S, int OPT, bool TILE = false>
__device__ __forceinline__ void update_cell(const Stage2Args& a, const Geom& g, const Offs& o, const int pos[3],
                                            double qdt_d, double qdt2_d, double tdep, double drvA,
                                            double& numax_out, const TileView<S>* tv = nullptr) {
  static_assert(!TILE || (OPT & (OPT_DIVB | OPT_RES | OPT_RES1 | OPT_PRE | OPT_PART_A | OPT_PART_B)) == 0,
                "the tile form computes the default sources with inline cross terms");
  using PR = Pairs<NDIM>;
  using T = S;
  constexpr int NP = 2 * NDIR + 2, E = NDIR + 1, B0 = NDIR + 1;
  T numax = T(0);
  {
    // stencil fields at c and its neighbours (st); the cell's own global fields at cg
    const int st[3] = {1, TILE ? tv->st1 : (int)g.st[1], TILE ? 0 : (int)g.st[2]};
    const int c = TILE ? tv->c : pos[0] + st[1] * pos[1] + st[2] * pos[2];
    const long cg = TILE ? tv->cg : (long)c;
    const long stg[3] = {1, g.st[1], g.st[2]};
    auto W = [&](int iw) {
      if constexpr (TILE) return tv->W[iw];
      else return (const S*)a.fW[iw] + o.P;
    };
    auto Df = [&](int i) {
      if constexpr (TILE) return tv->D[i];
      else return (const S*)a.fD[i] + o.I;
    };
    auto FF = [&](int d, int iw) {
      if constexpr (TILE) return tv->F[d][iw];
      else return (const S*)a.fF[d][iw] + o.I;
    };
    auto QQ = [&](int ip) {
      if constexpr (TILE) return tv->Q[ip];
      else return (const S*)a.fQ[ip] + o.I;
    };
    auto BG = [&](int i) { return a.fBG[i] + o.B; };
    const S* base = (const S*)a.base + o.P;
    const long sP = a.sP;
    T acc[NP];
    if constexpr ((OPT & OPT_PART_B) != 0) {
      const S* part = (const S*)a.out + o.P;  // part A's sums after centdiff4 and gravity
#pragma unroll
      for (int iw = 0; iw < NP; ++iw) acc[iw] = part[iw * sP + cg];
    } else {
#pragma unroll
      for (int iw = 0; iw < NP; ++iw) acc[iw] = base[iw * sP + cg];
    }
    T dxv[NDIM];
#pragma unroll
    for (int d = 0; d < NDIM; ++d) dxv[d] = (T)__ldg(a.fDX[d] + o.X + cg);
    // gradient4 (src/vacgrid.t:684): -(q(+2) - 8(q(+1)-q(-1)) - q(-2))/dx/12, zero on
    // the first and last two mesh cells along its dimension (:690-709)
    bool z4[NDIM];
#pragma unroll
    for (int d = 0; d < NDIM; ++d) z4[d] = pos[d] <= g.lo[d] + 1 || pos[d] >= g.hi[d] - 1;
    auto g4 = [&](const S* q, int s, T dxd) {
      return -(ldt<TILE>(q, c + 2 * s) - T(8) * (ldt<TILE>(q, c + s) - ldt<TILE>(q, c - s)) - ldt<TILE>(q, c - 2 * s)) / dxd / T(12);
    };
    const T qdt = (T)qdt_d;

    const T q2 = (T)qdt2_d;
    // --- centdiff4 (src/vaccd.t:35-70) -----------------------------------------
    if constexpr ((OPT & OPT_PART_B) == 0) {
#pragma unroll
    for (int d = 0; d < NDIM; ++d) {
      if (d < a.dmin || d > a.dmax) continue;
      if (!z4[d]) {
#pragma unroll
        for (int iw = 0; iw < NP; ++iw) {
          if (iw == B0 + 1 + d) continue;  // no flux of b_d along d
          if (!((a.iwmask >> iw) & 1u)) continue;
          acc[iw] = acc[iw] - qdt * g4(FF(d, iw), st[d], dxv[d]);
        }
      }
      if ((a.iwmask >> E) & 1u) {
        const S* vd = Df(1 + d);
        if (!z4[d]) {
          // getptotal_bg, src/vacphys0.t.mhd:221
          double bgs = 0.0;
#pragma unroll
          for (int C = 0; C < NDIR; ++C) bgs = bgs + __ldg(BG(2 + C) + cg) * __ldg(BG(2 + C) + cg);
          const T fb = (T)((a.gamma - 1.0) * __ldg(BG(0) + cg) - 0.5 * (a.gamma - 2.0) * bgs);
          acc[E] = acc[E] - qdt * g4(vd, st[d], dxv[d]) * fb;
        }
#pragma unroll
        for (int di = 0; di < NDIM; ++di) {
          if (di < a.dmin || di > a.dmax || z4[di]) continue;
          acc[E] = acc[E] + qdt * (T)__ldg(BG(2 + di) + cg) * (T)__ldg(BG(2 + d) + cg) * g4(vd, st[di], dxv[di]);
        }
      }
    }

    // --- gravity, src/vacusr.gravity.t:46-78 ---------------------------------------
    if (a.grav_on) {
      const T rho = ldt<TILE>(W(0), c);
#pragma unroll
      for (int d = 0; d < NDIM; ++d)
        if (((a.iwmask >> (1 + d)) & 1u) && fabs(a.grav[d]) > kSmall)
          acc[1 + d] = acc[1 + d] + q2 * (T)a.grav[d] * rho;
      if ((a.iwmask >> E) & 1u) {
        const T rt = ldt<TILE>(Df(0), c);
#pragma unroll
        for (int d = 0; d < NDIM; ++d)
          if (fabs(a.grav[d]) > kSmall) acc[E] = acc[E] + q2 * (T)a.grav[d] * rho * ldt<TILE>(W(1 + d), c) / rt;
      }
    }
    }  // centdiff4 and gravity
    if constexpr ((OPT & OPT_PART_A) != 0) {
      S* part = (S*)a.out + o.P;
#pragma unroll
      for (int iw = 0; iw < NP; ++iw) part[iw * sP + cg] = acc[iw];
    } else {

    // --- hyperdiffusion, src/vacusr.viscosity.t:2-221 --------------------------------
    if (a.visc_on) {
      // gradient1* zero rule: edge mesh cells along a non-periodic dimension
      bool z1[NDIM];
#pragma unroll
      for (int d = 0; d < NDIM; ++d)
        z1[d] = (a.zero1[d][0] && pos[d] == g.lo[d]) || (a.zero1[d][1] && pos[d] == g.hi[d]);
      auto nus = [&](int ip, int k, int j, T dxk, T& nl, T& nr) {
        const S* Qp = QQ(ip);
        nr = ldt<TILE>(Qp, j) * dxk;
        nl = ldt<TILE>(Qp, j - st[k]) * dxk;
      };
      // density and the "173" energy, :45-64
#pragma unroll
      for (int pass = 0; pass < 2; ++pass) {
        const S* q = pass == 0 ? W(0) : Df(NDIR + 1);
        const int tgt = pass == 0 ? 0 : E;
#pragma unroll
        for (int k = 0; k < NDIM; ++k) {
          T nl, nr;
          nus(pass == 0 ? PR::rho(k) : PR::e(k), k, c, dxv[k], nl, nr);
          numax = fmaxT(numax, fmaxT(nr, nl));
          const T qc = ldt<TILE>(q, c);
          const T gL = z1[k] ? T(0) : (qc - ldt<TILE>(q, c - st[k])) / dxv[k];
          const T gR = z1[k] ? T(0) : (ldt<TILE>(q, c + st[k]) - qc) / dxv[k];
          const T tL = (nl + T(0)) * gL, tR = (nr + T(0)) * gR;
          acc[tgt] = acc[tgt] + (tR - tL) / dxv[k] * q2;
        }
      }
      // momentum, :69-133
      const S* rtf = Df(0);
#pragma unroll
      for (int k = 0; k < NDIM; ++k) {
        const int sk = st[k];
        const T dxk = dxv[k];
        const T rC = ldt<TILE>(rtf, c);
        const T rL = (rC + ldt<TILE>(rtf, c - sk)) / T(2), rR = (ldt<TILE>(rtf, c + sk) + rC) / T(2);
#pragma unroll
        for (int l = 0; l < NDIM; ++l) {
          const S* q = Df(1 + l);  // v_l
          T nl, nr;
          nus(PR::v(l, k), k, c, dxk, nl, nr);
          numax = fmaxT(numax, fmaxT(nr, nl));
          const T qc = ldt<TILE>(q, c);
          const T gL = z1[k] ? T(0) : (qc - ldt<TILE>(q, c - sk)) / dxk;
          const T gR = z1[k] ? T(0) : (ldt<TILE>(q, c + sk) - qc) / dxk;
          const T tL = (nl + T(0)) * gL, tR = (nr + T(0)) * gR;
          const S* ml = W(1 + l);
          const T mc = ldt<TILE>(ml, c);
          const T VL = (mc + ldt<TILE>(ml, c - sk)) / T(2), VR = (ldt<TILE>(ml, c + sk) + mc) / T(2);
          const T t2m = (rR * tR - rL * tL) / dxk / T(2);
          const T t2e = (VR * tR - VL * tL) / dxk / T(2);
          // ii1=0: i=k, ii0=l
          acc[1 + l] = acc[1 + l] + t2m * q2;
          acc[E] = acc[E] + t2e * q2;
          if (l == k) {
            // ii1=1 with l==k takes the i==k branch a second time
            acc[1 + l] = acc[1 + l] + t2m * q2;
            acc[E] = acc[E] + t2e * q2;
          } else {
            // ii1=1: i=l, ii0=k
            const int sl = st[l];
            T Tm[2], Te[2];
#pragma unroll
            for (int sg = 0; sg < 2; ++sg) {
              const int j = sg ? c + sl : c - sl;
              const long jg = sg ? cg + stg[l] : cg - stg[l];
              const int pl = pos[l] + (sg ? 1 : -1);
              T H = T(0);
              if (pl >= g.lo[l] && pl <= g.hi[l]) {  // nu vanishes outside the mesh
                if constexpr ((OPT & OPT_PRE) != 0) {
                  H = ldt<TILE>((const S*)a.fX[Cross<NDIM>::m(l, k)] + o.I, j);
                } else {
                  const T dxkj = (T)__ldg(a.fDX[k] + o.X + jg);
                  T njl, njr;
                  nus(PR::v(l, k), k, j, dxkj, njl, njr);
                  const T gC = z1[k] ? T(0) : (ldt<TILE>(q, j + sk) - ldt<TILE>(q, j - sk)) / dxkj / T(2);
                  H = gC * (njl + njr + T(2) * T(0)) / T(2) / T(2);
                }
              }
              Tm[sg] = ldt<TILE>(rtf, j) * H;
              Te[sg] = ldt<TILE>(W(1 + k), j) * H;
            }
            const T dxl = dxv[l];
            const T tCm = z1[l] ? T(0) : (Tm[1] - Tm[0]) / dxl / T(2);
            const T tCe = z1[l] ? T(0) : (Te[1] - Te[0]) / dxl / T(2);
            acc[1 + k] = acc[1 + k] + tCm * q2;
            acc[E] = acc[E] + tCe * q2;
          }
        }
      }
      // magnetic field, :139-215
#pragma unroll
      for (int k = 0; k < NDIM; ++k)
#pragma unroll
        for (int l = 0; l < NDIM; ++l) {
          if (k == l) continue;
          const int sk = st[k], sl = st[l];
          const T dxk = dxv[k];
          const S* q = W(B0 + 1 + l);  // b_l
          T nl, nr;
          nus(PR::b(l, k), k, c, dxk, nl, nr);
          numax = fmaxT(numax, fmaxT(nr, nl));
          // ii1=0: ii0=k, m=l, sB=-1, j=k (m /= k branch)
          {
            T K[2], Ke[2];
#pragma unroll
            for (int sg = 0; sg < 2; ++sg) {
              const int j = sg ? c + sl : c - sl;
              const long jg = sg ? cg + stg[l] : cg - stg[l];
              const int pl = pos[l] + (sg ? 1 : -1);
              T Kv = T(0);
              if (pl >= g.lo[l] && pl <= g.hi[l]) {
                if constexpr ((OPT & OPT_PRE) != 0) {
                  Kv = ldt<TILE>((const S*)a.fX[Cross<NDIM>::b(l, k)] + o.I, j);
                } else {
                  const T dxkj = (T)__ldg(a.fDX[k] + o.X + jg);
                  T njl, njr;
                  nus(PR::b(l, k), k, j, dxkj, njl, njr);
                  const T gC = z1[k] ? T(0) : (ldt<TILE>(q, j + sk) - ldt<TILE>(q, j - sk)) / dxkj / T(2);
                  Kv = gC * (njl + njr) / T(2);
                }
              }
              K[sg] = Kv;
              Ke[sg] = Kv * ldt<TILE>(W(B0 + 1 + k), j);
            }
            const T dxl = dxv[l];
            const T tC = z1[l] ? T(0) : (K[1] - K[0]) / dxl / T(2);
            const T tCe = z1[l] ? T(0) : (Ke[1] - Ke[0]) / dxl / T(2);
            acc[B0 + 1 + k] = acc[B0 + 1 + k] + T(-1) * tC * q2;
            acc[E] = acc[E] + T(-1) * tCe * q2;
          }
          // ii1=1: ii0=l, m=k, sB=+1, j=l (m == k branch)
          {
            const T qc = ldt<TILE>(q, c), qm = ldt<TILE>(q, c - sk), qp = ldt<TILE>(q, c + sk);
            const T BL = (qc + qm) / T(2), BR = (qp + qc) / T(2);
            const T gL = z1[k] ? T(0) : (qc - qm) / dxk;
            const T gR = z1[k] ? T(0) : (qp - qc) / dxk;
            const T tL = nl * gL, tR = nr * gR;
            acc[B0 + 1 + l] = acc[B0 + 1 + l] + T(1) * (tR - tL) / dxk * q2;
            acc[E] = acc[E] + T(1) * (tR * BR - tL * BL) / dxk * q2;
          }
        }
    }

    // --- user driver: tdep from the host, spatial profiles precomputed there -----------
    if (a.driver != DRV_NONE) {
      const T rtn = (T)((double)acc[0] + __ldg(BG(1) + cg));
      if (a.driver == DRV_SLOG) {
        // src/vacusr.f:1355-1375 (x1 vertical; m2, m3 driven)
        const T vvx = (T)(__ldg(a.drv + o.X + cg) * tdep * drvA);
        const T vvy = (T)(__ldg(a.drv + a.sX + o.X + cg) * tdep * drvA);
        if (NDIR >= 3) {
          acc[2] = acc[2] + rtn * vvx * q2;
          acc[3 % NP] = acc[3 % NP] + rtn * vvy * q2;
        }
        acc[E] = acc[E] + rtn * (vvx * vvx + vvy * vvy + T(0) * T(0)) * q2 / T(2);
      } else {
        const T v = (T)(drvA * tdep * __ldg(a.drv + o.X + cg) * __ldg(a.drv + a.sX + o.X + cg));
        const int comp = (a.driver == DRV_STRAT) ? 1 : 2;
        acc[comp] = acc[comp] + rtn * v * q2;
        acc[E] = acc[E] + rtn * (v * v) * q2 / T(2);
      }
    }

    // --- addsource (src/vacphys.mhd0.t:225-258) after specialsource, as addsource2
    // orders them (src/vac.t:569-571): the resistive term, then Powell's; both
    // read wCT only
    // b + bg at cell n, summed in FP64
    auto Bat = [&](int C, int n) { return (T)((double)ldt<TILE>(W(B0 + 1 + C), n) + __ldg(BG(2 + C) + n)); };

    // --- resistivity, addsource_res2 (src/vacphys.mhdres.t:231-301), constant eta ------
    // J = curl(b+bg) by getcurrent (:48-95) at the 2*ndim face neighbours, with the
    // module's gradient -(q(+1)-q(-1))/dx/2 (:304-317); each term is that gradient of
    // J eta qdt (b) or of B J eta qdt (e) on the mesh.  Walking the neighbour
    // direction d outermost keeps the reference's order of additions: d is jdir of
    // the b loop and idir of the e loop.
    constexpr int IDM = res_idirmin(NDIM, NDIR);
    auto curr = [&](int n, T J[3]) {
#pragma unroll
      for (int i = IDM; i < 3; ++i) {
        J[i] = T(0);
#pragma unroll
        for (int j = 0; j < NDIM; ++j)
#pragma unroll
          for (int k = 0; k < NDIR; ++k) {
            const int l = lvc3(i, j, k);
            if (l == 0) continue;
            const int sj = st[j];
            const T dxn = (T)__ldg(a.fDX[j] + o.X + n);
            const T gr = -(Bat(k, n + sj) - Bat(k, n - sj)) / dxn / T(2);
            J[i] = (l == 1) ? J[i] + gr : J[i] - gr;
          }
      }
    };
    if constexpr ((OPT & OPT_RES) != 0) {
      if constexpr (IDM < 3) {
        const T eta = (T)a.eta;
#pragma unroll
        for (int d = 0; d < NDIM; ++d) {
          const int s = st[d];
          T Jp[3], Jm[3];
          curr(c + s, Jp);
          curr(c - s, Jm);
          const T dxd = dxv[d];
#pragma unroll
          for (int i = 0; i < NDIR; ++i) {
            if (!((a.iwmask >> (B0 + 1 + i)) & 1u)) continue;
#pragma unroll
            for (int k = IDM; k < 3; ++k) {
              const int l = lvc3(i, d, k);
              if (l == 0) continue;
              const T gr = -(Jp[k] * eta * q2 - Jm[k] * eta * q2) / dxd / T(2);
              acc[B0 + 1 + i] = (l == 1) ? acc[B0 + 1 + i] - gr : acc[B0 + 1 + i] + gr;
            }
          }
          if ((a.iwmask >> E) & 1u) {
#pragma unroll
            for (int j = 0; j < NDIR; ++j) {
#pragma unroll
              for (int k = IDM; k < 3; ++k) {
                const int l = lvc3(d, j, k);
                if (l == 0) continue;
                const T up = Bat(j, c + s) * Jp[k] * eta * q2, um = Bat(j, c - s) * Jm[k] * eta * q2;
                const T gr = -(up - um) / dxd / T(2);
                acc[E] = (l == 1) ? acc[E] + gr : acc[E] - gr;
              }
            }
          }
        }
      }
    }

    // --- resistivity, compact form addsource_res1 (src/vacphys.mhdres.t:96-220) --------
    // per idir in order: eta times the 3-point Laplacian of B_idir = b_idir + bg_idir
    // (:160-173, the sum starting from zero) into b_idir and, times B_idir, into e
    // (:191-201); then eta J**2 into e (:205-214), J from getcurrent at this cell
    if constexpr ((OPT & OPT_RES1) != 0) {
      const T eta = (T)a.eta;
#pragma unroll
      for (int i = 0; i < NDIR; ++i) {
        const T Bc = Bat(i, c);
        T lap = T(0);
#pragma unroll
        for (int d = 0; d < NDIM; ++d) {
          const int s = st[d];
          const T dxd = dxv[d];
          lap = lap + (Bat(i, c + s) - T(2) * Bc + Bat(i, c - s)) / (dxd * dxd);
        }
        lap = lap * eta;
        if ((a.iwmask >> (B0 + 1 + i)) & 1u) acc[B0 + 1 + i] = acc[B0 + 1 + i] + q2 * lap;
        if ((a.iwmask >> E) & 1u) acc[E] = acc[E] + q2 * lap * Bc;
      }
      if constexpr (IDM < 3) {
        if ((a.iwmask >> E) & 1u) {
          T J[3];
          curr(c, J);
          T j2 = T(0);
#pragma unroll
          for (int i = IDM; i < 3; ++i) j2 = j2 + J[i] * J[i];
          acc[E] = acc[E] + q2 * eta * j2;
        }
      }
    }

    // --- Powell div B source, addsource_divb (src/vacphys.mhd0.t:263-297) ----------------
    // div B is getdivb's sum over every dimension of gradient4(b+bg) (:106-144)
    if constexpr (NDIM > 1 && (OPT & OPT_DIVB) != 0) {
      T divb = T(0);
#pragma unroll
      for (int d = 0; d < NDIM; ++d) {
        T gd = T(0);
        if (!z4[d]) {
          const int s = st[d];
          gd = -(Bat(d, c + 2 * s) - T(8) * (Bat(d, c + s) - Bat(d, c - s)) - Bat(d, c - 2 * s)) / dxv[d] / T(12);
        }
        divb = divb + gd;
      }
      divb = q2 * divb;
      const T rt = ldt<TILE>(Df(0), c);
      T sm = T(0);
#pragma unroll
      for (int C = 0; C < NDIR; ++C) {
        const T mC = ldt<TILE>(W(1 + C), c);
        const T BC = Bat(C, c);
        if ((a.iwmask >> (1 + C)) & 1u) acc[1 + C] = acc[1 + C] - BC * divb;
        if ((a.iwmask >> (B0 + 1 + C)) & 1u) acc[B0 + 1 + C] = acc[B0 + 1 + C] - mC / rt * divb;
        sm = (C == 0) ? mC * BC : sm + mC * BC;
      }
      if ((a.iwmask >> E) & 1u) acc[E] = acc[E] - sm / rt * divb;
    }

    // --- store with the Runge-Kutta epilogue (src/vac.t:450,454) ---------------------
    S* out = (S*)a.out + o.P;
    if (a.epi == EPI_PLAIN) {
#pragma unroll
      for (int iw = 0; iw < NP; ++iw) out[iw * sP + cg] = acc[iw];
    } else if (a.epi == EPI_RK4_S3) {
      S* w1 = (S*)a.aux1 + o.P;
      const S* w2 = (const S*)a.aux2 + o.P;
#pragma unroll
      for (int iw = 0; iw < NP; ++iw) {
        const T w3 = acc[iw];
        out[iw * sP + cg] = w3;
        w1[iw * sP + cg] = (w1[iw * sP + cg] + T(2) * w2[iw * sP + cg] + w3 - T(4) * base[iw * sP + cg]) / T(3);
      }
    } else {
      const S* w1 = (const S*)a.aux1 + o.P;
#pragma unroll
      for (int iw = 0; iw < NP; ++iw) out[iw * sP + cg] = acc[iw] + w1[iw * sP + cg];
    }

    }  // part B
    }
  numax_out = fmax(numax_out, (double)numax);
}

// ---------------------------------------------------------------------------
// single-grid kernels
// ---------------------------------------------------------------------------
// resident blocks per SM of the face and setnu passes (measured at 128^3, like
// the update's below: face 1.11 -> 0.82 ms in FP64 at 4 blocks, nu 1.04 -> 0.98
// ms in FP64 at 6; FP32 setnu is fastest at the 80 registers of 3 blocks, which
// the compiler chose without a bound until the argument struct grew)
#ifndef SAC_FACE_MINB_F64
#define SAC_FACE_MINB_F64 4
#endif
#ifndef SAC_FACE_MINB_F32
#define SAC_FACE_MINB_F32 4
#endif
#ifndef SAC_NU_MINB_F64
#define SAC_NU_MINB_F64 6
#endif
#ifndef SAC_NU_MINB_F32
#define SAC_NU_MINB_F32 3
#endif

template <int NDIM, int NDIR, typename S>
__global__ void __launch_bounds__(256, sizeof(S) == 8 ? SAC_FACE_MINB_F64 : SAC_FACE_MINB_F32)
    k_face(const Stage2Args a, int do_ctot) {
  __shared__ double sh[32];
  const Geom& g = a.g;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  double cm[NDIM];
#pragma unroll
  for (int d = 0; d < NDIM; ++d) cm[d] = 0.0;
  if (c < (int)g.ncell) {
    const int p0 = c % g.n[0], p1 = (c / g.n[0]) % g.n[1], p2 = c / (g.n[0] * g.n[1]);
    const bool mesh = do_ctot && p0 >= g.lo[0] && p0 <= g.hi[0] && p1 >= g.lo[1] && p1 <= g.hi[1] &&
                      p2 >= g.lo[2] && p2 <= g.hi[2];
    face_cell<NDIM, NDIR, S>(a, Offs{0, 0, 0, 0}, c, mesh, a.gamma, cm);
  }
  if (do_ctot) {
#pragma unroll
    for (int d = 0; d < NDIM; ++d) block_max_to((unsigned long long*)&a.ctot[d], cm[d], sh);
  }
}

template <int NDIM, int NDIR, typename S>
__global__ void __launch_bounds__(256, sizeof(S) == 8 ? SAC_NU_MINB_F64 : SAC_NU_MINB_F32)
    k_nu(const Stage2Args a) {
  const Geom& g = a.g;
  int ext[3], p[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) ext[d] = (d < NDIM) ? (g.hi[d] - g.lo[d] + 2) : 1;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ext[0] * ext[1] * ext[2]) return;
  p[0] = t % ext[0];
  p[1] = (t / ext[0]) % ext[1];
  p[2] = t / (ext[0] * ext[1]);
#pragma unroll
  for (int d = 0; d < 3; ++d) p[d] += (d < NDIM) ? g.lo[d] - 1 : 0;
  const int c = p[0] + (int)g.st[1] * p[1] + (int)g.st[2] * p[2];
  nu_cell<NDIM, NDIR, S>(a, g, Offs{0, 0, 0, 0}, c, p, a.ctot);
}

// k_cross body at the mesh cell pos: for every l != k the centred half-sums of
// addsource_visc's cross derivatives at this cell, which the update of the cells
// on either side along l uses (src/vacusr.viscosity.t:117-118 for the momenta,
// :195-197 for the field) -- the same expressions as the update's inline form
template <int NDIM, int NDIR, typename S>
__device__ __forceinline__ void cross_cell(const Stage2Args& a, const Geom& g, const Offs& o, const int pos[3]) {
  using PR = Pairs<NDIM>;
  using CR = Cross<NDIM>;
  using T = S;
  constexpr int B0 = NDIR + 1;
  const int st[3] = {1, (int)g.st[1], (int)g.st[2]};
  const int c = pos[0] + st[1] * pos[1] + st[2] * pos[2];
#pragma unroll
  for (int k = 0; k < NDIM; ++k) {
    const int sk = st[k];
    const bool z1 = (a.zero1[k][0] && pos[k] == g.lo[k]) || (a.zero1[k][1] && pos[k] == g.hi[k]);
    const T dxk = (T)__ldg(a.fDX[k] + o.X + c);
#pragma unroll
    for (int l = 0; l < NDIM; ++l) {
      if (l == k) continue;
      {  // momentum: v_l along k
        const S* q = (const S*)a.fD[1 + l] + o.I;
        const S* Qp = (const S*)a.fQ[PR::v(l, k)] + o.I;
        const T nr = ld(Qp, c) * dxk, nl = ld(Qp, c - sk) * dxk;
        const T gC = z1 ? T(0) : (ld(q, c + sk) - ld(q, c - sk)) / dxk / T(2);
        ((S*)a.fX[CR::m(l, k)] + o.I)[c] = gC * (nl + nr + T(2) * T(0)) / T(2) / T(2);
      }
      {  // field: b_l along k
        const S* q = (const S*)a.fW[B0 + 1 + l] + o.P;
        const S* Qp = (const S*)a.fQ[PR::b(l, k)] + o.I;
        const T nr = ld(Qp, c) * dxk, nl = ld(Qp, c - sk) * dxk;
        const T gC = z1 ? T(0) : (ld(q, c + sk) - ld(q, c - sk)) / dxk / T(2);
        ((S*)a.fX[CR::b(l, k)] + o.I)[c] = gC * (nl + nr) / T(2);
      }
    }
  }
}

// 8 resident blocks per SM (32 registers): measured at 128^3 in FP64, setnu plus
// k_cross 1.565 -> 1.499 ms per RK4 step against the unbounded 44 registers
#ifndef SAC_CROSS_MINB
#define SAC_CROSS_MINB 8
#endif
template <int NDIM, int NDIR, typename S>
__global__ void __launch_bounds__(256, SAC_CROSS_MINB) k_cross(const Stage2Args a) {
  const Geom& g = a.g;
  int pos[3];
  pos[0] = g.lo[0] + blockIdx.x * blockDim.x + threadIdx.x;
  pos[1] = g.lo[1] + blockIdx.y * blockDim.y + threadIdx.y;
  pos[2] = g.lo[2] + blockIdx.z * blockDim.z + threadIdx.z;
  if (pos[0] <= g.hi[0] && pos[1] <= g.hi[1] && pos[2] <= g.hi[2])
    cross_cell<NDIM, NDIR, S>(a, g, Offs{0, 0, 0, 0}, pos);
}

// Resident blocks of 256 threads per SM that the register budget is sized for.
// The update is latency-bound; filling more warp slots beats keeping every
// value in registers (measured at 128^3: FP64 1.91 -> 1.55 ms per launch going
// from 2 to 4 blocks, FP32 0.95 -> 0.53 ms going from 2 to 8, the extra spills
// served from L1).
#ifndef SAC_UPDATE_MINB_F64
#define SAC_UPDATE_MINB_F64 4
#endif
#ifndef SAC_UPDATE_MINB_F32
#define SAC_UPDATE_MINB_F32 8
#endif

// the 3D update's block shape per storage type (256 threads; x along the
// contiguous dimension)
#ifndef SAC_UPDATE_BLK3_F64_X
#define SAC_UPDATE_BLK3_F64_X 8
#define SAC_UPDATE_BLK3_F64_Y 8
#define SAC_UPDATE_BLK3_F64_Z 4
#endif
#ifndef SAC_UPDATE_BLK3_F32_X
#define SAC_UPDATE_BLK3_F32_X 32
#define SAC_UPDATE_BLK3_F32_Y 4
#define SAC_UPDATE_BLK3_F32_Z 2
#endif

// The FP64 3D update runs in two parts (bit 0; bit 1 would split the FP32 one):
// part A (centdiff4 and gravity) needs fewer registers and runs at 5 resident
// blocks per SM without spills, part B (hyperdiffusion to the epilogue) at 4.
// Measured at 128^3 on one B200, same box: 2.92e8 -> 3.00e8 FP64 cell-updates/s
// (update 4.47 -> 4.27 ms per step); at 4 blocks for both parts no gain; the
// FP32 update split at 8 / 6 blocks is 1 % slower and stays whole.
#ifndef SAC_UPDATE_SPLIT
#define SAC_UPDATE_SPLIT 1
#endif
#ifndef SAC_UPDATE_A_MINB_F64
#define SAC_UPDATE_A_MINB_F64 5
#endif
#ifndef SAC_UPDATE_B_MINB_F64
#define SAC_UPDATE_B_MINB_F64 4
#endif
#ifndef SAC_UPDATE_A_MINB_F32
#define SAC_UPDATE_A_MINB_F32 8
#endif
#ifndef SAC_UPDATE_B_MINB_F32
#define SAC_UPDATE_B_MINB_F32 8
#endif
template <typename S, int OPT>
constexpr int update_minb() {
  return sizeof(S) != 8 ? ((OPT & OPT_PART_A) ? SAC_UPDATE_A_MINB_F32
                                              : ((OPT & OPT_PART_B) ? SAC_UPDATE_B_MINB_F32 : SAC_UPDATE_MINB_F32))
                        : ((OPT & OPT_PART_A) ? SAC_UPDATE_A_MINB_F64
                                              : ((OPT & OPT_PART_B) ? SAC_UPDATE_B_MINB_F64 : SAC_UPDATE_MINB_F64));
}

template <int NDIM, int NDIR, typename S, int OPT>
__global__ void __launch_bounds__(256, update_minb<S, OPT>())
    k_update(const Stage2Args a) {
  __shared__ double sh[32];
  const Geom& g = a.g;
  int pos[3];
  pos[0] = g.lo[0] + blockIdx.x * blockDim.x + threadIdx.x;
  pos[1] = g.lo[1] + blockIdx.y * blockDim.y + threadIdx.y;
  pos[2] = g.lo[2] + blockIdx.z * blockDim.z + threadIdx.z;
  double numax = 0.0;
  if (pos[0] <= g.hi[0] && pos[1] <= g.hi[1] && pos[2] <= g.hi[2])
    update_cell<NDIM, NDIR, S, OPT>(a, g, Offs{0, 0, 0, 0}, pos, a.qdt, a.qdt2, a.tdep, a.drvA, numax);
  if constexpr ((OPT & OPT_PART_A) == 0) {
    if (a.visc_on) block_max_to(a.maxnu, numax, sh);
  }
}

// ---------------------------------------------------------------------------
// batched kernels: persistent CTAs walk a tile list; each tile belongs to one
// instance, whose geometry, offsets and dt come from the instance tables
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool tile_cell(const Tile& tl, const Geom& g, const int lo[3], const int hi[3],
                                          int p[3]) {
  p[0] = tl.p[0] + threadIdx.x;
  p[1] = tl.p[1] + threadIdx.y;
  p[2] = tl.p[2] + threadIdx.z;
  for (int d = 0; d < 3; ++d)
    if (p[d] < lo[d] || p[d] > hi[d]) return false;
  return true;
}

// The batched passes run 1D/2D cells, whose register needs differ from the 3D
// stage's: they keep the bounds measured on the batch (the 3D ones above cost
// the 4096-instance OT batch 3 % in FP64 and 22 % in FP32).
#ifndef SAC_BATCH_UPDATE_MINB_F64
#define SAC_BATCH_UPDATE_MINB_F64 2
#endif
#ifndef SAC_BATCH_UPDATE_MINB_F32
#define SAC_BATCH_UPDATE_MINB_F32 2
#endif

template <int NDIM, int NDIR, typename S>
__global__ void __launch_bounds__(256) kb_face(const BatchStageArgs b, double gamma) {
  __shared__ double sh[32];
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    const Tile tl = b.tiles[t];
    if (b.dyn[tl.inst].dt == 0.0) continue;  // finished (tmax): nothing to compute
    const InstInfo I = b.inst[tl.inst];  // a register copy: stores cannot alias it
    const Geom& g = I.g;
    const int lo[3] = {0, 0, 0}, hi[3] = {g.n[0] - 1, g.n[1] - 1, g.n[2] - 1};
    int p[3];
    double cm[NDIM];
#pragma unroll
    for (int d = 0; d < NDIM; ++d) cm[d] = 0.0;
    if (tile_cell(tl, g, lo, hi, p)) {
      const int c = p[0] + (int)g.st[1] * p[1] + (int)g.st[2] * p[2];
      const bool mesh = p[0] >= g.lo[0] && p[0] <= g.hi[0] && p[1] >= g.lo[1] && p[1] <= g.hi[1] &&
                        p[2] >= g.lo[2] && p[2] <= g.hi[2];
      face_cell<NDIM, NDIR, S>(b.a, I.o, c, mesh, gamma, cm);
    }
#pragma unroll
    for (int d = 0; d < NDIM; ++d) block_max_to(&b.dyn[tl.inst].ctot[d], cm[d], sh);
  }
}

template <int NDIM, int NDIR, typename S>
__global__ void __launch_bounds__(256) kb_nu(const BatchStageArgs b) {
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    const Tile tl = b.tiles[t];
    if (b.dyn[tl.inst].dt == 0.0) continue;
    const InstInfo I = b.inst[tl.inst];  // a register copy: stores cannot alias it
    const Geom& g = I.g;
    int lo[3], hi[3], p[3];
    for (int d = 0; d < 3; ++d) {
      lo[d] = d < NDIM ? g.lo[d] - 1 : 0;
      hi[d] = d < NDIM ? g.hi[d] : 0;
    }
    if (tile_cell(tl, g, lo, hi, p)) {
      const int c = p[0] + (int)g.st[1] * p[1] + (int)g.st[2] * p[2];
      nu_cell<NDIM, NDIR, S>(b.a, g, I.o, c, p, b.dyn[tl.inst].ctot);
    }
  }
}

template <int NDIM, int NDIR, typename S, int OPT>
__global__ void __launch_bounds__(256, sizeof(S) == 8 ? SAC_BATCH_UPDATE_MINB_F64 : SAC_BATCH_UPDATE_MINB_F32)
    kb_update(const BatchStageArgs b) {
  __shared__ double sh[32];
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) {
    const Tile tl = b.tiles[t];
    const InstInfo I = b.inst[tl.inst];  // a register copy: stores cannot alias it
    const Geom& g = I.g;
    int p[3];
    double numax = 0.0;
    if (b.dyn[tl.inst].dt != 0.0 && tile_cell(tl, g, g.lo, g.hi, p)) {
      // the RK4 stage steps of advect, src/vac.t:442-452; every stage sees the
      // driver at the step's start time t (advect1 is called with t)
      const InstDyn& D = b.dyn[tl.inst];
      const double dt = D.dt, drvA = D.drvA, omega = D.omega, tnow = D.t;
      const double qdt = b.stage == 0 ? dt / 2 : b.stage == 1 ? dt / 2 : b.stage == 2 ? dt : dt / 6;
      const double qdt2 = qdt * ((double)(b.a.dmax - b.a.dmin) + 1.0) / (double)g.ndim;
      const double tdep = b.a.driver != DRV_NONE ? sin(omega * tnow) : 0.0;
      update_cell<NDIM, NDIR, S, OPT>(b.a, g, I.o, p, qdt, qdt2, tdep, drvA, numax);
    }
    if (b.a.visc_on) block_max_to(&b.dyn[tl.inst].maxnu, numax, sh);
  }
}

// getdt_courant per instance: max over its mesh of cmax/dx (src/vac.t:667-694),
// for tile t of b's list (a whole block; sh: 32 doubles of shared memory)
template <int NDIM, int NDIR, typename S>
__device__ __forceinline__ void courant_tile(const BatchStageArgs& b, int t, double gamma, double* sh) {
  constexpr int E = NDIR + 1;
  {
    const Tile tl = b.tiles[t];
    const InstDyn& Dy = b.dyn[tl.inst];
    if (Dy.tmax > 0.0 && Dy.t >= Dy.tmax) return;  // finished: its dt will be 0
    const InstInfo I = b.inst[tl.inst];  // a register copy: stores cannot alias it
    const Geom& g = I.g;
    int p[3];
    double best = 0.0;
    if (tile_cell(tl, g, g.lo, g.hi, p)) {
      const int c = p[0] + (int)g.st[1] * p[1] + (int)g.st[2] * p[2];
      auto W = [&](int iw) { return (double)((const S*)b.a.fW[iw])[I.o.P + c]; };
      auto BG = [&](int i) { return b.a.fBG[i][I.o.B + c]; };
      const double rho = W(0), rhob = BG(1), eb = BG(0);
      const double rt = rho + rhob;
      double m2 = 0, b2 = 0, bb = 0, bgs = 0, Bt2 = 0;
#pragma unroll
      for (int C = 0; C < NDIR; ++C) m2 = m2 + W(1 + C) * W(1 + C);
#pragma unroll
      for (int C = 0; C < NDIR; ++C) b2 = b2 + W(E + 1 + C) * W(E + 1 + C);
#pragma unroll
      for (int C = 0; C < NDIR; ++C) bb = bb + W(E + 1 + C) * BG(2 + C);
      double q = 0.5 * m2 / rt;
      q = q + 0.5 * b2 + bb;
      const double pr = (gamma - 1.0) * (W(E) - q);
#pragma unroll
      for (int C = 0; C < NDIR; ++C) bgs = bgs + BG(2 + C) * BG(2 + C);
      const double cs2 = gamma * (pr + (gamma - 1.0) * (eb - 0.5 * bgs)) / rt;
#pragma unroll
      for (int C = 0; C < NDIR; ++C) {
        const double B = W(E + 1 + C) + BG(2 + C);
        Bt2 = Bt2 + B * B;
      }
      const double cf2 = Bt2 / rt + cs2;
#pragma unroll
      for (int d = 0; d < NDIM; ++d) {
        const double Bd = W(E + 1 + d) + BG(2 + d);
        const double cmax = sqrt(0.5 * (cf2 + sqrt(cf2 * cf2 - 4.0 * cs2 * (Bd * Bd) / rt))) + fabs(W(1 + d) / rt);
        const double r = cmax / b.a.fDX[d][I.o.X + c];
        best = (r != r) ? r : fmax(best, r);
      }
    }
    block_max_to(&b.dyn[tl.inst].courant, best, sh);
  }
}

template <int NDIM, int NDIR, typename S>
__global__ void __launch_bounds__(256) kb_courant(const BatchStageArgs b, double gamma) {
  __shared__ double sh[32];
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) courant_tile<NDIM, NDIR, S>(b, t, gamma, sh);
}

// ---------------------------------------------------------------------------
// launchers (instantiated per storage type in stage_f64.cu / stage_f32.cu)
// ---------------------------------------------------------------------------
template <typename Fn>
void dispatch_nd(const Geom& g, Fn&& f) {
  const int nd = g.ndim, nr = g.ndir;
  if (nd == 1 && nr == 1) f(std::integral_constant<int, 1>{}, std::integral_constant<int, 1>{});
  else if (nd == 1 && nr == 2) f(std::integral_constant<int, 1>{}, std::integral_constant<int, 2>{});
  else if (nd == 1 && nr == 3) f(std::integral_constant<int, 1>{}, std::integral_constant<int, 3>{});
  else if (nd == 2 && nr == 2) f(std::integral_constant<int, 2>{}, std::integral_constant<int, 2>{});
  else if (nd == 2 && nr == 3) f(std::integral_constant<int, 2>{}, std::integral_constant<int, 3>{});
  else f(std::integral_constant<int, 3>{}, std::integral_constant<int, 3>{});
}

template <typename S>
void launch_face(const Stage2Args& a0, int do_ctot, cudaStream_t st) {
  Stage2Args a = a0;
  fill_field_ptrs(a, sizeof(S));
  const int N = (int)a.g.ncell;
  dispatch_nd(a.g, [&](auto ND, auto NR) {
    k_face<decltype(ND)::value, decltype(NR)::value, S><<<(unsigned)((N + 255) / 256), 256, 0, st>>>(a, do_ctot);
  });
}

template <typename S>
void launch_nu(const Stage2Args& a0, cudaStream_t st) {
  Stage2Args a = a0;
  fill_field_ptrs(a, sizeof(S));
  long nb = 1;
  for (int d = 0; d < a.g.ndim; ++d) nb *= (a.g.hi[d] - a.g.lo[d] + 2);
  dispatch_nd(a.g, [&](auto ND, auto NR) {
    k_nu<decltype(ND)::value, decltype(NR)::value, S><<<(unsigned)((nb + 255) / 256), 256, 0, st>>>(a);
  });
}

template <typename S>
void launch_update(const Stage2Args& a0, cudaStream_t st) {
  Stage2Args a = a0;
  fill_field_ptrs(a, sizeof(S));
  const Geom& g = a.g;
  dispatch_nd(g, [&](auto ND, auto NR) {
    constexpr int NDIM = decltype(ND)::value;
    dim3 blk = NDIM == 1 ? dim3(256, 1, 1)
                         : (NDIM == 2 ? dim3(32, 8, 1)
                                      : (sizeof(S) == 8 ? dim3(SAC_UPDATE_BLK3_F64_X, SAC_UPDATE_BLK3_F64_Y, SAC_UPDATE_BLK3_F64_Z)
                                                        : dim3(SAC_UPDATE_BLK3_F32_X, SAC_UPDATE_BLK3_F32_Y, SAC_UPDATE_BLK3_F32_Z)));
    const int n0 = g.hi[0] - g.lo[0] + 1, n1 = g.hi[1] - g.lo[1] + 1, n2 = g.hi[2] - g.lo[2] + 1;
    dim3 grd((n0 + blk.x - 1) / blk.x, (n1 + blk.y - 1) / blk.y, (n2 + blk.z - 1) / blk.z);
    constexpr int NDIR = decltype(NR)::value;
    // the optional sources present for this shape: Powell's needs ndim > 1, the
    // resistive one a current component (ndir > 1)
    const int ropt = a.res_on ? (a.res_compact ? OPT_RES1 : (NDIR > 1 ? OPT_RES : 0)) : 0;
    const int opt = ((NDIM > 1 && a.divb_on) ? OPT_DIVB : 0) | ropt;
    // the FP64 single grid takes the precomputed cross terms (k_cross runs
    // whenever hyperdiffusion does; without it the terms are never reached):
    // measured at 128^3 the update fell from 5.53 to 4.41 ms per step for 0.59
    // ms of k_cross.  The FP32 update, held to 32 registers, was slower with
    // them (2.11 -> 2.39 ms) and computes them inline.
    constexpr int P = sizeof(S) == 8 ? OPT_PRE : 0;
    if constexpr (NDIM > 1) {
      if (opt == OPT_DIVB) {
        k_update<NDIM, NDIR, S, P | OPT_DIVB><<<grd, blk, 0, st>>>(a);
        return;
      }
      if (opt == (OPT_DIVB | OPT_RES)) {
        k_update<NDIM, NDIR, S, P | OPT_DIVB | OPT_RES><<<grd, blk, 0, st>>>(a);
        return;
      }
      if (opt == (OPT_DIVB | OPT_RES1)) {
        k_update<NDIM, NDIR, S, P | OPT_DIVB | OPT_RES1><<<grd, blk, 0, st>>>(a);
        return;
      }
    }
    if constexpr (NDIR > 1) {
      if (opt == OPT_RES) {
        k_update<NDIM, NDIR, S, P | OPT_RES><<<grd, blk, 0, st>>>(a);
        return;
      }
    }
    if (opt == OPT_RES1) {
      k_update<NDIM, NDIR, S, P | OPT_RES1><<<grd, blk, 0, st>>>(a);
      return;
    }
    // SAC_UPDATE_SPLIT bit 0: the FP64 3D update in two parts; bit 1: the FP32 one
    if constexpr (NDIM == 3 && (SAC_UPDATE_SPLIT & (sizeof(S) == 8 ? 1 : 2)) != 0) {
      k_update<NDIM, NDIR, S, P | OPT_PART_A><<<grd, blk, 0, st>>>(a);
      k_update<NDIM, NDIR, S, P | OPT_PART_B><<<grd, blk, 0, st>>>(a);
      return;
    }
    k_update<NDIM, NDIR, S, P><<<grd, blk, 0, st>>>(a);
  });
}

template <typename S>
void launch_cross(const Stage2Args& a0, cudaStream_t st) {
  Stage2Args a = a0;
  fill_field_ptrs(a, sizeof(S));
  const Geom& g = a.g;
  if (g.ndim < 2 || sizeof(S) != 8) return;  // no pair l != k; FP32 computes them inline
  dispatch_nd(g, [&](auto ND, auto NR) {
    constexpr int NDIM = decltype(ND)::value;
    if constexpr (NDIM > 1) {
      const dim3 blk = NDIM == 2 ? dim3(32, 8, 1) : dim3(32, 4, 2);
      const int n0 = g.hi[0] - g.lo[0] + 1, n1 = g.hi[1] - g.lo[1] + 1, n2 = g.hi[2] - g.lo[2] + 1;
      const dim3 grd((n0 + blk.x - 1) / blk.x, (n1 + blk.y - 1) / blk.y, (n2 + blk.z - 1) / blk.z);
      k_cross<NDIM, decltype(NR)::value, S><<<grd, blk, 0, st>>>(a);
    }
  });
}

// persistent grid: enough CTAs to fill every SM, each walking the tile list
inline unsigned persistent_grid(int ntiles, int per_sm) {
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const long want = (long)nsm * per_sm;
  return (unsigned)(ntiles < want ? ntiles : want);
}

template <typename S>
void launch_batch_face(const BatchStageArgs& b0, double gamma, cudaStream_t st) {
  BatchStageArgs b = b0;
  fill_field_ptrs(b.a, sizeof(S));
  if (!b.ntiles) return;
  dispatch_nd(b.a.g, [&](auto ND, auto NR) {
    kb_face<decltype(ND)::value, decltype(NR)::value, S><<<persistent_grid(b.ntiles, 8), dim3(32, 8, 1), 0, st>>>(
        b, gamma);
  });
}

template <typename S>
void launch_batch_nu(const BatchStageArgs& b0, cudaStream_t st) {
  BatchStageArgs b = b0;
  fill_field_ptrs(b.a, sizeof(S));
  if (!b.ntiles) return;
  dispatch_nd(b.a.g, [&](auto ND, auto NR) {
    kb_nu<decltype(ND)::value, decltype(NR)::value, S><<<persistent_grid(b.ntiles, 8), dim3(32, 8, 1), 0, st>>>(b);
  });
}

template <typename S>
void launch_batch_update(const BatchStageArgs& b0, dim3 blk, cudaStream_t st) {
  BatchStageArgs b = b0;
  fill_field_ptrs(b.a, sizeof(S));
  if (!b.ntiles) return;
  dispatch_nd(b.a.g, [&](auto ND, auto NR) {
    // Powell's term for ndim > 1, the resistive one for ndir > 1
    constexpr int NDIM = decltype(ND)::value;
    constexpr int NDIR = decltype(NR)::value;
    const unsigned grid = persistent_grid(b.ntiles, 2);
    const int opt = ((NDIM > 1 && b.a.divb_on) ? OPT_DIVB : 0) | ((NDIR > 1 && b.a.res_on) ? OPT_RES : 0);
    if constexpr (NDIM > 1) {
      if (opt == OPT_DIVB) {
        kb_update<NDIM, NDIR, S, OPT_DIVB><<<grid, blk, 0, st>>>(b);
        return;
      }
      if (opt == (OPT_DIVB | OPT_RES)) {
        kb_update<NDIM, NDIR, S, OPT_DIVB | OPT_RES><<<grid, blk, 0, st>>>(b);
        return;
      }
    }
    if constexpr (NDIR > 1) {
      if (opt == OPT_RES) {
        kb_update<NDIM, NDIR, S, OPT_RES><<<grid, blk, 0, st>>>(b);
        return;
      }
    }
    kb_update<NDIM, NDIR, S, 0><<<grid, blk, 0, st>>>(b);
  });
}

template <typename S>
void launch_batch_courant(const BatchStageArgs& b0, double gamma, cudaStream_t st) {
  BatchStageArgs b = b0;
  fill_field_ptrs(b.a, sizeof(S));
  if (!b.ntiles) return;
  dispatch_nd(b.a.g, [&](auto ND, auto NR) {
    kb_courant<decltype(ND)::value, decltype(NR)::value, S>
        <<<persistent_grid(b.ntiles, 8), dim3(32, 8, 1), 0, st>>>(b, gamma);
  });
}

}  // namespace sacgpu
