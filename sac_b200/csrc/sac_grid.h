// sac_grid.h -- gridsetup1 (src/vacgrid.t:556-661) on the host: extrapolate the
// coordinates into the ghost layers and one layer beyond, then
// dx = (x(+1) - x(-1))/2 over the whole grid.  Shared by the single-grid and the
// batched contexts so that both see the same cell widths as the reference.
#pragma once
#include <cmath>
#include <cstdlib>
#include <vector>

namespace sacgpu {

// g: n, lo, hi, st, ncell, ndim set.  x: ndim blocks of g.ncell (mesh part read;
// the ghost part too when fullgridini).  Outputs the full-grid x and dx.
inline void gridsetup1(const int n[3], const int lo[3], const int hi[3], int ndim, long ncell, const double* x,
                       bool fullgridini, std::vector<double>& hx, std::vector<double>& hdx) {
  const long st1 = n[0], st2 = (long)n[0] * n[1];
  int qn[3], qo[3];
  for (int d = 0; d < 3; ++d) {
    qn[d] = (d < ndim) ? n[d] + 2 : 1;
    qo[d] = (d < ndim) ? 1 : 0;
  }
  const long qc = (long)qn[0] * qn[1] * qn[2];
  std::vector<double> qx((size_t)ndim * qc, 0.0);
  auto qid = [&](int i, int j, int k) { return (i + qo[0]) + (long)qn[0] * ((j + qo[1]) + (long)qn[1] * (k + qo[2])); };
  auto gid = [&](int i, int j, int k) { return i + st1 * j + st2 * k; };
  for (int jd = 0; jd < ndim; ++jd)
    for (int k = 0; k < n[2]; ++k)
      for (int j = 0; j < n[1]; ++j)
        for (int i = 0; i < n[0]; ++i) qx[jd * qc + qid(i, j, k)] = x[jd * ncell + gid(i, j, k)];
  for (int d = 0; d < ndim; ++d) {
    int lo3[3], hi3[3];
    for (int e = 0; e < 3; ++e) {
      lo3[e] = (e < ndim) ? -1 : 0;
      hi3[e] = (e < ndim) ? n[e] : 0;
    }
    for (int side = 0; side < 2; ++side) {
      int a, b, ixe, ixf;
      if (side == 0) {  // upper layers first
        b = n[d];
        a = fullgridini ? n[d] : hi[d] + 1;
        ixe = a - 1;
        ixf = ixe - 1;
      } else {
        a = -1;
        b = fullgridini ? -1 : lo[d] - 1;
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
                const int m = std::abs(ixe - q);
                qx[jd * qc + qid(i, j, k)] = (double)(1 + m) * qx[jd * qc + qid(ie[0], ie[1], ie[2])] -
                                             (double)m * qx[jd * qc + qid(iff[0], iff[1], iff[2])];
              }
        }
    }
  }
  hx.assign((size_t)ndim * ncell, 0.0);
  hdx.assign((size_t)ndim * ncell, 0.0);
  for (int jd = 0; jd < ndim; ++jd)
    for (int k = 0; k < n[2]; ++k)
      for (int j = 0; j < n[1]; ++j)
        for (int i = 0; i < n[0]; ++i) hx[jd * ncell + gid(i, j, k)] = qx[jd * qc + qid(i, j, k)];
  for (int d = 0; d < ndim; ++d)
    for (int k = 0; k < n[2]; ++k)
      for (int j = 0; j < n[1]; ++j)
        for (int i = 0; i < n[0]; ++i) {
          int p[3] = {i, j, k}, m[3] = {i, j, k};
          p[d] += 1;
          m[d] -= 1;
          hdx[d * ncell + gid(i, j, k)] = 0.5 * (qx[d * qc + qid(p[0], p[1], p[2])] - qx[d * qc + qid(m[0], m[1], m[2])]);
        }
}

// Spatial profiles of the Gaussian velocity drivers on the full grid, two
// blocks of ncell: the stratified workload (user 4: horizontal Gaussian of width
// up[4] about (up[2], up[3]) times a vertical one of width up[6] about x1=up[5])
// and the flux tube (user 5: a Gaussian of width up[3] about x1=up[2] times one
// of width up[5] about x2=up[4]).  The time factor A sin(omega t) is applied in
// the stage update.
inline void gauss_driver_profiles(int user, int ndim, long ncell, const double* hx, const double* up,
                                  double* out) {
  for (long q = 0; q < ncell; ++q) {
    const double x1 = hx[q], x2 = ndim > 1 ? hx[ncell + q] : 0.0, x3 = ndim > 2 ? hx[2 * ncell + q] : 0.0;
    if (user == 4) {
      const double xx = ndim > 1 ? x2 - up[2] : 0.0, yy = ndim > 2 ? x3 - up[3] : 0.0, zz = x1 - up[5];
      out[q] = std::exp(-(xx * xx + yy * yy) / (up[4] * up[4]));
      out[ncell + q] = std::exp(-(zz * zz) / (up[6] * up[6]));
    } else {
      const double zz = x1 - up[2], xx = x2 - up[4];
      out[q] = std::exp(-(zz * zz) / (up[3] * up[3]));
      out[ncell + q] = std::exp(-(xx * xx) / (up[5] * up[5]));
    }
  }
}

}  // namespace sacgpu
