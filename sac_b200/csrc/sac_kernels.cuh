// sac_kernels.cuh -- shared device code: geometry, reductions, the getdt_courant
// reduction and the one-pass ghost-cell fill (getboundary).  The stage kernels
// live in sac_stage.cuh.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace sacgpu {

constexpr double kSmall = 1.0e-99;  // smalldouble, src/vacdef.t:50
constexpr int kMaxDim = 3;

// Boundary codes (typeB strings of src/vacgrid.t:257-470)
enum BType : int8_t {
  BT_CONT = 0, BT_FIXED, BT_CONT1, BT_FIXED1, BT_GRAD1, BT_PERIODIC, BT_SYMM, BT_SYMM0, BT_ASYMM,
  BT_CONTCD4, BT_ZERO
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

// Offsets of one grid's blocks inside the arrays of the four families: advanced
// state (P: w, w1, w2, w3), background (B), per-stage intermediates (I: D, F, R)
// and grid (X: dx, driver profiles).  A single grid has all offsets 0.
struct Offs {
  long P, B, I, X;
};

// ---- many independent grids (the batched path) -----------------------------
struct InstInfo {
  Geom g;  // the grid of this instance
  Offs o;  // where its blocks start
};

// per-instance values the device updates during a step
struct InstDyn {
  double dt, t;
  double mindx2[3];  // min over the mesh of dx^2 per dimension (getdt_visc)
  double dtgrav;     // getdt_grav, fixed at the first step
  double drvA, omega;  // velocity driver amplitude and angular frequency (tdep = sin(omega t))
  double tmax;         // > 0: the run ends at exactly this time (tmaxexact); the instance then
                       // takes dt = 0 steps that leave its state untouched
  unsigned long long ctot[3], maxnu, courant;  // bits of non-negative maxima
  int it, bad;       // step counter; set when a reduction met NaN/Inf
  int visc_dt_seen;  // getdt_visc has run once, overwriting dtdiffpar with 0.25
};

// one unit of work: a tile of blockDim cells starting at p (local coordinates)
struct Tile {
  int inst;
  int p[3];
};

// 256 consecutive ghost cells of one instance (ghost-slab enumeration of k_bound)
struct GhostChunk {
  int inst;
  int start;
};

// Explicitly rounded arithmetic (never contracted into an FMA).  Used where the
// reference's rounding must be reproduced bit for bit: the inputs of setnu's
// max|d3|/max|d1| ratio, which is ill-conditioned where a field is constant up to
// rounding, and the boundary extrapolations/combinations.
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double div_rn(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float div_rn(float a, float b) { return __fdiv_rn(a, b); }

// Division that skips the divide for a zero numerator, bit-identical to n / d:
// for a finite nonzero d, n / d is a zero exactly when n is one, with the sign of
// n times the sign of d, which n * d gives.  The shortcut is taken only where d
// is finite and nonzero.  An FP64 division whose numerator is zero leaves the
// fast path of the divide (measured on B200: 3.6x the time of one with a normal
// numerator); k_face divides the momenta, which are exactly zero over most of a
// run that starts from rest, by rho'+rhob.  FP32 storage keeps its plain
// (approximate) division.
template <typename T>
__device__ __forceinline__ T dvs(T n, T d) {
  if constexpr (sizeof(T) == 8) {
    if (n == T(0) && d != T(0) && fabs(d) <= 1.7976931348623157e308) return n * d;
  }
  return n / d;
}
__device__ __forceinline__ double dvs_rn(double n, double d) {
  if (n == 0.0 && d != 0.0 && fabs(d) <= 1.7976931348623157e308) return __dmul_rn(n, d);
  return __ddiv_rn(n, d);
}
__device__ __forceinline__ float dvs_rn(float n, float d) { return __fdiv_rn(n, d); }

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
// getdt_courant (src/vac.t:641-699), evaluated in FP64
// ---------------------------------------------------------------------------
// max over dimensions of cmax/dx at mesh cell (i0,i1,i2); NaN when any is NaN
template <int NDIR, typename S>
__device__ __forceinline__ double courant_cell(const Geom& g, const S* __restrict__ wp,
                                               const double* __restrict__ bgv, const double* __restrict__ dx,
                                               int i0, int i1, int i2, double gamma) {
  const long N = g.ncell;
  const long c = i0 + g.st[1] * i1 + g.st[2] * i2;
  constexpr int E = NDIR + 1;
  const double rho = (double)wp[c], rhob = bgv[N + c], eb = bgv[c];
  const double rt = rho + rhob;
  double m2 = 0, b2 = 0, bb = 0, bgs = 0, Bt2 = 0;
  double m[NDIR], b[NDIR];
#pragma unroll
  for (int C = 0; C < NDIR; ++C) {
    m[C] = (double)wp[(1 + C) * N + c];
    b[C] = (double)wp[(E + 1 + C) * N + c];
  }
#pragma unroll
  for (int C = 0; C < NDIR; ++C) m2 = m2 + m[C] * m[C];
#pragma unroll
  for (int C = 0; C < NDIR; ++C) b2 = b2 + b[C] * b[C];
#pragma unroll
  for (int C = 0; C < NDIR; ++C) bb = bb + b[C] * bgv[(2 + C) * N + c];
  double q = 0.5 * m2 / rt;
  q = q + 0.5 * b2 + bb;
  const double p = (gamma - 1.0) * ((double)wp[E * N + c] - q);
#pragma unroll
  for (int C = 0; C < NDIR; ++C) bgs = bgs + bgv[(2 + C) * N + c] * bgv[(2 + C) * N + c];
  const double cs2 = gamma * (p + (gamma - 1.0) * (eb - 0.5 * bgs)) / rt;
#pragma unroll
  for (int C = 0; C < NDIR; ++C) {
    double B = b[C] + bgv[(2 + C) * N + c];
    Bt2 = Bt2 + B * B;
  }
  const double cf2 = Bt2 / rt + cs2;
  double best = 0.0;
#pragma unroll
  for (int d = 0; d < NDIR; ++d) {  // ndim <= ndir: unrolled, m and b stay in registers
    if (d >= g.ndim) break;
    const double Bd = b[d] + bgv[(2 + d) * N + c];
    double cmax = sqrt(0.5 * (cf2 + sqrt(cf2 * cf2 - 4.0 * cs2 * (Bd * Bd) / rt))) + fabs(m[d] / rt);
    double r = cmax / dx[d * N + c];
    if (r != r) return r;
    best = fmax(best, r);
  }
  return best;
}

// NaN-sticky running max of non-negative values
__device__ __forceinline__ double max_sticky(double best, double r) {
  return (r != r || best != best) ? __longlong_as_double(0x7ff8000000000000ll) : fmax(best, r);
}

// k_courant: max over the mesh of courant_cell, one atomic per block
template <int NDIR, typename S>
__global__ void k_courant(const __grid_constant__ Geom g, const S* __restrict__ wp, const double* __restrict__ bgv,
                          const double* __restrict__ dx, unsigned long long* out, double gamma) {
  __shared__ double sh[32];
  double best = 0.0;
  // 32-bit decode: sac_set_grid keeps the grid's cell offsets below 2^31
  const unsigned nm0 = g.hi[0] - g.lo[0] + 1, nm1 = g.hi[1] - g.lo[1] + 1, nm2 = g.hi[2] - g.lo[2] + 1;
  const unsigned tot = nm0 * nm1 * nm2;
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += gridDim.x * blockDim.x) {
    const unsigned q = t / nm0;
    const int i0 = g.lo[0] + (int)(t - q * nm0);
    const int i1 = g.lo[1] + (int)(q % nm1);
    const int i2 = g.lo[2] + (int)(q / nm1);
    best = max_sticky(best, courant_cell<NDIR, S>(g, wp, bgv, dx, i0, i1, i2, gamma));
  }
  block_max_to(out, best, sh);
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
  void* A;                          // perturbed block of the target array (np vars, storage type)
  double* bgA;                      // background block (nw-np vars)
  const int8_t* __restrict__ type;  // [iw*nB + iB]
  const int* __restrict__ fixed;    // [iw*nB + iB] 1 once fixB holds values
  const double* __restrict__ fixB;  // compact slabs, region iB at fixoff[iB]
  long fixoff[6];
  long slab[6];                     // cells per variable in region iB
  long sA, oA;                      // field stride and offset of the advanced blocks (A, aux)
  long sB, oB;                      // field stride and offset of the background block
  int pairshift[3][2];              // periodic source offset along d for lower/upper ghosts
  int init;                         // first call: fixed acts as cont, or keeps the values read (fullgridini)
  int fullgridini;
  int mode;                         // 0 plain, 1 RK4 stage-3 epilogue, 2 RK4 final combination
  void* aux1;                       // w1 (mode 1: written; mode 2: read)
  const void* aux2;                 // w2 (mode 1)
  const void* basep;                // w (mode 1)
};

__device__ __forceinline__ long fix_index(const Geom& g, int d, bool up, int p0, int p1, int p2) {
  const int e0 = g.ndim > 0 ? g.n[0] : 1, e1 = g.ndim > 1 ? g.n[1] : 1;
  const int x0 = d == 0 ? g.lo[0] : e0, x1 = d == 1 ? g.lo[1] : e1;  // the slab's extent
  const int pd = d == 0 ? p0 : (d == 1 ? p1 : p2);
  const int qd = up ? pd - (g.hi[d] + 1) : pd;
  const int q0 = d == 0 ? qd : p0, q1 = d == 1 ? qd : p1, q2 = d == 2 ? qd : p2;
  return q0 + (long)x0 * (q1 + (long)x1 * q2);
}

template <typename S>
__device__ __forceinline__ double bc_read(const BcArgs& a, int iw, long c) {
  const int np = a.g.np;
  return iw < np ? (double)((const S*)a.A)[(long)iw * a.sA + a.oA + c] : a.bgA[(long)(iw - np) * a.sB + a.oB + c];
}

// Value of variable iw at cell (p0,p1,p2) (mesh or ghost).  fixed_leaf/leaf
// report a chain that ended in a stored fixB value (needed by the RK4 final
// combination).  The coordinates are scalars, so that replacing the one along
// the ghost dimension is a select rather than a store to a local array.
template <int DEPTH, typename S>
__device__ double bc_resolve(const BcArgs& a, int iw, int p0, int p1, int p2, bool& fixed_leaf, long& leaf) {
  const long c = p0 + a.g.st[1] * p1 + a.g.st[2] * p2;
  int d = -1;
  if (a.g.ndim > 0 && (p0 < a.g.lo[0] || p0 > a.g.hi[0])) d = 0;
  if (a.g.ndim > 1 && (p1 < a.g.lo[1] || p1 > a.g.hi[1])) d = 1;
  if (a.g.ndim > 2 && (p2 < a.g.lo[2] || p2 > a.g.hi[2])) d = 2;
  if constexpr (DEPTH == 0) {
    return bc_read<S>(a, iw, c);
  } else {
    if (d < 0) return bc_read<S>(a, iw, c);
    const int pd = d == 0 ? p0 : (d == 1 ? p1 : p2);
    const int lo = a.g.lo[d], hi = a.g.hi[d];
    const bool up = pd > hi;
    const int iB = 2 * d + (up ? 1 : 0);
    const int nB = 2 * a.g.ndim;
    const int t = a.type[iw * nB + iB];
    const int edge = up ? hi : lo;
    auto at = [&](int q) {
      return bc_resolve<DEPTH - 1, S>(a, iw, d == 0 ? q : p0, d == 1 ? q : p1, d == 2 ? q : p2, fixed_leaf, leaf);
    };
    const bool isfixed = a.fixed[iw * nB + iB] != 0;
    auto fbv = [&]() { return a.fixB[a.fixoff[iB] + (long)iw * a.slab[iB] + fix_index(a.g, d, up, p0, p1, p2)]; };
    switch (t) {
      case BT_CONT:
        return at(edge);
      case BT_FIXED:
        if (isfixed) {
          fixed_leaf = true;
          leaf = c;
          return fbv();
        }
        if (a.init && a.fullgridini) return bc_read<S>(a, iw, c);
        return at(edge);
      case BT_PERIODIC:
        return at(pd + a.pairshift[d][up ? 1 : 0]);
      case BT_SYMM:
      case BT_SYMM0:
        return at(up ? 2 * hi + 1 - pd : 2 * lo - 1 - pd);
      case BT_ASYMM:
        return -at(up ? 2 * hi + 1 - pd : 2 * lo - 1 - pd);
      case BT_CONTCD4: {  // reflection about the edge cell, src/vacgrid.t:261-293
        const int n = up ? pd - hi : lo - pd;
        return at(up ? hi - n : lo + n);
      }
      default: {  // cont1, fixed1, grad1, src/vacgrid.t:373-409
        if (isfixed) {
          if (t == BT_GRAD1) return fbv() + at(edge);
          fixed_leaf = true;
          leaf = c;
          return fbv();
        }
        if (t != BT_CONT1 && a.init && a.fullgridini) return bc_read<S>(a, iw, c);
        const int f = up ? edge - 1 : edge + 1;
        const int n = abs(pd - edge);
        const double ve = at(edge), vf = at(f);
        return sub_rn(mul_rn((double)(n + 1), ve), mul_rn((double)n, vf));
      }
    }
  }
}

// number of ghost cells in each slab of highest ghost dimension d
__host__ __device__ inline void ghost_slabs(const Geom& g, long ns[3]) {
  for (int d = 0; d < 3; ++d) {
    ns[d] = 0;
    if (d >= g.ndim) continue;
    long n = 2L * g.lo[d];
    for (int e = 0; e < g.ndim; ++e) {
      if (e < d) n *= g.n[e];
      if (e > d) n *= (g.hi[e] - g.lo[e] + 1);
    }
    ns[d] = n;
  }
}

// Ghost cells enumerated slab by slab: slab d holds the cells whose highest ghost
// dimension is d (all coordinates for dims < d, mesh coordinates for dims > d).
template <typename S>
__device__ void bound_cell(const BcArgs& a, long t, const long ns[3], int iw0, int iw1) {
  const Geom& g = a.g;
  int d;
  long r;
  if (t < ns[0]) {
    d = 0;
    r = t;
  } else if (t < ns[0] + ns[1]) {
    d = 1;
    r = t - ns[0];
  } else {
    d = 2;
    r = t - ns[0] - ns[1];
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
  // 32-bit decode: a slab holds fewer cells than the grid, whose cell offsets
  // sac_set_grid keeps below 2^31
  const unsigned ur = (unsigned)r, e0 = (unsigned)ext[0], e1 = (unsigned)ext[1];
  const unsigned q0 = ur / e0;
  int p[3];
  p[0] = (int)(ur - q0 * e0);
  p[1] = (int)(q0 % e1);
  p[2] = (int)(q0 / e1);
  for (int e = 0; e < 3; ++e) p[e] += off[e];
  if (p[d] >= g.lo[d]) p[d] = g.hi[d] + 1 + (p[d] - g.lo[d]);  // upper layers
  const long c = p[0] + g.st[1] * p[1] + g.st[2] * p[2];
  for (int iw = iw0; iw < iw1; ++iw) {
    bool fl = false;
    long leaf = 0;
    double v = bc_resolve<3, S>(a, iw, p[0], p[1], p[2], fl, leaf);
    const bool pert = iw < g.np;
    S* A = (S*)a.A;
    S* w1 = (S*)a.aux1;
    if (a.mode == 2 && pert && fl) v = (double)((S)v + w1[(long)iw * a.sA + a.oA + leaf]);
    if (pert)
      A[(long)iw * a.sA + a.oA + c] = (S)v;
    else
      a.bgA[(long)(iw - g.np) * a.sB + a.oB + c] = v;
    if (a.mode == 1 && pert) {
      const long o = (long)iw * a.sA + a.oA + c;
      const S* w2 = (const S*)a.aux2;
      const S* w0 = (const S*)a.basep;
      w1[o] = div_rn(sub_rn(add_rn(add_rn(w1[o], S(2) * w2[o]), (S)v), S(4) * w0[o]), S(3));
    }
  }
}

// __grid_constant__: the resolver takes the parameters by reference, which
// would otherwise copy the whole struct to each thread's stack
template <typename S>
__global__ void k_bound(const __grid_constant__ BcArgs a, long nslab0, long nslab1, long nslab2, int nvar) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const long ns[3] = {nslab0, nslab1, nslab2};
  if (t >= nslab0 + nslab1 + nslab2) return;
  bound_cell<S>(a, t, ns, 0, nvar);
}

// batched: persistent CTAs of 256 threads walk the ghost chunks of all instances.
// The instance's arguments live in shared memory, written once per chunk by one
// thread: a per-thread copy would put the whole struct on every thread's stack.
// One chunk t per call (a whole block); a: the block's shared copy.
template <typename S>
__device__ __forceinline__ void bound_chunk(const BcArgs& proto, const InstInfo* __restrict__ inst,
                                            const GhostChunk* __restrict__ chunks, int t, int nvar,
                                            const InstDyn* __restrict__ dyn, BcArgs& a) {
  {
    const GhostChunk ch = chunks[t];
    if (dyn && dyn[ch.inst].dt == 0.0) return;  // a finished instance keeps its state (uniform per block)
    __syncthreads();  // the previous chunk's readers are done with a
    if (threadIdx.x == 0) {
      a = proto;
      const InstInfo& I = inst[ch.inst];
      a.g = I.g;
      a.oA = I.o.P;
      a.oB = I.o.B;
      for (int d = 0; d < 3; ++d) {  // periodic sources one mesh extent away (src/vacgrid.t:109-120)
        const int nm = d < a.g.ndim ? a.g.hi[d] - a.g.lo[d] + 1 : 0;
        a.pairshift[d][0] = nm;
        a.pairshift[d][1] = -nm;
      }
    }
    __syncthreads();
    long ns[3];
    ghost_slabs(a.g, ns);
    const long k = (long)ch.start + threadIdx.x;
    if (k < ns[0] + ns[1] + ns[2]) bound_cell<S>(a, k, ns, 0, nvar);
  }
}

template <typename S>
__global__ void __launch_bounds__(256) kb_bound(const __grid_constant__ BcArgs proto, const InstInfo* __restrict__ inst,
                                                const GhostChunk* __restrict__ chunks, int nchunks, int nvar,
                                                const InstDyn* __restrict__ dyn) {
  __shared__ BcArgs a;
  for (int t = blockIdx.x; t < nchunks; t += gridDim.x) bound_chunk<S>(proto, inst, chunks, t, nvar, dyn, a);
}

// Store fixB of region (d,up) for variable iw after the first fill
// (src/vacgrid.t:476-507); grad1 stores the difference to the edge value.
template <typename S>
__global__ void k_fixcapture(Geom g, const S* __restrict__ A, const double* __restrict__ bgA, double* fixB,
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
  auto rd = [&](long cc) { return iw < g.np ? (double)A[(long)iw * g.ncell + cc] : bgA[(long)(iw - g.np) * g.ncell + cc]; };
  double v = rd(c);
  if (grad) {
    const int edge = up ? g.hi[d] : g.lo[d];
    v = v - rd(c + (long)(edge - p[d]) * g.st[d]);
  }
  fixB[off + (long)iw * slab + t] = v;
}

// ---------------------------------------------------------------------------
// user boundary regions (&boundlist ixB^LIM, idimB, upperB; src/vacgrid.t:71-99):
// getboundary fills region iB = 1..nB in order (src/vacgrid.t:227-471), one
// launch per region.  Every source a region reads lies outside it along idimB (the
// edge, the inner edge, the mirror image, the periodic pair or fixB), so the cells
// of one region are independent and one parallel pass per region, in region
// order, is the sequential result; corners that several regions cover take the
// value of the last one, as in the reference.
// ---------------------------------------------------------------------------
struct RegionArgs {
  Geom g;
  void* A;                          // advanced block (np variables, storage type), field stride g.ncell
  double* bgA;                      // background block (nw-np variables)
  const int8_t* __restrict__ type;  // [iw*nB + iB]
  const int* __restrict__ fixed;    // [iw*nB + iB] 1 once fixB holds values
  const double* __restrict__ fixB;  // this region's slab: nw blocks of `cells` values
  int lo[3], hi[3];                 // the region (0-based, inclusive; 0..0 beyond ndim)
  long shift;                       // periodic: cell offset of the source (the pair moved by dixB)
  long cells;
  int d, up, iB, nB;
  int fullgridini;  // a fixed-type variable not yet in fixB keeps the values read
};

__device__ __forceinline__ void region_cell(const RegionArgs& a, long t, int p[3]) {
  const unsigned e0 = a.hi[0] - a.lo[0] + 1, e1 = a.hi[1] - a.lo[1] + 1;
  const unsigned ut = (unsigned)t, q = ut / e0;
  p[0] = a.lo[0] + (int)(ut - q * e0);
  p[1] = a.lo[1] + (int)(q % e1);
  p[2] = a.lo[2] + (int)(q / e1);
}

template <typename S>
__global__ void __launch_bounds__(256) k_bound_region(const __grid_constant__ RegionArgs a, int iw0, int nvar) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= a.cells) return;
  const Geom& g = a.g;
  int p[3];
  region_cell(a, t, p);
  const long N = g.ncell, sd = g.st[a.d];
  const long c = p[0] + g.st[1] * p[1] + g.st[2] * p[2];
  const int pd = p[a.d];
  auto rd = [&](int iw, long cc) {
    return iw < g.np ? (double)((const S*)a.A)[(long)iw * N + cc] : a.bgA[(long)(iw - g.np) * N + cc];
  };
  const int ixe = a.up ? a.lo[a.d] - 1 : a.hi[a.d] + 1;  // the edge the region copies from
  for (int iw = iw0; iw < nvar; ++iw) {
    const int ty = a.type[iw * a.nB + a.iB];
    const bool isfixed = a.fixed[iw * a.nB + a.iB] != 0;
    double v;
    bool store = true;
    switch (ty) {
      case BT_CONT:
      case BT_FIXED:  // src/vacgrid.t:343-368
        if (isfixed)
          v = a.fixB[(long)iw * a.cells + t];
        else if (ty == BT_CONT || !a.fullgridini)
          v = rd(iw, c + (long)(ixe - pd) * sd);
        else
          store = false;
        break;
      case BT_PERIODIC:  // :411-413
        v = rd(iw, c + a.shift);
        break;
      case BT_SYMM:
      case BT_SYMM0:
      case BT_ASYMM: {  // :414-446
        const int m = a.up ? 2 * a.lo[a.d] - 1 : 2 * a.hi[a.d] + 1;
        v = rd(iw, c + (long)(m - 2 * pd) * sd);
        if (ty == BT_ASYMM) v = -v;
        break;
      }
      case BT_ZERO:     // :295-346: contCD4's copy, on the primitive variables (k_primitive before)
      case BT_CONTCD4: {  // :261-293: the plane ixmin, then the plane ixmax
        const int se = a.up ? a.lo[a.d] - 2 : a.hi[a.d] + 3, see = a.up ? a.lo[a.d] - 3 : a.hi[a.d] + 2;
        if (pd == a.hi[a.d])
          v = rd(iw, c + (long)(see - pd) * sd);
        else if (pd == a.lo[a.d])
          v = rd(iw, c + (long)(se - pd) * sd);
        else
          store = false;
        break;
      }
      default: {  // cont1, fixed1, grad1, :369-409
        if (isfixed) {
          v = a.fixB[(long)iw * a.cells + t];
          if (ty == BT_GRAD1) v = v + rd(iw, c + (long)(ixe - pd) * sd);
        } else if (ty == BT_CONT1 || !a.fullgridini) {
          const int ixf = a.up ? ixe - 1 : ixe + 1;
          const int n = abs(pd - ixe);
          v = sub_rn(mul_rn((double)(n + 1), rd(iw, c + (long)(ixe - pd) * sd)),
                     mul_rn((double)n, rd(iw, c + (long)(ixf - pd) * sd)));
        } else {
          store = false;
        }
        break;
      }
    }
    if (!store) continue;
    if (iw < g.np)
      ((S*)a.A)[(long)iw * N + c] = (S)v;
    else
      a.bgA[(long)(iw - g.np) * N + c] = v;
  }
}

// primitive and conserve over the whole grid (src/vacphys0.t.mhd:5-52), around the
// copy of a 'zero' variable: p = getpthermal into the e slot and v = m/(rho'+rhob)
// into the m slots; then e = p/(gamma-1) + ((rho'+rhob) v^2 + b^2)/2 + b.bg and
// m = (rho'+rhob) v, in the reference's order of operations
template <int NDIR, typename S>
__global__ void __launch_bounds__(256) k_primitive(const __grid_constant__ Geom g, S* __restrict__ A,
                                                   const double* __restrict__ bg, double gamma) {
  const long N = g.ncell;
  constexpr int E = NDIR + 1;
  for (long c = blockIdx.x * (long)blockDim.x + threadIdx.x; c < N; c += (long)gridDim.x * blockDim.x) {
    const double rho = (double)A[c], rhob = bg[N + c];
    double m2 = 0.0, b2 = 0.0, bb = 0.0, m[NDIR];
#pragma unroll
    for (int C = 0; C < NDIR; ++C) {
      m[C] = (double)A[(1 + C) * N + c];
      m2 = m2 + m[C] * m[C];
    }
    double q = 0.5 * m2 / (rho + rhob);
#pragma unroll
    for (int C = 0; C < NDIR; ++C) {
      const double b = (double)A[(E + 1 + C) * N + c];
      b2 = b2 + b * b;
    }
#pragma unroll
    for (int C = 0; C < NDIR; ++C) bb = bb + (double)A[(E + 1 + C) * N + c] * bg[(2 + C) * N + c];
    q = q + 0.5 * b2 + bb;
    A[E * N + c] = (S)((gamma - 1.0) * ((double)A[E * N + c] - q));
#pragma unroll
    for (int C = 0; C < NDIR; ++C) A[(1 + C) * N + c] = (S)(m[C] / (rho + rhob));
  }
}

template <int NDIR, typename S>
__global__ void __launch_bounds__(256) k_conserve(const __grid_constant__ Geom g, S* __restrict__ A,
                                                  const double* __restrict__ bg, double gamma) {
  const long N = g.ncell;
  constexpr int E = NDIR + 1;
  for (long c = blockIdx.x * (long)blockDim.x + threadIdx.x; c < N; c += (long)gridDim.x * blockDim.x) {
    const double rt = (double)A[c] + bg[N + c];
    double v2 = 0.0, b2 = 0.0, bb = 0.0, v[NDIR];
#pragma unroll
    for (int C = 0; C < NDIR; ++C) {
      v[C] = (double)A[(1 + C) * N + c];
      v2 = v2 + v[C] * v[C];
    }
#pragma unroll
    for (int C = 0; C < NDIR; ++C) {
      const double b = (double)A[(E + 1 + C) * N + c];
      b2 = b2 + b * b;
    }
#pragma unroll
    for (int C = 0; C < NDIR; ++C) bb = bb + (double)A[(E + 1 + C) * N + c] * bg[(2 + C) * N + c];
    A[E * N + c] = (S)((double)A[E * N + c] / (gamma - 1.0) + 0.5 * (rt * v2 + b2) + bb);
#pragma unroll
    for (int C = 0; C < NDIR; ++C) A[(1 + C) * N + c] = (S)(rt * v[C]);
  }
}

// fixB of a user region for variable iw after the first fill (src/vacgrid.t:476-507):
// the values, or for grad1 their differences to the region's edge
template <typename S>
__global__ void __launch_bounds__(256) k_fixcapture_region(const __grid_constant__ RegionArgs a, double* fixB,
                                                           int iw, int grad) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= a.cells) return;
  const Geom& g = a.g;
  int p[3];
  region_cell(a, t, p);
  const long N = g.ncell;
  const long c = p[0] + g.st[1] * p[1] + g.st[2] * p[2];
  auto rd = [&](long cc) {
    return iw < g.np ? (double)((const S*)a.A)[(long)iw * N + cc] : a.bgA[(long)(iw - g.np) * N + cc];
  };
  double v = rd(c);
  if (grad) {
    const int ixe = a.up ? a.lo[a.d] - 1 : a.hi[a.d] + 1;
    v = v - rd(c + (long)(ixe - p[a.d]) * g.st[a.d]);
  }
  fixB[(long)iw * a.cells + t] = v;
}

// storage conversions for the FP32 path
template <typename D, typename S>
__global__ void k_convert(D* __restrict__ dst, const S* __restrict__ src, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    dst[i] = (D)src[i];
}

}  // namespace sacgpu
