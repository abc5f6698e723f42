// sac_stage2d.cuh -- one RK stage of 2D grids in one kernel per tile.
//
// A CTA takes a tile of TX x TY mesh cells of one instance and computes, in
// shared memory, everything the stage's update of those cells reads:
//   phase 1  over the tile grown by 3 cells (setnu's windows reach that far): the
//            derived fields rho'+rhob, v, the "173" energy (k_face's getv and
//            tmp_nu), rho', m and b, and the fluxes along x (rows of the tile, x
//            grown by 2) and along y (columns, y grown by 2) -- the k_face
//            arithmetic (face_eval);
//   phase 2  setnu's face quotients along x and along y at the faces the update
//            and its inline cross terms read (c and c - s_k, at the tile's cells
//            and one cell around) -- the k_nu arithmetic (face_quotient), with
//            c_tot of the stage from kb_ctot;
//   phase 3  the update of each cell (update_cell in its tile form: the stencil
//            fields from shared memory, the cell's own base, background, widths,
//            driver profiles and outputs in global memory), with the RK epilogue.
// So the fluxes and setnu quotients never go to HBM.  Every value is computed by
// the same device functions as the three-pass stage, in the same order, so the
// results are those of the three-pass stage bit for bit.
#pragma once
#include "sac_stage.cuh"

namespace sacgpu {

// shared-memory layout of a TX x TY tile (row stride BW = TX + 6; box row 0 is
// the grid row y0 - 3): the point fields over all BH = TY + 6 rows, the x fluxes
// over the tile's rows, the y fluxes over the tile's rows grown by 2, the x
// quotients over the rows grown by 1, the y quotients over the rows from y0 - 1
template <int NDIR, typename S, int TX, int TY>
struct Tile2D {
  static constexpr int H = 3, BW = TX + 2 * H, BH = TY + 2 * H;
  static constexpr int NP = 2 * NDIR + 2, NFL = NP - 1;  // fluxes per dimension (no b_d along d)
  static constexpr int NPF = 9;                          // rho', m_x, m_y, b_x, b_y, rho_t, v_x, v_y, e173
  static constexpr int NQ = 5;                           // setnu pairs per dimension in 2D
  static constexpr int FX_R0 = H, FX_NR = TY;            // box rows of each family
  static constexpr int FY_R0 = H - 2, FY_NR = TY + 4;
  static constexpr int QX_R0 = H - 1, QX_NR = TY + 2;
  static constexpr int QY_R0 = H - 1, QY_NR = TY + 1;
  static constexpr int P_OFF = 0;
  static constexpr int FX_OFF = P_OFF + NPF * BW * BH;
  static constexpr int FY_OFF = FX_OFF + NFL * BW * FX_NR;
  static constexpr int QX_OFF = FY_OFF + NFL * BW * FY_NR;
  static constexpr int QY_OFF = QX_OFF + NQ * BW * QX_NR;
  static constexpr int ELEMS = QY_OFF + NQ * BW * QY_NR;
  static constexpr int BYTES = ELEMS * (int)sizeof(S);
  // point-field slots
  static constexpr int P_RHO = 0, P_M = 1, P_B = 3, P_RT = 5, P_V = 6, P_E173 = 8;
  // flux slot of variable iw along d (b_d has none)
  static __device__ __forceinline__ constexpr int fslot(int d, int iw) { return iw < NDIR + 2 + d ? iw : iw - 1; }
  // the setnu pair of Pairs<2> in slot j of dimension k: rho, e173, v_x, v_y, b_l
  static __device__ __forceinline__ constexpr int qpair(int k, int j) {
    return j == 0 ? k : j == 1 ? 2 + k : j == 2 ? 4 + k : j == 3 ? 6 + k : (k == 0 ? 9 : 8);
  }
};

// c_tot of the stage per instance: getcmax's maxima over the mesh of the stage
// input, the k_face arithmetic (face_eval with no fluxes), one atomic per block
template <int NDIM, int NDIR, typename S>
__device__ __forceinline__ void ctot_tile(const BatchStageArgs& b, int t, double gamma, double* sh) {
  {
    const Tile tl = b.tiles[t];
    if (b.dyn[tl.inst].dt == 0.0) return;  // finished (tmax): nothing to compute
    const InstInfo I = b.inst[tl.inst];
    const Geom& g = I.g;
    int p[3];
    double cm[NDIM];
#pragma unroll
    for (int d = 0; d < NDIM; ++d) cm[d] = 0.0;
    if (tile_cell(tl, g, g.lo, g.hi, p)) {
      const long c = p[0] + g.st[1] * p[1] + g.st[2] * p[2];
      face_eval<NDIM, NDIR, S>(b.a, I.o, c, true, gamma, cm, 0u, [](int, S) {}, [](int, int, S) {});
    }
#pragma unroll
    for (int d = 0; d < NDIM; ++d) block_max_to(&b.dyn[tl.inst].ctot[d], cm[d], sh);
  }
}

template <int NDIM, int NDIR, typename S>
__global__ void __launch_bounds__(256) kb_ctot(const __grid_constant__ BatchStageArgs b, double gamma) {
  __shared__ double sh[32];
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) ctot_tile<NDIM, NDIR, S>(b, t, gamma, sh);
}

// the fused stage of tile t of a tile list of 2D instances (a whole block of
// TX*TY threads; smraw: the tile memory, shred: 32 doubles of shared memory)
template <int NDIR, typename S, int TX, int TY>
__device__ __forceinline__ void stage2d_tile(const BatchStageArgs& b, int t, unsigned char* smraw, double* shred) {
  using L = Tile2D<NDIR, S, TX, TY>;
  constexpr int NDIM = 2, H = L::H, BW = L::BW, BH = L::BH, NT = TX * TY;
  constexpr int E = NDIR + 1;
  S* sm = reinterpret_cast<S*>(smraw);
  const int tid = threadIdx.x;
  {
    const Tile tl = b.tiles[t];
    const InstDyn& Dy = b.dyn[tl.inst];
    const bool live = Dy.dt != 0.0;  // uniform over the block
    if (!live) return;
    const InstInfo I = b.inst[tl.inst];
    const Geom& g = I.g;
    const int x0 = tl.p[0], y0 = tl.p[1];  // the tile's first mesh cell
    __syncthreads();  // the previous tile's readers are done with the tile memory
    // ---- phase 1: point fields and fluxes --------------------------------------
    for (int idx = tid; idx < BW * BH; idx += NT) {
      const int by = idx / BW, bx = idx - by * BW;
      const int gx = x0 - H + bx, gy = y0 - H + by;
      if (gx < 0 || gx >= g.n[0] || gy < 0 || gy >= g.n[1]) continue;
      const long c = gx + g.st[1] * gy;
      const unsigned fd = ((by >= L::FX_R0 && by < L::FX_R0 + L::FX_NR && bx >= H - 2 && bx < H + TX + 2) ? 1u : 0u) |
                          ((bx >= H && bx < H + TX && by >= L::FY_R0 && by < L::FY_R0 + L::FY_NR) ? 2u : 0u);
      double cm[NDIM];
      face_eval<NDIM, NDIR, S>(
          b.a, I.o, c, false, b.a.gamma, cm, fd,
          [&](int i, S v) {
            if (i == 0) sm[L::P_OFF + L::P_RT * BW * BH + idx] = v;
            else if (i <= NDIM) sm[L::P_OFF + (L::P_V + i - 1) * BW * BH + idx] = v;
            else if (i == NDIR + 1) sm[L::P_OFF + L::P_E173 * BW * BH + idx] = v;
          },
          [&](int d, int iw, S v) {
            if (d == 0)
              sm[L::FX_OFF + L::fslot(0, iw) * BW * L::FX_NR + (by - L::FX_R0) * BW + bx] = v;
            else
              sm[L::FY_OFF + L::fslot(1, iw) * BW * L::FY_NR + (by - L::FY_R0) * BW + bx] = v;
          });
      const S* w0 = (const S*)b.a.fW[0] + I.o.P;
      sm[L::P_OFF + L::P_RHO * BW * BH + idx] = w0[c];
#pragma unroll
      for (int l = 0; l < NDIM; ++l) {
        sm[L::P_OFF + (L::P_M + l) * BW * BH + idx] = ((const S*)b.a.fW[1 + l] + I.o.P)[c];
        sm[L::P_OFF + (L::P_B + l) * BW * BH + idx] = ((const S*)b.a.fW[E + 1 + l] + I.o.P)[c];
      }
    }
    __syncthreads();
    // ---- phase 2: setnu's face quotients ---------------------------------------
    const double* ctotp = (const double*)Dy.ctot;
    auto pfield = [&](int slot) { return (const S*)(sm + L::P_OFF + slot * BW * BH); };
    auto qsrc = [&](int k, int j) {  // the q of pair slot j along k, src/vacusr.viscosity.t:284-301
      return j == 0 ? pfield(L::P_RHO) : j == 1 ? pfield(L::P_E173) : j == 2 ? pfield(L::P_V) : j == 3 ? pfield(L::P_V + 1)
                                                                                           : pfield(L::P_B + (1 - k));
    };
#pragma unroll
    for (int k = 0; k < NDIM; ++k) {
      const int c0 = H - 1, nc = k == 0 ? TX + 1 : TX + 2;  // box columns
      const int r0 = k == 0 ? L::QX_R0 : L::QY_R0, nr = k == 0 ? L::QX_NR : L::QY_NR;
      const int off = k == 0 ? L::QX_OFF : L::QY_OFF;
      const int s = k == 0 ? 1 : BW;
      const double ct = ctotp[k];
      const S p04 = (S)(ct * 0.04), p4 = (S)(ct * 0.4);  // c_hyp, src/vacusr.viscosity.t:284-290
      for (int q = tid; q < nc * nr; q += NT) {
        const int rr = q / nc, cc = q - rr * nc;
        const int bx = c0 + cc, by = r0 + rr;
        const int gx = x0 - H + bx, gy = y0 - H + by;
        // the faces k_nu computes: lo-1 .. hi in every dimension
        if (gx < g.lo[0] - 1 || gx > g.hi[0] || gy < g.lo[1] - 1 || gy > g.hi[1]) continue;
        const int cb = bx + by * BW;
        const int pos = k == 0 ? gx : gy, lo = g.lo[k], hi = g.hi[k];
        S* qo = sm + off + (by - r0) * BW + bx;
#pragma unroll
        for (int j = 0; j < L::NQ; ++j)
          qo[j * BW * nr] = face_quotient<true>(qsrc(k, j), cb, s, pos, lo, hi, (j == 2 || j == 3) ? p4 : p04);
      }
    }
    __syncthreads();
    // ---- phase 3: the update of the tile's cells --------------------------------
    double numax = 0.0;
    {
      const int tx = tid % TX, ty = tid / TX;
      int pos[3] = {x0 + tx, y0 + ty, 0};
      if (pos[0] <= g.hi[0] && pos[1] <= g.hi[1]) {
        TileView<S> tv;
        for (int i = 0; i < 8; ++i) tv.W[i] = nullptr;
        for (int i = 0; i < 6; ++i) tv.D[i] = nullptr;
        for (int d = 0; d < 3; ++d)
          for (int i = 0; i < 8; ++i) tv.F[d][i] = nullptr;
        for (int i = 0; i < 21; ++i) tv.Q[i] = nullptr;
        tv.W[0] = pfield(L::P_RHO);
#pragma unroll
        for (int l = 0; l < NDIM; ++l) {
          tv.W[1 + l] = pfield(L::P_M + l);
          tv.W[E + 1 + l] = pfield(L::P_B + l);
          tv.D[1 + l] = pfield(L::P_V + l);
        }
        tv.D[0] = pfield(L::P_RT);
        tv.D[NDIR + 1] = pfield(L::P_E173);
#pragma unroll
        for (int iw = 0; iw < L::NP; ++iw) {
          if (iw != E + 1) tv.F[0][iw] = sm + L::FX_OFF + L::fslot(0, iw) * BW * L::FX_NR - L::FX_R0 * BW;
          if (iw != E + 2) tv.F[1][iw] = sm + L::FY_OFF + L::fslot(1, iw) * BW * L::FY_NR - L::FY_R0 * BW;
        }
#pragma unroll
        for (int j = 0; j < L::NQ; ++j) {
          tv.Q[L::qpair(0, j)] = sm + L::QX_OFF + j * BW * L::QX_NR - L::QX_R0 * BW;
          tv.Q[L::qpair(1, j)] = sm + L::QY_OFF + j * BW * L::QY_NR - L::QY_R0 * BW;
        }
        tv.st1 = BW;
        tv.c = (H + tx) + (H + ty) * BW;
        tv.cg = pos[0] + g.st[1] * pos[1];
        // the RK4 stage steps of advect, src/vac.t:442-452; every stage sees the
        // driver at the step's start time t (advect1 is called with t)
        const double dt = Dy.dt, drvA = Dy.drvA, omega = Dy.omega, tnow = Dy.t;
        const double qdt = b.stage == 0 ? dt / 2 : b.stage == 1 ? dt / 2 : b.stage == 2 ? dt : dt / 6;
        const double qdt2 = qdt * ((double)(b.a.dmax - b.a.dmin) + 1.0) / (double)g.ndim;
        const double tdep = b.a.driver != DRV_NONE ? sin(omega * tnow) : 0.0;
        update_cell<NDIM, NDIR, S, 0, true>(b.a, g, I.o, pos, qdt, qdt2, tdep, drvA, numax, &tv);
      }
    }
    if (b.a.visc_on) block_max_to(&b.dyn[tl.inst].maxnu, numax, shred);
  }
}

// resident CTAs per SM the fused stage is compiled for: FP64 2 (its 97.6 KB of
// tile memory allows no more; 128 registers), FP32 4 (64 registers, no spills for
// ndir 2)
#ifndef SAC_STAGE2D_MINB_F64
#define SAC_STAGE2D_MINB_F64 2
#endif
#ifndef SAC_STAGE2D_MINB_F32
#define SAC_STAGE2D_MINB_F32 4
#endif
template <int NDIR, typename S, int TX, int TY>
__global__ void __launch_bounds__(TX * TY, sizeof(S) == 4 ? SAC_STAGE2D_MINB_F32 : SAC_STAGE2D_MINB_F64)
    kb_stage2d(const __grid_constant__ BatchStageArgs b) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ double shred[32];
  for (int t = blockIdx.x; t < b.ntiles; t += gridDim.x) stage2d_tile<NDIR, S, TX, TY>(b, t, smraw, shred);
}

// shared-memory bytes of the fused 2D stage for a tile shape
template <int NDIR, typename S, int TX, int TY>
constexpr int stage2d_smem() {
  return Tile2D<NDIR, S, TX, TY>::BYTES;
}

// tile shapes of the fused stage (the autotuner times each; sac_stage_api.h
// gives the host the same table)
__host__ __device__ constexpr int stage2d_tx(int i) { return i == 0 ? 32 : 16; }
__host__ __device__ constexpr int stage2d_ty(int i) { return i == 0 ? 8 : 8; }

template <typename S>
void launch_batch_ctot(const BatchStageArgs& b0, cudaStream_t st) {
  BatchStageArgs b = b0;
  fill_field_ptrs(b.a, sizeof(S));
  if (!b.ntiles) return;
  dispatch_nd(b.a.g, [&](auto ND, auto NR) {
    kb_ctot<decltype(ND)::value, decltype(NR)::value, S><<<persistent_grid(b.ntiles, 8), dim3(32, 8, 1), 0, st>>>(
        b, b.a.gamma);
  });
}

// the fused stage over the tile list b.tiles of shape `shape` (tiles at mesh
// origins spaced by the shape); instances must be 2D
template <typename S>
cudaError_t launch_batch_stage2d(const BatchStageArgs& b0, int shape, cudaStream_t st) {
  BatchStageArgs b = b0;
  fill_field_ptrs(b.a, sizeof(S));
  if (!b.ntiles) return cudaSuccess;
  auto go = [&](auto NRC, auto SH) -> cudaError_t {
    constexpr int NDIR = decltype(NRC)::value, I = decltype(SH)::value;
    constexpr int TX = stage2d_tx(I), TY = stage2d_ty(I);
    constexpr int smem = stage2d_smem<NDIR, S, TX, TY>();
    auto* k = kb_stage2d<NDIR, S, TX, TY>;
    static int per_sm = 0;  // per instantiation: the resident CTAs the tile memory allows
    if (!per_sm) {
      cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
      if (e != cudaSuccess) return e;
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, TX * TY, smem);
      if (e != cudaSuccess) return e;
      if (per_sm < 1) per_sm = 1;
    }
    k<<<persistent_grid(b.ntiles, per_sm), TX * TY, smem, st>>>(b);
    return cudaGetLastError();
  };
  auto by_shape = [&](auto NRC) -> cudaError_t {
    if (shape == 1) return go(NRC, std::integral_constant<int, 1>{});
    return go(NRC, std::integral_constant<int, 0>{});
  };
  if (b.a.g.ndim != 2) return cudaErrorInvalidValue;
  if (b.a.g.ndir == 3) return by_shape(std::integral_constant<int, 3>{});
  return by_shape(std::integral_constant<int, 2>{});
}

}  // namespace sacgpu
