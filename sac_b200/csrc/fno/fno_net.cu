// fno_net.cu -- the Fourier neural operator: parameters, forward, backward, Adam.
//
// Activations are channel-first per sample, v[b][c][s][f] (f fastest), BF16.  A
// Fourier layer is
//     z = W v + b + K(v),   v' = GELU(z)  (no activation after the last layer)
// where the spectral convolution K keeps m1 = 24 low and 24 high frequencies
// along s and the m2 = 24 lowest along f.  It runs as truncated real DFTs on the
// tensor cores (tcgen05 GEMMs against constant cos/sin tables):
//     F1  T[(b,c),j,s]   = sum_f v[(b,c,s),f] Fy[j,f]          j: Re/Im of ky < 24
//     F2  Z[(b,c),j,r]   = sum_s T[(b,c),j,s] Fx[r,s]          r: cos/-sin rows of 48 kx
//     MIX P[(b,o),j',r]  = complex mode-wise channel mixing with R[kx,ky,i,o]
//     F4  Y[(b,o),s,j']  = sum_r P[(b,o),j',r] Fx[r,s]
//     F5  spec[(b,o,s),f]= sum_j' Y[(b,o,s),j'] Hy[f,j']        (Hermitian weights, 1/(S F))
//     F6  z = W v + spec + b, GELU                              (channel-mixing GEMM)
// which equals irfft2(R . rfft2(v)[modes]).  Lift (16 -> 32 channels) and
// projection (32 -> 128 -> 6) are channel-mixing GEMMs with fused GELU.  The
// backward pass runs the transposed chain with the same engine; weight and bias
// gradients accumulate in FP32; Adam keeps FP32 master weights and refreshes the
// BF16 copies the GEMMs read.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "fno_gemm.cuh"
#include "fno_host.h"
#include "fno_proj.cuh"
#include "sac_fno.h"

using namespace fno;

namespace {

constexpr int kJ = 48;  // 2 * m2 (Re, Im of ky = 0..23)
constexpr int kR = 96;  // 2 * 2 * m1 rows (cos, -sin) of 48 kx

// ---------------------------------------------------------------------------
// small kernels
// ---------------------------------------------------------------------------
__global__ void k_f2bf(bf16* dst, const float* src, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    dst[i] = __float2bfloat16(src[i]);
}

// mode-wise complex channel mixing, one block per ky and 8 consecutive kx rows
// q0..q0+7 (so that each row of Z and P is read and written in 32-byte runs):
//   U = Z[q,ky]-Z[48+q,24+ky] + i(Z[q,24+ky]+Z[48+q,ky]),  O[o] = sum_i U[i] R[i,o]
//   P[ky][q]=Or, P[ky][48+q]=Oi, P[24+ky][q]=Oi, P[24+ky][48+q]=-Or
// Shared memory: R of the 8 modes as [i][o][j] and U as [(b,i)][j], j = q - q0
// fastest, so that a warp's reads of both are conflict-free.
constexpr int kMixQ = 8;
__global__ void __launch_bounds__(256) k_mix_fwd(const float* __restrict__ zt, const bf16* __restrict__ Rr,
                                                 const bf16* __restrict__ Ri, bf16* __restrict__ pt, int B, int W,
                                                 int m2) {
  extern __shared__ float sh[];
  float* rr = sh;
  float* ri = rr + kMixQ * W * W;
  float* ur = ri + kMixQ * W * W;
  float* ui = ur + kMixQ * B * W;
  const int ky = blockIdx.x % m2, q0 = (blockIdx.x / m2) * kMixQ;
  const int WW = W * W;
  // the loads of each loop are issued in groups of 8 before their stores, so that
  // a thread has several in flight (one block per SM leaves few warps to hide them)
  for (int t0 = threadIdx.x; t0 < kMixQ * WW; t0 += 8 * blockDim.x) {
    bf16 vr[8], vi[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int t = t0 + u * blockDim.x;
      if (t < kMixQ * WW) {
        const int j = t / WW, e = t - j * WW;  // e = i*W + o of mode (q0 + j, ky)
        const long moff = ((long)(q0 + j) * m2 + ky) * WW;
        vr[u] = Rr[moff + e];
        vi[u] = Ri[moff + e];
      }
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int t = t0 + u * blockDim.x;
      if (t < kMixQ * WW) {
        const int j = t / WW, e = t - j * WW;
        rr[e * kMixQ + j] = __bfloat162float(vr[u]);
        ri[e * kMixQ + j] = __bfloat162float(vi[u]);
      }
    }
  }
  const int JR = kJ * kR;
  for (int t0 = threadIdx.x; t0 < kMixQ * B * W; t0 += 4 * blockDim.x) {
    float z0[4], z1[4], z2[4], z3[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int t = t0 + u * blockDim.x;
      if (t < kMixQ * B * W) {
        const int bc = t / kMixQ, q = q0 + (t % kMixQ);
        const float* z = zt + (long)bc * JR;
        z0[u] = z[ky * kR + q];
        z1[u] = z[(m2 + ky) * kR + 48 + q];
        z2[u] = z[(m2 + ky) * kR + q];
        z3[u] = z[ky * kR + 48 + q];
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int t = t0 + u * blockDim.x;
      if (t < kMixQ * B * W) {
        ur[t] = z0[u] - z1[u];
        ui[t] = z2[u] + z3[u];
      }
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < kMixQ * B * W; t += blockDim.x) {
    const int bo = t / kMixQ, j = t % kMixQ, b = bo / W, o = bo % W, q = q0 + j;
    float orr = 0.f, oii = 0.f;
    for (int i = 0; i < W; ++i) {
      const float a = ur[(b * W + i) * kMixQ + j], c = ui[(b * W + i) * kMixQ + j];
      const float xr = rr[(i * W + o) * kMixQ + j], xi = ri[(i * W + o) * kMixQ + j];
      orr += a * xr - c * xi;
      oii += a * xi + c * xr;
    }
    bf16* p = pt + (long)bo * JR;
    p[ky * kR + q] = __float2bfloat16(orr);
    p[ky * kR + 48 + q] = __float2bfloat16(oii);
    p[(m2 + ky) * kR + q] = __float2bfloat16(oii);
    p[(m2 + ky) * kR + 48 + q] = __float2bfloat16(-orr);
  }
}

// the same mixing with one block per (q, ky) mode, for widths whose 8-mode
// shared memory would not fit
//   U = Z[q,ky]-Z[48+q,24+ky] + i(Z[q,24+ky]+Z[48+q,ky]),  O[o] = sum_i U[i] R[i,o]
//   P[ky][q]=Or, P[ky][48+q]=Oi, P[24+ky][q]=Oi, P[24+ky][48+q]=-Or
__global__ void __launch_bounds__(256) k_mix_fwd_mode(const float* __restrict__ zt, const bf16* __restrict__ Rr,
                                                 const bf16* __restrict__ Ri, bf16* __restrict__ pt, int B, int W,
                                                 int m2) {
  extern __shared__ float sh[];
  float* rr = sh;
  float* ri = rr + W * W;
  float* ur = ri + W * W;
  float* ui = ur + B * W;
  const int mode = blockIdx.x, q = mode / m2, ky = mode % m2;
  const long moff = (long)mode * W * W;
  for (int t = threadIdx.x; t < W * W; t += blockDim.x) {
    rr[t] = __bfloat162float(Rr[moff + t]);
    ri[t] = __bfloat162float(Ri[moff + t]);
  }
  const int JR = kJ * kR;
  for (int t = threadIdx.x; t < B * W; t += blockDim.x) {
    const float* z = zt + (long)t * JR;
    ur[t] = z[ky * kR + q] - z[(m2 + ky) * kR + 48 + q];
    ui[t] = z[(m2 + ky) * kR + q] + z[ky * kR + 48 + q];
  }
  __syncthreads();
  for (int t = threadIdx.x; t < B * W; t += blockDim.x) {
    const int b = t / W, o = t % W;
    float orr = 0.f, oii = 0.f;
    for (int i = 0; i < W; ++i) {
      const float a = ur[b * W + i], c = ui[b * W + i], xr = rr[i * W + o], xi = ri[i * W + o];
      orr += a * xr - c * xi;
      oii += a * xi + c * xr;
    }
    bf16* p = pt + (long)t * JR;
    p[ky * kR + q] = __float2bfloat16(orr);
    p[ky * kR + 48 + q] = __float2bfloat16(oii);
    p[(m2 + ky) * kR + q] = __float2bfloat16(oii);
    p[(m2 + ky) * kR + 48 + q] = __float2bfloat16(-orr);
  }
}

// backward of k_mix_fwd with one block per ky and 8 consecutive kx rows (the
// per-mode k_mix_bwd below, regrouped as k_mix_fwd is): dZ (bf16) and dR += (fp32).
// Shared memory: R as [o][i][j] (a warp of the dZ phase reads consecutive i),
// U as [(b,i)][j] and G as [(b,o)][j], j = q - q0 fastest; the loads are issued
// in groups.  The sums run over o and over b in the per-mode kernel's order.
__global__ void __launch_bounds__(256) k_mix_bwd_g(const float* __restrict__ dpt, const float* __restrict__ zt,
                                                   const bf16* __restrict__ Rr, const bf16* __restrict__ Ri,
                                                   bf16* __restrict__ dzt, float* __restrict__ dRr,
                                                   float* __restrict__ dRi, int B, int W, int m2) {
  extern __shared__ float sh[];
  float* rr = sh;
  float* ri = rr + kMixQ * W * W;
  float* ur = ri + kMixQ * W * W;
  float* ui = ur + kMixQ * B * W;
  float* gr = ui + kMixQ * B * W;
  float* gi = gr + kMixQ * B * W;
  const int ky = blockIdx.x % m2, q0 = (blockIdx.x / m2) * kMixQ;
  const int WW = W * W, JR = kJ * kR;
  for (int t0 = threadIdx.x; t0 < kMixQ * WW; t0 += 8 * blockDim.x) {
    bf16 vr[8], vi[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int t = t0 + u * blockDim.x;
      if (t < kMixQ * WW) {
        const int j = t / WW, e = t - j * WW;  // e = i*W + o of mode (q0 + j, ky)
        const long moff = ((long)(q0 + j) * m2 + ky) * WW;
        vr[u] = Rr[moff + e];
        vi[u] = Ri[moff + e];
      }
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int t = t0 + u * blockDim.x;
      if (t < kMixQ * WW) {
        const int j = t / WW, e = t - j * WW, i = e / W, o = e - i * W;
        rr[(o * W + i) * kMixQ + j] = __bfloat162float(vr[u]);
        ri[(o * W + i) * kMixQ + j] = __bfloat162float(vi[u]);
      }
    }
  }
  for (int t0 = threadIdx.x; t0 < kMixQ * B * W; t0 += 2 * blockDim.x) {
    float z[2][4], g[2][4];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int t = t0 + u * blockDim.x;
      if (t < kMixQ * B * W) {
        const int bc = t / kMixQ, q = q0 + (t % kMixQ);
        const float* zz = zt + (long)bc * JR;
        const float* gg = dpt + (long)bc * JR;
        z[u][0] = zz[ky * kR + q], z[u][1] = zz[(m2 + ky) * kR + 48 + q];
        z[u][2] = zz[(m2 + ky) * kR + q], z[u][3] = zz[ky * kR + 48 + q];
        g[u][0] = gg[ky * kR + q], g[u][1] = gg[(m2 + ky) * kR + 48 + q];
        g[u][2] = gg[ky * kR + 48 + q], g[u][3] = gg[(m2 + ky) * kR + q];
      }
    }
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int t = t0 + u * blockDim.x;
      if (t < kMixQ * B * W) {
        ur[t] = z[u][0] - z[u][1];
        ui[t] = z[u][2] + z[u][3];
        gr[t] = g[u][0] - g[u][1];
        gi[t] = g[u][2] + g[u][3];
      }
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < kMixQ * B * W; t += blockDim.x) {  // t = ((b, i), j)
    const int bi = t / kMixQ, j = t % kMixQ, b = bi / W, i = bi % W, q = q0 + j;
    float dur = 0.f, dui = 0.f;
    for (int o = 0; o < W; ++o) {
      const float a = gr[(b * W + o) * kMixQ + j], c = gi[(b * W + o) * kMixQ + j];
      const float xr = rr[(o * W + i) * kMixQ + j], xi = ri[(o * W + i) * kMixQ + j];
      dur += a * xr + c * xi;
      dui += -a * xi + c * xr;
    }
    bf16* p = dzt + (long)bi * JR;
    p[ky * kR + q] = __float2bfloat16(dur);
    p[(m2 + ky) * kR + 48 + q] = __float2bfloat16(-dur);
    p[(m2 + ky) * kR + q] = __float2bfloat16(dui);
    p[ky * kR + 48 + q] = __float2bfloat16(dui);
  }
  for (int t = threadIdx.x; t < kMixQ * WW; t += blockDim.x) {  // t = ((i, o), j)
    const int io = t / kMixQ, j = t % kMixQ, i = io / W, o = io % W;
    float sr = 0.f, si = 0.f;
    for (int b = 0; b < B; ++b) {
      const float a = gr[(b * W + o) * kMixQ + j], c = gi[(b * W + o) * kMixQ + j];
      const float u = ur[(b * W + i) * kMixQ + j], v = ui[(b * W + i) * kMixQ + j];
      sr += a * u + c * v;
      si += -a * v + c * u;
    }
    const long moff = ((long)(q0 + j) * m2 + ky) * WW;
    dRr[moff + io] += sr;
    dRi[moff + io] += si;
  }
}

// backward of k_mix_fwd: dZ (bf16) and dR += (fp32), one block per mode
__global__ void __launch_bounds__(256) k_mix_bwd(const float* __restrict__ dpt, const float* __restrict__ zt,
                                                 const bf16* __restrict__ Rr, const bf16* __restrict__ Ri,
                                                 bf16* __restrict__ dzt, float* __restrict__ dRr,
                                                 float* __restrict__ dRi, int B, int W, int m2) {
  extern __shared__ float sh[];
  float* rr = sh;
  float* ri = rr + W * W;
  float* ur = ri + W * W;
  float* ui = ur + B * W;
  float* gr = ui + B * W;
  float* gi = gr + B * W;
  const int mode = blockIdx.x, q = mode / m2, ky = mode % m2;
  const long moff = (long)mode * W * W;
  const int JR = kJ * kR;
  for (int t = threadIdx.x; t < W * W; t += blockDim.x) {
    rr[t] = __bfloat162float(Rr[moff + t]);
    ri[t] = __bfloat162float(Ri[moff + t]);
  }
  for (int t = threadIdx.x; t < B * W; t += blockDim.x) {
    const float* z = zt + (long)t * JR;
    ur[t] = z[ky * kR + q] - z[(m2 + ky) * kR + 48 + q];
    ui[t] = z[(m2 + ky) * kR + q] + z[ky * kR + 48 + q];
    const float* g = dpt + (long)t * JR;
    gr[t] = g[ky * kR + q] - g[(m2 + ky) * kR + 48 + q];
    gi[t] = g[ky * kR + 48 + q] + g[(m2 + ky) * kR + q];
  }
  __syncthreads();
  for (int t = threadIdx.x; t < B * W; t += blockDim.x) {  // t = (b, i)
    const int b = t / W, i = t % W;
    float dur = 0.f, dui = 0.f;
    for (int o = 0; o < W; ++o) {
      const float a = gr[b * W + o], c = gi[b * W + o], xr = rr[i * W + o], xi = ri[i * W + o];
      dur += a * xr + c * xi;
      dui += -a * xi + c * xr;
    }
    bf16* p = dzt + (long)t * JR;
    p[ky * kR + q] = __float2bfloat16(dur);
    p[(m2 + ky) * kR + 48 + q] = __float2bfloat16(-dur);
    p[(m2 + ky) * kR + q] = __float2bfloat16(dui);
    p[ky * kR + 48 + q] = __float2bfloat16(dui);
  }
  for (int t = threadIdx.x; t < W * W; t += blockDim.x) {  // t = (i, o)
    const int i = t / W, o = t % W;
    float sr = 0.f, si = 0.f;
    for (int b = 0; b < B; ++b) {
      const float a = gr[b * W + o], c = gi[b * W + o], u = ur[b * W + i], v = ui[b * W + i];
      sr += a * u + c * v;
      si += -a * v + c * u;
    }
    dRr[moff + t] += sr;
    dRi[moff + t] += si;
  }
}

// out[c] += sum over b, p of d[b][c][p]  (bias gradients)
__global__ void __launch_bounds__(256) k_chan_sum(const bf16* __restrict__ d, float* __restrict__ out, int B, int C,
                                                  long P) {
  __shared__ float sh[8];
  const int c = blockIdx.y;
  float s = 0.f;
  const long tot = (long)B * P;
  for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < tot; k += (long)gridDim.x * blockDim.x) {
    const long b = k / P, p = k % P;
    s += __bfloat162float(d[(b * C + c) * P + p]);
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
    atomicAdd(out + c, t);
  }
}

// Adam with decoupled weight decay on the FP32 masters; refresh the BF16 copies
__global__ void k_adam(float* __restrict__ w, bf16* __restrict__ wb, const float* __restrict__ g,
                       float* __restrict__ m, float* __restrict__ v, long n, float lr, float b1, float b2,
                       float eps, float wd, float c1, float c2, float gscale) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const float gi = g[i] * gscale;
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    float x = w[i] * (1.f - lr * wd);
    x -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = x;
    wb[i] = __float2bfloat16(x);
  }
}

__global__ void k_sumsq(const float* __restrict__ g, long n, float* out) {
  float s = 0.f;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    s += g[i] * g[i];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

// loss = mean (y - t)^2 over the first cout channels; dy = 2 (y - t) / n as BF16
// in a buffer of cpad >= cout channels (the padding channels are zeroed)
__global__ void k_mse(const float* __restrict__ y, const bf16* __restrict__ t, bf16* __restrict__ dy, float* loss,
                      int B, int cout, int cpad, long P, float inv_n) {
  float s = 0.f;
  const long tot = (long)B * cpad * P;
  for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < tot; k += (long)gridDim.x * blockDim.x) {
    const long p = k % P, c = (k / P) % cpad, b = k / (P * cpad);
    float g = 0.f;
    if (c < cout) {
      const long o = (b * cout + c) * P + p;
      const float e = y[o] - __bfloat162float(t[o]);
      s += e * e;
      g = 2.f * e * inv_n;
    }
    dy[k] = __float2bfloat16(g);
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, s * inv_n);
}

// network input x[b][c][s][f] (bf16, cin channels):
//   0..nst-1  the state channel times scale[b*nst + c] (normalised perturbation)
//   nst..     per-sample feature planes feat[b*nfeat + k]
//   then      s/S - 1/2 and f/F, the remaining channels zero
template <typename T>
__global__ void k_features(const T* __restrict__ st, const float* __restrict__ scale,
                           const float* __restrict__ feat, bf16* __restrict__ x, int B, int nst, int nfeat, int cin,
                           int S, int F) {
  const long P = (long)S * F;
  const long tot = (long)B * cin * P;
  for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < tot; k += (long)gridDim.x * blockDim.x) {
    const long p = k % P;
    const int c = (int)((k / P) % cin), b = (int)(k / (P * cin));
    float v = 0.f;
    if (c < nst) {
      v = (float)st[((long)b * nst + c) * P + p] * (scale ? scale[b * nst + c] : 1.f);
    } else if (c < nst + nfeat) {
      v = feat[b * nfeat + (c - nst)];
    } else if (c == nst + nfeat) {
      v = (float)(p / F) / (float)S - 0.5f;
    } else if (c == nst + nfeat + 1) {
      v = (float)(p % F) / (float)F;
    }
    x[k] = __float2bfloat16(v);
  }
}

// st[b][c][p] += scale[b*nst+c] * y[b][c][p]   (apply the predicted increment)
__global__ void k_apply(float* __restrict__ st, const float* __restrict__ y, const float* __restrict__ scale,
                        int B, int nst, long P) {
  const long tot = (long)B * nst * P;
  for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < tot; k += (long)gridDim.x * blockDim.x) {
    const long bc = k / P;
    st[k] += scale[bc] * y[k];
  }
}

unsigned grid_for(long n) {
  long g = (n + 255) / 256;
  return (unsigned)(g < 148L * 32 ? (g < 1 ? 1 : g) : 148L * 32);
}

}  // namespace

// ===========================================================================
// the network object
// ===========================================================================
struct sac_fno {
  sac_fno_config cfg{};
  std::string err;
  cudaStream_t st = nullptr;
  int S = 0, F = 0, W = 0, L = 0, H = 0, cin = 0, cout = 0, cpad = 0, m1 = 0, m2 = 0, nmodes = 0;
  bool mix_grouped = false;  // k_mix_fwd's 8-mode blocks fit in shared memory
  size_t mix_bwd_max = 0;     // the shared memory k_mix_bwd_g may take (0: not used)
  long P = 0;
  // parameters: FP32 masters, BF16 copies, gradients, Adam moments (one buffer each)
  long nparam = 0;
  float *w = nullptr, *g = nullptr, *am = nullptr, *av = nullptr;
  bf16* wb = nullptr;
  struct Seg {
    long off, n;
  };
  Seg sP, sPb, sQ1, sQ1b, sQ2, sQ2b;
  std::vector<Seg> sW, sWb, sRr, sRi;
  // DFT tables (bf16)
  bf16 *Fy = nullptr, *FyT = nullptr, *Fx = nullptr, *Gx = nullptr, *Hy = nullptr, *HyT = nullptr;
  // activations of the last forward
  int Bmax = 0, Blast = 0;
  const bf16* xin = nullptr;
  std::vector<bf16*> act, pre;
  std::vector<float*> zt;
  bf16 *hpre = nullptr, *h = nullptr;
  // scratch
  bf16 *tp = nullptr, *pt = nullptr, *yb = nullptr, *dz = nullptr, *dz2 = nullptr, *dyt = nullptr, *dzt = nullptr,
       *dtp = nullptr, *dhpre = nullptr, *dyb = nullptr;
  float *spec = nullptr, *dvacc = nullptr, *dpt = nullptr, *scal = nullptr;
  int* errw = nullptr;
  int wait_tries = 0;  // GemmDesc::wait_tries of every launch (0: default bound)
};

namespace {

int fail(sac_fno* n, const std::string& m) {
  if (n) n->err = m;
  set_error(m);
  return 1;
}

#define FK(call)                                                                        \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess) {                                                            \
      if (n) n->err = std::string(#call) + ": " + cudaGetErrorString(e_);               \
      set_error(n ? n->err : std::string(cudaGetErrorString(e_)));                      \
      return 3;                                                                         \
    }                                                                                   \
  } while (0)

#define GK(desc)                      \
  do {                                \
    GemmDesc d_ = (desc);             \
    d_.wait_tries = n->wait_tries;    \
    int rc_ = gemm(d_, n->st);        \
    if (rc_) return rc_;              \
  } while (0)

GemmDesc gd(int M, int N, int K, int batch = 1) {
  GemmDesc d;
  std::memset(&d, 0, sizeof(d));
  d.M = M;
  d.N = N;
  d.K = K;
  d.batch = batch;
  d.ksplit = 1;
  d.a_msplit = 1 << 30;
  d.b_nsplit = 1 << 30;
  d.c_msplit = 1 << 30;
  d.alpha = 1.f;
  return d;
}

// row index m = p (a pixel) within sample b; X[b][k][p] as an MN-major operand
void a_chanfirst(GemmDesc& d, const bf16* x, int K, long P) {
  d.a = x;
  d.a_mn_major = 1;
  d.a_m0 = 1;
  d.a_k = P;
  d.a_b = (long)K * P;
}
// C[b][n][p]
void c_chanfirst(GemmDesc& d, void* c, int N, long P, int bf) {
  d.c = c;
  d.c_m0 = 1;
  d.c_n = P;
  d.c_b = (long)N * P;
  d.c_bf16 = bf;
}

// ---------------------------------------------------------------------------
// train: keep what the backward pass needs (pre-activations, the input pointer)
int forward(sac_fno* n, const bf16* x, float* y, int B, bool train) {
  const int S = n->S, F = n->F, W = n->W, H = n->H;
  const long P = n->P;
  n->xin = train ? x : nullptr;
  n->Blast = B;
  // lift: v0[b][o][p] = sum_c Pw[o][c] x[b][c][p] + pb[o]
  {
    GemmDesc d = gd((int)P, W, n->cin, B);
    a_chanfirst(d, x, n->cin, P);
    d.b = n->wb + n->sP.off;
    d.b_n = n->cin;
    d.b_k = 1;
    c_chanfirst(d, n->act[0], W, P, 1);
    d.bias_n = n->w + n->sPb.off;
    d.err = n->errw;
    GK(d);
  }
  for (int l = 0; l < n->L; ++l) {
    const bf16* v = n->act[l];
    // F1: T[(b,c)][j][s] = sum_f v[(b,c,s)][f] Fy[j][f]
    {
      GemmDesc d = gd(B * W * S, kJ, F);
      d.a = v;
      d.a_m0 = F;
      d.a_k = 1;
      d.b = n->Fy;
      d.b_n = F;
      d.b_k = 1;
      d.c = n->tp;
      d.c_msplit = S;
      d.c_m0 = 1;
      d.c_m1 = (long)kJ * S;
      d.c_n = S;
      d.c_bf16 = 1;
      d.err = n->errw;
      GK(d);
    }
    // F2: Z[(b,c,j)][r] = sum_s T[(b,c,j)][s] Fx[r][s]  (rows r, so that the store is coalesced)
    {
      GemmDesc d = gd(kR, B * W * kJ, S);
      d.a = n->Fx;
      d.a_m0 = S;
      d.a_k = 1;
      d.b = n->tp;
      d.b_n = S;
      d.b_k = 1;
      d.c = n->zt[l];
      d.c_m0 = 1;
      d.c_n = kR;
      d.err = n->errw;
      GK(d);
    }
    // spectral mixing
    {
      if (n->mix_grouped) {
        const size_t sm = sizeof(float) * kMixQ * (2 * W * W + 2 * B * W);
        k_mix_fwd<<<n->nmodes / kMixQ, 256, sm, n->st>>>(n->zt[l], n->wb + n->sRr[l].off, n->wb + n->sRi[l].off,
                                                         n->pt, B, W, n->m2);
      } else {
        const size_t sm = sizeof(float) * (2 * W * W + 2 * B * W);
        k_mix_fwd_mode<<<n->nmodes, 256, sm, n->st>>>(n->zt[l], n->wb + n->sRr[l].off, n->wb + n->sRi[l].off,
                                                      n->pt, B, W, n->m2);
      }
      FK(cudaGetLastError());
    }
    // F4: Y[(b,o)][s][j'] = sum_r P[(b,o),j'][r] Fx[r][s]   (rows (b,o,j'))
    {
      GemmDesc d = gd(B * W * kJ, S, kR);
      d.a = n->pt;
      d.a_m0 = kR;
      d.a_k = 1;
      d.b = n->Gx;
      d.b_n = kR;
      d.b_k = 1;
      d.c = n->yb;
      d.c_msplit = kJ;
      d.c_m0 = 1;
      d.c_m1 = (long)S * kJ;
      d.c_n = kJ;
      d.c_bf16 = 1;
      d.err = n->errw;
      GK(d);
    }
    // F5 and F6 in one GEMM where a 128-row tile of pixels lies in one row s (F a
    // multiple of 128): z[b][o][p] = sum_i W[o][i] v[b][i][p] + sum_j' Hy[f][j'] Y[(b,o),s][j']
    // + b[o] accumulates both products in the tile's TMEM accumulator, so the
    // spectral term never goes to memory
    const bool fused56 = F % kBM == 0;
    if (fused56) {
      GemmDesc d = gd((int)P, W, W, B);
      a_chanfirst(d, v, W, P);
      d.b = n->wb + n->sW[l].off;
      d.b_n = W;
      d.b_k = 1;
      d.K2 = kJ;
      d.a2 = n->Hy;  // A2(p, j') = Hy[p % F][j']
      d.a2_msplit = F;
      d.a2_m0 = kJ;
      d.a2_k = 1;
      d.b2 = n->yb;  // B2(o, j') = Y[(b,o)][s][j'], s = p0 / F for the tile at p0
      d.b2_n = (long)S * kJ;
      d.b2_k = 1;
      d.b2_b = (long)W * S * kJ;
      d.b2_m = kJ;
      d.b2_mdiv = F;
      c_chanfirst(d, n->act[l + 1], W, P, 1);
      d.bias_n = n->w + n->sWb[l].off;
      if (l < n->L - 1) {
        d.act = ACT_GELU;
        d.pre = train ? n->pre[l] : nullptr;
      }
      d.err = n->errw;
      GK(d);
      continue;
    }
    // F5: spec[(b,o,s)][f] = sum_j' Y[(b,o,s)][j'] Hy[f][j']  (rows f)
    {
      GemmDesc d = gd(F, B * W * S, kJ);
      d.a = n->Hy;
      d.a_m0 = kJ;
      d.a_k = 1;
      d.b = n->yb;
      d.b_n = kJ;
      d.b_k = 1;
      d.c = n->spec;
      d.c_m0 = 1;
      d.c_n = F;
      d.err = n->errw;
      GK(d);
    }
    // F6: z[b][o][p] = sum_i W[o][i] v[b][i][p] + spec + b[o];  v' = GELU(z)
    {
      GemmDesc d = gd((int)P, W, W, B);
      a_chanfirst(d, v, W, P);
      d.b = n->wb + n->sW[l].off;
      d.b_n = W;
      d.b_k = 1;
      c_chanfirst(d, n->act[l + 1], W, P, 1);
      d.add = n->spec;
      d.bias_n = n->w + n->sWb[l].off;
      if (l < n->L - 1) {
        d.act = ACT_GELU;
        d.pre = train ? n->pre[l] : nullptr;
      }
      d.err = n->errw;
      GK(d);
    }
  }
  // projection: h = GELU(Q1 v_L + q1b), y = Q2 h + q2b; for inference in one
  // kernel that keeps h on chip (fno_proj.cuh)
  if (!train && H == kProjH && W <= kBK && W % 8 == 0 && n->cpad <= kProjN2 && P % 8 == 0) {
    ProjArgs pa{};
    pa.v = n->act[n->L];
    pa.q1 = n->wb + n->sQ1.off;
    pa.q1b = n->w + n->sQ1b.off;
    pa.q2 = n->wb + n->sQ2.off;
    pa.q2b = n->w + n->sQ2b.off;
    pa.y = y;
    pa.P = P;
    pa.B = B;
    pa.W = W;
    pa.cout = n->cout;
    pa.cpad = n->cpad;
    pa.err = n->errw;
    pa.wait_tries = n->wait_tries;
    static int per_sm = 0;
    if (!per_sm) {
      // resident CTAs per SM from the kernel's own limits: shared memory (with the
      // largest carveout), TMEM (kProjH of 512 columns each) and registers
      FK(cudaFuncSetAttribute(k_proj_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, kProjSmem));
      FK(cudaFuncSetAttribute(k_proj_infer, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
      cudaFuncAttributes fa{};
      FK(cudaFuncGetAttributes(&fa, k_proj_infer));
      int dev = 0, smem_sm = 0, regs_sm = 0;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
      cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
      const int by_smem = smem_sm / (kProjSmem + (int)fa.sharedSizeBytes + 1024);
      const int by_tmem = 512 / kProjH;
      const int by_regs = fa.numRegs > 0 ? regs_sm / (fa.numRegs * kThreads) : by_tmem;
      per_sm = std::max(1, std::min(std::min(by_smem, by_tmem), by_regs));
    }
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const long ntiles = (P + kBM - 1) / kBM * B;
    const unsigned grid = (unsigned)std::min<long>(ntiles, (long)nsm * per_sm);
    k_proj_infer<<<grid, kThreads, kProjSmem, n->st>>>(pa);
    FK(cudaGetLastError());
    return 0;
  }
  {
    GemmDesc d = gd((int)P, H, W, B);
    a_chanfirst(d, n->act[n->L], W, P);
    d.b = n->wb + n->sQ1.off;
    d.b_n = W;
    d.b_k = 1;
    c_chanfirst(d, n->h, H, P, 1);
    d.bias_n = n->w + n->sQ1b.off;
    d.act = ACT_GELU;
    d.pre = train ? n->hpre : nullptr;
    d.err = n->errw;
    GK(d);
  }
  {
    GemmDesc d = gd((int)P, n->cout, H, B);
    a_chanfirst(d, n->h, H, P);
    d.b = n->wb + n->sQ2.off;
    d.b_n = H;
    d.b_k = 1;
    c_chanfirst(d, y, n->cout, P, 0);
    d.bias_n = n->w + n->sQ2b.off;
    d.err = n->errw;
    GK(d);
  }
  return 0;
}

// weight gradient dWt[r][c] += sum_{b,p} dout[b][r][p] * in[b][c][p]  (split over p)
int wgrad(sac_fno* n, const bf16* dout, int R, const bf16* in, int C, float* gout, int B) {
  const long P = n->P;
  GemmDesc d = gd(R, C, (int)P, B);
  d.a = dout;
  d.a_m0 = P;
  d.a_k = 1;
  d.a_b = (long)R * P;
  d.b = in;
  d.b_n = P;
  d.b_k = 1;
  d.b_b = (long)C * P;
  d.c = gout;
  d.c_m0 = C;
  d.c_n = 1;
  d.c_b = 0;
  d.c_mode = C_ATOMIC;
  d.ksplit = (int)std::min<long>(64, std::max<long>(1, P / 1024));
  if (d.ksplit * B > 65535) d.ksplit = 65535 / B;
  d.err = n->errw;
  GK(d);
  return 0;
}

int bias_grad(sac_fno* n, const bf16* d, int C, float* out, int B) {
  dim3 grid(64, C);
  k_chan_sum<<<grid, 256, 0, n->st>>>(d, out, B, C, n->P);
  FK(cudaGetLastError());
  return 0;
}

// dy: [B][cpad][P] bf16 (gradient of the loss w.r.t. y; padding channels zero)
int backward(sac_fno* n, const bf16* dy) {
  const int B = n->Blast, S = n->S, F = n->F, W = n->W, H = n->H, cpad = n->cpad;
  const long P = n->P;
  float* gw = n->g;
  // y = Q2 h + q2b
  int rc;
  // dy holds cpad channels (the ones past cout are zero, as are those rows of Q2)
  if ((rc = wgrad(n, dy, cpad, n->h, H, gw + n->sQ2.off, B))) return rc;
  if ((rc = bias_grad(n, dy, cpad, gw + n->sQ2b.off, B))) return rc;
  {  // dhpre[b][q][p] = GELU'(hpre) * sum_k Q2[k][q] dy[b][k][p]
    GemmDesc d = gd((int)P, H, cpad, B);
    a_chanfirst(d, dy, cpad, P);
    d.b = n->wb + n->sQ2.off;  // Q2[k][q], k padded to cpad rows
    d.b_mn_major = 1;
    d.b_n = 1;
    d.b_k = H;
    c_chanfirst(d, n->dhpre, H, P, 1);
    d.act = ACT_GELU_GRAD;
    d.pre = n->hpre;
    d.err = n->errw;
    GK(d);
  }
  if ((rc = wgrad(n, n->dhpre, H, n->act[n->L], W, gw + n->sQ1.off, B))) return rc;
  if ((rc = bias_grad(n, n->dhpre, H, gw + n->sQ1b.off, B))) return rc;
  {  // dz_{L-1}[b][o][p] = sum_q Q1[q][o] dhpre[b][q][p]   (no activation after the last layer)
    GemmDesc d = gd((int)P, W, H, B);
    a_chanfirst(d, n->dhpre, H, P);
    d.b = n->wb + n->sQ1.off;
    d.b_mn_major = 1;
    d.b_n = 1;
    d.b_k = W;
    c_chanfirst(d, n->dz, W, P, 1);
    d.err = n->errw;
    GK(d);
  }
  for (int l = n->L - 1; l >= 0; --l) {
    const bf16* v = n->act[l];
    bf16* dzl = n->dz;  // gradient w.r.t. z_l
    if ((rc = wgrad(n, dzl, W, v, W, gw + n->sW[l].off, B))) return rc;
    if ((rc = bias_grad(n, dzl, W, gw + n->sWb[l].off, B))) return rc;
    {  // pointwise path: dvacc[b][i][p] = sum_o W[o][i] dz[b][o][p]
      GemmDesc d = gd((int)P, W, W, B);
      a_chanfirst(d, dzl, W, P);
      d.b = n->wb + n->sW[l].off;
      d.b_mn_major = 1;
      d.b_n = 1;
      d.b_k = W;
      c_chanfirst(d, n->dvacc, W, P, 0);
      d.err = n->errw;
      GK(d);
    }
    {  // B5: dY[(b,o)][j'][s] = sum_f dz[(b,o,s)][f] Hy[f][j']
      GemmDesc d = gd(B * W * S, kJ, F);
      d.a = dzl;
      d.a_m0 = F;
      d.a_k = 1;
      d.b = n->HyT;
      d.b_n = F;
      d.b_k = 1;
      d.c = n->dyt;
      d.c_msplit = S;
      d.c_m0 = 1;
      d.c_m1 = (long)kJ * S;
      d.c_n = S;
      d.c_bf16 = 1;
      d.err = n->errw;
      GK(d);
    }
    {  // B4: dP[(b,o),j'][r] = sum_s dY[(b,o),j'][s] Fx[r][s]  (rows r)
      GemmDesc d = gd(kR, B * W * kJ, S);
      d.a = n->Fx;
      d.a_m0 = S;
      d.a_k = 1;
      d.b = n->dyt;
      d.b_n = S;
      d.b_k = 1;
      d.c = n->dpt;
      d.c_m0 = 1;
      d.c_n = kR;
      d.err = n->errw;
      GK(d);
    }
    {  // B3: mixing backward -> dZ, dR
      const size_t smg = sizeof(float) * kMixQ * (2 * W * W + 4 * B * W);
      if (smg <= n->mix_bwd_max) {
        k_mix_bwd_g<<<n->nmodes / kMixQ, 256, smg, n->st>>>(n->dpt, n->zt[l], n->wb + n->sRr[l].off,
                                                           n->wb + n->sRi[l].off, n->dzt, gw + n->sRr[l].off,
                                                           gw + n->sRi[l].off, B, W, n->m2);
      } else {
        const size_t sm = sizeof(float) * (2 * W * W + 4 * B * W);
        k_mix_bwd<<<n->nmodes, 256, sm, n->st>>>(n->dpt, n->zt[l], n->wb + n->sRr[l].off, n->wb + n->sRi[l].off,
                                                 n->dzt, gw + n->sRr[l].off, gw + n->sRi[l].off, B, W, n->m2);
      }
      FK(cudaGetLastError());
    }
    {  // B2: dT[(b,c),j][s] = sum_r dZ[(b,c),j][r] Fx[r][s]  (rows s)
      GemmDesc d = gd(S, B * W * kJ, kR);
      d.a = n->Gx;
      d.a_m0 = kR;
      d.a_k = 1;
      d.b = n->dzt;
      d.b_n = kR;
      d.b_k = 1;
      d.c = n->dtp;
      d.c_m0 = 1;
      d.c_n = S;
      d.c_bf16 = 1;
      d.err = n->errw;
      GK(d);
    }
    {  // B1: dv[(b,c,s)][f] = dvacc + sum_j dT[(b,c)][j][s] Fy[j][f], then GELU' of the layer
       // below  (rows f; B rows n = (b,c,s) read MN-major from dT[(b,c)][j][s])
      GemmDesc d = gd(F, B * W * S, kJ);
      d.a = n->FyT;
      d.a_m0 = kJ;
      d.a_k = 1;
      d.b = n->dtp;
      d.b_mn_major = 1;
      d.b_n = 1;
      d.b_nsplit = S;
      d.b_n1 = (long)kJ * S;
      d.b_k = S;
      d.c = n->dz2;
      d.c_m0 = 1;
      d.c_n = F;
      d.c_bf16 = 1;
      d.add = n->dvacc;
      if (l > 0) {
        d.act = ACT_GELU_GRAD;
        d.pre = n->pre[l - 1];
      }
      d.err = n->errw;
      GK(d);
    }
    std::swap(n->dz, n->dz2);  // dz now holds the gradient w.r.t. z_{l-1} (or v_0)
  }
  // lift: v0 = Pw x + pb
  if ((rc = wgrad(n, n->dz, W, n->xin, n->cin, gw + n->sP.off, B))) return rc;
  if ((rc = bias_grad(n, n->dz, W, gw + n->sPb.off, B))) return rc;
  return 0;
}

void make_tables(int S, int F, int m1, int m2, std::vector<float>& Fy, std::vector<float>& Fx,
                 std::vector<float>& Hy) {
  const double tp = 2.0 * M_PI;
  Fy.assign((size_t)kJ * F, 0.f);
  for (int j = 0; j < m2; ++j)
    for (int f = 0; f < F; ++f) {
      const double a = tp * (double)((long)j * f % F) / F;
      Fy[(size_t)j * F + f] = (float)std::cos(a);
      Fy[(size_t)(m2 + j) * F + f] = (float)-std::sin(a);
    }
  Fx.assign((size_t)kR * S, 0.f);
  for (int q = 0; q < 2 * m1; ++q) {
    const int kx = q < m1 ? q : S - 2 * m1 + q;
    for (int s = 0; s < S; ++s) {
      const double a = tp * (double)((long)kx * s % S) / S;
      Fx[(size_t)q * S + s] = (float)std::cos(a);
      Fx[(size_t)(2 * m1 + q) * S + s] = (float)-std::sin(a);
    }
  }
  Hy.assign((size_t)F * kJ, 0.f);
  const double norm = 1.0 / ((double)S * F);
  for (int f = 0; f < F; ++f)
    for (int j = 0; j < m2; ++j) {
      const double wgt = (j == 0 ? 1.0 : 2.0) * norm;
      const double a = tp * (double)((long)j * f % F) / F;
      Hy[(size_t)f * kJ + j] = (float)(wgt * std::cos(a));
      Hy[(size_t)f * kJ + m2 + j] = (float)(-wgt * std::sin(a));
    }
}

template <typename T>
int upload(sac_fno* n, T** dst, const std::vector<float>& src, bool bf) {
  if (bf) {
    std::vector<bf16> h(src.size());
    for (size_t i = 0; i < src.size(); ++i) h[i] = __float2bfloat16(src[i]);
    FK(cudaMalloc(dst, sizeof(bf16) * h.size()));
    FK(cudaMemcpy(*dst, h.data(), sizeof(bf16) * h.size(), cudaMemcpyHostToDevice));
  } else {
    FK(cudaMalloc(dst, sizeof(float) * src.size()));
    FK(cudaMemcpy(*dst, src.data(), sizeof(float) * src.size(), cudaMemcpyHostToDevice));
  }
  return 0;
}

std::vector<float> transpose(const std::vector<float>& a, int rows, int cols) {
  std::vector<float> t((size_t)rows * cols);
  for (int r = 0; r < rows; ++r)
    for (int c = 0; c < cols; ++c) t[(size_t)c * rows + r] = a[(size_t)r * cols + c];
  return t;
}

}  // namespace

extern "C" {

void sac_fno_default_config(sac_fno_config* c) {
  std::memset(c, 0, sizeof(*c));
  c->S = 256;
  c->F = 256;
  c->width = 32;
  c->layers = 4;
  c->modes1 = 24;
  c->modes2 = 24;
  c->hidden = 128;
  c->cin = 16;
  c->cout = 6;
  c->max_batch = 16;
  c->device = 0;
}

int sac_fno_create(const sac_fno_config* cfg, sac_fno** out) {
  sac_fno* n = nullptr;
  if (!cfg || !out) return fail(n, "sac_fno_create: null argument");
  *out = nullptr;
  if (cfg->modes1 != 24 || cfg->modes2 != 24) return fail(n, "sac_fno_create: 24 x 24 modes are built in");
  if (cfg->width % 16 || cfg->width > 64 || cfg->cin % 16 || cfg->hidden % 16 || cfg->cout < 1 || cfg->cout > 16 ||
      cfg->S % 8 || cfg->F % 8 || cfg->S < 2 * cfg->modes1 + 2 || cfg->F < 2 * cfg->modes2 + 2 ||
      cfg->layers < 1 || cfg->max_batch < 1 || cfg->max_batch > 64)
    return fail(n, "sac_fno_create: unsupported configuration");
  n = new sac_fno();
  n->cfg = *cfg;
  n->S = cfg->S;
  n->F = cfg->F;
  n->W = cfg->width;
  n->L = cfg->layers;
  n->H = cfg->hidden;
  n->cin = cfg->cin;
  n->cout = cfg->cout;
  n->cpad = (cfg->cout + 7) / 8 * 8;
  n->m1 = cfg->modes1;
  n->m2 = cfg->modes2;
  n->nmodes = 2 * n->m1 * n->m2;
  n->P = (long)n->S * n->F;
  n->Bmax = cfg->max_batch;
  if (cudaSetDevice(cfg->device) != cudaSuccess || cudaStreamCreateWithFlags(&n->st, cudaStreamNonBlocking)) {
    delete n;
    return fail(nullptr, "sac_fno_create: no device");
  }
  {  // the grouped forward mode mixing holds R and U of 8 modes for the whole batch
    const size_t mix = sizeof(float) * kMixQ * (2 * (size_t)n->W * n->W + 2 * (size_t)n->Bmax * n->W);
    n->mix_grouped = mix <= 227 * 1024 && (2 * n->m1) % kMixQ == 0 &&
                     cudaFuncSetAttribute(k_mix_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mix) ==
                         cudaSuccess;
    cudaGetLastError();  // a refused attribute leaves the per-mode form
    // the grouped backward holds R, U and G of 8 modes for the training batch
    const size_t mb = std::min<size_t>(227 * 1024, sizeof(float) * kMixQ *
                                                       (2 * (size_t)n->W * n->W + 4 * (size_t)n->Bmax * n->W));
    if ((2 * n->m1) % kMixQ == 0 &&
        cudaFuncSetAttribute(k_mix_bwd_g, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mb) == cudaSuccess)
      n->mix_bwd_max = mb;
    cudaGetLastError();
    const size_t one = sizeof(float) * (2 * (size_t)n->W * n->W + 2 * (size_t)n->Bmax * n->W);
    if (!n->mix_grouped &&
        cudaFuncSetAttribute(k_mix_fwd_mode, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)one) != cudaSuccess) {
      cudaStreamDestroy(n->st);
      delete n;
      return fail(nullptr, "sac_fno_create: width and max_batch too large for the mode mixing's shared memory");
    }
  }
  // parameter segments (each a multiple of 8 elements, 16-byte aligned in bf16)
  long off = 0;
  auto seg = [&](long cnt) {
    sac_fno::Seg s{off, cnt};
    off += (cnt + 7) / 8 * 8;
    return s;
  };
  const int W = n->W;
  n->sP = seg((long)W * n->cin);
  n->sPb = seg(W);
  for (int l = 0; l < n->L; ++l) {
    n->sW.push_back(seg((long)W * W));
    n->sWb.push_back(seg(W));
    n->sRr.push_back(seg((long)n->nmodes * W * W));
    n->sRi.push_back(seg((long)n->nmodes * W * W));
  }
  n->sQ1 = seg((long)n->H * W);
  n->sQ1b = seg(n->H);
  n->sQ2 = seg((long)n->cpad * n->H);  // rows cout..cpad-1 stay zero
  n->sQ2b = seg(n->cpad);
  n->nparam = off;
  const long np = n->nparam;
  FK(cudaMalloc(&n->w, sizeof(float) * np));
  FK(cudaMalloc(&n->g, sizeof(float) * np));
  FK(cudaMalloc(&n->am, sizeof(float) * np));
  FK(cudaMalloc(&n->av, sizeof(float) * np));
  FK(cudaMalloc(&n->wb, sizeof(bf16) * np));
  FK(cudaMemset(n->w, 0, sizeof(float) * np));
  FK(cudaMemset(n->g, 0, sizeof(float) * np));
  FK(cudaMemset(n->am, 0, sizeof(float) * np));
  FK(cudaMemset(n->av, 0, sizeof(float) * np));
  FK(cudaMemset(n->wb, 0, sizeof(bf16) * np));
  // DFT tables
  std::vector<float> Fy, Fx, Hy;
  make_tables(n->S, n->F, n->m1, n->m2, Fy, Fx, Hy);
  int rc;
  if ((rc = upload(n, &n->Fy, Fy, true)) || (rc = upload(n, &n->FyT, transpose(Fy, kJ, n->F), true)) ||
      (rc = upload(n, &n->Fx, Fx, true)) || (rc = upload(n, &n->Gx, transpose(Fx, kR, n->S), true)) ||
      (rc = upload(n, &n->Hy, Hy, true)) || (rc = upload(n, &n->HyT, transpose(Hy, n->F, kJ), true))) {
    sac_fno_destroy(n);
    return rc;
  }
  // activations and scratch for max_batch samples
  const long B = n->Bmax, P = n->P, BWP = B * W * P;
  for (int l = 0; l <= n->L; ++l) {
    bf16* p;
    FK(cudaMalloc(&p, sizeof(bf16) * BWP));
    n->act.push_back(p);
  }
  for (int l = 0; l < n->L; ++l) {
    bf16* p;
    FK(cudaMalloc(&p, sizeof(bf16) * BWP));
    n->pre.push_back(p);
    float* z;
    FK(cudaMalloc(&z, sizeof(float) * B * W * kJ * kR));
    n->zt.push_back(z);
  }
  FK(cudaMalloc(&n->hpre, sizeof(bf16) * B * n->H * P));
  FK(cudaMalloc(&n->h, sizeof(bf16) * B * n->H * P));
  FK(cudaMalloc(&n->dhpre, sizeof(bf16) * B * n->H * P));
  FK(cudaMalloc(&n->tp, sizeof(bf16) * B * W * kJ * n->S));
  FK(cudaMalloc(&n->dtp, sizeof(bf16) * B * W * kJ * n->S));
  FK(cudaMalloc(&n->dyt, sizeof(bf16) * B * W * kJ * n->S));
  FK(cudaMalloc(&n->pt, sizeof(bf16) * B * W * kJ * kR));
  FK(cudaMalloc(&n->dzt, sizeof(bf16) * B * W * kJ * kR));
  FK(cudaMalloc(&n->dpt, sizeof(float) * B * W * kJ * kR));
  FK(cudaMalloc(&n->yb, sizeof(bf16) * B * W * n->S * kJ));
  FK(cudaMalloc(&n->spec, sizeof(float) * BWP));
  FK(cudaMalloc(&n->dvacc, sizeof(float) * BWP));
  FK(cudaMalloc(&n->dz, sizeof(bf16) * BWP));
  FK(cudaMalloc(&n->dz2, sizeof(bf16) * BWP));
  FK(cudaMalloc(&n->scal, sizeof(float) * 4));
  FK(cudaMalloc(&n->errw, sizeof(int)));
  FK(cudaMemset(n->errw, 0, sizeof(int)));
  *out = n;
  return 0;
}

void sac_fno_destroy(sac_fno* n) {
  if (!n) return;
  cudaSetDevice(n->cfg.device);
  if (n->st) cudaStreamSynchronize(n->st);
  for (void* p : {(void*)n->w, (void*)n->g, (void*)n->am, (void*)n->av, (void*)n->wb, (void*)n->Fy, (void*)n->FyT,
                  (void*)n->Fx, (void*)n->Gx, (void*)n->Hy, (void*)n->HyT, (void*)n->hpre, (void*)n->h,
                  (void*)n->dhpre, (void*)n->tp, (void*)n->dtp, (void*)n->dyt, (void*)n->pt, (void*)n->dzt,
                  (void*)n->dpt, (void*)n->yb, (void*)n->spec, (void*)n->dvacc, (void*)n->dz, (void*)n->dz2,
                  (void*)n->scal, (void*)n->errw})
    if (p) cudaFree(p);
  for (auto* p : n->act) cudaFree(p);
  for (auto* p : n->pre) cudaFree(p);
  for (auto* p : n->zt) cudaFree(p);
  if (n->st) cudaStreamDestroy(n->st);
  delete n;
}

const char* sac_fno_error(const sac_fno* n) { return n ? n->err.c_str() : "null network"; }
long sac_fno_num_params(const sac_fno* n) { return n ? n->nparam : 0; }
void* sac_fno_stream(const sac_fno* n) { return n ? (void*)n->st : nullptr; }

// FP32 parameters (host), in segment order; the BF16 copies follow
int sac_fno_set_params(sac_fno* n, const float* host) {
  if (!n || !host) return fail(n, "sac_fno_set_params: null argument");
  FK(cudaSetDevice(n->cfg.device));
  FK(cudaMemcpyAsync(n->w, host, sizeof(float) * n->nparam, cudaMemcpyHostToDevice, n->st));
  k_f2bf<<<grid_for(n->nparam), 256, 0, n->st>>>(n->wb, n->w, n->nparam);
  FK(cudaGetLastError());
  FK(cudaStreamSynchronize(n->st));
  return 0;
}

int sac_fno_get_params(sac_fno* n, float* host) {
  if (!n || !host) return fail(n, "sac_fno_get_params: null argument");
  FK(cudaSetDevice(n->cfg.device));
  FK(cudaMemcpyAsync(host, n->w, sizeof(float) * n->nparam, cudaMemcpyDeviceToHost, n->st));
  FK(cudaStreamSynchronize(n->st));
  return 0;
}

int sac_fno_get_grads(sac_fno* n, float* host) {
  if (!n || !host) return fail(n, "sac_fno_get_grads: null argument");
  FK(cudaSetDevice(n->cfg.device));
  FK(cudaMemcpyAsync(host, n->g, sizeof(float) * n->nparam, cudaMemcpyDeviceToHost, n->st));
  FK(cudaStreamSynchronize(n->st));
  return 0;
}

// offsets of the named parameter groups (host array of 2*(6 + 4*layers) longs:
// offset, count for P, Pb, then per layer W, Wb, Rr, Ri, then Q1, Q1b, Q2, Q2b)
int sac_fno_param_layout(const sac_fno* n, long* out) {
  if (!n || !out) return 1;
  int k = 0;
  auto put = [&](const sac_fno::Seg& s) {
    out[k++] = s.off;
    out[k++] = s.n;
  };
  put(n->sP);
  put(n->sPb);
  for (int l = 0; l < n->L; ++l) {
    put(n->sW[l]);
    put(n->sWb[l]);
    put(n->sRr[l]);
    put(n->sRi[l]);
  }
  put(n->sQ1);
  put(n->sQ1b);
  put(n->sQ2);
  put(n->sQ2b);
  return 0;
}

// PyTorch-style initialisation: 1x1 layers U(-1/sqrt(fan_in), 1/sqrt(fan_in)),
// spectral weights U(-1, 1) / (width * width)
int sac_fno_init(sac_fno* n, unsigned long long seed) {
  if (!n) return 1;
  std::vector<float> h((size_t)n->nparam, 0.f);
  std::mt19937_64 rng(seed);
  auto fill = [&](const sac_fno::Seg& s, double bound, long rows_valid = -1, long row_len = 0) {
    std::uniform_real_distribution<double> u(-bound, bound);
    for (long i = 0; i < s.n; ++i) {
      const bool valid = rows_valid < 0 || i / row_len < rows_valid;
      h[(size_t)(s.off + i)] = valid ? (float)u(rng) : 0.f;
    }
  };
  const double bl = 1.0 / std::sqrt((double)n->cin);
  fill(n->sP, bl);
  fill(n->sPb, bl);
  for (int l = 0; l < n->L; ++l) {
    const double bw = 1.0 / std::sqrt((double)n->W);
    fill(n->sW[l], bw);
    fill(n->sWb[l], bw);
    fill(n->sRr[l], 1.0 / ((double)n->W * n->W));
    fill(n->sRi[l], 1.0 / ((double)n->W * n->W));
  }
  fill(n->sQ1, 1.0 / std::sqrt((double)n->W));
  fill(n->sQ1b, 1.0 / std::sqrt((double)n->W));
  fill(n->sQ2, 1.0 / std::sqrt((double)n->H), n->cout, n->H);
  fill(n->sQ2b, 1.0 / std::sqrt((double)n->H), n->cout, 1);
  return sac_fno_set_params(n, h.data());
}

int sac_fno_zero_grad(sac_fno* n) {
  if (!n) return 1;
  FK(cudaMemsetAsync(n->g, 0, sizeof(float) * n->nparam, n->st));
  return 0;
}

// x: [B][cin][S][F] bf16 (kept by the caller until sac_fno_backward);
// y: [B][cout][S][F] float
int sac_fno_forward(sac_fno* n, const void* x, float* y, int B) {
  if (!n || !x || !y) return fail(n, "sac_fno_forward: null argument");
  if (B < 1 || B > n->Bmax) return fail(n, "sac_fno_forward: batch outside 1..max_batch");
  FK(cudaSetDevice(n->cfg.device));
  return forward(n, (const bf16*)x, y, B, true);
}

// the forward pass without what training needs (no pre-activation stores); a
// backward pass cannot follow it
int sac_fno_infer(sac_fno* n, const void* x, float* y, int B) {
  if (!n || !x || !y) return fail(n, "sac_fno_infer: null argument");
  if (B < 1 || B > n->Bmax) return fail(n, "sac_fno_infer: batch outside 1..max_batch");
  FK(cudaSetDevice(n->cfg.device));
  return forward(n, (const bf16*)x, y, B, false);
}

// dy: [B][cpad][S][F] bf16 with cpad = cout rounded up to 8 (padding channels zero)
int sac_fno_backward(sac_fno* n, const void* dy) {
  if (!n || !dy) return fail(n, "sac_fno_backward: null argument");
  if (!n->xin) return fail(n, "sac_fno_backward: no forward pass to differentiate");
  FK(cudaSetDevice(n->cfg.device));
  return backward(n, (const bf16*)dy);
}

// mean squared error over the cout channels; writes dy (bf16, cpad channels)
// and adds the loss to *loss (device float)
int sac_fno_mse(sac_fno* n, const float* y, const void* target, void* dy, float* loss, int B) {
  if (!n || !y || !target || !dy || !loss) return fail(n, "sac_fno_mse: null argument");
  const long tot = (long)B * n->cout * n->P;
  k_mse<<<grid_for((long)B * n->cpad * n->P), 256, 0, n->st>>>(y, (const bf16*)target, (bf16*)dy, loss, B,
                                                               n->cout, n->cpad, n->P, 1.0f / (float)tot);
  FK(cudaGetLastError());
  return 0;
}

// one Adam step (bias-corrected, decoupled weight decay); the gradient is
// clipped to global L2 norm clip (<= 0: no clipping)
int sac_fno_adam(sac_fno* n, float lr, float b1, float b2, float eps, float wd, int step, float clip) {
  if (!n || step < 1) return fail(n, "sac_fno_adam: bad argument");
  float gscale = 1.f;
  if (clip > 0.f) {
    FK(cudaMemsetAsync(n->scal, 0, sizeof(float), n->st));
    k_sumsq<<<grid_for(n->nparam), 256, 0, n->st>>>(n->g, n->nparam, n->scal);
    float ss = 0.f;
    FK(cudaMemcpyAsync(&ss, n->scal, sizeof(float), cudaMemcpyDeviceToHost, n->st));
    FK(cudaStreamSynchronize(n->st));
    const float norm = std::sqrt(ss);
    if (!(norm == norm)) return fail(n, "sac_fno_adam: non-finite gradient");
    if (norm > clip) gscale = clip / norm;
  }
  const float c1 = 1.f - std::pow(b1, (float)step), c2 = 1.f - std::pow(b2, (float)step);
  k_adam<<<grid_for(n->nparam), 256, 0, n->st>>>(n->w, n->wb, n->g, n->am, n->av, n->nparam, lr, b1, b2, eps, wd,
                                                 c1, c2, gscale);
  FK(cudaGetLastError());
  // the padding rows of Q2 stay zero (zero gradient, zero moments, decay keeps 0)
  return 0;
}

// assemble the network input from a state (float or bf16) and per-sample features
int sac_fno_features(sac_fno* n, const void* state, int state_bf16, const float* scale, const float* feat,
                     int nfeat, void* x, int B, int nst) {
  if (!n || !state || !x) return fail(n, "sac_fno_features: null argument");
  if (nst + nfeat + 2 > n->cin) return fail(n, "sac_fno_features: too many channels for cin");
  const long tot = (long)B * n->cin * n->P;
  if (state_bf16)
    k_features<bf16><<<grid_for(tot), 256, 0, n->st>>>((const bf16*)state, scale, feat, (bf16*)x, B, nst, nfeat,
                                                       n->cin, n->S, n->F);
  else
    k_features<float><<<grid_for(tot), 256, 0, n->st>>>((const float*)state, scale, feat, (bf16*)x, B, nst, nfeat,
                                                        n->cin, n->S, n->F);
  FK(cudaGetLastError());
  return 0;
}

int sac_fno_apply(sac_fno* n, float* state, const float* y, const float* scale, int B, int nst) {
  if (!n || !state || !y || !scale) return fail(n, "sac_fno_apply: null argument");
  k_apply<<<grid_for((long)B * nst * n->P), 256, 0, n->st>>>(state, y, scale, B, nst, n->P);
  FK(cudaGetLastError());
  return 0;
}

// error word of the GEMMs (bit 0: a bounded wait timed out); synchronises; reset clears it
int sac_fno_check(sac_fno* n, int reset) {
  if (!n) return 1;
  int e = 0;
  FK(cudaMemcpyAsync(&e, n->errw, sizeof(int), cudaMemcpyDeviceToHost, n->st));
  FK(cudaStreamSynchronize(n->st));
  if (reset) FK(cudaMemsetAsync(n->errw, 0, sizeof(int), n->st));
  if (e) return fail(n, "a tensor-core wait timed out (error word " + std::to_string(e) + ")") + 6;
  return 0;
}

int sac_fno_set_wait_tries(sac_fno* n, int tries) {
  if (!n) return 1;
  n->wait_tries = tries < 0 ? -1 : tries;
  return 0;
}

}  // extern "C"
