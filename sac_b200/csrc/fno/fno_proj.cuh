// fno_proj.cuh -- the FNO's projection for inference in one kernel:
//
//   y[b][k][p] = q2b[k] + sum_q Q2[k][q] GELU(q1b[q] + sum_c Q1[q][c] v[b][c][p])
//
// Persistent CTAs of 128 threads walk tiles of 128 pixels of one sample.  Per
// tile: the tile of v (MN-major, pixels contiguous) goes to shared memory and one
// thread issues the first product into a 128-column TMEM accumulator (hidden
// channels); each thread reads its pixel's row back with tcgen05.ld, adds the
// bias, applies GELU and writes the BF16 hidden row into shared memory in the
// K-major operand layout; the second product (N = 16, the output channels padded
// with zero rows) then runs on the tensor cores into the first 16 columns of the
// same accumulator, and the epilogue stores the cout outputs.  So the 128 hidden
// channels of a pixel never leave the SM.  Q1, Q2 and the biases are loaded once
// per CTA.  Every mbarrier wait is bounded; on time-out the kernel sets bit 0 of
// the error word, drains the MMAs in flight, frees its TMEM and returns.
#pragma once
#include "fno_gemm.cuh"

namespace fno {

struct ProjArgs {
  const bf16* v;   // [B][W][P]
  const bf16* q1;  // [H][W], H = 128
  const float* q1b;
  const bf16* q2;  // [cpad][H]
  const float* q2b;
  float* y;        // [B][cout][P]
  long P;
  int B, W, cout, cpad;
  int* err;
  int wait_tries;
};

constexpr int kProjH = 128, kProjN2 = 16;
// shared memory: A1 (128 x 64), B1 (128 x 64), hidden A2 (2 x 128 x 64), B2 (2 x 16 x 64)
constexpr int kProjA1 = 0, kProjB1 = kBM * kBK * 2, kProjA2 = kProjB1 + kProjH * kBK * 2,
              kProjB2 = kProjA2 + 2 * kBM * kBK * 2, kProjSmem = kProjB2 + 2 * kProjN2 * kBK * 2;

__global__ void __launch_bounds__(kThreads, 3) k_proj_infer(const ProjArgs a) {
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ uint64_t bar;
  __shared__ uint32_t tmem_sh;
  __shared__ float b1s[kProjH];
  __shared__ float b2s[kProjN2];
  const int tid = threadIdx.x, warp = tid >> 5;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_sh)),
                 "r"(kProjH));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  // the weights, once: Q1 as a 128 x 64 K-major B tile (k >= W zero), Q2 as two
  // 16 x 64 K-major tiles (rows >= cpad zero)
  {
    Tile16<kProjH> t1;
    load_tile<kProjH>(t1, a.q1, a.W, 0, 1 << 30, 1, 0, 0, kProjH, 0, a.W);
    store_tile<kProjH>(t1, smem + kProjB1, 0);
#pragma unroll
    for (int kt = 0; kt < 2; ++kt) {
      Tile16<kProjN2> t2;
      load_tile<kProjN2>(t2, a.q2, kProjH, 0, 1 << 30, 1, 0, 0, a.cpad, kt * kBK, kProjH);
      store_tile<kProjN2>(t2, smem + kProjB2 + kt * kProjN2 * kBK * 2, 0);
    }
    b1s[tid] = a.q1b[tid];  // kThreads == kProjH
    if (tid < kProjN2) b2s[tid] = tid < a.cout ? a.q2b[tid] : 0.0f;
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = tmem_sh;
  const uint32_t id1 = umma_idesc(kProjH, 1, 0), id2 = umma_idesc(kProjN2, 0, 0);
  const int tries = a.wait_tries == 0 ? kWaitTries : (a.wait_tries < 0 ? 0 : a.wait_tries);
  const long tps = (a.P + kBM - 1) / kBM, ntiles = tps * a.B;
  const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
  uint32_t phase = 0;  // commits waited on so far (the barrier's parity)
  bool ok = true, pending = false;
  for (long t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int b = (int)(t / tps);
    const long p0 = (t % tps) * kBM;
    const bf16* vb = a.v + (long)b * a.W * a.P;
    {  // the tile of v: 128 pixels x W channels, MN-major
      Tile16<kBM> ta;
      load_tile<kBM>(ta, vb + p0, 1, 0, 1 << 30, a.P, 1, 0, (int)min((long)kBM, a.P - p0), 0, a.W);
      store_tile<kBM>(ta, smem + kProjA1, 1);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (tid == 0) {  // hidden = v Q1^T, K = W <= 64 (k past W is zero)
      asm volatile("tcgen05.fence::after_thread_sync;");
      const uint32_t a0 = smem_u32(smem + kProjA1), b0 = smem_u32(smem + kProjB1);
      for (int kk = 0; kk < (a.W + 15) / 16; ++kk) {
        const uint64_t da = tile_desc<kBM>(a0, 1, kk), db = tile_desc<kProjH>(b0, 0, kk);
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(tmem),
            "l"(da), "l"(db), "r"(id1), "r"(kk > 0 ? 1u : 0u), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(&bar))
                   : "memory");
    }
    pending = true;
    if (!mbar_wait(&bar, phase & 1, tries)) ok = false;
    if (__syncthreads_or(!ok)) break;
    pending = false;
    ++phase;
    asm volatile("tcgen05.fence::after_thread_sync;");
    // GELU(hidden + q1b) -> BF16 rows of the K-major hidden operand: core
    // (row group r/8, k chunk q/8) at (r/8*8 + q/8 % 8)*128 B + (r%8)*16 of k tile q/64
    const int r = tid;
#pragma unroll 1
    for (int cc = 0; cc < kProjH; cc += 16) {
      uint32_t v[16];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
          : "r"(tmem + lane_base + (uint32_t)cc));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      uint32_t h[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const float x0 = gelu_f(__uint_as_float(v[2 * j]) + b1s[cc + 2 * j]);
        const float x1 = gelu_f(__uint_as_float(v[2 * j + 1]) + b1s[cc + 2 * j + 1]);
        const __nv_bfloat162 pr = __floats2bfloat162_rn(x0, x1);
        h[j] = *reinterpret_cast<const uint32_t*>(&pr);
      }
#pragma unroll
      for (int half = 0; half < 2; ++half) {
        const int q = cc + 8 * half, kt = q / kBK, kc = (q % kBK) / 8;
        uint8_t* dst = smem + kProjA2 + kt * kBM * kBK * 2 + ((r / 8) * 8 + kc) * 128 + (r % 8) * 16;
        *reinterpret_cast<uint4*>(dst) = make_uint4(h[4 * half], h[4 * half + 1], h[4 * half + 2], h[4 * half + 3]);
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (tid == 0) {  // y = hidden Q2^T into columns 0..15 (the hidden accumulator was read)
      asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll
      for (int kt = 0; kt < 2; ++kt) {
        const uint32_t a0 = smem_u32(smem + kProjA2 + kt * kBM * kBK * 2);
        const uint32_t b0 = smem_u32(smem + kProjB2 + kt * kProjN2 * kBK * 2);
#pragma unroll
        for (int kk = 0; kk < kBK / 16; ++kk) {
          const uint64_t da = tile_desc<kBM>(a0, 0, kk), db = tile_desc<kProjN2>(b0, 0, kk);
          asm volatile(
              "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
              " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(tmem),
              "l"(da), "l"(db), "r"(id2), "r"((kt | kk) ? 1u : 0u), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
        }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(&bar))
                   : "memory");
    }
    pending = true;
    if (!mbar_wait(&bar, phase & 1, tries)) ok = false;
    if (__syncthreads_or(!ok)) break;
    pending = false;
    ++phase;
    asm volatile("tcgen05.fence::after_thread_sync;");
    {
      uint32_t v[16];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
          : "r"(tmem + lane_base));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      const long p = p0 + r;
      if (p < a.P) {
        float* yb = a.y + (long)b * a.cout * a.P + p;
#pragma unroll
        for (int k = 0; k < kProjN2; ++k)
          if (k < a.cout) yb[(long)k * a.P] = __uint_as_float(v[k]) + b2s[k];
      }
    }
    // the next tile's first product overwrites the accumulator and A1: every
    // thread's reads are done once all pass the barrier after its A1 store
    asm volatile("tcgen05.fence::before_thread_sync;");
  }
  if (!ok) {
    if (tid == 0 && a.err) atomicOr(a.err, 1);
    if (pending) mbar_wait(&bar, phase & 1);  // drain the MMAs in flight (default bound)
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kProjH));
}

}  // namespace fno
