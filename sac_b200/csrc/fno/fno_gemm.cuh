// fno_gemm.cuh -- BF16 GEMM on the 5th-generation tensor cores (tcgen05, sm_100a).
//
//   C(m,n) = epilogue( alpha * sum_k A(m,k) * B(n,k) )
//
// One CTA of 128 threads computes a 128 x BN tile.  Operand tiles of 64 k are
// staged in shared memory in the canonical no-swizzle UMMA layouts (core
// matrices of 8 rows x 16 bytes), K-major or MN-major as the operand is laid out
// in global memory, double buffered; one elected thread issues
// tcgen05.mma.cta_group::1.kind::f16 (BF16 x BF16 -> FP32) into a TMEM
// accumulator and commits to an mbarrier, while all threads load the next tile.
// The epilogue reads the accumulator back with tcgen05.ld (warp w owns TMEM lanes
// 32w..32w+31, i.e. tile rows) and applies bias / residual add / GELU / GELU'
// before storing FP32 or BF16, plain, accumulated or atomically.
//
// Every wait on an mbarrier is bounded: on time-out the kernel raises a flag in
// the error word, skips the rest of its work, frees its TMEM and returns.
#pragma once
#include <cuda_bf16.h>
#include <cstdint>

namespace fno {

using bf16 = __nv_bfloat16;

enum EpiAct : int { ACT_NONE = 0, ACT_GELU = 1, ACT_GELU_GRAD = 2 };
enum CMode : int { C_STORE = 0, C_ACCUM = 1, C_ATOMIC = 2 };

// Addressing of a matrix whose row index m is split as m = (m / msplit, m % msplit):
//   addr(m, x) = base + bz*s_b + (m / msplit)*s_m1 + (m % msplit)*s_m0 + x*s_x
struct GemmDesc {
  int M, N, K;      // problem per batch item
  int batch;        // batch items (grid.z = batch * ksplit)
  int ksplit;       // K split into ksplit chunks (results combined by C_ATOMIC)
  // A(m, k)
  const bf16* a;
  long a_m0, a_m1, a_k, a_b;
  int a_msplit;
  int a_mn_major;   // 1: a_m0 == 1 (8 consecutive m contiguous); 0: a_k == 1
  // B(n, k)
  const bf16* b;
  long b_n, b_k, b_b;
  int b_mn_major;   // 1: b_n == 1; 0: b_k == 1
  // C(m, n) and the epilogue tensors that share its addressing
  void* c;
  long c_m0, c_m1, c_n, c_b;
  int c_msplit;
  int c_bf16;       // 0: float, 1: bf16
  int c_mode;       // CMode
  float alpha;
  const float* bias_n;  // + bias_n[n]
  const float* add;     // + add(m, n), float, C addressing
  int act;              // EpiAct
  bf16* pre;            // ACT_GELU: stores the pre-activation; ACT_GELU_GRAD: reads it
  int* err;             // error word (bit 0: an mbarrier wait timed out)
  // B rows split like A's: n = (n / b_nsplit, n % b_nsplit) -> (n / b_nsplit)*b_n1 + (n % b_nsplit)*b_n
  long b_n1;
  int b_nsplit;
  // bound of the pipeline's mbarrier waits in tries of at most ~5 ms each:
  // 0 = the default kWaitTries, > 0 = that many, < 0 = none (the first wait gives
  // up at once; a test of the time-out path).  The wait that drains the MMAs in
  // flight before the accumulator is released always keeps the default bound.
  int wait_tries;
  // a second product accumulated into the same tile when K2 > 0:
  //   C = epilogue(alpha * (sum_k A(m,k) B(n,k) + sum_k2 A2(m,k2) B2(n,k2)))
  // A2 is addressed like A; B2 like B without a row split, its base moved by
  // (m0 / b2_mdiv) * b2_m for the tile whose first row is m0 (b2_mdiv a multiple of
  // the tile height, so that all rows of a tile read the same B2 block)
  int K2;
  int a2_msplit, a2_mn_major;
  const bf16* a2;
  long a2_m0, a2_m1, a2_k, a2_b;
  const bf16* b2;
  long b2_n, b2_k, b2_b, b2_m;
  int b2_mn_major, b2_mdiv;
};

constexpr int kBM = 128, kBK = 64, kThreads = 128;

// Epilogue forms compiled as separate kernels, so that the per-element work
// carries no test of runtime flags; EPI_GENERIC reads every flag at run time.
struct EpiForm {
  bool generic, bias, add, bf16, atomic;
  int act;
};
enum EpiKind : int {
  EPI_GENERIC = 0,
  EPI_F32,             // store float
  EPI_BF16,            // store bf16
  EPI_BF16_BIAS,       // + bias, bf16
  EPI_F32_BIAS,        // + bias, float
  EPI_BF16_BIAS_GELU,  // + bias, GELU (pre stored), bf16
  EPI_BF16_BIAS_ADD,   // + bias + add, bf16
  EPI_BF16_BIAS_ADD_GELU,
  EPI_BF16_ADD,        // + add, bf16
  EPI_BF16_ADD_GRAD,   // (acc + add) * GELU'(pre), bf16
  EPI_BF16_GRAD,       // acc * GELU'(pre), bf16
  EPI_F32_ATOMIC,      // atomic add, float
  EPI_KINDS
};
__host__ __device__ constexpr EpiForm epi_form(int k) {
  return k == EPI_F32                  ? EpiForm{false, false, false, false, false, ACT_NONE}
         : k == EPI_BF16               ? EpiForm{false, false, false, true, false, ACT_NONE}
         : k == EPI_BF16_BIAS          ? EpiForm{false, true, false, true, false, ACT_NONE}
         : k == EPI_F32_BIAS           ? EpiForm{false, true, false, false, false, ACT_NONE}
         : k == EPI_BF16_BIAS_GELU     ? EpiForm{false, true, false, true, false, ACT_GELU}
         : k == EPI_BF16_BIAS_ADD      ? EpiForm{false, true, true, true, false, ACT_NONE}
         : k == EPI_BF16_BIAS_ADD_GELU ? EpiForm{false, true, true, true, false, ACT_GELU}
         : k == EPI_BF16_ADD           ? EpiForm{false, false, true, true, false, ACT_NONE}
         : k == EPI_BF16_ADD_GRAD      ? EpiForm{false, false, true, true, false, ACT_GELU_GRAD}
         : k == EPI_BF16_GRAD          ? EpiForm{false, false, false, true, false, ACT_GELU_GRAD}
         : k == EPI_F32_ATOMIC         ? EpiForm{false, false, false, false, true, ACT_NONE}
                                       : EpiForm{true, false, false, false, false, ACT_NONE};
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// UMMA shared-memory descriptor, no swizzle: start, leading and stride byte
// offsets in 16-byte units, version 1 (bits 46-48) for sm_100.
__device__ __forceinline__ uint64_t umma_sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, M=128
__host__ __device__ constexpr uint32_t umma_idesc(int n, int a_mn, int b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
         ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kBM >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

constexpr int kWaitTries = 400;  // ~2 s

// bounded wait for the phase with the given parity; false on time-out
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int tries = kWaitTries) {
  const uint32_t a = smem_u32(bar);
  for (int it = 0; it < tries; ++it) {  // each try suspends for at most ~5 ms
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred P1;\n mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2, %3;\n selp.b32 %0, 1, 0, P1;\n}"
        : "=r"(ok)
        : "r"(a), "r"(parity), "r"(5000000u)
        : "memory");
    if (ok) return true;
  }
  return false;
}

// GELU in its tanh form (Hendrycks and Gimpel): 0.5 x (1 + tanh(u)),
// u = c0 (x + c1 x^3), c0 = sqrt(2/pi), c1 = 0.044715, with the SFU's tanh
// (tanh.approx.f32, relative error near 2^-11, below the BF16 rounding of the
// activations it feeds); its derivative 0.5 (1 + t) + 0.5 x (1 - t^2) c0 (1 + 3 c1 x^2)
__device__ __forceinline__ float tanh_sfu(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float gelu_f(float x) {
  const float u = 0.7978845608028654f * fmaf(0.044715f * x, x * x, x);
  return 0.5f * x * (1.0f + tanh_sfu(u));
}
__device__ __forceinline__ float gelu_grad_f(float x) {
  const float x2 = x * x;
  const float t = tanh_sfu(0.7978845608028654f * fmaf(0.044715f * x, x2, x));
  return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * (0.7978845608028654f * fmaf(0.134145f, x2, 1.0f));
}

// the 16-byte chunks one thread moves for a ROWS x 64 operand tile
template <int ROWS>
struct Tile16 {
  static constexpr int CPT = ROWS * 8 / kThreads;
  uint4 v[CPT];
};

// Load the 128 x 64 (A) or BN x 64 (B) operand tile chunks this thread owns into
// registers.  rows: tile rows; mn_major selects the mapping; zero outside.
template <int ROWS>
__device__ __forceinline__ void load_tile(Tile16<ROWS>& t, const bf16* base, long s_m0, long s_m1, int msplit, long s_k,
                                          int mn_major, int row0, int nrows, int k0, int kend) {
  static_assert(ROWS % 16 == 0, "tile rows");
#pragma unroll
  for (int i = 0; i < Tile16<ROWS>::CPT; ++i) {
    const int id = threadIdx.x + kThreads * i;  // < ROWS*8 chunks of 8 elements
    uint4 val = make_uint4(0, 0, 0, 0);
    {
      int r, k;
      if (!mn_major) {  // 8 consecutive k of one row
        const int rr = id & 7, kc = (id >> 3) & 7, rg = id >> 6;
        r = rg * 8 + rr;
        k = k0 + kc * 8;
      } else {  // 8 consecutive rows of one k
        const int k8 = id & 7, mc = (id >> 3) % (ROWS / 8), kg = (id >> 3) / (ROWS / 8);
        r = mc * 8;
        k = k0 + kg * 8 + k8;
      }
      const int m = row0 + r;
      if (m < nrows && k < kend) {
        const long off = (long)(m / msplit) * s_m1 + (long)(m % msplit) * s_m0 + (long)k * s_k;
        val = __ldg(reinterpret_cast<const uint4*>(base + off));
      }
    }
    t.v[i] = val;
  }
}

// Store the chunks into the canonical layout:
//   K-major : core (row group g, k chunk c) at (g*8 + c)*128 B, row r%8 at +16*(r%8)
//             -> LBO (k chunk stride) 128 B, SBO (row group stride) 1024 B
//   MN-major: core (k group q, row chunk c) at (q*ROWS/8 + c)*128 B, k%8 at +16*(k%8)
//             -> LBO (k group stride) ROWS*16 B, SBO (row chunk stride) 128 B
template <int ROWS>
__device__ __forceinline__ void store_tile(const Tile16<ROWS>& t, uint8_t* sm, int mn_major) {
#pragma unroll
  for (int i = 0; i < Tile16<ROWS>::CPT; ++i) {
    const int id = threadIdx.x + kThreads * i;
    {
      int off;
      if (!mn_major) {
        const int rr = id & 7, kc = (id >> 3) & 7, rg = id >> 6;
        off = (rg * 8 + kc) * 128 + rr * 16;
      } else {
        const int k8 = id & 7, mc = (id >> 3) % (ROWS / 8), kg = (id >> 3) / (ROWS / 8);
        off = (kg * (ROWS / 8) + mc) * 128 + k8 * 16;
      }
      *reinterpret_cast<uint4*>(sm + off) = t.v[i];
    }
  }
}

template <int ROWS>
__device__ __forceinline__ uint64_t tile_desc(uint32_t saddr, int mn_major, int kstep) {
  // one MMA covers 16 k: two K-major k chunks or two MN-major k groups
  if (!mn_major) return umma_sdesc(saddr + kstep * 256, 128, 1024);
  return umma_sdesc(saddr + kstep * 2 * ROWS * 16, ROWS * 16, 128);
}

template <int BN, int EPI>
__global__ void __launch_bounds__(kThreads, BN <= 64 ? 4 : BN <= 128 ? 3 : 1) k_gemm(const GemmDesc d) {
  constexpr int A_BYTES = kBM * kBK * 2, B_BYTES = BN * kBK * 2, STAGE = A_BYTES + B_BYTES;
  constexpr int TCOLS = BN <= 32 ? 32 : BN <= 64 ? 64 : BN <= 128 ? 128 : 256;
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ uint64_t bar[2];
  __shared__ uint32_t tmem_sh;

  const int tid = threadIdx.x, warp = tid >> 5;
  const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * BN;
  const int zb = blockIdx.z / d.ksplit, zk = blockIdx.z % d.ksplit;
  const int kper = ((d.K + d.ksplit - 1) / d.ksplit + kBK - 1) / kBK * kBK;
  const int kbeg = zk * kper, kend = min(d.K, kbeg + kper);
  const int nk1 = kend > kbeg ? (kend - kbeg + kBK - 1) / kBK : 0;
  const int nk = nk1 + (d.K2 > 0 ? (d.K2 + kBK - 1) / kBK : 0);  // k tiles of both products
  const bf16* A = d.a + (long)zb * d.a_b;
  const bf16* B = d.b + (long)zb * d.b_b;
  const bf16* A2 = d.K2 > 0 ? d.a2 + (long)zb * d.a2_b : nullptr;
  const bf16* B2 = d.K2 > 0 ? d.b2 + (long)zb * d.b2_b + (long)(m0 / d.b2_mdiv) * d.b2_m : nullptr;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_sh)),
                 "r"(TCOLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = tmem_sh;
  const uint32_t idesc1 = umma_idesc(BN, d.a_mn_major, d.b_mn_major);
  const uint32_t idesc2 = umma_idesc(BN, d.a2_mn_major, d.b2_mn_major);
  const int tries = d.wait_tries == 0 ? kWaitTries : (d.wait_tries < 0 ? 0 : d.wait_tries);

  Tile16<kBM> ta;
  Tile16<BN> tb;
  bool ok = true;
  int issued = 0;  // k tiles whose MMAs were issued and committed
  for (int kt = 0; kt < nk; ++kt) {
    const int s = kt & 1;
    const bool first = kt < nk1;  // uniform: a k tile of the first product or of the second
    const int a_mn = first ? d.a_mn_major : d.a2_mn_major, b_mn = first ? d.b_mn_major : d.b2_mn_major;
    uint8_t* sa = smem + s * STAGE;
    uint8_t* sb = sa + A_BYTES;
    if (first) {
      const int k0 = kbeg + kt * kBK;
      load_tile<kBM>(ta, A, d.a_m0, d.a_m1, d.a_msplit, d.a_k, d.a_mn_major, m0, d.M, k0, kend);
      load_tile<BN>(tb, B, d.b_n, d.b_n1, d.b_nsplit, d.b_k, d.b_mn_major, n0, d.N, k0, kend);
    } else {
      const int k0 = (kt - nk1) * kBK;
      load_tile<kBM>(ta, A2, d.a2_m0, d.a2_m1, d.a2_msplit, d.a2_k, d.a2_mn_major, m0, d.M, k0, d.K2);
      load_tile<BN>(tb, B2, d.b2_n, 0, 1 << 30, d.b2_k, d.b2_mn_major, n0, d.N, k0, d.K2);
    }
    if (kt >= 2 && !mbar_wait(&bar[s], ((kt - 2) >> 1) & 1, tries)) ok = false;  // stage s free again
    if (__syncthreads_or(!ok)) {
      ok = false;
      break;
    }
    store_tile<kBM>(ta, sa, a_mn);
    store_tile<BN>(tb, sb, b_mn);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;");
      const uint32_t a0 = smem_u32(sa), b0 = smem_u32(sb);
#pragma unroll
      for (int kk = 0; kk < kBK / 16; ++kk) {
        const uint64_t da = tile_desc<kBM>(a0, a_mn, kk);
        const uint64_t db = tile_desc<BN>(b0, b_mn, kk);
        const uint32_t acc = (kt > 0 || kk > 0) ? 1u : 0u;
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(tmem),
            "l"(da), "l"(db), "r"(first ? idesc1 : idesc2), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(&bar[s]))
                   : "memory");
    }
    issued = kt + 1;
  }
  if (ok && issued > 0 && !mbar_wait(&bar[(issued - 1) & 1], ((issued - 1) >> 1) & 1, tries)) ok = false;
  if (__syncthreads_or(!ok)) {
    if (tid == 0 && d.err) atomicOr(d.err, 1);
    // let the MMAs in flight drain (bounded) before the accumulator is released
    if (issued > 0) mbar_wait(&bar[(issued - 1) & 1], ((issued - 1) >> 1) & 1);
  } else if (nk > 0 || d.c_mode == C_STORE) {
    asm volatile("tcgen05.fence::after_thread_sync;");
    const int r = warp * 32 + (tid & 31);
    const int m = m0 + r;
    const long crow = m < d.M ? (long)zb * d.c_b + (long)(m / d.c_msplit) * d.c_m1 + (long)(m % d.c_msplit) * d.c_m0 : 0;
#pragma unroll 1
    for (int cc = 0; cc < BN; cc += 16) {
      uint32_t v[16];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)cc;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (m >= d.M) continue;
      // all loads of the chunk first (independent, so they overlap), then the
      // arithmetic, then the stores; columns past N are masked, not branched on
      constexpr EpiForm E = epi_form(EPI);
      const bool has_bias = E.generic ? d.bias_n != nullptr : E.bias;
      const bool has_add = E.generic ? d.add != nullptr : E.add;
      const int act = E.generic ? d.act : E.act;
      const bool out_bf16 = E.generic ? d.c_bf16 != 0 : E.bf16;
      const int mode = E.generic ? d.c_mode : (E.atomic ? C_ATOMIC : C_STORE);
      const bool store_pre = d.pre != nullptr;  // uniform: inference passes no pre buffer
      float x[16], ad[16], pr[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int n = n0 + cc + j;
        const bool in = n < d.N;
        const long o = crow + (long)n * d.c_n;
        x[j] = nk > 0 ? d.alpha * __uint_as_float(v[j]) : 0.0f;
        ad[j] = (in && has_add) ? __ldg(d.add + o) : 0.0f;
        pr[j] = (in && act == ACT_GELU_GRAD) ? __bfloat162float(d.pre[o]) : 0.0f;
        if (in && has_bias) x[j] += __ldg(d.bias_n + n);
      }
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int n = n0 + cc + j;
        if (n >= d.N) continue;
        const long o = crow + (long)n * d.c_n;
        float y = x[j] + ad[j];
        if (act == ACT_GELU) {
          if (store_pre) d.pre[o] = __float2bfloat16(y);
          y = gelu_f(y);
        } else if (act == ACT_GELU_GRAD) {
          y *= gelu_grad_f(pr[j]);
        }
        if (out_bf16) {
          bf16* C = (bf16*)d.c;
          if (mode == C_ACCUM) y += __bfloat162float(C[o]);
          C[o] = __float2bfloat16(y);
        } else {
          float* C = (float*)d.c;
          if (mode == C_ATOMIC)
            atomicAdd(C + o, y);
          else if (mode == C_ACCUM)
            C[o] += y;
          else
            C[o] = y;
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TCOLS));
}

template <int BN>
constexpr int gemm_smem_bytes() {
  return 2 * (kBM * kBK * 2 + BN * kBK * 2);
}

}  // namespace fno
