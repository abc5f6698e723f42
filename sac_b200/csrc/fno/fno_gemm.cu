// fno_gemm.cu -- host launcher of the tcgen05 GEMM (libsacfno.so).
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <string>

#include "fno_gemm.cuh"
#include "fno_host.h"
#include "sac_fno.h"

namespace fno {

static_assert(sizeof(sac_fno_gemm_desc) == sizeof(GemmDesc), "the C descriptor mirrors GemmDesc");

thread_local std::string g_err;

void set_error(const std::string& m) { g_err = m; }

namespace {

bool aligned16(const void* p) { return ((uintptr_t)p & 15) == 0; }

template <int BN, int EPI>
cudaError_t launch_kind(const GemmDesc& d, cudaStream_t st) {
  constexpr int smem = gemm_smem_bytes<BN>();
  static bool attr = false;  // per process; the attribute is per device function
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k_gemm<BN, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  dim3 grid((unsigned)((d.M + kBM - 1) / kBM), (unsigned)((d.N + BN - 1) / BN), (unsigned)(d.batch * d.ksplit));
  k_gemm<BN, EPI><<<grid, kThreads, smem, st>>>(d);
  return cudaGetLastError();
}

// the compiled epilogue form that matches the descriptor (EPI_GENERIC otherwise)
int epi_kind(const GemmDesc& d) {
  const bool bias = d.bias_n != nullptr, add = d.add != nullptr;
  if (d.c_mode == C_ATOMIC)
    return (!d.c_bf16 && !bias && !add && d.act == ACT_NONE) ? EPI_F32_ATOMIC : EPI_GENERIC;
  if (d.c_mode != C_STORE) return EPI_GENERIC;
  for (int k = 1; k < EPI_KINDS; ++k) {
    const EpiForm f = epi_form(k);
    if (f.atomic) continue;
    if (f.bias == bias && f.add == add && f.bf16 == (d.c_bf16 != 0) && f.act == d.act) return k;
  }
  return EPI_GENERIC;
}

template <int BN>
cudaError_t launch_bn(const GemmDesc& d, cudaStream_t st) {
  switch (epi_kind(d)) {
    case EPI_F32: return launch_kind<BN, EPI_F32>(d, st);
    case EPI_BF16: return launch_kind<BN, EPI_BF16>(d, st);
    case EPI_BF16_BIAS: return launch_kind<BN, EPI_BF16_BIAS>(d, st);
    case EPI_F32_BIAS: return launch_kind<BN, EPI_F32_BIAS>(d, st);
    case EPI_BF16_BIAS_GELU: return launch_kind<BN, EPI_BF16_BIAS_GELU>(d, st);
    case EPI_BF16_BIAS_ADD: return launch_kind<BN, EPI_BF16_BIAS_ADD>(d, st);
    case EPI_BF16_BIAS_ADD_GELU: return launch_kind<BN, EPI_BF16_BIAS_ADD_GELU>(d, st);
    case EPI_BF16_ADD: return launch_kind<BN, EPI_BF16_ADD>(d, st);
    case EPI_BF16_ADD_GRAD: return launch_kind<BN, EPI_BF16_ADD_GRAD>(d, st);
    case EPI_BF16_GRAD: return launch_kind<BN, EPI_BF16_GRAD>(d, st);
    case EPI_F32_ATOMIC: return launch_kind<BN, EPI_F32_ATOMIC>(d, st);
    default: return launch_kind<BN, EPI_GENERIC>(d, st);
  }
}

}  // namespace

int gemm(const GemmDesc& d, cudaStream_t st) {
  auto bad = [](const char* m) {
    set_error(std::string("sac_fno_gemm: ") + m);
    return 1;
  };
  if (d.M <= 0 || d.N <= 0 || d.K <= 0 || d.batch <= 0 || d.ksplit <= 0) return bad("empty or negative sizes");
  if (d.K % 8) return bad("K must be a multiple of 8");
  if ((long)d.batch * d.ksplit > 65535) return bad("batch * ksplit exceeds the grid limit");
  if (!d.a || !d.b || !d.c) return bad("null operand");
  if (!aligned16(d.a) || !aligned16(d.b)) return bad("operands must be 16-byte aligned");
  if (d.a_msplit <= 0 || d.c_msplit <= 0) return bad("msplit must be positive");
  if (d.a_mn_major) {
    if (d.a_m0 != 1) return bad("MN-major A needs a_m0 == 1");
    if (d.M % 8 || d.a_msplit % 8 || d.a_k % 8 || d.a_m1 % 8 || d.a_b % 8) return bad("MN-major A alignment");
  } else {
    if (d.a_k != 1) return bad("K-major A needs a_k == 1");
    if (d.a_m0 % 8 || d.a_m1 % 8 || d.a_b % 8) return bad("K-major A alignment");
  }
  if (d.b_nsplit <= 0) return bad("b_nsplit must be positive");
  if (d.b_mn_major) {
    if (d.b_n != 1) return bad("MN-major B needs b_n == 1");
    if (d.N % 8 || d.b_nsplit % 8 || d.b_k % 8 || d.b_n1 % 8 || d.b_b % 8) return bad("MN-major B alignment");
  } else {
    if (d.b_k != 1) return bad("K-major B needs b_k == 1");
    if (d.b_n % 8 || d.b_n1 % 8 || d.b_b % 8) return bad("K-major B alignment");
  }
  if (d.K2 < 0) return bad("negative K2");
  if (d.K2 > 0) {
    if (d.K2 % 8) return bad("K2 must be a multiple of 8");
    if (d.ksplit != 1) return bad("a second product needs ksplit == 1");
    if (!d.a2 || !d.b2) return bad("null second operand");
    if (!aligned16(d.a2) || !aligned16(d.b2)) return bad("second operands must be 16-byte aligned");
    if (d.a2_msplit <= 0) return bad("a2_msplit must be positive");
    if (d.b2_mdiv <= 0 || d.b2_mdiv % kBM) return bad("b2_mdiv must be a positive multiple of 128");
    if (d.a2_mn_major) {
      if (d.a2_m0 != 1) return bad("MN-major A2 needs a2_m0 == 1");
      if (d.M % 8 || d.a2_msplit % 8 || d.a2_k % 8 || d.a2_m1 % 8 || d.a2_b % 8) return bad("MN-major A2 alignment");
    } else {
      if (d.a2_k != 1) return bad("K-major A2 needs a2_k == 1");
      if (d.a2_m0 % 8 || d.a2_m1 % 8 || d.a2_b % 8) return bad("K-major A2 alignment");
    }
    if (d.b2_mn_major) {
      if (d.b2_n != 1) return bad("MN-major B2 needs b2_n == 1");
      if (d.N % 8 || d.b2_k % 8 || d.b2_b % 8 || d.b2_m % 8) return bad("MN-major B2 alignment");
    } else {
      if (d.b2_k != 1) return bad("K-major B2 needs b2_k == 1");
      if (d.b2_n % 8 || d.b2_b % 8 || d.b2_m % 8) return bad("K-major B2 alignment");
    }
  }
  if (d.c_mode == C_ATOMIC && d.c_bf16) return bad("atomic accumulation needs a float C");
  if (d.ksplit > 1 && d.c_mode != C_ATOMIC) return bad("ksplit > 1 needs c_mode atomic");
  if (d.act == ACT_GELU_GRAD && !d.pre) return bad("GELU' needs the pre-activation");
  if (d.c_mode == C_ATOMIC && (d.act != ACT_NONE || d.bias_n || d.add))
    return bad("atomic accumulation takes no bias, add or activation");
  // widest tile that covers N, narrowed while the grid would leave SMs idle
  int bn = d.N <= 16 ? 16 : d.N <= 32 ? 32 : d.N <= 48 ? 48 : d.N <= 64 ? 64 : d.N <= 96 ? 96 : d.N <= 128 ? 128 : 256;
  const long mt = (d.M + kBM - 1) / kBM * (long)d.batch * d.ksplit;
  while (bn > 64 && bn % 64 == 0 && mt * ((d.N + bn - 1) / bn) < 2L * 148) bn /= 2;
  cudaError_t e;
  switch (bn) {
    case 16: e = launch_bn<16>(d, st); break;
    case 32: e = launch_bn<32>(d, st); break;
    case 48: e = launch_bn<48>(d, st); break;
    case 64: e = launch_bn<64>(d, st); break;
    case 96: e = launch_bn<96>(d, st); break;
    case 128: e = launch_bn<128>(d, st); break;
    default: e = launch_bn<256>(d, st); break;
  }
  if (e != cudaSuccess) {
    set_error(std::string("sac_fno_gemm: ") + cudaGetErrorString(e));
    return 3;
  }
  return 0;
}

}  // namespace fno

extern "C" {

int sac_fno_gemm(const sac_fno_gemm_desc* d, void* stream) {
  if (!d) return 1;
  fno::GemmDesc g;
  std::memcpy(&g, d, sizeof(g));
  return fno::gemm(g, (cudaStream_t)stream);
}

const char* sac_fno_last_error(void) { return fno::g_err.c_str(); }

}  // extern "C"
