/*
 * sac_fno.h -- C-ABI of the Fourier-neural-operator surrogate (libsacfno.so).
 *
 * No reference counterpart: the surrogate is a library extension that advances a
 * 2D perturbation state by a fixed number of solver steps per call.  Device
 * pointers are passed in and out; every call is asynchronous on the given CUDA
 * stream unless stated.
 */
#ifndef SAC_FNO_H
#define SAC_FNO_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- BF16 GEMM on the tensor cores (tcgen05), the engine of every layer ----
 *   C(m,n) = epilogue(alpha * sum_k A(m,k) * B(n,k))
 * Row index splits: addr(m, x) = base + batch*s_b + (m / msplit)*s_m1 + (m % msplit)*s_m0 + x*s_x.
 * A is K-major (a_k == 1) or MN-major (a_m0 == 1, a_mn_major = 1); B likewise with
 * b_k / b_n.  Requirements: K % 8 == 0; 16-byte aligned operands and 8-element
 * aligned strides across the contiguous chunks; M (resp. N) % 8 == 0 and
 * msplit % 8 == 0 for an MN-major A (resp. B).
 * Epilogue: + bias_n[n], + add(m,n) (float, C addressing), then act: 1 = GELU
 * (the pre-activation is stored to pre when given), 2 = multiply by GELU'(pre).
 * c_mode: 0 store, 1 accumulate, 2 atomic add (float C; with ksplit > 1). */
typedef struct sac_fno_gemm_desc {
  int M, N, K, batch, ksplit;
  const void* a;
  long a_m0, a_m1, a_k, a_b;
  int a_msplit, a_mn_major;
  const void* b;
  long b_n, b_k, b_b;
  int b_mn_major;
  void* c;
  long c_m0, c_m1, c_n, c_b;
  int c_msplit, c_bf16, c_mode;
  float alpha;
  const float* bias_n;
  const float* add;
  int act;
  void* pre;
  int* err;
} sac_fno_gemm_desc;

/* 0 on success; 1 on an argument that breaks the requirements (message in
 * sac_fno_last_error); 3 on a CUDA launch error. */
int sac_fno_gemm(const sac_fno_gemm_desc* d, void* cuda_stream);
const char* sac_fno_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* SAC_FNO_H */
