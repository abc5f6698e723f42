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
 * b_k / b_n and its own row split (b_nsplit, b_n1).  Requirements: K % 8 == 0;
 * 16-byte aligned operands and 8-element aligned strides across the contiguous
 * chunks; M (resp. N) % 8 == 0 and the split % 8 == 0 for an MN-major A (resp. B).
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
  long b_n1;    /* B rows split like A's: (n / b_nsplit)*b_n1 + (n % b_nsplit)*b_n */
  int b_nsplit;
  int wait_tries; /* bound of the tensor-core pipeline waits, in tries of at most ~5 ms:
                   * 0 = default (400), > 0 = that many, -1 = none: the first wait gives
                   * up at once, sets bit 0 of *err and the kernel returns (a test of the
                   * time-out path; MMAs already issued are still drained with the default
                   * bound before the accumulator is released) */
  /* a second product accumulated into the same tile when K2 > 0:
   *   C = epilogue(alpha * (sum_k A(m,k) B(n,k) + sum_k2 A2(m,k2) B2(n,k2)))
   * A2 is addressed like A; B2 like B without a row split, its base moved by
   * (m0 / b2_mdiv) * b2_m for the 128-row tile whose first row is m0 (b2_mdiv a
   * multiple of 128).  Needs ksplit = 1. */
  int K2;
  int a2_msplit, a2_mn_major;
  const void* a2;
  long a2_m0, a2_m1, a2_k, a2_b;
  const void* b2;
  long b2_n, b2_k, b2_b, b2_m;
  int b2_mn_major, b2_mdiv;
} sac_fno_gemm_desc;

/* 0 on success; 1 on an argument that breaks the requirements (message in
 * sac_fno_last_error); 3 on a CUDA launch error. */
int sac_fno_gemm(const sac_fno_gemm_desc* d, void* cuda_stream);
const char* sac_fno_last_error(void);

/* ---- the network ----
 * FNO on an S x F grid: lift cin -> width (1x1), `layers` Fourier layers
 * z = W v + b + irfft2(R . rfft2(v)[24 x 24 corner modes]), GELU between layers,
 * projection width -> hidden (GELU) -> cout.  BF16 weights and activations,
 * FP32 accumulation and FP32 master weights.  Tensors are channel-first per
 * sample: x[b][c][s][f], f fastest. */
typedef struct sac_fno_config {
  int S, F;              /* grid (multiples of 8, at least 50) */
  int width, layers;     /* 32, 4 */
  int modes1, modes2;    /* 24, 24 (built in) */
  int hidden;            /* projection width, 128 */
  int cin, cout;         /* input channels (multiple of 16), outputs (<= 16) */
  int max_batch;         /* activations are held for this many samples (<= 64) */
  int device;
} sac_fno_config;
typedef struct sac_fno sac_fno;

void sac_fno_default_config(sac_fno_config* c);
int sac_fno_create(const sac_fno_config* c, sac_fno** out);
void sac_fno_destroy(sac_fno* n);
const char* sac_fno_error(const sac_fno* n);
void* sac_fno_stream(const sac_fno* n);   /* every call below is enqueued here */
long sac_fno_num_params(const sac_fno* n);
/* out[2*(6 + 4*layers)]: offset, count of each parameter group in the flat FP32
 * vector: P, Pb, then per
 * layer W, Wb, R.re, R.im (R[kx][ky][i][o], kx: 24 low then 24 high), then Q1, Q1b,
 * Q2, Q2b (Q2 padded to cout rounded up to 8 rows) */
int sac_fno_param_layout(const sac_fno* n, long* out);
int sac_fno_init(sac_fno* n, unsigned long long seed);
int sac_fno_set_params(sac_fno* n, const float* host);   /* synchronous */
int sac_fno_get_params(sac_fno* n, float* host);         /* synchronous */
int sac_fno_get_grads(sac_fno* n, float* host);          /* synchronous */
int sac_fno_zero_grad(sac_fno* n);
/* x: [B][cin][S][F] bf16, kept unchanged by the caller until sac_fno_backward;
 * y: [B][cout][S][F] float */
int sac_fno_forward(sac_fno* n, const void* x, float* y, int B);
/* the same output without storing what the backward pass needs (inference) */
int sac_fno_infer(sac_fno* n, const void* x, float* y, int B);
/* dy: [B][cout8][S][F] bf16, cout8 = cout rounded up to 8 (extra channels zero);
 * accumulates the parameter gradients of the last forward pass */
int sac_fno_backward(sac_fno* n, const void* dy);
/* loss += mean over the cout channels of (y - target)^2 (device float);
 * dy = its gradient (bf16, cout8 channels); target bf16 [B][cout][S][F] */
int sac_fno_mse(sac_fno* n, const float* y, const void* target, void* dy, float* loss, int B);
/* Adam with bias correction and decoupled weight decay; step counts from 1;
 * clip > 0 rescales the gradient to that global L2 norm (synchronises) */
int sac_fno_adam(sac_fno* n, float lr, float b1, float b2, float eps, float wd, int step, float clip);
/* x[b][c] = state[b][c] * scale[b*nst + c] for c < nst (state float or bf16,
 * [B][nst][S][F]); then nfeat constant planes feat[b*nfeat + k]; then the
 * coordinates s/S - 1/2 and f/F; the remaining channels zero */
int sac_fno_features(sac_fno* n, const void* state, int state_bf16, const float* scale, const float* feat,
                     int nfeat, void* x, int B, int nst);
/* state[b][c] += scale[b*nst + c] * y[b][c]  (float, [B][nst][S][F]) */
int sac_fno_apply(sac_fno* n, float* state, const float* y, const float* scale, int B, int nst);
/* synchronises; 7 when a tensor-core wait timed out since the last reset */
int sac_fno_check(sac_fno* n, int reset);
/* wait_tries of every GEMM the network launches (see sac_fno_gemm_desc; 0 =
 * default, -1 = give up at once, for testing the time-out report) */
int sac_fno_set_wait_tries(sac_fno* n, int tries);

#ifdef __cplusplus
}
#endif
#endif /* SAC_FNO_H */
