/*
 * naja_mlp.h -- C ABI of the learned-rounding network's kernels (sm_100a).
 *
 * The rounding network maps a conditioned model's bound ratios
 * log(u_new / u_base) to a diagonal-plus-low-rank affine rounding
 * y = (diag(exp(d)) + U U^T) z + c of its polytope.  It has no counterpart
 * in quothbonney/naja (the reference's nearest precedents are the pair
 * schedule warmup, src/rounding/runtime_warmup.cpp:16-108, and the Dikin
 * preconditioner, src/rounding/dikin_precondition.cpp:36-183, which stays
 * the fallback).  Training and inference run on these kernels: BF16 operands
 * with FP32 accumulation on the tensor cores (tcgen05, accumulator in tensor
 * memory), FP32 master weights and Adam moments.
 *
 * Layouts: every matrix is row-major with an explicit row pitch in elements;
 * BF16 pitches are multiples of 8 (16-byte rows) and BF16 bases 16-byte
 * aligned.  All pointers are device memory; calls are asynchronous on
 * `stream` (a cudaStream_t, NULL = legacy default stream).  Return values
 * are naja status codes (naja_chr.h); naja_last_error() has the message.
 */
#ifndef NAJA_MLP_H
#define NAJA_MLP_H

#ifdef __cplusplus
extern "C" {
#endif

/* What the GEMM epilogue writes for element (m, n), v = acc + bias[n]:
 *   c_f32      (optional)  C[m*ldc + n] = v, or C += v with accumulate
 *   act        (optional)  BF16 g(v) at act[m*ld_act + n]
 *   act_t      (optional)  BF16 g(v) at act_t[n*ld_act_t + m]
 * with g = GELU (erf form) when gelu != 0, else the identity. */
typedef struct naja_gemm_epilogue {
  const float* bias;
  float* c_f32;
  int ldc;
  int accumulate;
  void* act;
  int ld_act;
  void* act_t;
  int ld_act_t;
  int gelu;
} naja_gemm_epilogue;

/* D (M x N) = A (M x K) B (N x K)^T, A and B BF16 row-major (K contiguous),
 * FP32 accumulation; D goes through the epilogue. */
int naja_gemm_bf16(int M, int N, int K, const void* A, int lda, const void* B, int ldb,
                   const naja_gemm_epilogue* epi, void* stream);

/* Synchronises `stream` and reports (and clears) a bounded wait that a
 * naja_gemm_bf16 launch gave up since the last check. */
int naja_mlp_check(void* stream);

/* FP32 (rows x cols, ld_src) -> BF16 copy (ld_dst) and/or transposed BF16
 * copy (cols x rows, ld_dst_t); either output may be NULL. */
int naja_cast_bf16(int rows, int cols, const float* src, int ld_src, void* dst, int ld_dst, void* dst_t,
                   int ld_dst_t, void* stream);

/* dpre = dact * GELU'(pre) for (rows x cols) FP32 matrices (pitch ld); writes
 * dpre as FP32 (ld), BF16 (ld_bf) and transposed BF16 (ld_bf_t). */
int naja_gelu_backward(int rows, int cols, const float* dact, const float* pre, int ld, float* dpre,
                       void* dpre_bf, int ld_bf, void* dpre_bf_t, int ld_bf_t, void* stream);

/* Weighted mean-squared error over (rows x cols): loss = sum w[n] (out - t)^2
 * / rows, accumulated into *loss (one double, device memory); the gradient
 * 2 w[n] (out - t) / rows is written as FP32 (ld), BF16 (ld_bf) and
 * transposed BF16 (ld_bf_t). */
int naja_mse_grad(int rows, int cols, const float* out, const float* target, int ld, const float* w,
                  double* loss, float* grad, void* grad_bf, int ld_bf, void* grad_bf_t, int ld_bf_t,
                  void* stream);

/* db[n] = sum_m d[m*ld + n] over (rows x cols). */
int naja_col_sum(int rows, int cols, const float* d, int ld, float* db, void* stream);

/* Adam step on FP32 master weights W (rows x cols, ld) with moments m, v and
 * gradient g (same layout); refreshes the BF16 copy (ld_bf) and transposed
 * BF16 copy (ld_bf_t) when given.  step is 1-based. */
int naja_adam(int rows, int cols, float* W, const float* g, float* m, float* v, int ld, float lr, float beta1,
              float beta2, float eps, int step, void* w_bf, int ld_bf, void* w_bf_t, int ld_bf_t,
              void* stream);

#ifdef __cplusplus
}
#endif
#endif /* NAJA_MLP_H */
