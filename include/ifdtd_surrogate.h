/*
 * ifdtd_surrogate.h - kernels of the learned receiver-trace surrogate.
 *
 * No counterpart in the reference: ruddyscent/ionosphere-fdtd has no
 * surrogate model.  These entry points are the forward and backward building
 * blocks of a small network trained on traces the FDTD engine generates: a
 * BF16 tensor-core GEMM with FP32 accumulation and the elementwise training
 * steps.  All pointers are device pointers; bf16 arrays are passed as void*.
 * Every call is asynchronous on `stream` and returns an ifdtd_status
 * (ifdtd.h); ifdtd_last_error gives the message.
 */
#ifndef IFDTD_SURROGATE_H
#define IFDTD_SURROGATE_H

#include <stdint.h>

#include "ifdtd.h"

#ifdef __cplusplus
extern "C" {
#endif

/* c (m x n, fp32, row-major, leading dimension ldc) = alpha * op(a) op(b) + beta * c.
 * op(a) is m x k: a is bf16 row-major m x k (trans_a = 0) or k x m (trans_a = 1).
 * op(b) is k x n: b is bf16 row-major k x n (trans_b = 0) or n x k (trans_b = 1). */
int32_t ifdtd_nn_gemm(int32_t m, int32_t n, int32_t k, const void* a, int32_t lda, int32_t trans_a, const void* b,
                      int32_t ldb, int32_t trans_b, float alpha, float beta, float* c, int32_t ldc, void* stream);
/* The same product on the 5th-generation tensor cores: tcgen05.mma (bf16 inputs, fp32 accumulation
 * in tensor memory), one 128 x 128 tile of c per 128-thread CTA, K in chunks of 64 staged in shared
 * memory.  Same arguments and result as ifdtd_nn_gemm up to fp32 rounding of the accumulation. */
int32_t ifdtd_nn_gemm_tc(int32_t m, int32_t n, int32_t k, const void* a, int32_t lda, int32_t trans_a, const void* b,
                         int32_t ldb, int32_t trans_b, float alpha, float beta, float* c, int32_t ldc, void* stream);
/* ifdtd_nn_gemm_tc with a caller-owned device workspace (workspace_bytes may be 0): when the
 * output tiles would leave most SMs idle and K is long (the weight gradients of the decoder, whose K
 * is the number of rows), K is split over CTAs that write fp32 partial tiles into the workspace
 * (at most workspace_bytes / (4 m n) splits), and a second kernel adds them in split order, so the
 * result is the same on every run.  Calls that share a workspace must not overlap on the GPU. */
int32_t ifdtd_nn_gemm_tc_ws(int32_t m, int32_t n, int32_t k, const void* a, int32_t lda, int32_t trans_a, const void* b,
                            int32_t ldb, int32_t trans_b, float alpha, float beta, float* c, int32_t ldc, void* workspace,
                            int64_t workspace_bytes, void* stream);
/* Status word of ifdtd_nn_gemm_tc: bit 0 set when an mbarrier wait ran out its 0.2 s bound (that
 * call's result is then invalid).  Reading it synchronises the device; reset != 0 clears it. */
int32_t ifdtd_nn_gemm_tc_status(int32_t reset, int32_t* out);
/* z (rows x cols, fp32) += bias (cols); y_bf16 = act(z) (act 0 identity, 1 SiLU; y may be NULL). */
int32_t ifdtd_nn_bias_act(int32_t rows, int32_t cols, float* z, const float* bias, int32_t act, void* y_bf16,
                          void* stream);
/* dz = dy * act'(z), written as fp32 and as bf16. */
int32_t ifdtd_nn_act_grad(int32_t rows, int32_t cols, const float* z, const float* dy, int32_t act, float* dz,
                          void* dz_bf16, void* stream);
/* out[c] = sum over the rows of x[r, c] (bias gradients). */
int32_t ifdtd_nn_col_sum(int32_t rows, int32_t cols, const float* x, float* out, void* stream);
/* grad = 2 (pred - target) / n; *loss += mean squared error (loss must start at 0). */
int32_t ifdtd_nn_mse(int32_t n, const float* pred, const float* target, float* grad, float* loss, void* stream);
/* Row-weighted squared error over a rows x cols array: *loss += sum_r row_weight[r] * sum_c (pred - target)^2
 * / (rows * cols), grad = 2 row_weight[r] (pred - target) / (rows * cols) (loss must start at 0). */
int32_t ifdtd_nn_wmse(int32_t rows, int32_t cols, const float* pred, const float* target, const float* row_weight,
                      float* grad, float* loss, void* stream);
/* One Adam step (bias-corrected, step >= 1) on fp32 weights w; w_bf16 (may be NULL) receives the bf16 copy. */
int32_t ifdtd_nn_adam(int32_t n, float* w, const float* g, float* m, float* v, float lr, float beta1, float beta2,
                      float eps, int32_t step, void* w_bf16, void* stream);
/* y (bf16) = x (fp32), n elements. */
int32_t ifdtd_nn_to_bf16(int64_t n, const float* x, void* y, void* stream);

#ifdef __cplusplus
}
#endif

#endif
