// Kernels of the learned trace surrogate: a BF16 tensor-core GEMM with FP32
// accumulation (forward and both backward products of every layer) and the
// elementwise steps of training (bias + SiLU, its derivative, column sums,
// mean-squared error, Adam).  The network is a small MLP followed by
// non-overlapping transposed convolutions; with activations kept channels-last
// every one of its layers is a dense product over rows, so this one GEMM serves
// all of them.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <string>

#include "../../include/ifdtd_surrogate.h"
#include "errors.cuh"

namespace ifdtd {
namespace nn {

constexpr int BM = 64, BN = 64, BK = 32, PAD = 8, THREADS = 128;

__device__ __forceinline__ uint32_t pack2(__nv_bfloat16 lo, __nv_bfloat16 hi) {
  return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

// C (M x N, fp32, row-major, ldc) = alpha * op(A) op(B) + beta * C, with op(A)
// M x K and op(B) K x N.  A is row-major M x K (ta = 0) or K x M (ta = 1); B is
// row-major K x N (tb = 0) or N x K (tb = 1).  A 64 x 64 tile per CTA, four
// warps of 32 x 32, each of 2 x 4 mma.m16n8k16 (bf16 inputs, fp32 accumulate);
// shared tiles hold A as [m][k] and B as [n][k], zero outside the matrices.
__global__ void __launch_bounds__(THREADS) gemm_bf16(int M, int N, int K, const __nv_bfloat16* __restrict__ A, int lda,
                                                     int ta, const __nv_bfloat16* __restrict__ B, int ldb, int tb,
                                                     float alpha, float beta, float* __restrict__ C, int ldc) {
  __shared__ __align__(16) __nv_bfloat16 As[BM][BK + PAD];
  __shared__ __align__(16) __nv_bfloat16 Bs[BN][BK + PAD];
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;  // row tiles on x (up to 2^31 - 1 of them)
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  const int g = lane >> 2, t = lane & 3;
  float acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.f;
  const __nv_bfloat16 zero = __float2bfloat16(0.f);
  for (int k0 = 0; k0 < K; k0 += BK) {
    for (int e = threadIdx.x; e < BM * BK; e += THREADS) {
      const int r = e / BK, c = e % BK, gm = m0 + r, gk = k0 + c;
      As[r][c] = (gm < M && gk < K) ? (ta ? A[(size_t)gk * lda + gm] : A[(size_t)gm * lda + gk]) : zero;
    }
    for (int e = threadIdx.x; e < BN * BK; e += THREADS) {
      const int r = e / BK, c = e % BK, gn = n0 + r, gk = k0 + c;
      Bs[r][c] = (gn < N && gk < K) ? (tb ? B[(size_t)gn * ldb + gk] : B[(size_t)gk * ldb + gn]) : zero;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; kk += 16) {
      uint32_t a[2][4], b[4][2];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int r = wm + 16 * i + g;
        a[i][0] = pack2(As[r][kk + 2 * t], As[r][kk + 2 * t + 1]);
        a[i][1] = pack2(As[r + 8][kk + 2 * t], As[r + 8][kk + 2 * t + 1]);
        a[i][2] = pack2(As[r][kk + 2 * t + 8], As[r][kk + 2 * t + 9]);
        a[i][3] = pack2(As[r + 8][kk + 2 * t + 8], As[r + 8][kk + 2 * t + 9]);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int n = wn + 8 * j + g;
        b[j][0] = pack2(Bs[n][kk + 2 * t], Bs[n][kk + 2 * t + 1]);
        b[j][1] = pack2(Bs[n][kk + 2 * t + 8], Bs[n][kk + 2 * t + 9]);
      }
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
          asm volatile(
              "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
              "{%0, %1, %2, %3};"
              : "+f"(acc[i][j][0]), "+f"(acc[i][j][1]), "+f"(acc[i][j][2]), "+f"(acc[i][j][3])
              : "r"(a[i][0]), "r"(a[i][1]), "r"(a[i][2]), "r"(a[i][3]), "r"(b[j][0]), "r"(b[j][1]));
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int row = m0 + wm + 16 * i + g + 8 * h;
        if (row >= M) continue;
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const int col = n0 + wn + 8 * j + 2 * t + q;
          if (col >= N) continue;
          float* p = C + (size_t)row * ldc + col;
          const float v = alpha * acc[i][j][2 * h + q];
          *p = beta == 0.f ? v : v + beta * *p;
        }
      }
}

__device__ __forceinline__ float silu(float z) { return z / (1.f + expf(-z)); }
__device__ __forceinline__ float silu_grad(float z) {
  const float s = 1.f / (1.f + expf(-z));
  return s * (1.f + z * (1.f - s));
}

// z += bias (per column); y = act(z) as bf16 (act 0: identity, 1: SiLU)
__global__ void bias_act(int rows, int cols, float* __restrict__ z, const float* __restrict__ bias, int act,
                         __nv_bfloat16* __restrict__ y) {
  const size_t n = (size_t)rows * cols;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float v = z[i] + bias[i % cols];
    z[i] = v;
    if (y) y[i] = __float2bfloat16(act ? silu(v) : v);
  }
}

// dz = dy * act'(z), as fp32 and as bf16
__global__ void act_grad(int rows, int cols, const float* __restrict__ z, const float* __restrict__ dy, int act,
                         float* __restrict__ dz, __nv_bfloat16* __restrict__ dz16) {
  const size_t n = (size_t)rows * cols;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float v = act ? dy[i] * silu_grad(z[i]) : dy[i];
    dz[i] = v;
    dz16[i] = __float2bfloat16(v);
  }
}

// out[c] = sum over rows of x[r, c]: one 256-thread block per column, rows
// strided over the threads, then a fixed-order tree (the same bits every run)
__global__ void col_sum(int rows, int cols, const float* __restrict__ x, float* __restrict__ out) {
  __shared__ float part[256];
  const int c = blockIdx.x;
  float s = 0.f;
  for (int r = threadIdx.x; r < rows; r += blockDim.x) s += x[(size_t)r * cols + c];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[c] = part[0];
}

// grad = 2 (p - t) / n; loss[0] += sum (p - t)^2 / n (one atomic per block)
__global__ void mse(int n, const float* __restrict__ p, const float* __restrict__ t, float* __restrict__ grad,
                    float* __restrict__ loss) {
  __shared__ float part[256];
  float s = 0.f;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float d = p[i] - t[i];
    grad[i] = 2.f * d / (float)n;
    s += d * d;
  }
  part[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(loss, part[0] / (float)n);
}

// Row-weighted squared error: loss += sum_r w[r] sum_c (p - t)^2 / (rows * cols),
// grad = 2 w[r] (p - t) / (rows * cols) (w[r] = 1 / mean square of target row
// r makes every trace count by its relative error)
__global__ void wmse(int rows, int cols, const float* __restrict__ p, const float* __restrict__ t,
                     const float* __restrict__ w, float* __restrict__ grad, float* __restrict__ loss) {
  __shared__ float part[256];
  const int n = rows * cols;
  float s = 0.f;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float d = p[i] - t[i], wr = w[i / cols];
    grad[i] = 2.f * wr * d / (float)n;
    s += wr * d * d;
  }
  part[threadIdx.x] = s;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if (threadIdx.x < k) part[threadIdx.x] += part[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(loss, part[0] / (float)n);
}

// Adam on fp32 master weights; the bf16 copy the GEMMs read is refreshed
__global__ void adam(int n, float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                     float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2,
                     __nv_bfloat16* __restrict__ w16) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    if (w16) w16[i] = __float2bfloat16(wi);
  }
}

__global__ void to_bf16(size_t n, const float* __restrict__ x, __nv_bfloat16* __restrict__ y) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    y[i] = __float2bfloat16(x[i]);
}

int grid1d(size_t n) {
  const size_t b = (n + 255) / 256;
  return (int)(b < 1 ? 1 : (b > 148 * 8 ? 148 * 8 : b));
}

int launched(const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return record_error(IFDTD_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return IFDTD_OK;
}

}  // namespace nn
}  // namespace ifdtd

using namespace ifdtd::nn;

extern "C" {

int32_t ifdtd_nn_gemm(int32_t m, int32_t n, int32_t k, const void* a, int32_t lda, int32_t trans_a, const void* b,
                      int32_t ldb, int32_t trans_b, float alpha, float beta, float* c, int32_t ldc, void* stream) {
  if (m <= 0 || n <= 0 || k <= 0 || !a || !b || !c) return ifdtd::record_error(IFDTD_ERR_ARGUMENT, "bad gemm shape");
  if (lda < (trans_a ? m : k) || ldb < (trans_b ? k : n) || ldc < n)
    return ifdtd::record_error(IFDTD_ERR_ARGUMENT, "gemm leading dimension too small");
  if ((n + BN - 1) / BN > 65535) return ifdtd::record_error(IFDTD_ERR_ARGUMENT, "gemm has too many columns");
  const dim3 grid((m + BM - 1) / BM, (n + BN - 1) / BN);
  gemm_bf16<<<grid, THREADS, 0, (cudaStream_t)stream>>>(m, n, k, (const __nv_bfloat16*)a, lda, trans_a != 0,
                                                          (const __nv_bfloat16*)b, ldb, trans_b != 0, alpha, beta, c,
                                                          ldc);
  return launched("gemm_bf16");
}

int32_t ifdtd_nn_bias_act(int32_t rows, int32_t cols, float* z, const float* bias, int32_t act, void* y_bf16,
                          void* stream) {
  if (rows <= 0 || cols <= 0 || !z || !bias || act < 0 || act > 1)
    return ifdtd::record_error(IFDTD_ERR_ARGUMENT, "bad bias_act arguments");
  bias_act<<<grid1d((size_t)rows * cols), 256, 0, (cudaStream_t)stream>>>(rows, cols, z, bias, act,
                                                                           (__nv_bfloat16*)y_bf16);
  return launched("bias_act");
}

int32_t ifdtd_nn_act_grad(int32_t rows, int32_t cols, const float* z, const float* dy, int32_t act, float* dz,
                          void* dz_bf16, void* stream) {
  if (rows <= 0 || cols <= 0 || !z || !dy || !dz || !dz_bf16 || act < 0 || act > 1)
    return ifdtd::record_error(IFDTD_ERR_ARGUMENT, "bad act_grad arguments");
  act_grad<<<grid1d((size_t)rows * cols), 256, 0, (cudaStream_t)stream>>>(rows, cols, z, dy, act, dz,
                                                                           (__nv_bfloat16*)dz_bf16);
  return launched("act_grad");
}

int32_t ifdtd_nn_col_sum(int32_t rows, int32_t cols, const float* x, float* out, void* stream) {
  if (rows <= 0 || cols <= 0 || !x || !out) return ifdtd::record_error(IFDTD_ERR_ARGUMENT, "bad col_sum arguments");
  col_sum<<<cols, 256, 0, (cudaStream_t)stream>>>(rows, cols, x, out);
  return launched("col_sum");
}

int32_t ifdtd_nn_mse(int32_t n, const float* pred, const float* target, float* grad, float* loss, void* stream) {
  if (n <= 0 || !pred || !target || !grad || !loss) return ifdtd::record_error(IFDTD_ERR_ARGUMENT, "bad mse arguments");
  mse<<<grid1d((size_t)n), 256, 0, (cudaStream_t)stream>>>(n, pred, target, grad, loss);
  return launched("mse");
}

int32_t ifdtd_nn_wmse(int32_t rows, int32_t cols, const float* pred, const float* target, const float* row_weight,
                      float* grad, float* loss, void* stream) {
  if (rows <= 0 || cols <= 0 || (int64_t)rows * cols >= (int64_t)1 << 31 || !pred || !target || !row_weight || !grad || !loss)
    return ifdtd::record_error(IFDTD_ERR_ARGUMENT, "bad wmse arguments");
  wmse<<<grid1d((size_t)rows * cols), 256, 0, (cudaStream_t)stream>>>(rows, cols, pred, target, row_weight, grad, loss);
  return launched("wmse");
}

int32_t ifdtd_nn_adam(int32_t n, float* w, const float* g, float* m, float* v, float lr, float beta1, float beta2,
                      float eps, int32_t step, void* w_bf16, void* stream) {
  if (n <= 0 || !w || !g || !m || !v || step < 1) return ifdtd::record_error(IFDTD_ERR_ARGUMENT, "bad adam arguments");
  const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
  adam<<<grid1d((size_t)n), 256, 0, (cudaStream_t)stream>>>(n, w, g, m, v, lr, beta1, beta2, eps, c1, c2,
                                                           (__nv_bfloat16*)w_bf16);
  return launched("adam");
}

int32_t ifdtd_nn_to_bf16(int64_t n, const float* x, void* y, void* stream) {
  if (n <= 0 || !x || !y) return ifdtd::record_error(IFDTD_ERR_ARGUMENT, "bad to_bf16 arguments");
  to_bf16<<<grid1d((size_t)n), 256, 0, (cudaStream_t)stream>>>((size_t)n, x, (__nv_bfloat16*)y);
  return launched("to_bf16");
}

}  // extern "C"
