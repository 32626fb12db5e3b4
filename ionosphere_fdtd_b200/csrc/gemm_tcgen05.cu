// BF16 GEMM of the trace surrogate on the 5th-generation tensor cores
// (tcgen05.mma, sm_100a): C (M x N, fp32) = alpha * op(A) op(B) + beta * C.
//
// One CTA of 128 threads (one warpgroup) computes a 128 x 128 tile of C.  The
// accumulator lives in tensor memory: warp 0 allocates 128 TMEM columns (fp32,
// one column per output column, lane = output row).  K runs in chunks of 64:
// all threads stage the chunk's A tile (128 rows x 64) and B tile (128 output
// columns x 64) in shared memory, K-major, in the no-swizzle core-matrix
// layout the MMA reads (8 rows x 16 bytes per core matrix, 128 bytes apart
// along K, 1024 bytes apart along M / N), zero outside the matrices, so ragged
// shapes and both transposes need no special case in the MMA.  One elected
// thread issues four tcgen05.mma (M 128, N 128, K 16 each, bf16 inputs, fp32
// accumulate) per chunk and commits them to the chunk's mbarrier; two stages
// let the next chunk load while the MMAs of the previous one run.  The
// epilogue reads the accumulator with tcgen05.ld (each warp its 32 TMEM lanes)
// and writes alpha * acc + beta * C.
//
// Every mbarrier wait is bounded by the global timer (0.2 s).  A wait that runs
// out sets bit 0 of the module status word (ifdtd_nn_gemm_tc_status), the CTA
// skips its remaining chunks and its epilogue, waits (again bounded) for the
// MMAs it issued, frees its tensor memory and returns.  No operand is another
// GPU's memory and no copy uses cluster multicast.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <string>

#include "../../include/ifdtd_surrogate.h"
#include "errors.cuh"

namespace ifdtd {
namespace tc {

constexpr int TM = 128, TN = 128, TK = 64, THREADS = 128, STAGES = 2;
constexpr int A_BYTES = TM * TK * 2, B_BYTES = TN * TK * 2, STAGE_BYTES = A_BYTES + B_BYTES;
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024;  // + room to align the stages to 1024 bytes
constexpr uint32_t TMEM_COLS = 128;
constexpr uint64_t kWaitNs = 200ull * 1000 * 1000;

__device__ int g_status;

// Instruction descriptor of tcgen05.mma.kind::f16: fp32 accumulator (bits 4-5
// = 1), A and B bf16 (bits 7-9 and 10-12 = 1), both K-major (bits 15, 16 = 0),
// N >> 3 at bits 17-22, M >> 4 at bits 24-28; dense, no negation.
constexpr uint32_t kInstrDesc =
    (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TN >> 3) << 17) | ((uint32_t)(TM >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

// Shared-memory matrix descriptor: start address >> 4 (bits 0-13), leading
// byte offset >> 4 (bits 16-29: the next core matrix along K, 128 B), stride
// byte offset >> 4 (bits 32-45: the next 8-row group, 1024 B), the sm_100
// descriptor version 1 (bits 46-48), base offset 0, no swizzle (bits 61-63 = 0).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)(128u >> 4) << 16) | ((uint64_t)(1024u >> 4) << 32) |
         ((uint64_t)1 << 46);
}

// Byte offset of the 16-byte row piece (row, k-group) in a 128 x 64 tile: core
// matrix (row / 8, kg) at ((row / 8) * 8 + kg) * 128, row % 8 at 16 * (row % 8).
__device__ __forceinline__ uint32_t core_offset(int row, int kg) {
  return (uint32_t)((((row >> 3) << 3) + kg) * 128 + ((row & 7) << 4));
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for the phase of `bar` with this parity; false (and the status
// bit set) when it did not complete within kWaitNs.
__device__ __forceinline__ bool wait_bounded(uint32_t bar, uint32_t parity) {
  if (mbar_try(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  for (uint32_t i = 1; i < (1u << 30); ++i) {
    if (mbar_try(bar, parity)) return true;
    if ((i & 15u) == 0 && global_ns() - t0 > kWaitNs) break;
  }
  atomicOr(&g_status, 1);
  return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// The 8 bf16 of op(X)[row][k0 .. k0 + 7] (zero outside rows x cols) as one
// 16-byte piece.  op(X) is rows x cols: X row-major rows x cols (trans = 0,
// contiguous along k) or cols x rows (trans = 1, strided); `vec` allows one
// 16-byte load when the piece lies inside a contiguous row.
__device__ __forceinline__ uint4 load_piece(const __nv_bfloat16* __restrict__ X, int ld, int trans, int rows, int cols,
                                            int row, int k0, bool vec) {
  uint4 v = make_uint4(0u, 0u, 0u, 0u);
  if (row >= rows || k0 >= cols) return v;
  if (!trans && vec && k0 + 8 <= cols) return __ldg(reinterpret_cast<const uint4*>(X + (size_t)row * ld + k0));
  uint16_t h[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const int k = k0 + q;
    h[q] = k < cols ? __bfloat16_as_ushort(trans ? X[(size_t)k * ld + row] : X[(size_t)row * ld + k]) : (uint16_t)0;
  }
  v.x = (uint32_t)h[0] | ((uint32_t)h[1] << 16);
  v.y = (uint32_t)h[2] | ((uint32_t)h[3] << 16);
  v.z = (uint32_t)h[4] | ((uint32_t)h[5] << 16);
  v.w = (uint32_t)h[6] | ((uint32_t)h[7] << 16);
  return v;
}

// Split K (blockIdx.z = split, kps chunks each): with `partial` set, CTA z
// writes its raw tile sums to partial[z] (M x N, leading dimension N) and a
// second kernel adds the splits in order; otherwise kps covers all chunks and
// the CTA writes alpha * acc + beta * C.
__global__ void __launch_bounds__(THREADS) gemm_tcgen05(int M, int N, int K, const __nv_bfloat16* __restrict__ A,
                                                        int lda, int ta, const __nv_bfloat16* __restrict__ B, int ldb,
                                                        int tb, float alpha, float beta, float* __restrict__ C,
                                                        int ldc, int kps, float* __restrict__ partial) {
  extern __shared__ unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t mma_done[STAGES];
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;
  unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  const int m0 = blockIdx.x * TM, n0 = blockIdx.y * TN;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mma_done[s])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    abort_flag = 0;
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  const bool vec_a = !ta && lda % 8 == 0 && (reinterpret_cast<uintptr_t>(A) & 15) == 0;
  const bool vec_b = tb && ldb % 8 == 0 && (reinterpret_cast<uintptr_t>(B) & 15) == 0;
  const int c_first = blockIdx.z * kps;
  const int nk = max(0, min((K + TK - 1) / TK - c_first, kps));  // this split's chunks
  int issued = 0;  // chunks whose MMAs were issued (thread 0)
  for (int c = 0; c < nk; ++c) {
    const int s = c % STAGES;
    // the stage is free once the MMAs of chunk c - STAGES, which read it, are done
    if (c >= STAGES && !wait_bounded(smem_u32(&mma_done[s]), (uint32_t)((c - STAGES) / STAGES) & 1u)) abort_flag = 1;
    __syncthreads();
    if (abort_flag) break;
    unsigned char* as = smem + s * STAGE_BYTES;
    unsigned char* bs = as + A_BYTES;
    const int k0 = (c_first + c) * TK;
    // piece p: row (p >> 6) * 8 + (p & 7), k-group (p >> 3) & 7, so consecutive
    // threads fill consecutive 16-byte slots of one core matrix
    for (int p = threadIdx.x; p < TM * (TK / 8); p += THREADS) {
      const int row = ((p >> 6) << 3) + (p & 7), kg = (p >> 3) & 7;
      *reinterpret_cast<uint4*>(as + core_offset(row, kg)) = load_piece(A, lda, ta, M, K, m0 + row, k0 + 8 * kg, vec_a);
      // op(B) is K x N: the tile's row n holds op(B)[k][n0 + n] along k
      *reinterpret_cast<uint4*>(bs + core_offset(row, kg)) =
          load_piece(B, ldb, !tb, N, K, n0 + row, k0 + 8 * kg, vec_b);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    if (threadIdx.x == 0) {
      tc_fence_after();
      const uint32_t a0 = smem_u32(as), b0 = smem_u32(bs);
#pragma unroll
      for (int kk = 0; kk < TK / 16; ++kk) {
        const uint64_t ad = smem_desc(a0 + kk * 256), bd = smem_desc(b0 + kk * 256);
        const uint32_t acc = (c > 0 || kk > 0) ? 1u : 0u;
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
            "l"(ad), "l"(bd), "r"(kInstrDesc), "r"(acc)
            : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(&mma_done[s]))
                   : "memory");
      issued = c + 1;
    }
  }
  // every thread waits for the last issued chunk's commit (it covers all earlier MMAs)
  __syncthreads();
  const int done_chunks = abort_flag ? -1 : nk;
  if (nk == 0 && threadIdx.x == 0) abort_flag = 1;  // an empty split (not launched by the host) writes nothing
  bool ok = true;
  if (done_chunks > 0) {
    const int last = nk - 1;
    ok = wait_bounded(smem_u32(&mma_done[last % STAGES]), (uint32_t)(last / STAGES) & 1u);
  } else if (threadIdx.x == 0 && issued > 0) {
    // aborted: wait (bounded) for the MMAs already issued before freeing TMEM
    wait_bounded(smem_u32(&mma_done[(issued - 1) % STAGES]), (uint32_t)((issued - 1) / STAGES) & 1u);
  }
  if (!ok) abort_flag = 1;
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (!abort_flag) {
    const int row = m0 + 32 * warp + lane;
    const uint32_t lane_base = tmem + ((uint32_t)(32 * warp) << 16);
#pragma unroll 1
    for (int cb = 0; cb < TN; cb += 16) {
      uint32_t r[16];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
          "%15}, [%16];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
            "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
          : "r"(lane_base + (uint32_t)cb));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (row < M && partial) {
        float* prow = partial + ((size_t)blockIdx.z * M + row) * N;
#pragma unroll
        for (int q = 0; q < 16; ++q)
          if (n0 + cb + q < N) prow[n0 + cb + q] = __uint_as_float(r[q]);
      } else if (row < M) {
        float* crow = C + (size_t)row * ldc;
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          const int col = n0 + cb + q;
          if (col < N) {
            const float v = alpha * __uint_as_float(r[q]);
            crow[col] = beta == 0.f ? v : v + beta * crow[col];
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
  }
}

// C = alpha * (sum of the splits' partial tiles, in split order) + beta * C.
__global__ void splitk_reduce(int M, int N, int splits, const float* __restrict__ partial, float alpha, float beta,
                              float* __restrict__ C, int ldc) {
  const size_t n = (size_t)M * N;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    float acc = partial[i];
    for (int z = 1; z < splits; ++z) acc += partial[(size_t)z * n + i];
    const size_t row = i / N, col = i - row * N;
    float* p = C + row * ldc + col;
    const float v = alpha * acc;
    *p = beta == 0.f ? v : v + beta * *p;
  }
}

// Splits of K for a product of `tiles` output tiles and nk chunks of 64: only
// when the tiles leave most SMs idle and K is long, at least 4 chunks per
// split, at most 2 CTAs per SM in total, within the workspace.
int choose_splits(int tiles, int nk, size_t mn, size_t workspace_bytes) {
  if (workspace_bytes == 0 || tiles >= 74 || nk < 8) return 1;
  int s = std::min(nk / 4, std::max(1, 296 / tiles));
  s = (int)std::min<size_t>((size_t)s, workspace_bytes / (mn * sizeof(float)));
  return std::max(1, s);
}

}  // namespace tc
}  // namespace ifdtd


// ---------------------------------------------------------------------------
// TMA-fed kernel for the K-major / K-major case (op(A) = A row-major M x K,
// op(B) = B^T with B row-major N x K: the forward products of the surrogate
// and square benchmark products).  Persistent: one CTA of 6 warps per SM
// walks 128 x 256 output tiles in grouped order.  Warp 0 (one lane) streams
// 64-wide K chunks of A (128 x 64) and B (256 x 64) with 2-D TMA tile loads
// (128-byte swizzle, zero fill outside the matrices) into a 4-stage ring,
// completing on the stage's "full" mbarrier by transaction count; warp 1 (one
// lane) waits on "full", issues four tcgen05.mma (M 128, N 256, K 16) per
// chunk and commits them to the stage's "empty" mbarrier, which frees the
// stage for the producer.  The accumulator alternates between two 256-column
// halves of the CTA's 512 TMEM columns: after a tile's last chunk the MMA lane
// commits to that half's "acc_full" barrier and goes on with the next tile in
// the other half, while warps 2-5 read the finished half with tcgen05.ld
// (each from the 32 TMEM lanes of its warp index modulo 4), write C and arrive
// on the half's "acc_empty" barrier.  Every wait is bounded as in the generic
// kernel; a wait that runs out sets the status bit and a stop flag, every role
// leaves its loop, and the CTA waits (bounded) for the MMAs it issued before it
// frees the tensor memory.  Loads read this GPU's memory only, without
// multicast.
// ---------------------------------------------------------------------------
namespace ifdtd {
namespace tc {

constexpr int XM = 128, XN = 256, XK = 64, XSTAGES = 4, XTHREADS = 192;
constexpr int XA_BYTES = XM * XK * 2, XB_BYTES = XN * XK * 2, XSTAGE = XA_BYTES + XB_BYTES;
constexpr int XSMEM = XSTAGES * XSTAGE + 1024;
constexpr uint32_t XTMEM_COLS = 512;  // two 256-column accumulators: a tile's epilogue overlaps the next tile's MMAs
constexpr int XGROUP = 8;              // tile rasterisation: M-tiles per group
// fp32 accumulator, bf16 A and B, both K-major, N 256, M 128
constexpr uint32_t kInstrDescX =
    (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(XN >> 3) << 17) | ((uint32_t)(XM >> 4) << 24);

// K-major operand with the 128-byte swizzle: rows of 128 bytes (64 bf16),
// 8-row groups 1024 bytes apart (stride byte offset), the leading byte offset
// unused (1), descriptor version 1, layout 2 (128-byte swizzle).  The K step of
// 16 elements inside the 128-byte atom advances the start address by 32 bytes.
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t addr) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024u >> 4) << 32) | ((uint64_t)1 << 46) |
         ((uint64_t)2 << 61);
}

__device__ __forceinline__ void mbar_init_x(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

// Output tile t of a tiles_m x tiles_n grid in grouped order: XGROUP M-tiles
// sweep each N column together, so the CTAs running at once share B panels
// (and A panels within a group) in L2.
__device__ __forceinline__ void tile_coords(int t, int tiles_m, int tiles_n, int& tm, int& tn) {
  const int per_group = XGROUP * tiles_n;
  const int g = t / per_group, first = g * XGROUP;
  const int rows = min(tiles_m - first, XGROUP);
  const int r = t - g * per_group;
  tm = first + r % rows;
  tn = r / rows;
}

__device__ __forceinline__ void mbar_arrive_x(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tc_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__global__ void __launch_bounds__(XTHREADS) gemm_tcgen05_tma(const __grid_constant__ CUtensorMap map_a,
                                                             const __grid_constant__ CUtensorMap map_b, int M, int N,
                                                             int K, float alpha, float beta, float* __restrict__ C,
                                                             int ldc, int tiles_m, int tiles_n) {
  extern __shared__ unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t full[XSTAGES], empty[XSTAGES], acc_full[2], acc_empty[2], drain;
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;
  unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nk = (K + XK - 1) / XK, n_tiles = tiles_m * tiles_n;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"(XTMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (threadIdx.x == 32) {
    for (int s = 0; s < XSTAGES; ++s) {
      mbar_init_x(smem_u32(&full[s]), 1);
      mbar_init_x(smem_u32(&empty[s]), 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init_x(smem_u32(&acc_full[b]), 1);
      mbar_init_x(smem_u32(&acc_empty[b]), 4);  // one arrival per epilogue warp
    }
    mbar_init_x(smem_u32(&drain), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    abort_flag = 0;
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  volatile int* stop = &abort_flag;
  if (warp == 0 && lane == 0) {
    // producer: every chunk of every tile of this CTA, through the ring
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&map_a)) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&map_b)) : "memory");
    int g = 0;
    for (int t = blockIdx.x; t < n_tiles && !*stop; t += gridDim.x) {
      int tm, tn;
      tile_coords(t, tiles_m, tiles_n, tm, tn);
      for (int c = 0; c < nk; ++c, ++g) {
        const int s = g % XSTAGES;
        if (g >= XSTAGES && !wait_bounded(smem_u32(&empty[s]), (uint32_t)((g - XSTAGES) / XSTAGES) & 1u)) *stop = 1;
        if (*stop) break;
        const uint32_t as = smem_u32(smem + s * XSTAGE), bs = as + XA_BYTES;
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(&full[s])), "r"(XSTAGE)
                     : "memory");
        tma_load_2d(as, &map_a, c * XK, tm * XM, smem_u32(&full[s]));
        tma_load_2d(bs, &map_b, c * XK, tn * XN, smem_u32(&full[s]));
      }
    }
  } else if (warp == 1 && lane == 0) {
    // MMA issuer: tile i accumulates in TMEM columns (i % 2) * 256
    int g = 0, i = 0;
    for (int t = blockIdx.x; t < n_tiles && !*stop; t += gridDim.x, ++i) {
      const int b = i & 1;
      if (i >= 2 && !wait_bounded(smem_u32(&acc_empty[b]), (uint32_t)((i - 2) / 2) & 1u)) *stop = 1;
      if (*stop) break;
      tc_fence_after();
      const uint32_t d = tmem + (uint32_t)(b * XN);
      for (int c = 0; c < nk; ++c, ++g) {
        const int s = g % XSTAGES;
        if (!wait_bounded(smem_u32(&full[s]), (uint32_t)(g / XSTAGES) & 1u)) *stop = 1;
        if (*stop) break;
        tc_fence_after();
        const uint32_t as = smem_u32(smem + s * XSTAGE), bs = as + XA_BYTES;
#pragma unroll
        for (int kk = 0; kk < XK / 16; ++kk) {
          const uint64_t ad = smem_desc_sw128(as + kk * 32), bd = smem_desc_sw128(bs + kk * 32);
          const uint32_t acc = (c > 0 || kk > 0) ? 1u : 0u;
          asm volatile(
              "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
              " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d),
              "l"(ad), "l"(bd), "r"(kInstrDescX), "r"(acc)
              : "memory");
        }
        tc_commit(smem_u32(&empty[s]));  // frees the stage once these MMAs are done
      }
      if (*stop) break;
      tc_commit(smem_u32(&acc_full[b]));  // the tile's accumulator is complete
    }
    // "drain" fires once every MMA this thread issued has completed (also after a stop)
    tc_commit(smem_u32(&drain));
  } else if (warp >= 2) {
    // epilogue: warp w reads TMEM lanes 32 (w % 4) .. 32 (w % 4) + 31
    const int quarter = warp & 3;
    int i = 0;
    for (int t = blockIdx.x; t < n_tiles; t += gridDim.x, ++i) {
      const int b = i & 1;
      if (!__all_sync(0xFFFFFFFFu, wait_bounded(smem_u32(&acc_full[b]), (uint32_t)(i / 2) & 1u))) {
        *stop = 1;
        break;
      }
      tc_fence_after();
      int tm, tn;
      tile_coords(t, tiles_m, tiles_n, tm, tn);
      const int row = tm * XM + 32 * quarter + lane, n0 = tn * XN;
      const uint32_t lane_base = tmem + ((uint32_t)(32 * quarter) << 16) + (uint32_t)(b * XN);
#pragma unroll 1
      for (int cb = 0; cb < XN; cb += 16) {
        uint32_t r[16];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
            "%15}, [%16];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
              "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
            : "r"(lane_base + (uint32_t)cb));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (row < M) {
          float* crow = C + (size_t)row * ldc;
#pragma unroll
          for (int q = 0; q < 16; ++q) {
            const int col = n0 + cb + q;
            if (col < N) {
              const float v = alpha * __uint_as_float(r[q]);
              crow[col] = beta == 0.f ? v : v + beta * crow[col];
            }
          }
        }
      }
      // the accumulator may be overwritten once all four warps have read it
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive_x(smem_u32(&acc_empty[b]));
    }
  }
  __syncwarp();
  // no MMA may still write TMEM when it is freed
  if (!wait_bounded(smem_u32(&drain), 0u)) *stop = 1;
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(XTMEM_COLS) : "memory");
  }
}

// 2-D tensor map of a row-major rows x K bf16 matrix with leading dimension
// ld, boxes of box_rows x 64 with the 128-byte swizzle (zero fill outside).
bool encode_kmajor(CUtensorMap* map, const void* base, int rows, int K, int ld, int box_rows) {
  static PFN_cuTensorMapEncodeTiled encode = nullptr;
  if (!encode) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn)
      return false;
    encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled>(fn);
  }
  const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  const cuuint32_t box[2] = {(cuuint32_t)XK, (cuuint32_t)box_rows};
  const cuuint32_t elem[2] = {1, 1};
  return encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, elem,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace tc
}  // namespace ifdtd

extern "C" {

int32_t ifdtd_nn_gemm_tc_ws(int32_t m, int32_t n, int32_t k, const void* a, int32_t lda, int32_t trans_a, const void* b,
                            int32_t ldb, int32_t trans_b, float alpha, float beta, float* c, int32_t ldc, void* workspace,
                            int64_t workspace_bytes, void* stream) {
  using namespace ifdtd::tc;
  if (m <= 0 || n <= 0 || k <= 0 || !a || !b || !c) return ifdtd::record_error(IFDTD_ERR_ARGUMENT, "bad gemm shape");
  if (lda < (trans_a ? m : k) || ldb < (trans_b ? k : n) || ldc < n)
    return ifdtd::record_error(IFDTD_ERR_ARGUMENT, "gemm leading dimension too small");
  if ((n + TN - 1) / TN > 65535) return ifdtd::record_error(IFDTD_ERR_ARGUMENT, "gemm has too many columns");
  if (workspace_bytes < 0 || (workspace_bytes > 0 && !workspace))
    return ifdtd::record_error(IFDTD_ERR_ARGUMENT, "bad gemm workspace");
  // the opt-in above 48 KiB of dynamic shared memory holds per device; setting it is cheap
  cudaError_t e = cudaFuncSetAttribute(gemm_tcgen05, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
  if (e != cudaSuccess) return ifdtd::record_error(IFDTD_ERR_CUDA, std::string("gemm_tcgen05 attribute: ") + cudaGetErrorString(e));
  // the TMA-fed kernel: both operands K-major (trans_a = 0, trans_b = 1), 16-byte aligned rows, and
  // enough output tiles to spread over the SMs
  const bool kmajor = !trans_a && trans_b && lda % 8 == 0 && ldb % 8 == 0 && k % 8 == 0 &&
                      (reinterpret_cast<uintptr_t>(a) & 15) == 0 && (reinterpret_cast<uintptr_t>(b) & 15) == 0;
  if (kmajor && (size_t)((m + XM - 1) / XM) * ((n + XN - 1) / XN) >= 32) {
    CUtensorMap ma, mb;
    if (encode_kmajor(&ma, a, m, k, lda, XM) && encode_kmajor(&mb, b, n, k, ldb, XN)) {
      e = cudaFuncSetAttribute(gemm_tcgen05_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, XSMEM);
      if (e != cudaSuccess)
        return ifdtd::record_error(IFDTD_ERR_CUDA, std::string("gemm_tcgen05_tma attribute: ") + cudaGetErrorString(e));
      int dev = 0, sms = 148;
      if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      const int tiles_m = (m + XM - 1) / XM, tiles_n = (n + XN - 1) / XN;
      // persistent: one CTA per SM (the ring takes 198 KB of shared memory), each walking its tiles
      const int grid = std::min(tiles_m * tiles_n, std::max(sms, 1));
      gemm_tcgen05_tma<<<grid, XTHREADS, XSMEM, (cudaStream_t)stream>>>(ma, mb, m, n, k, alpha, beta, c, ldc, tiles_m,
                                                                        tiles_n);
      e = cudaGetLastError();
      if (e != cudaSuccess) return ifdtd::record_error(IFDTD_ERR_CUDA, std::string("gemm_tcgen05_tma: ") + cudaGetErrorString(e));
      return IFDTD_OK;
    }
  }
  const int tm = (m + TM - 1) / TM, tn = (n + TN - 1) / TN, nk = (k + TK - 1) / TK;
  const int want = choose_splits(tm * tn, nk, (size_t)m * n, (size_t)workspace_bytes);
  const int kps = (nk + want - 1) / want, splits = (nk + kps - 1) / kps;
  cudaStream_t st = (cudaStream_t)stream;
  float* partial = splits > 1 ? static_cast<float*>(workspace) : nullptr;
  gemm_tcgen05<<<dim3(tm, tn, splits), THREADS, SMEM_BYTES, st>>>(m, n, k, (const __nv_bfloat16*)a, lda, trans_a != 0,
                                                                  (const __nv_bfloat16*)b, ldb, trans_b != 0, alpha,
                                                                  beta, c, ldc, kps, partial);
  e = cudaGetLastError();
  if (e != cudaSuccess) return ifdtd::record_error(IFDTD_ERR_CUDA, std::string("gemm_tcgen05: ") + cudaGetErrorString(e));
  if (partial) {
    const size_t mn = (size_t)m * n;
    const int blocks = (int)std::min<size_t>((mn + 255) / 256, 148 * 8);
    splitk_reduce<<<blocks, 256, 0, st>>>(m, n, splits, partial, alpha, beta, c, ldc);
    e = cudaGetLastError();
    if (e != cudaSuccess) return ifdtd::record_error(IFDTD_ERR_CUDA, std::string("splitk_reduce: ") + cudaGetErrorString(e));
  }
  return IFDTD_OK;
}

int32_t ifdtd_nn_gemm_tc(int32_t m, int32_t n, int32_t k, const void* a, int32_t lda, int32_t trans_a, const void* b,
                         int32_t ldb, int32_t trans_b, float alpha, float beta, float* c, int32_t ldc, void* stream) {
  return ifdtd_nn_gemm_tc_ws(m, n, k, a, lda, trans_a, b, ldb, trans_b, alpha, beta, c, ldc, nullptr, 0, stream);
}

int32_t ifdtd_nn_gemm_tc_status(int32_t reset, int32_t* out) {
  using namespace ifdtd::tc;
  int v = 0;
  cudaError_t e = cudaMemcpyFromSymbol(&v, g_status, sizeof(int));
  if (e == cudaSuccess && reset) {
    const int zero = 0;
    e = cudaMemcpyToSymbol(g_status, &zero, sizeof(int));
  }
  if (e != cudaSuccess) return ifdtd::record_error(IFDTD_ERR_CUDA, std::string("gemm status: ") + cudaGetErrorString(e));
  if (out) *out = v;
  return IFDTD_OK;
}

}  // extern "C"
