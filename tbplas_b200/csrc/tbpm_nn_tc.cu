// tcgen05 (5th-generation tensor core) GEMM of the learned C(t) tail network:
//   C[M,N] = alpha * A[M,K] . B[N,K]^T + beta * C     (A, B BF16, K contiguous; C FP32)
//
// One CTA computes a 128 x 256 tile of C with 128 threads (4 warps), warp
// specialised:
//  * warp 0 (one lane) is the TMA producer: a 4-stage ring of shared-memory
//    stages, each a 128 x 64 tile of A and a 256 x 64 tile of B brought by
//    cp.async.bulk.tensor with the 128-byte swizzle; a `full` mbarrier per
//    stage carries the byte count, an `empty` mbarrier tells when the tensor
//    core has read the stage;
//  * warp 1 (one lane) issues tcgen05.mma (kind::f16: BF16 in, FP32
//    accumulate, M = 128, N = 256, K = 16 per instruction) and a
//    tcgen05.commit per stage that arrives on its `empty` barrier;
//  * the 128 x 256 FP32 accumulator lives in tensor memory (256 columns
//    allocated by warp 0);
//  * epilogue (all warps): each warp reads its 32 TMEM lanes (rows) with
//    tcgen05.ld, transposes 32 x 32 blocks through shared memory and writes
//    alpha * acc + beta * C one contiguous 128-byte row segment per store.
// Every mbarrier wait is bounded.  When a bound runs out the kernel records
// the failure in g_tc_status, stops issuing work, waits (bounded) for its
// copies in flight, frees its TMEM and returns; tbpm_nn_tc_status() reports
// it to the host.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <stdint.h>

#include <mutex>

#include "tbpm_b200.h"

namespace {

constexpr int TM = 128, TN = 256, TK = 64;  // CTA tile; TK * 2 B = one 128-byte swizzle row
constexpr int STAGES = 4;
constexpr int STAGE_A = TM * TK * 2;  // 16 KB
constexpr int STAGE_B = TN * TK * 2;  // 32 KB
constexpr int SMEM_BYTES = STAGES * (STAGE_A + STAGE_B) + 1024 + 256;
constexpr unsigned long long kWaitLimit = 1ull << 22;  // try_wait rounds per wait

__device__ int g_tc_status = 0;  // 0 ok, 1 a bounded wait ran out

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// true when the phase with the given parity has completed; gives up after
// kWaitLimit rounds
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (unsigned long long i = 0; i < kWaitLimit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// Shared-memory matrix descriptor of a K-major tile written by TMA with the
// 128-byte swizzle: rows of 128 B, 8-row groups 1024 B apart.
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);           // start address
  d |= (uint64_t)1 << 16;                           // leading byte offset (unused here)
  d |= (uint64_t)((1024 >> 4) & 0x3FFF) << 32;     // stride byte offset
  d |= (uint64_t)1 << 46;                           // descriptor version
  d |= (uint64_t)2 << 61;                           // 128-byte swizzle
  return d;
}

// Instruction descriptor: D F32, A and B BF16, both K-major, M = 128, N = 256.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TN >> 3) << 17) |
                            ((uint32_t)(TM >> 4) << 24);

__device__ __forceinline__ void mma_bf16_tc(uint32_t tmem_d, uint64_t a, uint64_t b,
                                            uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(bar))
      : "memory");
}

__global__ void __launch_bounds__(128, 1)
    gemm_tn_bf16_tc_kernel(const __grid_constant__ CUtensorMap map_a,
                           const __grid_constant__ CUtensorMap map_b, float* __restrict__ C,
                           int ldc, int M, int N, int K, float alpha, float beta) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // 1024-byte aligned stage buffers (the swizzle atom), then the barriers
  unsigned char* base = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  unsigned char* sa = base;
  unsigned char* sb = base + STAGES * STAGE_A;
  uint64_t* full = reinterpret_cast<uint64_t*>(sb + STAGES * STAGE_B);
  uint64_t* empty = full + STAGES;
  uint64_t* done = empty + STAGES;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  __shared__ int failed;
  __shared__ int issued;  // k-tiles whose loads were issued

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.y * TM, n0 = blockIdx.x * TN;
  const int kt_n = (K + TK - 1) / TK;

  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
    failed = 0;
    issued = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile(
        "tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 256;" ::"r"(
            smem_u32(tmem_slot))
        : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // TMA producer
    for (int kt = 0; kt < kt_n; ++kt) {
      const int s = kt % STAGES;
      if (kt >= STAGES && !mbar_wait(&empty[s], ((kt / STAGES) - 1) & 1)) {
        failed = 1;
        break;
      }
      if (*(volatile int*)&failed) break;
      mbar_expect_tx(&full[s], STAGE_A + STAGE_B);
      tma_load_2d(sa + s * STAGE_A, &map_a, kt * TK, m0, &full[s]);
      tma_load_2d(sb + s * STAGE_B, &map_b, kt * TK, n0, &full[s]);
      issued = kt + 1;
    }
  } else if (warp == 1 && lane == 0) {
    // MMA issuer
    bool ok = true;
    for (int kt = 0; kt < kt_n; ++kt) {
      const int s = kt % STAGES;
      if (!mbar_wait(&full[s], (kt / STAGES) & 1)) {
        ok = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a0 = smem_u32(sa + s * STAGE_A), b0 = smem_u32(sb + s * STAGE_B);
#pragma unroll
      for (int k = 0; k < TK / 16; ++k)
        mma_bf16_tc(tmem, smem_desc_sw128(a0 + 32 * k), smem_desc_sw128(b0 + 32 * k),
                    (kt > 0 || k > 0) ? 1u : 0u);
      mma_commit(&empty[s]);
    }
    // committed on failure too: `done` then tracks every MMA already issued,
    // so the CTA never frees its tensor memory under a running MMA
    mma_commit(done);
    if (!ok) failed = 1;
  }
  __syncthreads();
  bool good = !failed;
  if (!mbar_wait(done, 0)) good = false;
  if (!good) {
    if (tid == 0) {
      atomicExch(&g_tc_status, 1);
      // let the copies already issued land before the CTA's memory goes away
      const int n_iss = issued;
      for (int kt = n_iss - STAGES > 0 ? n_iss - STAGES : 0; kt < n_iss; ++kt)
        (void)mbar_wait(&full[kt % STAGES], (kt / STAGES) & 1);
    }
  } else {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // the stage buffers are free now: 32 x 33 floats per warp for the transpose
    float* tile = reinterpret_cast<float*>(base) + warp * 32 * 33;
    for (int c0 = 0; c0 < TN; c0 += 32) {
      if (n0 + c0 >= N) break;
      uint32_t v[32];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,"
          "%12,%13,%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,"
          "%31}, [%32];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
            "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
            "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]),
            "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
            "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]),
            "=r"(v[30]), "=r"(v[31])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      // lane holds row (warp*32 + lane), columns c0..c0+31: transpose so that
      // each store of the warp covers one row's 32 consecutive columns
#pragma unroll
      for (int j = 0; j < 32; ++j) tile[lane * 33 + j] = __uint_as_float(v[j]);
      __syncwarp();
      const int col = n0 + c0 + lane;
      for (int j = 0; j < 32; ++j) {
        const int row = m0 + warp * 32 + j;
        if (row < M && col < N) {
          float* p = C + (int64_t)row * ldc + col;
          const float x = alpha * tile[j * 33 + lane];
          *p = beta == 0.f ? x : x + beta * *p;
        }
      }
      __syncwarp();
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 256;" ::"r"(tmem)
                 : "memory");
  }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    (void)cudaGetLastError();
  });
  return fn;
}

// rows x K BF16 operand with row stride ld elements, box_rows x 64 boxes, 128-byte swizzle
bool make_map(CUtensorMap* map, const void* ptr, int rows, int K, int ld, int box_rows) {
  auto fn = encode_fn();
  if (!fn) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  const cuuint32_t box[2] = {(cuuint32_t)TK, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1, 1};
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims, strides,
            box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

}  // namespace

extern "C" {

int tbpm_nn_gemm_tn(const void* A, int lda, const void* B, int ldb, float* C, int ldc,
                       int M, int N, int K, float alpha, float beta, void* stream) {
  if (!A || !B || !C || M < 1 || N < 1 || K < 1 || K % 8 || lda % 8 || ldb % 8 || lda < K ||
      ldb < K || ldc < N)
    return TBPM_ERR_ARG;
  if ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B)) & 15) return TBPM_ERR_ARG;
  CUtensorMap ma, mb;
  if (!make_map(&ma, A, M, K, lda, TM) || !make_map(&mb, B, N, K, ldb, TN)) return TBPM_ERR_CUDA;
  if (cudaFuncSetAttribute(gemm_tn_bf16_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           SMEM_BYTES) != cudaSuccess)
    return TBPM_ERR_CUDA;
  const dim3 grid((N + TN - 1) / TN, (M + TM - 1) / TM);
  gemm_tn_bf16_tc_kernel<<<grid, 128, SMEM_BYTES, (cudaStream_t)stream>>>(ma, mb, C, ldc, M, N,
                                                                          K, alpha, beta);
  return cudaGetLastError() == cudaSuccess ? TBPM_OK : TBPM_ERR_CUDA;
}

int tbpm_nn_tc_status(int* failed) {
  if (!failed) return TBPM_ERR_ARG;
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, g_tc_status, sizeof(int)) != cudaSuccess) return TBPM_ERR_CUDA;
  *failed = v;
  const int zero = 0;
  if (cudaMemcpyToSymbol(g_tc_status, &zero, sizeof(int)) != cudaSuccess) return TBPM_ERR_CUDA;
  return TBPM_OK;
}

}  // extern "C"
