// BF16 kernels of the learned C(t) tail extrapolator (training and inference),
// FP32 accumulation.  Device-pointer C ABI (include/tbpm_b200.h, tbpm_nn_*);
// the caller owns all buffers and the stream.
//
//  gemm_tn_bf16_kernel  C[M,N] = alpha * A[M,K] . B[N,K]^T + beta * C  (A, B
//                       BF16 with K contiguous, C FP32) through mma.sync
//                       m16n8k16, 128x128x32 block tiles, cp.async double
//                       buffering, ldmatrix fragments: tbpm_nn_gemm_tn_mma, an
//                       independent implementation kept to check the tcgen05
//                       GEMM (tbpm_nn_tc.cu) that the network uses.  Every
//                       dense/convolution product of the network (forward, data
//                       gradient, weight gradient) is this GEMM after an im2col
//                       or a transpose.
//  im2col / col2im      1-D convolution <-> GEMM reshaping, channel-last [B][L][C]
//  bias_act / act_back  bias + GELU (exact erf form) and its derivative
//  colsum, mse, adam, cast, transpose
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "tbpm_b200.h"

namespace {

constexpr int BM = 128, BN = 128, BK = 32, PAD = 8;  // smem row = 40 bf16 = 80 B
constexpr int LDS = BK + PAD;

__device__ __forceinline__ void cp_async_16(void* smem, const void* gmem, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int n = valid ? 16 : 0;  // zero-fill when out of range
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}

__device__ __forceinline__ void ldmatrix_x4(unsigned& r0, unsigned& r1, unsigned& r2,
                                            unsigned& r3, const void* smem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(s));
}

__device__ __forceinline__ void mma_bf16(float* d, const unsigned* a, const unsigned* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// 256 threads = 8 warps as 2 (M) x 4 (N); warp tile 64 x 32.
__global__ void __launch_bounds__(256) gemm_tn_bf16_kernel(const __nv_bfloat16* __restrict__ A,
                                                           int lda,
                                                           const __nv_bfloat16* __restrict__ B,
                                                           int ldb, float* __restrict__ C,
                                                           int ldc, int M, int N, int K,
                                                           float alpha, float beta) {
  __shared__ __align__(16) __nv_bfloat16 As[2][BM][LDS];
  __shared__ __align__(16) __nv_bfloat16 Bs[2][BN][LDS];
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int wm = warp >> 2, wn = warp & 3;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  float acc[4][4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.f;

  auto load_stage = [&](int stage, int k0) {
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int c = tid + i * 256;  // 512 chunks of 16 B per operand tile
      const int row = c >> 2, kc = (c & 3) * 8;
      const int gk = k0 + kc;
      const int gm = m0 + row, gn = n0 + row;
      const bool va = gm < M && gk < K;
      const bool vb = gn < N && gk < K;
      cp_async_16(&As[stage][row][kc], va ? (const void*)(A + (int64_t)gm * lda + gk) : (const void*)A, va);
      cp_async_16(&Bs[stage][row][kc], vb ? (const void*)(B + (int64_t)gn * ldb + gk) : (const void*)B, vb);
    }
    asm volatile("cp.async.commit_group;\n" ::);
  };

  const int kt_n = (K + BK - 1) / BK;
  load_stage(0, 0);
  for (int kt = 0; kt < kt_n; ++kt) {
    const int st = kt & 1;
    if (kt + 1 < kt_n) {
      load_stage(st ^ 1, (kt + 1) * BK);
      asm volatile("cp.async.wait_group 1;\n" ::);
    } else {
      asm volatile("cp.async.wait_group 0;\n" ::);
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; kk += 16) {
      unsigned af[4][4], bf[4][2];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int r = wm * 64 + i * 16 + (lane & 15);
        const int k = kk + (lane >> 4) * 8;
        ldmatrix_x4(af[i][0], af[i][1], af[i][2], af[i][3], &As[st][r][k]);
      }
#pragma unroll
      for (int j = 0; j < 4; j += 2) {
        const int q = lane >> 3, r8 = lane & 7;
        const int n = wn * 32 + j * 8 + (q >> 1) * 8 + r8;
        const int k = kk + (q & 1) * 8;
        unsigned x0, x1, x2, x3;
        ldmatrix_x4(x0, x1, x2, x3, &Bs[st][n][k]);
        bf[j][0] = x0;
        bf[j][1] = x1;
        bf[j + 1][0] = x2;
        bf[j + 1][1] = x3;
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) mma_bf16(acc[i][j], af[i], bf[j]);
    }
    __syncthreads();
  }
  // epilogue
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int row = m0 + wm * 64 + i * 16 + (lane >> 2) + h * 8;
        const int col = n0 + wn * 32 + j * 8 + (lane & 3) * 2;
        if (row < M) {
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            if (col + e < N) {
              float* p = C + (int64_t)row * ldc + col + e;
              const float v = alpha * acc[i][j][h * 2 + e];
              *p = beta == 0.f ? v : v + beta * *p;
            }
          }
        }
      }
}

__global__ void transpose_bf16_kernel(const __nv_bfloat16* in, int rows, int cols,
                                      __nv_bfloat16* out) {
  __shared__ __nv_bfloat16 tile[32][33];
  const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
  for (int y = threadIdx.y; y < 32; y += blockDim.y) {
    const int r = by + y, c = bx + threadIdx.x;
    if (r < rows && c < cols) tile[y][threadIdx.x] = in[(int64_t)r * cols + c];
  }
  __syncthreads();
  for (int y = threadIdx.y; y < 32; y += blockDim.y) {
    const int c = bx + y, r = by + threadIdx.x;
    if (c < cols && r < rows) out[(int64_t)c * rows + r] = tile[threadIdx.x][y];
  }
}

// Xcol[(b*Lout + lo)][j*C + c] = X[b][lo*s + j - p][c] (0 outside)
__global__ void im2col_kernel(const __nv_bfloat16* X, int Bn, int L, int C, int k, int s, int p,
                              int Lout, __nv_bfloat16* Xcol) {
  const int64_t total = (int64_t)Bn * Lout * k * C;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(g % C);
    int64_t t = g / C;
    const int j = (int)(t % k);
    t /= k;
    const int lo = (int)(t % Lout);
    const int b = (int)(t / Lout);
    const int l = lo * s + j - p;
    Xcol[g] = (l >= 0 && l < L) ? X[((int64_t)b * L + l) * C + c] : __float2bfloat16(0.f);
  }
}

// dX[b][l][c] = sum over (lo, j) with lo*s + j - p = l of dXcol[(b*Lout+lo)][j*C + c]
__global__ void col2im_kernel(const float* dXcol, int Bn, int L, int C, int k, int s, int p,
                              int Lout, float* dX) {
  const int64_t total = (int64_t)Bn * L * C;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(g % C);
    const int64_t t = g / C;
    const int l = (int)(t % L);
    const int b = (int)(t / L);
    float acc = 0.f;
    for (int j = 0; j < k; ++j) {
      const int num = l + p - j;
      if (num < 0 || num % s) continue;
      const int lo = num / s;
      if (lo >= Lout) continue;
      acc += dXcol[((int64_t)b * Lout + lo) * ((int64_t)k * C) + (int64_t)j * C + c];
    }
    dX[g] = acc;
  }
}

__device__ __forceinline__ float gelu(float x) {
  return 0.5f * x * (1.f + erff(x * 0.70710678118654752f));
}
__device__ __forceinline__ float gelu_grad(float x) {
  const float cdf = 0.5f * (1.f + erff(x * 0.70710678118654752f));
  const float pdf = 0.39894228040143268f * __expf(-0.5f * x * x);
  return cdf + x * pdf;
}

__global__ void bias_act_kernel(const float* Z, const float* bias, int M, int N, int act,
                                float* pre, __nv_bfloat16* out_bf16, float* out_f32) {
  const int64_t total = (int64_t)M * N;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (int64_t)gridDim.x * blockDim.x) {
    const float z = Z[g] + (bias ? bias[g % N] : 0.f);
    if (pre) pre[g] = z;
    const float a = act == 1 ? gelu(z) : z;
    if (out_bf16) out_bf16[g] = __float2bfloat16(a);
    if (out_f32) out_f32[g] = a;
  }
}

__global__ void act_backward_kernel(const float* dA, const float* pre, int64_t total, int act,
                                    float* dZ, __nv_bfloat16* dZ_bf16) {
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (int64_t)gridDim.x * blockDim.x) {
    const float d = act == 1 ? dA[g] * gelu_grad(pre[g]) : dA[g];
    if (dZ) dZ[g] = d;
    if (dZ_bf16) dZ_bf16[g] = __float2bfloat16(d);
  }
}

// out[n] = sum_m Z[m][n] (fixed order per column)
__global__ void colsum_kernel(const float* Z, int M, int N, float* out) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  float s = 0.f;
  for (int m = 0; m < M; ++m) s += Z[(int64_t)m * N + n];
  out[n] = s;
}

// grad = 2 (pred - target) / (M N); partial squared errors per block
__global__ void mse_kernel(const float* pred, const float* target, int64_t total, float* grad,
                           double* block_sums) {
  __shared__ double red[256];
  double s = 0.0;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (int64_t)gridDim.x * blockDim.x) {
    const float d = pred[g] - target[g];
    if (grad) grad[g] = 2.f * d / (float)total;
    s += (double)d * d;
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) block_sums[blockIdx.x] = red[0];
}

__global__ void mse_finalize_kernel(const double* block_sums, int n_blocks, int64_t total,
                                    double* loss) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0.0;
    for (int i = 0; i < n_blocks; ++i) s += block_sums[i];
    *loss = s / (double)total;
  }
}

// AdamW (decoupled weight decay) on FP32 master weights; optional BF16 copy.
__global__ void adam_kernel(float* w, const float* g, float* m, float* v, int64_t n, float lr,
                            float b1, float b2, float eps, float wd, float bc1, float bc2,
                            __nv_bfloat16* w_bf16) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    float wi = w[i] * (1.f - lr * wd);
    wi -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
    w[i] = wi;
    if (w_bf16) w_bf16[i] = __float2bfloat16(wi);
  }
}

__global__ void cast_bf16_kernel(const float* in, int64_t n, __nv_bfloat16* out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = __float2bfloat16(in[i]);
}

int grid_1d(int64_t n) {
  const int64_t b = (n + 255) / 256;
  return (int)(b < 65535 * 8 ? (b < 1 ? 1 : b) : 65535 * 8);
}

int status(cudaError_t e) {
  if (e == cudaSuccess) return TBPM_OK;
  (void)cudaGetLastError();
  return TBPM_ERR_CUDA;
}

}  // namespace

extern "C" {

int tbpm_nn_gemm_tn_mma(const void* A, int lda, const void* B, int ldb, float* C, int ldc,
                        int M, int N, int K, float alpha, float beta, void* stream) {
  if (!A || !B || !C || M < 1 || N < 1 || K < 1 || K % 8 || lda % 8 || ldb % 8 || lda < K ||
      ldb < K || ldc < N)
    return TBPM_ERR_ARG;
  if ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B)) & 15) return TBPM_ERR_ARG;
  const dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM);
  gemm_tn_bf16_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(
      (const __nv_bfloat16*)A, lda, (const __nv_bfloat16*)B, ldb, C, ldc, M, N, K, alpha, beta);
  return status(cudaGetLastError());
}

int tbpm_nn_transpose_bf16(const void* in, int rows, int cols, void* out, void* stream) {
  if (!in || !out || rows < 1 || cols < 1) return TBPM_ERR_ARG;
  const dim3 grid((cols + 31) / 32, (rows + 31) / 32), block(32, 8);
  transpose_bf16_kernel<<<grid, block, 0, (cudaStream_t)stream>>>(
      (const __nv_bfloat16*)in, rows, cols, (__nv_bfloat16*)out);
  return status(cudaGetLastError());
}

int tbpm_nn_im2col(const void* X, int batch, int L, int C, int k, int s, int p, int Lout,
                   void* Xcol, void* stream) {
  if (!X || !Xcol || batch < 1 || L < 1 || C < 1 || k < 1 || s < 1 || p < 0 || Lout < 1)
    return TBPM_ERR_ARG;
  const int64_t total = (int64_t)batch * Lout * k * C;
  im2col_kernel<<<grid_1d(total), 256, 0, (cudaStream_t)stream>>>(
      (const __nv_bfloat16*)X, batch, L, C, k, s, p, Lout, (__nv_bfloat16*)Xcol);
  return status(cudaGetLastError());
}

int tbpm_nn_col2im(const float* dXcol, int batch, int L, int C, int k, int s, int p, int Lout,
                   float* dX, void* stream) {
  if (!dXcol || !dX || batch < 1 || L < 1 || C < 1 || k < 1 || s < 1 || p < 0 || Lout < 1)
    return TBPM_ERR_ARG;
  const int64_t total = (int64_t)batch * L * C;
  col2im_kernel<<<grid_1d(total), 256, 0, (cudaStream_t)stream>>>(dXcol, batch, L, C, k, s, p,
                                                                    Lout, dX);
  return status(cudaGetLastError());
}

int tbpm_nn_bias_act(const float* Z, const float* bias, int M, int N, int act, float* pre,
                     void* out_bf16, float* out_f32, void* stream) {
  if (!Z || M < 1 || N < 1 || act < 0 || act > 1) return TBPM_ERR_ARG;
  bias_act_kernel<<<grid_1d((int64_t)M * N), 256, 0, (cudaStream_t)stream>>>(
      Z, bias, M, N, act, pre, (__nv_bfloat16*)out_bf16, out_f32);
  return status(cudaGetLastError());
}

int tbpm_nn_act_backward(const float* dA, const float* pre, int64_t n, int act, float* dZ,
                         void* dZ_bf16, void* stream) {
  if (!dA || (act == 1 && !pre) || n < 1) return TBPM_ERR_ARG;
  act_backward_kernel<<<grid_1d(n), 256, 0, (cudaStream_t)stream>>>(dA, pre, n, act, dZ,
                                                                     (__nv_bfloat16*)dZ_bf16);
  return status(cudaGetLastError());
}

int tbpm_nn_colsum(const float* Z, int M, int N, float* out, void* stream) {
  if (!Z || !out || M < 1 || N < 1) return TBPM_ERR_ARG;
  colsum_kernel<<<(N + 255) / 256, 256, 0, (cudaStream_t)stream>>>(Z, M, N, out);
  return status(cudaGetLastError());
}

// loss (device double) = mean (pred - target)^2; grad (optional) = d loss / d pred.
// work: device scratch of at least 256 doubles.
int tbpm_nn_mse(const float* pred, const float* target, int64_t n, float* grad, double* work,
                double* loss, void* stream) {
  if (!pred || !target || !work || !loss || n < 1) return TBPM_ERR_ARG;
  const int nb = (int)((n + 255) / 256 < 256 ? (n + 255) / 256 : 256);
  mse_kernel<<<nb, 256, 0, (cudaStream_t)stream>>>(pred, target, n, grad, work);
  mse_finalize_kernel<<<1, 32, 0, (cudaStream_t)stream>>>(work, nb, n, loss);
  return status(cudaGetLastError());
}

int tbpm_nn_adam(float* w, const float* g, float* m, float* v, int64_t n, float lr, float b1,
                 float b2, float eps, float weight_decay, int step, void* w_bf16, void* stream) {
  if (!w || !g || !m || !v || n < 1 || step < 1) return TBPM_ERR_ARG;
  float bc1 = 1.f, bc2 = 1.f;
  for (int i = 0; i < step && i < 100000; ++i) {
    bc1 *= b1;
    bc2 *= b2;
  }
  bc1 = 1.f - bc1;
  bc2 = 1.f - bc2;
  adam_kernel<<<grid_1d(n), 256, 0, (cudaStream_t)stream>>>(w, g, m, v, n, lr, b1, b2, eps,
                                                            weight_decay, bc1, bc2,
                                                            (__nv_bfloat16*)w_bf16);
  return status(cudaGetLastError());
}

int tbpm_nn_cast_bf16(const float* in, int64_t n, void* out, void* stream) {
  if (!in || !out || n < 1) return TBPM_ERR_ARG;
  cast_bf16_kernel<<<grid_1d(n), 256, 0, (cudaStream_t)stream>>>(in, n, (__nv_bfloat16*)out);
  return status(cudaGetLastError());
}

}  // extern "C"
