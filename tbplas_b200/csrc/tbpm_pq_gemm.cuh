// The Kubo-Bastin moment contraction of tbpm_kbdc (tbpm.f90:898-957) as one
// complex GEMM with split K:
//
//   cs[i][j] = sum_n conj(P[n, i]) * Q[n, j]      i < m (bra vectors of a chunk),
//                                                 j < nk (ket vectors), n < N
//
// P and Q are column-major N x m and N x nk (column i of P starts at P + i*N):
// both operands are contiguous along the reduction index, as in a "TN" GEMM.
// The reference forms these m*nk inner products one at a time (n_kernel^2
// serial dot products); here a grid of 64 x 64 output tiles and S slices of
// the N rows each accumulate their share in registers.
//
// pq_gemm_kernel: 256 threads, output tile 64 (i) x 64 (j), 16 rows of n per
// step staged in shared memory (row length padded to 65 complex values, so the
// transposing stores and the broadcast reads are free of bank conflicts).
// Thread (tx, ty) owns outputs i = ty + 16a, j = tx + 16b (a, b < 4): per step
// it reads 4 + 4 staged values and does 16 complex FMAs.  The next step's
// loads are issued into registers before the current step is computed.  The
// block writes its slice's partial tile to ws[slice][j][i] (FP64).
//
// pq_reduce_kernel sums the slices in a fixed order and adds
// g_i g_j * scale * cs[i][j] to mu[i0 + i + nk*j] (FP64), so results are
// deterministic.  FP32 operands accumulate in FP32 within a slice and in FP64
// across slices.
#pragma once

#include "tbpm_common.cuh"

namespace tbpm {

constexpr int kPqTile = 64;
constexpr int kPqK = 16;
constexpr int kPqPad = kPqTile + 1;

template <typename R>
__global__ void __launch_bounds__(256) pq_gemm_kernel(const typename Cx<R>::t* __restrict__ P,
                                                      const typename Cx<R>::t* __restrict__ Q,
                                                      int64_t N, int m, int nk, int64_t rows_per_slice,
                                                      double2* __restrict__ ws) {
  using C = typename Cx<R>::t;
  __shared__ C sP[kPqK][kPqPad];
  __shared__ C sQ[kPqK][kPqPad];
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;
  const int j0 = blockIdx.x * kPqTile, i0 = blockIdx.y * kPqTile;
  const int slice = blockIdx.z;
  const int64_t n_lo = (int64_t)slice * rows_per_slice;
  const int64_t n_hi = n_lo + rows_per_slice < N ? n_lo + rows_per_slice : N;
  // loader mapping: row k = tid & 15 of the step, columns (tid >> 4) + 16q
  const int lk = tid & 15, lc = tid >> 4;
  R acc_re[4][4], acc_im[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc_re[a][b] = acc_im[a][b] = (R)0;
  C pr[4], qr[4];
  auto load = [&](int64_t n0) {
    const int64_t n = n0 + lk;
    const bool in = n < n_hi;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int i = i0 + lc + 16 * q, j = j0 + lc + 16 * q;
      C zero;
      zero.x = zero.y = (R)0;
      pr[q] = (in && i < m) ? P[(int64_t)i * N + n] : zero;
      qr[q] = (in && j < nk) ? Q[(int64_t)j * N + n] : zero;
    }
  };
  if (n_lo < n_hi) load(n_lo);
  for (int64_t n0 = n_lo; n0 < n_hi; n0 += kPqK) {
    __syncthreads();  // the previous step's reads are done
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      sP[lk][lc + 16 * q] = pr[q];
      sQ[lk][lc + 16 * q] = qr[q];
    }
    __syncthreads();
    if (n0 + kPqK < n_hi) load(n0 + kPqK);  // in flight during the step
#pragma unroll
    for (int k = 0; k < kPqK; ++k) {
      C p[4], q[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) p[a] = sP[k][ty + 16 * a];
#pragma unroll
      for (int b = 0; b < 4; ++b) q[b] = sQ[k][tx + 16 * b];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          // conj(p) * q
          acc_re[a][b] = fma(p[a].x, q[b].x, fma(p[a].y, q[b].y, acc_re[a][b]));
          acc_im[a][b] = fma(p[a].x, q[b].y, fma(-p[a].y, q[b].x, acc_im[a][b]));
        }
    }
  }
  double2* out = ws + (int64_t)slice * m * nk;
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int i = i0 + ty + 16 * a, j = j0 + tx + 16 * b;
      if (i < m && j < nk)
        out[(int64_t)j * m + i] = make_double2((double)acc_re[a][b], (double)acc_im[a][b]);
    }
}

// mu[(i0 + i) + nk*j] += g[i0+i] g[j] * scale * sum_s ws[s][j][i]
__global__ void pq_reduce_kernel(const double2* __restrict__ ws, int slices, int m, int nk,
                                 int i0, const double* __restrict__ g, double scale,
                                 double2* __restrict__ mu) {
  const int64_t total = (int64_t)m * nk;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    double re = 0.0, im = 0.0;
    for (int s = 0; s < slices; ++s) {
      const double2 v = ws[(int64_t)s * total + e];
      re += v.x;
      im += v.y;
    }
    const int ii = (int)(e % m);
    const int j = (int)(e / m);
    const int i = i0 + ii;
    const double w = g[i] * g[j];
    double2& o = mu[(int64_t)i + (int64_t)nk * j];
    o.x += w * re * scale;
    o.y += w * im * scale;
  }
}

}  // namespace tbpm
