// Segmented kernels for batches of uneven realisations packed into one
// block-diagonal Hamiltonian: segment k owns rows [seg_off[k], seg_off[k+1]).
// Each realisation has its own n_s random states (normalised over its own
// rows) and its own correlation function; all of them are propagated by the
// same Chebyshev-term launches.
//
// Launch shape: grid (n_chunks, n_seg), 256 threads; block (chunk, seg) owns a
// contiguous chunk of rows_per_chunk rows of segment seg, so every partial sum
// has a fixed owner and the reductions are deterministic.
#pragma once

#include "tbpm_kernels.cuh"

namespace tbpm {

// Fixed-order reduction of per-thread values over the row slots of a block
// (rpp slots x ns columns x nv values), then one partial per (column, value).
__device__ __forceinline__ void seg_block_reduce(double* smem, const double* vals, int nv,
                                                 int slot, int col, int rpp, int ns) {
  const int width = ns * nv;
  for (int q = 0; q < nv; ++q) smem[slot * width + col * nv + q] = vals[q];
  __syncthreads();
  tree_reduce_slots(smem, rpp, width, slot, col, ns);
}

// mode 0: partial sums of |z|^2 per (segment, column);
// mode 1: write z / sqrt(sum[segment*ns + column]) (random.f90:36-69 per
// realisation; key iseed*49741 with iseed = seed*(seg*ns + col + 1); counter =
// row index inside the segment).
template <typename R>
__global__ void __launch_bounds__(256) seg_state_kernel(const int64_t* seg_off, int ns,
                                                        long long seed, int kind,
                                                        int64_t rows_per_chunk, int mode,
                                                        const double* sums,
                                                        typename Cx<R>::t* out,
                                                        double* partials) {
  __shared__ double smem[256];
  const int seg = blockIdx.y;
  const int slot = threadIdx.x / ns;
  const int col = threadIdx.x - slot * ns;
  const int rpp = blockDim.x / ns;
  const int64_t s0 = seg_off[seg], s1 = seg_off[seg + 1];
  const int64_t c0 = s0 + (int64_t)blockIdx.x * rows_per_chunk;
  const int64_t c1 = min(c0 + rows_per_chunk, s1);
  const long long key = seed * ((long long)seg * ns + col + 1) * 49741LL;
  const double two_pi = 6.283185307179586476925286766559;
  const double den = mode == 1 ? sqrt(sums[(int64_t)seg * ns + col]) : 1.0;
  double acc = 0.0;
  if (slot < rpp) {
    for (int64_t r = c0 + slot; r < c1; r += rpp) {
      double f, g;
      philox_uniform_pair(key, r - s0, &f, &g);
      const double az2 = kind == 0 ? -1.0 * log(1.0 - f) : 1.0;
      if (mode == 0) {
        acc += az2;
      } else {
        double sn, cs;
        sincos(two_pi * g, &sn, &cs);
        const double m = sqrt(az2);
        typename Cx<R>::t o;
        o.x = (R)((m * cs) / den);
        o.y = (R)((m * sn) / den);
        out[r * ns + col] = o;
      }
    }
  }
  if (mode == 0) {
    seg_block_reduce(smem, &acc, 1, slot, col, rpp, ns);
    if (slot == 0)
      partials[((int64_t)seg * ns + col) * gridDim.x + blockIdx.x] = smem[col];
  }
}

// <ref|x> and <x|x> per (segment, column): partials[((seg*ns + col)*3 + q)*n_chunks + chunk]
template <typename R>
__global__ void __launch_bounds__(256) seg_corr_kernel(const int64_t* seg_off, int ns,
                                                       int64_t rows_per_chunk,
                                                       const typename Cx<R>::t* x,
                                                       const typename Cx<R>::t* ref,
                                                       double* partials) {
  __shared__ double smem[256 * 3];
  const int seg = blockIdx.y;
  const int slot = threadIdx.x / ns;
  const int col = threadIdx.x - slot * ns;
  const int rpp = blockDim.x / ns;
  const int64_t s0 = seg_off[seg], s1 = seg_off[seg + 1];
  const int64_t c0 = s0 + (int64_t)blockIdx.x * rows_per_chunk;
  const int64_t c1 = min(c0 + rows_per_chunk, s1);
  double v[3] = {0.0, 0.0, 0.0};
  if (slot < rpp) {
    for (int64_t r = c0 + slot; r < c1; r += rpp) {
      const typename Cx<R>::t a = ldg_c(x + r * ns + col);
      const typename Cx<R>::t f = ldg_c(ref + r * ns + col);
      const double xr = (double)a.x, xi = (double)a.y, fr = (double)f.x, fi = (double)f.y;
      v[0] += fr * xr + fi * xi;
      v[1] += fr * xi - fi * xr;
      v[2] += xr * xr + xi * xi;
    }
  }
  seg_block_reduce(smem, v, 3, slot, col, rpp, ns);
  if (slot == 0) {
    for (int q = 0; q < 3; ++q)
      partials[(((int64_t)seg * ns + col) * 3 + q) * gridDim.x + blockIdx.x] = smem[col * 3 + q];
  }
}

}  // namespace tbpm
