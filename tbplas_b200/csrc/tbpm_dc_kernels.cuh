// DC-conductivity kernels (tbpm.f90:497-718, SUBROUTINE tbpm_dccond).
//
// Phase 1 keeps the quasi-eigenstate block QE[N][n_en][B] (row-major over
// orbitals, then energies, then states) and folds a window of T propagated
// states per update:  QE_ib += sum_tau c_{tau,i} psi+_tau + conj(c_{tau,i}) psi-_tau
// with c_{tau,i} = W(t) exp(i E_i t dt)  (tbpm.f90:626-638).
//
// Phase 2 uses the Hermiticity of the current operator J (h_ji = conj(h_ij),
// dr_ji = -dr_ij, cython/sample.pyx:242-254):
//   <J wf0_J(t) | J wfE_i> = <J J wf0_J(t) | wfE_i>,
// so one J application per step replaces the 2*n_en current products per step
// of the reference, and the normalisation of QE_i cancels against
// |<wf0|QE_i/|QE_i|>|:  dc(k,i,t) = <u_k(t)|QE_i> / |<wf0|QE_i>|.
#pragma once

#include "tbpm_common.cuh"

namespace tbpm {

constexpr int kMaxWindow = 16;   // phase-1 window (states folded per QE update)
constexpr int kMaxProject = 8;   // phase-2 window (steps per QE projection)

template <typename R>
struct StatePtrs {
  const typename Cx<R>::t* p[kMaxWindow];
};

// Rows of the window states staged per pass of the QE kernels.
__host__ __device__ constexpr int qe_tile_rows(int nb) { return nb >= 32 ? 1 : 32 / nb; }

// Shared memory of qe_accum_kernel for nb states and `threads` elements per block.
__host__ __device__ constexpr size_t qe_accum_smem(int n_en, int nb, int threads) {
  // a chunk of `threads` consecutive elements spans at most threads / nb + 2 energies
  return sizeof(double2) *
         ((size_t)kMaxWindow * (size_t)(n_en < threads / nb + 2 ? n_en : threads / nb + 2) +
          (size_t)qe_tile_rows(nb) * kMaxWindow * 2 * nb);
}
// Shared memory of qe_project_kernel.
__host__ __device__ constexpr size_t qe_project_smem(int nb) {
  return sizeof(double2) * (size_t)qe_tile_rows(nb) * kMaxProject * 2 * nb;
}

// QE[r][i][b] (+)= sum_tau c[tau][i] * pos_tau[r][b] + conj(c[tau][i]) * neg_tau[r][b]
// pos/neg columns of a window state: b and nb + b (ld = 2 nb).  init: start
// from wf0[r][b] (tbpm.f90:600-603).
// Grid: x strides over tiles of qe_tile_rows(nb) rows, y over chunks of
// blockDim.x elements (i, b) of a row.  The block stages the coefficients of
// its energies once and the window values of a row tile (converted to double
// once, instead of once per energy) in shared memory; each thread then folds
// the window into its element of every row of the tile, in the same order and
// with the same arithmetic as one thread per element.
template <typename R>
__global__ void __launch_bounds__(256) qe_accum_kernel(typename Cx<R>::t* qe, int64_t n_rows,
                                                       int n_en, int nb, StatePtrs<R> win,
                                                       int T, const double2* coef, int init,
                                                       const typename Cx<R>::t* wf0) {
  extern __shared__ double2 qsm[];
  const int n_ib = n_en * nb;
  const int ld = 2 * nb;
  const int RS = qe_tile_rows(nb);
  const int ib0 = blockIdx.y * blockDim.x;
  const int ib = ib0 + threadIdx.x;
  const bool active = ib < n_ib;
  const int i = (active ? ib : ib0) / nb;
  const int b = active ? ib - i * nb : 0;
  const int i0 = ib0 / nb;
  const int ni = min(n_en, (ib0 + (int)blockDim.x - 1) / nb + 1) - i0;
  double2* sc = qsm;                    // [kMaxWindow][ni]
  double2* sw = qsm + kMaxWindow * ni;  // [RS][kMaxWindow][ld]
  for (int q = threadIdx.x; q < T * ni; q += blockDim.x) {
    const int tau = q / ni;
    const int ii = q - tau * ni;
    sc[tau * ni + ii] = coef[tau * n_en + i0 + ii];
  }
  for (int64_t rb = (int64_t)blockIdx.x * RS; rb < n_rows; rb += (int64_t)gridDim.x * RS) {
    const int nr = (int)min((int64_t)RS, n_rows - rb);
    __syncthreads();  // the previous tile is consumed (and the coefficients staged)
#pragma unroll
    for (int tau = 0; tau < kMaxWindow; ++tau) {
      if (tau < T) {
        const typename Cx<R>::t* src = win.p[tau] + rb * ld;
        for (int q = threadIdx.x; q < nr * ld; q += blockDim.x) {
          const int rr = q / ld;
          const typename Cx<R>::t v = ldg_c(src + q);
          sw[(rr * kMaxWindow + tau) * ld + (q - rr * ld)] = make_double2((double)v.x, (double)v.y);
        }
      }
    }
    __syncthreads();
    if (!active) continue;
    for (int rr = 0; rr < nr; ++rr) {
      const int64_t r = rb + rr;
      const int64_t g = r * n_ib + ib;
      double qr, qi;
      if (init) {
        const typename Cx<R>::t w = wf0[r * nb + b];
        qr = (double)w.x;
        qi = (double)w.y;
      } else {
        const typename Cx<R>::t q = qe[g];
        qr = (double)q.x;
        qi = (double)q.y;
      }
      const double2* wr = sw + rr * kMaxWindow * ld;
#pragma unroll
      for (int tau = 0; tau < kMaxWindow; ++tau) {
        if (tau < T) {
          const double2 c = sc[tau * ni + (i - i0)];
          const double2 p = wr[tau * ld + b];
          const double2 m = wr[tau * ld + nb + b];
          const double pr = p.x, pi = p.y, mr = m.x, mi = m.y;
          // c*p + conj(c)*m
          qr += c.x * pr - c.y * pi + c.x * mr + c.y * mi;
          qi += c.x * pi + c.y * pr + c.x * mi - c.y * mr;
        }
      }
      typename Cx<R>::t o;
      o.x = (R)qr;
      o.y = (R)qi;
      qe[g] = o;
    }
  }
}

// Tall-skinny reductions over orbitals with one thread per (energy, state)
// element: block partial sums of conj(u_tau[r][k*nb + b]) * QE[r][i][b] for
// tau < T, k in {0, 1} (mode 0), or of conj(wf0[r][b]) * QE[r][i][b] (mode 1,
// T = 1, k = 0).  partials[((tau*2 + k) * n_en*nb + ib) * 2 + {re,im}][block x].
// Grid: x over row ranges of rows_per_tile, y over chunks of blockDim.x
// elements.  The u values of a tile of rows are staged in shared memory as
// double (converted once, not once per energy); each thread sums its rows in
// order, with the accumulators in registers (compile-time indices only).
template <typename R>
__global__ void __launch_bounds__(256) qe_project_kernel(const typename Cx<R>::t* qe,
                                                         int64_t n_rows, int64_t rows_per_tile,
                                                         int n_en, int nb, StatePtrs<R> u,
                                                         int T, int mode,
                                                         const typename Cx<R>::t* wf0,
                                                         double* partials) {
  extern __shared__ double2 qsm[];
  const int64_t r0 = (int64_t)blockIdx.x * rows_per_tile;
  const int64_t r1 = min(r0 + rows_per_tile, n_rows);
  const int n_ib = n_en * nb;
  const int K = mode == 0 ? 2 : 1;
  const int ld = 2 * nb;
  const int RS = qe_tile_rows(nb);
  const int ib = blockIdx.y * blockDim.x + threadIdx.x;
  const bool active = ib < n_ib;
  const int b = active ? ib % nb : 0;
  double ar[2 * kMaxProject], ai[2 * kMaxProject];
#pragma unroll
  for (int q = 0; q < 2 * kMaxProject; ++q) ar[q] = ai[q] = 0.0;
  for (int64_t rb = r0; rb < r1; rb += RS) {
    const int nr = (int)min((int64_t)RS, r1 - rb);
    __syncthreads();  // the previous tile is consumed
    if (mode == 1) {
      for (int q = threadIdx.x; q < nr * nb; q += blockDim.x) {
        const typename Cx<R>::t v = ldg_c(wf0 + rb * nb + q);
        qsm[q] = make_double2((double)v.x, (double)v.y);
      }
    } else {
#pragma unroll
      for (int tau = 0; tau < kMaxProject; ++tau) {
        if (tau < T) {
          const typename Cx<R>::t* src = u.p[tau] + rb * ld;
          for (int q = threadIdx.x; q < nr * ld; q += blockDim.x) {
            const int rr = q / ld;
            const typename Cx<R>::t v = ldg_c(src + q);
            qsm[(rr * kMaxProject + tau) * ld + (q - rr * ld)] =
                make_double2((double)v.x, (double)v.y);
          }
        }
      }
    }
    __syncthreads();
    if (!active) continue;
    for (int rr = 0; rr < nr; ++rr) {
      const typename Cx<R>::t qv = qe[(rb + rr) * n_ib + ib];
      const double qr = (double)qv.x, qi = (double)qv.y;
      if (mode == 1) {
        const double2 w = qsm[rr * nb + b];
        ar[0] += w.x * qr + w.y * qi;
        ai[0] += w.x * qi - w.y * qr;
      } else {
        const double2* ur = qsm + rr * kMaxProject * ld;
#pragma unroll
        for (int tau = 0; tau < kMaxProject; ++tau) {
          if (tau < T) {
#pragma unroll
            for (int k = 0; k < 2; ++k) {
              const double2 w = ur[tau * ld + k * nb + b];
              ar[tau * 2 + k] += w.x * qr + w.y * qi;
              ai[tau * 2 + k] += w.x * qi - w.y * qr;
            }
          }
        }
      }
    }
  }
  if (!active) return;
#pragma unroll
  for (int q = 0; q < 2 * kMaxProject; ++q) {
    if (q < T * K) {
      const int64_t o = (int64_t)q * n_ib + ib;
      partials[(o * 2 + 0) * gridDim.x + blockIdx.x] = ar[q];
      partials[(o * 2 + 1) * gridDim.x + blockIdx.x] = ai[q];
    }
  }
}

// out[v] = sum over blocks of partials[v][block], fixed order; block per value.
__global__ void __launch_bounds__(256) reduce_rows_kernel(const double* partials, int n_blocks,
                                                          int64_t n_values, double* out) {
  __shared__ double red[256];
  for (int64_t v = blockIdx.x; v < n_values; v += gridDim.x) {
    const double* p = partials + v * n_blocks;
    double s = 0.0;
    for (int i = threadIdx.x; i < n_blocks; i += blockDim.x) s += p[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
      if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
      __syncthreads();
    }
    if (threadIdx.x == 0) out[v] = red[0];
    __syncthreads();
  }
}

// Current products on a block of 2*nb columns: out[r][b] = (J_x in_x)[r][b],
// out[r][nb + b] = (J_y in_y)[r][b], where in_x / in_y are columns x_off + b /
// y_off + b of `in` (row stride in_ld).  J_d = i * rescale * hop * d.
template <typename R>
__global__ void __launch_bounds__(256) jj_apply_kernel(
    const int32_t* indptr, const int32_t* indices, const typename Cx<R>::t* hop, const R* dx,
    const R* dy, double rescale, int64_t n_rows, int nb, const typename Cx<R>::t* in, int in_ld,
    int x_off, int y_off, typename Cx<R>::t* out) {
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= n_rows * 2 * nb) return;
  const int64_t r = gid / (2 * nb);
  const int col = (int)(gid - r * 2 * nb);
  const int k = col / nb;
  const int b = col - k * nb;
  const R* d = k == 0 ? dx : dy;
  const int src_col = (k == 0 ? x_off : y_off) + b;
  const R s = (R)rescale;
  R vr = 0, vi = 0;
  const int j0 = __ldg(indptr + r), j1 = __ldg(indptr + r + 1);
  for (int j = j0; j < j1; ++j) {
    const int c = __ldg(indices + j);
    const typename Cx<R>::t h = ldg_c(hop + j);
    const R dd = __ldg(d + j);
    const R jr = (-s * h.y) * dd, ji = (s * h.x) * dd;
    const typename Cx<R>::t w = ldg_c(in + (int64_t)c * in_ld + src_col);
    vr = fma(jr, w.x, fma(-ji, w.y, vr));
    vi = fma(jr, w.y, fma(ji, w.x, vi));
  }
  typename Cx<R>::t o;
  o.x = vr;
  o.y = vi;
  out[r * 2 * nb + col] = o;
}

// dst[r][b] = dst[r][nb + b] = src[r][b]   (wf_pos = wf_neg = wf0)
template <typename R>
__global__ void dup_columns_kernel(const typename Cx<R>::t* src, int64_t n_rows, int nb,
                                   typename Cx<R>::t* dst) {
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= n_rows * nb) return;
  const int64_t r = gid / nb;
  const int b = (int)(gid - r * nb);
  const typename Cx<R>::t v = src[gid];
  dst[r * 2 * nb + b] = v;
  dst[r * 2 * nb + nb + b] = v;
}

}  // namespace tbpm
