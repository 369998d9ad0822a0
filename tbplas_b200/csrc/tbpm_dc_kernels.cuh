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

// QE[r][i][b] (+)= sum_tau c[tau][i] * pos_tau[r][b] + conj(c[tau][i]) * neg_tau[r][b]
// pos/neg columns of a window state: b and nb + b (ld = 2 nb).  init: start
// from wf0[r][b] (tbpm.f90:600-603).
template <typename R>
__global__ void __launch_bounds__(256) qe_accum_kernel(typename Cx<R>::t* qe, int64_t n_rows,
                                                       int n_en, int nb, StatePtrs<R> win,
                                                       int T, const double2* coef, int init,
                                                       const typename Cx<R>::t* wf0) {
  const int64_t total = n_rows * n_en * nb;
  const int ld = 2 * nb;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = g / ((int64_t)n_en * nb);
    const int rem = (int)(g - r * n_en * nb);
    const int i = rem / nb;
    const int b = rem - i * nb;
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
    for (int tau = 0; tau < T; ++tau) {
      const double2 c = __ldg(coef + tau * n_en + i);
      const typename Cx<R>::t p = ldg_c(win.p[tau] + r * ld + b);
      const typename Cx<R>::t m = ldg_c(win.p[tau] + r * ld + nb + b);
      const double pr = (double)p.x, pi = (double)p.y, mr = (double)m.x, mi = (double)m.y;
      // c*p + conj(c)*m
      qr += c.x * pr - c.y * pi + c.x * mr + c.y * mi;
      qi += c.x * pi + c.y * pr + c.x * mi - c.y * mr;
    }
    typename Cx<R>::t o;
    o.x = (R)qr;
    o.y = (R)qi;
    qe[g] = o;
  }
}

// Tall-skinny reductions over orbitals with one thread per (energy, state)
// element: block partial sums of conj(u_tau[r][k*nb + b]) * QE[r][i][b] for
// tau < T, k in {0, 1} (mode 0), or of conj(wf0[r][b]) * QE[r][i][b] (mode 1,
// T = 1, k = 0).  partials[((tau*2 + k) * n_en*nb + ib) * 2 + {re,im}][block].
template <typename R>
__global__ void __launch_bounds__(256) qe_project_kernel(const typename Cx<R>::t* qe,
                                                         int64_t n_rows, int64_t rows_per_tile,
                                                         int n_en, int nb, StatePtrs<R> u,
                                                         int T, int mode,
                                                         const typename Cx<R>::t* wf0,
                                                         double* partials) {
  const int64_t r0 = (int64_t)blockIdx.x * rows_per_tile;
  const int64_t r1 = min(r0 + rows_per_tile, n_rows);
  const int n_ib = n_en * nb;
  const int K = mode == 0 ? 2 : 1;
  const int n_out = T * K * n_ib;
  for (int ib = threadIdx.x; ib < n_ib; ib += blockDim.x) {
    const int b = ib % nb;
    double ar[2 * kMaxProject], ai[2 * kMaxProject];
#pragma unroll
    for (int q = 0; q < 2 * kMaxProject; ++q) ar[q] = ai[q] = 0.0;
    for (int64_t r = r0; r < r1; ++r) {
      const typename Cx<R>::t qv = qe[r * n_ib + ib];
      const double qr = (double)qv.x, qi = (double)qv.y;
      if (mode == 1) {
        const typename Cx<R>::t w = ldg_c(wf0 + r * nb + b);
        ar[0] += (double)w.x * qr + (double)w.y * qi;
        ai[0] += (double)w.x * qi - (double)w.y * qr;
      } else {
#pragma unroll
        for (int tau = 0; tau < kMaxProject; ++tau) {
          if (tau < T) {
#pragma unroll
            for (int k = 0; k < 2; ++k) {
              const typename Cx<R>::t w = ldg_c(u.p[tau] + r * 2 * nb + k * nb + b);
              ar[tau * 2 + k] += (double)w.x * qr + (double)w.y * qi;
              ai[tau * 2 + k] += (double)w.x * qi - (double)w.y * qr;
            }
          }
        }
      }
    }
    for (int q = 0; q < T * K; ++q) {
      const int64_t o = (int64_t)q * n_ib + ib;
      partials[(o * 2 + 0) * gridDim.x + blockIdx.x] = ar[q];
      partials[(o * 2 + 1) * gridDim.x + blockIdx.x] = ai[q];
    }
  }
  (void)n_out;
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
