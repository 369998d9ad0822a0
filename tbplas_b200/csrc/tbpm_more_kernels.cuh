// Kernels of the TBPM drivers beyond DOS / AC / DC / psi(t):
//  dynamical polarisation  (tbpm.f90:355-493, funcs.f90:125-149)
//  quasi-eigenstates       (tbpm.f90:721-830; the QE accumulation is shared with DC)
//  Kubo-Bastin mu_mn       (tbpm.f90:836-960)
//  Haydock recursion       (propagation.f90:85-155)
#pragma once

#include "tbpm_common.cuh"
#include "tbpm_kernels.cuh"

namespace tbpm {

// up to kMaxCols q-points per launch
struct QBlock {
  double q[kMaxCols][3];
};

// q.r in the reference's order (q1*x + q2*y) + q3*z, without FMA contraction
__device__ __forceinline__ double q_dot_r(const double* q, double x, double y, double z) {
  return __dadd_rn(__dadd_rn(__dmul_rn(q[0], x), __dmul_rn(q[1], y)), __dmul_rn(q[2], z));
}

// Block of nq*nb + nb columns: psi1 of q-point k and state b at column k*nb + b
// gets exp(-i q_k.r) wf0_b (tbpm.f90:456), psi2 of state b (column nq*nb + b)
// gets wf0_b.
template <typename R>
__global__ void dens_init_kernel(const typename Cx<R>::t* W, const double* sx, const double* sy,
                                 const double* sz, QBlock qb, int nq, int nb, int64_t n_rows,
                                 typename Cx<R>::t* A) {
  const int ld = (nq + 1) * nb;
  const int64_t total = n_rows * ld;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = g / ld;
    const int col = (int)(g - r * ld);
    const int k = col / nb;
    const int b = col - k * nb;
    const typename Cx<R>::t w = W[r * nb + b];
    typename Cx<R>::t o = w;
    if (k < nq) {
      double sn, cs;
      sincos(q_dot_r(qb.q[k], sx[r], sy[r], sz[r]), &sn, &cs);
      // (cs - i sn) * w
      const double wr = (double)w.x, wi = (double)w.y;
      o.x = (R)(cs * wr + sn * wi);
      o.y = (R)(cs * wi - sn * wr);
    }
    A[g] = o;
  }
}

// Partials of <psi2_b | exp(i q_k.r) psi1_{k,b}> (re, im) and <psi2_b|psi2_b>
// for every (k, b): partials[((k*nb + b)*3 + v) * gridDim.x + block].
// One thread per (k, b) column of a row slot; rows grid-stride.
template <typename R>
__global__ void __launch_bounds__(256) dens_corr_kernel(const typename Cx<R>::t* A,
                                                        const double* sx, const double* sy,
                                                        const double* sz, QBlock qb, int nq,
                                                        int nb, int64_t n_rows,
                                                        double* partials) {
  extern __shared__ double smem[];
  const int tpr = nq * nb;
  const int slot = threadIdx.x / tpr;
  const int lane = threadIdx.x - slot * tpr;
  const int rpp = blockDim.x / tpr;
  const int k = lane / nb;
  const int b = lane - k * nb;
  const int ld = (nq + 1) * nb;
  double cr = 0.0, ci = 0.0, nn = 0.0;
  for (int64_t r = (int64_t)blockIdx.x * rpp + slot; r < n_rows;
       r += (int64_t)gridDim.x * rpp) {
    const typename Cx<R>::t p1 = A[r * ld + lane];
    const typename Cx<R>::t p2 = A[r * ld + nq * nb + b];
    double sn, cs;
    sincos(q_dot_r(qb.q[k], sx[r], sy[r], sz[r]), &sn, &cs);
    const double ar = (double)p1.x, ai = (double)p1.y;
    const double wr = cs * ar - sn * ai, wi = cs * ai + sn * ar;  // exp(i q.r) psi1
    const double qr = (double)p2.x, qi = (double)p2.y;
    cr += qr * wr + qi * wi;
    ci += qr * wi - qi * wr;
    nn += qr * qr + qi * qi;
  }
  const int width = tpr * 3;
  smem[slot * width + lane * 3 + 0] = cr;
  smem[slot * width + lane * 3 + 1] = ci;
  smem[slot * width + lane * 3 + 2] = nn;
  __syncthreads();
  tree_reduce_slots(smem, rpp, width, slot, lane, tpr);
  if (slot == 0) {
#pragma unroll
    for (int v = 0; v < 3; ++v)
      partials[(int64_t)(lane * 3 + v) * gridDim.x + blockIdx.x] = smem[lane * 3 + v];
  }
}

// Block partials of sum_r |QE[r][ib]|^2, one thread per (energy, state) ib;
// partials[ib * gridDim.x + block].
template <typename R>
__global__ void __launch_bounds__(256) qe_sqnorm_kernel(const typename Cx<R>::t* qe,
                                                        int64_t n_rows, int64_t rows_per_tile,
                                                        int n_ib, double* partials) {
  const int64_t r0 = (int64_t)blockIdx.x * rows_per_tile;
  const int64_t r1 = min(r0 + rows_per_tile, n_rows);
  for (int ib = threadIdx.x; ib < n_ib; ib += blockDim.x) {
    double s = 0.0;
    for (int64_t r = r0; r < r1; ++r) {
      const typename Cx<R>::t q = qe[r * n_ib + ib];
      s += (double)q.x * (double)q.x + (double)q.y * (double)q.y;
    }
    partials[(int64_t)ib * gridDim.x + blockIdx.x] = s;
  }
}

// acc[r][i] += scale * sum_b |QE[r][i][b]|^2 / nrm2[i*nb + b]   (tbpm.f90:803-813)
template <typename R>
__global__ void qe_density_kernel(const typename Cx<R>::t* qe, int64_t n_rows, int n_en, int nb,
                                  const double* nrm2, double scale, double* acc) {
  const int64_t total = n_rows * n_en;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = g / n_en;
    const int i = (int)(g - r * n_en);
    double s = 0.0;
    for (int b = 0; b < nb; ++b) {
      const typename Cx<R>::t q = qe[(r * n_en + i) * nb + b];
      s += ((double)q.x * (double)q.x + (double)q.y * (double)q.y) / nrm2[i * nb + b];
    }
    acc[g] += scale * s;
  }
}

// ---- single-vector kernels (Kubo-Bastin, Haydock) ---------------------------

// y = alpha * (H x) + beta * z, H = D + O (z may alias y; beta == 0 ignores z)
template <typename R>
__global__ void cheb_vec_kernel(const int32_t* indptr, const int32_t* indices,
                                const typename Cx<R>::t* hop, const typename Cx<R>::t* diag,
                                int64_t n_rows, double alpha, double beta,
                                const typename Cx<R>::t* x, const typename Cx<R>::t* z,
                                typename Cx<R>::t* y) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n_rows;
       r += (int64_t)gridDim.x * blockDim.x) {
    double vr = 0.0, vi = 0.0;
    if (diag) {
      const typename Cx<R>::t d = diag[r], w = x[r];
      vr = (double)d.x * (double)w.x - (double)d.y * (double)w.y;
      vi = (double)d.x * (double)w.y + (double)d.y * (double)w.x;
    }
    const int j0 = __ldg(indptr + r), j1 = __ldg(indptr + r + 1);
    for (int j = j0; j < j1; ++j) {
      const typename Cx<R>::t h = ldg_c(hop + j);
      const typename Cx<R>::t w = ldg_c(x + __ldg(indices + j));
      vr += (double)h.x * (double)w.x - (double)h.y * (double)w.y;
      vi += (double)h.x * (double)w.y + (double)h.y * (double)w.x;
    }
    double orr = alpha * vr, oi = alpha * vi;
    if (beta != 0.0) {
      const typename Cx<R>::t zz = z[r];
      orr += beta * (double)zz.x;
      oi += beta * (double)zz.y;
    }
    typename Cx<R>::t o;
    o.x = (R)orr;
    o.y = (R)oi;
    y[r] = o;
  }
}

// y = J_d x with J_d = i * rescale * hop * d on the off-diagonal entries
// (funcs.f90:12-33 + csr.F90:71-101)
template <typename R>
__global__ void current_vec_kernel(const int32_t* indptr, const int32_t* indices,
                                   const typename Cx<R>::t* hop, const R* d, double rescale,
                                   int64_t n_rows, const typename Cx<R>::t* x,
                                   typename Cx<R>::t* y) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n_rows;
       r += (int64_t)gridDim.x * blockDim.x) {
    double vr = 0.0, vi = 0.0;
    const int j0 = __ldg(indptr + r), j1 = __ldg(indptr + r + 1);
    for (int j = j0; j < j1; ++j) {
      const typename Cx<R>::t h = ldg_c(hop + j);
      const double dd = (double)__ldg(d + j);
      const double jr = -rescale * (double)h.y * dd, ji = rescale * (double)h.x * dd;
      const typename Cx<R>::t w = ldg_c(x + __ldg(indices + j));
      vr += jr * (double)w.x - ji * (double)w.y;
      vi += jr * (double)w.y + ji * (double)w.x;
    }
    typename Cx<R>::t o;
    o.x = (R)vr;
    o.y = (R)vi;
    y[r] = o;
  }
}

// Haydock step, part 1: pb = rescale * H p2 and partials of <p2|pb>
// (partials[v * gridDim.x + block], v = re, im)
template <typename R>
__global__ void __launch_bounds__(256) haydock_apply_kernel(
    const int32_t* indptr, const int32_t* indices, const typename Cx<R>::t* hop,
    const typename Cx<R>::t* diag, int64_t n_rows, double rescale, const typename Cx<R>::t* p2,
    typename Cx<R>::t* pb, double* partials) {
  __shared__ double red[2][256];
  double cr = 0.0, ci = 0.0;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n_rows;
       r += (int64_t)gridDim.x * blockDim.x) {
    double vr = 0.0, vi = 0.0;
    if (diag) {
      const typename Cx<R>::t d = diag[r], w = p2[r];
      vr = (double)d.x * (double)w.x - (double)d.y * (double)w.y;
      vi = (double)d.x * (double)w.y + (double)d.y * (double)w.x;
    }
    const int j0 = __ldg(indptr + r), j1 = __ldg(indptr + r + 1);
    for (int j = j0; j < j1; ++j) {
      const typename Cx<R>::t h = ldg_c(hop + j);
      const typename Cx<R>::t w = ldg_c(p2 + __ldg(indices + j));
      vr += (double)h.x * (double)w.x - (double)h.y * (double)w.y;
      vi += (double)h.x * (double)w.y + (double)h.y * (double)w.x;
    }
    vr *= rescale;
    vi *= rescale;
    typename Cx<R>::t o;
    o.x = (R)vr;
    o.y = (R)vi;
    pb[r] = o;
    const typename Cx<R>::t s = p2[r];
    const double sr = (double)s.x, si = (double)s.y;
    cr += sr * (double)o.x + si * (double)o.y;
    ci += sr * (double)o.y - si * (double)o.x;
  }
  red[0][threadIdx.x] = cr;
  red[1][threadIdx.x] = ci;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      red[0][threadIdx.x] += red[0][threadIdx.x + w];
      red[1][threadIdx.x] += red[1][threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = red[0][0];
    partials[gridDim.x + blockIdx.x] = red[1][0];
  }
}

// Haydock step, part 2: pb = -a*p2 - b_prev*p1 + pb (a = coef[0..1] complex,
// b_prev = *bprev, absent when bprev is null) and partials of <pb|pb>
template <typename R>
__global__ void __launch_bounds__(256) haydock_orth_kernel(int64_t n_rows, const double* a,
                                                           const double* bprev,
                                                           const typename Cx<R>::t* p2,
                                                           const typename Cx<R>::t* p1,
                                                           typename Cx<R>::t* pb,
                                                           double* partials) {
  __shared__ double red[256];
  const double ar = -a[0], ai = -a[1];
  const double bb = bprev ? -*bprev : 0.0;
  double nn = 0.0;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n_rows;
       r += (int64_t)gridDim.x * blockDim.x) {
    const typename Cx<R>::t x = p2[r], z = pb[r];
    double vr = ar * (double)x.x - ai * (double)x.y;
    double vi = ar * (double)x.y + ai * (double)x.x;
    if (bprev) {
      const typename Cx<R>::t y = p1[r];
      vr += bb * (double)y.x;
      vi += bb * (double)y.y;
    }
    vr += (double)z.x;
    vi += (double)z.y;
    typename Cx<R>::t o;
    o.x = (R)vr;
    o.y = (R)vi;
    pb[r] = o;
    nn += (double)o.x * (double)o.x + (double)o.y * (double)o.y;
  }
  red[threadIdx.x] = nn;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) partials[blockIdx.x] = red[0];
}

// Fixed-order sum of n_parts partials of n_vals values into out (one block);
// mode 1 takes the square root of value 0 (a norm).
__global__ void __launch_bounds__(256) small_reduce_kernel(const double* partials, int n_parts,
                                                           int n_vals, int mode, double* out) {
  __shared__ double red[256];
  for (int v = 0; v < n_vals; ++v) {
    double s = 0.0;
    for (int i = threadIdx.x; i < n_parts; i += blockDim.x) s += partials[v * n_parts + i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
      if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
      __syncthreads();
    }
    if (threadIdx.x == 0) out[v] = (mode == 1 && v == 0) ? sqrt(red[0]) : red[0];
    __syncthreads();
  }
}

// y = x / *b (b on the device)
template <typename R>
__global__ void scale_inv_kernel(int64_t n_rows, const double* b, const typename Cx<R>::t* x,
                                 typename Cx<R>::t* y) {
  const double s = *b;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n_rows;
       r += (int64_t)gridDim.x * blockDim.x) {
    const typename Cx<R>::t v = x[r];
    typename Cx<R>::t o;
    o.x = (R)((double)v.x / s);
    o.y = (R)((double)v.y / s);
    y[r] = o;
  }
}

}  // namespace tbpm

namespace tbpm {

// analysis.f90:6-69 (cond_from_trace) with kpm.f90:31-56 (get_gamma_mn):
// out[k-1] = sum_{m,n} Re(Gamma_mn(x_k) mu_mn), x_k = k * pi / ne_integral,
// one block per energy; cos(m x), sin(m x) are tabulated in shared memory and
// the threads walk the rows m of mu (column-major), so the reads coalesce.
//   Gamma_mn = (cos x - i n sin x) cos(m x) e^{i n x} + (cos x + i m sin x) cos(n x) e^{-i m x}
__global__ void __launch_bounds__(256) gamma_trace_kernel(const double2* mu, int nk,
                                                          int ne_integral, double* out) {
  extern __shared__ double tab[];  // [0, nk): cos(m x), [nk, 2nk): sin(m x)
  __shared__ double red[256];
  const int k = blockIdx.x + 1;
  const double x = k * (3.14159265358979323846 / ne_integral);
  for (int m = threadIdx.x; m < nk; m += blockDim.x) {
    double s, c;
    sincos(m * x, &s, &c);
    tab[m] = c;
    tab[nk + m] = s;
  }
  __syncthreads();
  double sx, cx;
  sincos(x, &sx, &cx);
  double acc = 0.0;
  for (int n = 0; n < nk; ++n) {
    const double cn = tab[n], sn = tab[nk + n];
    const double a1 = cx * cn + n * sx * sn;  // Re of (cx - i n sx)(Cn + i Sn)
    const double b1 = cx * sn - n * sx * cn;  // Im of the same
    const double2* col = mu + (int64_t)n * nk;
    for (int m = threadIdx.x; m < nk; m += blockDim.x) {
      const double cm = tab[m], sm = tab[nk + m];
      const double re = cm * a1 + cn * (cx * cm + m * sx * sm);
      const double im = cm * b1 + cn * (m * sx * cm - cx * sm);
      const double2 v = col[m];
      acc += re * v.x - im * v.y;
    }
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = red[0];
}

}  // namespace tbpm
