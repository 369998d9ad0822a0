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

// ---- quasi-eigenstate kernels: cp.async double-buffered row tiles -----------
//
// Both QE kernels walk tiles of qe_tile_rows rows.  While a block works on tile
// j, the raw values of tile j+1 (window states, and the block's slice of QE)
// are on their way into shared memory (cp.async, no registers held); a short
// pass converts each staged value to double once; the tile's arithmetic then
// reads shared memory only.  Two barriers per tile.

#ifndef TBPM_QE_MINB_A
#define TBPM_QE_MINB_A 2
#endif
#ifndef TBPM_QE_MINB_P
#define TBPM_QE_MINB_P 2
#endif
#ifndef TBPM_QE_ROWS_A
#define TBPM_QE_ROWS_A 4
#endif
// rows per tile of qe_project_kernel, and of qe_accum_kernel (fewer: its tile
// holds 16 window states)
template <typename R>
__host__ __device__ constexpr int qe_tile_rows(int nb) {
  return nb >= 64 ? 1 : (64 / nb < 8 ? 64 / nb : 8);
}
template <typename R>
__host__ __device__ constexpr int qe_accum_rows(int nb) {
  return nb >= 64 ? 1 : (64 / nb < TBPM_QE_ROWS_A ? 64 / nb : TBPM_QE_ROWS_A);
}

// One complex value into shared memory, asynchronously.
template <typename C>
__device__ __forceinline__ void qe_cp_async(C* dst, const C* src) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  if constexpr (sizeof(C) == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void qe_cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void qe_cp_wait_all() {
  asm volatile("cp.async.wait_group 0;" ::: "memory");
}

// Energies per thread of the QE kernels: a thread updates (or projects) the
// elements of kQeG energies for one state b, so every staged window / u value
// it reads from shared memory serves kQeG elements.
constexpr int kQeG = 2;

// Threads per block of qe_accum_kernel: a multiple of nb (so that the kQeG
// elements of a thread share their state b), at most 256.
__host__ __device__ constexpr int qe_accum_threads(int n_en, int nb) {
  return nb * ((n_en + kQeG - 1) / kQeG < 256 / nb ? (n_en + kQeG - 1) / kQeG : 256 / nb);
}
// Threads per block of qe_project_kernel (K threads per element: one per k).
__host__ __device__ constexpr int qe_project_threads(int n_en, int nb, int K) {
  return K * nb *
         ((n_en + kQeG - 1) / kQeG < 256 / (K * nb) ? (n_en + kQeG - 1) / kQeG : 256 / (K * nb));
}

// Shared memory of qe_accum_kernel.
template <typename R>
__host__ __device__ constexpr size_t qe_accum_smem(int n_en, int nb) {
  return (size_t)qe_accum_rows<R>(nb) * kMaxWindow * 2 * nb * sizeof(double2) +     // S | D
         (size_t)kMaxWindow * kQeG * (size_t)(qe_accum_threads(n_en, nb) / nb) *
             sizeof(double2);                                                       // coefficients
}
// Shared memory of qe_project_kernel.
template <typename R>
__host__ __device__ constexpr size_t qe_project_smem(int n_en, int nb, int K) {
  return (sizeof(R) == 4 ? (size_t)qe_tile_rows<R>(nb) * kMaxProject * 2 * nb * sizeof(double2)
                         : 0) +                                                     // converted u
         2 * (size_t)qe_tile_rows<R>(nb) * kMaxProject * 2 * nb * 2 * sizeof(R) +   // raw u
         2 * (size_t)qe_tile_rows<R>(nb) * kQeG * (qe_project_threads(n_en, nb, K) / K) * 2 *
             sizeof(R);                                                             // raw QE
}

// QE[r][i][b] (+)= sum_tau c[tau][i] * pos_tau[r][b] + conj(c[tau][i]) * neg_tau[r][b]
// pos/neg columns of a window state: b and nb + b (ld = 2 nb).  init: start
// from wf0[r][b] (tbpm.f90:600-603).
// c p + conj(c) m = Re(c) (p + m) + i Im(c) (p - m): the sum S = p + m and the
// difference D = p - m of a row are formed once, in double, per staged tile,
// and every energy then needs 4 FMAs per window state instead of 8.
// Block: qe_accum_threads(n_en, nb) threads; thread t owns the elements
// ib_lo + t + g * blockDim.x (g < kQeG): state b = t % nb, kQeG energies, for
// every row of a tile; a coefficient read from shared memory serves the rows
// of the tile and an S / D value serves kQeG energies.  A thread's QE values
// of a tile are loaded before the tile's window values are staged, so both
// are in flight together.  (The window tile is staged with plain loads: a
// second, asynchronously filled buffer would halve the resident blocks.)
// Grid: x strides over row tiles, y over chunks of kQeG * blockDim.x elements.
template <typename R>
__global__ void __launch_bounds__(256, TBPM_QE_MINB_A) qe_accum_kernel(
    typename Cx<R>::t* qe, int64_t n_rows, int n_en, int nb, StatePtrs<R> win, int T,
    const double2* coef, int init, const typename Cx<R>::t* wf0) {
  using C = typename Cx<R>::t;
  constexpr int RM = TBPM_QE_ROWS_A;
  extern __shared__ double2 qsm[];
  const int n_ib = n_en * nb;
  const int ld = 2 * nb;
  const int RS = qe_accum_rows<R>(nb);
  const int NT = blockDim.x;  // a multiple of nb
  const int EBE = kQeG * NT;  // elements of a row the block covers
  const int ib_lo = blockIdx.y * EBE;
  const int eb = min(EBE, n_ib - ib_lo);
  const int t = threadIdx.x;
  const int b = t % nb;
  const int i_lo = ib_lo / nb;
  const int ni = min(n_en - i_lo, EBE / nb);
  bool act[kQeG];
  int il[kQeG];  // energy of element g, relative to i_lo
#pragma unroll
  for (int g = 0; g < kQeG; ++g) {
    act[g] = t + g * NT < eb;
    il[g] = (t + g * NT) / nb;
  }
  const int TW = kMaxWindow * ld;                  // staged values of one row
  double2* sd = qsm;                               // [RS][TW] S | D
  double2* sc = qsm + RS * TW;                     // [kMaxWindow][ni]
  for (int q = threadIdx.x; q < T * ni; q += blockDim.x) {
    const int tau = q / ni;
    const int ii = q - tau * ni;
    sc[tau * ni + ii] = coef[tau * n_en + i_lo + ii];
  }
  for (int64_t rb = (int64_t)blockIdx.x * RS; rb < n_rows; rb += (int64_t)gridDim.x * RS) {
    const int nr = (int)min((int64_t)RS, n_rows - rb);
    C q0[RM][kQeG];
#pragma unroll
    for (int rr = 0; rr < RM; ++rr)
#pragma unroll
      for (int g = 0; g < kQeG; ++g)
        if (rr < nr && act[g])
          q0[rr][g] = init ? wf0[(rb + rr) * nb + b] : qe[(rb + rr) * n_ib + ib_lo + t + g * NT];
    __syncthreads();  // the previous tile is consumed (and the coefficients staged)
#pragma unroll
    for (int tau = 0; tau < kMaxWindow; ++tau) {
      if (tau < T) {
        const C* src = win.p[tau] + rb * ld;
        for (int q = threadIdx.x; q < nr * nb; q += blockDim.x) {
          const int rr = q / nb;
          const int bb = q - rr * nb;
          const C p = ldg_c(src + rr * ld + bb);
          const C m = ldg_c(src + rr * ld + nb + bb);
          double2* o = sd + rr * TW + tau * ld;
          o[bb] = make_double2((double)p.x + (double)m.x, (double)p.y + (double)m.y);
          o[nb + bb] = make_double2((double)p.x - (double)m.x, (double)p.y - (double)m.y);
        }
      }
    }
    __syncthreads();
    if (!act[0]) continue;
    double qr[RM][kQeG], qi[RM][kQeG];
#pragma unroll
    for (int rr = 0; rr < RM; ++rr)
#pragma unroll
      for (int g = 0; g < kQeG; ++g) {
        qr[rr][g] = (double)q0[rr][g].x;
        qi[rr][g] = (double)q0[rr][g].y;
      }
#pragma unroll
    for (int tau = 0; tau < kMaxWindow; ++tau) {
      if (tau < T) {
        double2 c[kQeG];
#pragma unroll
        for (int g = 0; g < kQeG; ++g) c[g] = act[g] ? sc[tau * ni + il[g]] : make_double2(0, 0);
#pragma unroll
        for (int rr = 0; rr < RM; ++rr) {
          if (rr < nr) {
            const double2 S = sd[rr * TW + tau * ld + b];
            const double2 D = sd[rr * TW + tau * ld + nb + b];
#pragma unroll
            for (int g = 0; g < kQeG; ++g) {
              qr[rr][g] += c[g].x * S.x - c[g].y * D.y;
              qi[rr][g] += c[g].x * S.y + c[g].y * D.x;
            }
          }
        }
      }
    }
#pragma unroll
    for (int rr = 0; rr < RM; ++rr)
#pragma unroll
      for (int g = 0; g < kQeG; ++g)
        if (rr < nr && act[g]) {
          C o;
          o.x = (R)qr[rr][g];
          o.y = (R)qi[rr][g];
          qe[(rb + rr) * n_ib + ib_lo + t + g * NT] = o;
        }
  }
}

// ---- quasi-eigenstate accumulation as FP64 matrix products (mma.sync) -------
//
// For a row r and state b the window update of qe_accum_kernel is, over the
// energies i,
//   QE_re[i] += sum_tau Re c[tau][i] S_tau.x - Im c[tau][i] D_tau.y
//   QE_im[i] += sum_tau Re c[tau][i] S_tau.y + Im c[tau][i] D_tau.x
// i.e. one real product  A (energies x 2T) . B (2T x (r, b, re/im))  added to
// the block QE, with A[i][tau] = Re c, A[i][16 + tau] = Im c (zero for tau >=
// T) shared by every row.  qe_accum_mma_kernel runs it on the FP64 tensor
// path (mma.sync m8n8k4 f64): a warp owns up to kQeMmaMT tiles of 8 energies
// and keeps their A fragments (8 k-steps of 4) in registers for the whole
// launch; for each tile of kQeMmaPairs (row, state) pairs the block stages S
// and D (double) in shared memory, and a warp then, per 8-column tile (4 pairs
// x re/im), loads the B fragments once and updates its energy tiles: the C
// fragment of a lane is exactly one complex QE element.  QE is read and
// written once per window.
constexpr int kQeMmaWarps = 8;
constexpr int kQeMmaMT = 4;      // energy tiles (of 8) per warp
constexpr int kQeMmaPairs = 32;  // (row, state) pairs per staged tile

__device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// Rows per staged tile: at least kQeMmaPairs pairs, and rows * nb a multiple
// of 4 (whole 8-column tiles).
__host__ __device__ constexpr int qe_mma_rows(int nb) {
  return (((kQeMmaPairs + nb - 1) / nb) + (4 / (nb % 4 == 0 ? 4 : (nb % 2 == 0 ? 2 : 1))) - 1) /
         (4 / (nb % 4 == 0 ? 4 : (nb % 2 == 0 ? 2 : 1))) *
         (4 / (nb % 4 == 0 ? 4 : (nb % 2 == 0 ? 2 : 1)));
}

// Shared memory of qe_accum_mma_kernel: S and D of a tile, [tau][pair].
__host__ __device__ constexpr size_t qe_mma_smem(int nb) {
  return (size_t)kMaxWindow * qe_mma_rows(nb) * nb * 2 * sizeof(double2);
}

// Grid: x walks tiles of qe_mma_rows(nb) rows grid-stride; y walks groups of
// kQeMmaWarps * kQeMmaMT energy tiles.  Block: kQeMmaWarps warps.
template <typename R>
__global__ void __launch_bounds__(kQeMmaWarps * 32, 2) qe_accum_mma_kernel(
    typename Cx<R>::t* qe, int64_t n_rows, int n_en, int nb, const __grid_constant__ StatePtrs<R> win, int T,
    const double2* coef, int init, const typename Cx<R>::t* wf0) {
  using C = typename Cx<R>::t;
  extern __shared__ double2 qsm[];
  const int RT = qe_mma_rows(nb);
  const int P = RT * nb;  // pairs of a tile; P % 4 == 0
  const int ld = 2 * nb;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  // The block's energy tiles [blockIdx.y * 32, +32) form n_mg groups of
  // kQeMmaMT; warp w takes group w % n_mg and, with the other warps of that
  // group, every cnt-th column tile (so few energies still use every warp).
  const int n_mt = (n_en + 7) / 8;
  const int mt_b = blockIdx.y * kQeMmaWarps * kQeMmaMT;
  const int n_mt_b = min(kQeMmaWarps * kQeMmaMT, n_mt - mt_b);
  const int n_mg = (n_mt_b + kQeMmaMT - 1) / kQeMmaMT;
  const int mg = warp % n_mg;
  const int nt_first = warp / n_mg;
  const int nt_step = (kQeMmaWarps - mg + n_mg - 1) / n_mg;
  const int mt0 = mt_b + mg * kQeMmaMT;
  // A fragments: A[i = 8*mt + g][k = 4*s + t]
  double afr[kQeMmaMT][8];
#pragma unroll
  for (int m = 0; m < kQeMmaMT; ++m) {
    const int i = (mt0 + m) * 8 + g;
#pragma unroll
    for (int st = 0; st < 8; ++st) {
      const int k = 4 * st + t;
      const int tau = k & 15;
      double v = 0.0;
      if (i < n_en && tau < T) {
        const double2 c = coef[tau * n_en + i];
        v = k < 16 ? c.x : c.y;
      }
      afr[m][st] = v;
    }
  }
  double2* sS = qsm;                          // [kMaxWindow][P]
  double2* sD = qsm + kMaxWindow * P;         // [kMaxWindow][P]
  for (int64_t r0 = (int64_t)blockIdx.x * RT; r0 < n_rows; r0 += (int64_t)gridDim.x * RT) {
    const int nr = (int)min((int64_t)RT, n_rows - r0);
    __syncthreads();  // the previous tile's S / D are consumed
    for (int q = threadIdx.x; q < kMaxWindow * P; q += blockDim.x) {
      const int tau = q / P;
      const int pr = q - tau * P;
      const int rr = pr / nb, bb = pr - rr * nb;
      double2 S = make_double2(0.0, 0.0), D = make_double2(0.0, 0.0);
      if (tau < T && rr < nr) {
        const C* src = win.p[tau] + (r0 + rr) * ld;
        const C pv = ldg_c(src + bb);
        const C mv = ldg_c(src + nb + bb);
        S = make_double2((double)pv.x + (double)mv.x, (double)pv.y + (double)mv.y);
        D = make_double2((double)pv.x - (double)mv.x, (double)pv.y - (double)mv.y);
      }
      sS[q] = S;
      sD[q] = D;
    }
    __syncthreads();
    for (int nt = nt_first; nt < P / 4; nt += nt_step) {
      // B fragment: B[k = 4*s + t][n = g]; column g is pair 4*nt + g/2, part g&1
      const int pb = 4 * nt + (g >> 1);
      const bool im = g & 1;
      double bfr[8];
#pragma unroll
      for (int st = 0; st < 8; ++st) {
        const int k = 4 * st + t;
        if (k < 16) {
          const double2 S = sS[k * P + pb];
          bfr[st] = im ? S.y : S.x;
        } else {
          const double2 D = sD[(k - 16) * P + pb];
          bfr[st] = im ? D.x : -D.y;
        }
      }
      // C fragment: energy 8*mt + g, pair 4*nt + t (re, im)
      const int pc = 4 * nt + t;
      const int rr = pc / nb, bb = pc - rr * nb;
      const bool row_ok = rr < nr;
      double c0[kQeMmaMT], c1[kQeMmaMT];
#pragma unroll
      for (int m = 0; m < kQeMmaMT; ++m) {
        const int i = (mt0 + m) * 8 + g;
        c0[m] = c1[m] = 0.0;
        if (row_ok && i < n_en) {
          const C v = init ? wf0[(r0 + rr) * nb + bb] : qe[((r0 + rr) * n_en + i) * nb + bb];
          c0[m] = (double)v.x;
          c1[m] = (double)v.y;
        }
      }
#pragma unroll
      for (int m = 0; m < kQeMmaMT; ++m) {
        if (mt0 + m < n_mt) {
#pragma unroll
          for (int st = 0; st < 8; ++st) dmma_8x8x4(c0[m], c1[m], afr[m][st], bfr[st]);
        }
      }
#pragma unroll
      for (int m = 0; m < kQeMmaMT; ++m) {
        const int i = (mt0 + m) * 8 + g;
        if (row_ok && i < n_en) {
          C o;
          o.x = (R)c0[m];
          o.y = (R)c1[m];
          qe[((r0 + rr) * n_en + i) * nb + bb] = o;
        }
      }
    }
  }
}

// Tall-skinny reductions over orbitals: block partial sums of
// conj(u_tau[r][k*nb + b]) * QE[r][i][b] for tau < T, k in {0, 1} (mode 0), or
// of conj(wf0[r][b]) * QE[r][i][b] (mode 1, T = 1, k = 0).
// partials[((tau*K + k) * n_en*nb + ib) * 2 + {re,im}][block x].
// Block: qe_project_threads(n_en, nb, K) threads; thread t has k = t % K and
// owns the elements ib_lo + t / K + g * (blockDim.x / K), g < kQeG (one state
// b, kQeG energies); its T x kQeG accumulators stay in registers.
// Grid: x over row ranges of rows_per_tile, y over chunks of elements.  Each
// thread sums its rows in order.
template <typename R>
__global__ void __launch_bounds__(256, TBPM_QE_MINB_P) qe_project_kernel(
    const typename Cx<R>::t* qe, int64_t n_rows, int64_t rows_per_tile, int n_en, int nb,
    StatePtrs<R> u, int T, int mode, const typename Cx<R>::t* wf0, double* partials) {
  using C = typename Cx<R>::t;
  extern __shared__ double2 qsm[];
  const int64_t r0 = (int64_t)blockIdx.x * rows_per_tile;
  const int64_t r1 = min(r0 + rows_per_tile, n_rows);
  const int n_ib = n_en * nb;
  const int K = mode == 0 ? 2 : 1;
  const int ld = 2 * nb;
  const int RS = qe_tile_rows<R>(nb);
  const int NE = blockDim.x / K;  // threads per k, a multiple of nb
  const int EBE = kQeG * NE;      // elements of a row the block covers
  const int ib_lo = blockIdx.y * EBE;
  const int eb = min(EBE, n_ib - ib_lo);
  const int k = threadIdx.x % K;
  const int e = threadIdx.x / K;
  const int b = e % nb;
  bool act[kQeG];
#pragma unroll
  for (int g = 0; g < kQeG; ++g) act[g] = e + g * NE < eb;
  const int UW = kMaxProject * ld;  // staged values of one row
  constexpr bool conv = sizeof(R) == 4;
  double2* dbl = qsm;                                               // [RS][UW] (FP32 only)
  C* raw_u = reinterpret_cast<C*>(qsm + (conv ? RS * UW : 0));      // [2][RS][UW]
  C* raw_q = raw_u + 2 * RS * UW;                                   // [2][RS][EBE]
  auto issue = [&](int64_t rb, int buf) {
    const int nr = (int)min((int64_t)RS, r1 - rb);
    C* du = raw_u + buf * RS * UW;
    if (mode == 0) {
#pragma unroll
      for (int tau = 0; tau < kMaxProject; ++tau) {
        if (tau < T) {
          const C* src = u.p[tau] + rb * ld;
          for (int q = threadIdx.x; q < nr * ld; q += blockDim.x) {
            const int rr = q / ld;
            qe_cp_async(du + rr * UW + tau * ld + (q - rr * ld), src + q);
          }
        }
      }
    } else {
      for (int q = threadIdx.x; q < nr * nb; q += blockDim.x) {
        const int rr = q / nb;
        qe_cp_async(du + rr * UW + (q - rr * nb), wf0 + rb * nb + q);
      }
    }
    C* dq = raw_q + buf * RS * EBE;
    for (int q = threadIdx.x; q < nr * eb; q += blockDim.x) {
      const int rr = q / eb;
      const int ee = q - rr * eb;
      qe_cp_async(dq + rr * EBE + ee, qe + (rb + rr) * n_ib + ib_lo + ee);
    }
  };
  double ar[kMaxProject][kQeG], ai[kMaxProject][kQeG];
#pragma unroll
  for (int q = 0; q < kMaxProject; ++q)
#pragma unroll
    for (int g = 0; g < kQeG; ++g) ar[q][g] = ai[q][g] = 0.0;
  if (r0 < r1) issue(r0, 0);
  qe_cp_commit();
  int j = 0;
  for (int64_t rb = r0; rb < r1; rb += RS, ++j) {
    const int nr = (int)min((int64_t)RS, r1 - rb);
    qe_cp_wait_all();
    __syncthreads();  // tile j is in shared memory; tile j-1 is consumed
    if (rb + RS < r1) issue(rb + RS, (j + 1) & 1);
    qe_cp_commit();
    const C* tu = raw_u + (j & 1) * RS * UW;
    const C* tq = raw_q + (j & 1) * RS * EBE;
    if constexpr (conv) {
      const int per_row = mode == 0 ? T * ld : nb;
      for (int q = threadIdx.x; q < nr * per_row; q += blockDim.x) {
        const int rr = q / per_row;
        const int w = q - rr * per_row;
        const C v = tu[rr * UW + w];
        dbl[rr * UW + w] = make_double2((double)v.x, (double)v.y);
      }
      __syncthreads();
    }
    if (!act[0]) continue;
    for (int rr = 0; rr < nr; ++rr) {
      double qr[kQeG], qi[kQeG];
#pragma unroll
      for (int g = 0; g < kQeG; ++g) {
        const C qv = act[g] ? tq[rr * EBE + e + g * NE] : C{};
        qr[g] = (double)qv.x;
        qi[g] = (double)qv.y;
      }
      if (mode == 1) {
        double2 w;
        if constexpr (conv)
          w = dbl[rr * UW + b];
        else
          w = make_double2((double)tu[rr * UW + b].x, (double)tu[rr * UW + b].y);
#pragma unroll
        for (int g = 0; g < kQeG; ++g) {
          ar[0][g] += w.x * qr[g] + w.y * qi[g];
          ai[0][g] += w.x * qi[g] - w.y * qr[g];
        }
      } else {
#pragma unroll
        for (int tau = 0; tau < kMaxProject; ++tau) {
          if (tau < T) {
            const int o = rr * UW + tau * ld + k * nb + b;
            double2 w;
            if constexpr (conv)
              w = dbl[o];
            else
              w = make_double2((double)tu[o].x, (double)tu[o].y);
#pragma unroll
            for (int g = 0; g < kQeG; ++g) {
              ar[tau][g] += w.x * qr[g] + w.y * qi[g];
              ai[tau][g] += w.x * qi[g] - w.y * qr[g];
            }
          }
        }
      }
    }
  }
#pragma unroll
  for (int g = 0; g < kQeG; ++g) {
    if (!act[g]) continue;
    const int ib = ib_lo + e + g * NE;
#pragma unroll
    for (int tau = 0; tau < kMaxProject; ++tau) {
      if (tau < (mode == 0 ? T : 1)) {
        const int64_t o = (int64_t)(tau * K + k) * n_ib + ib;
        partials[(o * 2 + 0) * gridDim.x + blockIdx.x] = ar[tau][g];
        partials[(o * 2 + 1) * gridDim.x + blockIdx.x] = ai[tau][g];
      }
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
