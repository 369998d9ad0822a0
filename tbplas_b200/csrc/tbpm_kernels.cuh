// TBPM device kernels (sm_100a).  All kernels are bandwidth-bound CSR / vector
// passes; none of them uses tensor cores.
//
//  cheb_term_kernel   one term of a three-term Chebyshev recurrence over a block
//                     of ld right-hand sides:  p_k = alpha*(H p_{k-1}) + beta*p_{k-2},
//                     with the Bessel/Fermi-weighted accumulation of up to three
//                     pending terms into the accumulator (the new state) and,
//                     on the last term of a time step, the correlation
//                     <ref|psi> and norm <psi|psi> per column (block partials).
//                     Replaces propagation.f90:12-82 + csr.F90:104-322 +
//                     math.F90:578-700 + the inner_prod calls of tbpm.f90.
//  finalize_kernel    fixed-order sum of block partials into out[step] (a
//                     device-side step counter makes the launch graph-replayable).
//  corr_kernel        <ref|x> and <x|x> per column (tbpm.f90:58 corr(0) etc.).
//  gen_state_kernel   Philox4x32-10 random states (random.f90:36-69 distribution).
//  current_apply_kernel  J_x psi, J_y psi with J = i*rescale*hop*dr built on the fly
//                     (funcs.f90:12-33 + csr.F90:71-101).
//  jcorr_kernel       the four AC correlations <psi2|J_b psi1_a> (tbpm.f90:320-327).
#pragma once

#include "tbpm_common.cuh"

namespace tbpm {

constexpr int kMaxCols = 64;

struct TermCoef {
  double alpha_re, alpha_im;  // multiplier of H*p_{k-1} (columns not in neg_mask)
  double beta;                // multiplier of p_{k-2}
  double w[2][3];             // flush weights [set][p_{k-2}, p_{k-1}, p_k]
  unsigned long long neg_mask;  // column c uses -alpha
  unsigned long long set_mask;  // column c uses weight set 1
  int nflush;                 // number of pending terms flushed (0..3)
  int acc_init;               // 1: acc = sum, 0: acc += sum
};

template <typename R, int V>
struct TermArgs {
  const int32_t* indptr;   // off-diagonal CSR of H
  const int32_t* indices;
  const typename Cx<R>::t* hop;
  const typename Cx<R>::t* diag;  // diagonal of H (null: none)
  int64_t n_rows;
  int64_t rows_per_tile;  // unused by the grid-stride kernels (kept for layout)
  int tpr;  // threads (packs) per row = ld / V
  const Pack<R, V>* gather;  // p_{k-1}
  const Pack<R, V>* pin;     // p_{k-2} (null when beta == 0)
  Pack<R, V>* pout;          // destination of p_k (null: not stored)
  Pack<R, V>* acc;           // accumulator (null when nflush == 0)
  const Pack<R, V>* ref;     // correlation reference (null: no partials)
  int ref_tpr;               // packs per row of ref; lanes >= ref_tpr correlate to 0
  double* partials;          // [(col*3 + v) * gridDim.x + block]
  TermCoef c;
};

// Kernel modes: 0 = recurrence only, 1 = recurrence + accumulator flush,
// 2 = flush + correlation/norm partials (last term of a time step).  Each
// mode is compiled separately so the common mode-0 terms keep few registers.
// Blocks have at most 256 threads; the minimum resident blocks per SM bound
// the registers per thread (4 blocks: 64 registers).
// (measured on B200: FP64 is fastest at 4 resident blocks in every mode, the
// FP32 recurrence-only mode at 5)
#ifndef TBPM_MINB_PLAIN_F64
#define TBPM_MINB_PLAIN_F64 4
#endif
#ifndef TBPM_MINB_PLAIN_F32
#define TBPM_MINB_PLAIN_F32 5
#endif
#ifndef TBPM_MINB_FLUSH
#define TBPM_MINB_FLUSH 4
#endif

// 32 bytes of state per thread (two complex128 or four complex64) hold twice
// the data in registers
#ifndef TBPM_MINB_F64_V2
#define TBPM_MINB_F64_V2 2
#endif
// (measured on B200: the FP32 recurrence-only mode is 2.5% faster at 3 resident
// blocks, 85 registers; FP64 is 5% slower there)
#ifndef TBPM_MINB_V32_PLAIN_F32
#define TBPM_MINB_V32_PLAIN_F32 3
#endif

template <typename R, int MODE, int V = 1>
struct TermBounds {
  static constexpr int min_blocks =
      sizeof(R) * V == 16
          ? (MODE == 0 ? (sizeof(R) == 8 ? TBPM_MINB_F64_V2 : TBPM_MINB_V32_PLAIN_F32)
                       : TBPM_MINB_F64_V2)
          : (MODE == 0 ? (sizeof(R) == 8 ? TBPM_MINB_PLAIN_F64 : TBPM_MINB_PLAIN_F32)
                       : TBPM_MINB_FLUSH);
};
// independent gathers issued per batch
#ifndef TBPM_BW
#define TBPM_BW 2
#endif
// L2 prefetch distance in sweep iterations (0: off)
#ifndef TBPM_PF_DIST
#define TBPM_PF_DIST 1
#endif

// Bulk prefetch of [p, p + bytes) into L2 (sm_90+ cp.async.bulk.prefetch);
// the range is trimmed to 16-byte granularity and to [lo, hi).
__device__ __forceinline__ void prefetch_l2(const void* p, int64_t bytes, const void* lo,
                                            const void* hi) {
  uintptr_t a = reinterpret_cast<uintptr_t>(p);
  uintptr_t e = a + (uintptr_t)bytes;
  const uintptr_t l = reinterpret_cast<uintptr_t>(lo), h = reinterpret_cast<uintptr_t>(hi);
  if (a < l) a = l;
  if (e > h) e = h;
  a = (a + 15) & ~(uintptr_t)15;
  e = e & ~(uintptr_t)15;
  if (e <= a) return;
  const uint32_t sz = (uint32_t)(e - a);
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"(sz) : "memory");
}

template <typename R, int V, int MODE>
__global__ void __launch_bounds__(256, (TermBounds<R, MODE, V>::min_blocks))
    cheb_term_kernel(const TermArgs<R, V> a) {
  extern __shared__ double smem[];
  constexpr int BW = TBPM_BW;
  const int tpr = a.tpr;
  const int slot = threadIdx.x / tpr;
  const int lane = threadIdx.x - slot * tpr;
  const int rpp = blockDim.x / tpr;
  // Persistent grid-stride schedule over row tiles of rpp rows: the resident
  // blocks sweep one narrow band of rows together, so the neighbour rows of
  // the gathered vector p_{k-1} are still in L2 when they are needed again.
  const int64_t stride = (int64_t)gridDim.x * rpp;
  // per-column selectors; the coefficients themselves stay in the parameter
  // bank and are picked at their point of use (keeps registers free)
  const unsigned neg_bits = (unsigned)(a.c.neg_mask >> (lane * V)) & ((1u << V) - 1u);
  const unsigned set_bits = (unsigned)(a.c.set_mask >> (lane * V)) & ((1u << V) - 1u);
  const R beta = (R)a.c.beta;
  const int nflush = MODE >= 1 ? a.c.nflush : 0;
  constexpr bool do_corr = MODE == 2;
  const bool ref_lane = do_corr && a.ref != nullptr && lane < a.ref_tpr;
  const bool need_own = a.diag != nullptr || nflush >= 2;

  double cre[V], cim[V], nrm[V];
#pragma unroll
  for (int v = 0; v < V; ++v) cre[v] = cim[v] = nrm[v] = 0.0;

  const int64_t row_bytes = (int64_t)tpr * sizeof(Pack<R, V>);
  const char* gather_end = reinterpret_cast<const char*>(a.gather + a.n_rows * tpr);
  for (int64_t r0 = (int64_t)blockIdx.x * rpp; r0 < a.n_rows; r0 += stride) {
    if (TBPM_PF_DIST > 0 && threadIdx.x == 0) {
      // the streamed tiles of this block TBPM_PF_DIST sweep iterations ahead:
      // their DRAM reads are in flight without holding registers
      const int64_t rp = r0 + TBPM_PF_DIST * stride;
      if (rp < a.n_rows) {
        const int64_t tile = (int64_t)rpp * row_bytes;
        const char* g = reinterpret_cast<const char*>(a.gather);
        prefetch_l2(g + rp * row_bytes, tile, g, gather_end);
        if (a.pin) {
          const char* p = reinterpret_cast<const char*>(a.pin);
          prefetch_l2(p + rp * row_bytes, tile, p, p + a.n_rows * row_bytes);
        }
        if (MODE >= 1 && !a.c.acc_init) {
          const char* q = reinterpret_cast<const char*>(a.acc);
          prefetch_l2(q + rp * row_bytes, tile, q, q + a.n_rows * row_bytes);
        }
      }
    }
    const int64_t r = r0 + slot;
    if (r >= a.n_rows) continue;
    const int64_t e = r * tpr + lane;
    Pack<R, V> pm2;
    if (a.pin) {
      pm2 = ldcs_pack(a.pin + e);
    } else {
#pragma unroll
      for (int k = 0; k < 2 * V; ++k) pm2.v[k] = (R)0;
    }
    Pack<R, V> own;
    if (need_own) own = ldg_pack(a.gather + e);
    const int j0 = __ldg(a.indptr + r);
    const int j1 = __ldg(a.indptr + r + 1);
    R sre[V], sim[V];
    if (a.diag) {
      const typename Cx<R>::t d = ldg_c(a.diag + r);
#pragma unroll
      for (int v = 0; v < V; ++v) {
        sre[v] = d.x * own.v[2 * v] - d.y * own.v[2 * v + 1];
        sim[v] = d.x * own.v[2 * v + 1] + d.y * own.v[2 * v];
      }
    } else {
#pragma unroll
      for (int v = 0; v < V; ++v) sre[v] = sim[v] = (R)0;
    }
    // off-diagonal neighbours in batches of BW independent gathers
    for (int jb = j0; jb < j1; jb += BW) {
      int cidx[BW];
      typename Cx<R>::t h[BW];
#pragma unroll
      for (int u = 0; u < BW; ++u) {
        if (jb + u < j1) {
          cidx[u] = __ldg(a.indices + jb + u);
          h[u] = ldg_c(a.hop + jb + u);
        } else {
          cidx[u] = -1;
        }
      }
      Pack<R, V> x[BW];
#pragma unroll
      for (int u = 0; u < BW; ++u)
        if (cidx[u] >= 0) x[u] = ldg_pack(a.gather + (int64_t)cidx[u] * tpr + lane);
#pragma unroll
      for (int u = 0; u < BW; ++u) {
        if (cidx[u] >= 0) {
#pragma unroll
          for (int v = 0; v < V; ++v) {
            sre[v] = fma(h[u].x, x[u].v[2 * v], fma(-h[u].y, x[u].v[2 * v + 1], sre[v]));
            sim[v] = fma(h[u].x, x[u].v[2 * v + 1], fma(h[u].y, x[u].v[2 * v], sim[v]));
          }
        }
      }
    }
    Pack<R, V> pk;
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const bool neg = (neg_bits >> v) & 1u;
      const R ar = (R)(neg ? -a.c.alpha_re : a.c.alpha_re);
      const R ai = (R)(neg ? -a.c.alpha_im : a.c.alpha_im);
      pk.v[2 * v] = fma(ar, sre[v], fma(-ai, sim[v], beta * pm2.v[2 * v]));
      pk.v[2 * v + 1] = fma(ar, sim[v], fma(ai, sre[v], beta * pm2.v[2 * v + 1]));
    }
    if (nflush > 0) {
      Pack<R, V> acc;
      if (!a.c.acc_init) acc = ldcs_pack(a.acc + e);
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const int set = (set_bits >> v) & 1u;
        const double w0 = set ? a.c.w[1][0] : a.c.w[0][0];
        const double w1 = set ? a.c.w[1][1] : a.c.w[0][1];
        const double w2 = set ? a.c.w[1][2] : a.c.w[0][2];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const int k = 2 * v + q;
          double t = a.c.acc_init ? 0.0 : (double)acc.v[k];
          if (nflush >= 3) t += w0 * (double)pm2.v[k];
          if (nflush >= 2) t += w1 * (double)own.v[k];
          t += w2 * (double)pk.v[k];
          acc.v[k] = (R)t;
        }
      }
      stcs_pack(a.acc + e, acc);
      if (do_corr) {
        Pack<R, V> rf;
        if (ref_lane) rf = ldcs_pack(a.ref + r * a.ref_tpr + lane);
#pragma unroll
        for (int v = 0; v < V; ++v) {
          const double xr = (double)acc.v[2 * v], xi = (double)acc.v[2 * v + 1];
          if (ref_lane) {
            const double fr = (double)rf.v[2 * v], fi = (double)rf.v[2 * v + 1];
            cre[v] += fr * xr + fi * xi;
            cim[v] += fr * xi - fi * xr;
          }
          nrm[v] += xr * xr + xi * xi;
        }
      }
    }
    if (a.pout) stcs_pack(a.pout + e, pk);
  }

  if (do_corr) {
    const int width = tpr * V * 3;
#pragma unroll
    for (int v = 0; v < V; ++v) {
      double* s = smem + slot * width + (lane * V + v) * 3;
      s[0] = cre[v];
      s[1] = cim[v];
      s[2] = nrm[v];
    }
    __syncthreads();
    tree_reduce_slots(smem, rpp, width, slot, lane, tpr);
    if (slot == 0) {
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const int col = lane * V + v;
#pragma unroll
        for (int q = 0; q < 3; ++q)
          a.partials[(int64_t)(col * 3 + q) * gridDim.x + blockIdx.x] = smem[col * 3 + q];
      }
    }
  }
}

// Sum block partials laid out as [value][n_blocks] into out[step][value];
// block b handles value b.  The last block to finish advances *step.
static __global__ void __launch_bounds__(256) finalize_kernel(const double* partials, int n_blocks,
                                                       int n_values, int* step,
                                                       unsigned int* done, double* out) {
  __shared__ double red[256];
  const int val = blockIdx.x;
  const double* p = partials + (int64_t)val * n_blocks;
  double s = 0.0;
  for (int i = threadIdx.x; i < n_blocks; i += blockDim.x) s += p[i];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  __shared__ int st;
  if (threadIdx.x == 0) {
    st = *((volatile int*)step);
    out[(int64_t)st * n_values + val] = red[0];
    __threadfence();
    const unsigned int prev = atomicAdd(done, 1u);
    if (prev == (unsigned int)n_values - 1) {
      *done = 0u;
      *step = st + 1;
      __threadfence();
    }
  }
}

// <ref|x> and <x|x> per column: partials [(col*3 + v) * grid + block].
template <typename R, int V>
__global__ void __launch_bounds__(512) corr_kernel(const Pack<R, V>* x, const Pack<R, V>* ref,
                                                   int64_t n_rows, int64_t rows_per_tile,
                                                   int tpr, int ref_tpr, double* partials) {
  extern __shared__ double smem[];
  const int slot = threadIdx.x / tpr;
  const int lane = threadIdx.x - slot * tpr;
  const int rpp = blockDim.x / tpr;
  (void)rows_per_tile;  // grid-stride over row tiles of rpp rows
  const bool ref_lane = ref != nullptr && lane < ref_tpr;
  double cre[V], cim[V], nrm[V];
#pragma unroll
  for (int v = 0; v < V; ++v) cre[v] = cim[v] = nrm[v] = 0.0;
  for (int64_t r = (int64_t)blockIdx.x * rpp + slot; r < n_rows;
       r += (int64_t)gridDim.x * rpp) {
    const Pack<R, V> xv = ldg_pack(x + r * tpr + lane);
    Pack<R, V> rf;
    if (ref_lane) rf = ldg_pack(ref + r * ref_tpr + lane);
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const double xr = (double)xv.v[2 * v], xi = (double)xv.v[2 * v + 1];
      if (ref_lane) {
        const double fr = (double)rf.v[2 * v], fi = (double)rf.v[2 * v + 1];
        cre[v] += fr * xr + fi * xi;
        cim[v] += fr * xi - fi * xr;
      }
      nrm[v] += xr * xr + xi * xi;
    }
  }
  const int width = tpr * V * 3;
#pragma unroll
  for (int v = 0; v < V; ++v) {
    double* s = smem + slot * width + (lane * V + v) * 3;
    s[0] = cre[v];
    s[1] = cim[v];
    s[2] = nrm[v];
  }
  __syncthreads();
  tree_reduce_slots(smem, rpp, width, slot, lane, tpr);
  if (slot == 0) {
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const int col = lane * V + v;
#pragma unroll
      for (int q = 0; q < 3; ++q)
        partials[(int64_t)(col * 3 + q) * gridDim.x + blockIdx.x] = smem[col * 3 + q];
    }
  }
}

// ---------------------------------------------------------------------------
// Philox4x32-10 counter-based generator (Salmon et al., SC'11): 10 rounds with
// multipliers 0xD2511F53 / 0xCD9E8D57 and Weyl key increments 0x9E3779B9 /
// 0xBB67AE85.  Counter = (element index lo, hi, 0x5442504D, 0), key = the
// 64-bit stream key.  Two 53-bit uniforms per element: f from words 0-1, g from
// words 2-3.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void philox_uniform_pair(int64_t key, int64_t j, double* f,
                                                    double* g) {
  uint32_t c0 = (uint32_t)(uint64_t)j, c1 = (uint32_t)((uint64_t)j >> 32);
  uint32_t c2 = 0x5442504Du, c3 = 0u;
  uint32_t k0 = (uint32_t)(uint64_t)key, k1 = (uint32_t)((uint64_t)key >> 32);
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
    const uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
    const uint32_t n0 = hi1 ^ c1 ^ k0;
    const uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  const double s = 1.0 / 9007199254740992.0;
  *f = ((double)(c0 >> 5) * 67108864.0 + (double)(c1 >> 6)) * s;
  *g = ((double)(c2 >> 5) * 67108864.0 + (double)(c3 >> 6)) * s;
}

struct StateKeys {
  long long key[kMaxCols];  // stream key per column (iseed * 49741)
};

// mode 0: partial sums of |z|^2 per column ([col * grid + block]).
// mode 1: write z / sqrt(sum[col]) into out (row-interleaved, ld = tpr*V).
template <typename R, int V>
__global__ void __launch_bounds__(512) gen_state_kernel(StateKeys keys, int kind,
                                                        int64_t n_rows, int64_t rows_per_tile,
                                                        int tpr, int mode, const double* sums,
                                                        int sums_stride, Pack<R, V>* out,
                                                        double* partials) {
  extern __shared__ double smem[];
  const int slot = threadIdx.x / tpr;
  const int lane = threadIdx.x - slot * tpr;
  const int rpp = blockDim.x / tpr;
  (void)rows_per_tile;  // grid-stride over row tiles of rpp rows
  const double two_pi = 6.283185307179586476925286766559;
  double acc[V];
  double den[V];
#pragma unroll
  for (int v = 0; v < V; ++v) {
    acc[v] = 0.0;
    den[v] = mode == 1 ? sqrt(sums[(int64_t)(lane * V + v) * sums_stride]) : 1.0;
  }
  for (int64_t r = (int64_t)blockIdx.x * rpp + slot; r < n_rows;
       r += (int64_t)gridDim.x * rpp) {
    Pack<R, V> o;
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const int col = lane * V + v;
      double f, g;
      philox_uniform_pair(keys.key[col], r, &f, &g);
      const double az2 = kind == 0 ? -1.0 * log(1.0 - f) : 1.0;
      if (mode == 0) {
        acc[v] += az2;
      } else {
        double sn, cs;
        sincos(two_pi * g, &sn, &cs);
        const double m = sqrt(az2);
        o.v[2 * v] = (R)((m * cs) / den[v]);
        o.v[2 * v + 1] = (R)((m * sn) / den[v]);
      }
    }
    if (mode == 1) out[r * tpr + lane] = o;
  }
  if (mode == 0) {
    const int width = tpr * V;
#pragma unroll
    for (int v = 0; v < V; ++v) smem[slot * width + lane * V + v] = acc[v];
    __syncthreads();
    tree_reduce_slots(smem, rpp, width, slot, lane, tpr);
    if (slot == 0) {
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const int col = lane * V + v;
        partials[(int64_t)col * gridDim.x + blockIdx.x] = smem[col];
      }
    }
  }
}

// AC set-up (tbpm.f90:277-281): for a block of B states wf0 [N][B], build the
// 3B-column block [J_x wf0 | J_y wf0 | wf0] where J_d = i*rescale*hop*d.
// One thread per (row, state); V = 1.
template <typename R>
__global__ void __launch_bounds__(512) current_apply_kernel(
    const int32_t* indptr, const int32_t* indices, const typename Cx<R>::t* hop,
    const R* dx, const R* dy, double rescale, int64_t n_rows, int B,
    const typename Cx<R>::t* wf0, typename Cx<R>::t* out) {
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= n_rows * B) return;
  const int64_t r = gid / B;
  const int b = (int)(gid - r * B);
  const R s = (R)rescale;
  R xr = 0, xi = 0, yr = 0, yi = 0;
  const int j0 = __ldg(indptr + r), j1 = __ldg(indptr + r + 1);
  for (int j = j0; j < j1; ++j) {
    const int c = __ldg(indices + j);
    const typename Cx<R>::t h = ldg_c(hop + j);
    // (i*s)*h = (-s*h.im, s*h.re); times dr
    const R jr = -s * h.y, ji = s * h.x;
    const R ddx = __ldg(dx + j), ddy = __ldg(dy + j);
    const typename Cx<R>::t w = ldg_c(wf0 + (int64_t)c * B + b);
    const R axr = jr * ddx, axi = ji * ddx, ayr = jr * ddy, ayi = ji * ddy;
    xr = fma(axr, w.x, fma(-axi, w.y, xr));
    xi = fma(axr, w.y, fma(axi, w.x, xi));
    yr = fma(ayr, w.x, fma(-ayi, w.y, yr));
    yi = fma(ayr, w.y, fma(ayi, w.x, yi));
  }
  const int64_t o = r * 3 * B;
  typename Cx<R>::t vx, vy;
  vx.x = xr;
  vx.y = xi;
  vy.x = yr;
  vy.y = yi;
  out[o + b] = vx;
  out[o + B + b] = vy;
  out[o + 2 * B + b] = wf0[r * B + b];
}

// AC correlations (tbpm.f90:320-327) for the 3B-column block
// psi = [psi1_x | psi1_y | psi2]: per state b the values
//   <psi2|J_x psi1_x>, <psi2|J_y psi1_x>, <psi2|J_x psi1_y>, <psi2|J_y psi1_y>
// and <psi2|psi2>; partials [(b*9 + v) * grid + block], v = re/im pairs then norm.
template <typename R>
#ifndef TBPM_JCORR_JB
#define TBPM_JCORR_JB 4  // neighbour entries whose loads are issued together
#endif
#ifndef TBPM_JCORR_MINB
#define TBPM_JCORR_MINB 2  // resident 256-thread blocks per SM the registers are bounded for
#endif
__global__ void __launch_bounds__(256, TBPM_JCORR_MINB) jcorr_kernel(
    const int32_t* indptr, const int32_t* indices, const typename Cx<R>::t* hop,
    const R* dx, const R* dy, double rescale, int64_t n_rows, int64_t rows_per_tile, int B,
    const typename Cx<R>::t* psi, double* partials) {
  extern __shared__ double smem[];
  const int tpr = B;
  const int slot = threadIdx.x / tpr;
  const int b = threadIdx.x - slot * tpr;
  const int rpp = blockDim.x / tpr;
  (void)rows_per_tile;  // grid-stride over row tiles of rpp rows
  const R s = (R)rescale;
  const int ld = 3 * B;
  double acc[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) acc[k] = 0.0;
  for (int64_t r = (int64_t)blockIdx.x * rpp + slot; r < n_rows;
       r += (int64_t)gridDim.x * rpp) {
    R xxr = 0, xxi = 0, yxr = 0, yxi = 0, xyr = 0, xyi = 0, yyr = 0, yyi = 0;
    const int j0 = __ldg(indptr + r), j1 = __ldg(indptr + r + 1);
    const typename Cx<R>::t p2 = ldg_c(psi + r * ld + 2 * B + b);
    // neighbours in batches of JB: every load of a batch is issued before the
    // first product, so the gathers overlap (the products keep the entry order)
    constexpr int JB = TBPM_JCORR_JB;
    for (int jb = j0; jb < j1; jb += JB) {
      int cc[JB];
      typename Cx<R>::t hh[JB];
      R ddx[JB], ddy[JB];
#pragma unroll
      for (int u = 0; u < JB; ++u) {
        cc[u] = -1;
        if (jb + u < j1) {
          cc[u] = __ldg(indices + jb + u);
          hh[u] = ldg_c(hop + jb + u);
          ddx[u] = __ldg(dx + jb + u);
          ddy[u] = __ldg(dy + jb + u);
        }
      }
      typename Cx<R>::t p1x[JB], p1y[JB];
#pragma unroll
      for (int u = 0; u < JB; ++u)
        if (cc[u] >= 0) {
          p1x[u] = ldg_c(psi + (int64_t)cc[u] * ld + b);
          p1y[u] = ldg_c(psi + (int64_t)cc[u] * ld + B + b);
        }
#pragma unroll
      for (int u = 0; u < JB; ++u) {
        if (cc[u] < 0) continue;
        const R jr = -s * hh[u].y, ji = s * hh[u].x;
        const R axr = jr * ddx[u], axi = ji * ddx[u], ayr = jr * ddy[u], ayi = ji * ddy[u];
        // J_x psi1_x, J_y psi1_x, J_x psi1_y, J_y psi1_y
        xxr = fma(axr, p1x[u].x, fma(-axi, p1x[u].y, xxr));
        xxi = fma(axr, p1x[u].y, fma(axi, p1x[u].x, xxi));
        yxr = fma(ayr, p1x[u].x, fma(-ayi, p1x[u].y, yxr));
        yxi = fma(ayr, p1x[u].y, fma(ayi, p1x[u].x, yxi));
        xyr = fma(axr, p1y[u].x, fma(-axi, p1y[u].y, xyr));
        xyi = fma(axr, p1y[u].y, fma(axi, p1y[u].x, xyi));
        yyr = fma(ayr, p1y[u].x, fma(-ayi, p1y[u].y, yyr));
        yyi = fma(ayr, p1y[u].y, fma(ayi, p1y[u].x, yyi));
      }
    }
    const double qr = (double)p2.x, qi = (double)p2.y;
    // conj(p2) * v
    acc[0] += qr * (double)xxr + qi * (double)xxi;
    acc[1] += qr * (double)xxi - qi * (double)xxr;
    acc[2] += qr * (double)yxr + qi * (double)yxi;
    acc[3] += qr * (double)yxi - qi * (double)yxr;
    acc[4] += qr * (double)xyr + qi * (double)xyi;
    acc[5] += qr * (double)xyi - qi * (double)xyr;
    acc[6] += qr * (double)yyr + qi * (double)yyi;
    acc[7] += qr * (double)yyi - qi * (double)yyr;
    acc[8] += qr * qr + qi * qi;
  }
  const int width = tpr * 9;
#pragma unroll
  for (int k = 0; k < 9; ++k) smem[slot * width + b * 9 + k] = acc[k];
  __syncthreads();
  tree_reduce_slots(smem, rpp, width, slot, b, tpr);
  if (slot == 0) {
#pragma unroll
    for (int k = 0; k < 9; ++k)
      partials[(int64_t)(b * 9 + k) * gridDim.x + blockIdx.x] = smem[b * 9 + k];
  }
}

}  // namespace tbpm
