// Chebyshev term with its streamed operands staged in shared memory by bulk
// copies (sm_100a): cheb_ring_kernel.
//
// The term computes the same values in the same order as cheb_term_kernel
// (tbpm_kernels.cuh): p_k = alpha*(H p_{k-1}) + beta*p_{k-2}, H = D + O, with the
// deferred Bessel/Fermi-weighted flush of up to three pending terms into the
// accumulator and, in MODE 2, the <ref|psi> / <psi|psi> block partials.  Only
// the way the operands reach the threads differs.
//
// A block is one producer warp and kRingConsumerWarps consumer warps.  The
// persistent grid walks row tiles grid-stride; tile i of a block goes to stage
// i % S of a ring of S shared-memory stages.  For each tile the producer warp
// issues 1-D bulk copies (cp.async.bulk global -> shared, completion counted in
// bytes on the stage's "full" mbarrier) of
//   * the tile's CSR slice: indptr, and the indices and hopping values of its
//     off-diagonal entries (when they fit the stage; else the consumers read
//     them from global memory),
//   * the diagonal D of its rows,
//   * its rows of p_{k-2}, of p_{k-1} (the row's own values) and of the
//     accumulator (flush terms that add to it).
// The copies of up to S-1 tiles are in flight at once and hold no registers:
// the DRAM latency of every streamed operand is off the consumers' critical
// path.  A consumer thread owns V columns of one row: it reads its CSR entries
// from shared memory, gathers the neighbour rows of p_{k-1} from global memory
// (they are L2 hits: the whole grid sweeps one band of rows), combines them
// with the staged operands and stores p_k and the accumulator.  Each consumer
// warp then arrives on the stage's "empty" mbarrier, which the producer waits
// for before reusing the stage.
//
// Every wait is bounded in time (kRingWaitNs).  A wait that runs out sets bit
// 0 of *status and the block stops; the producer then waits (bounded) for
// the copies it has issued before it leaves, so no copy lands in the shared
// memory of a block that has ended.  The host reads the status word at its
// next synchronisation and reports TBPM_ERR_TIMEOUT.
//
// Copy alignment (cp.async.bulk: 16-byte addresses and sizes): every window is
// widened to 16-byte boundaries.  The widened windows stay inside the
// allocations because device buffers are allocated in multiples of 256 bytes.
// A row of the state block must be a multiple of 16 bytes (FP64 always; FP32
// needs an even block width); the host uses cheb_term_kernel otherwise.
#pragma once

#include "tbpm_kernels.cuh"

namespace tbpm {

// (measured on B200, 2048^2 graphene, 16 states: 15 consumer warps in one block
// per SM beat 7 in two, 11 in one, 5 in three and 3 in four)
#ifndef TBPM_RING_WARPS
#define TBPM_RING_WARPS 15  // consumer warps per block
#endif
#ifndef TBPM_RING_MINB
#define TBPM_RING_MINB 1  // resident blocks per SM the stages are sized for
#endif
#ifndef TBPM_RING_STAGES
#define TBPM_RING_STAGES 3  // most stages per ring (measured on B200: 3 beats 4-8)
#endif
#ifndef TBPM_RING_LOCAL
#define TBPM_RING_LOCAL 0  // 1: neighbours inside the tile read from its staged p_{k-1} rows
#endif
#ifndef TBPM_RING_EVICT
#define TBPM_RING_EVICT 0  // 1: bulk copies of p_{k-2} and the accumulator marked evict-first in L2
#endif
constexpr int kRingConsumerWarps = TBPM_RING_WARPS;
constexpr int kRingConsumers = kRingConsumerWarps * 32;
constexpr int kRingThreads = kRingConsumers + 32;
constexpr int kRingMaxStages = TBPM_RING_STAGES;
constexpr int kRingMinBlocks = TBPM_RING_MINB;
constexpr unsigned long long kRingWaitNs = 2000000000ull;  // 2 s per wait
#ifndef TBPM_RING_GATHER
#define TBPM_RING_GATHER 3  // neighbour gathers issued together (measured: 3 beats 4)
#endif

// Shared-memory layout of one stage (byte offsets, 128-byte aligned parts)
// and the ring.  Offsets of absent parts are -1.
struct RingShape {
  int rows;         // rows per tile
  int stages;       // S
  int cap;          // CSR entries a stage holds (multiple of 4)
  int pin_off, own_off, acc_off, diag_off, ip_off, ix_off, hop_off;
  int hdr_off;      // window layouts: the stage's window table (kRingWinHdr bytes)
  int win_off;      // window layouts: rows of p_{k-1} covering the tile's columns
  int win_rows;     // window layouts: rows the window region holds
  int ref_off;      // MODE 2: rows of the correlation reference (-1: read from global)
  int stage_bytes;  // one stage
  int bar_off;      // 2*S mbarriers (full[S], empty[S]) after the stages
  int smem_bytes;   // total dynamic shared memory
};

template <typename R, int V>
struct RingArgs {
  TermArgs<R, V> t;
  RingShape s;
  unsigned int* status;  // bit 0: a bounded wait ran out
  const int* win;        // WIN kernels: per tile kRingWinInts ints (ring_window_kernel)
};

// Row windows (the WIN kernels): a tile's off-diagonal columns and its own
// rows are covered by at most kRingWinMax row ranges of p_{k-1}, staged into
// the stage's window region by bulk copies; the consumers read every operand
// from shared memory.  Record per tile: [0] = number of windows | (gather
// flag << 8), then (first row, row count) per window.  A tile whose columns do
// not fit (more windows, or more rows than the region) stages its own rows as
// its one window and gathers the neighbours from global memory.
constexpr int kRingWinMax = 4;
constexpr int kRingWinInts = 12;   // record size (3 x int4)
constexpr int kRingWinHdr = 64;    // stage table: flags, lo[4], base[4]
constexpr int kRingWinGap = 8;     // rows between two column runs merged into one window

__device__ __forceinline__ uint32_t ring_smem(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long ring_clock_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void ring_bar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void ring_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void ring_arrive_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}

// 1-D bulk copy of `bytes` (multiple of 16) from global `src` (16-byte aligned)
// to shared `dst`; completion is counted on mbarrier `bar`.
__device__ __forceinline__ void ring_copy(uint32_t dst, const void* src, uint32_t bytes,
                                          uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}

// The same copy with an L2 eviction-priority policy (createpolicy).
__device__ __forceinline__ void ring_copy_hint(uint32_t dst, const void* src, uint32_t bytes,
                                               uint32_t bar, uint64_t policy) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint "
      "[%0], [%1], %2, [%3], %4;" ::"r"(dst),
      "l"(src), "r"(bytes), "r"(bar), "l"(policy)
      : "memory");
}

__device__ __forceinline__ uint64_t ring_evict_first_policy() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}

// Wait for the phase of parity `parity` of mbarrier `bar`, at most kRingWaitNs.
__device__ __forceinline__ bool ring_wait(uint32_t bar, uint32_t parity) {
  const unsigned long long t0 = ring_clock_ns();
  for (;;) {
    for (int i = 0; i < 64; ++i) {
      uint32_t ok;
      asm volatile(
          "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
          " selp.u32 %0, 1, 0, p;\n}\n"
          : "=r"(ok)
          : "r"(bar), "r"(parity)
          : "memory");
      if (ok) return true;
    }
    if (ring_clock_ns() - t0 > kRingWaitNs) return false;
  }
}

template <typename R, int V>
__device__ __forceinline__ Pack<R, V> lds_pack(const char* p) {
  return *reinterpret_cast<const Pack<R, V>*>(p);
}

template <typename R, int V, int MODE, bool WIN>
__global__ void __launch_bounds__(kRingThreads, kRingMinBlocks)
    cheb_ring_kernel(const __grid_constant__ RingArgs<R, V> ra) {
  using C = typename Cx<R>::t;
  extern __shared__ __align__(128) char rsm[];
  const TermArgs<R, V>& a = ra.t;
  const RingShape& sh = ra.s;
  const int S = sh.stages;
  const int TR = sh.rows;
  const int64_t n = a.n_rows;
  const int tpr = a.tpr;
  const int tid = threadIdx.x;
  const uint32_t full0 = ring_smem(rsm + sh.bar_off);
  const uint32_t empty0 = full0 + 8u * (uint32_t)S;
  const int nflush = MODE >= 1 ? a.c.nflush : 0;
  const bool need_own = a.diag != nullptr || nflush >= 2;
  const bool add_acc = nflush > 0 && !a.c.acc_init;
  const int64_t row_bytes = (int64_t)tpr * sizeof(Pack<R, V>);
  const bool ref_staged = MODE == 2 && a.ref != nullptr && sh.ref_off >= 0;

  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      ring_bar_init(full0 + 8u * s, 1);
      ring_bar_init(empty0 + 8u * s, kRingConsumerWarps);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  double cre[V], cim[V], nrm[V];
#pragma unroll
  for (int v = 0; v < V; ++v) cre[v] = cim[v] = nrm[v] = 0.0;
  const int slot = tid / tpr;
  const int lane = tid - slot * tpr;

  if (tid >= kRingConsumers) {
    // ---------------- producer warp ----------------
    const int wl = tid & 31;
    int64_t issued = 0;
    bool ok = true;
    // CSR bounds of the next 32 tiles, one tile per lane, loaded a batch ahead
    auto bounds = [&](int64_t i, int* b0, int* b1) {
      const int64_t r0 = ((int64_t)blockIdx.x + i * gridDim.x) * TR;
      if (r0 < n) {
        const int64_t r1 = r0 + TR < n ? r0 + TR : n;
        *b0 = __ldg(a.indptr + r0);
        *b1 = __ldg(a.indptr + r1);
      } else {
        *b0 = *b1 = 0;
      }
    };
    int cur0, cur1, nxt0, nxt1;
    bounds(wl, &cur0, &cur1);
    bounds(32 + wl, &nxt0, &nxt1);
    // WIN: the window records of the same tiles
    auto record = [&](int64_t i, int4* w) {
      const int64_t t = (int64_t)blockIdx.x + i * gridDim.x;
      if (WIN && t * TR < n) {
        const int4* p = reinterpret_cast<const int4*>(ra.win + t * kRingWinInts);
        w[0] = p[0];
        w[1] = p[1];
        w[2] = p[2];
      } else {
        w[0] = w[1] = w[2] = make_int4(0, 0, 0, 0);
      }
    };
    int4 wcur[3], wnxt[3];
    if (WIN) {
      record(wl, wcur);
      record(32 + wl, wnxt);
    }
    for (int64_t i = 0;; ++i) {
      const int64_t r0 = ((int64_t)blockIdx.x + i * gridDim.x) * TR;
      if (r0 >= n) break;
      if (i > 0 && (i & 31) == 0) {
        cur0 = nxt0;
        cur1 = nxt1;
        bounds(i + 32 + wl, &nxt0, &nxt1);
        if (WIN) {
          wcur[0] = wnxt[0];
          wcur[1] = wnxt[1];
          wcur[2] = wnxt[2];
          record(i + 32 + wl, wnxt);
        }
      }
      int wr[9];
      if (WIN) {
        const int src = (int)(i & 31);
        wr[0] = __shfl_sync(0xffffffffu, wcur[0].x, src);
        wr[1] = __shfl_sync(0xffffffffu, wcur[0].y, src);
        wr[2] = __shfl_sync(0xffffffffu, wcur[0].z, src);
        wr[3] = __shfl_sync(0xffffffffu, wcur[0].w, src);
        wr[4] = __shfl_sync(0xffffffffu, wcur[1].x, src);
        wr[5] = __shfl_sync(0xffffffffu, wcur[1].y, src);
        wr[6] = __shfl_sync(0xffffffffu, wcur[1].z, src);
        wr[7] = __shfl_sync(0xffffffffu, wcur[1].w, src);
        wr[8] = __shfl_sync(0xffffffffu, wcur[2].x, src);
      }
      const int j0 = __shfl_sync(0xffffffffu, cur0, (int)(i & 31));
      const int j1 = __shfl_sync(0xffffffffu, cur1, (int)(i & 31));
      const int s = (int)(i % S);
      // the whole warp takes the same branch (the vote), so the shuffles above
      // stay convergent
      if (i >= S &&
          !__all_sync(0xffffffffu, ring_wait(empty0 + 8u * s, (uint32_t)(((i / S) + 1) & 1)))) {
        ok = false;
        break;
      }
      if (wl == 0) {
        char* st = rsm + (size_t)s * sh.stage_bytes;
        const uint32_t bar = full0 + 8u * s;
        const int nr = (int)(n - r0 < TR ? n - r0 : TR);
        // indptr[r0 .. r0+nr] from the 16-byte boundary at or below r0
        const int64_t r0a = r0 & ~(int64_t)3;
        const uint32_t ip_bytes = (uint32_t)(((r0 + nr + 1 - r0a + 3) & ~(int64_t)3) * 4);
        // off-diagonal entries [j0, j1) widened to multiples of 4 entries
        const int ja = j0 & ~3;
        const int cnt = ((j1 + 3) & ~3) - ja;
        const bool csr_in = cnt > 0 && cnt <= sh.cap;
        uint32_t bytes = ip_bytes;
        if (csr_in) bytes += (uint32_t)cnt * (4u + (uint32_t)sizeof(C));
        int64_t d0 = 0;
        uint32_t d_bytes = 0;
        if (a.diag) {
          constexpr int al = 16 / (int)sizeof(C);  // entries per 16 bytes
          d0 = r0 - r0 % al;
          d_bytes = (uint32_t)((r0 + nr - d0 + al - 1) / al * al) * (uint32_t)sizeof(C);
          bytes += d_bytes;
        }
        const uint32_t tile = (uint32_t)(nr * row_bytes);
        const uint32_t ref_tile = (uint32_t)(nr * a.ref_tpr * (int64_t)sizeof(Pack<R, V>));
        if (a.pin) bytes += tile;
        if (need_own && !WIN) bytes += tile;
        if (add_acc) bytes += tile;
        if (ref_staged) bytes += ref_tile;
        int n_w = 0;
        if (WIN) {
          // the stage's window table: lo[w] and base[w] = (row offset in the
          // region) - lo[w], so a column c of window w sits at row base[w] + c
          int* hdr = reinterpret_cast<int*>(st + sh.hdr_off);
          n_w = wr[0] & 0xff;
          int off = 0;
#pragma unroll
          for (int w = 0; w < kRingWinMax; ++w) {
            const int lo = wr[1 + 2 * w], len = wr[2 + 2 * w];
            hdr[1 + w] = w < n_w ? lo : 0x7fffffff;
            hdr[5 + w] = w < n_w ? off - lo : 0;
            if (w < n_w) off += len;
          }
          hdr[0] = wr[0];
          bytes += (uint32_t)(off * row_bytes);
        }
        ring_arrive_tx(bar, bytes);
        ring_copy(ring_smem(st + sh.ip_off), a.indptr + r0a, ip_bytes, bar);
        if (csr_in) {
          ring_copy(ring_smem(st + sh.ix_off), a.indices + ja, (uint32_t)cnt * 4u, bar);
          ring_copy(ring_smem(st + sh.hop_off), a.hop + ja, (uint32_t)cnt * sizeof(C), bar);
        }
        if (a.diag) ring_copy(ring_smem(st + sh.diag_off), a.diag + d0, d_bytes, bar);
        const int64_t e0 = r0 * tpr;
        if (TBPM_RING_EVICT) {
          // p_{k-2} and the accumulator are read once: keep L2 for p_{k-1}
          const uint64_t pol = ring_evict_first_policy();
          if (a.pin) ring_copy_hint(ring_smem(st + sh.pin_off), a.pin + e0, tile, bar, pol);
          if (add_acc) ring_copy_hint(ring_smem(st + sh.acc_off), a.acc + e0, tile, bar, pol);
        } else {
          if (a.pin) ring_copy(ring_smem(st + sh.pin_off), a.pin + e0, tile, bar);
          if (add_acc) ring_copy(ring_smem(st + sh.acc_off), a.acc + e0, tile, bar);
        }
        if (need_own && !WIN) ring_copy(ring_smem(st + sh.own_off), a.gather + e0, tile, bar);
        if (WIN) {
          int off = 0;
#pragma unroll
          for (int w = 0; w < kRingWinMax; ++w) {
            const int lo = wr[1 + 2 * w], len = wr[2 + 2 * w];
            if (w < n_w) {
              ring_copy(ring_smem(st + sh.win_off + (int64_t)off * row_bytes),
                        a.gather + (int64_t)lo * tpr, (uint32_t)(len * row_bytes), bar);
              off += len;
            }
          }
        }
        if (ref_staged)
          ring_copy(ring_smem(st + sh.ref_off), a.ref + r0 * a.ref_tpr, ref_tile, bar);
      }
      __syncwarp();
      ++issued;
    }
    if (!ok && wl == 0) atomicOr(ra.status, 1u);
    // the last S tiles' copies must land before the block may end
    const int64_t first = issued > S ? issued - S : 0;
    for (int64_t i = first; i < issued; ++i)
      if (!ring_wait(full0 + 8u * (int)(i % S), (uint32_t)((i / S) & 1))) {
        if (wl == 0) atomicOr(ra.status, 1u);
        break;
      }
  } else {
    // ---------------- consumer warps ----------------
    const unsigned neg_bits = (unsigned)(a.c.neg_mask >> (lane * V)) & ((1u << V) - 1u);
    const unsigned set_bits = (unsigned)(a.c.set_mask >> (lane * V)) & ((1u << V) - 1u);
    const R beta = (R)a.c.beta;
    constexpr bool do_corr = MODE == 2;
    const bool active = slot < TR;
    const bool ref_lane = do_corr && a.ref != nullptr && lane < a.ref_tpr;
    constexpr int GB = TBPM_RING_GATHER;
    for (int64_t i = 0;; ++i) {
      const int64_t r0 = ((int64_t)blockIdx.x + i * gridDim.x) * TR;
      if (r0 >= n) break;
      const int s = (int)(i % S);
      if (!__all_sync(0xffffffffu, ring_wait(full0 + 8u * s, (uint32_t)((i / S) & 1)))) {
        if ((tid & 31) == 0) atomicOr(ra.status, 1u);
        break;
      }
      const char* st = rsm + (size_t)s * sh.stage_bytes;
      const int64_t r = r0 + slot;
      if (active && r < n) {
        const int nr = (int)(n - r0 < TR ? n - r0 : TR);
        const int32_t* ip = reinterpret_cast<const int32_t*>(st + sh.ip_off) + (r0 & 3);
        const int j0 = ip[slot], j1 = ip[slot + 1];
        const int ja = ip[0] & ~3;
        const int cnt = ((ip[nr] + 3) & ~3) - ja;
        const bool csr_in = cnt > 0 && cnt <= sh.cap;
        const int32_t* ixs = reinterpret_cast<const int32_t*>(st + sh.ix_off) - ja;
        const C* hs = reinterpret_cast<const C*>(st + sh.hop_off) - ja;
        // WIN: row of column c in the window region (windows sorted by lo)
        const int* hdr = reinterpret_cast<const int*>(st + sh.hdr_off);
        const bool wgat = !WIN || ((hdr[0] >> 8) & 1);
        auto wrow = [&](int col) -> int64_t {
          int b = hdr[5];
          if (col >= hdr[2]) b = hdr[6];
          if (col >= hdr[3]) b = hdr[7];
          if (col >= hdr[4]) b = hdr[8];
          return (int64_t)b + col;
        };
        const char* wreg = st + sh.win_off;
        const int64_t e = r * tpr + lane;
        const int64_t te = (int64_t)slot * tpr + lane;  // pack index within the tile
        R sre[V], sim[V];
        Pack<R, V> own;
        bool first = true;
        for (int jb = j0; jb < j1 || first; jb += GB) {
          int cidx[GB];
          C h[GB];
#pragma unroll
          for (int u = 0; u < GB; ++u) {
            if (jb + u < j1) {
              cidx[u] = csr_in ? ixs[jb + u] : __ldg(a.indices + jb + u);
              h[u] = csr_in ? hs[jb + u] : ldg_c(a.hop + jb + u);
            } else {
              cidx[u] = -1;
            }
          }
          Pack<R, V> x[GB];
#pragma unroll
          for (int u = 0; u < GB; ++u)
            if (cidx[u] >= 0) {
              // neighbours inside the tile come from its staged rows of p_{k-1}
              const int64_t lc = (int64_t)cidx[u] - r0;
              if (WIN && !wgat)
                x[u] = lds_pack<R, V>(wreg + (wrow(cidx[u]) * tpr + lane) * sizeof(Pack<R, V>));
              else if (!WIN && TBPM_RING_LOCAL && need_own && lc >= 0 && lc < nr)
                x[u] = lds_pack<R, V>(st + sh.own_off + (lc * tpr + lane) * sizeof(Pack<R, V>));
              else
                x[u] = ldg_pack(a.gather + (int64_t)cidx[u] * tpr + lane);
            }
          if (first) {
            // staged operands while the gathers are in flight: sum = D p_{k-1}
            first = false;
            if (need_own)
              own = WIN ? lds_pack<R, V>(wreg + (wrow((int)r) * tpr + lane) * sizeof(Pack<R, V>))
                        : lds_pack<R, V>(st + sh.own_off + te * sizeof(Pack<R, V>));
            if (a.diag) {
              constexpr int al = 16 / (int)sizeof(C);
              const C d = reinterpret_cast<const C*>(st + sh.diag_off)[r - (r0 - r0 % al)];
#pragma unroll
              for (int v = 0; v < V; ++v) {
                sre[v] = d.x * own.v[2 * v] - d.y * own.v[2 * v + 1];
                sim[v] = d.x * own.v[2 * v + 1] + d.y * own.v[2 * v];
              }
            } else {
#pragma unroll
              for (int v = 0; v < V; ++v) sre[v] = sim[v] = (R)0;
            }
          }
#pragma unroll
          for (int u = 0; u < GB; ++u) {
            if (cidx[u] >= 0) {
#pragma unroll
              for (int v = 0; v < V; ++v) {
                sre[v] = fma(h[u].x, x[u].v[2 * v], fma(-h[u].y, x[u].v[2 * v + 1], sre[v]));
                sim[v] = fma(h[u].x, x[u].v[2 * v + 1], fma(h[u].y, x[u].v[2 * v], sim[v]));
              }
            }
          }
        }
        Pack<R, V> pm2;
        if (a.pin) {
          pm2 = lds_pack<R, V>(st + sh.pin_off + te * sizeof(Pack<R, V>));
        } else {
#pragma unroll
          for (int k = 0; k < 2 * V; ++k) pm2.v[k] = (R)0;
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
        if (a.pout) stcs_pack(a.pout + e, pk);
        if (nflush > 0) {
          Pack<R, V> acc;
          if (add_acc) acc = lds_pack<R, V>(st + sh.acc_off + te * sizeof(Pack<R, V>));
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
            if (ref_lane)
              rf = ref_staged ? lds_pack<R, V>(st + sh.ref_off +
                                               ((int64_t)slot * a.ref_tpr + lane) *
                                                   sizeof(Pack<R, V>))
                              : ldcs_pack(a.ref + r * a.ref_tpr + lane);
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
      }
      __syncwarp();
      if ((tid & 31) == 0) ring_arrive(empty0 + 8u * s);
    }
  }

  if constexpr (MODE == 2) {
    // block partials of the correlation and norm, reduced in a fixed order over
    // the rows of a tile; the stage buffers are free (every copy was consumed)
    __syncthreads();
    double* red = reinterpret_cast<double*>(rsm);
    const int width = tpr * V * 3;
    if (tid < kRingConsumers && slot < TR) {
#pragma unroll
      for (int v = 0; v < V; ++v) {
        double* p = red + slot * width + (lane * V + v) * 3;
        p[0] = cre[v];
        p[1] = cim[v];
        p[2] = nrm[v];
      }
    }
    __syncthreads();
    tree_reduce_slots(red, TR, width, slot, lane, tpr);
    if (tid < kRingConsumers && slot == 0) {
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const int col = lane * V + v;
#pragma unroll
        for (int q = 0; q < 3; ++q)
          a.partials[(int64_t)(col * 3 + q) * gridDim.x + blockIdx.x] = red[col * 3 + q];
      }
    }
  }
}

// ---- window plan ----------------------------------------------------------

// One thread per tile of TR rows: cover its own rows and the columns of its
// off-diagonal entries with row ranges, merging runs closer than kRingWinGap
// rows; at most kRingWinMax ranges and `budget` rows in total, else the tile
// is marked for global gathers with its own rows as its one window.
__global__ void ring_window_kernel(const int32_t* __restrict__ indptr,
                                   const int32_t* __restrict__ indices, int64_t n, int TR,
                                   int n_tiles, int budget, int* win, unsigned* n_gather) {
  constexpr int K = 8;  // runs tracked before the merge
  for (int T = blockIdx.x * blockDim.x + threadIdx.x; T < n_tiles; T += gridDim.x * blockDim.x) {
    const int64_t r0 = (int64_t)T * TR;
    const int64_t r1 = r0 + TR < n ? r0 + TR : n;
    int lo[K], hi[K];  // [lo, hi)
    int m = 1;
    lo[0] = (int)r0;
    hi[0] = (int)r1;
    bool over = false;
    const int j1 = indptr[r1];
    for (int j = indptr[r0]; j < j1 && !over; ++j) {
      const int c = indices[j];
      int k = 0;
      for (; k < m; ++k)
        if (c >= lo[k] - kRingWinGap && c < hi[k] + kRingWinGap) break;
      if (k < m) {
        lo[k] = c < lo[k] ? c : lo[k];
        hi[k] = c + 1 > hi[k] ? c + 1 : hi[k];
      } else if (m < K) {
        lo[m] = c;
        hi[m] = c + 1;
        ++m;
      } else {
        over = true;
      }
    }
    // sort by lo, then merge runs that overlap or lie within the gap
    for (int a = 1; a < m; ++a)
      for (int b = a; b > 0 && lo[b] < lo[b - 1]; --b) {
        const int tl = lo[b], th = hi[b];
        lo[b] = lo[b - 1];
        hi[b] = hi[b - 1];
        lo[b - 1] = tl;
        hi[b - 1] = th;
      }
    int q = 0;
    for (int a = 1; a < m; ++a) {
      if (lo[a] <= hi[q] + kRingWinGap) {
        hi[q] = hi[a] > hi[q] ? hi[a] : hi[q];
      } else {
        ++q;
        lo[q] = lo[a];
        hi[q] = hi[a];
      }
    }
    const int nw = q + 1;
    int rows = 0;
    for (int a = 0; a < nw; ++a) rows += hi[a] - lo[a];
    int* rec = win + (int64_t)T * kRingWinInts;
    if (over || nw > kRingWinMax || rows > budget) {
      rec[0] = 1 | (1 << 8);
      rec[1] = (int)r0;
      rec[2] = (int)(r1 - r0);
      for (int a = 3; a < kRingWinInts; ++a) rec[a] = 0;
      atomicAdd(n_gather, 1u);
    } else {
      rec[0] = nw;
      for (int a = 0; a < kRingWinMax; ++a) {
        rec[1 + 2 * a] = a < nw ? lo[a] : 0;
        rec[2 + 2 * a] = a < nw ? hi[a] - lo[a] : 0;
      }
      for (int a = 1 + 2 * kRingWinMax; a < kRingWinInts; ++a) rec[a] = 0;
    }
  }
}

}  // namespace tbpm
