// Two consecutive Chebyshev terms in one launch (sm_100a): cheb_pair_kernel.
//
// Terms k and k+1 of an expansion,
//   p_k     = alpha*(H p_{k-1}) + beta*p_{k-2}     ("first" term, item bit 0 = 0)
//   p_{k+1} = alpha*(H p_k)     + beta*p_{k-1}     ("second" term, item bit 0 = 1)
// run as one stream of work items, one item per (row tile, term).  A tile's
// second term needs p_k of every row its rows couple to, so it waits until the
// first term of each of those tiles is stored; it then reads p_k back while it
// is still in L2, and its own rows of p_{k-1}, its CSR slice and its diagonal
// are L2 hits too (the first term of the same tile read them shortly before).
// Against two single-term launches this saves the DRAM reads of p_{k-1}, p_k
// and the matrix once per pair: about a third of the bytes of the two terms.
// Every row is computed with the same operations in the same order as
// cheb_ring_kernel / cheb_term_kernel, so the results are bit-identical.
// (Measured on B200, 2048^2 graphene, 16 FP64 states: the launches move the
// modelled bytes, but a consumer warp spends as long on a second-term item as
// on a first-term one, waiting on its L2 gathers, so the pair takes longer
// than two ring launches; the library uses it only on request, term_kernel 3.)
//
// The second term overwrites p_{k-1} (its output p_{k+1} takes that buffer),
// which first terms of neighbouring tiles gather.  The dependency list of a
// tile is therefore the union of the tiles its rows read (columns) and the
// tiles whose rows read it (the transposed pattern): its second term runs
// only after the first term of every tile on the list, which covers both.
//
// Items follow a precomputed sequence (pair_seq_kernel): all first terms in
// tile order, each second term placed after the first terms of its whole list
// plus a margin of about the work in flight.  Block b takes one position of
// each round of G positions, in order (G blocks, launched cooperatively, so
// all are resident).
// Every dependency of an item lies earlier in the sequence and the flag of a
// finished item is stored by its consumers, whatever its producer waits on,
// so the earliest unfinished item can always proceed: no deadlock.
//
// A block is one producer warp and kRingConsumerWarps consumer warps around a
// ring of shared-memory stages, as in cheb_ring_kernel.  The producer stages
// each item's CSR slice, diagonal, p_{k-2} / p_{k-1} rows and accumulator by
// bulk copies (data that no block writes during the launch).  p_k, written
// during the launch, is read by the consumers with L2-only loads (ld.global.cg)
// after the producer has seen the flags of the item's dependencies (relaxed
// loads, then one acquire fence per second-term item).  The last consumer
// warp done with a first-term item (an acq_rel counter in shared memory)
// stores the tile's flag after a GPU-scope fence.  Flags hold the launch
// number + 1 (PairSync::epoch), so they never need resetting.
//
// Every wait is bounded in time (kRingWaitNs) and also ends when another block
// has reported a failure; a wait that runs out sets bit 0 of *status.
#pragma once

#include "tbpm_ring_kernels.cuh"

namespace tbpm {

constexpr int kPairDeps = 16;   // dependency tiles per tile (padded with -1)
constexpr int kPairEnd = -1;    // stage marker: no more items
// after the mbarriers: stage item codes, flag value, per-stage counts of
// consumer warps done (128 bytes), then the two terms' arguments
template <typename R, int V>
constexpr int pair_extra_smem() {
  return 128 + 2 * (int)((sizeof(TermArgs<R, V>) + 15) / 16 * 16);
}

struct PairSync {
  unsigned epoch;  // launches completed with this plan
  unsigned done;   // blocks finished in the current launch
  unsigned pad[2];
};

template <typename R, int V>
struct PairArgs {
  TermArgs<R, V> t[2];  // the first (k) and the second (k+1) term
  RingShape s;          // stage layout (the flush layout: with accumulator rows)
  const int4* seq;      // items: {2*tile + term, indptr[r0], indptr[r1], 0}
  int n_items;
  const int* deps;      // [tile][kPairDeps] tiles whose first term must be stored first
  unsigned* flags;      // [tile]: epoch + 1 once the tile's first term is stored
  PairSync* sync;
  unsigned* status;     // bit 0: a bounded wait ran out
};

__device__ __forceinline__ bool ring_test(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ unsigned ld_relaxed_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_relaxed_u32(unsigned* p, unsigned v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Producer: stage the operands of one item (lane 0 only).  Own rows of
// p_{k-1} are staged for the first term; the second term's own rows are p_k,
// which the consumers load themselves.
template <typename R, int V, int TERM>
__device__ __forceinline__ void pair_issue(const TermArgs<R, V>& a, const RingShape& sh, char* st,
                                           uint32_t bar, int64_t r0, int j0, int j1) {
  using C = typename Cx<R>::t;
  const int64_t n = a.n_rows;
  const int TR = sh.rows;
  const int nr = (int)(n - r0 < TR ? n - r0 : TR);
  const int64_t row_bytes = (int64_t)a.tpr * sizeof(Pack<R, V>);
  const int nflush = a.c.nflush;
  const bool need_own = TERM == 0 && (a.diag != nullptr || nflush >= 2);
  const bool add_acc = nflush > 0 && !a.c.acc_init;
  const int64_t r0a = r0 & ~(int64_t)3;
  const uint32_t ip_bytes = (uint32_t)(((r0 + nr + 1 - r0a + 3) & ~(int64_t)3) * 4);
  const int ja = j0 & ~3;
  const int cnt = ((j1 + 3) & ~3) - ja;
  const bool csr_in = cnt > 0 && cnt <= sh.cap;
  uint32_t bytes = ip_bytes;
  if (csr_in) bytes += (uint32_t)cnt * (4u + (uint32_t)sizeof(C));
  int64_t d0 = 0;
  uint32_t d_bytes = 0;
  if (a.diag) {
    constexpr int al = 16 / (int)sizeof(C);
    d0 = r0 - r0 % al;
    d_bytes = (uint32_t)((r0 + nr - d0 + al - 1) / al * al) * (uint32_t)sizeof(C);
    bytes += d_bytes;
  }
  const uint32_t tile = (uint32_t)(nr * row_bytes);
  if (a.pin) bytes += tile;
  if (need_own) bytes += tile;
  if (add_acc) bytes += tile;
  ring_arrive_tx(bar, bytes);
  ring_copy(ring_smem(st + sh.ip_off), a.indptr + r0a, ip_bytes, bar);
  if (csr_in) {
    ring_copy(ring_smem(st + sh.ix_off), a.indices + ja, (uint32_t)cnt * 4u, bar);
    ring_copy(ring_smem(st + sh.hop_off), a.hop + ja, (uint32_t)cnt * sizeof(C), bar);
  }
  if (a.diag) ring_copy(ring_smem(st + sh.diag_off), a.diag + d0, d_bytes, bar);
  const int64_t e0 = r0 * a.tpr;
  if (a.pin) ring_copy(ring_smem(st + sh.pin_off), a.pin + e0, tile, bar);
  if (add_acc) ring_copy(ring_smem(st + sh.acc_off), a.acc + e0, tile, bar);
  if (need_own) ring_copy(ring_smem(st + sh.own_off), a.gather + e0, tile, bar);
}

// Consumer: one row's V columns of one item, in cheb_ring_kernel's order.
// One code path for both terms (two inlined copies spill at 128 registers).
template <typename R, int V>
__device__ __forceinline__ void pair_rows(const TermArgs<R, V>& a, const RingShape& sh,
                                          const char* st, int64_t r0, int slot, int lane,
                                          const bool second) {
  using C = typename Cx<R>::t;
  const int TR = sh.rows;
  const int64_t n = a.n_rows;
  const int tpr = a.tpr;
  const int64_t r = r0 + slot;
  if (slot >= TR || r >= n) return;
  const int nflush = a.c.nflush;
  const bool need_own = a.diag != nullptr || nflush >= 2;
  const bool add_acc = nflush > 0 && !a.c.acc_init;
  const unsigned neg_bits = (unsigned)(a.c.neg_mask >> (lane * V)) & ((1u << V) - 1u);
  const unsigned set_bits = (unsigned)(a.c.set_mask >> (lane * V)) & ((1u << V) - 1u);
  const R beta = (R)a.c.beta;
  constexpr int GB = TBPM_RING_GATHER;
  const int nr = (int)(n - r0 < TR ? n - r0 : TR);
  const int32_t* ip = reinterpret_cast<const int32_t*>(st + sh.ip_off) + (r0 & 3);
  const int j0 = ip[slot], j1 = ip[slot + 1];
  const int ja = ip[0] & ~3;
  const int cnt = ((ip[nr] + 3) & ~3) - ja;
  const bool csr_in = cnt > 0 && cnt <= sh.cap;
  const int32_t* ixs = reinterpret_cast<const int32_t*>(st + sh.ix_off) - ja;
  const C* hs = reinterpret_cast<const C*>(st + sh.hop_off) - ja;
  const int64_t e = r * tpr + lane;
  const int64_t te = (int64_t)slot * tpr + lane;
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
        const Pack<R, V>* src = a.gather + (int64_t)cidx[u] * tpr + lane;
        x[u] = second ? ldcg_pack(src) : ldg_pack(src);
      }
    if (first) {
      first = false;
      if (need_own)
        own = second ? ldcg_pack(a.gather + e)
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
  if (a.pout) {
    // p_k is read back by the second term from L2: normal eviction priority
    if (second)
      stcs_pack(a.pout + e, pk);
    else
      stwb_pack(a.pout + e, pk);
  }
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
  }
}

template <typename R, int V>
__global__ void __launch_bounds__(kRingThreads, kRingMinBlocks)
    cheb_pair_kernel(const __grid_constant__ PairArgs<R, V> pa) {
  extern __shared__ __align__(128) char rsm[];
  const RingShape& sh = pa.s;
  const int S = sh.stages;
  const int TR = sh.rows;
  const int tid = threadIdx.x;
  const unsigned FULL = 0xffffffffu;
  const uint32_t full0 = ring_smem(rsm + sh.bar_off);
  const uint32_t empty0 = full0 + 8u * (uint32_t)S;
  // after the mbarriers: the item code of each stage (8 at most), this
  // launch's flag value, the consumer warps done with each stage's item
  volatile int* item_of = reinterpret_cast<volatile int*>(rsm + sh.bar_off + 16 * S);
  volatile unsigned* want_p =
      reinterpret_cast<volatile unsigned*>(rsm + sh.bar_off + 16 * S + 32);
  unsigned* done_cnt = reinterpret_cast<unsigned*>(rsm + sh.bar_off + 16 * S + 64);
  // the consumers read the arguments of an item's term from shared memory (a
  // runtime index into the kernel parameters costs a dependent load per field)
  constexpr int kArgBytes = (int)((sizeof(TermArgs<R, V>) + 15) / 16 * 16);
  TermArgs<R, V>* args = reinterpret_cast<TermArgs<R, V>*>(rsm + sh.bar_off + 16 * S + 128);
  TermArgs<R, V>* args1 =
      reinterpret_cast<TermArgs<R, V>*>(rsm + sh.bar_off + 16 * S + 128 + kArgBytes);

  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      ring_bar_init(full0 + 8u * s, 1);
      ring_bar_init(empty0 + 8u * s, kRingConsumerWarps);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    *want_p = ld_relaxed_u32(&pa.sync->epoch) + 1u;
    *args = pa.t[0];
    for (int s = 0; s < S; ++s) done_cnt[s] = 0u;
  }
  if (tid == 32) *args1 = pa.t[1];
  __syncthreads();
  const unsigned want = *want_p;

  if (tid >= kRingConsumers) {
    // ---------------- producer warp ----------------
    const int wl = tid & 31;
    const int64_t G = gridDim.x;
    const int64_t n_items = pa.n_items;
    bool ok = true;
    int64_t issued = 0;
    auto failed_elsewhere = [&]() {
      return *reinterpret_cast<volatile unsigned*>(pa.status) != 0u;
    };
    // Item q of this block is sequence position q * G + (blockIdx.x + q) % G:
    // round q of the sequence, at an offset that turns with the round, so a
    // block alternates between first and second terms where they alternate in
    // the sequence (a plain stride of an even G would give a block only one
    // kind).  Lane l holds the entry of item wbase + l, and of wbase + 32 + l.
    auto entry = [&](int64_t q) -> int4 {
      const int64_t p = q * G + ((int64_t)blockIdx.x + q) % G;
      return p < n_items ? pa.seq[p] : make_int4(kPairEnd, 0, 0, 0);
    };
    int64_t wbase = 0;
    int4 e_cur = entry(wl), e_nxt = entry(32 + wl);
    auto code_at = [&](int64_t q) -> int {  // q in [wbase, wbase + 64)
      const int d = (int)(q - wbase);
      const int c0 = __shfl_sync(FULL, e_cur.x, d & 31);
      const int c1 = __shfl_sync(FULL, e_nxt.x, d & 31);
      return d < 32 ? c0 : c1;
    };
    auto dep_row = [&](int code) -> int {  // lane's dependency of a second-term item
      return (code >= 0 && (code & 1) && wl < kPairDeps) ? pa.deps[(code >> 1) * kPairDeps + wl]
                                                          : -1;
    };
    // dependency rows and flag values, loaded one and two items ahead
    int dep0 = dep_row(code_at(0));
    unsigned fl0 = dep0 >= 0 ? ld_relaxed_u32(pa.flags + dep0) : want;
    int dep1 = dep_row(code_at(1));
    for (int64_t q = 0;; ++q) {
      if (q == wbase + 32) {
        e_cur = e_nxt;
        wbase += 32;
        e_nxt = entry(wbase + 32 + wl);
      }
      const int d = (int)(q - wbase);
      const int code = __shfl_sync(FULL, e_cur.x, d);
      const int j0 = __shfl_sync(FULL, e_cur.y, d);
      const int j1 = __shfl_sync(FULL, e_cur.z, d);
      if (code < 0) break;
      const int s = (int)(q % S);
      // the stage is free once the consumers are done with the item S back
      if (q >= S &&
          !__all_sync(FULL, ring_wait(empty0 + 8u * s, (uint32_t)(((q / S) + 1) & 1)))) {
        ok = false;
        break;
      }
      if (code & 1) {
        // second term: the first term of every dependency must be stored
        if (!__all_sync(FULL, fl0 == want)) {
          const unsigned long long t0 = ring_clock_ns();
          for (;;) {
            fl0 = dep0 >= 0 ? ld_relaxed_u32(pa.flags + dep0) : want;
            if (__all_sync(FULL, fl0 == want)) break;
            bool out = ring_clock_ns() - t0 > kRingWaitNs || failed_elsewhere();
            out = __shfl_sync(FULL, out, 0);
            if (out) {
              ok = false;
              break;
            }
          }
          if (!ok) break;
        }
        // acquire: the dependencies' rows of p_k before the consumers' loads
        asm volatile("fence.acq_rel.gpu;" ::: "memory");
      }
      if (wl == 0) {
        char* st = rsm + (size_t)s * sh.stage_bytes;
        const uint32_t bar = full0 + 8u * s;
        const int64_t r0 = (int64_t)(code >> 1) * TR;
        item_of[s] = code;
        if (code & 1)
          pair_issue<R, V, 1>(pa.t[1], sh, st, bar, r0, j0, j1);
        else
          pair_issue<R, V, 0>(pa.t[0], sh, st, bar, r0, j0, j1);
      }
      __syncwarp();
      ++issued;
      // look-ahead: flags of item q+1, dependency row of item q+2
      const unsigned fl1 = dep1 >= 0 ? ld_relaxed_u32(pa.flags + dep1) : want;
      const int dep2 = dep_row(code_at(q + 2));
      dep0 = dep1;
      fl0 = fl1;
      dep1 = dep2;
    }
    // no more items: mark the next stage as the end for the consumers
    bool end_sent = false;
    if (ok) {
      const int64_t q = issued;
      const int s = (int)(q % S);
      if (q >= S &&
          !__all_sync(FULL, ring_wait(empty0 + 8u * s, (uint32_t)(((q / S) + 1) & 1))))
        ok = false;
      if (ok) {
        if (wl == 0) {
          item_of[s] = kPairEnd;
          ring_arrive(full0 + 8u * s);
        }
        __syncwarp();
        end_sent = true;
      }
    }
    // (after the end marker the consumers wait for every issued stage, so
    // its copies land before the block ends)
    if (!ok) {
      if (wl == 0) atomicOr(pa.status, 1u);
      if (!end_sent && issued < S) {
        if (wl == 0) {
          item_of[(int)(issued % S)] = kPairEnd;
          ring_arrive(full0 + 8u * (int)(issued % S));
        }
      }
      // consumers may have stopped: the copies already issued must land
      // before the block may end
      const int64_t first = issued > S ? issued - S : 0;
      for (int64_t i = first; i < issued; ++i)
        if (!ring_wait(full0 + 8u * (int)(i % S), (uint32_t)((i / S) & 1))) break;
    }
  } else {
    // ---------------- consumer warps ----------------
    const int tpr = pa.t[0].tpr;
    const int slot = tid / tpr;
    const int lane = tid - slot * tpr;
    for (int64_t q = 0;; ++q) {
      const int s = (int)(q % S);
      if (!__all_sync(FULL, ring_wait(full0 + 8u * s, (uint32_t)((q / S) & 1)))) {
        if ((tid & 31) == 0) atomicOr(pa.status, 1u);
        break;
      }
      const int code = item_of[s];
      if (code < 0) break;
      const char* st = rsm + (size_t)s * sh.stage_bytes;
      const int64_t r0 = (int64_t)(code >> 1) * TR;
      pair_rows<R, V>((code & 1) ? *args1 : *args, sh, st, r0, slot, lane, (code & 1) != 0);
      __syncwarp();
      if ((tid & 31) == 0) {
        if ((code & 1) == 0) {
          // the last consumer warp done with a first-term item stores its flag:
          // the warps' rows (acq_rel count in shared memory), then one fence
          // and the flag (the release pattern at GPU scope)
          unsigned prev;
          asm volatile("atom.acq_rel.cta.shared::cta.add.u32 %0, [%1], 1;"
                       : "=r"(prev)
                       : "r"(ring_smem(done_cnt + s))
                       : "memory");
          if (prev == (unsigned)kRingConsumerWarps - 1u) {
            done_cnt[s] = 0u;
            asm volatile("fence.acq_rel.gpu;" ::: "memory");
            st_relaxed_u32(pa.flags + (code >> 1), want);
          }
        }
        ring_arrive(empty0 + 8u * s);
      }
    }
  }

  // the last block to finish advances the epoch
  __syncthreads();
  if (tid == 0) {
    __threadfence();
    const unsigned prev = atomicAdd(&pa.sync->done, 1u);
    if (prev == gridDim.x - 1) {
      pa.sync->done = 0u;
      __threadfence();
      pa.sync->epoch = want;
    }
  }
}

// ---- plan: dependency lists and the item sequence -------------------------

// One warp per tile: the distinct tiles its rows' columns fall in (the tile
// itself first).  More than kPairDeps sets bit 0 of *bad.
__global__ void pair_fwd_kernel(const int32_t* __restrict__ indptr,
                                const int32_t* __restrict__ indices, int64_t n, int TR,
                                int n_tiles, int* fwd, int* fcnt, unsigned* bad) {
  __shared__ int sets[8][kPairDeps];
  const unsigned FULL = 0xffffffffu;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int* set = sets[w];
  const int n_warps = (int)(gridDim.x * (blockDim.x >> 5));
  for (int T = (int)(blockIdx.x * (blockDim.x >> 5)) + w; T < n_tiles; T += n_warps) {
    const int64_t r0 = (int64_t)T * TR;
    const int64_t r1 = r0 + TR < n ? r0 + TR : n;
    const int j0 = indptr[r0], j1 = indptr[r1];
    if (lane == 0) set[0] = T;
    int cnt = 1;
    __syncwarp();
    for (int base = j0; base < j1; base += 32) {
      const int t = base + lane < j1 ? (int)(indices[base + lane] / TR) : -1;
      bool present = t < 0;
      const int lim = cnt < kPairDeps ? cnt : kPairDeps;
      for (int k = 0; k < lim; ++k) present |= set[k] == t;
      const unsigned grp = __match_any_sync(FULL, t);
      const bool lead = !present && lane == __ffs(grp) - 1;
      const unsigned lm = __ballot_sync(FULL, lead);
      const int pos = cnt + __popc(lm & ((1u << lane) - 1u));
      __syncwarp();
      if (lead && pos < kPairDeps) set[pos] = t;
      cnt += __popc(lm);
      __syncwarp();
    }
    if (cnt > kPairDeps) {
      if (lane == 0) atomicOr(bad, 1u);
      cnt = kPairDeps;
    }
    if (lane < kPairDeps) fwd[(int64_t)T * kPairDeps + lane] = lane < cnt ? set[lane] : -1;
    if (lane == 0) fcnt[T] = cnt;
    __syncwarp();
  }
}

// The transposed pattern: T is added to the list of every tile T reads.
__global__ void pair_rev_kernel(const int* fwd, const int* fcnt, int n_tiles, int* rev, int* rcnt,
                                unsigned* bad) {
  for (int T = blockIdx.x * blockDim.x + threadIdx.x; T < n_tiles; T += gridDim.x * blockDim.x) {
    for (int k = 0; k < fcnt[T]; ++k) {
      const int d = fwd[(int64_t)T * kPairDeps + k];
      if (d == T) continue;
      const int slot = atomicAdd(&rcnt[d], 1);
      if (slot < kPairDeps)
        rev[(int64_t)d * kPairDeps + slot] = T;
      else
        atomicOr(bad, 2u);
    }
  }
}

// Union of both lists per tile, the position of its second term (after the
// first term of tile min(last dependency + margin, n_tiles); n_tiles = at the
// end) and the count of tiles whose last dependency is within `near` tiles.
__global__ void pair_merge_kernel(const int* fwd, const int* fcnt, const int* rev,
                                  const int* rcnt, int n_tiles, int margin, int near, int* deps,
                                  int* ready, int* cnt_b, unsigned* bad, unsigned* n_near) {
  for (int T = blockIdx.x * blockDim.x + threadIdx.x; T < n_tiles; T += gridDim.x * blockDim.x) {
    int list[kPairDeps];
    int m = 0;
    const int nf = fcnt[T];
    for (int k = 0; k < nf; ++k) list[m++] = fwd[(int64_t)T * kPairDeps + k];
    const int nrv = rcnt[T] < kPairDeps ? rcnt[T] : kPairDeps;
    bool over = false;
    for (int k = 0; k < nrv; ++k) {
      const int d = rev[(int64_t)T * kPairDeps + k];
      bool present = false;
      for (int i = 0; i < m; ++i) present |= list[i] == d;
      if (present) continue;
      if (m < kPairDeps)
        list[m++] = d;
      else
        over = true;
    }
    if (over) atomicOr(bad, 4u);
    int last = T;
    for (int i = 0; i < m; ++i) last = list[i] > last ? list[i] : last;
    for (int i = 0; i < kPairDeps; ++i) deps[(int64_t)T * kPairDeps + i] = i < m ? list[i] : -1;
    const int64_t rd = (int64_t)last + margin;
    const int r = rd < n_tiles ? (int)rd : n_tiles;
    ready[T] = r;
    atomicAdd(&cnt_b[r], 1);
    if (last - T <= near) atomicAdd(n_near, 1u);
  }
}

// Items: the first term of tile a at position a + off_b[a] (second terms
// placed before it: those ready at tiles < a); the second term of tile T
// right after the first term of tile ready[T] (or after all first terms).
__global__ void pair_seq_kernel(const int32_t* __restrict__ indptr, int64_t n, int TR,
                                int n_tiles, const int* ready, const int64_t* off_b, int* g_cnt,
                                int4* seq) {
  for (int T = blockIdx.x * blockDim.x + threadIdx.x; T < n_tiles; T += gridDim.x * blockDim.x) {
    const int64_t r0 = (int64_t)T * TR;
    const int64_t r1 = r0 + TR < n ? r0 + TR : n;
    const int j0 = indptr[r0], j1 = indptr[r1];
    seq[T + off_b[T]] = make_int4(2 * T, j0, j1, 0);
    const int r = ready[T];
    const int64_t base = (int64_t)r + off_b[r] + (r < n_tiles ? 1 : 0);
    const int slot = atomicAdd(&g_cnt[r], 1);
    seq[base + slot] = make_int4(2 * T + 1, j0, j1, 0);
  }
}

}  // namespace tbpm
