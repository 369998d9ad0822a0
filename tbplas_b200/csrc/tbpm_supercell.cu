// Device-side assembly of the TBPM Hamiltonian of a periodic supercell.
//
// Replaces the host chain of the reference builder that produces the TBPM
// input:  SuperCell orbital positions (cython/super.pyx:569-612), the reduced
// hopping list (super.pyx:643-912, builder/super.py:687-790), Peierls phases
// (cython/sample.pyx:20-74), the rescale estimate (sample.pyx:77-116),
// rescaling (builder/sample.py:272-299) and the CSR builders
// Sample.build_ham_csr (sample.py:375-391) / build_ham_dxy (sample.py:417-461,
// sample.pyx:150-257).
//
// One thread owns one row (one orbital of the supercell).  It enumerates the
// row's entries straight from the primitive cell: the on-site term, the
// hopping terms whose bra is this orbital, and the conjugates of the terms
// whose ket is this orbital.  Every term carries the position it has in the
// reference's hopping list (its "key"), so that the row can be put in the
// reference's order: by column for build_ham_csr, on-site first and then list
// order for build_ham_dxy, and list order for the rescale row sums.  All
// floating-point steps use explicitly rounded intrinsics in the reference's
// evaluation order (no FMA contraction), so positions, dr, rescale and
// field-free values are bit-identical to the reference; Peierls factors go
// through the device sincos (within 2 ulp of the host libm).
//
// Passes: [vacancy map] -> [row sums + max, if the rescale is estimated] ->
// row counts -> exclusive scan -> fill.  The fill either writes the resident
// H = D + O form of the context (in its precision) or a full CSR for download.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "tbpm_b200.h"
#include "tbpm_common.cuh"
#include "tbpm_engine.cuh"
#include "tbpm_scan.cuh"

namespace tbpm {
namespace {

struct HopTerm {
  int r[3];
  int bra, ket;
  int is_pbc;
  double er, ei;
};

struct ScDev {
  double lat[9], S[9], origin[3];
  int dim[3], pbc[3];
  int n_orb, n_hop;
  int64_t n_rows, n_full;
  const double* frac;     // [n_orb][3]
  const double* pc_eng;   // [n_orb]
  const double* sc_eng;   // [n_rows] or null
  const HopTerm* hop;     // [n_hop]
  const int* fwd_off;     // terms whose bra is orbital o: fwd_ih[fwd_off[o] .. fwd_off[o+1])
  const int* fwd_ih;
  const int* bwd_off;     // terms whose ket is orbital o
  const int* bwd_ih;
  const int64_t* vac;     // sorted vacancy indices (full numbering)
  int64_t n_vac;
  const int32_t* inv;     // row -> full index (only with vacancies)
  int field, gauge;
  double gfac;            // field prefactor of the gauge (see phase())
  double scale;           // 1 / rescale
  int layout;             // TBPM_LAYOUT_CSR or TBPM_LAYOUT_DXY
  double cutoff;          // on-site cutoff of the DXY layout
  int need_dr;
};

struct Term {
  unsigned long long key;
  int col;
  int kind;  // 1: this row is the bra, 2: this row is the ket (conjugate)
  double vr, vi, dx, dy;
};

__device__ __forceinline__ int wrap_idx(int j, int n, int p) {
  if (!p) return (j < 0 || j >= n) ? -1 : j;
  int w = j % n;
  return w < 0 ? w + n : w;
}

__device__ __forceinline__ int floor_div(int j, int n) {
  int q = j / n;
  return (j % n != 0 && ((j < 0) != (n < 0))) ? q - 1 : q;
}

__device__ __forceinline__ int64_t lower_bound64(const int64_t* a, int64_t n, int64_t x) {
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (a[mid] < x)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

// row of supercell orbital g, or -1 if g is a vacancy (super.pyx:104-152)
__device__ __forceinline__ int64_t row_of(const ScDev& s, int64_t g) {
  if (s.n_vac == 0) return g;
  const int64_t lb = lower_bound64(s.vac, s.n_vac, g);
  if (lb < s.n_vac && s.vac[lb] == g) return -1;
  return g - lb;
}

__device__ __forceinline__ int64_t full_index(const ScDev& s, int ia, int ib, int ic, int o) {
  return (((int64_t)ia * s.dim[1] + ib) * s.dim[2] + ic) * s.n_orb + o;
}

// Cartesian position of supercell orbital (ia, ib, ic, o): super.pyx:602-611
// ((ra*L00 + rb*L10) + rc*L20), then + origin (super.py:682)
__device__ __forceinline__ void orb_pos(const ScDev& s, int ia, int ib, int ic, int o,
                                        double p[3]) {
  const double ra = __dadd_rn(s.frac[3 * o + 0], (double)ia);
  const double rb = __dadd_rn(s.frac[3 * o + 1], (double)ib);
  const double rc = __dadd_rn(s.frac[3 * o + 2], (double)ic);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    double v = __dadd_rn(__dmul_rn(ra, s.lat[k]), __dmul_rn(rb, s.lat[3 + k]));
    v = __dadd_rn(v, __dmul_rn(rc, s.lat[6 + k]));
    p[k] = __dadd_rn(v, s.origin[k]);
  }
}

// dr of a term i -> j whose unwrapped ket cell is (ja0, jb0, jc0)
// (super.pyx:736-753): ((((pj - pi) + na*S0) + nb*S1) + nc*S2)
__device__ __forceinline__ void term_dr(const ScDev& s, const double pi[3], const double pj[3],
                                        int ja0, int jb0, int jc0, double& dx, double& dy) {
  const double na = (double)floor_div(ja0, s.dim[0]);
  const double nb = (double)floor_div(jb0, s.dim[1]);
  const double nc = (double)floor_div(jc0, s.dim[2]);
  double d[2];
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    double v = __dsub_rn(pj[k], pi[k]);
    v = __dadd_rn(v, __dmul_rn(na, s.S[k]));
    v = __dadd_rn(v, __dmul_rn(nb, s.S[3 + k]));
    d[k] = __dadd_rn(v, __dmul_rn(nc, s.S[6 + k]));
  }
  dx = d[0];
  dy = d[1];
}

// Peierls phase of the term i -> j (sample.pyx:50-72); gfac carries
// factor*B (gauge 0), (-factor)*B (gauge 1) or (factor*0.5)*B (gauge 2)
__device__ __forceinline__ double phase(const ScDev& s, const double pi[3], const double pj[3],
                                        double dx, double dy) {
  if (s.gauge == 0) return __dmul_rn(__dmul_rn(s.gfac, dx), __dadd_rn(pj[1], pi[1]));
  if (s.gauge == 1) return __dmul_rn(__dmul_rn(s.gfac, dy), __dadd_rn(pj[0], pi[0]));
  const double sx = __dadd_rn(pj[0], pi[0]);
  const double sy = __dadd_rn(pj[1], pi[1]);
  return __dmul_rn(s.gfac, __dsub_rn(__dmul_rn(dx, sx), __dmul_rn(dy, sy)));
}

// h * (cos + i sin) with the operation order of a complex product
__device__ __forceinline__ void apply_phase(double ph, double& vr, double& vi) {
  double sn, cs;
  sincos(ph, &sn, &cs);
  const double r = __dsub_rn(__dmul_rn(vr, cs), __dmul_rn(vi, sn));
  const double i = __dadd_rn(__dmul_rn(vr, sn), __dmul_rn(vi, cs));
  vr = r;
  vi = i;
}

// position of term ih in the reference's hopping list
__device__ __forceinline__ unsigned long long term_key(const ScDev& s, bool is_pbc,
                                                       int64_t bra_cell, int64_t bra_row,
                                                       int ih) {
  if (s.n_vac == 0 && is_pbc)  // build_hop_pbc: cells, then terms
    return (unsigned long long)bra_cell * s.n_hop + ih;
  // build_hop_gen (all terms with vacancies, the non-periodic rest without):
  // rows, then terms; after the periodic list in the fast case
  const unsigned long long base = s.n_vac == 0 ? (1ull << 62) : 0ull;
  return base + (unsigned long long)bra_row * s.n_hop + ih;
}

// All hopping entries of row r (unsorted); returns their count and the raw
// on-site energy.
template <int MAXT>
__device__ int gather_row(const ScDev& s, int64_t r, Term* t, double& e_raw) {
  const int64_t g = s.n_vac ? (int64_t)s.inv[r] : r;
  const int o = (int)(g % s.n_orb);
  const int64_t cell = g / s.n_orb;
  const int ic = (int)(cell % s.dim[2]);
  const int ib = (int)((cell / s.dim[2]) % s.dim[1]);
  const int ia = (int)(cell / ((int64_t)s.dim[2] * s.dim[1]));
  e_raw = s.sc_eng ? s.sc_eng[r] : s.pc_eng[o];
  const bool pos = s.field || s.need_dr;
  double p_me[3] = {0, 0, 0};
  if (pos) orb_pos(s, ia, ib, ic, o, p_me);
  int n = 0;
  for (int k = s.fwd_off[o]; k < s.fwd_off[o + 1]; ++k) {
    const int ih = s.fwd_ih[k];
    const HopTerm h = s.hop[ih];
    const int ja0 = ia + h.r[0], jb0 = ib + h.r[1], jc0 = ic + h.r[2];
    const int ja = wrap_idx(ja0, s.dim[0], s.pbc[0]);
    const int jb = wrap_idx(jb0, s.dim[1], s.pbc[1]);
    const int jc = wrap_idx(jc0, s.dim[2], s.pbc[2]);
    if (ja < 0 || jb < 0 || jc < 0) continue;
    const int64_t col = row_of(s, full_index(s, ja, jb, jc, h.ket));
    if (col < 0 || n >= MAXT) continue;
    Term& e = t[n++];
    e.key = term_key(s, h.is_pbc, cell, r, ih);
    e.col = (int)col;
    e.kind = 1;
    e.vr = h.er;
    e.vi = h.ei;
    e.dx = e.dy = 0.0;
    if (pos) {
      double pj[3];
      orb_pos(s, ja, jb, jc, h.ket, pj);
      term_dr(s, p_me, pj, ja0, jb0, jc0, e.dx, e.dy);
      if (s.field) apply_phase(phase(s, p_me, pj, e.dx, e.dy), e.vr, e.vi);
    }
  }
  for (int k = s.bwd_off[o]; k < s.bwd_off[o + 1]; ++k) {
    const int ih = s.bwd_ih[k];
    const HopTerm h = s.hop[ih];
    // bra cell (sa, sb, sc) with (sa + R) wrapped == this cell
    int sa = wrap_idx(ia - h.r[0], s.dim[0], s.pbc[0]);
    int sb = wrap_idx(ib - h.r[1], s.dim[1], s.pbc[1]);
    int sc = wrap_idx(ic - h.r[2], s.dim[2], s.pbc[2]);
    if (sa < 0 || sb < 0 || sc < 0) continue;
    const int64_t g_bra = full_index(s, sa, sb, sc, h.bra);
    const int64_t col = row_of(s, g_bra);
    if (col < 0 || n >= MAXT) continue;
    Term& e = t[n++];
    const int64_t bra_cell = g_bra / s.n_orb;
    e.key = term_key(s, h.is_pbc, bra_cell, col, ih);
    e.col = (int)col;
    e.kind = 2;
    e.vr = h.er;
    e.vi = h.ei;
    e.dx = e.dy = 0.0;
    if (pos) {
      double pb[3];
      orb_pos(s, sa, sb, sc, h.bra, pb);
      // dr and phase of the term as the bra row stores it
      term_dr(s, pb, p_me, sa + h.r[0], sb + h.r[1], sc + h.r[2], e.dx, e.dy);
      if (s.field) apply_phase(phase(s, pb, p_me, e.dx, e.dy), e.vr, e.vi);
    }
  }
  return n;
}

template <class Less>
__device__ __forceinline__ void insertion_sort(Term* t, int n, Less less) {
  for (int i = 1; i < n; ++i) {
    Term x = t[i];
    int j = i - 1;
    while (j >= 0 && less(x, t[j])) {
      t[j + 1] = t[j];
      --j;
    }
    t[j + 1] = x;
  }
}

struct ByKey {
  __device__ bool operator()(const Term& a, const Term& b) const { return a.key < b.key; }
};
struct ByCol {
  __device__ bool operator()(const Term& a, const Term& b) const {
    return a.col < b.col || (a.col == b.col && a.key < b.key);
  }
};

// x * (scale + 0i) as a complex product (builder/sample.py:296-297)
__device__ __forceinline__ void scale_c(double scale, double& vr, double& vi) {
  const double r = __dsub_rn(__dmul_rn(vr, scale), __dmul_rn(vi, 0.0));
  const double i = __dadd_rn(__dmul_rn(vr, 0.0), __dmul_rn(vi, scale));
  vr = r;
  vi = i;
}

// An output entry of row r after ordering, merging and rescaling.
struct Out {
  int col;
  double vr, vi, dx, dy;
};

// Final entries of row r in the layout's order (at most MAXT + 1).
template <int MAXT>
__device__ int row_entries(const ScDev& s, int64_t r, Term* t, Out* out) {
  double e_raw;
  const int n = gather_row<MAXT>(s, r, t, e_raw);
  const double d = __dmul_rn(e_raw, s.scale);
  for (int i = 0; i < n; ++i) {
    scale_c(s.scale, t[i].vr, t[i].vi);
    if (t[i].kind == 2) {
      t[i].vi = -t[i].vi;
      t[i].dx = -t[i].dx;
      t[i].dy = -t[i].dy;
    }
  }
  int m = 0;
  if (s.layout == TBPM_LAYOUT_DXY) {
    if (fabs(d) >= s.cutoff) out[m++] = Out{(int)r, d, 0.0, 0.0, 0.0};
    insertion_sort(t, n, ByKey());
    for (int i = 0; i < n; ++i) out[m++] = Out{t[i].col, t[i].vr, t[i].vi, t[i].dx, t[i].dy};
    return m;
  }
  // build_ham_csr = (diag + half) + half^H: per column ((d or 0) + h) + b with
  // absent parts 0 (scipy's sparse sum), explicit zeros dropped
  insertion_sort(t, n, ByCol());
  bool diag_done = false;
  int i = 0;
  while (i < n || !diag_done) {
    const int col = (!diag_done && (i >= n || (int)r <= t[i].col)) ? (int)r : t[i].col;
    double hr = 0.0, hi = 0.0, br = 0.0, bi = 0.0, dx = 0.0, dy = 0.0;
    bool first = true;
    while (i < n && t[i].col == col) {
      if (t[i].kind == 1) {
        hr = __dadd_rn(hr, t[i].vr);
        hi = __dadd_rn(hi, t[i].vi);
      } else {
        br = __dadd_rn(br, t[i].vr);
        bi = __dadd_rn(bi, t[i].vi);
      }
      if (first) {
        dx = t[i].dx;
        dy = t[i].dy;
        first = false;
      }
      ++i;
    }
    if (col == (int)r) diag_done = true;
    const double vr = __dadd_rn(__dadd_rn(col == (int)r ? d : 0.0, hr), br);
    const double vi = __dadd_rn(__dadd_rn(0.0, hi), bi);
    if (vr != 0.0 || vi != 0.0) out[m++] = Out{col, vr, vi, dx, dy};
  }
  return m;
}

// ---- passes ---------------------------------------------------------------

__global__ void sc_inverse_kernel(ScDev s, int32_t* inv) {
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < s.n_full;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = row_of(s, g);
    if (r >= 0) inv[r] = (int32_t)g;
  }
}

// get_rescale (sample.pyx:105-115): orb_eng + sum of |h| in list order; block
// maxima into bmax
template <int MAXT>
__global__ void __launch_bounds__(256) sc_rowsum_kernel(ScDev s, double* bmax) {
  Term t[MAXT];
  double best = -INFINITY;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < s.n_rows;
       r += (int64_t)gridDim.x * blockDim.x) {
    double sum;
    const int n = gather_row<MAXT>(s, r, t, sum);
    insertion_sort(t, n, ByKey());
    for (int i = 0; i < n; ++i) {
      const double a = __dsqrt_rn(__dadd_rn(__dmul_rn(t[i].vr, t[i].vr),
                                            __dmul_rn(t[i].vi, t[i].vi)));
      sum = __dadd_rn(sum, a);
    }
    best = fmax(best, sum);
  }
  __shared__ double red[256];
  red[threadIdx.x] = best;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) bmax[blockIdx.x] = red[0];
}

// entries per row: all of them (full CSR) or the off-diagonal ones (resident
// H = D + O); diag_rows counts rows with an on-site entry
template <int MAXT>
__global__ void __launch_bounds__(256) sc_count_kernel(ScDev s, int split, int32_t* count,
                                                       unsigned long long* diag_rows) {
  Term t[MAXT];
  Out o[MAXT + 1];
  unsigned long long nd = 0;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < s.n_rows;
       r += (int64_t)gridDim.x * blockDim.x) {
    const int m = row_entries<MAXT>(s, r, t, o);
    int c = m, dg = 0;
    for (int i = 0; i < m; ++i) dg += (o[i].col == (int)r);
    if (split) c -= dg;
    nd += dg > 0;
    count[r] = c;
  }
  for (int w = 16; w > 0; w >>= 1) nd += __shfl_xor_sync(0xffffffffu, nd, w);
  if ((threadIdx.x & 31) == 0 && nd) atomicAdd(diag_rows, nd);
}

// full CSR for download
template <int MAXT>
__global__ void __launch_bounds__(256) sc_fill_full_kernel(ScDev s, const int64_t* off,
                                                           int32_t* indices, double2* val,
                                                           double* dx, double* dy) {
  Term t[MAXT];
  Out o[MAXT + 1];
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < s.n_rows;
       r += (int64_t)gridDim.x * blockDim.x) {
    const int m = row_entries<MAXT>(s, r, t, o);
    int64_t p = off[r];
    for (int i = 0; i < m; ++i, ++p) {
      indices[p] = o[i].col;
      val[p] = make_double2(o[i].vr, o[i].vi);
      if (dx) {
        dx[p] = o[i].dx;
        dy[p] = o[i].dy;
      }
    }
  }
}

// resident H = D + O of the context, in precision R
template <int MAXT, typename R>
__global__ void __launch_bounds__(256) sc_fill_split_kernel(
    ScDev s, const int64_t* off, int32_t* indptr, int32_t* indices,
    typename Cx<R>::t* val, R* dx, R* dy, typename Cx<R>::t* diag) {
  using C = typename Cx<R>::t;
  Term t[MAXT];
  Out o[MAXT + 1];
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < s.n_rows;
       r += (int64_t)gridDim.x * blockDim.x) {
    const int m = row_entries<MAXT>(s, r, t, o);
    int64_t p = off[r];
    indptr[r] = (int32_t)p;
    if (r == s.n_rows - 1) indptr[s.n_rows] = (int32_t)off[s.n_rows];
    double gr = 0.0, gi = 0.0;
    for (int i = 0; i < m; ++i) {
      if (o[i].col == (int)r) {
        gr = __dadd_rn(gr, o[i].vr);
        gi = __dadd_rn(gi, o[i].vi);
        continue;
      }
      indices[p] = o[i].col;
      C v;
      v.x = (R)o[i].vr;
      v.y = (R)o[i].vi;
      val[p] = v;
      if (dx) {
        dx[p] = (R)o[i].dx;
        dy[p] = (R)o[i].dy;
      }
      ++p;
    }
    if (diag) {
      C v;
      v.x = (R)gr;
      v.y = (R)gi;
      diag[r] = v;
    }
  }
}

// ---- host side ---------------------------------------------------------------

struct Tables {
  DevMem frac, pc_eng, sc_eng, hop, fwd_off, fwd_ih, bwd_off, bwd_ih, vac, inv;
};

template <typename T>
void upload(DevMem& m, const T* src, size_t count, cudaStream_t st) {
  m.ensure(std::max<size_t>(count, 1) * sizeof(T));
  if (count) TBPM_CK(cudaMemcpyAsync(m.p, src, count * sizeof(T), cudaMemcpyHostToDevice, st));
}

int grid_for(int64_t n, int threads) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t want = (n + threads - 1) / threads;
  return (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)sms * 16));
}

struct Prepared {
  ScDev s{};
  Tables tb;
  int maxt = 0;
  double rescale = 1.0;
};

void prepare(tbpm_ctx* c, const tbpm_supercell* sc, int layout, double cutoff, Prepared& P) {
  if (!sc || !sc->lat_vec || !sc->orb_pos || !sc->orb_eng)
    throw Error{TBPM_ERR_ARG, "supercell: null primitive-cell array"};
  if (sc->n_orb < 1) throw Error{TBPM_ERR_ARG, "supercell: no orbitals"};
  if (sc->n_hop < 0 || (sc->n_hop > 0 && (!sc->hop_ind || !sc->hop_eng)))
    throw Error{TBPM_ERR_ARG, "supercell: null hopping arrays"};
  if (sc->n_hop > 65535) throw Error{TBPM_ERR_ARG, "supercell: more than 65535 hopping terms"};
  if (layout != TBPM_LAYOUT_CSR && layout != TBPM_LAYOUT_DXY)
    throw Error{TBPM_ERR_ARG, "supercell: unknown layout"};
  if (sc->b_field != 0.0 && (sc->gauge < 0 || sc->gauge > 2))
    throw Error{TBPM_ERR_ARG, "Illegal gauge (0, 1 or 2)"};
  ScDev& s = P.s;
  const int n_orb = sc->n_orb, n_hop = sc->n_hop;
  for (int k = 0; k < 3; ++k) {
    if (sc->dim[k] < 1) throw Error{TBPM_ERR_ARG, "supercell: dimension must be positive"};
    s.dim[k] = sc->dim[k];
    s.pbc[k] = sc->pbc[k] ? 1 : 0;
  }
  // SuperCell dimension check (builder/super.py:132-139)
  for (int k = 0; k < 3; ++k) {
    int rmax = 0;
    for (int h = 0; h < n_hop; ++h) rmax = std::max(rmax, std::abs(sc->hop_ind[5 * h + k]));
    if (n_hop > 0 && sc->dim[k] < 2 * rmax + 1)
      throw Error{TBPM_ERR_ARG, "supercell: dimension " + std::to_string(k) +
                                    " must be at least " + std::to_string(2 * rmax + 1)};
  }
  const int64_t n_cells = (int64_t)s.dim[0] * s.dim[1] * s.dim[2];
  const int64_t n_full = n_cells * n_orb;
  if (n_full > (int64_t)INT32_MAX) throw Error{TBPM_ERR_ARG, "supercell: more than 2^31-1 orbitals"};
  std::vector<HopTerm> hop((size_t)std::max(n_hop, 1));
  std::vector<std::vector<int>> fwd(n_orb), bwd(n_orb);
  for (int h = 0; h < n_hop; ++h) {
    const int32_t* q = sc->hop_ind + 5 * h;
    if (q[3] < 0 || q[3] >= n_orb || q[4] < 0 || q[4] >= n_orb)
      throw Error{TBPM_ERR_ARG, "supercell: hopping orbital index out of range"};
    if (q[0] == 0 && q[1] == 0 && q[2] == 0 && q[3] == q[4])
      throw Error{TBPM_ERR_ARG, "supercell: on-site term given as a hopping"};
    HopTerm& t = hop[h];
    bool pb = true;
    for (int k = 0; k < 3; ++k) {
      t.r[k] = q[k];
      if (!s.pbc[k] && q[k] != 0) pb = false;
    }
    t.bra = q[3];
    t.ket = q[4];
    t.is_pbc = pb ? 1 : 0;
    t.er = sc->hop_eng[2 * h];
    t.ei = sc->hop_eng[2 * h + 1];
    fwd[q[3]].push_back(h);
    bwd[q[4]].push_back(h);
  }
  std::vector<int> fo(n_orb + 1, 0), bo(n_orb + 1, 0), fi, bi;
  int maxt = 0;
  for (int o = 0; o < n_orb; ++o) {
    fo[o + 1] = fo[o] + (int)fwd[o].size();
    bo[o + 1] = bo[o] + (int)bwd[o].size();
    fi.insert(fi.end(), fwd[o].begin(), fwd[o].end());
    bi.insert(bi.end(), bwd[o].begin(), bwd[o].end());
    maxt = std::max(maxt, (int)(fwd[o].size() + bwd[o].size()));
  }
  if (maxt > 64)
    throw Error{TBPM_ERR_ARG, "supercell: more than 64 hopping terms touch one orbital"};
  P.maxt = maxt;
  const int64_t n_vac = sc->vac_id_sc ? sc->n_vac : 0;
  for (int64_t v = 0; v < n_vac; ++v) {
    if (sc->vac_id_sc[v] < 0 || sc->vac_id_sc[v] >= n_full)
      throw Error{TBPM_ERR_ARG, "supercell: vacancy index out of range"};
    if (v && sc->vac_id_sc[v] <= sc->vac_id_sc[v - 1])
      throw Error{TBPM_ERR_ARG, "supercell: vacancy indices must be sorted and unique"};
  }
  const int64_t n_rows = n_full - n_vac;
  if (n_rows < 1) throw Error{TBPM_ERR_ARG, "supercell: every orbital is a vacancy"};
  // lattice of the supercell: pc lattice rows times dim (builder/super.py:865-868)
  for (int i = 0; i < 3; ++i)
    for (int k = 0; k < 3; ++k) {
      s.lat[3 * i + k] = sc->lat_vec[3 * i + k];
      s.S[3 * i + k] = sc->lat_vec[3 * i + k] * (double)sc->dim[i];
    }
  for (int k = 0; k < 3; ++k) s.origin[k] = sc->origin ? sc->origin[k] : 0.0;
  s.n_orb = n_orb;
  s.n_hop = n_hop;
  s.n_rows = n_rows;
  s.n_full = n_full;
  s.n_vac = n_vac;
  s.layout = layout;
  s.cutoff = cutoff;
  s.need_dr = 0;
  s.field = sc->b_field != 0.0 ? 1 : 0;
  s.gauge = sc->gauge;
  const double factor = M_PI / 4135.666734;  // sample.pyx:48
  if (s.gauge == 0)
    s.gfac = factor * sc->b_field;
  else if (s.gauge == 1)
    s.gfac = -factor * sc->b_field;
  else
    s.gfac = factor * 0.5 * sc->b_field;

  cudaStream_t st = c->stream;
  Tables& T = P.tb;
  std::vector<double> frac(3 * (size_t)n_orb);
  for (size_t i = 0; i < frac.size(); ++i) frac[i] = sc->orb_pos[i];
  upload(T.frac, frac.data(), frac.size(), st);
  upload(T.pc_eng, sc->orb_eng, (size_t)n_orb, st);
  upload(T.hop, hop.data(), hop.size(), st);
  upload(T.fwd_off, fo.data(), fo.size(), st);
  upload(T.bwd_off, bo.data(), bo.size(), st);
  upload(T.fwd_ih, fi.data(), fi.size(), st);
  upload(T.bwd_ih, bi.data(), bi.size(), st);
  s.frac = T.frac.as<double>();
  s.pc_eng = T.pc_eng.as<double>();
  s.hop = T.hop.as<HopTerm>();
  s.fwd_off = T.fwd_off.as<int>();
  s.fwd_ih = T.fwd_ih.as<int>();
  s.bwd_off = T.bwd_off.as<int>();
  s.bwd_ih = T.bwd_ih.as<int>();
  s.sc_eng = nullptr;
  if (sc->sc_orb_eng) {
    upload(T.sc_eng, sc->sc_orb_eng, (size_t)n_rows, st);
    s.sc_eng = T.sc_eng.as<double>();
  }
  s.vac = nullptr;
  s.inv = nullptr;
  if (n_vac) {
    upload(T.vac, sc->vac_id_sc, (size_t)n_vac, st);
    s.vac = T.vac.as<int64_t>();
    T.inv.ensure((size_t)n_rows * 4);
    s.inv = T.inv.as<int32_t>();
    sc_inverse_kernel<<<grid_for(n_full, 256), 256, 0, st>>>(s, T.inv.as<int32_t>());
    TBPM_CK(cudaGetLastError());
  }
  // rescale: fixed, or estimated like Sample.get_rescale on the unscaled terms
  if (sc->rescale > 0.0) {
    P.rescale = sc->rescale;
  } else {
    const int grid = grid_for(n_rows, 256);
    DevMem bmax;
    bmax.ensure((size_t)grid * 8);
    s.scale = 1.0;
    switch (maxt <= 8 ? 8 : maxt <= 16 ? 16 : maxt <= 32 ? 32 : 64) {
      case 8: sc_rowsum_kernel<8><<<grid, 256, 0, st>>>(s, bmax.as<double>()); break;
      case 16: sc_rowsum_kernel<16><<<grid, 256, 0, st>>>(s, bmax.as<double>()); break;
      case 32: sc_rowsum_kernel<32><<<grid, 256, 0, st>>>(s, bmax.as<double>()); break;
      default: sc_rowsum_kernel<64><<<grid, 256, 0, st>>>(s, bmax.as<double>()); break;
    }
    TBPM_CK(cudaGetLastError());
    std::vector<double> h((size_t)grid);
    TBPM_CK(cudaMemcpyAsync(h.data(), bmax.p, (size_t)grid * 8, cudaMemcpyDeviceToHost, st));
    TBPM_CK(cudaStreamSynchronize(st));
    double m = -INFINITY;
    for (double v : h) m = std::max(m, v);
    if (!(m > 0.0) || !std::isfinite(m))
      throw Error{TBPM_ERR_ARG, "supercell: estimated rescale factor is not positive"};
    P.rescale = m;
  }
  // builder/sample.py:296-297: values times (1.0 / factor)
  s.scale = 1.0 / P.rescale;
}

template <int MAXT>
void launch_count(const Prepared& P, int split, int32_t* count, unsigned long long* nd,
                  cudaStream_t st) {
  sc_count_kernel<MAXT><<<grid_for(P.s.n_rows, 256), 256, 0, st>>>(P.s, split, count, nd);
}

void count_rows(const Prepared& P, int split, int32_t* count, unsigned long long* nd,
                cudaStream_t st) {
  const int m = P.maxt;
  if (m <= 8)
    launch_count<8>(P, split, count, nd, st);
  else if (m <= 16)
    launch_count<16>(P, split, count, nd, st);
  else if (m <= 32)
    launch_count<32>(P, split, count, nd, st);
  else
    launch_count<64>(P, split, count, nd, st);
  TBPM_CK(cudaGetLastError());
}

template <int MAXT>
void launch_fill_full(const Prepared& P, const int64_t* off, int32_t* ix, double2* v,
                      double* dx, double* dy, cudaStream_t st) {
  sc_fill_full_kernel<MAXT><<<grid_for(P.s.n_rows, 256), 256, 0, st>>>(P.s, off, ix, v, dx, dy);
}

template <int MAXT, typename R>
void launch_fill_split(const Prepared& P, const int64_t* off, Ham& h, bool dxy, bool diag,
                       cudaStream_t st) {
  using C = typename Cx<R>::t;
  sc_fill_split_kernel<MAXT, R><<<grid_for(P.s.n_rows, 256), 256, 0, st>>>(
      P.s, off, h.indptr.as<int32_t>(), h.indices.as<int32_t>(), h.hop.as<C>(),
      dxy ? h.dx.as<R>() : nullptr, dxy ? h.dy.as<R>() : nullptr,
      diag ? h.diag.as<C>() : nullptr);
}

template <typename R>
void fill_split(const Prepared& P, const int64_t* off, Ham& h, bool dxy, bool diag,
                cudaStream_t st) {
  const int m = P.maxt;
  if (m <= 8)
    launch_fill_split<8, R>(P, off, h, dxy, diag, st);
  else if (m <= 16)
    launch_fill_split<16, R>(P, off, h, dxy, diag, st);
  else if (m <= 32)
    launch_fill_split<32, R>(P, off, h, dxy, diag, st);
  else
    launch_fill_split<64, R>(P, off, h, dxy, diag, st);
  TBPM_CK(cudaGetLastError());
}

}  // namespace

// Build the Hamiltonian of the supercell and keep it resident in the context
// (in place of tbpm_ham_upload of a host CSR).
void drv_supercell_ham(tbpm_ctx* c, const tbpm_supercell* sc, int layout, double cutoff,
                       int64_t* n_rows, int64_t* nnz, double* rescale) {
  Phase phase("tbpm_supercell_ham");
  Prepared P;
  prepare(c, sc, layout, cutoff, P);
  const bool dxy = layout == TBPM_LAYOUT_DXY;
  P.s.need_dr = dxy ? 1 : 0;
  cudaStream_t st = c->stream;
  const int64_t n = P.s.n_rows;
  DevMem count, off, nd;
  count.ensure((size_t)n * 4);
  off.ensure((size_t)(n + 1) * 8);
  nd.ensure(8);
  TBPM_CK(cudaMemsetAsync(nd.p, 0, 8, st));
  count_rows(P, 1, count.as<int32_t>(), nd.as<unsigned long long>(), st);
  const int64_t n_off = scan_counts(count.as<int32_t>(), n, off.as<int64_t>(), st);
  unsigned long long n_diag = 0;
  TBPM_CK(cudaMemcpyAsync(&n_diag, nd.p, 8, cudaMemcpyDeviceToHost, st));
  TBPM_CK(cudaStreamSynchronize(st));
  if (n_off > (int64_t)INT32_MAX)
    throw Error{TBPM_ERR_ARG, "supercell: more than 2^31-1 off-diagonal entries"};
  count.release();
  c->graph.reset();
  c->sess.active = false;
  Ham& h = c->ham;
  h.n = 0;
  const bool fp64 = c->opts.precision == TBPM_PREC_FP64;
  const size_t rs = fp64 ? 8 : 4;
  h.indptr.ensure((size_t)(n + 1) * 4);
  h.indices.ensure((size_t)std::max<int64_t>(n_off, 1) * 4);
  h.hop.ensure((size_t)std::max<int64_t>(n_off, 1) * 2 * rs);
  const bool has_diag = n_diag > 0;
  if (has_diag) h.diag.ensure((size_t)n * 2 * rs);
  if (dxy) {
    h.dx.ensure((size_t)std::max<int64_t>(n_off, 1) * rs);
    h.dy.ensure((size_t)std::max<int64_t>(n_off, 1) * rs);
  }
  if (fp64)
    fill_split<double>(P, off.as<int64_t>(), h, dxy, has_diag, st);
  else
    fill_split<float>(P, off.as<int64_t>(), h, dxy, has_diag, st);
  TBPM_CK(cudaStreamSynchronize(st));
  h.has_diag = has_diag;
  h.has_dxy = dxy;
  h.prec = c->opts.precision;
  h.n = n;
  h.nnz = n_off;
  h.rescale = P.rescale;
  ++h.gen;
  if (n_rows) *n_rows = n;
  if (nnz) *nnz = n_off + (int64_t)n_diag;
  if (rescale) *rescale = P.rescale;
}

// Build the full CSR of the supercell and copy it to host arrays (sizes only
// when indptr is null).
void drv_supercell_csr(tbpm_ctx* c, const tbpm_supercell* sc, int layout, double cutoff,
                       int64_t* n_rows, int64_t* nnz, double* rescale, int64_t* indptr,
                       int32_t* indices, double* hop, double* dx, double* dy) {
  Phase phase("tbpm_supercell_csr");
  Prepared P;
  prepare(c, sc, layout, cutoff, P);
  const bool dxy = layout == TBPM_LAYOUT_DXY;
  const bool want_dr = dxy && dx && dy;
  P.s.need_dr = want_dr ? 1 : 0;
  cudaStream_t st = c->stream;
  const int64_t n = P.s.n_rows;
  DevMem count, off, nd;
  count.ensure((size_t)n * 4);
  off.ensure((size_t)(n + 1) * 8);
  nd.ensure(8);
  TBPM_CK(cudaMemsetAsync(nd.p, 0, 8, st));
  count_rows(P, 0, count.as<int32_t>(), nd.as<unsigned long long>(), st);
  const int64_t total = scan_counts(count.as<int32_t>(), n, off.as<int64_t>(), st);
  count.release();
  if (n_rows) *n_rows = n;
  if (nnz) *nnz = total;
  if (rescale) *rescale = P.rescale;
  if (!indptr) return;
  if (!indices || !hop) throw Error{TBPM_ERR_ARG, "supercell: null output array"};
  DevMem ix, val, ddx, ddy;
  ix.ensure((size_t)std::max<int64_t>(total, 1) * 4);
  val.ensure((size_t)std::max<int64_t>(total, 1) * 16);
  if (want_dr) {
    ddx.ensure((size_t)std::max<int64_t>(total, 1) * 8);
    ddy.ensure((size_t)std::max<int64_t>(total, 1) * 8);
  }
  const int m = P.maxt;
  double* px = want_dr ? ddx.as<double>() : nullptr;
  double* py = want_dr ? ddy.as<double>() : nullptr;
  if (m <= 8)
    launch_fill_full<8>(P, off.as<int64_t>(), ix.as<int32_t>(), val.as<double2>(), px, py, st);
  else if (m <= 16)
    launch_fill_full<16>(P, off.as<int64_t>(), ix.as<int32_t>(), val.as<double2>(), px, py, st);
  else if (m <= 32)
    launch_fill_full<32>(P, off.as<int64_t>(), ix.as<int32_t>(), val.as<double2>(), px, py, st);
  else
    launch_fill_full<64>(P, off.as<int64_t>(), ix.as<int32_t>(), val.as<double2>(), px, py, st);
  TBPM_CK(cudaGetLastError());
  TBPM_CK(cudaMemcpyAsync(indptr, off.p, (size_t)(n + 1) * 8, cudaMemcpyDeviceToHost, st));
  if (total) {
    TBPM_CK(cudaMemcpyAsync(indices, ix.p, (size_t)total * 4, cudaMemcpyDeviceToHost, st));
    TBPM_CK(cudaMemcpyAsync(hop, val.p, (size_t)total * 16, cudaMemcpyDeviceToHost, st));
    if (want_dr) {
      TBPM_CK(cudaMemcpyAsync(dx, ddx.p, (size_t)total * 8, cudaMemcpyDeviceToHost, st));
      TBPM_CK(cudaMemcpyAsync(dy, ddy.p, (size_t)total * 8, cudaMemcpyDeviceToHost, st));
    }
  }
  TBPM_CK(cudaStreamSynchronize(st));
}

}  // namespace tbpm
