// TEST INFRASTRUCTURE ONLY -- the CPU oracle for the TBPM hot path.
//
// A plain C++17/OpenMP restatement of the reference TBPLaS Fortran core
// (tbplas/fortran/*.f90 of deepmodeling/tbplas 1.6.0, non-MKL / non-BLAS /
// non-FFTW branches).  It exists so that tests, the smoke check and the
// CPU-baseline leg of bench.py can check and time the CUDA product against the
// reference algorithm.  Nothing in the product links or calls this file.
//
// The reference Fortran cannot be compiled on this machine (no Fortran
// compiler), so the oracle is pinned by (a) exact-diagonalisation known answers
// for the Chebyshev propagator and the Fermi operator, (b) the reference's own
// Python layer (Sample CSR builders, Bessel series, Analyzer), driven with this
// oracle behind an f2py-compatible shim, and (c) the Philox4x32-10 published
// known-answer vectors for the random-state stream.  The gfortran intrinsic
// RANDOM_NUMBER stream of the reference is not reproducible; the random-state
// *distribution* and seed plumbing are restated and the uniform source is the
// counter-based Philox stream shared (by specification, not by code) with the
// CUDA generator.
//
// Arithmetic follows the Fortran expression order where it is cheap to do so
// (e.g. csr.F90 accumulates `a*values(j)*in(k) + out(i)` left to right).

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

struct zc {
  double re, im;
};

inline zc zmk(double r, double i) { return zc{r, i}; }
inline zc zadd(zc a, zc b) { return zc{a.re + b.re, a.im + b.im}; }
inline zc zsub(zc a, zc b) { return zc{a.re - b.re, a.im - b.im}; }
inline zc zmul(zc a, zc b) {
  return zc{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
inline zc dmul(double a, zc b) { return zc{a * b.re, a * b.im}; }
inline zc zconj(zc a) { return zc{a.re, -a.im}; }
inline zc zdivd(zc a, double b) { return zc{a.re / b, a.im / b}; }
inline double zabs(zc a) { return std::hypot(a.re, a.im); }

constexpr double kPi = 3.14159265358979323846;  // const.f90:8

enum {
  ORC_OK = 0,
  ORC_ERR_ARG = 1,
  ORC_ERR_NORM = 2,
};

struct Csr {
  const int32_t* indptr;
  const int32_t* indices;
  const zc* values;
  int64_t n;
};

// csr.F90:71-101 (csr_mv): out(i) = values(j)*in(k) + out(i)
void csr_mv(const Csr& m, const zc* in, zc* out) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < m.n; ++i) {
    zc o = zmk(0, 0);
    for (int32_t j = m.indptr[i]; j < m.indptr[i + 1]; ++j)
      o = zadd(zmul(m.values[j], in[m.indices[j]]), o);
    out[i] = o;
  }
}

// csr.F90:140-171 (amv_z): out(i) = a*values(j)*in(k) + out(i), out zeroed
void amv_z(zc a, const Csr& m, const zc* in, zc* out) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < m.n; ++i) {
    zc o = zmk(0, 0);
    for (int32_t j = m.indptr[i]; j < m.indptr[i + 1]; ++j)
      o = zadd(zmul(zmul(a, m.values[j]), in[m.indices[j]]), o);
    out[i] = o;
  }
}

// csr.F90:104-137 (amv_d): real scale a
void amv_d(double a, const Csr& m, const zc* in, zc* out) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < m.n; ++i) {
    zc o = zmk(0, 0);
    for (int32_t j = m.indptr[i]; j < m.indptr[i + 1]; ++j)
      o = zadd(zmul(dmul(a, m.values[j]), in[m.indices[j]]), o);
    out[i] = o;
  }
}

// csr.F90:209-239 (amxpy_z): out(i) = a*values(j)*in(k) + out(i)
void amxpy_z(zc a, const Csr& m, const zc* in, zc* out) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < m.n; ++i) {
    zc o = out[i];
    for (int32_t j = m.indptr[i]; j < m.indptr[i + 1]; ++j)
      o = zadd(zmul(zmul(a, m.values[j]), in[m.indices[j]]), o);
    out[i] = o;
  }
}

// csr.F90:242-281 (amxpby_d): out(i) = b*out(i); out(i) += a*values(j)*in(k)
void amxpby_d(double a, const Csr& m, const zc* in, double b, zc* out) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < m.n; ++i) {
    zc o = dmul(b, out[i]);
    for (int32_t j = m.indptr[i]; j < m.indptr[i + 1]; ++j)
      o = zadd(zmul(dmul(a, m.values[j]), in[m.indices[j]]), o);
    out[i] = o;
  }
}

// math.F90:478-489 (dot_z = DOT_PRODUCT(X, Y)): serial sum of conjg(X)*Y
zc inner_prod(const zc* x, const zc* y, int64_t n) {
  zc s = zmk(0, 0);
  for (int64_t i = 0; i < n; ++i) s = zadd(s, zmul(zconj(x[i]), y[i]));
  return s;
}

// math.F90:504-515 (norm_z): sqrt(dble(DOT_PRODUCT(X, X)))
double norm_z(const zc* x, int64_t n) { return std::sqrt(inner_prod(x, x, n).re); }

// propagation.f90:12-49 (cheb_wf_timestep)
void cheb_wf_timestep(const Csr& h, const double* bes, int n_bes, const zc* wf_in,
                      bool fwd, zc* wf_out, std::vector<zc>& t0,
                      std::vector<zc>& t1) {
  const int64_t n = h.n;
  const zc img_dt = fwd ? zmk(0, 1) : zmk(0, -1);
  const zc m1 = zmk(-img_dt.re, -img_dt.im);
  const zc m2 = zmk(-2 * img_dt.re, -2 * img_dt.im);
  amv_z(m1, h, wf_in, t0.data());  // Tcheb0 = amv(-img_dt, H, wf_in)
  amv_z(m2, h, t0.data(), t1.data());
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) t1[i] = zadd(t1[i], wf_in[i]);  // .pAdd.
  const double a = bes[0], b = 2 * bes[1], c = 2 * bes[2];
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i)  // math.F90:684-700 axpbypcz
    wf_out[i] = zadd(zadd(dmul(a, wf_in[i]), dmul(b, t0[i])), dmul(c, t1[i]));
  zc* p0 = t0.data();
  zc* p1 = t1.data();
  for (int k = 3; k < n_bes; ++k) {
    zc* p2 = p0;
    amxpy_z(m2, h, p1, p0);  // p2 = -2*img_dt*H*p1 + p0
    const double w = 2 * bes[k];
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) wf_out[i] = zadd(dmul(w, p2[i]), wf_out[i]);
    p0 = p1;
    p1 = p2;
  }
}

// propagation.f90:52-82 (Fermi)
void fermi_op(const Csr& h, const double* coef, int n_coef, const zc* wf_in,
              zc* wf_out, std::vector<zc>& t0, std::vector<zc>& t1) {
  const int64_t n = h.n;
  csr_mv(h, wf_in, t0.data());
  amv_d(2.0, h, t0.data(), t1.data());
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) t1[i] = zsub(t1[i], wf_in[i]);  // .pSub.
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i)
    wf_out[i] = zadd(zadd(dmul(coef[0], wf_in[i]), dmul(coef[1], t0[i])),
                     dmul(coef[2], t1[i]));
  zc* p0 = t0.data();
  zc* p1 = t1.data();
  for (int k = 3; k < n_coef; ++k) {
    zc* p2 = p0;
    amxpby_d(2.0, h, p1, -1.0, p0);
    const double w = coef[k];
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) wf_out[i] = zadd(dmul(w, p2[i]), wf_out[i]);
    p0 = p1;
    p1 = p2;
  }
}

// funcs.f90:175-192 (check_norm): returns true when the norm is broken
bool norm_broken(const zc* wf, int64_t n, zc norm_ref, double eps) {
  const double dnorm = zabs(zsub(inner_prod(wf, wf, n), norm_ref));
  return std::isnan(dnorm) || !std::isfinite(dnorm) || dnorm > eps;
}

// funcs.f90:12-33 (current_coefficient): cur = (i*value)*hop*dr
void current_coefficient(const zc* hop, const double* dr, int64_t n_hop, double value,
                         std::vector<zc>& cur) {
  const zc alpha = zmk(0, value);
  cur.resize(n_hop);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n_hop; ++i) {
    const zc ah = zmul(alpha, hop[i]);
    cur[i] = zmk(ah.re * dr[i], ah.im * dr[i]);
  }
}

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC'11): 10 rounds of the 4x32 Philox S-box with the paper's
// multipliers and Weyl key increments.
// ---------------------------------------------------------------------------
inline void philox4x32_10(uint32_t ctr[4], uint32_t key0, uint32_t key1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
  uint32_t k0 = key0, k1 = key1;
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)M0 * ctr[0];
    const uint64_t p1 = (uint64_t)M1 * ctr[2];
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    const uint32_t n0 = hi1 ^ ctr[1] ^ k0;
    const uint32_t n2 = hi0 ^ ctr[3] ^ k1;
    ctr[0] = n0;
    ctr[1] = lo1;
    ctr[2] = n2;
    ctr[3] = lo0;
    k0 += W0;
    k1 += W1;
  }
}

// Two uniform doubles in [0,1) with 53-bit resolution for element j of the
// stream keyed by iseed.  The same mapping is specified for the CUDA generator.
inline void uniform_pair(int64_t iseed, int64_t j, double* f, double* g) {
  uint32_t c[4] = {(uint32_t)(uint64_t)j, (uint32_t)((uint64_t)j >> 32), 0x5442504Du,
                   0x00000000u};
  philox4x32_10(c, (uint32_t)(uint64_t)iseed, (uint32_t)((uint64_t)iseed >> 32));
  const double s = 1.0 / 9007199254740992.0;  // 2^-53
  *f = ((double)(c[0] >> 5) * 67108864.0 + (double)(c[1] >> 6)) * s;
  *g = ((double)(c[2] >> 5) * 67108864.0 + (double)(c[3] >> 6)) * s;
}

// random.f90:36-69 (random_state): |z|^2 ~ Exp(1), phase ~ U[0, 2pi),
// normalised by sqrt(sum |z|^2).  The seed passed by the drivers is
// seed*(i_sample + rank*n_ran_samples) (tbpm.f90:57); random.f90:52 then uses
// iseed*49741 to seed the stream, which is kept here as the Philox key.
// kind 0: exponential modulus (reference); kind 1: unit modulus.
void random_state(zc* wf, int64_t n, int64_t iseed, int kind) {
  const int64_t key = iseed * 49741;
  double sum = 0;
  for (int64_t i = 0; i < n; ++i) {
    double f, g;
    uniform_pair(key, i, &f, &g);
    const double abs_z_sq = kind == 0 ? -1.0 * std::log(1.0 - f) : 1.0;
    const double ph = 2 * kPi * g;
    const double r = std::sqrt(abs_z_sq);
    wf[i] = zmk(r * std::cos(ph), r * std::sin(ph));
    sum += abs_z_sq;
  }
  const double d = std::sqrt(sum);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) wf[i] = zdivd(wf[i], d);
}

// fft.F90:18-72 (fft1d_inplace, non-FFTW branch): in-place radix-2 DIF with
// bit-reversal at the end.  n must be a power of two.
void fft1d_inplace(zc* x, int64_t n, int sgn) {
  int64_t ncur = n;
  for (;;) {
    const int64_t ntmp = ncur;
    const double e = 2.0 * kPi / (double)ncur;
    ncur = ncur / 2;
    if (ncur < 1) break;
#pragma omp parallel for schedule(static)
    for (int64_t j = 1; j <= ncur; ++j) {
      const double ang = (double)sgn * e * (double)(j - 1);
      const zc w = zmk(std::cos(ang), std::sin(ang));
      for (int64_t i = j; i <= n; i += ntmp) {
        const int64_t itmp = i + ncur;
        const zc ctmp = zsub(x[i - 1], x[itmp - 1]);
        x[i - 1] = zadd(x[i - 1], x[itmp - 1]);
        x[itmp - 1] = zmul(ctmp, w);
      }
    }
  }
  int64_t j = 1;
  for (int64_t i = 1; i <= n - 1; ++i) {
    if (i < j) {
      const zc t = x[j - 1];
      x[j - 1] = x[i - 1];
      x[i - 1] = t;
    }
    int64_t k = n / 2;
    while (k < j) {
      j -= k;
      k /= 2;
    }
    j += k;
  }
}

// funcs.f90:36-57 (Fermi_dist)
double fermi_dist(double beta, double ef, double energy) {
  if (energy >= ef) {
    const double x = std::exp(beta * (ef - energy));
    return x / (1 + x);
  }
  const double x = std::exp(beta * (energy - ef));
  return 1 / (1 + x);
}

// kpm.f90:8-29 (jackson_kernel), first element pre-halved
void jackson_kernel(double* g, int64_t n_kernel) {
  g[0] = 0.5;
  const double q = kPi / (double)n_kernel;
  const double cotq = std::cos(q) / std::sin(q);
  for (int64_t k = 1; k < n_kernel; ++k)
    g[k] = ((double)(n_kernel - k) * std::cos(q * k) + cotq * std::sin(q * k)) /
           (double)n_kernel;
}

}  // namespace

extern "C" {

int orc_version(void) { return 1; }

void orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

int orc_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void orc_philox4x32_10(uint32_t* ctr, uint32_t key0, uint32_t key1) {
  philox4x32_10(ctr, key0, key1);
}

// random.f90:36-69 with the Philox uniform source (see random_state above)
void orc_random_state(double* wf, int64_t n, int64_t iseed, int kind) {
  random_state(reinterpret_cast<zc*>(wf), n, iseed, kind);
}

// funcs.f90:60-123 (get_Fermi_cheb_coef).  coef must hold nr_fermi doubles;
// returns n_cheb.
int orc_fermi_cheb_coef(double* coef, int nr_fermi, double beta, double mu,
                        int one_minus_fermi, double eps) {
  if (nr_fermi < 4 || (nr_fermi & (nr_fermi - 1))) return -1;
  std::vector<zc> cc(nr_fermi);
  const double r0 = 2 * kPi / nr_fermi;
  for (int i = 1; i <= nr_fermi; ++i) {
    const double energy = std::cos((double)(i - 1) * r0);
    const double f = fermi_dist(beta, mu, energy);
    cc[i - 1] = zmk(one_minus_fermi ? 1.0 - f : f, 0.0);
  }
  fft1d_inplace(cc.data(), nr_fermi, -1);
  int n_cheb = nr_fermi / 2;
  std::vector<double> kernel(n_cheb);
  jackson_kernel(kernel.data(), n_cheb);
  for (int i = 0; i < nr_fermi; ++i) coef[i] = 0.0;
  for (int i = 1; i <= n_cheb; ++i)
    coef[i - 1] = kernel[i - 1] * cc[i - 1].re / n_cheb;
  // truncation (funcs.f90:116-121); coef(n_cheb+1) is 0 here (it is an
  // unset element of the work array in the reference)
  for (int i = 1; i <= n_cheb; ++i) {
    if (std::fabs(coef[i - 1]) < eps && std::fabs(coef[i]) < eps) {
      n_cheb = i;
      break;
    }
  }
  return n_cheb;
}

// propagation.f90:12-49: one forward/backward time step of n_states vectors
int orc_cheb_timestep(const double* bes, int n_bes, const int32_t* indptr,
                      const int32_t* indices, const double* hop, int64_t n,
                      const double* wf_in, double* wf_out, int fwd) {
  if (n_bes < 3 || n < 1) return ORC_ERR_ARG;
  Csr h{indptr, indices, reinterpret_cast<const zc*>(hop), n};
  std::vector<zc> t0(n), t1(n);
  cheb_wf_timestep(h, bes, n_bes, reinterpret_cast<const zc*>(wf_in), fwd != 0,
                   reinterpret_cast<zc*>(wf_out), t0, t1);
  return ORC_OK;
}

// propagation.f90:52-82: Fermi operator applied to one vector
int orc_fermi(const double* coef, int n_coef, const int32_t* indptr,
              const int32_t* indices, const double* hop, int64_t n, const double* wf_in,
              double* wf_out) {
  if (n_coef < 3 || n < 1) return ORC_ERR_ARG;
  Csr h{indptr, indices, reinterpret_cast<const zc*>(hop), n};
  std::vector<zc> t0(n), t1(n);
  fermi_op(h, coef, n_coef, reinterpret_cast<const zc*>(wf_in), reinterpret_cast<zc*>(wf_out),
           t0, t1);
  return ORC_OK;
}

// tbpm.f90:6-93 (tbpm_dos).  wf0 (n_samples x n, complex) holds the initial
// states; when wf0 is null they are generated by random_state with the seed
// rule of tbpm.f90:57.  corr: complex[n_timestep+1].
int orc_tbpm_dos(const double* bes, int n_bes, const int32_t* indptr,
                 const int32_t* indices, const double* hop, int64_t n, const double* wf0_in,
                 int seed, int n_timestep, int n_samples, int rank, int chk_step,
                 double chk_thr, int state_kind, double* corr_out) {
  if (n_bes < 3 || n < 1 || n_timestep < 1 || n_samples < 1) return ORC_ERR_ARG;
  Csr h{indptr, indices, reinterpret_cast<const zc*>(hop), n};
  zc* corr = reinterpret_cast<zc*>(corr_out);
  for (int t = 0; t <= n_timestep; ++t) corr[t] = zmk(0, 0);
  std::vector<zc> wf0(n), wft(n), tmp(n), t0(n), t1(n);
  for (int s = 1; s <= n_samples; ++s) {
    if (wf0_in)
      std::memcpy(wf0.data(), wf0_in + 2 * (int64_t)(s - 1) * n, sizeof(zc) * n);
    else
      random_state(wf0.data(), n, (int64_t)seed * (s + rank * n_samples), state_kind);
    zc cv = inner_prod(wf0.data(), wf0.data(), n);
    corr[0] = zadd(corr[0], zdivd(cv, n_samples));
    cheb_wf_timestep(h, bes, n_bes, wf0.data(), true, wft.data(), t0, t1);
    cv = inner_prod(wf0.data(), wft.data(), n);
    corr[1] = zadd(corr[1], zdivd(cv, n_samples));
    const zc norm_ref = inner_prod(wft.data(), wft.data(), n);
    for (int t = 2; t <= n_timestep; ++t) {
      if (t == chk_step && norm_broken(wft.data(), n, norm_ref, chk_thr)) return ORC_ERR_NORM;
      cheb_wf_timestep(h, bes, n_bes, wft.data(), true, tmp.data(), t0, t1);
      wft.swap(tmp);
      cv = inner_prod(wf0.data(), wft.data(), n);
      corr[t] = zadd(corr[t], zdivd(cv, n_samples));
    }
  }
  return ORC_OK;
}

// tbpm.f90:193-351 (tbpm_accond).  corr: complex (4, n_timestep) F-order.
int orc_tbpm_accond(const double* bes, int n_bes, double beta, double mu,
                    const int32_t* indptr, const int32_t* indices, const double* hop,
                    int64_t n, int64_t nnz, double h_rescale, const double* dx,
                    const double* dy, const double* wf0_in, int seed, int n_timestep,
                    int n_samples, int nr_fermi, double fermi_precision, int rank,
                    int chk_step, double chk_thr, int state_kind, double* corr_out) {
  if (n_bes < 3 || n < 1 || n_timestep < 1 || n_samples < 1) return ORC_ERR_ARG;
  zc* corr = reinterpret_cast<zc*>(corr_out);
  for (int64_t i = 0; i < 4 * (int64_t)n_timestep; ++i) corr[i] = zmk(0, 0);
  const zc* hz = reinterpret_cast<const zc*>(hop);
  std::vector<zc> curx, cury;
  current_coefficient(hz, dx, nnz, h_rescale, curx);
  current_coefficient(hz, dy, nnz, h_rescale, cury);
  Csr cx{indptr, indices, curx.data(), n}, cy{indptr, indices, cury.data(), n};
  Csr h{indptr, indices, hz, n};
  std::vector<double> coef_f(nr_fermi + 1), coef_omf(nr_fermi + 1);
  const int n_f = orc_fermi_cheb_coef(coef_f.data(), nr_fermi, beta, mu, 0, fermi_precision);
  const int n_omf =
      orc_fermi_cheb_coef(coef_omf.data(), nr_fermi, beta, mu, 1, fermi_precision);
  if (n_f < 3 || n_omf < 3) return ORC_ERR_ARG;
  std::vector<zc> wf0(n), wf1(n), px(n), py(n), p2(n), tmp(n), t0(n), t1(n);
  for (int s = 1; s <= n_samples; ++s) {
    if (wf0_in)
      std::memcpy(wf0.data(), wf0_in + 2 * (int64_t)(s - 1) * n, sizeof(zc) * n);
    else
      random_state(wf0.data(), n, (int64_t)seed * (s + rank * n_samples), state_kind);
    csr_mv(cx, wf0.data(), tmp.data());
    fermi_op(h, coef_omf.data(), n_omf, tmp.data(), px.data(), t0, t1);
    csr_mv(cy, wf0.data(), tmp.data());
    fermi_op(h, coef_omf.data(), n_omf, tmp.data(), py.data(), t0, t1);
    fermi_op(h, coef_f.data(), n_f, wf0.data(), p2.data(), t0, t1);
    // t = 1 correlations are evaluated but not accumulated (tbpm.f90:284-302)
    const zc norm_ref = inner_prod(p2.data(), p2.data(), n);
    for (int t = 2; t <= n_timestep; ++t) {
      if (t == chk_step && norm_broken(p2.data(), n, norm_ref, chk_thr)) return ORC_ERR_NORM;
      cheb_wf_timestep(h, bes, n_bes, px.data(), true, tmp.data(), t0, t1);
      px.swap(tmp);
      cheb_wf_timestep(h, bes, n_bes, py.data(), true, tmp.data(), t0, t1);
      py.swap(tmp);
      cheb_wf_timestep(h, bes, n_bes, p2.data(), true, tmp.data(), t0, t1);
      p2.swap(tmp);
      zc cv[4];
      csr_mv(cx, px.data(), wf1.data());
      cv[0] = inner_prod(p2.data(), wf1.data(), n);
      csr_mv(cy, px.data(), wf1.data());
      cv[1] = inner_prod(p2.data(), wf1.data(), n);
      csr_mv(cx, py.data(), wf1.data());
      cv[2] = inner_prod(p2.data(), wf1.data(), n);
      csr_mv(cy, py.data(), wf1.data());
      cv[3] = inner_prod(p2.data(), wf1.data(), n);
      for (int k = 0; k < 4; ++k)
        corr[k + 4 * (int64_t)(t - 1)] =
            zadd(corr[k + 4 * (int64_t)(t - 1)], zdivd(cv[k], n_samples));
    }
  }
  return ORC_OK;
}

// tbpm.f90:497-718 (tbpm_dccond).  dos_corr: complex[n_timestep];
// dc_corr: complex (2, n_energies, n_timestep) F-order, first n_en_inds of the
// energy axis filled.
int orc_tbpm_dccond(const double* bes, int n_bes, const int32_t* indptr,
                    const int32_t* indices, const double* hop, int64_t n, int64_t nnz,
                    double h_rescale, const double* dx, const double* dy,
                    const double* wf0_in, int seed, int n_timestep, int n_samples,
                    double t_step, const double* energies, int n_energies,
                    const int32_t* en_inds, int n_en_inds, int rank, int chk_step,
                    double chk_thr, int state_kind, double* dos_out, double* dc_out) {
  if (n_bes < 3 || n < 1 || n_timestep < 1 || n_samples < 1 || n_en_inds < 0 ||
      n_en_inds > n_energies)
    return ORC_ERR_ARG;
  zc* dos = reinterpret_cast<zc*>(dos_out);
  zc* dc = reinterpret_cast<zc*>(dc_out);
  for (int t = 0; t < n_timestep; ++t) dos[t] = zmk(0, 0);
  for (int64_t i = 0; i < 2 * (int64_t)n_energies * n_timestep; ++i) dc[i] = zmk(0, 0);
  const zc* hz = reinterpret_cast<const zc*>(hop);
  Csr h{indptr, indices, hz, n};
  std::vector<zc> curx, cury;
  current_coefficient(hz, dx, nnz, h_rescale, curx);
  current_coefficient(hz, dy, nnz, h_rescale, cury);
  Csr cx{indptr, indices, curx.data(), n}, cy{indptr, indices, cury.data(), n};
  std::vector<zc> wf0(n), wpos(n), wneg(n), wfe(n), tmp(n), t0(n), t1(n);
  std::vector<zc> qe((size_t)n * n_en_inds), w0j1(n), w0j2(n), wej1(n), wej2(n);
  auto dc_at = [&](int k, int i, int t) -> zc& {
    return dc[k + 2 * ((int64_t)i + (int64_t)n_energies * t)];
  };
  for (int s = 1; s <= n_samples; ++s) {
    if (wf0_in)
      std::memcpy(wf0.data(), wf0_in + 2 * (int64_t)(s - 1) * n, sizeof(zc) * n);
    else
      random_state(wf0.data(), n, (int64_t)seed * (s + rank * n_samples), state_kind);
    wpos = wf0;
    wneg = wf0;
    for (int i = 0; i < n_en_inds; ++i)
      std::memcpy(&qe[(size_t)i * n], wf0.data(), sizeof(zc) * n);
    const zc norm_ref = inner_prod(wf0.data(), wf0.data(), n);
    for (int t = 1; t <= n_timestep; ++t) {
      if (t == chk_step && (norm_broken(wpos.data(), n, norm_ref, chk_thr) ||
                            norm_broken(wneg.data(), n, norm_ref, chk_thr)))
        return ORC_ERR_NORM;
      cheb_wf_timestep(h, bes, n_bes, wpos.data(), true, tmp.data(), t0, t1);
      wpos.swap(tmp);
      cheb_wf_timestep(h, bes, n_bes, wneg.data(), false, tmp.data(), t0, t1);
      wneg.swap(tmp);
      const zc cv = inner_prod(wf0.data(), wpos.data(), n);
      dos[t - 1] = zadd(dos[t - 1], zdivd(cv, n_samples));
      const double W = 0.5 * (1 + std::cos(kPi * t / n_timestep));  // Hanning
#pragma omp parallel for schedule(static)
      for (int i = 0; i < n_en_inds; ++i) {
        const double x = energies[en_inds[i]] * (double)t * t_step;
        const zc P = zmk(std::cos(x), std::sin(x));
        const zc Pc = zconj(P);
        zc* q = &qe[(size_t)i * n];
        for (int64_t j = 0; j < n; ++j) {
          q[j] = zadd(q[j], dmul(W, zmul(P, wpos[j])));
          q[j] = zadd(q[j], dmul(W, zmul(Pc, wneg[j])));
        }
      }
    }
    for (int i = 0; i < n_en_inds; ++i) {
      zc* q = &qe[(size_t)i * n];
      const double qs = norm_z(q, n);
      for (int64_t j = 0; j < n; ++j) q[j] = zdivd(q[j], qs);
    }
    csr_mv(cx, wf0.data(), w0j1.data());
    csr_mv(cy, wf0.data(), w0j2.data());
    for (int t = 1; t <= n_timestep; ++t) {
      if (t >= 2) {
        cheb_wf_timestep(h, bes, n_bes, w0j1.data(), true, tmp.data(), t0, t1);
        w0j1.swap(tmp);
        cheb_wf_timestep(h, bes, n_bes, w0j2.data(), true, tmp.data(), t0, t1);
        w0j2.swap(tmp);
      }
      for (int i = 0; i < n_en_inds; ++i) {
        const zc* q = &qe[(size_t)i * n];
        const double a = zabs(inner_prod(wf0.data(), q, n));
        for (int64_t j = 0; j < n; ++j) wfe[j] = zdivd(q[j], a);
        csr_mv(cx, wfe.data(), wej1.data());
        csr_mv(cy, wfe.data(), wej2.data());
        const zc c1 = inner_prod(w0j1.data(), wej1.data(), n);
        const zc c2 = inner_prod(w0j2.data(), wej2.data(), n);
        dc_at(0, i, t - 1) = zadd(dc_at(0, i, t - 1), zdivd(c1, n_samples));
        dc_at(1, i, t - 1) = zadd(dc_at(1, i, t - 1), zdivd(c2, n_samples));
      }
    }
  }
  return ORC_OK;
}

// tbpm.f90:1029-1093 (tbpm_psi_t).  psi_t: complex (n, n_time_log) F-order.
int orc_tbpm_psi_t(const double* bes, int n_bes, const int32_t* indptr,
                   const int32_t* indices, const double* hop, int64_t n, const double* psi0,
                   const int32_t* time_log, int n_time_log, int n_timestep, int chk_step,
                   double chk_thr, double* psi_t_out) {
  if (n_bes < 3 || n < 1 || n_time_log < 1) return ORC_ERR_ARG;
  Csr h{indptr, indices, reinterpret_cast<const zc*>(hop), n};
  zc* out = reinterpret_cast<zc*>(psi_t_out);
  std::vector<zc> wft(n), tmp(n), t0(n), t1(n);
  std::memcpy(wft.data(), psi0, sizeof(zc) * n);
  const zc norm_ref = inner_prod(wft.data(), wft.data(), n);
  int ptr = 1;
  for (int t = 1; t <= n_timestep; ++t) {
    if (time_log[ptr - 1] == t - 1) {
      std::memcpy(out + (size_t)(ptr - 1) * n, wft.data(), sizeof(zc) * n);
      if (ptr < n_time_log) ++ptr;
    }
    if (t == chk_step && norm_broken(wft.data(), n, norm_ref, chk_thr)) return ORC_ERR_NORM;
    cheb_wf_timestep(h, bes, n_bes, wft.data(), true, tmp.data(), t0, t1);
    wft.swap(tmp);
  }
  if (time_log[ptr - 1] == n_timestep)
    std::memcpy(out + (size_t)(ptr - 1) * n, wft.data(), sizeof(zc) * n);
  return ORC_OK;
}

// funcs.f90:125-149 (density_coef): exp(+-i q.r) per orbital
static void density_coef(int64_t n, const double* x, const double* y, const double* z,
                         const double* q, zc* dq, zc* dmq) {
  for (int64_t i = 0; i < n; ++i) {
    const double p = q[0] * x[i] + q[1] * y[i] + q[2] * z[i];
    dq[i] = zmk(std::cos(p), std::sin(p));
    dmq[i] = zmk(std::cos(p), -std::sin(p));
  }
}

// tbpm.f90:355-493 (tbpm_dyn_pol).  q_points: C order [n_q][3].
// corr: real (n_q, n_timestep) F-order.
int orc_tbpm_dyn_pol(const double* bes, int n_bes, double beta, double mu,
                     const int32_t* indptr, const int32_t* indices, const double* hop,
                     int64_t n, const double* site_x, const double* site_y,
                     const double* site_z, const double* q_points, int n_q,
                     const double* wf0_in, int seed, int n_timestep, int n_samples,
                     int nr_fermi, double fermi_precision, int rank, int chk_step,
                     double chk_thr, int state_kind, double* corr) {
  if (n_bes < 3 || n < 1 || n_timestep < 1 || n_samples < 1 || n_q < 1) return ORC_ERR_ARG;
  for (int64_t i = 0; i < (int64_t)n_q * n_timestep; ++i) corr[i] = 0.0;
  Csr h{indptr, indices, reinterpret_cast<const zc*>(hop), n};
  std::vector<double> coef_f(nr_fermi + 1), coef_omf(nr_fermi + 1);
  const int n_f = orc_fermi_cheb_coef(coef_f.data(), nr_fermi, beta, mu, 0, fermi_precision);
  const int n_omf =
      orc_fermi_cheb_coef(coef_omf.data(), nr_fermi, beta, mu, 1, fermi_precision);
  if (n_f < 3 || n_omf < 3) return ORC_ERR_ARG;
  std::vector<zc> dq(n), dmq(n), wf0(n), wf1(n), psi1(n), psi2(n), tmp(n), t0(n), t1(n);
  for (int iq = 0; iq < n_q; ++iq) {
    density_coef(n, site_x, site_y, site_z, q_points + 3 * iq, dq.data(), dmq.data());
    for (int s = 1; s <= n_samples; ++s) {
      if (wf0_in)
        std::memcpy(wf0.data(), wf0_in + 2 * (int64_t)(s - 1) * n, sizeof(zc) * n);
      else
        random_state(wf0.data(), n, (int64_t)seed * (s + rank * n_samples), state_kind);
      for (int64_t i = 0; i < n; ++i) tmp[i] = zmul(dmq[i], wf0[i]);
      fermi_op(h, coef_omf.data(), n_omf, tmp.data(), psi1.data(), t0, t1);
      fermi_op(h, coef_f.data(), n_f, wf0.data(), psi2.data(), t0, t1);
      for (int64_t i = 0; i < n; ++i) wf1[i] = zmul(dq[i], psi1[i]);
      corr[iq] += inner_prod(psi2.data(), wf1.data(), n).im / n_samples;
      const zc norm_ref = inner_prod(psi2.data(), psi2.data(), n);
      for (int t = 2; t <= n_timestep; ++t) {
        if (t == chk_step && norm_broken(psi2.data(), n, norm_ref, chk_thr))
          return ORC_ERR_NORM;
        cheb_wf_timestep(h, bes, n_bes, psi1.data(), true, tmp.data(), t0, t1);
        psi1.swap(tmp);
        cheb_wf_timestep(h, bes, n_bes, psi2.data(), true, tmp.data(), t0, t1);
        psi2.swap(tmp);
        for (int64_t i = 0; i < n; ++i) wf1[i] = zmul(dq[i], psi1[i]);
        corr[iq + (int64_t)n_q * (t - 1)] += inner_prod(psi2.data(), wf1.data(), n).im / n_samples;
      }
    }
  }
  return ORC_OK;
}

// tbpm.f90:721-830 (tbpm_eigenstates).  wf_qe: real (n_energies, n) F-order.
int orc_tbpm_eigenstates(const double* bes, int n_bes, const int32_t* indptr,
                         const int32_t* indices, const double* hop, int64_t n,
                         const double* wf0_in, int seed, int n_timestep, int n_samples,
                         double t_step, const double* energies, int n_en, int rank,
                         int chk_step, double chk_thr, int state_kind, double* wf_qe) {
  if (n_bes < 3 || n < 1 || n_timestep < 1 || n_samples < 1 || n_en < 1) return ORC_ERR_ARG;
  for (int64_t i = 0; i < (int64_t)n_en * n; ++i) wf_qe[i] = 0.0;
  Csr h{indptr, indices, reinterpret_cast<const zc*>(hop), n};
  std::vector<zc> wf0(n), wp(n), wm(n), tmp(n), t0(n), t1(n), wfq((size_t)n * n_en);
  for (int s = 1; s <= n_samples; ++s) {
    if (wf0_in)
      std::memcpy(wf0.data(), wf0_in + 2 * (int64_t)(s - 1) * n, sizeof(zc) * n);
    else
      random_state(wf0.data(), n, (int64_t)seed * (s + rank * n_samples), state_kind);
    wp = wf0;
    wm = wf0;
    for (int i = 0; i < n_en; ++i)
      std::memcpy(wfq.data() + (size_t)i * n, wf0.data(), sizeof(zc) * n);
    const zc norm_ref = inner_prod(wf0.data(), wf0.data(), n);
    for (int k = 1; k <= n_timestep; ++k) {
      if (k == chk_step && (norm_broken(wp.data(), n, norm_ref, chk_thr) ||
                            norm_broken(wm.data(), n, norm_ref, chk_thr)))
        return ORC_ERR_NORM;
      cheb_wf_timestep(h, bes, n_bes, wp.data(), true, tmp.data(), t0, t1);
      wp.swap(tmp);
      cheb_wf_timestep(h, bes, n_bes, wm.data(), false, tmp.data(), t0, t1);
      wm.swap(tmp);
      const double W = 0.5 * (1 + std::cos(kPi * k / n_timestep));  // Hanning window
      for (int i = 0; i < n_en; ++i) {
        const double ph = energies[i] * k * t_step;
        const zc P = zmk(std::cos(ph), std::sin(ph));
        zc* q = wfq.data() + (size_t)i * n;
        for (int64_t j = 0; j < n; ++j) {
          q[j] = zadd(q[j], dmul(W, zmul(P, wp[j])));
          q[j] = zadd(q[j], dmul(W, zmul(zconj(P), wm[j])));
        }
      }
    }
    for (int i = 0; i < n_en; ++i) {
      zc* q = wfq.data() + (size_t)i * n;
      const double qs = norm_z(q, n);
      for (int64_t j = 0; j < n; ++j) q[j] = zdivd(q[j], qs);
      for (int64_t j = 0; j < n; ++j) {
        const double a = zabs(q[j]);
        wf_qe[i + (int64_t)n_en * j] += a * a / n_samples;
      }
    }
  }
  return ORC_OK;
}

// tbpm.f90:836-960 (tbpm_kbdc).  direction 1: J_x, 2: J_y on the ket side.
// mu: complex (n_kernel, n_kernel) F-order.
int orc_tbpm_kbdc(const int32_t* indptr, const int32_t* indices, const double* hop,
                  int64_t n, int64_t nnz, double h_rescale, const double* dx, const double* dy,
                  const double* wf0_in, int seed, int n_samples, int n_kernel, int direction,
                  int rank, int state_kind, double* mu_out) {
  if (n < 1 || n_samples < 1 || n_kernel < 2 || (direction != 1 && direction != 2))
    return ORC_ERR_ARG;
  const zc* hz = reinterpret_cast<const zc*>(hop);
  zc* mu = reinterpret_cast<zc*>(mu_out);
  for (int64_t i = 0; i < (int64_t)n_kernel * n_kernel; ++i) mu[i] = zmk(0, 0);
  std::vector<zc> curx, cury;
  current_coefficient(hz, dx, nnz, h_rescale, curx);
  if (direction == 2) current_coefficient(hz, dy, nnz, h_rescale, cury);
  Csr h{indptr, indices, hz, n}, cx{indptr, indices, curx.data(), n};
  Csr cy{indptr, indices, direction == 2 ? cury.data() : curx.data(), n};
  std::vector<double> g(n_kernel);
  jackson_kernel(g.data(), n_kernel);
  std::vector<zc> win(n), w0(n), w1(n), w2(n), dk((size_t)n * n_kernel);
  std::vector<zc> cmu((size_t)n_kernel * n_kernel);
  auto col = [&](int j) { return dk.data() + (size_t)j * n; };
  for (int s = 1; s <= n_samples; ++s) {
    if (wf0_in)
      std::memcpy(win.data(), wf0_in + 2 * (int64_t)(s - 1) * n, sizeof(zc) * n);
    else
      random_state(win.data(), n, (int64_t)seed * (s + rank * n_samples), state_kind);
    std::memcpy(col(0), win.data(), sizeof(zc) * n);
    csr_mv(h, col(0), col(1));
    for (int j = 2; j < n_kernel; ++j) {
      csr_mv(h, col(j - 1), col(j));
      zc* y = col(j);
      const zc* x = col(j - 2);
      for (int64_t i = 0; i < n; ++i) y[i] = zadd(dmul(-1.0, x[i]), dmul(2.0, y[i]));
    }
    const Csr& cj = direction == 1 ? cx : cy;
    for (int j = 0; j < n_kernel; ++j) {
      std::memcpy(w0.data(), col(j), sizeof(zc) * n);
      csr_mv(cj, w0.data(), col(j));
    }
    csr_mv(cx, win.data(), w0.data());
    for (int j = 0; j < n_kernel; ++j) cmu[(size_t)j * n_kernel] = inner_prod(w0.data(), col(j), n);
    csr_mv(h, w0.data(), w1.data());
    for (int j = 0; j < n_kernel; ++j)
      cmu[1 + (size_t)j * n_kernel] = inner_prod(w1.data(), col(j), n);
    zc* p0 = w0.data();
    zc* p1 = w1.data();
    for (int i = 2; i < n_kernel; ++i) {
      zc* p2 = p0;
      amxpby_d(2.0, h, p1, -1.0, p0);  // p2 = 2 H p1 - p0, in place of p0
      for (int j = 0; j < n_kernel; ++j)
        cmu[i + (size_t)j * n_kernel] = inner_prod(p2, col(j), n);
      p0 = p1;
      p1 = p2;
    }
    for (int j = 0; j < n_kernel; ++j)
      for (int i = 0; i < n_kernel; ++i) {
        const size_t o = i + (size_t)j * n_kernel;
        mu[o] = zadd(mu[o], zdivd(dmul(g[i] * g[j], cmu[o]), n_samples));
      }
  }
  return ORC_OK;
}

// propagation.f90:85-155 (Haydock_coef) for one start vector n1 (overwritten).
static void haydock_coef(const Csr& h, double h_rescale, zc* n1, int n_depth, zc* coefa,
                         double* coefb) {
  const int64_t n = h.n;
  std::vector<zc> n2(n), nbuf(n);
  amv_d(h_rescale, h, n1, nbuf.data());
  coefa[0] = inner_prod(n1, nbuf.data(), n);
  for (int64_t i = 0; i < n; ++i) nbuf[i] = zadd(zmul(zmk(-coefa[0].re, -coefa[0].im), n1[i]), nbuf[i]);
  coefb[0] = norm_z(nbuf.data(), n);
  for (int64_t i = 0; i < n; ++i) n2[i] = zdivd(nbuf[i], coefb[0]);
  zc* p1 = n1;
  zc* p2 = n2.data();
  zc* pb = nbuf.data();
  for (int d = 1; d < n_depth; ++d) {
    amv_d(h_rescale, h, p2, pb);
    coefa[d] = inner_prod(p2, pb, n);
    const zc a = zmk(-coefa[d].re, -coefa[d].im);
    const double b = -coefb[d - 1];
    for (int64_t i = 0; i < n; ++i) pb[i] = zadd(zadd(zmul(a, p2[i]), dmul(b, p1[i])), pb[i]);
    coefb[d] = norm_z(pb, n);
    for (int64_t i = 0; i < n; ++i) pb[i] = zdivd(pb[i], coefb[d]);
    zc* sw = p1;
    p1 = p2;
    p2 = pb;
    pb = sw;
  }
}

// tbpm.f90:963-1026 (ldos_haydock): sample-averaged Haydock coefficients.
// wf_sites (optional, complex [n_samples][n_sites]) replaces the random site
// amplitudes.  coefa: complex[n_depth], coefb: real[n_depth].
int orc_haydock_coef(const int32_t* site_indices, int n_sites, const int32_t* indptr,
                     const int32_t* indices, const double* hop, int64_t n, double h_rescale,
                     const double* wf_sites, int seed, int n_depth, int n_samples,
                     int state_kind, double* coefa_out, double* coefb) {
  if (n < 1 || n_sites < 1 || n_depth < 1 || n_samples < 1) return ORC_ERR_ARG;
  Csr h{indptr, indices, reinterpret_cast<const zc*>(hop), n};
  zc* ca = reinterpret_cast<zc*>(coefa_out);
  for (int d = 0; d < n_depth; ++d) {
    ca[d] = zmk(0, 0);
    coefb[d] = 0.0;
  }
  std::vector<zc> tmp(n_sites), wf0(n), a(n_depth);
  std::vector<double> b(n_depth);
  for (int s = 1; s <= n_samples; ++s) {
    if (wf_sites)
      std::memcpy(tmp.data(), wf_sites + 2 * (int64_t)(s - 1) * n_sites, sizeof(zc) * n_sites);
    else
      random_state(tmp.data(), n_sites, (int64_t)seed * s, state_kind);
    std::fill(wf0.begin(), wf0.end(), zmk(0, 0));
    for (int i = 0; i < n_sites; ++i) {
      if (site_indices[i] < 0 || site_indices[i] >= n) return ORC_ERR_ARG;
      wf0[site_indices[i]] = tmp[i];
    }
    haydock_coef(h, h_rescale, wf0.data(), n_depth, a.data(), b.data());
    for (int d = 0; d < n_depth; ++d) {
      ca[d] = zadd(ca[d], zdivd(a[d], n_samples));
      coefb[d] += b[d] / n_samples;
    }
  }
  return ORC_OK;
}

// analysis.f90:6-69 (cond_from_trace) with kpm.f90:31-56 (get_gamma_mn) and
// funcs.f90:36-57 (Fermi_dist).  mu_mn: complex (n_kernel, n_kernel) F-order.
int orc_cond_from_trace(const double* mu_mn_in, int n_kernel, const double* mu, int n_mu,
                        double h_rescale, double beta, int ne_integral, double* cond) {
  if (n_kernel < 1 || ne_integral < 2) return ORC_ERR_ARG;
  const zc* mu_mn = reinterpret_cast<const zc*>(mu_mn_in);
  const double dE = kPi / ne_integral;
  const int ne = ne_integral - 1;
  std::vector<double> energy(ne), sum_gamma_mu(ne);
  for (int k = 1; k <= ne; ++k) {
    energy[k - 1] = k * dE;
    const double x = energy[k - 1];
    const double sx = std::sin(x), cx = std::cos(x);
    double sum = 0.0;
#pragma omp parallel for reduction(+ : sum) schedule(static)
    for (int j = 0; j < n_kernel; ++j) {
      for (int i = 0; i < n_kernel; ++i) {
        const zc a = zmul(dmul(std::cos(i * x), zmk(cx, -j * sx)),
                          zmk(std::cos(j * x), std::sin(j * x)));
        const zc b = zmul(dmul(std::cos(j * x), zmk(cx, i * sx)),
                          zmk(std::cos(i * x), -std::sin(i * x)));
        const zc g = zadd(a, b);
        sum += zmul(g, mu_mn[i + (size_t)n_kernel * j]).re;
      }
    }
    sum_gamma_mu[k - 1] = sum;
  }
  for (int i = 0; i < n_mu; ++i) {
    double dcx = 0.0;
    for (int k = 0; k < ne; ++k) {
      const double s = std::sin(energy[k]);
      const double div = s * s * s;
      const double en = std::cos(energy[k]) * h_rescale;
      const double fd = fermi_dist(beta, mu[i], en);
      dcx += sum_gamma_mu[k] * fd * dE / div;
    }
    cond[i] = dcx;
  }
  return ORC_OK;
}

}  // extern "C"
