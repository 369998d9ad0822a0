// Windowed trigonometric sums of the TBPM Analyzer on the device.
//
// The Analyzer's transforms of correlation functions (tbplas/tbpm/analysis.py)
// are sums over the time index k of window-weighted correlation values times
// cos / sin of (frequency or energy) x time:
//   * calc_ac_cond (analysis.py:161-243):   sum_k 2 w_k sin(omega_i k dt) Im c_ab(k),
//     for tnr frequencies: tnr^2 terms per component;
//   * calc_dyn_pol (analysis.py:245-308):   sum_k w_k c_q(k) (cos + i sin)(omega_i k dt),
//     n_q x tnr^2 terms;
//   * calc_dc_cond (analysis.py:375-458):   sum_k w_k Re(exp(-i E_i k dt) c_a(E_i, k)),
//     each energy with its own correlation row;
//   * calc_diff_coeff (analysis.py:460-511): the cumulative trapezoid over time of
//     the same terms.
// tbpm_trig_sums computes the first three, one warp per output with a fixed
// shuffle-reduction order (deterministic), and tbpm_trig_cumtrapz the fourth,
// one thread per row in the order of scipy's cumulative_trapezoid (the sum of
// (d_m (y_m + y_{m+1})) / 2 over m).  Phases are formed as the host does:
// (x_i * k) * dt, or x_i * (k * dt) for phase_kdt = 1.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <vector>

#include "tbpm_b200.h"
#include "tbpm_engine.cuh"

namespace {

__device__ __forceinline__ double trig_phase(double x, int k, double dt, int phase_kdt) {
  return phase_kdt ? x * ((double)k * dt) : (x * (double)k) * dt;
}

// out_c[o] = sum_k w_k a[q][k] cos(phase), out_s[o] = sum_k w_k b[q][k] sin(phase)
// for output o = r * n_x + i; q = r (shared rows) or q = o (a row per output).
__global__ void trig_sums_kernel(const double* __restrict__ w, int n_k,
                                 const double* __restrict__ a, const double* __restrict__ b,
                                 int n_rows, const double* __restrict__ x, int n_x, double dt,
                                 int per_output, int phase_kdt, double* out_c, double* out_s) {
  const int lane = threadIdx.x & 31;
  const int64_t n_out = (int64_t)n_rows * n_x;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x / 32);
  for (int64_t o = (int64_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5); o < n_out;
       o += warps) {
    const int r = (int)(o / n_x);
    const int i = (int)(o - (int64_t)r * n_x);
    const int64_t q = per_output ? o : (int64_t)r;
    const double* ar = a ? a + q * n_k : nullptr;
    const double* br = b ? b + q * n_k : nullptr;
    const double xi = x[i];
    double sc = 0.0, ss = 0.0;
    for (int k = lane; k < n_k; k += 32) {
      double sn, cs;
      sincos(trig_phase(xi, k, dt, phase_kdt), &sn, &cs);
      if (ar) sc += w[k] * (ar[k] * cs);
      if (br) ss += w[k] * (br[k] * sn);
    }
#pragma unroll
    for (int m = 16; m > 0; m >>= 1) {
      sc += __shfl_xor_sync(0xffffffffu, sc, m);
      ss += __shfl_xor_sync(0xffffffffu, ss, m);
    }
    if (lane == 0) {
      if (out_c) out_c[o] = sc;
      if (out_s) out_s[o] = ss;
    }
  }
}

// out[q][0] = 0, out[q][j] = out[q][j-1] + (d_{j-1} (y_{j-1} + y_j)) / 2 with
// y_k = (a[q][k] cos(x_q k dt) + b[q][k] sin(x_q k dt)) * w_k
__global__ void trig_cumtrapz_kernel(const double* __restrict__ w, int n_k,
                                     const double* __restrict__ a, const double* __restrict__ b,
                                     int n_rows, const double* __restrict__ x, double dt,
                                     const double* __restrict__ d, double* out) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n_rows; q += gridDim.x * blockDim.x) {
    const double* aq = a + (int64_t)q * n_k;
    const double* bq = b + (int64_t)q * n_k;
    double* oq = out + (int64_t)q * n_k;
    auto term = [&](int k) {
      double sn, cs;
      sincos(trig_phase(x[q], k, dt, 0), &sn, &cs);
      // rounded as the host's (cos * re + sin * im) * w, without contraction
      return __dmul_rn(__dadd_rn(__dmul_rn(cs, aq[k]), __dmul_rn(sn, bq[k])), w[k]);
    };
    double acc = 0.0;
    oq[0] = 0.0;
    double y0 = term(0);
    for (int k = 1; k < n_k; ++k) {
      const double y1 = term(k);
      acc += (d[k - 1] * (y1 + y0)) / 2.0;
      oq[k] = acc;
      y0 = y1;
    }
  }
}

int fail(tbpm_ctx* c, int code, const char* msg) {
  c->err = msg;
  return code;
}

int fail_cuda(tbpm_ctx* c, cudaError_t e, const char* what) {
  (void)cudaGetLastError();
  char buf[256];
  std::snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
  c->err = buf;
  return TBPM_ERR_CUDA;
}

// Device copies of the host inputs, laid out one after another in c->anl
// (256-byte aligned parts); returns the device address of each.
struct Staged {
  std::vector<double*> dev;
};

int stage_inputs(tbpm_ctx* c, const std::vector<std::pair<const double*, size_t>>& in,
                 size_t out_doubles, Staged* st, double** out_dev) {
  auto al = [](size_t n) { return (n * sizeof(double) + 255) & ~(size_t)255; };
  size_t total = al(out_doubles);
  for (const auto& p : in) total += p.first ? al(p.second) : 0;
  try {
    c->anl.ensure(total);
  } catch (const tbpm::Error& e) {
    return fail(c, e.code, "device memory for the Analyzer sums");
  }
  char* q = c->anl.as<char>();
  for (const auto& p : in) {
    if (!p.first) {
      st->dev.push_back(nullptr);
      continue;
    }
    double* d = reinterpret_cast<double*>(q);
    const cudaError_t e = cudaMemcpyAsync(d, p.first, p.second * sizeof(double),
                                          cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return fail_cuda(c, e, "Analyzer input upload");
    st->dev.push_back(d);
    q += al(p.second);
  }
  *out_dev = reinterpret_cast<double*>(q);
  return TBPM_OK;
}

}  // namespace

extern "C" int tbpm_trig_sums(tbpm_ctx* c, const double* w, int n_k, const double* a,
                              const double* b, int n_rows, const double* x, int n_x, double dt,
                              int per_output, int phase_kdt, double* out_cos, double* out_sin) {
  if (!c) return TBPM_ERR_ARG;
  if (!w || !x || n_k < 1 || n_rows < 1 || n_x < 1)
    return fail(c, TBPM_ERR_ARG, "tbpm_trig_sums: empty or null input");
  if ((out_cos && !a) || (out_sin && !b) || (!out_cos && !out_sin))
    return fail(c, TBPM_ERR_ARG, "tbpm_trig_sums: each requested sum needs its coefficients");
  const size_t rows = per_output ? (size_t)n_rows * n_x : (size_t)n_rows;
  const size_t n_out = (size_t)n_rows * n_x;
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) return fail_cuda(c, e, "cudaSetDevice");
  Staged st;
  double* out_dev = nullptr;
  int rc = stage_inputs(c,
                        {{w, (size_t)n_k},
                         {out_cos ? a : nullptr, rows * n_k},
                         {out_sin ? b : nullptr, rows * n_k},
                         {x, (size_t)n_x}},
                        2 * n_out, &st, &out_dev);
  if (rc != TBPM_OK) return rc;
  const int threads = 256;
  const int64_t blocks = std::min<int64_t>(((int64_t)n_out + 7) / 8, 148 * 64);
  trig_sums_kernel<<<(int)blocks, threads, 0, c->stream>>>(
      st.dev[0], n_k, st.dev[1], st.dev[2], n_rows, st.dev[3], n_x, dt, per_output ? 1 : 0,
      phase_kdt ? 1 : 0, out_cos ? out_dev : nullptr, out_sin ? out_dev + n_out : nullptr);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail_cuda(c, e, "trig_sums_kernel launch");
  if (out_cos)
    e = cudaMemcpyAsync(out_cos, out_dev, n_out * sizeof(double), cudaMemcpyDeviceToHost,
                        c->stream);
  if (e == cudaSuccess && out_sin)
    e = cudaMemcpyAsync(out_sin, out_dev + n_out, n_out * sizeof(double),
                        cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return fail_cuda(c, e, "tbpm_trig_sums");
  c->launches = 1;
  c->err.clear();
  return TBPM_OK;
}

extern "C" int tbpm_trig_cumtrapz(tbpm_ctx* c, const double* w, int n_k, const double* a,
                                  const double* b, int n_rows, const double* x, double dt,
                                  const double* spacing, double* out) {
  if (!c) return TBPM_ERR_ARG;
  if (!w || !a || !b || !x || !out || n_k < 1 || n_rows < 1 || (n_k > 1 && !spacing))
    return fail(c, TBPM_ERR_ARG, "tbpm_trig_cumtrapz: empty or null input");
  const size_t n_out = (size_t)n_rows * n_k;
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) return fail_cuda(c, e, "cudaSetDevice");
  Staged st;
  double* out_dev = nullptr;
  int rc = stage_inputs(c,
                        {{w, (size_t)n_k},
                         {a, n_out},
                         {b, n_out},
                         {x, (size_t)n_rows},
                         {n_k > 1 ? spacing : nullptr, (size_t)std::max(n_k - 1, 1)}},
                        n_out, &st, &out_dev);
  if (rc != TBPM_OK) return rc;
  trig_cumtrapz_kernel<<<(n_rows + 127) / 128, 128, 0, c->stream>>>(
      st.dev[0], n_k, st.dev[1], st.dev[2], n_rows, st.dev[3], dt, st.dev[4], out_dev);
  e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(out, out_dev, n_out * sizeof(double), cudaMemcpyDeviceToHost,
                        c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return fail_cuda(c, e, "tbpm_trig_cumtrapz");
  c->launches = 1;
  c->err.clear();
  return TBPM_OK;
}
