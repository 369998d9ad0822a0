// tbpm_cheb_timestep_noalloc: one Chebyshev time step that allocates nothing.
//
// Who needs it: callers that must not call cudaMalloc themselves or have the
// library call it.  Examples are a host framework whose caching allocator
// already owns almost all of HBM (a stray cudaMalloc would fail or fragment
// its pool), and a latency-critical loop where allocation after start-up is
// forbidden.  Such callers hand in device buffers from their own allocator.
// The two Chebyshev work vectors this step needs live in a fixed
// file-scope device array instead of being allocated.
//
// Limits and rules (also stated in include/tbpm_b200.h):
//  * The work array holds kNoAllocScratchBytes = 16 MiB.  It is part of the
//    library image, so every GPU that loads the library keeps it until the
//    process exits.  Its first 256 bytes hold a status word; the rest fits
//    2 * n_rows * n_states complex128 values with n_rows * n_states <=
//    kNoAllocMaxValues = (16 MiB - 256) / 32 = 524,280; larger requests are
//    rejected with TBPM_ERR_ARG before any work is enqueued.
//  * The caller's arrays must be device (or managed) memory usable on the
//    context's device, wf and hop 16-byte aligned (the kernels move them in
//    16-byte loads) and indptr/indices 4-byte aligned; anything else is
//    rejected on the host with TBPM_ERR_ARG before any launch.
//  * The first call on a context resolves the device address of the array
//    (cudaGetSymbolAddress, with the context's device current) and keeps it
//    in the context; make that first call before any stream capture.  A
//    context created after a cudaDeviceReset resolves it afresh.
//  * Every call shares the one array, and it keeps the last call's contents.
//    Calls that overlap on the GPU (other host threads, other streams) race
//    on it: serialise them.  The status word at its start is cleared by each
//    call before use; the work vectors are always written before they are
//    read.
//  * The call is synchronous: it validates the CSR on the device, waits for
//    the verdict, enqueues the step on the context stream and waits for it.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <mutex>

#include "tbpm_b200.h"
#include "tbpm_engine.cuh"
#include "tbpm_kernels.cuh"

namespace {

constexpr size_t kNoAllocScratchBytes = (size_t)16 << 20;
constexpr size_t kStatusBytes = 256;  // status word area at the start of the array
// n_rows * n_states that the two complex128 work vectors may hold
constexpr long long kNoAllocMaxValues =
    (long long)((kNoAllocScratchBytes - kStatusBytes) / (2 * sizeof(double2)));
static_assert(kNoAllocMaxValues == 524280, "documented limit of the work array");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of g_noalloc_scratch for the context's device (which must be
// current), looked up on the context's first call and kept in it.  In host
// code the symbol name is only a host-side stand-in, never a device address.
cudaError_t scratch_address(tbpm_ctx* c, void** out) {
  std::lock_guard<std::mutex> lock(c->noalloc_mutex);
  if (!c->noalloc_scratch) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    c->noalloc_scratch = p;
  }
  *out = c->noalloc_scratch;
  return cudaSuccess;
}

// indptr[0] == 0, non-decreasing, indptr[n] == nnz
__global__ void noalloc_check_rows(const int32_t* indptr, int64_t n, int64_t nnz,
                                   unsigned int* status) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t a = indptr[i], b = indptr[i + 1];
    if (b < a || (i == 0 && a != 0) || (i == n - 1 && (int64_t)b != nnz)) atomicOr(status, 1u);
  }
}

// 0 <= indices[j] < n (only launched after the row check passed, so every j
// is inside [0, nnz))
__global__ void noalloc_check_cols(const int32_t* indices, int64_t n, int64_t nnz,
                                   unsigned int* status) {
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < nnz;
       j += (int64_t)gridDim.x * blockDim.x) {
    const int32_t c = indices[j];
    if (c < 0 || (int64_t)c >= n) atomicOr(status, 2u);
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

// A caller's array: `align`-byte aligned, and device or managed memory that the
// context's device can read (a host pointer, or another GPU's buffer, would
// fault inside the kernels).  Queries only; nothing is allocated.
int check_array(tbpm_ctx* c, const void* p, size_t align, const char* name) {
  char buf[200];
  if (reinterpret_cast<uintptr_t>(p) % align != 0) {
    std::snprintf(buf, sizeof buf, "%s must be %zu-byte aligned", name, align);
    return fail(c, TBPM_ERR_ARG, buf);
  }
  cudaPointerAttributes at{};
  const cudaError_t e = cudaPointerGetAttributes(&at, p);
  if (e != cudaSuccess) (void)cudaGetLastError();
  const bool ok = e == cudaSuccess && (at.type == cudaMemoryTypeManaged ||
                                       (at.type == cudaMemoryTypeDevice && at.device == c->device));
  if (!ok) {
    std::snprintf(buf, sizeof buf,
                  "%s must be device (or managed) memory of the context's device %d", name,
                  c->device);
    return fail(c, TBPM_ERR_ARG, buf);
  }
  return TBPM_OK;
}

}  // namespace

extern "C" int tbpm_cheb_timestep_noalloc(tbpm_ctx* c, const double* bes, int n_bes,
                                          const int32_t* indptr, const int32_t* indices,
                                          const double* hop, int64_t n_rows, int64_t nnz,
                                          double* wf, int n_states, int forward) {
  using namespace tbpm;
  if (!c) return TBPM_ERR_ARG;
  if (!bes || n_bes < 3) return fail(c, TBPM_ERR_ARG, "at least 3 Bessel coefficients required");
  if (!indptr || !wf || (nnz > 0 && (!indices || !hop)))
    return fail(c, TBPM_ERR_ARG, "null array argument");
  if (n_rows < 1 || nnz < 0 || n_rows > INT32_MAX || nnz > INT32_MAX)
    return fail(c, TBPM_ERR_ARG, "n_rows / nnz out of range");
  if (n_states < 1 || n_states > 64) return fail(c, TBPM_ERR_ARG, "n_states must be 1..64");
  const size_t vec_bytes = (size_t)n_rows * (size_t)n_states * sizeof(double2);
  if ((long long)n_rows * n_states > kNoAllocMaxValues) {
    char buf[200];
    std::snprintf(buf, sizeof buf,
                  "tbpm_cheb_timestep_noalloc: n_rows*n_states = %lld exceeds the %lld "
                  "complex128 values its fixed 16 MiB work array holds",
                  (long long)n_rows * n_states, kNoAllocMaxValues);
    return fail(c, TBPM_ERR_ARG, buf);
  }
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) return fail_cuda(c, e, "cudaSetDevice");
  int rc = check_array(c, wf, 16, "wf");
  if (rc == TBPM_OK) rc = check_array(c, indptr, 4, "indptr");
  if (rc == TBPM_OK && nnz > 0) rc = check_array(c, indices, 4, "indices");
  if (rc == TBPM_OK && nnz > 0) rc = check_array(c, hop, 16, "hop");
  if (rc != TBPM_OK) return rc;
  void* base = nullptr;
  e = scratch_address(c, &base);
  if (e != cudaSuccess) return fail_cuda(c, e, "cudaGetSymbolAddress(noalloc scratch)");
  unsigned int* status = reinterpret_cast<unsigned int*>(base);
  auto* X = reinterpret_cast<Pack<double, 1>*>(static_cast<unsigned char*>(base) + kStatusBytes);
  auto* Y = reinterpret_cast<Pack<double, 1>*>(reinterpret_cast<unsigned char*>(X) + vec_bytes);
  auto* A = reinterpret_cast<Pack<double, 1>*>(wf);
  cudaStream_t s = c->stream;

  // ---- validate the CSR on the device (kernels below never read out of it)
  e = cudaMemsetAsync(status, 0, sizeof(unsigned int), s);
  if (e != cudaSuccess) return fail_cuda(c, e, "cudaMemsetAsync(status)");
  noalloc_check_rows<<<256, 256, 0, s>>>(indptr, n_rows, nnz, status);
  unsigned int flag = 0;
  e = cudaMemcpyAsync(&flag, status, sizeof flag, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail_cuda(c, e, "CSR row check");
  if (flag) return fail(c, TBPM_ERR_ARG, "invalid indptr (must start at 0, not decrease, end at nnz)");
  if (nnz > 0) {
    noalloc_check_cols<<<256, 256, 0, s>>>(indices, n_rows, nnz, status);
    e = cudaMemcpyAsync(&flag, status, sizeof flag, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail_cuda(c, e, "CSR column check");
    if (flag) return fail(c, TBPM_ERR_ARG, "column index out of range");
  }

  // ---- one time step, the schedule of propagation.f90:33-48 with the
  // deferred three-term flush: p_1 -> X, p_2 -> Y, p_k over p_{k-2}
  const int tpr = n_states;
  const int rpp = std::max(1, 128 / tpr);
  const int threads = rpp * tpr;
  auto grid_for = [&](const void* kernel) {
    int per_sm = 0, sms = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0) !=
            cudaSuccess ||
        per_sm < 1)
      per_sm = 1;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device) !=
            cudaSuccess ||
        sms < 1)
      sms = 148;
    (void)cudaGetLastError();
    const int64_t tiles = (n_rows + rpp - 1) / rpp;
    return (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)per_sm * sms, tiles));
  };
  const int grid0 = grid_for(reinterpret_cast<const void*>(cheb_term_kernel<double, 1, 0>));
  const int grid1 = grid_for(reinterpret_cast<const void*>(cheb_term_kernel<double, 1, 1>));
  const double sgn = forward ? 1.0 : -1.0;
  auto w = [&](int k) { return k == 0 ? bes[0] : 2 * bes[k]; };
  int last_flush = -1;
  for (int k = 1; k < n_bes; ++k) {
    TermArgs<double, 1> a{};
    a.indptr = indptr;
    a.indices = indices;
    a.hop = reinterpret_cast<const double2*>(hop);
    a.diag = nullptr;  // diagonal entries stay in the CSR
    a.n_rows = n_rows;
    a.rows_per_tile = rpp;
    a.tpr = tpr;
    if (k == 1) {
      a.c.alpha_re = 0.0;
      a.c.alpha_im = -1.0 * sgn;
      a.c.beta = 0.0;
      a.gather = A;
      a.pin = nullptr;
      a.pout = X;
    } else {
      a.c.alpha_re = 0.0;
      a.c.alpha_im = -2.0 * sgn;
      a.c.beta = 1.0;
      a.gather = (k - 1) & 1 ? X : Y;
      a.pin = (k == 2) ? A : ((k & 1) ? X : Y);
      a.pout = (k < n_bes - 1) ? ((k & 1) ? X : Y) : nullptr;
      const int pending = k - last_flush;
      if (k == 2 || pending == 3 || k == n_bes - 1) {
        a.c.nflush = pending;
        a.c.acc_init = (k == 2) ? 1 : 0;
        for (int set = 0; set < 2; ++set) {
          a.c.w[set][0] = pending >= 3 ? w(k - 2) : 0.0;
          a.c.w[set][1] = pending >= 2 ? w(k - 1) : 0.0;
          a.c.w[set][2] = w(k);
        }
        a.acc = A;
        last_flush = k;
      }
    }
    if (a.c.nflush > 0)
      cheb_term_kernel<double, 1, 1><<<grid1, threads, 0, s>>>(a);
    else
      cheb_term_kernel<double, 1, 0><<<grid0, threads, 0, s>>>(a);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail_cuda(c, e, "cheb_term_kernel launch");
  }
  e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail_cuda(c, e, "time step");
  c->err.clear();
  return TBPM_OK;
}
