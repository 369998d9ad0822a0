// Host-side engine of libtbpm_b200: device buffers, launch plans, CUDA-graph
// replay and the drivers behind the C ABI (include/tbpm_b200.h).
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <cstdint>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "tbpm_b200.h"

namespace tbpm {

struct Error {
  int code;
  std::string msg;
};

void throw_cuda(cudaError_t e, const char* what);
#define TBPM_CK(call)                                   \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) ::tbpm::throw_cuda(e_, #call); \
  } while (0)

// A named NVTX range over a scope (a driver or one of its phases), so that a
// timeline profiler shows where each call spends its time. NVTX3 is header
// only: with no profiler attached each push/pop is a test of a null pointer.
struct Phase {
  explicit Phase(const char* name) { nvtxRangePushA(name); }
  ~Phase() { nvtxRangePop(); }
  Phase(const Phase&) = delete;
  Phase& operator=(const Phase&) = delete;
};

// Grow-only device allocation, in multiples of 256 bytes (the bulk copies of
// the ring kernels widen their windows to 16-byte boundaries and rely on it).
struct DevMem {
  void* p = nullptr;
  size_t bytes = 0;
  void ensure(size_t n);
  void release();
  template <typename T>
  T* as() const {
    return reinterpret_cast<T*>(p);
  }
  DevMem() = default;
  DevMem(const DevMem&) = delete;
  DevMem& operator=(const DevMem&) = delete;
  ~DevMem() { release(); }
};

// H = D + O: the diagonal D (on-site terms, dense complex[N]) and the
// off-diagonal part O in CSR (indptr/indices/hop and the matching dx/dy).
// nnz counts the entries of O.
struct Ham {
  int prec = -1;
  int64_t n = 0, nnz = 0;
  DevMem indptr, indices, hop, dx, dy, diag;
  bool has_dxy = false;
  bool has_diag = false;
  double rescale = 1.0;
  uint64_t gen = 0;  // advanced by every upload or device build of a Hamiltonian
};

// Chebyshev-type expansion  out = sum_k w_k p_k,
//   p_0 = psi, p_1 = alpha1 * H p_0, p_k = alpha * H p_{k-1} + beta * p_{k-2}.
struct Expansion {
  int n_terms = 0;
  double alpha1_re = 0, alpha1_im = 0;
  double alpha_re = 0, alpha_im = 0;
  double beta = 0;
  std::vector<double> w[2];
  unsigned long long neg_mask = 0, set_mask = 0;
};

Expansion time_step_expansion(const double* bes, int n_bes);
Expansion fermi_expansion(const double* coef_a, int n_a, const double* coef_b, int n_b,
                          unsigned long long set_b_mask);

struct Tile {
  int threads = 256;
  int rpp = 1;
  int64_t rows_per_tile = 1;
  int grid = 1;
};

struct GraphCache {
  cudaGraphExec_t exec = nullptr;
  std::vector<unsigned char> key;
  int steps = 0;
  int64_t l_step = 0;   // launches of one captured step
  double b_step = 0;    // modelled HBM bytes of one captured step
  void reset();
  ~GraphCache() { reset(); }
};

// Work plan of the paired-term kernel (tbpm_pair_kernels.cuh) for one tile
// height: each tile's dependency list, the item sequence and the flags.
// Built on the device for the current Hamiltonian (gen), rebuilt after the
// next upload.
struct PairPlan {
  int rows = 0;          // rows per tile
  int grid = 0;          // launch grid the sequence margin was set for
  uint64_t ham_gen = 0;  // Hamiltonian it was built for
  bool forced = false;   // built ignoring the L2 window test
  bool usable = false;   // every list fits kPairDeps (and the window test passed)
  int n_tiles = 0;
  DevMem seq, deps, flags, sync;
};

// Row windows of the ring kernels (ring_window_kernel) for one tile height on
// the current Hamiltonian (gen).
struct WindowPlan {
  int rows = 0;
  uint64_t ham_gen = 0;
  int n_tiles = 0;
  DevMem win, n_gather;
};

// A plan asked for while a graph was being captured (its build launches
// kernels outside the graph, and the pair plan synchronises); ensure_graph
// builds it and captures again.  kind 0: pair plan, 1: window plan (rows only).
struct PairRequest {
  int rows, grid, stages;
  size_t tile_bytes;
  bool force;
  int kind = 0;
};

struct Session {
  bool active = false;
  int kind = 0;  // 1 = DOS
  int ld = 0;
  int V = 1;
  int rows_cap = 0;
  int rows_enqueued = 0;
  Expansion ex;
};

}  // namespace tbpm

struct tbpm_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  tbpm_options opts{};
  std::string err;
  tbpm::Ham ham;
  tbpm::DevMem A, X, Y, wf0, partials, out, ctr, stage, small, qe, coef, seg;
  tbpm::DevMem raw;  // device copy of an uploaded host CSR, kept for the next upload
  tbpm::DevMem status;  // bit 0: a bounded device-side wait ran out (cleared when read)
  tbpm::DevMem anl;     // inputs and outputs of the Analyzer's trigonometric sums
  std::vector<std::unique_ptr<tbpm::PairPlan>> pairs;  // paired-term plans, by tile height
  std::vector<std::unique_ptr<tbpm::WindowPlan>> windows;  // ring window plans, by tile height
  std::vector<tbpm::PairRequest> pair_requests;
  tbpm::DevMem pair_tmp;  // scratch of the plan build
  int64_t launches = 0;
  double model_bytes = 0;
  tbpm::Session sess;
  tbpm::GraphCache graph;
  // device address of the allocation-free time step's fixed work array on this
  // context's device (tbpm_noalloc.cu), looked up on its first call
  void* noalloc_scratch = nullptr;
  std::mutex noalloc_mutex;
};
