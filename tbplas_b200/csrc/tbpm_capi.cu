// extern "C" entry points of libtbpm_b200.so (declared in include/tbpm_b200.h).
// Every entry point converts internal exceptions into a status code and keeps
// the message for tbpm_last_error(); nothing here exits the process.
#include <cuda_runtime.h>

#include <cstdio>
#include <new>

#include "tbpm_b200.h"
#include "tbpm_engine.cuh"

namespace tbpm {
void drv_ham_upload(tbpm_ctx* c, const int32_t* indptr, const int32_t* indices,
                    const double* hop, int64_t n, int64_t nnz, const double* dx,
                    const double* dy, double rescale);
void drv_dos(tbpm_ctx* c, const double* bes, int n_bes, const double* wf0, int n_states,
             int seed, int rank, int n_ran_samples, int n_timestep, int chk_step,
             double chk_thr, double* corr, double* corr_per_state);
void drv_ac(tbpm_ctx* c, const double* bes, int n_bes, double beta, double mu,
            const double* wf0, int n_states, int seed, int rank, int n_ran_samples,
            int n_timestep, int nr_fermi, double fermi_precision, int chk_step, double chk_thr,
            double* corr);
void drv_dc_part(tbpm_ctx* c, const double* bes, int n_bes, const double* wf0, int first_state,
                 int n_states, int n_avg, int seed, int rank, int n_ran_samples, int n_timestep,
                 double t_step, const double* energies, int n_energies, const int32_t* en_inds,
                 int n_en_inds, int chk_step, double chk_thr, double* dos_corr, double* dc_corr,
                 bool zero);
void drv_dc(tbpm_ctx* c, const double* bes, int n_bes, const double* wf0, int n_states,
            int seed, int rank, int n_ran_samples, int n_timestep, double t_step,
            const double* energies, int n_energies, const int32_t* en_inds, int n_en_inds,
            int chk_step, double chk_thr, double* dos_corr, double* dc_corr);
void drv_psi_t(tbpm_ctx* c, const double* bes, int n_bes, const double* psi0,
               const int32_t* time_log, int n_log, int n_timestep, int chk_step,
               double chk_thr, double* psi_t);
void drv_random_states(tbpm_ctx* c, int64_t n, int seed, int first_sample, int n_states,
                       int rank, int n_ran_samples, int kind, double* wf);
void drv_fermi_coef(int nr_fermi, double beta, double mu, int one_minus, double eps,
                    double* coef, int* n_cheb);
void drv_expansion_apply(tbpm_ctx* c, const Expansion& ex, double* wf, int n_states);
void drv_session_dos_begin(tbpm_ctx* c, const double* bes, int n_bes, int n_states, int seed,
                           int rank, int n_ran_samples, int n_timestep);
void drv_dos_segmented(tbpm_ctx* c, const double* bes, int n_bes, const int64_t* seg_off,
                       int n_seg, int n_states, int seed, int n_timestep, int chk_step,
                       double chk_thr, double* corr, double* corr_per_state);
void drv_session_advance(tbpm_ctx* c, int n_steps);
void drv_session_read(tbpm_ctx* c, double* corr, double* norms, int* n_done);
void drv_selftest_wait_timeout(tbpm_ctx* c);
void drv_session_dos_resume(tbpm_ctx* c, const double* bes, int n_bes, int n_states,
                            const double* wf0, const double* psi, const double* corr,
                            const double* norms, int n_done, int n_timestep);
void drv_session_export(tbpm_ctx* c, double* wf0, double* psi);
void drv_dyn_pol(tbpm_ctx* c, const double* bes, int n_bes, double beta, double mu,
                 const double* sx, const double* sy, const double* sz, const double* q_points,
                 int n_q, const double* wf0, int n_states, int seed, int rank,
                 int n_ran_samples, int n_timestep, int nr_fermi, double fermi_precision,
                 int chk_step, double chk_thr, double* corr);
void drv_eigenstates(tbpm_ctx* c, const double* bes, int n_bes, const double* wf0,
                     int n_states, int seed, int rank, int n_ran_samples, int n_timestep,
                     double t_step, const double* energies, int n_energies, int chk_step,
                     double chk_thr, double* wf_qe);
void drv_kbdc(tbpm_ctx* c, const double* wf0, int n_states, int seed, int rank,
              int n_ran_samples, int n_kernel, int direction, double* mu);
void drv_haydock(tbpm_ctx* c, const int32_t* sites, int n_sites, const double* wf_sites,
                 int n_samples, int n_depth, double h_rescale, double* coefa, double* coefb);
void drv_cond_from_trace(tbpm_ctx* c, const double* mu_mn, int nk, const double* mu, int n_mu,
                         double h_rescale, double beta, int ne_integral, double* cond);
void drv_supercell_ham(tbpm_ctx* c, const tbpm_supercell* sc, int layout, double cutoff,
                       int64_t* n_rows, int64_t* nnz, double* rescale);
void drv_supercell_csr(tbpm_ctx* c, const tbpm_supercell* sc, int layout, double cutoff,
                       int64_t* n_rows, int64_t* nnz, double* rescale, int64_t* indptr,
                       int32_t* indices, double* hop, double* dx, double* dy);
}  // namespace tbpm

namespace {

tbpm_options default_options() {
  tbpm_options o{};
  o.precision = TBPM_PREC_FP64;
  o.batch = 16;
  o.state_kind = TBPM_STATE_EXP;
  o.verbose = 0;
  o.threads_per_block = 0;
  o.rows_per_tile = 0;
  o.steps_per_graph = 16;
  o.use_graphs = 1;
  o.fp32_chk_thr = 1e-4;
  o.vector_width = 0;
  o.term_kernel = 0;
  o.dc_budget_gb = 0.0;
  return o;
}

template <class F>
int guarded(tbpm_ctx* c, F&& f) {
  if (!c) return TBPM_ERR_ARG;
  try {
    TBPM_CK(cudaSetDevice(c->device));
    f();
    c->err.clear();
    return TBPM_OK;
  } catch (const tbpm::Error& e) {
    c->err = e.msg;
    return e.code;
  } catch (const std::bad_alloc&) {
    c->err = "host allocation failed";
    return TBPM_ERR_OOM;
  } catch (...) {
    c->err = "unknown error";
    return TBPM_ERR_CUDA;
  }
}

// Host CSR arguments of the f2py-style drivers: upload when given.
void maybe_upload(tbpm_ctx* c, const int32_t* indptr, const int32_t* indices,
                  const double* hop, int64_t n_rows, int64_t nnz, const double* dx,
                  const double* dy, double rescale) {
  if (indptr) tbpm::drv_ham_upload(c, indptr, indices, hop, n_rows, nnz, dx, dy, rescale);
}

}  // namespace

extern "C" {

int tbpm_version(void) { return 1; }

int tbpm_create(int device, tbpm_ctx** out) {
  if (!out) return TBPM_ERR_ARG;
  *out = nullptr;
  int n_dev = 0;
  if (cudaGetDeviceCount(&n_dev) != cudaSuccess || n_dev < 1) {
    (void)cudaGetLastError();
    return TBPM_ERR_CUDA;
  }
  if (device < 0 || device >= n_dev) return TBPM_ERR_ARG;
  tbpm_ctx* c = new (std::nothrow) tbpm_ctx();
  if (!c) return TBPM_ERR_OOM;
  c->device = device;
  c->opts = default_options();
  if (cudaSetDevice(device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
    (void)cudaGetLastError();
    delete c;
    return TBPM_ERR_CUDA;
  }
  // status word of the kernels' bounded waits (zero = no wait ran out)
  try {
    c->status.ensure(256);
  } catch (...) {
    cudaStreamDestroy(c->stream);
    delete c;
    return TBPM_ERR_OOM;
  }
  if (cudaMemset(c->status.p, 0, 256) != cudaSuccess) {
    (void)cudaGetLastError();
    cudaStreamDestroy(c->stream);
    delete c;
    return TBPM_ERR_CUDA;
  }
  *out = c;
  return TBPM_OK;
}

int tbpm_destroy(tbpm_ctx* c) {
  if (!c) return TBPM_OK;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  c->graph.reset();
  c->ham.indptr.release();
  c->ham.indices.release();
  c->ham.hop.release();
  c->ham.dx.release();
  c->ham.dy.release();
  c->ham.diag.release();
  cudaStreamDestroy(c->stream);
  delete c;
  return TBPM_OK;
}

const char* tbpm_last_error(const tbpm_ctx* c) { return c ? c->err.c_str() : "null context"; }

int tbpm_set_options(tbpm_ctx* c, const tbpm_options* o) {
  if (!c || !o) return TBPM_ERR_ARG;
  if (o->precision != TBPM_PREC_FP64 && o->precision != TBPM_PREC_FP32) {
    c->err = "precision must be TBPM_PREC_FP64 or TBPM_PREC_FP32";
    return TBPM_ERR_ARG;
  }
  if (o->state_kind != TBPM_STATE_EXP && o->state_kind != TBPM_STATE_UNIT) {
    c->err = "unknown state_kind";
    return TBPM_ERR_ARG;
  }
  if (o->batch < 0 || o->threads_per_block < 0 || o->rows_per_tile < 0 ||
      o->steps_per_graph < 0 || !(o->fp32_chk_thr >= 0) || o->vector_width < 0 ||
      o->vector_width > 2 || o->term_kernel < 0 || o->term_kernel > 4 ||
      !(o->dc_budget_gb >= 0)) {
    c->err = "negative option";
    return TBPM_ERR_ARG;
  }
  c->opts = *o;
  c->graph.reset();
  return TBPM_OK;
}

int tbpm_get_options(const tbpm_ctx* c, tbpm_options* o) {
  if (!c || !o) return TBPM_ERR_ARG;
  *o = c->opts;
  return TBPM_OK;
}

void* tbpm_get_stream(const tbpm_ctx* c) { return c ? (void*)c->stream : nullptr; }

int tbpm_last_stats(const tbpm_ctx* c, int64_t* launches, double* model_bytes) {
  if (!c) return TBPM_ERR_ARG;
  if (launches) *launches = c->launches;
  if (model_bytes) *model_bytes = c->model_bytes;
  return TBPM_OK;
}

int tbpm_ham_upload(tbpm_ctx* c, const int32_t* indptr, const int32_t* indices,
                    const double* hop, int64_t n_rows, int64_t nnz, const double* dx,
                    const double* dy, double rescale) {
  return guarded(c, [&] {
    tbpm::drv_ham_upload(c, indptr, indices, hop, n_rows, nnz, dx, dy, rescale);
  });
}

int tbpm_supercell_ham(tbpm_ctx* c, const tbpm_supercell* sc, int layout,
                       double orb_eng_cutoff, int64_t* n_rows, int64_t* nnz,
                       double* rescale) {
  return guarded(c, [&] {
    tbpm::drv_supercell_ham(c, sc, layout, orb_eng_cutoff, n_rows, nnz, rescale);
  });
}

int tbpm_supercell_csr(tbpm_ctx* c, const tbpm_supercell* sc, int layout,
                       double orb_eng_cutoff, int64_t* n_rows, int64_t* nnz, double* rescale,
                       int64_t* indptr, int32_t* indices, double* hop, double* dx,
                       double* dy) {
  return guarded(c, [&] {
    tbpm::drv_supercell_csr(c, sc, layout, orb_eng_cutoff, n_rows, nnz, rescale, indptr,
                            indices, hop, dx, dy);
  });
}

int tbpm_dyn_pol(tbpm_ctx* c, const double* bes, int n_bes, double beta, double mu,
                 const int32_t* indptr, const int32_t* indices, const double* hop,
                 int64_t n_rows, int64_t nnz, double h_rescale, const double* dx,
                 const double* dy, const double* site_x, const double* site_y,
                 const double* site_z, int seed, int n_timestep, int n_ran_samples,
                 int nr_fermi, double fermi_precision, const double* q_points, int n_q_points,
                 int rank, int wfn_chk_step, double wfn_chk_thr, double* corr) {
  return guarded(c, [&] {
    maybe_upload(c, indptr, indices, hop, n_rows, nnz, dx, dy, h_rescale);
    tbpm::drv_dyn_pol(c, bes, n_bes, beta, mu, site_x, site_y, site_z, q_points, n_q_points,
                      nullptr, n_ran_samples, seed, rank, n_ran_samples, n_timestep, nr_fermi,
                      fermi_precision, wfn_chk_step, wfn_chk_thr, corr);
  });
}

int tbpm_dyn_pol_states(tbpm_ctx* c, const double* bes, int n_bes, double beta, double mu,
                        const int32_t* indptr, const int32_t* indices, const double* hop,
                        int64_t n_rows, int64_t nnz, const double* site_x,
                        const double* site_y, const double* site_z, const double* q_points,
                        int n_q_points, const double* wf0, int n_states, int n_timestep,
                        int nr_fermi, double fermi_precision, int wfn_chk_step,
                        double wfn_chk_thr, double* corr) {
  return guarded(c, [&] {
    if (!wf0) throw tbpm::Error{TBPM_ERR_ARG, "null initial states"};
    maybe_upload(c, indptr, indices, hop, n_rows, nnz, nullptr, nullptr, 1.0);
    tbpm::drv_dyn_pol(c, bes, n_bes, beta, mu, site_x, site_y, site_z, q_points, n_q_points,
                      wf0, n_states, 0, 0, n_states, n_timestep, nr_fermi, fermi_precision,
                      wfn_chk_step, wfn_chk_thr, corr);
  });
}

int tbpm_eigenstates(tbpm_ctx* c, const double* bes, int n_bes, const int32_t* indptr,
                     const int32_t* indices, const double* hop, int64_t n_rows, int64_t nnz,
                     int seed, int n_timestep, int n_ran_samples, double t_step,
                     const double* energies, int n_energies, int rank, int wfn_chk_step,
                     double wfn_chk_thr, double* wf_qe) {
  return guarded(c, [&] {
    maybe_upload(c, indptr, indices, hop, n_rows, nnz, nullptr, nullptr, 1.0);
    tbpm::drv_eigenstates(c, bes, n_bes, nullptr, n_ran_samples, seed, rank, n_ran_samples,
                          n_timestep, t_step, energies, n_energies, wfn_chk_step, wfn_chk_thr,
                          wf_qe);
  });
}

int tbpm_eigenstates_states(tbpm_ctx* c, const double* bes, int n_bes, const int32_t* indptr,
                            const int32_t* indices, const double* hop, int64_t n_rows,
                            int64_t nnz, const double* wf0, int n_states, int n_timestep,
                            double t_step, const double* energies, int n_energies,
                            int wfn_chk_step, double wfn_chk_thr, double* wf_qe) {
  return guarded(c, [&] {
    if (!wf0) throw tbpm::Error{TBPM_ERR_ARG, "null initial states"};
    maybe_upload(c, indptr, indices, hop, n_rows, nnz, nullptr, nullptr, 1.0);
    tbpm::drv_eigenstates(c, bes, n_bes, wf0, n_states, 0, 0, n_states, n_timestep, t_step,
                          energies, n_energies, wfn_chk_step, wfn_chk_thr, wf_qe);
  });
}

int tbpm_kbdc(tbpm_ctx* c, int seed, const int32_t* indptr, const int32_t* indices,
              const double* hop, int64_t n_rows, int64_t nnz, double h_rescale,
              const double* dx, const double* dy, int n_ran_samples, int n_kernel,
              int direction, int rank, double* mu) {
  return guarded(c, [&] {
    maybe_upload(c, indptr, indices, hop, n_rows, nnz, dx, dy, h_rescale);
    tbpm::drv_kbdc(c, nullptr, n_ran_samples, seed, rank, n_ran_samples, n_kernel, direction,
                   mu);
  });
}

int tbpm_kbdc_states(tbpm_ctx* c, const int32_t* indptr, const int32_t* indices,
                     const double* hop, int64_t n_rows, int64_t nnz, double h_rescale,
                     const double* dx, const double* dy, const double* wf0, int n_states,
                     int n_kernel, int direction, double* mu) {
  return guarded(c, [&] {
    if (!wf0) throw tbpm::Error{TBPM_ERR_ARG, "null initial states"};
    maybe_upload(c, indptr, indices, hop, n_rows, nnz, dx, dy, h_rescale);
    tbpm::drv_kbdc(c, wf0, n_states, 0, 0, n_states, n_kernel, direction, mu);
  });
}

int tbpm_haydock_coef(tbpm_ctx* c, const int32_t* indptr, const int32_t* indices,
                      const double* hop, int64_t n_rows, int64_t nnz, double h_rescale,
                      const int32_t* site_indices, int n_sites, const double* wf_sites,
                      int n_samples, int n_depth, double* coefa, double* coefb) {
  return guarded(c, [&] {
    maybe_upload(c, indptr, indices, hop, n_rows, nnz, nullptr, nullptr, h_rescale);
    tbpm::drv_haydock(c, site_indices, n_sites, wf_sites, n_samples, n_depth, h_rescale, coefa,
                      coefb);
  });
}

int tbpm_cond_from_trace(tbpm_ctx* c, const double* mu_mn, int n_kernel, const double* mu,
                         int n_mu, double h_rescale, double beta, int ne_integral,
                         double fermi_precision, int rank, double* cond) {
  (void)fermi_precision;  // unused by the reference too (its cut-off is commented out)
  (void)rank;
  return guarded(c, [&] {
    tbpm::drv_cond_from_trace(c, mu_mn, n_kernel, mu, n_mu, h_rescale, beta, ne_integral, cond);
  });
}

int tbpm_ham_release(tbpm_ctx* c) {
  return guarded(c, [&] {
    cudaStreamSynchronize(c->stream);
    c->graph.reset();
    c->sess.active = false;
    c->ham.indptr.release();
    c->ham.indices.release();
    c->ham.hop.release();
    c->ham.dx.release();
    c->ham.dy.release();
    c->ham.diag.release();
    c->raw.release();
    c->ham.has_diag = false;
    c->ham.n = 0;
    c->ham.nnz = 0;
    c->ham.has_dxy = false;
    c->ham.prec = -1;
    ++c->ham.gen;
  });
}

int tbpm_dos(tbpm_ctx* c, const double* bes, int n_bes, const int32_t* indptr,
             const int32_t* indices, const double* hop, int64_t n_rows, int64_t nnz, int seed,
             int n_timestep, int n_ran_samples, int rank, int wfn_chk_step, double wfn_chk_thr,
             double* corr) {
  return guarded(c, [&] {
    maybe_upload(c, indptr, indices, hop, n_rows, nnz, nullptr, nullptr, 1.0);
    tbpm::drv_dos(c, bes, n_bes, nullptr, n_ran_samples, seed, rank, n_ran_samples, n_timestep,
                  wfn_chk_step, wfn_chk_thr, corr, nullptr);
  });
}

int tbpm_dos_states(tbpm_ctx* c, const double* bes, int n_bes, const int32_t* indptr,
                    const int32_t* indices, const double* hop, int64_t n_rows, int64_t nnz,
                    const double* wf0, int n_states, int n_timestep, int wfn_chk_step,
                    double wfn_chk_thr, double* corr, double* corr_per_state) {
  return guarded(c, [&] {
    if (!wf0) throw tbpm::Error{TBPM_ERR_ARG, "wf0 is null"};
    maybe_upload(c, indptr, indices, hop, n_rows, nnz, nullptr, nullptr, 1.0);
    tbpm::drv_dos(c, bes, n_bes, wf0, n_states, 0, 0, n_states, n_timestep, wfn_chk_step,
                  wfn_chk_thr, corr, corr_per_state);
  });
}

int tbpm_accond(tbpm_ctx* c, const double* bes, int n_bes, double beta, double mu,
                const int32_t* indptr, const int32_t* indices, const double* hop,
                int64_t n_rows, int64_t nnz, double h_rescale, const double* dx,
                const double* dy, int seed, int n_timestep, int n_ran_samples, int nr_fermi,
                double fermi_precision, int rank, int wfn_chk_step, double wfn_chk_thr,
                double* corr) {
  return guarded(c, [&] {
    maybe_upload(c, indptr, indices, hop, n_rows, nnz, dx, dy, h_rescale);
    tbpm::drv_ac(c, bes, n_bes, beta, mu, nullptr, n_ran_samples, seed, rank, n_ran_samples,
                 n_timestep, nr_fermi, fermi_precision, wfn_chk_step, wfn_chk_thr, corr);
  });
}

int tbpm_accond_states(tbpm_ctx* c, const double* bes, int n_bes, double beta, double mu,
                       const int32_t* indptr, const int32_t* indices, const double* hop,
                       int64_t n_rows, int64_t nnz, double h_rescale, const double* dx,
                       const double* dy, const double* wf0, int n_states, int n_timestep,
                       int nr_fermi, double fermi_precision, int wfn_chk_step,
                       double wfn_chk_thr, double* corr) {
  return guarded(c, [&] {
    if (!wf0) throw tbpm::Error{TBPM_ERR_ARG, "wf0 is null"};
    maybe_upload(c, indptr, indices, hop, n_rows, nnz, dx, dy, h_rescale);
    tbpm::drv_ac(c, bes, n_bes, beta, mu, wf0, n_states, 0, 0, n_states, n_timestep, nr_fermi,
                 fermi_precision, wfn_chk_step, wfn_chk_thr, corr);
  });
}

int tbpm_dccond(tbpm_ctx* c, const double* bes, int n_bes, double beta, double mu,
                const int32_t* indptr, const int32_t* indices, const double* hop,
                int64_t n_rows, int64_t nnz, double h_rescale, const double* dx,
                const double* dy, int seed, int n_timestep, int n_ran_samples, double t_step,
                const double* energies, int n_energies, const int32_t* en_inds,
                int n_en_inds, int rank, int wfn_chk_step, double wfn_chk_thr,
                double* dos_corr, double* dc_corr) {
  (void)beta;
  (void)mu;  // passed but unused by the reference (tbpm.f90:497-718)
  return guarded(c, [&] {
    maybe_upload(c, indptr, indices, hop, n_rows, nnz, dx, dy, h_rescale);
    tbpm::drv_dc(c, bes, n_bes, nullptr, n_ran_samples, seed, rank, n_ran_samples, n_timestep,
                 t_step, energies, n_energies, en_inds, n_en_inds, wfn_chk_step, wfn_chk_thr,
                 dos_corr, dc_corr);
  });
}

int tbpm_dccond_states(tbpm_ctx* c, const double* bes, int n_bes, const int32_t* indptr,
                       const int32_t* indices, const double* hop, int64_t n_rows,
                       int64_t nnz, double h_rescale, const double* dx, const double* dy,
                       const double* wf0, int n_states, int n_timestep, double t_step,
                       const double* energies, int n_energies, const int32_t* en_inds,
                       int n_en_inds, int wfn_chk_step, double wfn_chk_thr,
                       double* dos_corr, double* dc_corr) {
  return guarded(c, [&] {
    if (!wf0) throw tbpm::Error{TBPM_ERR_ARG, "wf0 is null"};
    maybe_upload(c, indptr, indices, hop, n_rows, nnz, dx, dy, h_rescale);
    tbpm::drv_dc(c, bes, n_bes, wf0, n_states, 0, 0, n_states, n_timestep, t_step, energies,
                 n_energies, en_inds, n_en_inds, wfn_chk_step, wfn_chk_thr, dos_corr, dc_corr);
  });
}

int tbpm_dccond_accumulate(tbpm_ctx* c, const double* bes, int n_bes, const double* wf0,
                           int seed, int rank, int n_ran_samples, int first_state, int n_states,
                           int n_timestep, double t_step, const double* energies,
                           int n_energies, const int32_t* en_inds, int n_en_inds,
                           int wfn_chk_step, double wfn_chk_thr, double* dos_corr,
                           double* dc_corr) {
  return guarded(c, [&] {
    if (n_states < 1 || first_state < 0 || first_state + n_states > n_ran_samples)
      throw tbpm::Error{TBPM_ERR_ARG, "states outside [0, n_ran_samples)"};
    tbpm::drv_dc_part(c, bes, n_bes, wf0, first_state, n_states, n_ran_samples, seed, rank,
                      n_ran_samples, n_timestep, t_step, energies, n_energies, en_inds,
                      n_en_inds, wfn_chk_step, wfn_chk_thr, dos_corr, dc_corr, false);
  });
}

int tbpm_psi_t(tbpm_ctx* c, const double* bes, int n_bes, const int32_t* indptr,
               const int32_t* indices, const double* hop, int64_t n_rows, int64_t nnz,
               const double* psi0, const int32_t* time_log, int n_time_log, int n_timestep,
               int wfn_chk_step, double wfn_chk_thr, double* psi_t) {
  return guarded(c, [&] {
    if (!psi0 || !psi_t) throw tbpm::Error{TBPM_ERR_ARG, "null psi0 / psi_t"};
    maybe_upload(c, indptr, indices, hop, n_rows, nnz, nullptr, nullptr, 1.0);
    tbpm::drv_psi_t(c, bes, n_bes, psi0, time_log, n_time_log, n_timestep, wfn_chk_step,
                    wfn_chk_thr, psi_t);
  });
}

int tbpm_random_states(tbpm_ctx* c, int64_t n_rows, int seed, int first_sample, int n_states,
                       int rank, int n_ran_samples, int state_kind, double* wf) {
  return guarded(c, [&] {
    if (!wf) throw tbpm::Error{TBPM_ERR_ARG, "null output"};
    tbpm::drv_random_states(c, n_rows, seed, first_sample, n_states, rank, n_ran_samples,
                            state_kind, wf);
  });
}

int tbpm_fermi_cheb_coef(int nr_fermi, double beta, double mu, int one_minus_fermi, double eps,
                         double* coef, int* n_cheb) {
  if (!coef || !n_cheb) return TBPM_ERR_ARG;
  try {
    tbpm::drv_fermi_coef(nr_fermi, beta, mu, one_minus_fermi, eps, coef, n_cheb);
    return TBPM_OK;
  } catch (const tbpm::Error& e) {
    return e.code;
  } catch (...) {
    return TBPM_ERR_ARG;
  }
}

int tbpm_cheb_timestep(tbpm_ctx* c, const double* bes, int n_bes, double* wf, int n_states,
                       int forward) {
  return guarded(c, [&] {
    if (!bes || n_bes < 3 || !wf) throw tbpm::Error{TBPM_ERR_ARG, "bad arguments"};
    tbpm::Expansion ex = tbpm::time_step_expansion(bes, n_bes);
    if (!forward) ex.neg_mask = ~0ull;
    tbpm::drv_expansion_apply(c, ex, wf, n_states);
  });
}

int tbpm_fermi_apply(tbpm_ctx* c, const double* coef, int n_coef, double* wf, int n_states) {
  return guarded(c, [&] {
    if (!coef || n_coef < 3 || !wf) throw tbpm::Error{TBPM_ERR_ARG, "bad arguments"};
    const tbpm::Expansion ex = tbpm::fermi_expansion(coef, n_coef, coef, n_coef, 0ull);
    tbpm::drv_expansion_apply(c, ex, wf, n_states);
  });
}

int tbpm_dos_segmented(tbpm_ctx* c, const double* bes, int n_bes, const int32_t* indptr,
                       const int32_t* indices, const double* hop, int64_t n_rows, int64_t nnz,
                       const int64_t* seg_offsets, int n_seg, int n_states, int seed,
                       int n_timestep, int wfn_chk_step, double wfn_chk_thr, double* corr,
                       double* corr_per_state) {
  return guarded(c, [&] {
    maybe_upload(c, indptr, indices, hop, n_rows, nnz, nullptr, nullptr, 1.0);
    tbpm::drv_dos_segmented(c, bes, n_bes, seg_offsets, n_seg, n_states, seed, n_timestep,
                            wfn_chk_step, wfn_chk_thr, corr, corr_per_state);
  });
}

int tbpm_session_dos_begin(tbpm_ctx* c, const double* bes, int n_bes, int n_states, int seed,
                           int rank, int n_ran_samples, int n_timestep) {
  return guarded(c, [&] {
    tbpm::drv_session_dos_begin(c, bes, n_bes, n_states, seed, rank, n_ran_samples, n_timestep);
  });
}

int tbpm_session_advance(tbpm_ctx* c, int n_steps) {
  return guarded(c, [&] { tbpm::drv_session_advance(c, n_steps); });
}

int tbpm_session_read(tbpm_ctx* c, double* corr, double* norms, int* n_done) {
  return guarded(c, [&] { tbpm::drv_session_read(c, corr, norms, n_done); });
}

int tbpm_selftest_wait_timeout(tbpm_ctx* c) {
  return guarded(c, [&] { tbpm::drv_selftest_wait_timeout(c); });
}

int tbpm_session_export(tbpm_ctx* c, double* wf0, double* psi) {
  return guarded(c, [&] { tbpm::drv_session_export(c, wf0, psi); });
}

int tbpm_session_dos_resume(tbpm_ctx* c, const double* bes, int n_bes, int n_states,
                            const double* wf0, const double* psi, const double* corr,
                            const double* norms, int n_done, int n_timestep) {
  return guarded(c, [&] {
    tbpm::drv_session_dos_resume(c, bes, n_bes, n_states, wf0, psi, corr, norms, n_done,
                                 n_timestep);
  });
}

}  // extern "C"
