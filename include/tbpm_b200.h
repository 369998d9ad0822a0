/*
 * tbpm_b200.h -- C ABI of libtbpm_b200.so, the B200 (sm_100a) replacement of
 * the TBPM numeric core of TBPLaS (deepmodeling/tbplas 1.6.0), i.e. of the f2py
 * extension module `tbplas.fortran.f2py` built from tbplas/fortran/tbpm.f90.
 *
 * Conventions
 *  - Only plain C types cross this boundary.  Complex numbers are interleaved
 *    (re, im) doubles, exactly as numpy complex128 lays them out.
 *  - CSR arrays are 0-based (indptr[n_rows+1], indices[nnz], hop[nnz] complex),
 *    the layout produced by tbplas Sample.build_ham_csr / build_ham_dxy after
 *    f2py's cast of the index arrays to int32 (csr.F90:20-24).
 *  - Multi-dimensional outputs use the Fortran (column-major) layout that f2py
 *    returns, so a caller can wrap them with numpy order='F' unchanged.
 *  - Every function returns a status code (TBPM_OK on success); on failure
 *    tbpm_last_error() describes the problem.  The library never exits the
 *    process and never traps the GPU.  Where the reference Fortran calls
 *    `stop` (funcs.f90:175-192 check_norm) this library returns TBPM_ERR_NORM.
 *  - The random initial states of the reference come from gfortran's intrinsic
 *    RANDOM_NUMBER, which cannot be reproduced; this library draws the same
 *    distribution (random.f90:36-69) from a Philox4x32-10 stream keyed by the
 *    same seed rule (tbpm.f90:57).  The *_states entry points take the initial
 *    states from the caller instead.
 *  - Calls on one context are serialised on the context's CUDA stream.
 */
#ifndef TBPM_B200_H
#define TBPM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define TBPM_OK 0
#define TBPM_ERR_ARG 1     /* invalid argument (shape, size, range) */
#define TBPM_ERR_NORM 2    /* wave-function norm check failed (check_norm) */
#define TBPM_ERR_NAN 3     /* NaN / Inf detected */
#define TBPM_ERR_CUDA 4    /* CUDA runtime error */
#define TBPM_ERR_TIMEOUT 5 /* a bounded device-side wait expired */
#define TBPM_ERR_OOM 6     /* device allocation failed */
#define TBPM_ERR_STATE 7   /* call out of order (e.g. no Hamiltonian uploaded) */

/* arithmetic of the propagation */
#define TBPM_PREC_FP64 0 /* complex128 states, SpMV and reductions */
#define TBPM_PREC_FP32 1 /* complex64 states and SpMV; FP64 coefficients,
                            rescaling and correlation reductions */

/* random initial state distributions */
#define TBPM_STATE_EXP 0  /* |z|^2 ~ Exp(1), phase ~ U[0,2pi) (random.f90:36-69) */
#define TBPM_STATE_UNIT 1 /* |z| = 1, phase ~ U[0,2pi) */

typedef struct tbpm_ctx tbpm_ctx;

typedef struct tbpm_options {
  int precision;         /* TBPM_PREC_FP64 (default) or TBPM_PREC_FP32 */
  int batch;             /* states propagated together as one block; 0 = 16 */
  int state_kind;        /* TBPM_STATE_EXP (default) or TBPM_STATE_UNIT */
  int verbose;           /* 1: print progress like the reference on rank 0 */
  int threads_per_block; /* 0 = tuned default */
  int rows_per_tile;     /* 0 = tuned default */
  int steps_per_graph;   /* time steps captured per CUDA graph; 0 = 16 */
  int use_graphs;        /* 1 (default): replay captured CUDA graphs */
  double fp32_chk_thr;   /* lower bound of the norm-check threshold in FP32
                            mode (default 1e-4); FP64 uses wfn_chk_thr as is */
  int vector_width;      /* complex values per thread and load.  FP32: 0 = automatic
                            (4, with 256-bit accesses, when the block width is a
                            multiple of 4, else 2 when even), 1, 2.  FP64: 0 = automatic
                            (two complex128 per thread with 256-bit accesses when the
                            block width allows), 1 = one (128-bit accesses), 2 */
  int term_kernel;       /* Chebyshev-term kernel: 0 = automatic (the shared-memory
                            ring fed by bulk copies wherever a row of the state
                            block is a multiple of 16 bytes and the rows make at
                            least two ring tiles per SM, else the grid-stride
                            kernel), 1 = the grid-stride kernel with plain loads,
                            2 = the ring where it applies, 3 = two terms per
                            launch (the second term of a tile after the first
                            term of every tile it couples to, p_k read back from
                            L2) where every tile couples to at most 16 tiles,
                            4 = the ring with each tile's neighbour rows staged
                            as row windows where they fit; 3 and 4 measured
                            slower than the ring on the benchmark workload */
  double dc_budget_gb;   /* device memory (GiB) the DC driver may give its quasi-
                            eigenstate block and state ring; 0 = the free memory.
                            Fewer states per batch, then energy chunks (each
                            repeating the batch's propagation), keep it inside. */
} tbpm_options;

/* ---- context ------------------------------------------------------------ */

/* Create a context on CUDA device `device` with its own non-blocking stream. */
int tbpm_create(int device, tbpm_ctx** ctx);
int tbpm_destroy(tbpm_ctx* ctx);
const char* tbpm_last_error(const tbpm_ctx* ctx);
int tbpm_set_options(tbpm_ctx* ctx, const tbpm_options* opts);
int tbpm_get_options(const tbpm_ctx* ctx, tbpm_options* opts);
/* The cudaStream_t (as void*) all work of the context is enqueued on. */
void* tbpm_get_stream(const tbpm_ctx* ctx);
/* Statistics of the last propagation: kernel launches enqueued and the
 * algorithmic HBM bytes they move (CSR and every vector pass of the fused
 * schedule counted once; neighbour re-reads assumed to hit L2). */
int tbpm_last_stats(const tbpm_ctx* ctx, int64_t* kernel_launches, double* model_bytes);
int tbpm_version(void);

/* ---- resident Hamiltonian ------------------------------------------------ */

/* Upload a CSR Hamiltonian (host arrays) to the device in the context's
 * precision.  dx, dy (float64[nnz]) are optional (NULL) and needed by the AC
 * and DC drivers; `rescale` is Sample.rescale (used for the current operator,
 * funcs.f90:12-33).  Replaces make_csr_matrix (csr.F90:45-68). */
int tbpm_ham_upload(tbpm_ctx* ctx, const int32_t* indptr, const int32_t* indices,
                    const double* hop, int64_t n_rows, int64_t nnz, const double* dx,
                    const double* dy, double rescale);
int tbpm_ham_release(tbpm_ctx* ctx);

/* ---- supercell Hamiltonian assembled on the device ------------------------ */

/* entry layouts */
#define TBPM_LAYOUT_CSR 0 /* Sample.build_ham_csr (builder/sample.py:375-391):
                             columns sorted, on-site terms != 0, zeros dropped */
#define TBPM_LAYOUT_DXY 1 /* Sample.build_ham_dxy, algo "fast"
                             (cython/sample.pyx:150-257): on-site term first when
                             |E| >= cutoff, then hopping terms in the reference's
                             list order, with dx, dy */

/* A periodic supercell of a primitive cell, in the arrays a tbplas
 * PrimitiveCell / SuperCell / Sample hold (builder/primitive.py:957-1055,
 * builder/super.py:848-912).  Host pointers. */
typedef struct tbpm_supercell {
  const double* lat_vec;    /* [3][3] lattice vectors of the primitive cell (rows), nm */
  const double* origin;     /* [3] lattice origin, nm (NULL: 0) */
  int n_orb;                /* orbitals in the primitive cell */
  const double* orb_pos;    /* [n_orb][3] fractional orbital positions */
  const double* orb_eng;    /* [n_orb] on-site energies, eV */
  int n_hop;                /* reduced hopping terms (PrimitiveCell.hop_ind) */
  const int32_t* hop_ind;   /* [n_hop][5]: ra, rb, rc, bra orbital, ket orbital */
  const double* hop_eng;    /* [n_hop] complex (re, im) hopping energies, eV */
  int32_t dim[3];           /* supercell dimension */
  int32_t pbc[3];           /* periodic boundary conditions (0/1) */
  const int64_t* vac_id_sc; /* sorted, unique vacancy indices, numbering
                               ((ia*dim[1] + ib)*dim[2] + ic)*n_orb + o; NULL: none */
  int64_t n_vac;
  const double* sc_orb_eng; /* optional [n_rows] on-site energies of the supercell
                               orbitals in eV before rescaling (Sample.orb_eng, e.g.
                               with disorder); NULL: primitive-cell values */
  double b_field;           /* Peierls field along -z in Tesla (0: none), applied
                               before rescaling as Sample.set_magnetic_field */
  int gauge;                /* 0, 1 or 2 (cython/sample.pyx:20-74) */
  double rescale;           /* > 0: Sample.rescale_ham(rescale); <= 0: estimated
                               like Sample.get_rescale (cython/sample.pyx:77-116) */
} tbpm_supercell;

/* Assemble the Hamiltonian of a supercell on the device and keep it resident
 * in the context, in place of Sample.build_ham_csr / build_ham_dxy + a host
 * CSR upload (tbpm_ham_upload).  The TBPM drivers then run on it with
 * indptr == NULL.  layout: TBPM_LAYOUT_CSR for DOS / LDOS / psi_t,
 * TBPM_LAYOUT_DXY (with dx, dy) for AC / DC; orb_eng_cutoff is the DXY
 * on-site cutoff (eV after rescaling, reference default 1e-5).
 * Returns the row count, the entry count of the full CSR and the rescale
 * factor used.  Positions, dr, the rescale estimate and field-free values are
 * bit-identical to the reference builder; Peierls factors are within 2 ulp. */
int tbpm_supercell_ham(tbpm_ctx* ctx, const tbpm_supercell* sc, int layout,
                       double orb_eng_cutoff, int64_t* n_rows, int64_t* nnz,
                       double* rescale);

/* As tbpm_supercell_ham, but copies the full CSR of the layout to host
 * arrays: indptr int64[n_rows+1], indices int32[nnz], hop complex128[nnz],
 * dx, dy float64[nnz] (DXY only; may be NULL).  With indptr == NULL only
 * n_rows, nnz and rescale are returned (call twice to size the arrays). */
int tbpm_supercell_csr(tbpm_ctx* ctx, const tbpm_supercell* sc, int layout,
                       double orb_eng_cutoff, int64_t* n_rows, int64_t* nnz, double* rescale,
                       int64_t* indptr, int32_t* indices, double* hop, double* dx,
                       double* dy);

/* ---- f2py-equivalent drivers (host buffers in, host buffers out) --------- */

/* tbpm_dos -- replaces tbpm.f90:6-93 (SUBROUTINE tbpm_dos) as called from
 * Solver.calc_corr_dos (tbpm/solver.py:256-284).
 * corr: complex128[n_timestep + 1].  Uses the uploaded Hamiltonian when
 * indptr == NULL, otherwise uploads (indptr, indices, hop) first. */
int tbpm_dos(tbpm_ctx* ctx, const double* bes, int n_bes, const int32_t* indptr,
             const int32_t* indices, const double* hop, int64_t n_rows, int64_t nnz,
             int seed, int n_timestep, int n_ran_samples, int rank, int wfn_chk_step,
             double wfn_chk_thr, double* corr);

/* As tbpm_dos with caller-supplied initial states wf0 (complex128
 * [n_states][n_rows], C order).  corr_per_state (optional, complex128
 * [n_states][n_timestep + 1]) receives the unaveraged correlations. */
int tbpm_dos_states(tbpm_ctx* ctx, const double* bes, int n_bes, const int32_t* indptr,
                    const int32_t* indices, const double* hop, int64_t n_rows, int64_t nnz,
                    const double* wf0, int n_states, int n_timestep, int wfn_chk_step,
                    double wfn_chk_thr, double* corr, double* corr_per_state);

/* tbpm_accond -- replaces tbpm.f90:193-351 (SUBROUTINE tbpm_accond) as called
 * from Solver.calc_corr_ac_cond (tbpm/solver.py:317-352).
 * corr: complex128 (4, n_timestep) Fortran order (xx, xy, yx, yy); column 1
 * (t = 1) is zero as in the reference. */
int tbpm_accond(tbpm_ctx* ctx, const double* bes, int n_bes, double beta, double mu,
                const int32_t* indptr, const int32_t* indices, const double* hop,
                int64_t n_rows, int64_t nnz, double h_rescale, const double* dx,
                const double* dy, int seed, int n_timestep, int n_ran_samples, int nr_fermi,
                double fermi_precision, int rank, int wfn_chk_step, double wfn_chk_thr,
                double* corr);

/* As tbpm_accond with caller-supplied initial states (complex128 [n_states][n_rows]). */
int tbpm_accond_states(tbpm_ctx* ctx, const double* bes, int n_bes, double beta, double mu,
                       const int32_t* indptr, const int32_t* indices, const double* hop,
                       int64_t n_rows, int64_t nnz, double h_rescale, const double* dx,
                       const double* dy, const double* wf0, int n_states, int n_timestep,
                       int nr_fermi, double fermi_precision, int wfn_chk_step,
                       double wfn_chk_thr, double* corr);

/* tbpm_dccond -- replaces tbpm.f90:497-718 (SUBROUTINE tbpm_dccond) as called
 * from Solver.calc_corr_dc_cond (tbpm/solver.py:393-441).
 * dos_corr: complex128[n_timestep]; dc_corr: complex128 (2, n_energies,
 * n_timestep) Fortran order, the first n_en_inds rows of the energy axis
 * filled (as in the reference). */
int tbpm_dccond(tbpm_ctx* ctx, const double* bes, int n_bes, double beta, double mu,
                const int32_t* indptr, const int32_t* indices, const double* hop,
                int64_t n_rows, int64_t nnz, double h_rescale, const double* dx,
                const double* dy, int seed, int n_timestep, int n_ran_samples, double t_step,
                const double* energies, int n_energies, const int32_t* en_inds,
                int n_en_inds, int rank, int wfn_chk_step, double wfn_chk_thr,
                double* dos_corr, double* dc_corr);

/* As tbpm_dccond with caller-supplied initial states (complex128 [n_states][n_rows]). */
int tbpm_dccond_states(tbpm_ctx* ctx, const double* bes, int n_bes, const int32_t* indptr,
                       const int32_t* indices, const double* hop, int64_t n_rows,
                       int64_t nnz, double h_rescale, const double* dx, const double* dy,
                       const double* wf0, int n_states, int n_timestep, double t_step,
                       const double* energies, int n_energies, const int32_t* en_inds,
                       int n_en_inds, int wfn_chk_step, double wfn_chk_thr,
                       double* dos_corr, double* dc_corr);

/* Part of a tbpm_dccond run on the resident Hamiltonian (uploaded with dx, dy):
 * the states [first_state, first_state + n_states) of a run of n_ran_samples
 * states.  Their contributions, each divided by n_ran_samples, are ADDED to
 * dos_corr and dc_corr (layouts as tbpm_dccond) in the order tbpm_dccond adds
 * them, so a run taken in consecutive parts with the outputs kept in between
 * reproduces the same sums; DC checkpointing saves the outputs between parts.
 * States are seeded as in tbpm_dccond (seed, rank, n_ran_samples), or, if wf0
 * is not NULL, wf0 = complex128 [n_states][n_rows] holds this part's states.
 * No counterpart in the reference (its run is one call). */
int tbpm_dccond_accumulate(tbpm_ctx* ctx, const double* bes, int n_bes, const double* wf0,
                           int seed, int rank, int n_ran_samples, int first_state, int n_states,
                           int n_timestep, double t_step, const double* energies,
                           int n_energies, const int32_t* en_inds, int n_en_inds,
                           int wfn_chk_step, double wfn_chk_thr, double* dos_corr,
                           double* dc_corr);

/* tbpm_psi_t -- replaces tbpm.f90:1029-1093 (SUBROUTINE tbpm_psi_t) as called
 * from Solver.calc_psi_t (tbpm/solver.py:543-600).
 * psi0: complex128[n_rows]; time_log: int32[n_time_log] sorted, unique, in
 * [0, n_timestep]; psi_t: complex128 (n_rows, n_time_log) Fortran order. */
int tbpm_psi_t(tbpm_ctx* ctx, const double* bes, int n_bes, const int32_t* indptr,
               const int32_t* indices, const double* hop, int64_t n_rows, int64_t nnz,
               const double* psi0, const int32_t* time_log, int n_time_log, int n_timestep,
               int wfn_chk_step, double wfn_chk_thr, double* psi_t);

/* tbpm_dyn_pol -- replaces tbpm.f90:355-493 (SUBROUTINE tbpm_dyn_pol) as called
 * from Solver.calc_corr_dyn_pol (tbpm/solver.py:354-390).
 * site_x/y/z: float64[n_rows] orbital positions (Sample.orb_pos columns);
 * q_points: float64 [n_q_points][3] (C order); corr: float64 (n_q_points,
 * n_timestep) Fortran order, corr(q, t) = Im <psi2(t)| exp(i q.r) psi1(t)>
 * averaged over the states.  The psi2 vectors of a batch are shared by all its
 * q-points (they do not depend on q). */
int tbpm_dyn_pol(tbpm_ctx* ctx, const double* bes, int n_bes, double beta, double mu,
                 const int32_t* indptr, const int32_t* indices, const double* hop,
                 int64_t n_rows, int64_t nnz, double h_rescale, const double* dx,
                 const double* dy, const double* site_x, const double* site_y,
                 const double* site_z, int seed, int n_timestep, int n_ran_samples,
                 int nr_fermi, double fermi_precision, const double* q_points, int n_q_points,
                 int rank, int wfn_chk_step, double wfn_chk_thr, double* corr);

/* As tbpm_dyn_pol with caller-supplied initial states (complex128 [n_states][n_rows]). */
int tbpm_dyn_pol_states(tbpm_ctx* ctx, const double* bes, int n_bes, double beta, double mu,
                        const int32_t* indptr, const int32_t* indices, const double* hop,
                        int64_t n_rows, int64_t nnz, const double* site_x,
                        const double* site_y, const double* site_z, const double* q_points,
                        int n_q_points, const double* wf0, int n_states, int n_timestep,
                        int nr_fermi, double fermi_precision, int wfn_chk_step,
                        double wfn_chk_thr, double* corr);

/* tbpm_eigenstates -- replaces tbpm.f90:721-830 (SUBROUTINE tbpm_eigenstates)
 * as called from Solver.calc_quasi_eigenstates (tbpm/solver.py:474-507).
 * wf_qe: float64 (n_energies, n_rows) Fortran order, the sample average of
 * |QE_i(r)|^2 of the normalised Hanning-windowed quasi-eigenstates. */
int tbpm_eigenstates(tbpm_ctx* ctx, const double* bes, int n_bes, const int32_t* indptr,
                     const int32_t* indices, const double* hop, int64_t n_rows, int64_t nnz,
                     int seed, int n_timestep, int n_ran_samples, double t_step,
                     const double* energies, int n_energies, int rank, int wfn_chk_step,
                     double wfn_chk_thr, double* wf_qe);

/* As tbpm_eigenstates with caller-supplied initial states. */
int tbpm_eigenstates_states(tbpm_ctx* ctx, const double* bes, int n_bes, const int32_t* indptr,
                            const int32_t* indices, const double* hop, int64_t n_rows,
                            int64_t nnz, const double* wf0, int n_states, int n_timestep,
                            double t_step, const double* energies, int n_energies,
                            int wfn_chk_step, double wfn_chk_thr, double* wf_qe);

/* tbpm_kbdc -- replaces tbpm.f90:836-960 (SUBROUTINE tbpm_kbdc) as called from
 * Solver.calc_hall_mu (tbpm/solver.py:443-472).  direction 1: J_x, 2: J_y on
 * the ket side.  mu: complex128 (n_kernel, n_kernel) Fortran order,
 * mu(m, n) = g_m g_n <T_m(H) J_x psi | J_dir T_n(H) psi> averaged over the
 * states (g: Jackson kernel).  The n_kernel^2 inner products run as complex
 * GEMMs (cuBLAS, loaded on first use); memory: (n_kernel + 134) vectors. */
int tbpm_kbdc(tbpm_ctx* ctx, int seed, const int32_t* indptr, const int32_t* indices,
              const double* hop, int64_t n_rows, int64_t nnz, double h_rescale,
              const double* dx, const double* dy, int n_ran_samples, int n_kernel,
              int direction, int rank, double* mu);

/* As tbpm_kbdc with caller-supplied initial states. */
int tbpm_kbdc_states(tbpm_ctx* ctx, const int32_t* indptr, const int32_t* indices,
                     const double* hop, int64_t n_rows, int64_t nnz, double h_rescale,
                     const double* dx, const double* dy, const double* wf0, int n_states,
                     int n_kernel, int direction, double* mu);

/* Haydock (Lanczos) coefficients of ldos_haydock -- replaces tbpm.f90:963-1026
 * with propagation.f90:85-155 (SUBROUTINE Haydock_coef), averaged over
 * n_samples start vectors whose amplitudes on the sites are wf_sites
 * (complex128 [n_samples][n_sites]).  coefa: complex128[n_depth],
 * coefb: float64[n_depth].  The Green function and LDOS on the energy grid
 * (funcs.f90:152-172) are evaluated by the caller. */
int tbpm_haydock_coef(tbpm_ctx* ctx, const int32_t* indptr, const int32_t* indices,
                      const double* hop, int64_t n_rows, int64_t nnz, double h_rescale,
                      const int32_t* site_indices, int n_sites, const double* wf_sites,
                      int n_samples, int n_depth, double* coefa, double* coefb);

/* cond_from_trace -- replaces analysis.f90:6-69 (SUBROUTINE cond_from_trace,
 * with kpm.f90:31-56 get_gamma_mn) as called from Analyzer.calc_hall_cond
 * (tbpm/analysis.py:513-575).  mu_mn: complex128 (n_kernel, n_kernel) Fortran
 * order; mu: chemical potentials (eV); cond: float64[n_mu], before the
 * Analyzer's prefactor.  The n_kernel^2 x (ne_integral-1) trace runs on the
 * GPU; the final Fermi integral on the host.  fermi_precision and rank are
 * accepted for the reference's argument list and unused, as there. */
int tbpm_cond_from_trace(tbpm_ctx* ctx, const double* mu_mn, int n_kernel, const double* mu,
                         int n_mu, double h_rescale, double beta, int ne_integral,
                         double fermi_precision, int rank, double* cond);

/* DOS correlations of many uneven realisations packed into one block-diagonal
 * Hamiltonian (a batch of samples; the TBPM loop of tbpm.f90:50-86 run for
 * every realisation at once).  Realisation k owns rows
 * [seg_offsets[k], seg_offsets[k+1]) (seg_offsets[0] = 0,
 * seg_offsets[n_seg] = n_rows) and n_states random states drawn over its own
 * rows with iseed = seed*(k*n_states + s + 1) and normalised there.  All
 * realisations share the Bessel series (one rescale factor).  The whole
 * propagation is captured as one CUDA graph and launched once.
 * corr: complex128 [n_seg][n_timestep+1] (state average per realisation);
 * corr_per_state (optional): complex128 [n_seg][n_states][n_timestep+1]. */
int tbpm_dos_segmented(tbpm_ctx* ctx, const double* bes, int n_bes, const int32_t* indptr,
                       const int32_t* indices, const double* hop, int64_t n_rows, int64_t nnz,
                       const int64_t* seg_offsets, int n_seg, int n_states, int seed,
                       int n_timestep, int wfn_chk_step, double wfn_chk_thr, double* corr,
                       double* corr_per_state);

/* ---- building blocks ----------------------------------------------------- */

/* Random initial states of the reference distribution (random.f90:36-69) with
 * the seed rule iseed = seed*(first_sample + i + rank*n_ran_samples) for
 * i = 0..n_states-1 (tbpm.f90:57, first_sample is 1-based).
 * wf: complex128 [n_states][n_rows]. */
int tbpm_random_states(tbpm_ctx* ctx, int64_t n_rows, int seed, int first_sample,
                       int n_states, int rank, int n_ran_samples, int state_kind,
                       double* wf);

/* Chebyshev coefficients of the Fermi (one_minus_fermi = 0) or 1 - Fermi
 * operator (funcs.f90:60-123 get_Fermi_cheb_coef); coef holds nr_fermi
 * doubles; returns n_cheb through *n_cheb. */
int tbpm_fermi_cheb_coef(int nr_fermi, double beta, double mu, int one_minus_fermi,
                         double eps, double* coef, int* n_cheb);

/* One time step psi <- exp(-/+ i H dt) psi of n_states states with the uploaded
 * Hamiltonian (propagation.f90:12-49 cheb_wf_timestep).
 * wf: complex128 [n_states][n_rows], in place. */
int tbpm_cheb_timestep(tbpm_ctx* ctx, const double* bes, int n_bes, double* wf,
                       int n_states, int forward);

/* Fermi operator f(H) psi of n_states states with the uploaded Hamiltonian
 * (propagation.f90:52-82 Fermi).  wf: complex128 [n_states][n_rows], in place. */
int tbpm_fermi_apply(tbpm_ctx* ctx, const double* coef, int n_coef, double* wf,
                     int n_states);

/* One time step psi <- exp(-/+ i H dt) psi that allocates no device memory.
 * No counterpart in the reference: it exists for callers that cannot call
 * cudaMalloc (or have the library call it), e.g. a framework whose caching
 * allocator owns nearly all of HBM, or a loop where allocation after start-up
 * is forbidden.  All array arguments except bes are DEVICE pointers from the
 * caller's own allocator: the full CSR (diagonal entries included) and
 * wf = complex128 [n_rows][n_states] row-interleaved, updated in place; they
 * must be memory of the context's device (or managed), wf and hop 16-byte
 * aligned, indptr and indices 4-byte aligned, else TBPM_ERR_ARG before any
 * launch.  The two work vectors come from a fixed 16 MiB array inside the
 * library (held by every GPU that loads it until exit; 256 bytes of it are a
 * status word), so n_rows * n_states may be at most (16 MiB - 256) / 32 =
 * 524,280; larger sizes return TBPM_ERR_ARG.  The first call on a context
 * looks up that array's device address (make it before any stream capture).  All
 * calls share the array: calls that overlap on the GPU race, so serialise
 * them.  The call validates the CSR on the device and is synchronous on the
 * context stream.  FP64 only. */
int tbpm_cheb_timestep_noalloc(tbpm_ctx* ctx, const double* bes, int n_bes,
                               const int32_t* indptr, const int32_t* indices,
                               const double* hop, int64_t n_rows, int64_t nnz, double* wf,
                               int n_states, int forward);

/* Self-test of the device-side failure path (no counterpart in the reference,
 * whose only failure check is check_norm): one block waits, with the bounded
 * wait of the Chebyshev-term ring kernels, on a shared-memory barrier that
 * nothing completes.  The wait gives up after 2 s and records it in the
 * context's status word; the call then returns TBPM_ERR_TIMEOUT, as a
 * propagation whose wait ran out would, and the context stays usable. */
int tbpm_selftest_wait_timeout(tbpm_ctx* ctx);

/* ---- Analyzer transforms on the device ---------------------------------- */

/* Window-weighted trigonometric sums of correlation functions, the
 * O(tnr^2) part of Analyzer.calc_ac_cond (analysis.py:161-243) and
 * calc_dyn_pol (:245-308) and the sums of calc_dc_cond (:375-458).  For output
 * o = r * n_x + i:
 *   out_cos[o] = sum_k w[k] a[q][k] cos(phase_ik),
 *   out_sin[o] = sum_k w[k] b[q][k] sin(phase_ik),
 * k < n_k, with phase_ik = (x[i] * k) * dt, or x[i] * (k * dt) when phase_kdt is
 * 1, and q = r (per_output = 0: a, b are [n_rows][n_k]) or q = o (per_output =
 * 1: a, b are [n_rows][n_x][n_k]).  Either output may be NULL (its coefficient
 * array is then not read).  Host arrays; synchronous. */
int tbpm_trig_sums(tbpm_ctx* ctx, const double* w, int n_k, const double* a, const double* b,
                   int n_rows, const double* x, int n_x, double dt, int per_output,
                   int phase_kdt, double* out_cos, double* out_sin);
/* The cumulative trapezoid of Analyzer.calc_diff_coeff (analysis.py:460-511):
 * for row q < n_rows, y_k = (a[q][k] cos(x[q] k dt) + b[q][k] sin(x[q] k dt)) w[k]
 * and out[q][0] = 0, out[q][j] = out[q][j-1] + (spacing[j-1] (y_{j-1} + y_j)) / 2
 * (scipy's cumulative_trapezoid over a grid with the given spacing).  Host
 * arrays; synchronous. */
int tbpm_trig_cumtrapz(tbpm_ctx* ctx, const double* w, int n_k, const double* a,
                       const double* b, int n_rows, const double* x, double dt,
                       const double* spacing, double* out);

/* ---- learned C(t) tail extrapolator: BF16 kernels, FP32 accumulation ------
 * No counterpart in the reference (TBPLaS has no learned component).  All
 * pointers are device pointers owned by the caller; `stream` is a
 * cudaStream_t (NULL = default stream); calls are asynchronous.  BF16 arrays
 * are __nv_bfloat16 (passed as void*).  Layouts are row-major; convolution
 * activations are channel-last [batch][length][channels]. */

/* C[M,N] = alpha * A[M,K] . B[N,K]^T + beta * C (A, B BF16 with K contiguous,
 * 16-byte aligned rows: K, lda, ldb multiples of 8; C FP32) on the
 * 5th-generation tensor cores: TMA (128-byte swizzle) into a 4-stage
 * shared-memory ring, tcgen05.mma (BF16 -> FP32) with the 128 x 128
 * accumulator in tensor memory, tcgen05.ld epilogue. */
int tbpm_nn_gemm_tn(const void* A, int lda, const void* B, int ldb, float* C, int ldc, int M,
                    int N, int K, float alpha, float beta, void* stream);
/* The same product through mma.sync m16n8k16 (an independent implementation,
 * kept to check the tensor-core GEMM). */
int tbpm_nn_gemm_tn_mma(const void* A, int lda, const void* B, int ldb, float* C, int ldc,
                        int M, int N, int K, float alpha, float beta, void* stream);
/* 1 in *failed if a bounded wait of the tensor-core GEMM ran out since the
 * last call (that launch wrote nothing to C); resets the flag.  Synchronous. */
int tbpm_nn_tc_status(int* failed);
/* out[c][r] = in[r][c] (BF16) */
int tbpm_nn_transpose_bf16(const void* in, int rows, int cols, void* out, void* stream);
/* Xcol[(b*Lout + lo)][j*C + c] = X[b][lo*stride + j - pad][c], zero outside */
int tbpm_nn_im2col(const void* X, int batch, int L, int C, int k, int stride, int pad,
                   int Lout, void* Xcol, void* stream);
/* dX[b][l][c] = sum of dXcol entries that im2col copied from X[b][l][c] (FP32) */
int tbpm_nn_col2im(const float* dXcol, int batch, int L, int C, int k, int stride, int pad,
                   int Lout, float* dX, void* stream);
/* a = act(Z + bias) (act 0: identity, 1: GELU, erf form); pre (optional)
 * receives Z + bias; outputs in BF16 and/or FP32 (either may be NULL). */
int tbpm_nn_bias_act(const float* Z, const float* bias, int M, int N, int act, float* pre,
                     void* out_bf16, float* out_f32, void* stream);
/* dZ = dA * act'(pre), FP32 and/or BF16 output */
int tbpm_nn_act_backward(const float* dA, const float* pre, int64_t n, int act, float* dZ,
                         void* dZ_bf16, void* stream);
/* out[n] = sum_m Z[m][n] (bias gradients) */
int tbpm_nn_colsum(const float* Z, int M, int N, float* out, void* stream);
/* loss = mean((pred - target)^2) (device double), grad = d loss / d pred
 * (optional); work: device scratch of >= 256 doubles */
int tbpm_nn_mse(const float* pred, const float* target, int64_t n, float* grad, double* work,
                double* loss, void* stream);
/* AdamW step on FP32 master weights (step counts from 1); optional BF16 copy */
int tbpm_nn_adam(float* w, const float* g, float* m, float* v, int64_t n, float lr, float b1,
                 float b2, float eps, float weight_decay, int step, void* w_bf16, void* stream);
int tbpm_nn_cast_bf16(const float* in, int64_t n, void* out, void* stream);

/* ---- device-resident propagation session (benchmarks, batching) --------- */

/* Start a DOS propagation of n_states random states (seed rule as
 * tbpm_random_states with first_sample = 1) on the uploaded Hamiltonian, with
 * room for n_timestep steps.  Records corr(0).  With CUDA graphs enabled the
 * graph of opts.steps_per_graph steps is captured and uploaded here, so that
 * tbpm_session_advance only replays it. */
int tbpm_session_dos_begin(tbpm_ctx* ctx, const double* bes, int n_bes, int n_states,
                           int seed, int rank, int n_ran_samples, int n_timestep);
/* Enqueue n_steps time steps on the context stream; returns without waiting. */
int tbpm_session_advance(tbpm_ctx* ctx, int n_steps);
/* Wait for the stream and copy the per-state correlations recorded so far:
 * corr complex128 [n_rows_done][n_states], norms float64 [n_rows_done][n_states]
 * (either may be NULL).  *n_done receives the number of recorded time rows. */
int tbpm_session_read(tbpm_ctx* ctx, double* corr, double* norms, int* n_done);

/* Checkpoint support (the reference has no counterpart: its long runs restart
 * from scratch).  Export copies the session's initial states wf0 and current
 * states psi (complex128 [n_states][n_rows]) to the host (either may be NULL);
 * with tbpm_session_read's rows this is everything a DOS run needs to go on. */
int tbpm_session_export(tbpm_ctx* ctx, double* wf0, double* psi);
/* Start a DOS session on the uploaded Hamiltonian from such a state: wf0, psi
 * and the n_done recorded rows (corr complex128 [n_done][n_states], norms
 * float64 [n_done][n_states]).  With n_done == 0 the session starts from wf0
 * (row 0 recorded, psi unused), i.e. tbpm_session_dos_begin with given
 * states.  A resumed run reproduces the uninterrupted one bit for bit. */
int tbpm_session_dos_resume(tbpm_ctx* ctx, const double* bes, int n_bes, int n_states,
                            const double* wf0, const double* psi, const double* corr,
                            const double* norms, int n_done, int n_timestep);

#ifdef __cplusplus
}
#endif

#endif /* TBPM_B200_H */
