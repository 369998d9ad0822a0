"""GPU parity of the TBPM drivers against the CPU oracle (identical inputs).

Tolerances: FP64 results must match the oracle to a relative 1e-10 (max
|diff| / max |oracle|); FP32-state results are compared with the stated
looser bounds.
"""

import math

import numpy as np
import pytest

import tbplas_b200 as tb
from tbplas_b200 import _native as nat
from tbplas_b200.fortran import f2py
from oracle import oracle

from conftest import bessel_series, rel_err, unit_states

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10


@pytest.fixture(autouse=True)
def _fp64_backend():
    f2py.set_backend(precision="fp64", batch=16, device=0, state_kind="exp",
                     use_graphs=True, threads_per_block=0, rows_per_tile=0)
    yield
    f2py.set_backend(precision="fp64", batch=16, state_kind="exp", use_graphs=True)


def _csr(s):
    h = s.build_ham_csr()
    return h.indptr, h.indices, h.data


def test_dos_fp64_matches_oracle(graphene_small, dos_bes):
    ip, ix, hv = _csr(graphene_small)
    wf0 = unit_states(5, ip.size - 1)
    gpu, per = f2py.tbpm_dos_states(dos_bes, ip, ix, hv, wf0, 48, 128, 1e-9, per_state=True)
    ref = oracle.tbpm_dos(dos_bes, ip, ix, hv, 48, wf0=wf0)
    assert rel_err(gpu, ref) < FP64_TOL
    for b in range(5):
        one = oracle.tbpm_dos(dos_bes, ip, ix, hv, 48, wf0=wf0[b])
        assert rel_err(per[b], one) < FP64_TOL


@pytest.mark.parametrize("batch,graphs", [(2, True), (3, False), (64, True)])
def test_dos_batching_and_graphs(graphene_small, dos_bes, batch, graphs):
    ip, ix, hv = _csr(graphene_small)
    wf0 = unit_states(5, ip.size - 1, seed=3)
    f2py.set_backend(batch=batch, use_graphs=graphs, steps_per_graph=4)
    gpu = f2py.tbpm_dos_states(dos_bes, ip, ix, hv, wf0, 37, 128, 1e-9)
    ref = oracle.tbpm_dos(dos_bes, ip, ix, hv, 37, wf0=wf0)
    assert rel_err(gpu, ref) < FP64_TOL


def test_dos_config1_graphene_100x100(dos_bes):
    """Graphene 100x100 PBC, t=-2.7, rescale 9, 1 unit-modulus state, 256 steps."""
    s = tb.make_graphene_sample(100, 100, rescale=9.0)
    ip, ix, hv = _csr(s)
    assert ip.size - 1 == 20000 and ix.size == 60000
    wf0 = unit_states(1, 20000)
    gpu = f2py.tbpm_dos_states(dos_bes, ip, ix, hv, wf0, 256, 128, 1e-9)
    ref = oracle.tbpm_dos(dos_bes, ip, ix, hv, 256, wf0=wf0)
    assert rel_err(gpu, ref) < FP64_TOL


def test_random_states_match_oracle():
    n = 1000
    got = f2py.random_states(n, seed=1337, n_states=3, rank=1, n_ran_samples=3)
    for i in range(3):
        ref = oracle.random_state(n, 1337 * (i + 1 + 1 * 3), kind=0)
        assert np.max(np.abs(got[i] - ref)) < 1e-14
    assert np.allclose(np.linalg.norm(got, axis=1), 1.0, atol=1e-14)


def test_dos_seeded_matches_oracle(graphene_small, dos_bes):
    ip, ix, hv = _csr(graphene_small)
    gpu = f2py.tbpm_dos(dos_bes, ip, ix, hv, 1337, 40, 3, "unused", 0, 128, 1e-9)
    ref = oracle.tbpm_dos(dos_bes, ip, ix, hv, 40, seed=1337, n_samples=3)
    assert rel_err(gpu, ref) < FP64_TOL


@pytest.mark.parametrize("forward", [True, False])
def test_cheb_timestep_matches_oracle(graphene_small, dos_bes, forward):
    ip, ix, hv = _csr(graphene_small)
    n = ip.size - 1
    wf = unit_states(3, n, seed=11)
    ctx = f2py._ctx()
    ip32, ix32 = ip.astype(np.int32), ix.astype(np.int32)
    ctx.call("tbpm_ham_upload", nat.ptr(ip32), nat.ptr(ix32), nat.ptr(hv), n, hv.size, None,
             None, 1.0)
    bes = np.asarray(dos_bes)
    got = np.ascontiguousarray(wf.copy())
    ctx.call("tbpm_cheb_timestep", nat.ptr(bes), bes.size, nat.ptr(got), 3, 1 if forward else 0)
    for b in range(3):
        ref = oracle.cheb_timestep(bes, ip, ix, hv, wf[b], forward=forward)
        assert rel_err(got[b], ref) < 1e-12


def test_fermi_apply_matches_oracle(graphene_small):
    ip, ix, hv = _csr(graphene_small)
    n = ip.size - 1
    beta = 9.0 / (tb.KB * 300)
    coef = nat.fermi_cheb_coef(2**15, beta, 0.0, False, 1e-12)
    wf = unit_states(2, n, seed=5)
    ctx = f2py._ctx()
    ip32, ix32 = ip.astype(np.int32), ix.astype(np.int32)
    ctx.call("tbpm_ham_upload", nat.ptr(ip32), nat.ptr(ix32), nat.ptr(hv), n, hv.size, None,
             None, 1.0)
    got = np.ascontiguousarray(wf.copy())
    ctx.call("tbpm_fermi_apply", nat.ptr(coef), coef.size, nat.ptr(got), 2)
    for b in range(2):
        ref = oracle.fermi(coef, ip, ix, hv, wf[b])
        assert rel_err(got[b], ref) < 1e-10


def _dxy(s):
    return s.build_ham_dxy()


def test_ac_fp64_matches_oracle(ac_bes):
    s = tb.make_graphene_sample(8, 6, disorder=0.6, rescale=9.0, seed=3)
    ip, ix, hv, dx, dy = _dxy(s)
    n = ip.size - 1
    wf0 = unit_states(3, n, seed=21)
    beta = 9.0 / (tb.KB * 300)
    gpu = f2py.tbpm_accond_states(ac_bes, beta, 0.0, ip, ix, hv, s.rescale, dx, dy, wf0, 24,
                                  2**15, 1e-12, 128, 1e-9)
    ref = oracle.tbpm_accond(ac_bes, beta, 0.0, ip, ix, hv, s.rescale, dx, dy, 24, wf0=wf0)
    assert gpu.shape == (4, 24) and gpu.flags.f_contiguous
    assert np.all(gpu[:, 0] == 0)
    assert rel_err(gpu, ref) < FP64_TOL


def test_ac_seeded_matches_oracle(ac_bes):
    s = tb.make_graphene_sample(6, 6, disorder=0.3, rescale=9.0, seed=4)
    ip, ix, hv, dx, dy = _dxy(s)
    beta = 9.0 / (tb.KB * 300)
    gpu = f2py.tbpm_accond(ac_bes, beta, 0.1 / 9.0, ip, ix, hv, s.rescale, dx, dy, 1337, 12, 2,
                           2**15, 1e-12, "unused", 0, 128, 1e-9)
    ref = oracle.tbpm_accond(ac_bes, beta, 0.1 / 9.0, ip, ix, hv, s.rescale, dx, dy, 12,
                             seed=1337, n_samples=2)
    assert rel_err(gpu, ref) < FP64_TOL


def _dc_energies(s, tnr, limits=(-0.5, 0.5)):
    en_range = s.energy_range
    energies = np.array([0.5 * i * en_range / tnr - en_range / 2. for i in range(tnr * 2)])
    qe = np.where((energies >= limits[0]) & (energies <= limits[1]))[0]
    return energies, qe


@pytest.mark.parametrize("tnr", [20, 37])
def test_dc_fp64_matches_oracle(dos_bes, tnr):
    s = tb.make_graphene_sample(8, 6, disorder=0.8, rescale=9.0, seed=9)
    ip, ix, hv, dx, dy = _dxy(s)
    n = ip.size - 1
    wf0 = unit_states(2, n, seed=31)
    energies, qe = _dc_energies(s, tnr, limits=(-2.0, 2.0))
    t_step = 2 * math.pi / s.energy_range
    dos, dc = f2py.tbpm_dccond_states(dos_bes, ip, ix, hv, s.rescale, dx, dy, wf0, tnr, t_step,
                                      energies, qe, 128, 1e-9)
    rdos, rdc = oracle.tbpm_dccond(dos_bes, ip, ix, hv, s.rescale, dx, dy, tnr, t_step,
                                   energies, qe, wf0=wf0)
    assert dc.shape == (2, 2 * tnr, tnr)
    assert rel_err(dos, rdos) < FP64_TOL
    assert rel_err(dc, rdc) < FP64_TOL
    assert np.all(dc[:, qe.size:, :] == 0)


def test_psi_t_matches_oracle(graphene_small, dos_bes):
    ip, ix, hv = _csr(graphene_small)
    n = ip.size - 1
    psi0 = unit_states(1, n, seed=41)[0]
    time_log = np.array([0, 1, 5, 17, 30])
    got = f2py.tbpm_psi_t(dos_bes, ip, ix, hv, psi0, time_log, 30, 128, 1e-9)
    ref = oracle.tbpm_psi_t(dos_bes, ip, ix, hv, psi0, time_log, 30)
    assert got.shape == (n, 5) and got.flags.f_contiguous
    assert rel_err(got, ref) < FP64_TOL
    assert np.allclose(np.linalg.norm(got, axis=0), 1.0, atol=1e-12)


def test_norm_check_reports_error_instead_of_stopping(dos_bes):
    """rescale below the spectral radius makes the Chebyshev series diverge:
    the reference `stop`s in check_norm, the library returns TBPM_ERR_NORM."""
    s = tb.make_graphene_sample(8, 8, rescale=2.0)
    ip, ix, hv = _csr(s)
    wf0 = unit_states(1, ip.size - 1)
    with pytest.raises(nat.NormError):
        f2py.tbpm_dos_states(dos_bes, ip, ix, hv, wf0, 16, 8, 1e-9)
    with pytest.raises(oracle.OracleError):
        oracle.tbpm_dos(dos_bes, ip, ix, hv, 16, wf0=wf0, chk_step=8)


def test_invalid_csr_rejected_before_launch(dos_bes):
    ip = np.array([0, 2, 3], dtype=np.int32)
    ix = np.array([1, 5, 0], dtype=np.int32)  # column 5 out of range
    hv = np.ones(3, dtype=np.complex128)
    with pytest.raises(ValueError):
        f2py.tbpm_dos_states(dos_bes, ip, ix, hv, unit_states(1, 2), 4, 128, 1e-9)


@pytest.mark.parametrize("indptr,indices", [([0, 3, 2], [0, 1, 1]),      # indptr decreases
                                            ([0, 1, 2], [0, -1]),         # negative column
                                            ([0, 2, 3], [0, 1, 2])])      # column == n
def test_invalid_csr_variants_rejected(dos_bes, indptr, indices):
    ip = np.array(indptr, dtype=np.int32)
    ix = np.array(indices, dtype=np.int32)
    hv = np.ones(ix.size, dtype=np.complex128)
    with pytest.raises(ValueError):
        f2py.tbpm_dos_states(dos_bes, ip, ix, hv, unit_states(1, 2), 4, 128, 1e-9)


@pytest.mark.parametrize("prec,tol", [("fp64", FP64_TOL), ("fp32", 2e-5)])
def test_repeated_and_unsorted_diagonal_entries(graphene_small, dos_bes, prec, tol):
    """Rows with the diagonal split into two entries, placed anywhere in the
    row: the upload sums them into D; the oracle multiplies them as given."""
    h = graphene_small.build_ham_csr()
    n = h.shape[0]
    rows, cols, vals = [], [], []
    for r in range(n):
        a, b = h.indptr[r], h.indptr[r + 1]
        c, v = list(h.indices[a:b]), list(h.data[a:b])
        if r % 3 == 0:
            c = [r] + c + [r]
            v = [0.01 + 0.002j] + v + [-0.03 + 0j]
        rows += [r] * len(c)
        cols += c
        vals += v
    ip = np.zeros(n + 1, dtype=np.int32)
    np.cumsum(np.bincount(rows, minlength=n), out=ip[1:])
    ix = np.array(cols, dtype=np.int32)
    hv = np.array(vals, dtype=np.complex128)
    wf0 = unit_states(3, n, seed=21)
    ref = oracle.tbpm_dos(dos_bes, ip, ix, hv, 24, wf0=wf0)
    f2py.set_backend(precision=prec)
    got = f2py.tbpm_dos_states(dos_bes, ip, ix, hv, wf0, 24, 128, 1e-9)
    assert rel_err(got, ref) < tol


@pytest.mark.parametrize("n_states", [4, 3])
def test_dos_fp32_error_bounds(graphene_small, dos_bes, n_states):
    ip, ix, hv = _csr(graphene_small)
    wf0 = unit_states(n_states, ip.size - 1, seed=13)
    f2py.set_backend(precision="fp32")
    got = f2py.tbpm_dos_states(dos_bes, ip, ix, hv, wf0, 64, 32, 1e-9)
    ref = oracle.tbpm_dos(dos_bes, ip, ix, hv, 64, wf0=wf0)
    assert rel_err(got, ref) < 2e-5


def test_session_matches_driver(graphene_small, dos_bes):
    ip, ix, hv = _csr(graphene_small)
    n = ip.size - 1
    ctx = f2py._ctx()
    ip32, ix32 = ip.astype(np.int32), ix.astype(np.int32)
    ctx.call("tbpm_ham_upload", nat.ptr(ip32), nat.ptr(ix32), nat.ptr(hv), n, hv.size, None,
             None, 9.0)
    bes = np.asarray(dos_bes)
    ctx.call("tbpm_session_dos_begin", nat.ptr(bes), bes.size, 4, 1337, 0, 4, 40)
    ctx.call("tbpm_session_advance", 17)
    ctx.call("tbpm_session_advance", 23)
    corr = np.zeros((41, 4), dtype=np.complex128)
    norms = np.zeros((41, 4))
    import ctypes
    nd = ctypes.c_int(0)
    ctx.call("tbpm_session_read", nat.ptr(corr), nat.ptr(norms), ctypes.byref(nd))
    assert nd.value == 41
    ref = oracle.tbpm_dos(bes, ip, ix, hv, 40, seed=1337, n_samples=4)
    assert rel_err(corr.mean(axis=1), ref) < FP64_TOL
    assert np.allclose(norms, 1.0, atol=1e-12)


def test_solver_drop_in(tmp_path, graphene_small):
    config = tb.Config()
    config.generic["nr_time_steps"] = 32
    config.generic["nr_random_samples"] = 3
    solver = tb.Solver(graphene_small, config, echo_details=False, directory=str(tmp_path),
                       prefix="t")
    corr = solver.calc_corr_dos()
    assert corr.shape == (33,)
    assert (tmp_path / "t.corr_DOS.npy").exists()
    h = graphene_small.build_ham_csr()
    bes = solver._get_bessel_series(solver._get_time_step())
    ref = oracle.tbpm_dos(bes, h.indptr, h.indices, h.data, 32, seed=1337, n_samples=3)
    assert rel_err(corr, ref) < FP64_TOL
    analyzer = tb.Analyzer(graphene_small, config, dimension=2)
    energies, dos = analyzer.calc_dos(corr)
    assert energies.shape == (64,) and abs(np.sum(dos) * (energies[1] - energies[0]) - 1) < 1e-12


@pytest.mark.parametrize("width", [1, 2])
@pytest.mark.parametrize("driver", ["dos", "ac", "dc", "psi_t"])
def test_fp64_values_per_thread_match_oracle(graphene_small, dos_bes, ac_bes, driver, width):
    """FP64 with one complex128 per thread (128-bit accesses) and with two
    (256-bit loads and stores, the default for even block widths): results must
    not depend on it."""
    f2py.set_backend(vector_width=width)
    try:
        if driver == "dos":
            ip, ix, hv = _csr(graphene_small)
            wf0 = unit_states(6, ip.size - 1, seed=12)
            got = f2py.tbpm_dos_states(dos_bes, ip, ix, hv, wf0, 30, 128, 1e-9)
            ref = oracle.tbpm_dos(dos_bes, ip, ix, hv, 30, wf0=wf0)
        elif driver == "ac":
            s = tb.make_graphene_sample(8, 6, disorder=0.6, rescale=9.0, seed=3)
            ip, ix, hv, dx, dy = _dxy(s)
            wf0 = unit_states(2, ip.size - 1, seed=21)
            beta = 9.0 / (tb.KB * 300)
            got = f2py.tbpm_accond_states(ac_bes, beta, 0.0, ip, ix, hv, s.rescale, dx, dy, wf0,
                                          16, 2**15, 1e-12, 128, 1e-9)
            ref = oracle.tbpm_accond(ac_bes, beta, 0.0, ip, ix, hv, s.rescale, dx, dy, 16,
                                     wf0=wf0)
        elif driver == "dc":
            s = tb.make_graphene_sample(8, 6, disorder=0.8, rescale=9.0, seed=9)
            ip, ix, hv, dx, dy = _dxy(s)
            wf0 = unit_states(2, ip.size - 1, seed=31)
            energies, qe = _dc_energies(s, 20, limits=(-2.0, 2.0))
            t_step = 2 * math.pi / s.energy_range
            got = f2py.tbpm_dccond_states(dos_bes, ip, ix, hv, s.rescale, dx, dy, wf0, 20,
                                          t_step, energies, qe, 128, 1e-9)
            ref = oracle.tbpm_dccond(dos_bes, ip, ix, hv, s.rescale, dx, dy, 20, t_step,
                                     energies, qe, wf0=wf0)
            assert rel_err(got[0], ref[0]) < FP64_TOL
            got, ref = got[1], ref[1]
        else:
            ip, ix, hv = _csr(graphene_small)
            psi0 = unit_states(1, ip.size - 1, seed=41)[0]
            got = f2py.tbpm_psi_t(dos_bes, ip, ix, hv, psi0, np.array([0, 3, 11]), 11, 128,
                                  1e-9)
            ref = oracle.tbpm_psi_t(dos_bes, ip, ix, hv, psi0, np.array([0, 3, 11]), 11)
        assert rel_err(got, ref) < FP64_TOL
    finally:
        f2py.set_backend(vector_width=0)


@pytest.mark.parametrize("width", [0, 1, 2])
@pytest.mark.parametrize("driver", ["dos", "ac", "dc"])
def test_fp32_values_per_thread_within_bounds(dos_bes, ac_bes, driver, width):
    """FP32 states with four complex64 per thread (256-bit accesses, the default
    when the block width is a multiple of 4), two, and one: each within the FP32
    bound of the oracle (2e-5 relative over these short runs), whatever the width."""
    s = tb.make_graphene_sample(8, 6, disorder=0.6, rescale=9.0, seed=3)
    ip, ix, hv, dx, dy = _dxy(s)
    n = ip.size - 1
    wf0 = unit_states(4, n, seed=27)
    f2py.set_backend(precision="fp32", vector_width=width)
    try:
        if driver == "dos":
            h = s.build_ham_csr()
            got = f2py.tbpm_dos_states(dos_bes, h.indptr, h.indices, h.data, wf0, 24, 128, 1e-9)
            ref = oracle.tbpm_dos(dos_bes, h.indptr, h.indices, h.data, 24, wf0=wf0)
        elif driver == "ac":
            beta = 9.0 / (tb.KB * 300)
            got = f2py.tbpm_accond_states(ac_bes, beta, 0.0, ip, ix, hv, s.rescale, dx, dy, wf0,
                                          12, 2**15, 1e-12, 128, 1e-9)
            ref = oracle.tbpm_accond(ac_bes, beta, 0.0, ip, ix, hv, s.rescale, dx, dy, 12,
                                     wf0=wf0)
        else:
            energies, qe = _dc_energies(s, 16, limits=(-2.0, 2.0))
            t_step = 2 * math.pi / s.energy_range
            got = f2py.tbpm_dccond_states(dos_bes, ip, ix, hv, s.rescale, dx, dy, wf0, 16,
                                          t_step, energies, qe, 128, 1e-9)[1]
            ref = oracle.tbpm_dccond(dos_bes, ip, ix, hv, s.rescale, dx, dy, 16, t_step,
                                     energies, qe, wf0=wf0)[1]
        assert rel_err(got, ref) < 2e-5
    finally:
        f2py.set_backend(precision="fp64", vector_width=0)


@pytest.mark.parametrize("driver", ["dos", "psi_t"])
def test_nan_initial_state_reports_nan_status(graphene_small, dos_bes, driver):
    """A NaN in an initial state makes every norm NaN: the norm check at
    wfn_chk_step returns TBPM_ERR_NAN (NanError, a NormError) instead of
    stopping the process as the reference's check_norm does."""
    ip, ix, hv = _csr(graphene_small)
    n = ip.size - 1
    wf0 = unit_states(2, n, seed=3)
    wf0[1, 7] = np.nan
    with pytest.raises(nat.NanError, match="NaN or infinite"):
        if driver == "dos":
            f2py.tbpm_dos_states(dos_bes, ip, ix, hv, wf0, 16, 8, 1e-9)
        else:
            f2py.tbpm_psi_t(dos_bes, ip, ix, hv, wf0[1], np.array([0, 4]), 16, 8, 1e-9)
    # the context stays usable
    got = f2py.tbpm_dos_states(dos_bes, ip, ix, hv, wf0[:1], 8, 4, 1e-9)
    assert rel_err(got, oracle.tbpm_dos(dos_bes, ip, ix, hv, 8, wf0=wf0[:1])) < FP64_TOL


def test_bounded_wait_runs_out_reports_timeout_and_context_stays_usable(graphene_small,
                                                                          dos_bes):
    """A device wait on a barrier that nothing completes gives up after its
    bound and the call returns TBPM_ERR_TIMEOUT; the next propagation on the
    same context is correct."""
    ctx = f2py._ctx()
    import time
    t0 = time.perf_counter()
    with pytest.raises(nat.DeviceTimeoutError):
        ctx.call("tbpm_selftest_wait_timeout")
    assert time.perf_counter() - t0 < 30
    ip, ix, hv = _csr(graphene_small)
    wf0 = unit_states(2, ip.size - 1, seed=9)
    got = f2py.tbpm_dos_states(dos_bes, ip, ix, hv, wf0, 8, 4, 1e-9)
    assert rel_err(got, oracle.tbpm_dos(dos_bes, ip, ix, hv, 8, wf0=wf0)) < FP64_TOL
