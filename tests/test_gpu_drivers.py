"""GPU parity of tbpm_dyn_pol, tbpm_eigenstates, tbpm_kbdc, the Haydock
recursion and cond_from_trace against the CPU oracle (identical inputs).

Tolerances: FP64 results must match the oracle to a relative 1e-10 (max
|diff| / max |oracle|); FP32-state results to the stated looser bounds.
"""

import math

import numpy as np
import pytest

import tbplas_b200 as tb
from tbplas_b200.fortran import f2py
from oracle import oracle

from conftest import bessel_series, rel_err, unit_states

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10


@pytest.fixture(autouse=True)
def _fp64_backend():
    f2py.set_backend(precision="fp64", batch=16, device=0, state_kind="exp", use_graphs=True)
    yield
    f2py.set_backend(precision="fp64", batch=16, state_kind="exp", use_graphs=True)


@pytest.fixture(scope="module")
def sample():
    s = tb.make_graphene_sample(16, 12, disorder=1.0, rescale=9.0, seed=21)
    s.set_magnetic_field(30.0)
    return s


def _beta_mu(s):
    return 1.0 / (tb.KB * 300) * s.rescale, 0.1 / s.rescale


@pytest.mark.parametrize("batch,n_q", [(16, 3), (4, 17)])
def test_dyn_pol_matches_oracle(sample, batch, n_q):
    """q-points shared by one propagated psi2 block; the second case needs
    several q-chunks (17 q-points at 4 states per batch)."""
    f2py.set_backend(batch=batch)
    h = sample.build_ham_csr()
    pos = sample.orb_pos
    rng = np.random.default_rng(3)
    q = rng.uniform(-3, 3, (n_q, 3))
    q[:, 2] = 0.0
    wf = unit_states(5, h.shape[0], seed=4)
    beta, mu = _beta_mu(sample)
    bes = bessel_series(math.pi / 2)
    gpu = f2py.tbpm_dyn_pol_states(bes, beta, mu, h.indptr, h.indices, h.data, pos[:, 0],
                                   pos[:, 1], pos[:, 2], q, wf, 30, 2**15, 1e-12, 128, 1e-9)
    ref = oracle.tbpm_dyn_pol(bes, beta, mu, h.indptr, h.indices, h.data, pos[:, 0],
                              pos[:, 1], pos[:, 2], q, 30, wf0=wf)
    assert gpu.shape == (n_q, 30) and gpu.flags.f_contiguous
    assert rel_err(gpu, ref) < FP64_TOL


def test_dyn_pol_seeded_states_follow_the_seed_rule(sample):
    h = sample.build_ham_csr()
    ip, ix, hop, dx, dy = sample.build_ham_dxy()
    pos = sample.orb_pos
    q = [[1.0, 0.5, 0.0]]
    beta, mu = _beta_mu(sample)
    bes = bessel_series(math.pi / 2)
    got = f2py.tbpm_dyn_pol(bes, beta, mu, ip, ix, hop, sample.rescale, dx, dy, pos[:, 0],
                            pos[:, 1], pos[:, 2], 7, 12, 3, 2**15, 1e-12, q, "", 1, 128, 1e-9)
    wf = f2py.random_states(h.shape[0], 7, 3, rank=1, n_ran_samples=3)
    ref = oracle.tbpm_dyn_pol(bes, beta, mu, ip, ix, hop, pos[:, 0], pos[:, 1], pos[:, 2], q,
                              12, wf0=wf)
    assert rel_err(got, ref) < FP64_TOL


def test_dyn_pol_fp32_error_bound(sample):
    h = sample.build_ham_csr()
    pos = sample.orb_pos
    q = [[1.3, 0.2, 0.0], [0.0, 2.0, 0.0]]
    wf = unit_states(4, h.shape[0], seed=5)
    beta, mu = _beta_mu(sample)
    bes = bessel_series(math.pi / 2)
    ref = oracle.tbpm_dyn_pol(bes, beta, mu, h.indptr, h.indices, h.data, pos[:, 0], pos[:, 1],
                              pos[:, 2], q, 24, wf0=wf)
    f2py.set_backend(precision="fp32")
    gpu = f2py.tbpm_dyn_pol_states(bes, beta, mu, h.indptr, h.indices, h.data, pos[:, 0],
                                   pos[:, 1], pos[:, 2], q, wf, 24, 2**15, 1e-12, 128, 1e-9)
    assert rel_err(gpu, ref) < 2e-5


@pytest.mark.parametrize("prec,tol", [("fp64", FP64_TOL), ("fp32", 2e-5)])
def test_eigenstates_match_oracle(sample, prec, tol):
    h = sample.build_ham_csr()
    wf = unit_states(3, h.shape[0], seed=6)
    t_step = 2 * math.pi / sample.energy_range
    energies = [-0.5, 0.0, 0.3, 1.1]
    bes = bessel_series(math.pi)
    ref = oracle.tbpm_eigenstates(bes, h.indptr, h.indices, h.data, 40, t_step, energies,
                                  wf0=wf)
    f2py.set_backend(precision=prec)
    gpu = f2py.tbpm_eigenstates_states(bes, h.indptr, h.indices, h.data, wf, 40, t_step,
                                       energies, 128, 1e-9)
    assert gpu.shape == (4, h.shape[0]) and gpu.flags.f_contiguous
    assert rel_err(gpu, ref) < tol
    # each quasi-eigenstate density is normalised: sum_r = 1 per energy
    norm_tol = 1e-9 if prec == "fp64" else 1e-4
    assert np.max(np.abs(gpu.sum(axis=1) - 1.0)) < norm_tol


def test_eigenstates_seeded(sample):
    h = sample.build_ham_csr()
    t_step = 2 * math.pi / sample.energy_range
    bes = bessel_series(math.pi)
    got = f2py.tbpm_eigenstates(bes, h.indptr, h.indices, h.data, 11, 20, 2, t_step, [0.0, 0.4],
                                0, 128, 1e-9)
    wf = f2py.random_states(h.shape[0], 11, 2)
    ref = oracle.tbpm_eigenstates(bes, h.indptr, h.indices, h.data, 20, t_step, [0.0, 0.4],
                                  wf0=wf)
    assert rel_err(got, ref) < FP64_TOL


@pytest.mark.parametrize("direction", [1, 2])
def test_kbdc_matches_oracle(sample, direction):
    """150 moments: more than one 128-column chunk of bra vectors."""
    ip, ix, hop, dx, dy = sample.build_ham_dxy()
    wf = unit_states(2, ip.size - 1, seed=7)
    gpu = f2py.tbpm_kbdc_states(ip, ix, hop, sample.rescale, dx, dy, wf, 150, direction)
    ref = oracle.tbpm_kbdc(ip, ix, hop, sample.rescale, dx, dy, 150, direction, wf0=wf)
    assert gpu.shape == (150, 150) and gpu.flags.f_contiguous
    assert rel_err(gpu, ref) < FP64_TOL


def test_kbdc_seeded_and_fp32(sample):
    ip, ix, hop, dx, dy = sample.build_ham_dxy()
    got = f2py.tbpm_kbdc(5, ip, ix, hop, sample.rescale, dx, dy, 2, 40, 1, 0)
    wf = f2py.random_states(ip.size - 1, 5, 2)
    ref = oracle.tbpm_kbdc(ip, ix, hop, sample.rescale, dx, dy, 40, 1, wf0=wf)
    assert rel_err(got, ref) < FP64_TOL
    f2py.set_backend(precision="fp32")
    got32 = f2py.tbpm_kbdc_states(ip, ix, hop, sample.rescale, dx, dy, wf, 40, 1)
    assert rel_err(got32, ref) < 1e-4


def test_haydock_matches_oracle(sample):
    h = sample.build_ham_csr()
    sites = [0, 57, 101]
    w = unit_states(2, 3, seed=8)
    a, b = f2py.haydock_coef(sites, h.indptr, h.indices, h.data, sample.rescale, 60, w)
    ra, rb = oracle.haydock_coef(sites, h.indptr, h.indices, h.data, sample.rescale, 60,
                                 wf_sites=w)
    assert rel_err(a, ra) < FP64_TOL and rel_err(b, rb) < FP64_TOL
    en, ldos = f2py.ldos_haydock(sites, 0.05, sample.energy_range, h.indptr, h.indices, h.data,
                                 sample.rescale, 3, 60, 100, 2, "")
    ws = f2py.random_states(3, 3, 2)
    ren, rldos = oracle.ldos_haydock(sites, 0.05, sample.energy_range, h.indptr, h.indices,
                                     h.data, sample.rescale, 3, 60, 100, 2, wf_sites=ws)
    assert np.array_equal(en, ren)
    assert rel_err(ldos, rldos) < 1e-9


def test_cond_from_trace_matches_oracle(sample):
    ip, ix, hop, dx, dy = sample.build_ham_dxy()
    wf = unit_states(1, ip.size - 1, seed=9)
    mu_mn = oracle.tbpm_kbdc(ip, ix, hop, sample.rescale, dx, dy, 64, 2, wf0=wf)
    mus = np.linspace(-0.3, 0.3, 7)
    beta = 1.0 / (tb.KB * 300)
    gpu = f2py.cond_from_trace(mu_mn, mus, sample.rescale, beta, 256, 1e-12, 0)
    ref = oracle.cond_from_trace(mu_mn, mus, sample.rescale, beta, 256)
    assert rel_err(gpu, ref) < FP64_TOL


def _solver(sample, cfg, tmp_path, name):
    return tb.Solver(sample, cfg, echo_details=False, directory=str(tmp_path), prefix=name)


def test_solver_methods_end_to_end(sample, tmp_path):
    """Solver.calc_corr_dyn_pol / calc_quasi_eigenstates / calc_hall_mu /
    calc_ldos_haydock on the GPU equal the oracle fed with the same seeded
    states; their output files are written."""
    cfg = tb.Config()
    cfg.generic["nr_time_steps"] = 20
    cfg.generic["nr_random_samples"] = 3
    cfg.dyn_pol["q_points"] = [[1.0, 0.2, 0.0], [0.3, 1.5, 0.0]]
    cfg.quasi_eigenstates["energies"] = [-0.2, 0.1]
    cfg.dckb["n_kernel"] = 32
    cfg.LDOS["site_indices"] = [5, 9]
    cfg.LDOS["recursion_depth"] = 25
    sv = _solver(sample, cfg, tmp_path, "e2e")
    n = sample.build_ham_csr().shape[0]
    wf = f2py.random_states(n, 1337, 3)
    beta, mu = sv._get_beta_mu_re()
    t = sv._get_time_step()
    ip, ix, hop, dx, dy = sample.build_ham_dxy()
    pos = sample.orb_pos
    dp = sv.calc_corr_dyn_pol()
    ref = oracle.tbpm_dyn_pol(sv._get_bessel_series(0.5 * t), beta, mu, ip, ix, hop,
                              pos[:, 0], pos[:, 1], pos[:, 2], cfg.dyn_pol["q_points"], 20,
                              wf0=wf)
    assert rel_err(dp, ref) < FP64_TOL
    assert (tmp_path / "e2e.corr_dyn_pol.npy").exists()
    h = sample.build_ham_csr()
    qe = sv.calc_quasi_eigenstates(save_data=True)
    ref = oracle.tbpm_eigenstates(sv._get_bessel_series(t), h.indptr, h.indices, h.data, 20, t,
                                  [-0.2, 0.1], wf0=wf)
    assert rel_err(qe, ref) < FP64_TOL
    mu_mn = sv.calc_hall_mu()
    ref = oracle.tbpm_kbdc(ip, ix, hop, sample.rescale, dx, dy, 32, 1, wf0=wf)
    assert rel_err(mu_mn, ref) < FP64_TOL
    en, ldos = sv.calc_ldos_haydock()
    ws = f2py.random_states(2, 1337, 3)
    ren, rldos = oracle.ldos_haydock([5, 9], cfg.LDOS["delta"], sample.energy_range, h.indptr,
                                     h.indices, h.data, sample.rescale, 1337, 25, 20, 3,
                                     wf_sites=ws)
    assert rel_err(ldos, rldos) < 1e-9
    an = tb.Analyzer(sample, cfg, dimension=2)
    q, om, dyn = an.calc_dyn_pol(dp)
    assert dyn.shape == (2, 20)
    e, cond = an.calc_hall_cond(mu_mn)
    assert cond.shape == (len(cfg.dckb["energies"]),) and np.all(np.isfinite(cond))


@pytest.mark.parametrize("dim", [2, 3])
def test_analyzer_hall_cond_matches_reference(dim):
    """calc_hall_cond with the GPU trace against the reference Analyzer's output
    (tests/golden/reference_drivers.npz)."""
    import os
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_drivers.npz"))
    s = tb.LatticeSample((8, 7))
    s.orb_eng = s.orb_eng + g["disorder"]
    s.rescale_ham(9.0)
    cfg = tb.Config()
    cfg.dckb["ne_integral"] = 128
    cfg.dckb["energies"] = [-0.2, -0.1, 0.0, 0.1, 0.2]
    an = tb.Analyzer(s, cfg, dimension=dim)
    for unit in ("h_bar", "h"):
        e, c = an.calc_hall_cond(g["hall/mu_mn_dir2"], unit=unit)
        assert np.array_equal(e, g[f"analyzer/dim{dim}/hall_energies"])
        assert rel_err(c, g[f"analyzer/dim{dim}/hall_{unit}"]) < FP64_TOL


def test_dyn_pol_on_device_sample_equals_host_route(tmp_path):
    kw = dict(disorder=0.8, vacancy_rate=0.01, seed=13)
    dev = tb.make_graphene_device_sample(30, 24, rescale=9.0, **kw)
    host = tb.make_graphene_sample(30, 24, rescale=9.0, **kw)
    assert np.array_equal(dev.orb_pos, host.orb_pos)
    cfg = tb.Config()
    cfg.generic["nr_time_steps"] = 16
    cfg.generic["nr_random_samples"] = 2
    cfg.dyn_pol["q_points"] = [[0.7, 0.7, 0.0]]
    a = _solver(dev, cfg, tmp_path, "dev").calc_corr_dyn_pol()
    b = _solver(host, cfg, tmp_path, "host").calc_corr_dyn_pol()
    assert rel_err(a, b) < 1e-12
