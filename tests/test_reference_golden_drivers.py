"""Host-side parity for the dynamical-polarisation, quasi-eigenstate, Hall and
Haydock paths with the reference's Python layer (no GPU).

tests/golden/reference_drivers.npz was written by
tests/golden/make_golden_drivers.py: the reference Solver driving the CPU
oracle through its f2py layer with injected states, and the reference
Analyzer on those results.  Here the oracle, fed with the parameters this
package's Solver derives, must reproduce the reference Solver's outputs, and
this package's Analyzer must reproduce the reference Analyzer.
"""

import os

import numpy as np
import pytest

import tbplas_b200 as tb
from oracle import oracle

from conftest import rel_err

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_drivers.npz")


@pytest.fixture(scope="module")
def g():
    return np.load(GOLDEN)


def _sample(g):
    s = tb.LatticeSample((8, 7))
    s.orb_eng = s.orb_eng + g["disorder"]
    s.rescale_ham(9.0)
    return s


def _config():
    cfg = tb.Config()
    cfg.generic["nr_time_steps"] = 32
    cfg.generic["nr_random_samples"] = 2
    cfg.dyn_pol["q_points"] = [[1.0, 0.0, 0.0], [0.5, 0.8, 0.0], [0.0, 0.0, 0.0]]
    cfg.dyn_pol["background_dielectric_constant"] = 2.5
    cfg.quasi_eigenstates["energies"] = [-0.3, 0.0, 0.2]
    cfg.dckb["n_kernel"] = 48
    cfg.dckb["ne_integral"] = 128
    cfg.dckb["energies"] = [-0.2, -0.1, 0.0, 0.1, 0.2]
    cfg.LDOS["site_indices"] = [3, 40]
    cfg.LDOS["recursion_depth"] = 30
    cfg.LDOS["delta"] = 0.05
    return cfg


def test_solver_parameters_reproduce_reference_driver_outputs(g, tmp_path):
    s = _sample(g)
    assert np.array_equal(s.orb_pos, g["orb_pos"])
    cfg = _config()
    solver = tb.Solver(s, cfg, echo_details=False, directory=str(tmp_path), prefix="t")
    states = g["states"]
    beta, mu = solver._get_beta_mu_re()
    t = solver._get_time_step()
    bes_half = solver._get_bessel_series(0.5 * t)
    bes = solver._get_bessel_series(t)
    ip, ix, hop, dx, dy = s.build_ham_dxy()
    pos = s.orb_pos
    dp = oracle.tbpm_dyn_pol(bes_half, beta, mu, ip, ix, hop, pos[:, 0], pos[:, 1], pos[:, 2],
                             cfg.dyn_pol["q_points"], 32, wf0=states)
    assert rel_err(dp, g["dyn_pol/corr"]) < 1e-13
    h = s.build_ham_csr()
    qe = oracle.tbpm_eigenstates(bes, h.indptr, h.indices, h.data, 32, t,
                                 cfg.quasi_eigenstates["energies"], wf0=states)
    assert rel_err(qe, g["qe/states"]) < 1e-13
    for d in (1, 2):
        mu_mn = oracle.tbpm_kbdc(ip, ix, hop, s.rescale, dx, dy, 48, d, wf0=states)
        assert rel_err(mu_mn, g[f"hall/mu_mn_dir{d}"]) < 1e-13
    sites = cfg.LDOS["site_indices"]
    en, ldos = oracle.ldos_haydock(sites, 0.05, s.energy_range, h.indptr, h.indices, h.data,
                                   s.rescale, 1337, 30, 32, 2, wf_sites=states[:, sites])
    assert np.array_equal(en, g["haydock/energies"])
    assert rel_err(ldos, g["haydock/ldos"]) < 1e-12


@pytest.mark.parametrize("dim", [2, 3])
def test_analyzer_dyn_pol_and_epsilon_match_reference(g, dim):
    an = tb.Analyzer(_sample(g), _config(), dimension=dim)
    q, om, dp = an.calc_dyn_pol(g["dyn_pol/corr"])
    assert np.array_equal(q, g[f"analyzer/dim{dim}/q_points"])
    assert np.array_equal(om, g[f"analyzer/dim{dim}/omegas"])
    assert rel_err(dp, g[f"analyzer/dim{dim}/dyn_pol"]) < 1e-12
    eps = an.calc_epsilon(g[f"analyzer/dim{dim}/dyn_pol"])
    assert rel_err(eps, g[f"analyzer/dim{dim}/epsilon"]) < 1e-14


def test_analyzer_epsilon_q0_matches_reference(g):
    an = tb.Analyzer(_sample(g), _config(), dimension=3)
    eps = an.calc_epsilon_q0(g["analyzer/eps_q0/omegas"], g["analyzer/eps_q0/ac"])
    assert rel_err(eps, g["analyzer/eps_q0/eps"]) < 1e-15
    with pytest.raises(ValueError):
        tb.Analyzer(_sample(g), _config(), dimension=2).calc_epsilon_q0(
            g["analyzer/eps_q0/omegas"], g["analyzer/eps_q0/ac"])


def test_hall_trace_oracle_matches_reference(g):
    """The oracle's cond_from_trace times the Analyzer prefactor reproduces
    the reference's calc_hall_cond (whose trace ran on the same oracle)."""
    s = _sample(g)
    cfg = _config()
    from math import pi
    raw = oracle.cond_from_trace(g["hall/mu_mn_dir2"], cfg.dckb["energies"], s.rescale,
                                 cfg.generic["beta"], 128)
    pref = 16 * s.nr_orbitals / (pi * s.energy_range ** 2) / s.area_unit_cell
    assert rel_err(raw * pref, g["analyzer/dim2/hall_h_bar"]) < 1e-14


def test_device_sample_positions_match_reference(g):
    d = tb.make_graphene_device_sample(8, 7, rescale=9.0)
    assert np.array_equal(d.orb_pos, g["orb_pos"])


def test_recorded_reference_solver_calls_replay_on_the_oracle():
    """tests/golden/reference_calls.npz (the reference Solver's own f2py calls,
    see make_golden_calls.py) replays through the oracle's f2py-compatible
    shim to the recorded results: the fixture and the oracle agree, so the GPU
    replay of the same calls checks the drop-in against the oracle."""
    calls_path = os.path.join(os.path.dirname(__file__), "golden", "reference_calls.npz")
    gc = np.load(calls_path)
    shim = oracle.F2pyShim()
    for k, name in enumerate(gc["calls"]):
        args = []
        for i, kind in enumerate(gc[f"call{k}/kinds"]):
            v = gc[f"call{k}/arg{i}"]
            args.append(v if kind == "array" else v.tolist() if kind == "list" else
                        str(v) if kind == "str" else int(v) if kind == "int" else float(v))
        got = getattr(shim, str(name))(*args)
        got = got if isinstance(got, tuple) else (got,)
        for j in range(int(gc[f"call{k}/n_results"])):
            assert np.array_equal(got[j], gc[f"call{k}/result{j}"]), (name, j)
