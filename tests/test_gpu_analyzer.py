"""The Analyzer's transforms on the GPU (tbpm_trig_sums, tbpm_trig_cumtrapz).

calc_ac_cond, calc_dyn_pol, calc_dc_cond and calc_diff_coeff with the device
sums must reproduce (1) the reference Analyzer's own outputs recorded in the
golden fixtures (tests/golden/reference_tbplas.npz, reference_drivers.npz,
generated from the reference package), to the tolerances the host tests use,
and (2) this package's numpy evaluation of the same formulas at the sizes
where the O(tnr^2) sums matter (tnr = 2048), to a relative 1e-10 of the
largest value (cos / sin of the device and of numpy differ in the last bit).
"""

import os

import numpy as np
import pytest

import tbplas_b200 as tb

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(__file__)


def _rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / np.max(np.abs(b)))


@pytest.fixture(scope="module")
def g():
    return np.load(os.path.join(HERE, "golden", "reference_tbplas.npz"))


@pytest.fixture(scope="module")
def gd():
    return np.load(os.path.join(HERE, "golden", "reference_drivers.npz"))


def _analyzer(spin, tnr, dim=2):
    s = tb.LatticeSample((7, 5))
    s.rescale_ham(9.0)
    cfg = tb.Config()
    cfg.generic["nr_time_steps"] = tnr
    cfg.generic["correct_spin"] = spin
    return tb.Analyzer(s, cfg, dimension=dim, backend="gpu")


@pytest.mark.parametrize("spin", [False, True])
def test_device_analyzer_matches_reference_outputs(g, spin):
    p = f"analyzer/spin{int(spin)}/"
    an = _analyzer(spin, 32)
    om, ac = an.calc_ac_cond(g["solver/corr_ac"])
    assert np.array_equal(om, g[p + "ac_omegas"])
    assert _rel(ac, g[p + "ac"]) < 1e-10
    en, dc = an.calc_dc_cond(g["solver/corr_dos_dc"], g["solver/corr_dc"])
    assert np.array_equal(en, g[p + "dc_energies"])
    assert _rel(dc, g[p + "dc"]) < 1e-10
    tm, dcoef = an.calc_diff_coeff(g["solver/corr_dc"])
    assert _rel(dcoef, g[p + "diff_coeff"]) < 1e-10


@pytest.mark.parametrize("dim", [2, 3])
def test_device_dyn_pol_matches_reference_outputs(gd, dim):
    s = tb.LatticeSample((8, 7))
    s.orb_eng = s.orb_eng + gd["disorder"]
    s.rescale_ham(9.0)
    cfg = tb.Config()
    cfg.generic["nr_time_steps"] = 32
    cfg.generic["nr_random_samples"] = 2
    cfg.dyn_pol["q_points"] = [[1.0, 0.0, 0.0], [0.5, 0.8, 0.0], [0.0, 0.0, 0.0]]
    cfg.dyn_pol["background_dielectric_constant"] = 2.5
    an = tb.Analyzer(s, cfg, dimension=dim, backend="gpu")
    _, _, dp = an.calc_dyn_pol(gd["dyn_pol/corr"])
    assert _rel(dp, gd[f"analyzer/dim{dim}/dyn_pol"]) < 1e-12


def test_device_and_host_transforms_agree_at_2048_steps():
    tnr = 2048
    rng = np.random.default_rng(7)
    s = tb.LatticeSample((7, 5))
    s.rescale_ham(9.0)
    cfg = tb.Config()
    cfg.generic["nr_time_steps"] = tnr
    cfg.DC_conductivity["energy_limits"] = (-1.0, 1.0)
    cfg.dyn_pol["q_points"] = [[1.0, 0.0, 0.0], [0.2, 0.3, 0.0]]
    decay = np.exp(-np.arange(tnr) / 600.0)
    corr_ac = (rng.standard_normal((4, tnr)) + 1j * rng.standard_normal((4, tnr))) * decay
    corr_dp = rng.standard_normal((2, tnr)) * decay
    corr_dos = np.exp(-1j * 0.3 * np.arange(tnr)) * decay
    corr_dc = (rng.standard_normal((2, 2 * tnr, tnr)) +
               1j * rng.standard_normal((2, 2 * tnr, tnr))) * decay
    dev = tb.Analyzer(s, cfg, dimension=2, backend="gpu")
    host = tb.Analyzer(s, cfg, dimension=2, backend="host")
    assert _rel(dev.calc_ac_cond(corr_ac)[1], host.calc_ac_cond(corr_ac)[1]) < 1e-10
    assert _rel(dev.calc_dyn_pol(corr_dp)[2], host.calc_dyn_pol(corr_dp)[2]) < 1e-10
    en_d, dc_d = dev.calc_dc_cond(corr_dos, corr_dc)
    en_h, dc_h = host.calc_dc_cond(corr_dos, corr_dc)
    assert en_d.size > 100 and np.array_equal(en_d, en_h)
    assert _rel(dc_d, dc_h) < 1e-10
    assert _rel(dev.calc_diff_coeff(corr_dc)[1], host.calc_diff_coeff(corr_dc)[1]) < 1e-10
