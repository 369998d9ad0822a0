"""Host-side parity with the reference's Python layer (golden fixtures).

tests/golden/reference_tbplas.npz was produced by tests/golden/make_golden.py
from the reference TBPLaS package itself (Sample builders, Solver parameter
handling, Analyzer).  These tests need no GPU.
"""

import math
import os
import pickle

import numpy as np
import pytest

import tbplas_b200 as tb

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_tbplas.npz")


@pytest.fixture(scope="module")
def g():
    return np.load(GOLDEN)


def _mine(key, g):
    if key == "g4x3":
        s = tb.LatticeSample((4, 3))
    elif key == "g7x5_dis":
        s = tb.LatticeSample((7, 5))
        s.orb_eng = s.orb_eng + g["g7x5_dis/disorder"]
    elif key == "g6x6_vac":
        s = tb.LatticeSample((6, 6), vacancies=g["g6x6_vac/vacancies"])
    elif key.startswith("g6x5_mag"):
        s = tb.LatticeSample((6, 5))
        s.set_magnetic_field(77.06, gauge=int(key[-1]))
    elif key == "g5x4_open":
        s = tb.LatticeSample((5, 4), pbc=(False, False))
    elif key == "g8x8_r10":
        s = tb.LatticeSample((8, 8))
        s.rescale_ham(10.0)
        return s
    s.rescale_ham(9.0)
    return s


SAMPLES = ["g4x3", "g7x5_dis", "g6x6_vac", "g6x5_mag0", "g6x5_mag1", "g6x5_mag2",
           "g5x4_open", "g8x8_r10"]


@pytest.mark.parametrize("key", SAMPLES)
def test_build_ham_csr_matches_reference(g, key):
    s = _mine(key, g)
    h = s.build_ham_csr()
    assert h.indptr.dtype == np.int32 and h.indices.dtype == np.int32
    assert np.array_equal(h.indptr, g[f"{key}/csr_indptr"])
    assert np.array_equal(h.indices, g[f"{key}/csr_indices"])
    ref = g[f"{key}/csr_data"]
    if key.startswith("g6x5_mag"):
        assert np.max(np.abs(h.data - ref)) < 1e-15
    else:
        assert np.array_equal(h.data.view(np.float64), ref.view(np.float64))  # bitwise


@pytest.mark.parametrize("key", SAMPLES)
def test_build_ham_dxy_matches_reference(g, key):
    s = _mine(key, g)
    ip, ix, hop, dx, dy = s.build_ham_dxy()
    assert ip.dtype == np.int64 and ix.dtype == np.int64
    assert np.array_equal(ip, g[f"{key}/dxy_indptr"])
    rip, rix = g[f"{key}/dxy_indptr"], g[f"{key}/dxy_indices"]
    # the reference leaves rows unsorted; compare each row as a set of entries
    for r in range(ip.size - 1):
        a = slice(ip[r], ip[r + 1])
        b = slice(rip[r], rip[r + 1])
        oa, ob = np.argsort(ix[a]), np.argsort(rix[b])
        assert np.array_equal(ix[a][oa], rix[b][ob])
        assert np.max(np.abs(hop[a][oa] - g[f"{key}/dxy_hop"][b][ob]), initial=0) < 1e-15
        assert np.max(np.abs(dx[a][oa] - g[f"{key}/dxy_dx"][b][ob]), initial=0) < 1e-15
        assert np.max(np.abs(dy[a][oa] - g[f"{key}/dxy_dy"][b][ob]), initial=0) < 1e-15


@pytest.mark.parametrize("key", SAMPLES)
def test_sample_properties_match_reference(g, key):
    s = _mine(key, g)
    assert np.max(np.abs(s.orb_pos - g[f"{key}/orb_pos"])) < 1e-15
    assert s.rescale == float(g[f"{key}/rescale"])
    assert s.energy_range == float(g[f"{key}/energy_range"])
    assert abs(s.area_unit_cell - float(g[f"{key}/area_unit_cell"])) < 1e-15
    assert abs(s.volume_unit_cell - float(g[f"{key}/volume_unit_cell"])) < 1e-15
    assert s.nr_orbitals == int(g[f"{key}/nr_orbitals"])
    assert s.extended == float(g[f"{key}/extended"])


def _solver(tmp_path, nt=64):
    s = tb.LatticeSample((7, 5))
    s.rescale_ham(9.0)
    cfg = tb.Config()
    cfg.generic["nr_time_steps"] = nt
    cfg.generic["nr_random_samples"] = 2  # as in make_golden.py
    return tb.Solver(s, cfg, echo_details=False, directory=str(tmp_path), prefix="p"), s, cfg


def test_solver_parameters_match_reference(g, tmp_path):
    solver, s, cfg = _solver(tmp_path)
    t = solver._get_time_step()
    assert t == float(g["solver/time_step"])
    assert np.array_equal(np.array(solver._get_bessel_series(t)), g["solver/bessel_dos"])
    assert np.array_equal(np.array(solver._get_bessel_series(0.5 * t)), g["solver/bessel_ac"])
    assert np.allclose(solver._get_beta_mu_re(), g["solver/beta_mu_re"], rtol=0, atol=0)
    gen = cfg.generic
    vals = [gen['Bessel_max'], gen['Bessel_precision'], gen['beta'], gen['mu'],
            gen['nr_random_samples'], gen['seed'], gen['wfn_check_steps'],
            gen['wfn_check_thr'], gen['nr_Fermi_fft_steps'], gen['Fermi_cheb_precision']]
    assert np.array_equal(np.array(vals, dtype=float), g["config/generic_values"])
    assert (tmp_path / "p.config.pkl").exists()


def test_bessel_max_too_low_raises(tmp_path):
    solver, s, cfg = _solver(tmp_path)
    cfg.generic["Bessel_max"] = 5
    with pytest.raises(ValueError, match="Bessel_max too low"):
        solver._get_bessel_series(solver._get_time_step())


def test_config_legality_and_roundtrip(tmp_path):
    cfg = tb.Config()
    cfg.generic["nr_time_steps"] = 77
    with open(tmp_path / "c.pkl", "wb") as f:
        pickle.dump(cfg, f)
    back = tb.read_config(str(tmp_path / "c.pkl"))
    assert back.generic["nr_time_steps"] == 77
    back.check_params()
    cfg.generic["nr_time_step"] = 3  # typo
    with pytest.raises(ValueError, match="Undefined parameter nr_time_step"):
        cfg.check_params()


def _analyzer(g, spin, tnr, dim=2):
    s = tb.LatticeSample((7, 5))
    s.rescale_ham(9.0)
    cfg = tb.Config()
    cfg.generic["nr_time_steps"] = tnr
    cfg.generic["correct_spin"] = spin
    return tb.Analyzer(s, cfg, dimension=dim)


@pytest.mark.parametrize("spin", [False, True])
def test_analyzer_matches_reference(g, spin):
    p = f"analyzer/spin{int(spin)}/"
    an = _analyzer(g, spin, 64)
    e, d = an.calc_dos(g["solver/corr_dos"])
    assert np.array_equal(e, g[p + "dos_energies"])
    assert np.max(np.abs(d - g[p + "dos"])) < 1e-12 * np.max(np.abs(g[p + "dos"]))
    an = _analyzer(g, spin, 32)
    om, ac = an.calc_ac_cond(g["solver/corr_ac"])
    assert np.array_equal(om, g[p + "ac_omegas"])
    assert np.max(np.abs(ac - g[p + "ac"])) < 1e-10 * np.max(np.abs(g[p + "ac"]))
    en, dc = an.calc_dc_cond(g["solver/corr_dos_dc"], g["solver/corr_dc"])
    assert np.array_equal(en, g[p + "dc_energies"])
    assert np.max(np.abs(dc - g[p + "dc"])) < 1e-10 * np.max(np.abs(g[p + "dc"]))
    tm, dcoef = an.calc_diff_coeff(g["solver/corr_dc"])
    assert np.allclose(tm, g[p + "diff_time"], rtol=1e-15, atol=0)
    assert np.max(np.abs(dcoef - g[p + "diff_coeff"])) < 1e-10 * np.max(np.abs(g[p + "diff_coeff"]))


def test_analyzer_dimension3_and_errors(g):
    # make_golden.py evaluates the 3-D case with correct_spin=True
    an = _analyzer(g, True, 32, dim=3)
    _, ac = an.calc_ac_cond(g["solver/corr_ac"])
    assert np.max(np.abs(ac - g["analyzer/dim3/ac"])) < 1e-10 * np.max(np.abs(g["analyzer/dim3/ac"]))
    with pytest.raises(ValueError):
        _analyzer(g, False, 32, dim=1)
