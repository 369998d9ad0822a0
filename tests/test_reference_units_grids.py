"""CPU part of the full-scale check against the reference's own curves
(tests/golden/reference_units.npz, see test_gpu_reference_units.py): the
frequency grids of Analyzer.calc_ac_cond and calc_dyn_pol depend only on the
configuration and the cell, so for the reference's unit configurations
(4096 x 4096 graphene, a = 0.142 nm, t = 3.0 eV, rescale 9, 1024 steps) they
must equal the reference's grids exactly.  No propagation is needed: the
correlations passed in are zeros.
"""

import os

import numpy as np
import pytest

import tbplas_b200 as tb
from tbplas_b200.supercell import DeviceSample

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_units.npz")
A = 0.142
T = 3.0


@pytest.fixture(scope="module")
def sample():
    lat = A * np.sqrt(3)
    g = np.pi / 3
    lat_vec = np.array([[lat, 0.0, 0.0], [lat * np.cos(g), lat * np.sin(g), 0.0],
                        [0.0, 0.0, 1.0]])
    lat_vec[np.abs(lat_vec) < 1e-15] = 0.0
    hop_ind = np.array([[0, 0, 0, 0, 1], [1, 0, 0, 1, 0], [0, 1, 0, 1, 0]], dtype=np.int32)
    return DeviceSample(lat_vec, np.zeros(3), [[0.0, 0.0, 0.0], [1 / 3., 1 / 3., 0.0]],
                        [0.0, 0.0], hop_ind, np.full(3, T, dtype=np.complex128),
                        (4096, 4096, 1), (True, True, False), rescale=9.0)


def _config(q=None, spin=False):
    cfg = tb.Config()
    cfg.generic["nr_random_samples"] = 1
    cfg.generic["nr_time_steps"] = 1024
    cfg.generic["correct_spin"] = spin
    if q is not None:
        cfg.dyn_pol["q_points"] = q
    return cfg


def test_ac_frequency_grid_equals_reference(sample):
    gold = np.load(GOLDEN)
    cfg = _config(spin=True)
    om, ac = tb.Analyzer(sample, cfg, dimension=2).calc_ac_cond(np.zeros((4, 1024), complex))
    assert np.array_equal(om, gold["omegas_ac"])
    assert ac.shape == gold["ac"].shape


@pytest.mark.parametrize("which,q", [
    ("dp", 1 / A * np.array([[0.86602540, 0.5, 0.0]])),
    ("eps", np.array([[4.122280922013927, 2.38, 0.0]])),
])
def test_dyn_pol_frequency_grids_equal_reference(sample, which, q):
    gold = np.load(GOLDEN)
    cfg = _config(q=q)
    an = tb.Analyzer(sample, cfg, dimension=2)
    _, om, dp = an.calc_dyn_pol(np.zeros((1, 1024)))
    assert np.array_equal(om, gold["omegas_" + which])
    assert dp.shape == gold[which].shape
