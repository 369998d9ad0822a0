"""The reference's end-to-end TBPM test (tests/test_graph.py:36-101, test_tbpm)
run through this package's Solver and Analyzer.

Same sample (test_graph.py:12-30: 100 x 100 periodic graphene, a = 0.246 nm,
t = 2.7 eV, rescale 9, assembled here on the GPU) and the same Config: 256
time steps, 4 random samples, correct_spin, dyn_pol at q = (1, 0, 0), DC
energy window -0.3..0.3 eV.  The reference test only plots; here every
correlation the Solver returns is compared with the oracle, fed with the
arguments the Solver passed to the f2py layer (captured on the way) and
drawing the same seeded states, to the FP64 bound of 1e-10.  The Analyzer
outputs are checked for their defining properties.
"""

import math

import numpy as np
import pytest

import tbplas_b200 as tb
from tbplas_b200.fortran import f2py
from tbplas_b200.supercell import DeviceSample
from oracle import oracle

from conftest import rel_err

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10


@pytest.fixture(scope="module")
def sample():
    a = 0.246
    vectors = np.array([[0.5 * a, 0.5 * math.sqrt(3) * a, 0.0],
                        [-0.5 * a, 0.5 * math.sqrt(3) * a, 0.0],
                        [0.0, 0.0, 1.0]])
    hop_ind = np.array([[0, 0, 0, 0, 1], [1, 0, 0, 1, 0], [0, 1, 0, 1, 0]], dtype=np.int32)
    return DeviceSample(vectors, np.zeros(3), [[0.0, 0.0, 0.0], [1 / 3., 1 / 3., 0.0]],
                        [0.0, 0.0], hop_ind, np.full(3, 2.7, dtype=np.complex128),
                        (100, 100, 1), (True, True, False), rescale=9.0)


@pytest.fixture(scope="module")
def config():
    cfg = tb.Config()
    cfg.generic["nr_time_steps"] = 256
    cfg.generic["nr_random_samples"] = 4
    cfg.generic["correct_spin"] = True
    cfg.dyn_pol["q_points"] = [[1., 0., 0.]]
    cfg.DC_conductivity["energy_limits"] = (-0.3, 0.3)
    cfg.LDOS["site_indices"] = [0]
    cfg.LDOS["delta"] = 0.1
    cfg.LDOS["recursion_depth"] = 2000
    return cfg


@pytest.fixture()
def captured(monkeypatch):
    """Record the arguments the Solver passes to the f2py layer."""
    calls = {}
    for name in ("tbpm_dos", "tbpm_accond", "tbpm_dyn_pol", "tbpm_dccond"):
        real = getattr(f2py, name)

        def wrap(*args, _real=real, _name=name):
            calls[_name] = args
            return _real(*args)

        monkeypatch.setattr(f2py, name, wrap)
    return calls


def test_reference_tbpm_workflow(sample, config, captured, tmp_path):
    f2py.set_backend(precision="fp64", batch=16, device=0)
    solver = tb.Solver(sample, config, echo_details=False, directory=str(tmp_path), prefix="g")
    solver.save_config()
    analyzer = tb.Analyzer(sample, config)
    h = sample.download_ham_csr()
    ip, ix, hv, dx, dy = sample.download_ham_dxy()
    seed, tnr, ns = config.generic["seed"], 256, 4

    # DOS
    corr_dos = solver.calc_corr_dos()
    bes = captured["tbpm_dos"][0]
    ref = oracle.tbpm_dos(bes, h.indptr, h.indices, h.data, tnr, seed=seed, n_samples=ns)
    assert rel_err(corr_dos, ref) < FP64_TOL
    energies, dos = analyzer.calc_dos(corr_dos)
    # normalised to 1, times 2 for spin (correct_spin, analysis.py:137-139)
    assert abs(np.sum(dos) * (energies[1] - energies[0]) - 2) < 1e-12

    # AC conductivity
    corr_ac = solver.calc_corr_ac_cond()
    a = captured["tbpm_accond"]
    ref = oracle.tbpm_accond(a[0], a[1], a[2], ip, ix, hv, a[6], dx, dy, tnr, seed=seed,
                             n_samples=ns, nr_fermi=a[12], fermi_precision=a[13])
    assert rel_err(corr_ac, ref) < FP64_TOL
    omegas, ac = analyzer.calc_ac_cond(corr_ac)
    assert ac.shape == (4, tnr) and np.all(np.isfinite(ac))

    # dynamical polarisation
    corr_dp = solver.calc_corr_dyn_pol()
    d = captured["tbpm_dyn_pol"]
    pos = sample.orb_pos
    ref = oracle.tbpm_dyn_pol(d[0], d[1], d[2], ip, ix, hv, pos[:, 0], pos[:, 1], pos[:, 2],
                              config.dyn_pol["q_points"], tnr, seed=seed, n_samples=ns,
                              nr_fermi=d[15], fermi_precision=d[16])
    assert rel_err(corr_dp, ref) < FP64_TOL
    q, om_dp, dp = analyzer.calc_dyn_pol(corr_dp)
    assert dp.shape == (1, tnr) and np.all(np.isfinite(dp))

    # DC conductivity
    corr_dos_dc, corr_dc = solver.calc_corr_dc_cond()
    c = captured["tbpm_dccond"]
    rdos, rdc = oracle.tbpm_dccond(c[0], ip, ix, hv, c[6], dx, dy, tnr, c[12], c[13], c[14],
                                   seed=seed, n_samples=ns)
    assert rel_err(corr_dos_dc, rdos) < FP64_TOL
    assert rel_err(corr_dc, rdc) < FP64_TOL
    en_dc, dc = analyzer.calc_dc_cond(corr_dos_dc, corr_dc)
    assert dc.shape == (2, c[14].size) and np.all(np.isfinite(dc))
