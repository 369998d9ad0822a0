"""GPU assembly of supercell Hamiltonians (tbpm_supercell_ham / _csr).

Parity targets:
* the reference builder itself (tests/golden/reference_supercell.npz): every
  index, the native entry order of build_ham_dxy, dr, the estimated rescale
  factor and every field-free value must be identical; with a Peierls field
  the factors come from the device sincos, so values are compared to 4e-16
  absolute (|h| <= 1 after rescaling, i.e. a few ulp);
* the numpy oracle (oracle/supercell_oracle.py, itself pinned to the same
  fixtures) on supercells too large for fixtures;
* the host route: a Solver run on a DeviceSample equals the run on the
  host-built CSR of the same sample (same seeds) to 1e-12 relative.
"""

import math
import os

import numpy as np
import pytest

import tbplas_b200 as tb
from tbplas_b200 import _native as nat
from tbplas_b200.fortran import f2py
from oracle.supercell_oracle import SampleOracle, SupercellSpec, sample_from_golden

from conftest import rel_err

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_supercell.npz")
FIELD_TOL = 4e-16


@pytest.fixture(scope="module")
def z():
    return np.load(GOLDEN)


@pytest.fixture(autouse=True)
def _backend():
    f2py.set_backend(precision="fp64", batch=16, device=0, state_kind="exp")
    yield
    f2py.set_backend(precision="fp64", batch=16, state_kind="exp")


def _device_from_golden(z, key):
    field, gauge = z[f"{key}/field"]
    r = float(z[f"{key}/rescale_arg"])
    return tb.DeviceSample(z[f"{key}/lat_vec"], z[f"{key}/origin"], z[f"{key}/orb_pos"],
                           z[f"{key}/orb_eng"], z[f"{key}/hop_ind"], z[f"{key}/hop_eng"],
                           z[f"{key}/dim"], z[f"{key}/pbc"], vac_id_sc=z[f"{key}/vac_id_sc"],
                           orb_eng_sc=z[f"{key}/sc_orb_eng"], b_field=float(field),
                           gauge=int(gauge), rescale=r if r > 0 else None)


def _values_match(a, b, field):
    if a.shape != b.shape:
        return False
    if field:
        return float(np.max(np.abs(a - b), initial=0.0)) <= FIELD_TOL
    return np.array_equal(a, b)


def _cases():
    return [str(k) for k in np.load(GOLDEN)["cases"]]


@pytest.mark.parametrize("key", _cases())
def test_device_csr_matches_reference_builder(z, key):
    s = _device_from_golden(z, key)
    field = float(z[f"{key}/field"][0]) != 0.0
    h = s.download_ham_csr()
    assert np.array_equal(h.indptr, z[f"{key}/csr_indptr"])
    assert np.array_equal(h.indices, z[f"{key}/csr_indices"])
    assert _values_match(h.data, z[f"{key}/csr_data"], field)
    if field:
        assert abs(s.rescale - float(z[f"{key}/rescale"])) <= 1e-14
    else:
        assert s.rescale == float(z[f"{key}/rescale"])


@pytest.mark.parametrize("key", _cases())
def test_device_dxy_matches_reference_builder_in_native_order(z, key):
    s = _device_from_golden(z, key)
    field = float(z[f"{key}/field"][0]) != 0.0
    ip, ix, hop, dx, dy = s.download_ham_dxy()
    assert np.array_equal(ip, z[f"{key}/dxy_indptr"])
    assert np.array_equal(ix, z[f"{key}/dxy_indices"])
    assert _values_match(hop, z[f"{key}/dxy_hop"], field)
    assert np.array_equal(dx, z[f"{key}/dxy_dx"])
    assert np.array_equal(dy, z[f"{key}/dxy_dy"])


def _graphene_spec(nx, ny, pbc, vac):
    lat = tb.LatticeSample((1, 1))
    return SupercellSpec(np.vstack([lat.a1, lat.a2, [0, 0, lat.c]]), np.zeros(3),
                         [[0, 0, 0], [1 / 3., 1 / 3., 0]], [0.0, 0.0],
                         [[0, 0, 0, 0, 1], [1, 0, 0, 1, 0], [0, 1, 0, 1, 0]],
                         [-2.7, -2.7, -2.7], (nx, ny, 1), (pbc, pbc, False), vac)


@pytest.mark.parametrize("field,gauge", [(0.0, 0), (77.06, 0), (120.0, 2)])
def test_large_graphene_matches_oracle(field, gauge):
    """300 x 200 graphene, 1% vacancies, Anderson disorder: the GPU CSR and
    DXY arrays equal the oracle's."""
    d = tb.make_graphene_device_sample(300, 200, disorder=1.0, vacancy_rate=0.01,
                                       b_field=field, gauge=gauge, rescale=None, seed=5)
    spec = _graphene_spec(300, 200, True, d.vac_id_sc)
    o = SampleOracle(spec, d.orb_eng_sc)
    if field:
        o.set_magnetic_field(field, gauge)
    o.rescale_ham(None)
    assert abs(d.rescale - o.rescale) <= (1e-14 if field else 0.0)
    h, ho = d.download_ham_csr(), o.build_ham_csr()
    assert np.array_equal(h.indptr, ho.indptr) and np.array_equal(h.indices, ho.indices)
    assert _values_match(h.data, ho.data, field)
    a, b = d.download_ham_dxy(), o.build_ham_dxy()
    for k in (0, 1, 3, 4):
        assert np.array_equal(a[k], b[k])
    assert _values_match(a[2], b[2], field)


def test_3d_mixed_boundaries_matches_oracle():
    """A 2-orbital 3-D lattice with an inter-orbital term across c, 24x18x12,
    periodic along a and c, open along b, with vacancies and a field."""
    lat = np.diag([0.3, 0.32, 0.35])
    hop_ind = [[1, 0, 0, 0, 0], [0, 1, 0, 0, 0], [0, 0, 1, 0, 0], [1, 0, 0, 1, 1],
               [0, 1, 0, 1, 1], [0, 0, 1, 1, 1], [0, 0, 0, 0, 1], [1, 0, -1, 1, 0]]
    hop_eng = [-1.0, -0.9 + 0.05j, -0.8, -1.0, -0.9 + 0.05j, -0.8, -0.4, 0.2j]
    dim = (24, 18, 12)
    n_full = 24 * 18 * 12 * 2
    rng = np.random.default_rng(11)
    vac = np.sort(rng.choice(n_full, size=97, replace=False))
    eng = rng.uniform(-0.3, 0.3, n_full - vac.size)
    spec = SupercellSpec(lat, [0.01, 0.02, -0.03], [[0, 0, 0], [0.5, 0.25, 0.1]], [0.0, 0.2],
                         hop_ind, hop_eng, dim, (True, False, True), vac)
    o = SampleOracle(spec, eng)
    o.set_magnetic_field(25.0, 2)
    o.rescale_ham(None)
    d = tb.DeviceSample(lat, [0.01, 0.02, -0.03], [[0, 0, 0], [0.5, 0.25, 0.1]], [0.0, 0.2],
                        hop_ind, hop_eng, dim, (True, False, True), vac_id_sc=vac,
                        orb_eng_sc=eng, b_field=25.0, gauge=2)
    h, ho = d.download_ham_csr(), o.build_ham_csr()
    assert np.array_equal(h.indptr, ho.indptr) and np.array_equal(h.indices, ho.indices)
    assert _values_match(h.data, ho.data, True)
    a, b = d.download_ham_dxy(), o.build_ham_dxy()
    for k in (0, 1, 3, 4):
        assert np.array_equal(a[k], b[k])
    assert _values_match(a[2], b[2], True)


def _solver(sample, tmp_path, tnr, name, backend=None):
    cfg = tb.Config()
    cfg.generic["nr_time_steps"] = tnr
    cfg.generic["nr_random_samples"] = 3
    cfg.DC_conductivity["energy_limits"] = (-0.5, 0.5)
    return tb.Solver(sample, cfg, echo_details=False, prefix=name,
                     directory=str(tmp_path), backend=backend)


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("fp32", 1e-5)])
def test_solver_on_device_sample_equals_host_route(tmp_path, prec, tol):
    """DOS, AC and DC through the Solver: device-assembled Hamiltonian vs the
    host-built CSR of the same graphene sample (vacancies, disorder, field)."""
    kw = dict(disorder=1.0, vacancy_rate=0.01, b_field=60.0, seed=9)
    dev = tb.make_graphene_device_sample(48, 40, rescale=9.0, **kw)
    host = tb.make_graphene_sample(48, 40, rescale=9.0, **kw)
    be = {"precision": prec}
    a = _solver(dev, tmp_path, 24, "dev", be)
    b = _solver(host, tmp_path, 24, "host", be)
    assert rel_err(a.calc_corr_dos(), b.calc_corr_dos()) < tol
    assert rel_err(a.calc_corr_ac_cond(), b.calc_corr_ac_cond()) < tol
    da, ca = a.calc_corr_dc_cond()
    db, cb = b.calc_corr_dc_cond()
    assert rel_err(da, db) < tol and rel_err(ca, cb) < tol
    psi0 = np.exp(2j * np.pi * np.random.default_rng(1).random(dev.num_orb))
    assert rel_err(a.calc_psi_t(psi0, [0, 5, 24]), b.calc_psi_t(psi0, [0, 5, 24])) < tol


def test_invalid_supercells_are_rejected():
    lat = np.eye(3) * 0.3
    with pytest.raises(ValueError, match="dimension"):
        tb.DeviceSample(lat, None, [[0, 0, 0]], [0.0], [[2, 0, 0, 0, 0]], [-1.0], (4, 1, 1),
                        (True, False, False), rescale=3.0).download_ham_csr()
    with pytest.raises(ValueError, match="on-site"):
        tb.DeviceSample(lat, None, [[0, 0, 0], [0.5, 0, 0]], [0.0, 0.0],
                        [[0, 0, 0, 1, 1]], [-1.0], (3, 1, 1), (True, False, False),
                        rescale=3.0).download_ham_csr()
    with pytest.raises(ValueError, match="vacancy"):
        tb.DeviceSample(lat, None, [[0, 0, 0]], [0.0], [[1, 0, 0, 0, 0]], [-1.0], (3, 1, 1),
                        (True, False, False), vac_id_sc=[5],
                        rescale=3.0).download_ham_csr()
    with pytest.raises(ValueError, match="orbital index"):
        tb.DeviceSample(lat, None, [[0, 0, 0]], [0.0], [[1, 0, 0, 0, 3]], [-1.0], (3, 1, 1),
                        (True, False, False), rescale=3.0).download_ham_csr()


def test_resident_build_replaces_upload_and_reports_sizes():
    """tbpm_supercell_ham returns the same sizes and rescale as the host copy
    and leaves a Hamiltonian the DOS driver runs on."""
    d = tb.make_graphene_device_sample(64, 64, disorder=0.5, rescale=None, seed=2)
    ctx = nat.get_context(0)
    n, nnz = d.build_ham_csr().indptr.make_resident(ctx)
    h = d.download_ham_csr(ctx)
    assert n == h.shape[0] and nnz == h.nnz
    host = tb.make_graphene_sample(64, 64, disorder=0.5, rescale=None, seed=2)
    assert d.rescale == host.rescale
    bes = [float(v) for v in np.array([0.3, 0.2, 0.1, 0.05])]
    c = f2py.tbpm_dos(bes, d.build_ham_csr().indptr, None, None, 3, 4, 2, "", 0, 128, 1e-9)
    assert c.shape == (5,) and abs(c[0] - 1.0) < 1e-12
