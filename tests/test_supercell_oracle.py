"""The numpy supercell oracle against the reference builder's own outputs.

tests/golden/reference_supercell.npz holds, for eleven supercells of five
primitive cells, the inputs of the builder and what the reference Sample
returned (tests/golden/make_golden_supercell.py).  The oracle must reproduce
build_ham_csr and build_ham_dxy exactly (every index, the native entry order
and, without a magnetic field, every value bit for bit).  With a field the
Peierls factors go through cos/sin, whose last bit may differ between libm
builds, so values there are compared to 1e-15 absolute (|h| <= 1).
"""

import os

import numpy as np
import pytest

from oracle.supercell_oracle import sample_from_golden

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_supercell.npz")


@pytest.fixture(scope="module")
def z():
    return np.load(GOLDEN)


def _cases():
    return [str(k) for k in np.load(GOLDEN)["cases"]]


def _same(a, b, field):
    if field:
        return a.shape == b.shape and np.max(np.abs(a - b), initial=0.0) < 1e-15
    return a.shape == b.shape and np.array_equal(a, b)


@pytest.mark.parametrize("key", _cases())
def test_oracle_reproduces_reference_builder(z, key):
    s = sample_from_golden(z, key)
    field = float(z[f"{key}/field"][0]) != 0.0
    assert np.array_equal(s.orb_pos, z[f"{key}/sc_orb_pos"])
    if field:
        assert abs(s.rescale - float(z[f"{key}/rescale"])) < 1e-14
    else:
        assert s.rescale == float(z[f"{key}/rescale"])
    h = s.build_ham_csr()
    assert np.array_equal(h.indptr, z[f"{key}/csr_indptr"])
    assert np.array_equal(h.indices, z[f"{key}/csr_indices"])
    assert _same(h.data, z[f"{key}/csr_data"], field)
    ip, ix, hop, dx, dy = s.build_ham_dxy()
    assert np.array_equal(ip, z[f"{key}/dxy_indptr"])
    assert np.array_equal(ix, z[f"{key}/dxy_indices"])
    assert _same(hop, z[f"{key}/dxy_hop"], field)
    assert np.array_equal(dx, z[f"{key}/dxy_dx"])
    assert np.array_equal(dy, z[f"{key}/dxy_dy"])
