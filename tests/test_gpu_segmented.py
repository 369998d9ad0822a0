"""Batched uneven realisations (block-diagonal packing) against the oracle.

Every realisation of the packed batch must give the same per-state DOS
correlation as a separate oracle run on that realisation alone with the same
random states (the Philox stream of realisation k, state s has
iseed = seed*(k*n_states + s + 1) and counts rows from the start of the
realisation).
"""

import math

import numpy as np
import pytest

import tbplas_b200 as tb
from tbplas_b200.fortran import f2py
from oracle import oracle

from conftest import bessel_series, rel_err

pytestmark = pytest.mark.gpu


def _realisations():
    specs = [(6, 5, 0.0, 0.0), (9, 7, 1.5, 0.02), (5, 8, 3.0, 0.01), (12, 4, 0.7, 0.0)]
    return [tb.make_graphene_sample(nx, ny, disorder=w, vacancy_rate=v, rescale=10.0, seed=41 + i)
            for i, (nx, ny, w, v) in enumerate(specs)]


@pytest.mark.parametrize("ns", [3, 4])
@pytest.mark.parametrize("prec,tol", [("fp64", 1e-10), ("fp32", 3e-5)])
def test_segmented_matches_separate_oracle_runs(prec, tol, ns):
    samples = _realisations()
    packed = tb.pack_samples(samples)
    tnr, seed = 40, 1337
    bes = bessel_series(2 * math.pi / packed.energy_range * packed.rescale)
    f2py.set_backend(precision=prec, device=0)
    try:
        corr, per = f2py.tbpm_dos_segmented(bes, packed.indptr, packed.indices, packed.data,
                                            packed.offsets, ns, seed, tnr, per_state=True)
    finally:
        f2py.set_backend(precision="fp64")
    assert corr.shape == (len(samples), tnr + 1)
    for k, s in enumerate(samples):
        h = s.build_ham_csr()
        for b in range(ns):
            iseed = seed * (k * ns + b + 1)
            ref = oracle.tbpm_dos(bes, h.indptr, h.indices, h.data, tnr, seed=iseed,
                                  n_samples=1)
            assert rel_err(per[k, b], ref) < tol
        assert np.allclose(corr[k], per[k].mean(axis=0), rtol=0, atol=1e-15)
        # <wf0|wf0> = 1 up to the rounding of the stored states
        assert abs(corr[k, 0] - 1.0) < (1e-12 if prec == "fp64" else 1e-6)


def test_segmented_rejects_bad_offsets():
    samples = _realisations()[:2]
    packed = tb.pack_samples(samples)
    bes = bessel_series(math.pi)
    bad = packed.offsets.copy()
    bad[-1] += 1
    with pytest.raises(ValueError):
        f2py.tbpm_dos_segmented(bes, packed.indptr, packed.indices, packed.data, bad, 2, 1, 4)
