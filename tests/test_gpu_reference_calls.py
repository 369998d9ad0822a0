"""The reference Solver's own calls, replayed through the drop-in f2py module.

tests/golden/reference_calls.npz holds every call the reference's Solver
(tbplas/tbpm/solver.py) made into its f2py core while running calc_corr_dos,
calc_corr_ac_cond, calc_corr_dc_cond, calc_corr_dyn_pol and calc_psi_t on a
disordered 9 x 7 graphene sample, recorded by tests/golden/make_golden_calls.py
in a container that held the reference package: the positional arguments as
the reference builds them (a list of Bessel coefficients, int32 or int64 CSR
arrays, output file names, scalars) and the CPU oracle's result.  Each call is
replayed, argument for argument, through tbplas_b200.fortran.f2py, which the
reference binds as `from ..fortran import f2py` when this package replaces its
Fortran core; the GPU results must equal the oracle's to a relative 1e-10.
"""

import os

import numpy as np
import pytest

from tbplas_b200.fortran import f2py

from conftest import rel_err

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_calls.npz")


@pytest.fixture(scope="module")
def g():
    return np.load(GOLDEN)


def _args(g, k):
    out = []
    for i, kind in enumerate(g[f"call{k}/kinds"]):
        v = g[f"call{k}/arg{i}"]
        if kind == "array":
            out.append(v)
        elif kind == "list":
            out.append(v.tolist())
        elif kind == "str":
            out.append(str(v))
        elif kind == "int":
            out.append(int(v))
        else:
            out.append(float(v))
    return out


@pytest.fixture(autouse=True)
def _backend():
    f2py.set_backend(precision="fp64", batch=16, device=0, state_kind="exp", use_graphs=True)
    yield


@pytest.mark.parametrize("name", ["tbpm_dos", "tbpm_accond", "tbpm_dccond", "tbpm_dyn_pol",
                                  "tbpm_psi_t"])
def test_reference_solver_call_replays_through_the_drop_in(g, name):
    calls = list(g["calls"])
    assert name in calls
    k = calls.index(name)
    got = getattr(f2py, name)(*_args(g, k))
    n_res = int(g[f"call{k}/n_results"])
    got = got if n_res > 1 else (got,)
    assert len(got) == n_res
    for j in range(n_res):
        ref = g[f"call{k}/result{j}"]
        assert got[j].shape == ref.shape
        assert rel_err(got[j], ref) < 1e-10
