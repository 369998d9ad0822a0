"""Checkpoint / resume of DOS runs (tbplas_b200.checkpoint).

An interruption is made on the host: the checkpoint callback raises, as a
process that is stopped between two checkpoints would.  The resumed run must
return what an uninterrupted tbpm_dos returns, bit for bit in FP64.
"""

import math
import os

import numpy as np
import pytest

import tbplas_b200 as tb
from tbplas_b200.checkpoint import dos_checkpointed
from tbplas_b200.fortran import f2py

from conftest import bessel_series, rel_err

pytestmark = pytest.mark.gpu


class Stop(Exception):
    pass


@pytest.fixture(autouse=True)
def _backend():
    f2py.set_backend(precision="fp64", batch=2, device=0, state_kind="exp")
    yield
    f2py.set_backend(precision="fp64", batch=16, state_kind="exp")


@pytest.fixture(scope="module")
def ham():
    s = tb.make_graphene_sample(24, 20, disorder=1.0, rescale=9.0, seed=3)
    return s.build_ham_csr()


def _stop_at(s0_stop, done_stop):
    def cb(s0, done):
        if s0 == s0_stop and done == done_stop:
            raise Stop()
    return cb


@pytest.mark.parametrize("stop", [(2, 21), (4, 0), (0, 11)])
def test_resume_reproduces_uninterrupted_run(tmp_path, ham, stop):
    bes = bessel_series(math.pi)
    ref = f2py.tbpm_dos(bes, ham.indptr, ham.indices, ham.data, 5, 40, 5, "", 0, 16, 1e-9)
    path = str(tmp_path / "ck.npz")
    with pytest.raises(Stop):
        dos_checkpointed(bes, ham.indptr, ham.indices, ham.data, 5, 40, 5, 0, 16, 1e-9, path,
                         every=10, on_checkpoint=_stop_at(*stop))
    assert os.path.exists(path)
    got = dos_checkpointed(bes, ham.indptr, ham.indices, ham.data, 5, 40, 5, 0, 16, 1e-9, path,
                           every=10)
    assert np.array_equal(got, ref)
    assert not os.path.exists(path)


def test_checkpoint_of_other_inputs_is_ignored(tmp_path, ham):
    bes = bessel_series(math.pi)
    path = str(tmp_path / "ck.npz")
    with pytest.raises(Stop):
        dos_checkpointed(bes, ham.indptr, ham.indices, ham.data, 5, 30, 3, 0, 16, 1e-9, path,
                         every=7, on_checkpoint=_stop_at(0, 15))
    got = dos_checkpointed(bes, ham.indptr, ham.indices, ham.data, 6, 30, 3, 0, 16, 1e-9, path,
                           every=7)
    ref = f2py.tbpm_dos(bes, ham.indptr, ham.indices, ham.data, 6, 30, 3, "", 0, 16, 1e-9)
    assert np.array_equal(got, ref)


def test_fp32_resume_and_solver_checkpoint(tmp_path, ham):
    bes = bessel_series(math.pi)
    f2py.set_backend(precision="fp32")
    path = str(tmp_path / "ck32.npz")
    plain = dos_checkpointed(bes, ham.indptr, ham.indices, ham.data, 9, 24, 3, 0, 16, 1e-9,
                             path, every=5)
    with pytest.raises(Stop):
        dos_checkpointed(bes, ham.indptr, ham.indices, ham.data, 9, 24, 3, 0, 16, 1e-9, path,
                         every=5, on_checkpoint=_stop_at(2, 11))
    got = dos_checkpointed(bes, ham.indptr, ham.indices, ham.data, 9, 24, 3, 0, 16, 1e-9,
                           path, every=5)
    assert np.array_equal(got, plain)
    ref32 = f2py.tbpm_dos(bes, ham.indptr, ham.indices, ham.data, 9, 24, 3, "", 0, 16, 1e-9)
    assert rel_err(got, ref32) < 1e-6
    f2py.set_backend(precision="fp64")
    s = tb.make_graphene_sample(24, 20, disorder=1.0, rescale=9.0, seed=3)
    cfg = tb.Config()
    cfg.generic["nr_time_steps"] = 30
    cfg.generic["nr_random_samples"] = 3
    a = tb.Solver(s, cfg, echo_details=False, directory=str(tmp_path), prefix="a",
                  checkpoint={"path": str(tmp_path / "solver.npz"), "every": 8})
    b = tb.Solver(s, cfg, echo_details=False, directory=str(tmp_path), prefix="b")
    assert np.array_equal(a.calc_corr_dos(), b.calc_corr_dos())


@pytest.mark.parametrize("stop_after", [2, 4])
def test_dc_resume_reproduces_uninterrupted_run(tmp_path, stop_after):
    """DC (tbpm_dccond) checkpointed between parts of two states: stopped after
    the first or second part and resumed, the result is bit-identical to the
    same run without interruption, and equals one tbpm_dccond call to the
    FP64 bar."""
    from tbplas_b200.checkpoint import dc_checkpointed
    s = tb.make_graphene_sample(10, 8, disorder=0.8, rescale=9.0, seed=5)
    ip, ix, hv, dx, dy = s.build_ham_dxy()
    tnr = 24
    en_range = s.energy_range
    energies = np.array([0.5 * i * en_range / tnr - en_range / 2. for i in range(2 * tnr)])
    sel = np.where((energies >= -2.0) & (energies <= 2.0))[0]
    bes = bessel_series(math.pi)
    t_step = 2 * math.pi / en_range
    args = (bes, ip, ix, hv, s.rescale, dx, dy, 1337, tnr, 5, t_step, energies, sel, 0, 16,
            1e-9)
    whole = dc_checkpointed(*args, str(tmp_path / "whole.npz"), states_per_part=2)
    path = str(tmp_path / "dc.npz")

    def cb(done):
        if done == stop_after:
            raise Stop()

    with pytest.raises(Stop):
        dc_checkpointed(*args, path, states_per_part=2, on_checkpoint=cb)
    assert os.path.exists(path)
    got = dc_checkpointed(*args, path, states_per_part=2)
    assert not os.path.exists(path)
    for k in (0, 1):
        assert np.array_equal(got[k], whole[k])
    ref = f2py.tbpm_dccond(bes, 0.0, 0.0, ip, ix, hv, s.rescale, dx, dy, 1337, tnr, 5, t_step,
                           energies, sel, "", "", 0, 16, 1e-9)
    for k in (0, 1):
        assert rel_err(got[k], ref[k]) < 1e-12
