"""Multi-rank host logic on CPU: two gloo ranks (no GPU).

Covers the random-sample decomposition of the reference (Solver._dist_sample,
seed rule seed*(i_sample + rank*n_ran_samples) of tbpm.f90:57), the
all_average collective (parallel.py:175-189) on Fortran-ordered complex
arrays, bcast, and failure detection: a rank that raises before the
collective makes the surviving rank's collective end with an error within the
process-group timeout instead of hanging.  The device compute of each rank is
replaced by the CPU oracle through a module-like stand-in, which is what the
host logic sees of it.
"""

import os
import socket
import sys
from datetime import timedelta

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _init(rank, world, port, timeout_s=30):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    os.environ["RANK"] = str(rank)
    os.environ["WORLD_SIZE"] = str(world)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=timedelta(seconds=timeout_s))
    return dist


def _worker_solver(rank, world, port, outdir, q):
    # one OpenMP thread per rank: two ranks share the host cores, and the oracle's
    # small parallel regions stall on oversubscribed barriers otherwise (torch,
    # imported with this module, has already started the OpenMP runtime)
    os.environ["OMP_NUM_THREADS"] = "1"
    import torch
    torch.set_num_threads(1)
    sys.path.insert(0, ROOT)
    try:
        dist = _init(rank, world, port)
        import tbplas_b200 as tb
        from tbplas_b200.tbpm import solver as solver_mod
        from oracle import oracle

        class CpuStandIn:
            """The f2py entry points the Solver calls, computed by the oracle."""

            def tbpm_dos(self, *a):
                return oracle.F2pyShim().tbpm_dos(*a)

            def set_backend(self, **kw):
                pass

        solver_mod.f2py = CpuStandIn()
        from tbplas_b200.parallel import MPIEnv
        env = MPIEnv(enable_mpi=True)
        x = np.asfortranarray(np.arange(6, dtype=np.complex128).reshape(2, 3) * (rank + 1)
                              + 1j * rank)
        xl = x.copy(order="F")
        avg = env.all_average(xl)
        untouched = bool(np.array_equal(xl, x))  # the local array keeps its values
        b = np.full(4, float(rank))
        env.bcast(b)
        s = tb.make_graphene_sample(6, 6, disorder=0.5, seed=3)
        cfg = tb.Config()
        cfg.generic["nr_time_steps"] = 16
        cfg.generic["nr_random_samples"] = 3
        solver = tb.Solver(s, cfg, enable_mpi=True, echo_details=False,
                           directory=os.path.join(outdir, f"r{rank}"), prefix="m")
        corr = solver.calc_corr_dos()
        q.put((rank, avg, b, corr, cfg.generic["nr_random_samples"], untouched))
        dist.barrier()
        dist.destroy_process_group()
    except Exception as e:  # report instead of hanging the parent
        q.put((rank, "error", repr(e), None, None, None))


def test_two_rank_sample_decomposition(tmp_path):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker_solver, args=(r, 2, port, str(tmp_path), q))
             for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(2):
        r = q.get(timeout=240)
        res[r[0]] = r
    for p in procs:
        p.join(timeout=60)
    for r in (0, 1):
        assert not isinstance(res[r][1], str), res[r][2]
    x0 = np.arange(6, dtype=np.complex128).reshape(2, 3)
    expect = (x0 * 1 + x0 * 2 + 1j) / 2
    for r in (0, 1):
        _, avg, b, corr, nrs, untouched = res[r]
        assert np.allclose(avg, expect)
        assert untouched
        assert np.all(b == 0.0)
        assert nrs == 4  # padded to a multiple of the number of ranks
    sys.path.insert(0, ROOT)
    import tbplas_b200 as tb
    from oracle import oracle
    import math
    s = tb.make_graphene_sample(6, 6, disorder=0.5, seed=3)
    h = s.build_ham_csr()
    from conftest import bessel_series
    ref = oracle.tbpm_dos(bessel_series(math.pi), h.indptr, h.indices, h.data, 16,
                          seed=1337, n_samples=4)
    assert np.max(np.abs(res[0][3] - ref)) < 1e-13
    assert np.array_equal(res[0][3], res[1][3])


def _worker_dc(rank, world, port, outdir, q):
    # one OpenMP thread per rank: two ranks share the host cores, and the oracle's
    # small parallel regions stall on oversubscribed barriers otherwise (torch,
    # imported with this module, has already started the OpenMP runtime)
    os.environ["OMP_NUM_THREADS"] = "1"
    import torch
    torch.set_num_threads(1)
    sys.path.insert(0, ROOT)
    try:
        dist = _init(rank, world, port)
        import tbplas_b200 as tb
        from tbplas_b200.tbpm import solver as solver_mod
        from oracle import oracle

        class CpuStandIn:
            def tbpm_dccond(self, *a):
                return oracle.F2pyShim().tbpm_dccond(*a)

            def set_backend(self, **kw):
                pass

        solver_mod.f2py = CpuStandIn()
        s = tb.make_graphene_sample(6, 5, disorder=0.4, seed=7)
        cfg = tb.Config()
        cfg.generic["nr_time_steps"] = 12
        cfg.generic["nr_random_samples"] = 3
        cfg.DC_conductivity["energy_limits"] = (-2.0, 2.0)
        solver = tb.Solver(s, cfg, enable_mpi=True, echo_details=False,
                           directory=os.path.join(outdir, f"r{rank}"), prefix="d")
        dos, dc = solver.calc_corr_dc_cond()
        q.put((rank, dos, dc, np.isfortran(dc)))
        dist.barrier()
        dist.destroy_process_group()
    except Exception as e:  # report instead of hanging the parent
        q.put((rank, "error", repr(e), None))


def test_two_rank_dc_conductivity(tmp_path):
    """DC: the (n_timestep,) DOS and the (2, 2*n_timestep, n_timestep) Fortran-
    ordered DC correlations are averaged over the ranks' samples (3 padded to
    4), and equal the single-process oracle over the same 4 seeded samples."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker_dc, args=(r, 2, port, str(tmp_path), q))
             for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(2):
        r = q.get(timeout=240)
        res[r[0]] = r
    for p in procs:
        p.join(timeout=60)
    for r in (0, 1):
        assert not isinstance(res[r][1], str), res[r][2]
    assert np.array_equal(res[0][1], res[1][1]) and np.array_equal(res[0][2], res[1][2])
    sys.path.insert(0, ROOT)
    import math
    import tbplas_b200 as tb
    from oracle import oracle
    from conftest import bessel_series
    s = tb.make_graphene_sample(6, 5, disorder=0.4, seed=7)
    ip, ix, hv, dx, dy = s.build_ham_dxy()
    tnr = 12
    en_range = s.energy_range
    energies = np.array([0.5 * i * en_range / tnr - en_range / 2. for i in range(2 * tnr)])
    sel = np.where((energies >= -2.0) & (energies <= 2.0))[0]
    t_step = 2 * math.pi / en_range
    rdos, rdc = oracle.tbpm_dccond(bessel_series(t_step * s.rescale), ip, ix, hv, s.rescale,
                                   dx, dy, tnr, t_step, energies, sel, seed=1337, n_samples=4)
    assert res[0][2].shape == (2, 2 * tnr, tnr)
    assert np.max(np.abs(res[0][1] - rdos)) < 1e-13
    assert np.max(np.abs(res[0][2] - rdc)) <= 1e-13 * max(1.0, np.max(np.abs(rdc)))


def _worker_ac(rank, world, port, outdir, q):
    # one OpenMP thread per rank: two ranks share the host cores, and the oracle's
    # small parallel regions stall on oversubscribed barriers otherwise (torch,
    # imported with this module, has already started the OpenMP runtime)
    os.environ["OMP_NUM_THREADS"] = "1"
    import torch
    torch.set_num_threads(1)
    sys.path.insert(0, ROOT)
    try:
        dist = _init(rank, world, port)
        import tbplas_b200 as tb
        from tbplas_b200.tbpm import solver as solver_mod
        from oracle import oracle

        class CpuStandIn:
            def tbpm_accond(self, *a):
                return oracle.F2pyShim().tbpm_accond(*a)

            def set_backend(self, **kw):
                pass

        solver_mod.f2py = CpuStandIn()
        s = tb.make_graphene_sample(5, 5, disorder=0.4, seed=8)
        cfg = tb.Config()
        cfg.generic["nr_time_steps"] = 10
        cfg.generic["nr_random_samples"] = 2
        solver = tb.Solver(s, cfg, enable_mpi=True, echo_details=False,
                           directory=os.path.join(outdir, f"r{rank}"), prefix="a")
        ac = solver.calc_corr_ac_cond()
        q.put((rank, ac, np.isfortran(ac)))
        dist.barrier()
        dist.destroy_process_group()
    except Exception as e:  # report instead of hanging the parent
        q.put((rank, "error", repr(e)))


def test_two_rank_ac_conductivity(tmp_path):
    """AC: each rank propagates its own samples (Fermi operators included); the
    (4, n_timestep) correlations averaged over the ranks equal the
    single-process oracle over the same seeded samples."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker_ac, args=(r, 2, port, str(tmp_path), q))
             for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(2):
        r = q.get(timeout=240)
        res[r[0]] = r
    for p in procs:
        p.join(timeout=60)
    for r in (0, 1):
        assert not isinstance(res[r][1], str), res[r][2]
    assert np.array_equal(res[0][1], res[1][1])
    sys.path.insert(0, ROOT)
    import math
    import tbplas_b200 as tb
    from oracle import oracle
    from conftest import bessel_series
    s = tb.make_graphene_sample(5, 5, disorder=0.4, seed=8)
    ip, ix, hv, dx, dy = s.build_ham_dxy()
    cfg = tb.Config()
    beta = cfg.generic["beta"] * s.rescale
    mu = cfg.generic["mu"] / s.rescale
    t_half = 0.5 * 2 * math.pi / s.energy_range
    ref = oracle.tbpm_accond(bessel_series(t_half * s.rescale), beta, mu, ip, ix, hv, s.rescale,
                             dx, dy, 10, seed=1337, n_samples=2)
    assert res[0][1].shape == (4, 10) and res[0][2]
    assert np.max(np.abs(res[0][1] - ref)) <= 1e-13 * max(1.0, np.max(np.abs(ref)))


def _worker_fail(rank, world, port, q):
    sys.path.insert(0, ROOT)
    try:
        dist = _init(rank, world, port, timeout_s=5)
        from tbplas_b200.parallel import MPIEnv
        env = MPIEnv(enable_mpi=True)
        if rank == 1:
            raise RuntimeError("rank 1 failed before the collective")
        env.all_average(np.ones(3, dtype=np.complex128))
        q.put((rank, "no error"))
    except Exception as e:
        q.put((rank, type(e).__name__))


def test_failed_rank_is_detected_by_survivor():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker_fail, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=30)
        if p.is_alive():
            p.kill()
    assert got[1] == "RuntimeError"
    assert got[0] != "no error"
