"""Multi-GPU launch logic of bench.py, on CPU.

`bench.py --gpus N` without a torchrun environment re-runs itself under
torch.distributed.run with N ranks on 127.0.0.1, with NCCL's communicator
report on stderr.  Every rank times its own states; the reported time is the
maximum over ranks, with the per-rank list beside it.  Two gloo ranks check
that reduction; the launcher is checked by the command it builds and by main()
handing a multi-GPU request to it.
"""

import os
import socket
import sys
from datetime import timedelta

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_torchrun_command_runs_this_script_as_n_ranks():
    cmd = bench.torchrun_command(4, 29512, ["--gpus", "4", "--steps", "8"])
    assert cmd[:3] == [sys.executable, "-m", "torch.distributed.run"]
    assert "--nnodes=1" in cmd and "--nproc-per-node=4" in cmd
    assert cmd[cmd.index("--master-addr") + 1] == "127.0.0.1"
    assert "--master-port=29512" in cmd
    assert cmd[-4:] == ["--gpus", "4", "--steps", "8"]
    assert os.path.samefile(cmd[-5], os.path.join(ROOT, "bench.py"))


def test_main_hands_multi_gpu_requests_to_the_launcher(monkeypatch):
    seen = {}

    def fake_launch(n, argv):
        seen["n"], seen["argv"] = n, list(argv)
        return 0

    monkeypatch.delenv("WORLD_SIZE", raising=False)
    monkeypatch.setattr(bench, "launch_ranks", fake_launch)
    monkeypatch.setattr(sys, "argv", ["bench.py", "--gpus", "2", "--steps", "4"])
    with pytest.raises(SystemExit) as e:
        bench.main()
    assert e.value.code == 0
    assert seen == {"n": 2, "argv": ["--gpus", "2", "--steps", "4"]}


def test_launcher_sends_nccl_report_to_stderr(monkeypatch):
    got = {}

    def fake_call(cmd, env):
        got["cmd"], got["env"] = cmd, env
        return 3

    monkeypatch.delenv("NCCL_DEBUG", raising=False)
    monkeypatch.delenv("NCCL_DEBUG_FILE", raising=False)
    monkeypatch.setattr(bench.subprocess, "call", fake_call)
    assert bench.launch_ranks(2, ["--gpus", "2"]) == 3
    assert got["env"]["NCCL_DEBUG"] == "INFO"
    assert got["env"]["NCCL_DEBUG_FILE"] == "/dev/stderr"
    assert "--nproc-per-node=2" in got["cmd"]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    os.environ["OMP_NUM_THREADS"] = "1"
    sys.path.insert(0, ROOT)
    try:
        import torch
        import torch.distributed as dist
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        dist.init_process_group("gloo", rank=rank, world_size=world,
                                timeout=timedelta(seconds=60))
        import bench as b
        mx, per = b.gather_rank_values(10.0 + 5.0 * rank, dist, torch.device("cpu"))
        q.put((rank, mx, per))
        dist.barrier()
        dist.destroy_process_group()
    except Exception as e:  # report instead of hanging the parent
        q.put((rank, "error", repr(e)))


def test_two_rank_timing_is_the_maximum_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(2):
        r = q.get(timeout=180)
        res[r[0]] = r
    for p in procs:
        p.join(timeout=60)
    for r in (0, 1):
        assert res[r][1] != "error", res[r][2]
        assert res[r][1] == 15.0
        assert res[r][2] == [10.0, 15.0]
