"""Process-parallel environment of the TBPM path over torch.distributed.

Replaces the mpi4py wrapper `MPIEnv` of the reference (tbplas/parallel.py:18-257)
with the same contract: rank/size/is_master, `all_average` (sum over ranks,
divided by the number of ranks, parallel.py:175-189), `bcast` from rank 0,
`barrier` and master-only printing.  One process drives one GPU; random
states are split across ranks by Solver._dist_sample exactly as in the
reference, and the only collective on the data path is the final average of
the correlation arrays (kilobytes to hundreds of megabytes).

With the NCCL backend the arrays are reduced on the GPU over NVLink; with
gloo (CPU tests) on the host.
"""

import os
from datetime import timedelta

import numpy as np

__all__ = ["MPIEnv", "init_distributed"]


def init_distributed(backend: str = None, timeout_s: float = 120.0) -> bool:
    """Initialise torch.distributed from the torchrun environment if needed.

    :return: True when a process group is available afterwards
    """
    import torch
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        return True
    if "RANK" not in os.environ or "WORLD_SIZE" not in os.environ:
        return False
    if backend is None:
        backend = "nccl" if torch.cuda.is_available() else "gloo"
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    kwargs = {"backend": backend, "timeout": timedelta(seconds=timeout_s)}
    if backend == "nccl":
        local = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(local)
        kwargs["device_id"] = torch.device("cuda", local)
    dist.init_process_group(**kwargs)
    return True


class MPIEnv:
    """Rank information and the collectives the TBPM drivers need.

    :param enable_mpi: use the torch.distributed process group (initialised
        from the torchrun environment when not yet initialised); when False
        the object describes a single process, as in the reference
    :param echo_details: print the parallelisation details on rank 0
    """

    def __init__(self, enable_mpi: bool = False, echo_details: bool = False) -> None:
        self._dist = None
        self._rank, self._size = 0, 1
        if enable_mpi:
            if not init_distributed():
                raise ImportError("no torch.distributed process group: launch with torchrun "
                                  "or call torch.distributed.init_process_group first")
            import torch.distributed as dist
            self._dist = dist
            self._rank = dist.get_rank()
            self._size = dist.get_world_size()
        if echo_details:
            spaces = " " * 2
            self.print("\nParallelization details:")
            if self.mpi_enabled:
                self.print(f"{spaces}{'Processes':16s} : {self._size:<6d}")
            else:
                self.print(f"{spaces}{'MPI disabled':16s}")
            self.print()

    # -- collectives ---------------------------------------------------------
    def _reduce_sum(self, data: np.ndarray) -> np.ndarray:
        import torch
        dist = self._dist
        backend = dist.get_backend()
        arr = np.asarray(data)
        order = "F" if (arr.ndim > 1 and arr.flags.f_contiguous
                        and not arr.flags.c_contiguous) else "C"
        # a copy: the reduction must not overwrite the caller's local array
        # (the reference's all_average reduces into a new buffer)
        flat = np.array(arr.reshape(-1, order=order), copy=True)
        t = torch.from_numpy(flat.view(np.float64) if np.iscomplexobj(flat) else flat)
        if backend == "nccl":
            t = t.to(torch.device("cuda", torch.cuda.current_device()))
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        out = t.cpu().numpy()
        if np.iscomplexobj(flat):
            out = out.view(np.complex128)
        return out.reshape(arr.shape, order=order)

    def all_average(self, data_local: np.ndarray) -> np.ndarray:
        """Average data over ranks (reference parallel.py:175-189)."""
        if not self.mpi_enabled:
            return data_local
        data = self._reduce_sum(data_local)
        data /= self._size
        return data

    def all_reduce(self, data_local: np.ndarray) -> np.ndarray:
        """Sum data over ranks."""
        if not self.mpi_enabled:
            return data_local
        return self._reduce_sum(data_local)

    def bcast(self, data_local: np.ndarray) -> None:
        """Broadcast data_local in place from rank 0."""
        if not self.mpi_enabled:
            return
        import torch
        arr = np.asarray(data_local)
        flat = np.ascontiguousarray(arr).reshape(-1)
        t = torch.from_numpy(flat.view(np.float64) if np.iscomplexobj(flat) else flat.copy())
        if self._dist.get_backend() == "nccl":
            t = t.to(torch.device("cuda", torch.cuda.current_device()))
        self._dist.broadcast(t, src=0)
        res = t.cpu().numpy()
        if np.iscomplexobj(flat):
            res = res.view(np.complex128)
        data_local[...] = res.reshape(arr.shape)

    def barrier(self) -> None:
        if self.mpi_enabled:
            self._dist.barrier()

    def print(self, text: str = "") -> None:
        if self.is_master:
            print(text, flush=True)

    @property
    def mpi_enabled(self) -> bool:
        return self._dist is not None

    @property
    def is_master(self) -> bool:
        return self._rank == 0

    @property
    def rank(self) -> int:
        return self._rank

    @property
    def size(self) -> int:
        return self._size
