"""Autotuner of the Chebyshev-term launch shape.

For a given Hamiltonian, block width (states propagated together) and
precision it times a few DOS time steps for every candidate of

* threads per block (rows per block sweep iteration = threads / columns),
* FP32 vector width (1 or 2 complex values per thread and load),

keeps the fastest and stores it in a JSON cache keyed by precision, block
width and the matrix shape (rows, entries per row).  `apply` sets the best
shape as the backend default of tbplas_b200.fortran.f2py.

    python -m tbplas_b200.autotune --nx 512 --ny 512 --states 16 --precision fp32
"""

import argparse
import ctypes
import json
import math
import os
import time
from typing import Dict, Iterable, Optional

import numpy as np

from . import _native as nat
from .fortran import f2py

DEFAULT_CACHE = os.path.join(os.path.expanduser("~"), ".cache", "tbplas_b200", "tune.json")


def _key(precision: str, n_states: int, n_rows: int, nnz: int) -> str:
    per_row = round(nnz / max(n_rows, 1), 1)
    size = int(round(math.log2(max(n_rows, 1))))
    return f"{precision}/ld{n_states}/2^{size}rows/{per_row}nnz"


def tune_dos(indptr, indices, hop, n_states: int, precision: str = "fp64",
             threads: Iterable[int] = (64, 128, 256), steps: int = 4,
             device: Optional[int] = None, bessel: Optional[np.ndarray] = None) -> Dict:
    """Time `steps` DOS time steps for every candidate launch shape on this
    Hamiltonian; return {"best": {...}, "timings": [...]}."""
    ctx = nat.get_context(device)
    ip = nat.as_c(indptr, np.int32)
    ix = nat.as_c(indices, np.int32)
    hv = nat.as_c(hop, np.complex128)
    n, nnz = ip.size - 1, hv.size
    if bessel is None:
        import scipy.special as spec
        bessel = np.array([spec.jv(i, math.pi) for i in range(20)])
    bes = nat.as_c(bessel, np.float64)
    prec = nat.PREC_FP64 if precision == "fp64" else nat.PREC_FP32
    # vector widths: 0 = the library's choice (32-byte accesses when the block
    # width allows: four complex64 / two complex128 per thread), 1, 2 forced
    if n_states % 2:
        widths = (0,)
    elif precision == "fp32":
        widths = (0, 1, 2)
    else:
        widths = (0, 1)
    timings = []
    saved = ctx.options
    try:
        for vw in widths:
            for tpb in threads:
                ctx.set_options(precision=prec, batch=n_states, threads_per_block=int(tpb),
                                vector_width=int(vw), use_graphs=1, steps_per_graph=steps)
                ctx.call("tbpm_ham_upload", nat.ptr(ip), nat.ptr(ix), nat.ptr(hv), n, nnz, None,
                         None, 1.0)
                ctx.call("tbpm_session_dos_begin", nat.ptr(bes), bes.size, n_states, 1, 0,
                         n_states, 2 * steps + 1)
                done = ctypes.c_int(0)
                ctx.call("tbpm_session_advance", steps)  # warm-up (graph capture)
                ctx.call("tbpm_session_read", None, None, ctypes.byref(done))
                t0 = time.perf_counter()
                ctx.call("tbpm_session_advance", steps)
                ctx.call("tbpm_session_read", None, None, ctypes.byref(done))
                ms = (time.perf_counter() - t0) * 1e3 / steps
                timings.append({"threads_per_block": int(tpb), "vector_width": int(vw),
                                "ms_per_step": ms})
    finally:
        ctx.check(ctx._lib.tbpm_set_options(ctx.handle, ctypes.byref(saved)))
    best = min(timings, key=lambda r: r["ms_per_step"])
    return {"key": _key(precision, n_states, n, nnz), "best": best, "timings": timings}


def save(result: Dict, path: str = DEFAULT_CACHE) -> None:
    os.makedirs(os.path.dirname(path), exist_ok=True)
    cache = load_cache(path)
    cache[result["key"]] = result["best"]
    with open(path, "w") as f:
        json.dump(cache, f, indent=1, sort_keys=True)


def load_cache(path: str = DEFAULT_CACHE) -> Dict:
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def apply(best: Dict) -> None:
    """Make a tuned shape the backend default."""
    f2py.set_backend(threads_per_block=int(best["threads_per_block"]),
                     vector_width=int(best.get("vector_width", 0)))


def lookup(precision: str, n_states: int, n_rows: int, nnz: int,
           path: str = DEFAULT_CACHE) -> Optional[Dict]:
    return load_cache(path).get(_key(precision, n_states, n_rows, nnz))


def main(argv=None) -> None:
    from .builder import make_graphene_sample
    ap = argparse.ArgumentParser()
    ap.add_argument("--nx", type=int, default=512)
    ap.add_argument("--ny", type=int, default=512)
    ap.add_argument("--states", type=int, default=16)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"])
    ap.add_argument("--disorder", type=float, default=1.0)
    ap.add_argument("--cache", default=DEFAULT_CACHE)
    args = ap.parse_args(argv)
    s = make_graphene_sample(args.nx, args.ny, disorder=args.disorder)
    h = s.build_ham_csr()
    r = tune_dos(h.indptr, h.indices, h.data, args.states, args.precision)
    save(r, args.cache)
    print(json.dumps(r))


if __name__ == "__main__":
    main()
