"""The TBPM workloads of the benchmark configurations, as runnable measurements.

    python -m tbplas_b200.workloads c1 c2 [--steps N] [--out results.jsonl]

c1  graphene 100x100 PBC (20,000 orbitals), t = -2.7 eV, rescale 9, one
    unit-modulus random-phase state, 256 steps, corr_dos (FP64).
c2  graphene 2048x2048 PBC (8,388,608 orbitals), Anderson U[-0.5, 0.5] eV,
    16 states as one block, corr_dos + corr_ac, FP64 and FP32 states; the
    FP32 error against FP64 is reported as DOS L1 (Analyzer.calc_dos, both
    normalised) and AC relative L2 (correlation arrays).
c3  64 graphene realisations, 256^2..1024^2 cells, 1% vacancies, W ~ U[0,3] eV,
    rescale 10, 4 states each, 512 steps, packed block-diagonally and
    propagated by one CUDA-graph launch.
c5  graphene 4096x4096 with Peierls phases for one flux quantum per 1024
    hexagons, Anderson W = 1 eV, corr_dc with FP32 states.

Every result is one JSON line (orbital-steps/s, seconds, errors).  Inputs are
seeded synthetic Hamiltonians and seeded Philox states.
"""

import argparse
import json
import math
import sys
import time

import numpy as np

from . import _native as nat
from .builder import make_graphene_sample
from .fortran import f2py
from .tbpm import Analyzer, Config, Solver


def bessel_series(time_scaled: float, precision: float = 1e-14):
    import scipy.special as spec
    out = []
    for i in range(250):
        v = spec.jv(i, time_scaled)
        if abs(v) > precision or abs(spec.jv(i + 1, time_scaled)) > precision:
            out.append(float(v))
        else:
            return out
    raise ValueError("Bessel_max too low")


def dos_l1(sample, corr_a, corr_b, tnr: int) -> float:
    """L1 distance sum_E |rho_a - rho_b| dE of the Analyzer DOS of two
    correlation functions (both normalised to 1)."""
    cfg = Config()
    cfg.generic["nr_time_steps"] = tnr
    an = Analyzer(sample, cfg, dimension=2)
    e, da = an.calc_dos(corr_a)
    _, db = an.calc_dos(corr_b)
    return float(np.sum(np.abs(da - db)) * (e[1] - e[0]))


def _timed(fn):
    t0 = time.perf_counter()
    r = fn()
    return r, time.perf_counter() - t0


def run_c1(steps: int = 256) -> dict:
    s = make_graphene_sample(100, 100, rescale=9.0)
    h = s.build_ham_csr()
    bes = bessel_series(math.pi)
    rng = np.random.default_rng(1337)
    wf = np.exp(2j * np.pi * rng.random(h.shape[0]))
    wf /= np.linalg.norm(wf)
    f2py.set_backend(precision="fp64", batch=16)
    f2py.tbpm_dos_states(bes, h.indptr, h.indices, h.data, wf, 8, 128, 1e-9)  # warm-up
    corr, sec = _timed(lambda: f2py.tbpm_dos_states(bes, h.indptr, h.indices, h.data, wf,
                                                    steps, 128, 1e-9))
    return {"workload": "c1 graphene 100x100, 1 state, corr_dos FP64", "steps": steps,
            "seconds": sec, "orbital_steps_per_s": h.shape[0] * steps / sec,
            "corr_1": [corr[1].real, corr[1].imag]}


def run_c2(steps_dos: int = 1024, steps_ac: int = 1024, n_states: int = 16) -> dict:
    s = make_graphene_sample(2048, 2048, disorder=1.0, rescale=9.0, seed=1337)
    h = s.build_ham_csr()
    ip, ix, hop, dx, dy = s.build_ham_dxy()
    bes_dos = bessel_series(math.pi)
    bes_ac = bessel_series(math.pi / 2)
    n = h.shape[0]
    beta = Config().generic["beta"] * s.rescale
    res = {"workload": "c2 graphene 2048x2048, W=1 eV, 16 states, corr_dos + corr_ac",
           "n_orbitals": n, "states": n_states, "steps_dos": steps_dos, "steps_ac": steps_ac}
    out = {}
    for prec in ("fp64", "fp32"):
        f2py.set_backend(precision=prec, batch=16)
        corr, sec = _timed(lambda: f2py.tbpm_dos(bes_dos, h.indptr, h.indices, h.data, 1337,
                                                 steps_dos, n_states, "", 0, 128, 1e-9))
        res[f"dos_{prec}_seconds"] = sec
        res[f"dos_{prec}_orbital_steps_per_s"] = n * n_states * steps_dos / sec
        ac, sec_ac = _timed(lambda: f2py.tbpm_accond(bes_ac, beta, 0.0, ip, ix, hop, s.rescale,
                                                     dx, dy, 1337, steps_ac, n_states,
                                                     2**15, 1e-12, "", 0, 128, 1e-9))
        res[f"ac_{prec}_seconds"] = sec_ac
        res[f"ac_{prec}_orbital_steps_per_s"] = n * n_states * steps_ac / sec_ac
        out[prec] = (corr, ac)
    res["fp32_dos_l1_vs_fp64"] = dos_l1(s, out["fp32"][0], out["fp64"][0], steps_dos)
    a64, a32 = out["fp64"][1], out["fp32"][1]
    res["fp32_ac_rel_l2_vs_fp64"] = float(np.linalg.norm(a32 - a64) / np.linalg.norm(a64))
    res["fp32_dos_corr_max_rel_vs_fp64"] = float(np.max(np.abs(out["fp32"][0] - out["fp64"][0]))
                                                 / np.max(np.abs(out["fp64"][0])))
    f2py.set_backend(precision="fp64")
    return res


RUNNERS = {"c1": run_c1, "c2": run_c2}


def main(argv=None) -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("workloads", nargs="+", choices=sorted(RUNNERS))
    ap.add_argument("--steps", type=int, default=None,
                    help="override the number of time steps (shorter runs)")
    ap.add_argument("--out", default=None)
    args = ap.parse_args(argv)
    for w in args.workloads:
        kw = {}
        if args.steps:
            kw = {"steps": args.steps} if w == "c1" else \
                 {"steps_dos": args.steps, "steps_ac": args.steps}
        r = RUNNERS[w](**kw)
        line = json.dumps(r)
        print(line, flush=True)
        if args.out:
            with open(args.out, "a") as f:
                f.write(line + "\n")


if __name__ == "__main__":
    main(sys.argv[1:])
