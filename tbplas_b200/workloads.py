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
import os
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


def _c3_sample(args):
    nx, ny, w, seed = args
    s = make_graphene_sample(nx, ny, disorder=w, vacancy_rate=0.01, rescale=10.0, seed=seed)
    h = s.build_ham_csr()
    return h.indptr.astype(np.int64), h.indices.astype(np.int32), h.data


def build_c3(n_real: int = 64, lo: int = 256, hi: int = 1024, seed: int = 1337, workers=None):
    """64 realisations with L_a, L_b ~ U{lo..hi} cells, W ~ U[0,3] eV, 1%
    vacancies, rescale 10 eV (max row sum 3*2.7 + 1.5 < 10), packed
    block-diagonally.  Built in a spawn-started process pool (host work only,
    before any CUDA use in the workers)."""
    import concurrent.futures as cf
    import multiprocessing as mp
    rng = np.random.default_rng(seed)
    specs = [(int(rng.integers(lo, hi + 1)), int(rng.integers(lo, hi + 1)),
              float(rng.uniform(0, 3)), seed + 1 + i) for i in range(n_real)]
    workers = workers or min(8, os.cpu_count() or 1)
    with cf.ProcessPoolExecutor(max_workers=workers,
                                mp_context=mp.get_context("spawn")) as ex:
        parts = list(ex.map(_c3_sample, specs))
    offsets = [0]
    ips, ixs, vals = [], [], []
    nnz = 0
    for ip, ix, v in parts:
        ips.append(ip[:-1] + nnz)
        ixs.append(ix + offsets[-1])
        vals.append(v)
        nnz += v.size
        offsets.append(offsets[-1] + ip.size - 1)
    indptr = np.concatenate(ips + [np.array([nnz])]).astype(np.int32)
    return (indptr, np.concatenate(ixs).astype(np.int32), np.concatenate(vals),
            np.array(offsets, dtype=np.int64), specs)


def run_c3(steps: int = 512, n_states: int = 4, n_real: int = 64, lo: int = 256,
           hi: int = 1024) -> dict:
    from . import autotune
    (ip, ix, hv, off, specs), t_build = _timed(lambda: build_c3(n_real, lo, hi))
    n = ip.size - 1
    bes = bessel_series(math.pi)  # dt*rescale = 2*pi/(2*rescale)*rescale
    res = {"workload": f"c3 {n_real} graphene realisations {lo}^2..{hi}^2, 1% vacancies, "
                       f"W~U[0,3] eV, rescale 10, {n_states} states each, packed, one graph",
           "n_orbitals_total": int(n), "nnz": int(hv.size), "steps": steps,
           "host_build_seconds": t_build}
    out = {}
    for prec in ("fp64", "fp32"):
        tuned = autotune.tune_dos(ip, ix, hv, n_states, prec, steps=2, bessel=bes)
        autotune.apply(tuned["best"])
        f2py.set_backend(precision=prec)
        corr, sec = _timed(lambda: f2py.tbpm_dos_segmented(bes, ip, ix, hv, off, n_states,
                                                           1337, steps))
        res[f"{prec}_tuned"] = tuned["best"]
        res[f"{prec}_seconds"] = sec
        res[f"{prec}_orbital_steps_per_s"] = n * n_states * steps / sec
        out[prec] = corr
    diff = np.abs(out["fp32"] - out["fp64"]).max(axis=1) / np.abs(out["fp64"]).max(axis=1)
    res["fp32_max_rel_corr_err_per_realisation"] = float(diff.max())
    f2py.set_backend(precision="fp64", threads_per_block=0, vector_width=0)
    return res


def run_c5(steps: int = 2048, n_states: int = 8, nx: int = 4096, precision: str = "fp32",
           energy_limits=(-0.5, 0.5)) -> dict:
    """DC conductivity of 4096x4096 graphene in a perpendicular field of one
    flux quantum per 1024 hexagons (B = h/e / (1024 * hexagon area) = 77.06 T,
    Peierls phases in the gauge A = (By, 0, 0)), Anderson W = 1 eV, through the
    drop-in Solver / Analyzer."""
    import tempfile
    t0 = time.perf_counter()
    s = make_graphene_sample(nx, nx, disorder=1.0, rescale=9.0, seed=1337)
    flux_quantum = 4135.667  # h/e in T nm^2
    b_field = flux_quantum / (1024 * s.area_unit_cell)
    s.set_magnetic_field(b_field, gauge=0)
    ham = s.build_ham_dxy()
    t_build = time.perf_counter() - t0

    class Prebuilt:  # the Sample interface with the arrays built once
        rescale = s.rescale
        energy_range = s.energy_range
        nr_orbitals = s.nr_orbitals
        area_unit_cell = s.area_unit_cell
        volume_unit_cell = s.volume_unit_cell
        extended = s.extended

        def build_ham_dxy(self):
            return ham

    cfg = Config()
    cfg.generic["nr_time_steps"] = steps
    cfg.generic["nr_random_samples"] = n_states
    cfg.DC_conductivity["energy_limits"] = energy_limits
    with tempfile.TemporaryDirectory() as d:
        solver = Solver(Prebuilt(), cfg, echo_details=False, directory=d, prefix="c5",
                        backend={"precision": precision, "batch": n_states})
        (corr_dos, corr_dc), sec = _timed(solver.calc_corr_dc_cond)
    an = Analyzer(Prebuilt(), cfg, dimension=2)
    energies, dc = an.calc_dc_cond(corr_dos, corr_dc)
    i0 = int(np.argmin(np.abs(energies)))
    n = ham[0].size - 1
    f2py.set_backend(precision="fp64", batch=16)
    return {"workload": f"c5 graphene {nx}x{nx}, B={b_field:.2f} T (flux h/e per 1024 "
                        f"hexagons), W=1 eV, {n_states} states, corr_dc {precision}",
            "n_orbitals": int(n), "steps": steps, "n_energies": int(energies.size),
            "host_build_seconds": t_build, "seconds": sec,
            "orbital_steps_per_s": n * n_states * steps / sec,
            "sigma_dc_xx_at_E0": float(dc[0, i0]), "sigma_dc_yy_at_E0": float(dc[1, i0]),
            "corr_dos_1": [float(corr_dos[0].real), float(corr_dos[0].imag)]}


def _realisation(args):
    nx, ny, w, vac, seed = args
    s = make_graphene_sample(nx, ny, disorder=w, vacancy_rate=vac, rescale=10.0, seed=seed)
    h = s.build_ham_csr()
    return h.indptr.astype(np.int64), h.indices.astype(np.int32), h.data


def _pack(parts):
    offsets, ips, ixs, vals, nnz = [0], [], [], [], 0
    for ip, ix, v in parts:
        ips.append(ip[:-1] + nnz)
        ixs.append(ix + offsets[-1])
        vals.append(v)
        nnz += v.size
        offsets.append(offsets[-1] + ip.size - 1)
    indptr = np.concatenate(ips + [np.array([nnz])]).astype(np.int32)
    return indptr, np.concatenate(ixs).astype(np.int32), np.concatenate(vals), \
        np.array(offsets, dtype=np.int64)


def generate_curves(specs, n_states: int, tnr: int, precision: str, seed: int,
                    pack: int = 16, workers=None):
    """Per-state DOS correlations of graphene realisations specs = [(nx, ny,
    W, vacancy_rate, seed)], propagated on the GPU in packs of `pack`
    realisations.  Returns (n_real, n_states, tnr+1) complex128 and the GPU
    seconds spent."""
    import concurrent.futures as cf
    import multiprocessing as mp
    workers = workers or min(8, os.cpu_count() or 1)
    out, gpu_sec = [], 0.0
    bes = bessel_series(math.pi)  # dt*rescale = pi for rescale 10 and dt = 2 pi / 20
    with cf.ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
        for p0 in range(0, len(specs), pack):
            parts = list(ex.map(_realisation, specs[p0:p0 + pack]))
            ip, ix, hv, off = _pack(parts)
            f2py.set_backend(precision=precision)
            (corr, per), sec = _timed(lambda: f2py.tbpm_dos_segmented(
                bes, ip, ix, hv, off, n_states, seed + p0, tnr, per_state=True))
            gpu_sec += sec
            out.append(per)
    f2py.set_backend(precision="fp64")
    return np.concatenate(out), gpu_sec


def run_c4(n_train: int = 128, n_test: int = 8, nx: int = 512, n_states: int = 8,
           n_ref_states: int = 64, tnr: int = 2048, n_in: int = 256, epochs: int = 200,
           seed: int = 2024, data: str = None) -> dict:
    """Learned tail extrapolator: train on GPU-generated C(t) of disordered
    graphene with vacancies, then compare the DOS of (n_in propagated steps +
    predicted tail) with plain propagation of n steps, against a converged
    reference (n_ref_states states, 2048 steps) on held-out realisations.

    Time-to-DOS: plain FP64 needs n steps with n_states states; the learned
    path needs n_in FP32 steps of the same states plus one network inference.
    `data`: npz cache of the generated curves (written when absent).
    """
    from .learned import TailNet, curves_to_xy, dos_l1, extend
    res = {"workload": f"c4 learned tail: {nx}x{nx} graphene, W~U[0,3] eV, vacancies 0-2%, "
                       f"{n_states} states, n_in={n_in} -> {tnr}",
           "n_train_curves": n_train * n_states, "n_test_realisations": n_test}
    if data and os.path.exists(data):
        d = np.load(data)
        train, ref, ev64, ev32 = d["train"], d["ref"], d["ev64"], d["ev32"]
        t_gen, t64, t32 = float(d["t_gen"]), float(d["t64"]), float(d["t32"])
    else:
        rng = np.random.default_rng(seed)
        mk = lambda k, s0: [(nx, nx, float(rng.uniform(0, 3)), float(rng.uniform(0, 0.02)),
                             s0 + i) for i in range(k)]
        train_specs = mk(n_train, 10_000)
        test_specs = mk(n_test, 20_000)
        train, t_gen = generate_curves(train_specs, n_states, tnr, "fp32", 1)
        ref32, _ = generate_curves(test_specs, n_ref_states, tnr, "fp32", 7)
        ref = ref32.mean(axis=1)
        ev64, t64 = generate_curves(test_specs, n_states, tnr, "fp64", 7)  # same first states
        ev32, t32 = generate_curves(test_specs, n_states, tnr, "fp32", 7)
        if data:
            np.savez(data, train=train.astype(np.complex64), ref=ref, ev64=ev64, ev32=ev32,
                     t_gen=t_gen, t64=t64, t32=t32)
    res["datagen_gpu_seconds"] = t_gen
    e_range = 20.0
    c64 = ev64.mean(axis=1)
    c32 = ev32.mean(axis=1)
    l1 = lambda cs: float(np.mean([dos_l1(cs[k], ref[k], e_range) for k in range(n_test)]))
    plain = {n: l1(c64[:, :n + 1]) for n in (128, 192, 256, 320, 384, 512, 768, 1024, 1536, 2048)}
    res["l1_plain_fp64"] = {str(k): v for k, v in plain.items()}
    res["l1_zero_tail_full_window"] = l1(np.concatenate(
        [c32[:, :n_in + 1], np.zeros((n_test, tnr - n_in), complex)], axis=1))
    sec_step64 = t64 / (n_test * tnr)
    sec_step32 = t32 / (n_test * tnr)
    res["seconds_per_step_fp64"] = sec_step64
    res["seconds_per_step_fp32"] = sec_step32
    variants = {
        "per_state_wd1e-2": dict(targets="state", wd=1e-2),
        "state_mean_wd1e-2": dict(targets="mean", wd=1e-2),
        "per_state_wd1e-1": dict(targets="state", wd=1e-1),
    }
    best_name, best_l1 = None, math.inf
    for name, v in variants.items():
        if v["targets"] == "state":
            x, y = curves_to_xy(train.reshape(-1, tnr + 1).astype(np.complex128), n_in,
                                tnr - n_in)
        else:
            x, y = curves_to_xy(train.mean(axis=1).astype(np.complex128), n_in, tnr - n_in)
        n_val = max(8, len(x) // 8)
        net = TailNet(n_in=n_in, n_out=tnr - n_in, seed=seed)
        net.fit_scales(x, y)
        hist, t_train = _timed(lambda: net.train(x[n_val:], y[n_val:], epochs=epochs, batch=64,
                                                 lr=1e-3, weight_decay=v["wd"],
                                                 x_val=x[:n_val], y_val=y[:n_val],
                                                 patience=30))
        if v["targets"] == "state":
            xs, _ = curves_to_xy(ev32.reshape(-1, tnr + 1), n_in, tnr - n_in)
            tail, t_inf = _timed(lambda: net.predict(xs))
            tail = tail.reshape(n_test, n_states, tnr - n_in, 2).mean(axis=1)
        else:
            xs, _ = curves_to_xy(c32, n_in, tnr - n_in)
            tail, t_inf = _timed(lambda: net.predict(xs))
        learned = extend(c32[:, :n_in + 1], tail)
        r = {"train_seconds": t_train, "best_epoch": hist["best_epoch"],
             "val_mse_initial": hist.get("val_initial"), "val_mse_best": hist.get("val_best"),
             "l1_learned": l1(learned), "inference_seconds": t_inf}
        res[f"variant_{name}"] = r
        if r["l1_learned"] < best_l1:
            best_name, best_l1 = name, r["l1_learned"]
            t_learned = n_in * sec_step32 + t_inf / n_test
    res["best_variant"] = best_name
    res["l1_learned"] = best_l1
    res["seconds_learned_per_realisation"] = t_learned
    n_best_plain = min(plain, key=plain.get)
    res["plain_best_steps"] = n_best_plain
    res["plain_best_l1"] = plain[n_best_plain]
    reach = [n for n in sorted(plain) if plain[n] <= best_l1]
    if reach:
        res["plain_steps_to_reach_learned_l1"] = reach[0]
        res["time_to_dos_speedup_learned_vs_plain_fp64"] = reach[0] * sec_step64 / t_learned
    else:
        res["plain_steps_to_reach_learned_l1"] = None
        res["time_to_dos_speedup_learned_vs_plain_fp64"] = None
    res["speedup_vs_full_plain_2048_fp64"] = tnr * sec_step64 / t_learned
    return res


RUNNERS = {"c1": run_c1, "c2": run_c2, "c3": run_c3, "c4": run_c4, "c5": run_c5}


def main(argv=None) -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("workloads", nargs="+", choices=sorted(RUNNERS))
    ap.add_argument("--steps", type=int, default=None,
                    help="override the number of time steps (shorter runs)")
    ap.add_argument("--out", default=None)
    ap.add_argument("--data", default=None, help="c4: npz cache of the generated curves")
    args = ap.parse_args(argv)
    for w in args.workloads:
        kw = {}
        if args.steps:
            kw = {"steps": args.steps} if w in ("c1", "c3", "c5") else \
                 {"steps_dos": args.steps, "steps_ac": args.steps}
        if w == "c4" and args.data:
            kw["data"] = args.data
        r = RUNNERS[w](**kw)
        line = json.dumps(r)
        print(line, flush=True)
        if args.out:
            with open(args.out, "a") as f:
                f.write(line + "\n")


if __name__ == "__main__":
    main(sys.argv[1:])
