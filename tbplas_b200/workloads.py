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

from .builder import LatticeSample, make_graphene_sample
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
           energy_limits=(-0.5, 0.5), builder: str = "device") -> dict:
    """DC conductivity of 4096x4096 graphene in a perpendicular field of one
    flux quantum per 1024 hexagons (B = h/e / (1024 * hexagon area) = 77.06 T,
    Peierls phases in the gauge A = (By, 0, 0)), Anderson W = 1 eV, through the
    drop-in Solver / Analyzer.  builder "device" assembles the Hamiltonian on
    the GPU (DeviceSample), "host" builds the CSR with numpy and uploads it."""
    import tempfile
    from .supercell import make_graphene_device_sample
    flux_quantum = 4135.667  # h/e in T nm^2
    b_field = flux_quantum / (1024 * LatticeSample((1, 1)).area_unit_cell)
    t0 = time.perf_counter()
    if builder == "device":
        f2py.set_backend(precision=precision, batch=n_states)
        sample = make_graphene_device_sample(nx, nx, disorder=1.0, b_field=b_field, gauge=0,
                                             rescale=9.0, seed=1337)
        n, _ = sample.build_ham_dxy()[0].make_resident(f2py._ctx())
        t_build = time.perf_counter() - t0
    else:
        s = make_graphene_sample(nx, nx, disorder=1.0, rescale=9.0, seed=1337)
        s.set_magnetic_field(b_field, gauge=0)
        ham = s.build_ham_dxy()
        t_build = time.perf_counter() - t0
        n = ham[0].size - 1

        class Prebuilt:  # the Sample interface with the arrays built once
            rescale = s.rescale
            energy_range = s.energy_range
            nr_orbitals = s.nr_orbitals
            area_unit_cell = s.area_unit_cell
            volume_unit_cell = s.volume_unit_cell
            extended = s.extended

            def build_ham_dxy(self):
                return ham

        sample = Prebuilt()

    cfg = Config()
    cfg.generic["nr_time_steps"] = steps
    cfg.generic["nr_random_samples"] = n_states
    cfg.DC_conductivity["energy_limits"] = energy_limits
    with tempfile.TemporaryDirectory() as d:
        solver = Solver(sample, cfg, echo_details=False, directory=d, prefix="c5",
                        backend={"precision": precision, "batch": n_states})
        (corr_dos, corr_dc), sec = _timed(solver.calc_corr_dc_cond)
    an = Analyzer(sample, cfg, dimension=2)
    energies, dc = an.calc_dc_cond(corr_dos, corr_dc)
    i0 = int(np.argmin(np.abs(energies)))
    f2py.set_backend(precision="fp64", batch=16)
    return {"workload": f"c5 graphene {nx}x{nx}, B={b_field:.2f} T (flux h/e per 1024 "
                        f"hexagons), W=1 eV, {n_states} states, corr_dc {precision}",
            "builder": builder, "n_orbitals": int(n), "steps": steps,
            "n_energies": int(energies.size), "energy_limits_eV": list(energy_limits),
            "build_seconds": t_build, "seconds": sec,
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


def _field_realisation(args):
    nx, ny, w, b_field, seed = args
    s = make_graphene_sample(nx, ny, disorder=w, rescale=9.0, seed=seed)
    s.set_magnetic_field(b_field, gauge=0)
    h = s.build_ham_csr()
    return h.indptr.astype(np.int64), h.indices.astype(np.int32), h.data


def _curves_from_parts(parts, n_states: int, tnr: int, precision: str, seed: int):
    """Per-state DOS correlations of the realisations in `parts` (CSR arrays),
    packed into one launch; returns them and the GPU seconds spent."""
    bes = bessel_series(math.pi)
    ip, ix, hv, off = _pack(parts)
    try:
        f2py.set_backend(precision=precision)
        (corr, per), sec = _timed(lambda: f2py.tbpm_dos_segmented(
            bes, ip, ix, hv, off, n_states, seed, tnr, per_state=True))
    finally:
        f2py.set_backend(precision="fp64")
    return per, sec


def generate_curves(specs, n_states: int, tnr: int, precision: str, seed: int,
                    pack: int = 16, workers=None, build=None):
    """Per-state DOS correlations of graphene realisations specs = [(nx, ny,
    W, vacancy_rate, seed)] (or the arguments of `build`), propagated on the
    GPU in packs of `pack` realisations.  Returns (n_real, n_states, tnr+1)
    complex128 and the GPU seconds spent."""
    import concurrent.futures as cf
    import multiprocessing as mp
    workers = workers or min(8, os.cpu_count() or 1)
    out, gpu_sec = [], 0.0
    bes = bessel_series(math.pi)  # dt*rescale = pi for rescale 10 and dt = 2 pi / 20
    build = build or _realisation
    with cf.ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
        for p0 in range(0, len(specs), pack):
            parts = list(ex.map(build, specs[p0:p0 + pack]))
            ip, ix, hv, off = _pack(parts)
            f2py.set_backend(precision=precision)
            (corr, per), sec = _timed(lambda: f2py.tbpm_dos_segmented(
                bes, ip, ix, hv, off, n_states, seed + p0, tnr, per_state=True))
            gpu_sec += sec
            out.append(per)
    f2py.set_backend(precision="fp64")
    return np.concatenate(out), gpu_sec


def _l1_mean(curves, refs, e_range: float = 20.0) -> float:
    # e_range: the energy range 2 * rescale of the samples (10 eV for c4)
    from .learned import dos_l1 as l1
    return float(np.mean([l1(curves[k], refs[k], e_range) for k in range(len(refs))]))


def _time_dos_paths(parts, n_states: int, steps_list, seed: int = 7) -> dict:
    """End-to-end seconds per realisation (host CSR in, correlation out) of
    the plain FP64 path (f2py.tbpm_dos, one realisation per call) and of the
    FP32 path with all realisations packed into one launch, for each number
    of steps in steps_list."""
    bes = bessel_series(math.pi)
    ip1, ix1, hv1 = parts[0]
    ip, ix, hv, off = _pack(parts)
    out = {}
    try:
        for n in steps_list:
            f2py.set_backend(precision="fp64")
            f2py.tbpm_dos(bes, ip1, ix1, hv1, seed, 8, n_states, "", 0, 1024, 1e-9)  # warm-up
            _, t64 = _timed(lambda: f2py.tbpm_dos(bes, ip1, ix1, hv1, seed, n, n_states, "", 0,
                                                  1 << 30, 1e-9))
            f2py.set_backend(precision="fp32")
            f2py.tbpm_dos_segmented(bes, ip, ix, hv, off, n_states, seed, 8)  # warm-up
            _, t32 = _timed(lambda: f2py.tbpm_dos_segmented(bes, ip, ix, hv, off, n_states,
                                                            seed, n, 1 << 30))
            out[n] = {"plain_fp64_seconds": t64, "fp32_batched_seconds": t32 / len(parts)}
    finally:
        f2py.set_backend(precision="fp64")
    return out


def _steps_to_reach(l1_by_steps: dict, target: float):
    ok = [n for n in sorted(l1_by_steps) if l1_by_steps[n] < target]
    return ok[0] if ok else None


def run_c4(n_train: int = 128, n_test: int = 8, nx: int = 512, n_states: int = 8,
           n_ref_states: int = 64, tnr: int = 2048, n_in: int = 256, epochs: int = 200,
           seed: int = 2024, data: str = None, target_l1: float = 1e-3) -> dict:
    """Learned tail extrapolator on disordered graphene with vacancies.

    Trains on GPU-generated C(t) (FP32, n_states states per realisation),
    then compares on held-out realisations the DOS of
      * plain FP64 propagation of n steps,
      * FP32 propagation of n steps, realisations packed into one launch,
      * n_in FP32 steps followed by the predicted tail (learned),
    with two error definitions: L1 against the full tnr-step FP64
    propagation of the same states, and L1 against a converged reference
    (n_ref_states states).  Time-to-DOS at L1 < target_l1 (same-state
    definition) uses end-to-end timings of each path.  `data`: npz cache of
    the generated curves (written when absent).
    """
    from .learned import TailNet, curves_to_xy, extend
    res = {"workload": f"c4 learned tail: {nx}x{nx} graphene, W~U[0,3] eV, vacancies 0-2%, "
                       f"{n_states} states, n_in={n_in} -> {tnr}",
           "n_train_curves": n_train * n_states, "n_test_realisations": n_test,
           "target_l1": target_l1}
    rng = np.random.default_rng(seed)
    mk = lambda k, s0: [(nx, nx, float(rng.uniform(0, 3)), float(rng.uniform(0, 0.02)),
                         s0 + i) for i in range(k)]
    train_specs = mk(n_train, 10_000)
    test_specs = mk(n_test, 20_000)
    if data and os.path.exists(data):
        d = np.load(data)
        train, ref, ev64, ev32 = d["train"], d["ref"], d["ev64"], d["ev32"]
        t_gen = float(d["t_gen"])
    else:
        train, t_gen = generate_curves(train_specs, n_states, tnr, "fp32", 1)
        ref32, _ = generate_curves(test_specs, n_ref_states, tnr, "fp32", 7)
        ref = ref32.mean(axis=1)
        ev64, t64 = generate_curves(test_specs, n_states, tnr, "fp64", 7)  # same first states
        ev32, t32 = generate_curves(test_specs, n_states, tnr, "fp32", 7)
        if data:
            np.savez(data, train=train.astype(np.complex64), ref=ref, ev64=ev64, ev32=ev32,
                     t_gen=t_gen, t64=t64, t32=t32)
    res["datagen_gpu_seconds"] = t_gen
    c64 = ev64.mean(axis=1)
    c32 = ev32.mean(axis=1)
    grid = (128, 256, 384, 512, 768, 1024, 1536, 1792, 1920, tnr)
    same64 = {n: _l1_mean(c64[:, :n + 1], c64) for n in grid}
    same32 = {n: _l1_mean(c32[:, :n + 1], c64) for n in grid}
    conv64 = {n: _l1_mean(c64[:, :n + 1], ref) for n in grid}
    res["l1_same_states_plain_fp64"] = {str(k): v for k, v in same64.items()}
    res["l1_same_states_fp32"] = {str(k): v for k, v in same32.items()}
    res["l1_converged_plain_fp64"] = {str(k): v for k, v in conv64.items()}
    res["l1_converged_reference_vs_same_states_full"] = _l1_mean(ref, c64)

    variants = {
        "per_state_wd1e-2": dict(targets="state", wd=1e-2),
        "state_mean_wd1e-2": dict(targets="mean", wd=1e-2),
        "per_state_wd1e-1": dict(targets="state", wd=1e-1),
    }
    best = None
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
             "l1_same_states": _l1_mean(learned, c64), "l1_converged": _l1_mean(learned, ref),
             "inference_seconds_per_realisation": t_inf / n_test}
        res[f"variant_{name}"] = r
        if best is None or r["l1_same_states"] < best[1]["l1_same_states"]:
            best = (name, r)
    res["best_variant"] = best[0]
    res["l1_same_states_learned"] = best[1]["l1_same_states"]
    res["l1_converged_learned"] = best[1]["l1_converged"]
    res["l1_same_states_truncated_at_n_in_fp32"] = same32[n_in]
    zero = np.zeros((n_test, tnr - n_in, 2))
    res["l1_same_states_zero_tail_fp32"] = _l1_mean(extend(c32[:, :n_in + 1], zero), c64)

    # time-to-DOS, same-state definition
    parts = [_realisation(sp) for sp in test_specs]
    n64 = _steps_to_reach(same64, target_l1)
    n32 = _steps_to_reach(same32, target_l1)
    need = sorted({n for n in (n64, n32, n_in) if n})
    times = _time_dos_paths(parts, n_states, need)
    res["seconds_per_realisation"] = {str(k): v for k, v in times.items()}
    t_plain = times[n64]["plain_fp64_seconds"] if n64 else None
    t_fp32 = times[n32]["fp32_batched_seconds"] if n32 else None
    learned_ok = best[1]["l1_same_states"] < target_l1
    t_learned = (times[n_in]["fp32_batched_seconds"] + best[1]["inference_seconds_per_realisation"]
                 if learned_ok else None)
    res["time_to_dos"] = {
        "plain_fp64": {"steps": n64, "seconds_per_realisation": t_plain},
        "fp32_batched": {"steps": n32, "seconds_per_realisation": t_fp32},
        "fp32_batched_learned": {"reached": learned_ok, "steps": n_in if learned_ok else None,
                                 "seconds_per_realisation": t_learned},
    }
    res["time_to_dos_speedup_fp32_batched_vs_plain_fp64"] = (
        t_plain / t_fp32 if t_plain and t_fp32 else None)
    res["time_to_dos_speedup_learned_vs_plain_fp64"] = (
        t_plain / t_learned if t_plain and t_learned else None)
    # the best plain accuracy against the converged reference, and what the
    # learned tail reaches there
    n_best = min(conv64, key=conv64.get)
    res["converged_best_plain_steps"] = n_best
    res["converged_best_plain_l1"] = conv64[n_best]
    return res


def run_c4c(n_train: int = 96, n_test: int = 16, nx: int = 48, n_states: int = 64,
            nx_test: int = None, n_states_test: int = None, pack_test: int = None,
            tnr: int = 512, n_in: int = 64, w_max: float = 0.2, width: int = 64,
            epochs: int = 300, seed: int = 5, target_l1: float = 1e-3) -> dict:
    """The learned tail where C(t) carries a deterministic tail: weakly
    disordered graphene (W ~ U[0, w_max] eV, no vacancies) whose DOS keeps
    sharp structure at full resolution.  The network is trained on the state
    averages of nx x nx realisations (n_states states each); held-out
    nx_test x nx_test realisations (n_states_test states) are propagated
    n_in steps in FP32 and extended by the predicted tail.  All DOS L1 errors
    are against the full tnr-step FP64 propagation of the same states.

    Timings are end to end per realisation: the FP64 reference run (one
    launch per pack_test realisations) gives the plain path, scaled to n
    steps where fewer suffice; the FP32 n_in-step run plus inference gives
    the learned path."""
    from .learned import TailNet, curves_to_xy, extend
    nx_test = nx_test or nx
    n_states_test = n_states_test or n_states
    pack_test = pack_test or n_test
    rng = np.random.default_rng(seed)
    mk = lambda k, s0, n: [(n, n, float(rng.uniform(0, w_max)), 0.0, s0 + i) for i in range(k)]
    train_specs = mk(n_train, 100, nx)
    test_specs = mk(n_test, 900, nx_test)
    pack_train = max(1, min(n_train, (1 << 23) // (2 * nx * nx)))
    train, t_gen = generate_curves(train_specs, n_states, tnr, "fp32", 1, pack=pack_train)
    ev64, t64 = generate_curves(test_specs, n_states_test, tnr, "fp64", 7, pack=pack_test)
    ev32, t32 = generate_curves(test_specs, n_states_test, n_in, "fp32", 7, pack=pack_test)
    c64, c32 = ev64.mean(axis=1), ev32.mean(axis=1)
    x, y = curves_to_xy(train.mean(axis=1), n_in, tnr - n_in)
    n_val = max(8, n_train // 6)
    net = TailNet(n_in=n_in, n_out=tnr - n_in, width=width, seed=3)
    net.fit_scales(x, y)
    hist, t_train = _timed(lambda: net.train(x[n_val:], y[n_val:], epochs=epochs, batch=16,
                                             lr=1e-3, weight_decay=1e-3, x_val=x[:n_val],
                                             y_val=y[:n_val], patience=60))
    xs, _ = curves_to_xy(c32, n_in, tnr - n_in)
    tail, t_inf = _timed(lambda: net.predict(xs))
    learned = extend(c32, tail)
    grid = sorted({n_in, 2 * n_in, 3 * n_in, 4 * n_in, tnr // 2, 3 * tnr // 4, 7 * tnr // 8, tnr})
    plain = {n: _l1_mean(c64[:, :n + 1], c64) for n in grid}
    l1_learned = _l1_mean(learned, c64)
    n_match = _steps_to_reach(plain, l1_learned)
    n_target = _steps_to_reach(plain, target_l1)
    t_plain_full = t64 / n_test
    t_learned = t32 / n_test + t_inf / n_test
    per_step = lambda n: t_plain_full * n / tnr if n else None
    return {"workload": f"c4c coherent tail: train {nx}x{nx} graphene x {n_states} states, "
                        f"test {nx_test}x{nx_test} x {n_states_test} states, "
                        f"W~U[0,{w_max}] eV, n_in={n_in} -> {tnr}",
            "n_train_realisations": n_train, "n_test_realisations": n_test,
            "datagen_gpu_seconds": t_gen, "train_seconds": t_train,
            "best_epoch": hist["best_epoch"], "val_mse_initial": hist.get("val_initial"),
            "val_mse_best": hist.get("val_best"),
            "l1_same_states_plain_fp64": {str(k): v for k, v in plain.items()},
            "l1_same_states_truncated_at_n_in_fp32": _l1_mean(c32, c64),
            "l1_same_states_zero_tail_fp32": _l1_mean(
                extend(c32, np.zeros((n_test, tnr - n_in, 2))), c64),
            "l1_same_states_learned": l1_learned,
            "plain_steps_to_match_learned": n_match,
            "plain_fp64_seconds_per_realisation_full": t_plain_full,
            "learned_seconds_per_realisation": t_learned,
            "time_to_dos_speedup_learned_vs_plain_fp64_at_learned_l1": (
                per_step(n_match) / t_learned if n_match else None),
            "target_l1": target_l1,
            "learned_reaches_target": l1_learned < target_l1,
            "plain_steps_to_reach_target": n_target,
            "time_to_dos_speedup_learned_vs_plain_fp64_at_target": (
                per_step(n_target) / t_learned if (n_target and l1_learned < target_l1)
                else None)}


def run_c4l(**kw) -> dict:
    """c4c at scale: the tail learned on 512^2 realisations (16 states,
    ballistic range of 512 steps ~ 430 cells stays inside the sample), tested
    on 2048^2 realisations with 64 states, where the stochastic part of the
    tail is small enough for a DOS L1 near 1e-3."""
    args = dict(n_train=256, n_test=2, nx=512, n_states=16, nx_test=2048, n_states_test=64,
                pack_test=1, w_max=0.5, width=128, epochs=300)
    args.update(kw)
    return run_c4c(**args)


def run_c5l(n_train: int = 64, nx_train: int = 1024, nx_test: int = 4096, n_states: int = 8,
            tnr: int = 2048, n_in: int = 256, epochs: int = 200, seed: int = 2025,
            target_l1: float = 1e-3, data: str = None) -> dict:
    """Configuration 5's plain vs learned-tail comparison, for the DOS: the
    tail network is trained on FP32 C(t) of nx_train^2 graphene in the same
    field (h/e per 1024 hexagons, 77.06 T) and disorder (W = 1 eV), then
    applied to the first n_in FP32 steps of a 4096^2 realisation and compared
    with plain FP64 propagation of the same states (DOS L1 against the full
    tnr-step FP64 curve).  Seconds per path scale the full runs' per-step
    times.  `data`: npz cache of the generated curves (written when absent)."""
    from .learned import TailNet, curves_to_xy, extend
    flux_quantum = 4135.667  # h/e in T nm^2
    b_field = flux_quantum / (1024 * LatticeSample((1, 1)).area_unit_cell)
    e_range = 18.0  # 2 * rescale
    res = {"workload": f"c5 learned tail (DOS): train {n_train} x {nx_train}^2, test {nx_test}^2, "
                       f"B={b_field:.2f} T, W=1 eV, {n_states} states, n_in={n_in} -> {tnr}",
           "n_train_curves": n_train * n_states, "target_l1": target_l1}
    if data and os.path.exists(data):
        d = np.load(data)
        train, ev64, ev32 = d["train"], d["ev64"], d["ev32"]
        t_gen, t64, t32 = float(d["t_gen"]), float(d["t64"]), float(d["t32"])
    else:
        train_specs = [(nx_train, nx_train, 1.0, b_field, 30_000 + i) for i in range(n_train)]
        train, t_gen = generate_curves(train_specs, n_states, tnr, "fp32", 1, pack=8,
                                       build=_field_realisation)
        parts, t_build = _timed(
            lambda: [_field_realisation((nx_test, nx_test, 1.0, b_field, 1337))])
        res["test_host_build_seconds"] = t_build
        ev64, t64 = _curves_from_parts(parts, n_states, tnr, "fp64", 7)
        ev32, t32 = _curves_from_parts(parts, n_states, tnr, "fp32", 7)
        if data:
            np.savez(data, train=train.astype(np.complex64), ev64=ev64, ev32=ev32, t_gen=t_gen,
                     t64=t64, t32=t32)
    res["n_train_curves"] = int(train.shape[0] * train.shape[1])
    res["datagen_gpu_seconds"] = t_gen
    res["test_fp64_seconds"] = t64
    res["test_fp32_seconds"] = t32
    c64, c32 = ev64.mean(axis=1), ev32.mean(axis=1)
    grid = (128, 256, 384, 512, 768, 1024, 1536, 1792, 1920, tnr)
    same64 = {n: _l1_mean(c64[:, :n + 1], c64, e_range) for n in grid}
    same32 = {n: _l1_mean(c32[:, :n + 1], c64, e_range) for n in grid}
    res["l1_same_states_plain_fp64"] = {str(k): v for k, v in same64.items()}
    res["l1_same_states_fp32"] = {str(k): v for k, v in same32.items()}
    best = None
    for name, targets in (("per_state", "state"), ("state_mean", "mean")):
        src = train.reshape(-1, tnr + 1) if targets == "state" else train.mean(axis=1)
        x, y = curves_to_xy(src.astype(np.complex128), n_in, tnr - n_in)
        n_val = max(2, len(x) // 8)  # validation curves (the mean targets are few)
        net = TailNet(n_in=n_in, n_out=tnr - n_in, seed=seed)
        net.fit_scales(x, y)
        hist, t_train = _timed(lambda: net.train(x[n_val:], y[n_val:], epochs=epochs, batch=64,
                                                 lr=1e-3, weight_decay=1e-2, x_val=x[:n_val],
                                                 y_val=y[:n_val], patience=30))
        if targets == "state":
            xs, _ = curves_to_xy(ev32.reshape(-1, tnr + 1), n_in, tnr - n_in)
            tail = net.predict(xs).reshape(1, n_states, tnr - n_in, 2).mean(axis=1)
        else:
            xs, _ = curves_to_xy(c32, n_in, tnr - n_in)
            tail = net.predict(xs)
        learned = extend(c32[:, :n_in + 1], tail)
        r = {"train_seconds": t_train, "best_epoch": hist["best_epoch"],
             "val_mse_initial": hist.get("val_initial"), "val_mse_best": hist.get("val_best"),
             "l1_same_states": _l1_mean(learned, c64, e_range)}
        res[f"variant_{name}"] = r
        if best is None or r["l1_same_states"] < best[1]["l1_same_states"]:
            best = (name, r)
    res["best_variant"] = best[0]
    res["l1_same_states_learned"] = best[1]["l1_same_states"]
    res["l1_same_states_truncated_at_n_in_fp32"] = same32[n_in]
    zero = np.zeros((1, tnr - n_in, 2))
    res["l1_same_states_zero_tail_fp32"] = _l1_mean(extend(c32[:, :n_in + 1], zero), c64,
                                                    e_range)
    n64 = _steps_to_reach(same64, target_l1)
    n32 = _steps_to_reach(same32, target_l1)
    learned_ok = best[1]["l1_same_states"] < target_l1
    per64, per32 = t64 / tnr, t32 / tnr
    res["time_to_dos"] = {
        "plain_fp64": {"steps": n64, "seconds": n64 * per64 if n64 else None},
        "fp32": {"steps": n32, "seconds": n32 * per32 if n32 else None},
        "fp32_learned": {"reached": learned_ok, "steps": n_in if learned_ok else None,
                         "seconds": n_in * per32 if learned_ok else None},
    }
    if n64 and learned_ok:
        res["time_to_dos_speedup_learned_vs_plain_fp64"] = (n64 * per64) / (n_in * per32)
    if n64 and n32:
        res["time_to_dos_speedup_fp32_vs_plain_fp64"] = (n64 * per64) / (n32 * per32)
    return res


RUNNERS = {"c1": run_c1, "c2": run_c2, "c3": run_c3, "c4": run_c4, "c4c": run_c4c, "c4l": run_c4l,
           "c5": run_c5, "c5l": run_c5l}


def main(argv=None) -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("workloads", nargs="+", choices=sorted(RUNNERS))
    ap.add_argument("--steps", type=int, default=None,
                    help="override the number of time steps (shorter runs)")
    ap.add_argument("--out", default=None)
    ap.add_argument("--data", default=None, help="c4, c5l: npz cache of the generated curves")
    ap.add_argument("--epochs", type=int, default=None, help="c4, c5l: training epochs")
    ap.add_argument("--n-train", type=int, default=None,
                    help="c4: training realisations (curves = realisations x states)")
    ap.add_argument("--n-states", type=int, default=None,
                    help="c4: states per realisation (training and test)")
    ap.add_argument("--builder", default="device", choices=["device", "host"],
                    help="c5: assemble the Hamiltonian on the GPU or on the host")
    ap.add_argument("--nx", type=int, default=None,
                    help="c5: cells per side (default 4096)")
    ap.add_argument("--energy-limits", type=float, nargs=2, default=None,
                    help="c5: energy window of the DC conductivity in eV (default -0.5 0.5); "
                         "the quasi-eigenstate block holds N x energies x states values")
    args = ap.parse_args(argv)
    for w in args.workloads:
        kw = {}
        if w == "c5l" and args.n_train:
            kw["n_train"] = args.n_train
        if w in ("c4", "c5l") and args.epochs:
            kw["epochs"] = args.epochs
        if w == "c5l" and args.data:
            kw["data"] = args.data
        if args.steps and w != "c5l":
            kw = {"steps": args.steps} if w in ("c1", "c3", "c5") else \
                 {"steps_dos": args.steps, "steps_ac": args.steps}
        if w == "c4" and args.data:
            kw["data"] = args.data
        if w == "c4" and args.n_train:
            kw["n_train"] = args.n_train
        if w == "c4" and args.n_states:
            kw["n_states"] = args.n_states
        if w == "c5":
            kw["builder"] = args.builder
            if args.nx:
                kw["nx"] = args.nx
            if args.energy_limits:
                kw["energy_limits"] = tuple(args.energy_limits)
        r = RUNNERS[w](**kw)
        line = json.dumps(r)
        print(line, flush=True)
        if args.out:
            with open(args.out, "a") as f:
                f.write(line + "\n")


if __name__ == "__main__":
    main(sys.argv[1:])
