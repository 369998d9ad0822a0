"""Benchmark of the TBPM hot path on B200.

Workload (the headline configuration): graphene 2048 x 2048 periodic
supercell (8,388,608 orbitals), t = -2.7 eV, Anderson on-site disorder
U[-0.5, 0.5] eV, rescale 9 eV (nnz = 33.5M), 16 random-phase states
propagated as one block; one bench step = one TBPM time step of the DOS
correlation (19 Chebyshev terms + the fused correlation) for the whole block.

  value   orbital-steps/s on the device (state block and Hamiltonian resident
          in HBM), CUDA events on the library stream, max over ranks
  e2e     the same metric through the public API f2py.tbpm_dos (host CSR and
          host result buffers; uploads, state generation, propagation and the
          result download inside the timed region)
  roofline  algorithmic HBM bytes of the Chebyshev-term kernel family per
          step / measured step time, against the measured HBM copy bandwidth
  cpu_baseline  the CPU oracle (C++/OpenMP restatement of the reference
          Fortran) on this host's cores, bounded sample of the same workload

  ac      the AC-conductivity time step of the same workload (48-column block
          [J_x psi | J_y psi | psi] of the 16 states: time-step expansion +
          the current correlations), device time per step from CUDA events
          around two f2py.tbpm_accond calls of different lengths (their set-up,
          Fermi operators included, cancels in the difference)
  parity  the first two time steps of two state columns of the timed session,
          against the CPU oracle on the same Hamiltonian and states

`--impl reference` times the CPU oracle alone (the reference Fortran cannot be
built on this image) and prints its own JSON line.

Multi-GPU: `--gpus N` without a torchrun environment re-launches this script
under torch.distributed.run with N ranks (one process per GPU, NCCL).  Every
rank propagates its own 16 states (weak scaling, the reference's random-sample
decomposition, seeds offset by rank); the correlation arrays are averaged with
one all_reduce at the end of the e2e call, the only data-path collective.
"""

import argparse
import json
import math
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NX = NY = 2048
N_STATES = 16
DISORDER_W = 1.0
RESCALE = 9.0
SEED = 1337
HBM_FALLBACK_GBS = 6650.0
# DRAM bytes (ncu dram__bytes_read.sum + dram__bytes_write.sum) over the
# algorithmic bytes of the same launches of the ring kernel, measured with ncu
# on the 1024x1024 case of this workload (0.985 in both the recurrence-only and
# the flush mode); traffic scales with the rows.
TRAFFIC_OVER_ALGORITHMIC_FP64 = 0.985
PARITY_TOL = 1e-10


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


def bessel_series(time_scaled, precision=1e-14):
    import scipy.special as spec
    out = []
    for i in range(250):
        v = spec.jv(i, time_scaled)
        if abs(v) > precision or abs(spec.jv(i + 1, time_scaled)) > precision:
            out.append(float(v))
        else:
            return out
    raise ValueError("Bessel_max too low")


def build_sample():
    import tbplas_b200 as tb
    t0 = time.time()
    s = tb.make_graphene_sample(NX, NY, disorder=DISORDER_W, rescale=RESCALE, seed=SEED)
    h = s.build_ham_csr()
    log(f"[bench] built {NX}x{NY} graphene: N={h.shape[0]} nnz={h.nnz} in {time.time() - t0:.1f}s")
    return s, h


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = os.path.join("/tmp", f"tbpm_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        rows = []
        with open(self.path) as f:
            for line in f:
                p = [x.strip() for x in line.split(",")]
                if len(p) >= 9:
                    rows.append(p)
        os.remove(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def algorithmic_bytes_per_step(n, nnz, ld, n_bes, real_bytes, paired=False, with_ref=True):
    """HBM bytes one time step of the fused kernel family must move.

    Per Chebyshev term k = 1..n_bes-1 the kernel reads the CSR once
    ((n+1)*4 + nnz*(4 + 2*real_bytes)) and the gathered vector p_{k-1} once
    (neighbour rows come from L2), reads p_{k-2} and writes p_k (not on the
    first and last term), and every third term flushes the accumulator
    (read + write; write only on the first flush); the last term also reads
    the correlation reference (with_ref).  With paired terms (two terms per
    launch) the second term of a pair reads p_k, its own rows of p_{k-1} and
    the CSR from L2: the pair saves the CSR and two vector passes.  Pairs are
    (1, 2), (3, 4), ... except a last term with the correlation and two flush
    terms in a row.  This mirrors the schedule of enqueue_expansion in
    tbplas_b200/csrc/tbpm_engine.cu.
    """
    sv = 2 * real_bytes
    vec = n * ld * sv
    mat = (n + 1) * 4 + nnz * (4 + sv)
    term, flush = {}, {}
    last_flush = -1
    for k in range(1, n_bes):
        b = mat + vec
        fl = False
        if k == 1:
            b += vec
        else:
            b += vec * (2 if k < n_bes - 1 else 1)
            pending = k - last_flush
            if k == 2 or pending == 3 or k == n_bes - 1:
                b += vec * (1 if k == 2 else 2)
                last_flush = k
                fl = True
        if k == n_bes - 1 and with_ref:
            b += vec  # correlation reference wf0
        term[k], flush[k] = b, fl
    total = 0.0
    k = 1
    while k < n_bes:
        if (paired and k + 1 < n_bes and not (with_ref and k + 1 == n_bes - 1)
                and not (flush[k] and flush[k + 1])):
            total += term[k] + term[k + 1] - mat - 2 * vec
            k += 2
        else:
            total += term[k]
            k += 1
    return total


def survey_model_bytes_per_orbital_step(n, nnz, ld, n_bes, real_bytes):
    """The 5-passes-per-term byte model (M + B*5*S_v*N per term + S_v)."""
    sv = 2 * real_bytes
    m = n * (nnz / n) * (sv + 4) + 4 * (n + 1)
    return ((n_bes - 1) * (m / (n * ld) + 5 * sv) + sv)


def ac_algorithmic_bytes_per_step(n, nnz, nb, n_bes, real_bytes, paired=False):
    """HBM bytes of one AC time step: the time-step expansion of the
    3*nb-column block (no correlation reference on its last term) plus the
    current-correlation pass, which reads the CSR with hop, dx and dy once
    and every column of the block once."""
    ld = 3 * nb
    sv = 2 * real_bytes
    exp = algorithmic_bytes_per_step(n, nnz, ld, n_bes, real_bytes, paired=paired,
                                     with_ref=False)
    jcorr = (n + 1) * 4 + nnz * (4 + sv + 2 * real_bytes) + n * ld * sv
    return exp + jcorr


def free_port():
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def torchrun_command(n_gpus, port, argv):
    """The command that runs this script as n_gpus ranks on one node."""
    return [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
            f"--nproc-per-node={int(n_gpus)}", "--master-addr", "127.0.0.1",
            f"--master-port={int(port)}", os.path.abspath(__file__)] + list(argv)


def launch_ranks(n_gpus, argv):
    """Re-run this script under torch.distributed.run with n_gpus ranks; NCCL
    reports its communicators (NCCL_DEBUG=INFO) on stderr, so stdout keeps the
    one JSON line of rank 0."""
    env = dict(os.environ)
    env.setdefault("NCCL_DEBUG", "INFO")
    env.setdefault("NCCL_DEBUG_SUBSYS", "INIT")
    env.setdefault("NCCL_DEBUG_FILE", "/dev/stderr")
    cmd = torchrun_command(n_gpus, free_port(), argv)
    log("[bench] launching", " ".join(cmd))
    return subprocess.call(cmd, env=env)


def gather_rank_values(value, dist, device):
    """(max over ranks, per-rank list) of a float, every rank taking part."""
    import torch
    world = dist.get_world_size()
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    parts = [torch.zeros_like(t) for _ in range(world)]
    dist.all_gather(parts, t)
    vals = [float(p.item()) for p in parts]
    return max(vals), vals


def parity_spot_check(ip, ix, hv, bes, corr_rows, rank, columns=(0, 1), steps=2):
    """Relative error (max |diff| / max |oracle|) of the first `steps` time steps
    of session columns against the CPU oracle with the same states: column b
    of the session holds iseed = SEED * (1 + b + rank * N_STATES)."""
    from oracle import oracle
    n = ip.size - 1
    worst = 0.0
    for b in columns:
        wf0 = oracle.random_state(n, SEED * (1 + b + rank * N_STATES), 0)
        ref = oracle.tbpm_dos(bes, ip, ix, hv, steps, wf0=wf0, chk_step=0)
        got = corr_rows[:steps + 1, b]
        worst = max(worst, float(np.max(np.abs(got - ref)) / np.max(np.abs(ref))))
    return worst


def time_ac(args, sample, rank, local, peak, paired):
    """Device time per AC time step (FP64, 16 states, 48-column block)."""
    import torch
    from tbplas_b200 import KB
    from tbplas_b200.fortran import f2py
    ip, ix, hv, dx, dy = sample.build_ham_dxy()
    ip = ip.astype(np.int32)
    ix = ix.astype(np.int32)
    n, nnz = ip.size - 1, ix.size
    bes = np.asarray(bessel_series(math.pi / 2))
    beta = sample.rescale / (KB * 300.0)
    G = 16
    f2py.set_backend(precision="fp64", batch=N_STATES, device=local, use_graphs=True,
                     steps_per_graph=G, vector_width=0, threads_per_block=0,
                     term_kernel=args.term_kernel)
    ctx = f2py._ctx()
    stream = torch.cuda.ExternalStream(ctx.stream)

    def run(tnr):
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        ev0.record(stream)
        f2py.tbpm_accond(bes, beta, 0.0, ip, ix, hv, sample.rescale, dx, dy, SEED, tnr,
                         N_STATES, 2 ** 15, 1e-12, "unused", rank, tnr + 1, 1e-9)
        ev1.record(stream)
        torch.cuda.synchronize()
        return ev0.elapsed_time(ev1)

    # t_n = 1 + (n - 1) propagated steps; both lengths replay whole graphs plus
    # the same remainder, so capture and set-up cancel in the difference
    short = 1 + G + 3
    extra = G * max(1, args.ac_graphs)
    run(short)  # warm-up (uploads, Fermi coefficients, capture)
    t1 = run(short)
    t2 = run(short + extra)
    ms = (t2 - t1) / extra
    alg = ac_algorithmic_bytes_per_step(n, nnz, N_STATES, bes.size, 8, paired=paired)
    gbs = alg / (ms * 1e-3) / 1e9
    return {"ms_per_step": ms, "orbital_steps_per_s": n * N_STATES / (ms * 1e-3),
            "alg_bytes_per_step": alg, "achieved_gbs": gbs, "roofline_frac": gbs / peak,
            "block_columns": 3 * N_STATES, "bessel_terms": int(bes.size),
            "method": f"CUDA events around f2py.tbpm_accond of {short} and {short + extra} "
                      f"time steps; ({extra} steps) / difference"}


def run_gpu(args):
    import torch
    import torch.distributed as dist
    from tbplas_b200 import _native as nat
    from tbplas_b200.fortran import f2py
    from tbplas_b200.parallel import init_distributed

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    distributed = world > 1
    torch.cuda.set_device(local)
    if distributed:
        init_distributed(backend="nccl", timeout_s=300)
    dev = torch.device("cuda", local)
    peak, peak_kind = measured_peak()

    sample, h = build_sample()
    n, nnz = h.shape[0], h.nnz
    ip = h.indptr.astype(np.int32)
    ix = h.indices.astype(np.int32)
    hv = np.ascontiguousarray(h.data)
    bes = np.asarray(bessel_series(2 * math.pi / sample.energy_range * sample.rescale))
    n_bes = bes.size
    G = 16  # time steps per captured CUDA graph

    ctx = nat.get_context(local)
    results = {}
    fp64_rows = None
    for prec_name, prec in (("fp64", nat.PREC_FP64), ("fp32", nat.PREC_FP32)):
        if prec_name == "fp32" and args.skip_fp32:
            continue
        ctx.set_options(precision=prec, batch=N_STATES, use_graphs=1, steps_per_graph=G,
                        vector_width=args.vector_width if prec_name == "fp64" else 0,
                        threads_per_block=args.threads if prec_name == "fp64" else 0,
                        term_kernel=args.term_kernel)
        ctx.call("tbpm_ham_upload", nat.ptr(ip), nat.ptr(ix), nat.ptr(hv), n, nnz, None, None,
                 sample.rescale)
        total = args.steps + args.warmup
        # the session captures and uploads its step graph here, outside the timing
        ctx.call("tbpm_session_dos_begin", nat.ptr(bes), n_bes, N_STATES, SEED, rank, N_STATES,
                 total)
        stream = torch.cuda.ExternalStream(ctx.stream)
        ctx.call("tbpm_session_advance", args.warmup)
        torch.cuda.synchronize()
        if distributed:
            dist.barrier()
        torch.cuda.synchronize()
        sampler = ClockSampler(local) if (rank == 0 and prec_name == "fp64") else None
        if sampler:
            sampler.start()
            time.sleep(0.3)
        l0, b0 = ctx.last_stats()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        ctx.call("tbpm_session_advance", args.steps)
        ev1.record(stream)
        torch.cuda.synchronize()
        l1, b1 = ctx.last_stats()
        if distributed:
            dist.barrier()
        torch.cuda.synchronize()
        clocks = sampler.stop() if sampler else None
        ms = ev0.elapsed_time(ev1)
        per_rank = [ms]
        if distributed:
            ms, per_rank = gather_rank_values(ms, dist, dev)
        ms_step = ms / args.steps
        launches = (l1 - l0)
        model_bytes_step = (b1 - b0) / args.steps
        rb = 8 if prec == nat.PREC_FP64 else 4
        # the library ran two terms per launch where its byte count matches
        # the paired schedule
        alg_single = algorithmic_bytes_per_step(n, nnz, N_STATES, n_bes, rb)
        alg_paired = algorithmic_bytes_per_step(n, nnz, N_STATES, n_bes, rb, paired=True)
        paired = abs(model_bytes_step - alg_paired) < abs(model_bytes_step - alg_single)
        alg = alg_paired if paired else alg_single
        corr = np.zeros((total + 1, N_STATES), dtype=np.complex128)
        norms = np.zeros((total + 1, N_STATES))
        import ctypes
        nd = ctypes.c_int(0)
        ctx.call("tbpm_session_read", nat.ptr(corr), nat.ptr(norms), ctypes.byref(nd))
        if prec_name == "fp64":
            fp64_rows = corr
        results[prec_name] = {
            "ms_per_step": ms_step,
            "per_rank_ms_per_step": [v / args.steps for v in per_rank],
            "orbital_steps_per_s": n * N_STATES * world / (ms_step * 1e-3),
            "launches": launches,
            "alg_bytes_per_step": alg,
            "alg_bytes_per_step_single_terms": alg_single,
            "paired_terms": bool(paired),
            "lib_model_bytes_per_step": model_bytes_step,
            "achieved_gbs": alg / (ms_step * 1e-3) / 1e9,
            "norm_drift": float(np.max(np.abs(norms[:nd.value] - norms[0]))),
            "clocks": clocks,
        }
        log(f"[bench] {prec_name}: {ms_step:.3f} ms/step, "
            f"{results[prec_name]['orbital_steps_per_s']:.3e} orbital-steps/s, "
            f"{results[prec_name]['achieved_gbs']:.0f} GB/s, launches {launches}")

    # ---- e2e through the public API (FP64, host buffers) -----------------
    f2py.set_backend(precision="fp64", batch=N_STATES, device=local, use_graphs=True,
                     steps_per_graph=G, vector_width=args.vector_width,
                     threads_per_block=args.threads, term_kernel=args.term_kernel)
    from tbplas_b200.parallel import MPIEnv
    env = MPIEnv(enable_mpi=distributed)
    e2e_steps = args.steps
    torch.cuda.synchronize()
    if distributed:
        dist.barrier()
    t0 = time.perf_counter()
    corr = f2py.tbpm_dos(bes, ip, ix, hv, SEED, e2e_steps, N_STATES, "unused", rank, 128, 1e-9)
    corr = env.all_average(corr)
    torch.cuda.synchronize()
    t_e2e = time.perf_counter() - t0
    if distributed:
        t_e2e, _ = gather_rank_values(t_e2e, dist, dev)
    h2d = ip.nbytes + ix.nbytes + hv.nbytes + bes.nbytes
    d2h = corr.nbytes
    e2e = {"value": n * N_STATES * e2e_steps * world / t_e2e, "unit": "orbital-steps/s",
           "h2d_bytes_per_step": h2d / e2e_steps, "d2h_bytes_per_step": d2h / e2e_steps,
           "steps": e2e_steps, "seconds": t_e2e,
           "note": "one f2py.tbpm_dos call of `steps` time steps per rank: CSR upload and "
                   "validation, state generation, propagation, result download"
                   + (", then the NCCL all_average of the correlation" if distributed else "")}

    # ---- AC time step of the same workload (FP64) -------------------------
    ac = None
    if not args.skip_ac:
        ac = time_ac(args, sample, rank, local, peak, results["fp64"]["paired_terms"])
        if distributed:
            ac_ms, ac_ranks = gather_rank_values(ac["ms_per_step"], dist, dev)
            ac["ms_per_step"] = ac_ms
            ac["per_rank_ms_per_step"] = ac_ranks
            ac["orbital_steps_per_s"] = n * N_STATES * world / (ac_ms * 1e-3)
            ac["achieved_gbs"] = ac["alg_bytes_per_step"] / (ac_ms * 1e-3) / 1e9
            ac["roofline_frac"] = ac["achieved_gbs"] / peak
        log(f"[bench] ac fp64: {ac['ms_per_step']:.3f} ms/step, {ac['achieved_gbs']:.0f} GB/s")

    # ---- parity of the timed session against the oracle -------------------
    parity = None
    if rank == 0 and not args.skip_parity:
        t0 = time.perf_counter()
        err = parity_spot_check(ip, ix, hv, bes, fp64_rows, rank)
        parity = {"rel_err": err, "tol": PARITY_TOL, "ok": bool(err <= PARITY_TOL),
                  "what": "FP64 session columns 0 and 1, time steps 0..2, vs the CPU oracle "
                          "with the same states (max |diff| / max |oracle|)",
                  "seconds": time.perf_counter() - t0}
        log(f"[bench] parity vs oracle: {err:.3e}")

    cpu = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        cpu = cpu_baseline(ip, ix, hv, bes, args.cpu_steps)

    if rank == 0:
        r64 = results["fp64"]
        line = {
            "metric": "orbital-steps/s (TBPM DOS time step, FP64)",
            "value": r64["orbital_steps_per_s"],
            "unit": "orbital-steps/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": r64["ms_per_step"],
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64 (complex128 states, SpMV and reductions)",
            "data": "synthetic: graphene supercell with seeded Anderson disorder and "
                    "seeded Philox random-phase states",
            "config": {"workload": "graphene 2048x2048 PBC, W=1 eV Anderson disorder, "
                                   "16 states as one block, corr_dos time step",
                       "n_orbitals": n, "nnz": nnz, "states_per_gpu": N_STATES,
                       "bessel_terms": n_bes, "rescale_eV": RESCALE,
                       "l2": "inputs larger than L2 (state block 2.1 GB FP64)",
                       "steps_per_graph": G,
                       "parallelism": f"replicas of independent state blocks x{world}"},
            "roofline": {
                "bound": "hbm",
                "achieved": r64["achieved_gbs"],
                "peak": peak,
                "unit": "GB/s",
                "frac": r64["achieved_gbs"] / peak,
                "peak_kind": peak_kind,
                "traffic": r64["alg_bytes_per_step"] * TRAFFIC_OVER_ALGORITHMIC_FP64,
                "traffic_note": "bytes per step: ncu DRAM bytes / algorithmic bytes = 0.985 on "
                                "the 1024x1024 case, scaled by rows to this workload",
                "alg_bytes_per_step": r64["alg_bytes_per_step"],
                "kernel": ("cheb_term_kernel<double,2,MODE>" if args.term_kernel == 1 else
                           "cheb_pair_kernel<double,2> + cheb_ring_kernel<double,2,2>"
                           if r64["paired_terms"] else "cheb_ring_kernel<double,2,MODE>") +
                          " (+ finalize_kernel, <1% of step)",
            },
            "e2e": e2e,
            "gpu_launches": int(r64["launches"]),
            "clocks": r64["clocks"],
            "per_rank_ms_per_step": r64["per_rank_ms_per_step"],
            "fp32": {k: results["fp32"][k] for k in ("ms_per_step", "orbital_steps_per_s",
                                                      "achieved_gbs", "alg_bytes_per_step")}
            if "fp32" in results else None,
            "ac": ac,
            "parity": parity,
            "cpu_baseline": cpu,
        }
        if "fp32" in results:
            line["fp32"]["roofline_frac"] = results["fp32"]["achieved_gbs"] / peak
            t64, t32 = r64["ms_per_step"], results["fp32"]["ms_per_step"]
            line["time_to_dos"] = {
                "target_l1": 1e-3,
                "fp64_ms_per_step": t64, "fp32_ms_per_step": t32,
                "fp32_batched_vs_plain_fp64": t64 / t32,
                "learned_vs_plain_fp64": None,
                "note": "DOS L1 of FP32 states against FP64 at full length is 5e-7, so both "
                        "reach L1 < 1e-3 only at the full horizon and the time-to-DOS ratio "
                        "is the ratio of step times on this workload. The learned tail does "
                        "not shorten the horizon on the W ~ U[0,3] eV 512^2 workload: trained "
                        "on 20,000 curves it reaches L1 = 0.0099, not 1e-3 (the tail beyond "
                        "256 steps is per-state noise); where the "
                        "tail is deterministic (weak disorder) it reached L1 < 1e-3 13x "
                        "faster than plain FP64 in a separate measurement, and in the "
                        "77 T field of 4096^2 graphene (Landau-level oscillations) it reaches "
                        "L1 = 1.7e-3 from 256 steps, which plain FP64 needs ~1920 steps "
                        "for (~14x), but not 1e-3. Below the 3x target on the specified "
                        "workload.",
            }
        print(json.dumps(line), flush=True)
    if distributed:
        dist.barrier()
        dist.destroy_process_group()


def cpu_baseline(ip, ix, hv, bes, steps):
    """The oracle (C++/OpenMP restatement of the reference Fortran) on all host
    cores: 1 random state of the same Hamiltonian, `steps` time steps."""
    from oracle import oracle
    L = oracle.lib(native=True)
    import ctypes
    threads = os.cpu_count() or 1
    L.orc_set_threads(threads)
    n = ip.size - 1
    wf0 = np.ascontiguousarray(oracle.random_state(n, SEED, 0)[None, :])
    corr = np.zeros(steps + 1, dtype=np.complex128)
    b = np.ascontiguousarray(bes)
    t0 = time.perf_counter()
    rc = L.orc_tbpm_dos(b.ctypes.data, b.size, ip.ctypes.data, ix.ctypes.data, hv.ctypes.data,
                        n, wf0.ctypes.data, SEED, steps, 1, 0, 0, 1e-9, 0, corr.ctypes.data)
    dt = time.perf_counter() - t0
    if rc != 0:
        return None
    return {"value": n * steps / dt, "unit": "orbital-steps/s", "cores": threads,
            "kind": "port",
            "sample": f"1 state x {steps} time steps of the 2048x2048 disordered graphene "
                      f"Hamiltonian (the benchmark uses 16 states per GPU), {dt:.1f} s"}


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle
    sample, h = build_sample()
    ip = h.indptr.astype(np.int32)
    ix = h.indices.astype(np.int32)
    hv = np.ascontiguousarray(h.data)
    n = ip.size - 1
    bes = np.asarray(bessel_series(2 * math.pi / sample.energy_range * sample.rescale))
    L = oracle.lib(native=True)
    threads = os.cpu_count() or 1
    L.orc_set_threads(threads)
    wf0 = np.ascontiguousarray(oracle.random_state(n, SEED, 0)[None, :])
    # one step of the reference arm = one time step of one state
    corr = np.zeros(args.steps + args.warmup + 1, dtype=np.complex128)
    L.orc_tbpm_dos(bes.ctypes.data, bes.size, ip.ctypes.data, ix.ctypes.data, hv.ctypes.data,
                   n, wf0.ctypes.data, SEED, args.warmup, 1, 0, 0, 1e-9, 0, corr.ctypes.data)
    t0 = time.perf_counter()
    L.orc_tbpm_dos(bes.ctypes.data, bes.size, ip.ctypes.data, ix.ctypes.data, hv.ctypes.data,
                   n, wf0.ctypes.data, SEED, args.steps, 1, 0, 0, 1e-9, 0, corr.ctypes.data)
    dt = time.perf_counter() - t0
    value = n * args.steps / dt
    line = {
        "impl": "reference",
        "metric": "orbital-steps/s (TBPM DOS time step, FP64)",
        "value": value,
        "unit": "orbital-steps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": dt / args.steps * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64 (complex128)",
        "data": "synthetic: graphene supercell with seeded Anderson disorder",
        "config": {"workload": "graphene 2048x2048 PBC, W=1 eV Anderson disorder, "
                               "corr_dos time step (1 state per step on the CPU)",
                   "n_orbitals": n, "nnz": int(ix.size)},
        "cpu_baseline": {"value": value, "unit": "orbital-steps/s", "cores": threads,
                         "kind": "port",
                         "sample": f"1 state x {args.steps} time steps (reference Fortran "
                                   f"not buildable here: C++/OpenMP restatement)"},
        "e2e": {"value": value, "unit": "orbital-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=64)
    ap.add_argument("--warmup", type=int, default=4)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-steps", type=int, default=8)
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-fp32", action="store_true")
    ap.add_argument("--skip-ac", action="store_true")
    ap.add_argument("--skip-parity", action="store_true")
    ap.add_argument("--ac-graphs", type=int, default=2,
                    help="16-step graphs in the difference of the AC timing")
    ap.add_argument("--vector-width", type=int, default=0, choices=[0, 1, 2],
                    help="FP64 complex values per thread: 0 library default (two, 256-bit "
                         "accesses), 1 one (128-bit accesses), 2 two")
    ap.add_argument("--term-kernel", type=int, default=0, choices=[0, 1, 2, 3, 4],
                    help="Chebyshev-term kernel: 0 library default (shared-memory ring fed by "
                         "bulk copies), 1 grid-stride kernel with plain loads, 2 ring, 3 two "
                         "terms per launch, 4 ring with row windows")
    ap.add_argument("--threads", type=int, default=0,
                    help="FP64 threads per block of the term kernel (0: library default)")
    ap.add_argument("--nx", type=int, default=2048,
                    help="cells along a1 (smaller values only for profiling captures)")
    ap.add_argument("--ny", type=int, default=2048)
    args = ap.parse_args()
    global NX, NY
    NX, NY = args.nx, args.ny
    if args.warmup < 3:
        args.warmup = 3
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # one process per GPU: re-run under torch.distributed.run
        sys.exit(launch_ranks(args.gpus, sys.argv[1:]))
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
