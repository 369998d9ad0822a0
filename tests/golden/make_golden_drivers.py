"""Generate tests/golden/reference_drivers.npz from the reference TBPLaS.

Run in a container that holds the reference source tree (read-only):

    python tests/golden/make_golden_drivers.py --ref <reference tree> --scratch <scratch dir>

As make_golden.py, it imports the reference package from a scratch copy with
the CPU oracle of this repository behind `tbplas.fortran.f2py` (the
reference's Fortran cannot be compiled here) and injected initial states.  It
records what the reference's own Solver passes through the f2py layer and
gets back for calc_corr_dyn_pol, calc_quasi_eigenstates, calc_hall_mu and
calc_ldos_haydock, and what the reference's Analyzer computes from those
results: calc_dyn_pol, calc_epsilon, calc_epsilon_q0 and calc_hall_cond.
"""

import argparse
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, HERE)

from make_golden import install_shims, prepare_scratch  # noqa: E402


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="root of the reference source tree")
    ap.add_argument("--scratch", required=True,
                    help="scratch directory for the cythonized copy of the reference")
    ap.add_argument("--out", default=os.path.join(HERE, "reference_drivers.npz"))
    args = ap.parse_args()

    from oracle import oracle
    shim_obj = oracle.F2pyShim()
    shim = types.ModuleType("tbplas.fortran.f2py")
    for name in ("tbpm_dos", "tbpm_accond", "tbpm_dccond", "tbpm_psi_t", "tbpm_dyn_pol",
                 "tbpm_eigenstates", "tbpm_kbdc", "ldos_haydock", "cond_from_trace"):
        setattr(shim, name, getattr(shim_obj, name))
    prepare_scratch(args.ref, args.scratch)
    install_shims(shim)
    sys.path.insert(0, args.scratch)
    import tbplas as tb

    out = {}
    rng = np.random.default_rng(4242)
    cell = tb.make_graphene_diamond()
    sc = tb.SuperCell(cell, dim=(8, 7, 1), pbc=(True, True, False))
    s = tb.Sample(sc)
    s.init_orb_eng()
    s.orb_eng += rng.uniform(-0.5, 0.5, s.orb_eng.size)
    out["disorder"] = s.orb_eng.copy()
    s.rescale_ham(9.0)
    n = s.build_ham_csr().shape[0]
    states = np.exp(2j * np.pi * rng.random((2, n)))
    states /= np.linalg.norm(states, axis=1, keepdims=True)
    out["states"] = states
    shim_obj.states = states

    cfg = tb.Config()
    cfg.generic["nr_time_steps"] = 32
    cfg.generic["nr_random_samples"] = 2
    cfg.dyn_pol["q_points"] = [[1.0, 0.0, 0.0], [0.5, 0.8, 0.0], [0.0, 0.0, 0.0]]
    cfg.dyn_pol["background_dielectric_constant"] = 2.5
    cfg.quasi_eigenstates["energies"] = [-0.3, 0.0, 0.2]
    cfg.dckb["n_kernel"] = 48
    cfg.dckb["ne_integral"] = 128
    cfg.dckb["energies"] = [-0.2, -0.1, 0.0, 0.1, 0.2]
    cfg.LDOS["site_indices"] = [3, 40]
    cfg.LDOS["recursion_depth"] = 30
    cfg.LDOS["delta"] = 0.05
    solver = tb.Solver(s, cfg, prefix="golden", directory=os.path.join(args.scratch, "sim"))
    out["dyn_pol/corr"] = solver.calc_corr_dyn_pol()
    out["qe/states"] = solver.calc_quasi_eigenstates()
    for d in (1, 2):
        cfg.dckb["direction"] = d
        out[f"hall/mu_mn_dir{d}"] = solver.calc_hall_mu()
    en, ldos = solver.calc_ldos_haydock()
    out["haydock/energies"] = en
    out["haydock/ldos"] = ldos
    out["orb_pos"] = s.orb_pos
    for dim in (2, 3):
        an = tb.Analyzer(s, cfg, dimension=dim)
        q, om, dp = an.calc_dyn_pol(out["dyn_pol/corr"])
        out[f"analyzer/dim{dim}/q_points"] = q
        out[f"analyzer/dim{dim}/omegas"] = om
        out[f"analyzer/dim{dim}/dyn_pol"] = dp
        out[f"analyzer/dim{dim}/epsilon"] = an.calc_epsilon(dp)
        for unit in ("h_bar", "h"):
            e, c = an.calc_hall_cond(out["hall/mu_mn_dir2"], unit=unit)
            out[f"analyzer/dim{dim}/hall_{unit}"] = c
        out[f"analyzer/dim{dim}/hall_energies"] = e
    an3 = tb.Analyzer(s, cfg, dimension=3)
    omegas = np.linspace(0.1, 2.0, 11)
    ac = rng.standard_normal((4, 11)) + 1j * rng.standard_normal((4, 11))
    out["analyzer/eps_q0/omegas"] = omegas
    out["analyzer/eps_q0/ac"] = ac
    out["analyzer/eps_q0/eps"] = an3.calc_epsilon_q0(omegas, ac)
    np.savez_compressed(args.out, **out)
    print(f"wrote {args.out}: {len(out)} arrays, {os.path.getsize(args.out) / 1024:.1f} KiB")


if __name__ == "__main__":
    main()
