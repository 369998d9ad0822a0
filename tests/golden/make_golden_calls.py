"""Record the reference Solver's own calls into its f2py core.

Run in a container that holds the reference source tree (read-only):

    python tests/golden/make_golden_calls.py --ref <reference tree> --scratch <scratch dir>

The reference package is prepared and imported as make_golden.py does
(cythonized copy, stub matplotlib, scipy alias), with `tbplas.fortran.f2py`
replaced by a recording module: every call the reference's Solver makes
(calc_corr_dos, calc_corr_ac_cond, calc_corr_dc_cond, calc_psi_t,
calc_corr_dyn_pol) is passed to the CPU oracle's f2py-compatible shim, and its
positional arguments, exactly as the Solver builds them (array dtypes and
shapes included), and the oracle's result are written to
tests/golden/reference_calls.npz.  A GPU test replays each recorded call
through tbplas_b200.fortran.f2py: the drop-in must accept the reference
Solver's argument lists as they are and return the oracle's results.
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
    ap.add_argument("--out", default=os.path.join(HERE, "reference_calls.npz"))
    args = ap.parse_args()

    from oracle import oracle
    shim_obj = oracle.F2pyShim()
    out = {}
    calls = []

    def recorder(name):
        fn = getattr(shim_obj, name)

        def call(*a):
            k = len(calls)
            calls.append(name)
            kinds = []
            for i, v in enumerate(a):
                if isinstance(v, np.ndarray):
                    out[f"call{k}/arg{i}"] = v
                    kinds.append("array")
                elif isinstance(v, (list, tuple)):
                    out[f"call{k}/arg{i}"] = np.asarray(v)
                    kinds.append("list")
                elif isinstance(v, str):
                    out[f"call{k}/arg{i}"] = np.array(v)
                    kinds.append("str")
                elif isinstance(v, (bool, np.bool_)):
                    out[f"call{k}/arg{i}"] = np.array(int(v))
                    kinds.append("int")
                elif isinstance(v, (int, np.integer)):
                    out[f"call{k}/arg{i}"] = np.array(int(v))
                    kinds.append("int")
                else:
                    out[f"call{k}/arg{i}"] = np.array(float(v))
                    kinds.append("float")
            out[f"call{k}/kinds"] = np.array(kinds)
            res = fn(*a)
            if isinstance(res, tuple):
                for j, r in enumerate(res):
                    out[f"call{k}/result{j}"] = r
                out[f"call{k}/n_results"] = np.array(len(res))
            else:
                out[f"call{k}/result0"] = res
                out[f"call{k}/n_results"] = np.array(1)
            return res
        return call

    shim = types.ModuleType("tbplas.fortran.f2py")
    for name in ("tbpm_dos", "tbpm_accond", "tbpm_dccond", "tbpm_psi_t", "tbpm_dyn_pol"):
        setattr(shim, name, recorder(name))

    prepare_scratch(args.ref, args.scratch)
    install_shims(shim)
    sys.path.insert(0, args.scratch)
    import tbplas as tb

    rng = np.random.default_rng(20241203)
    cell = tb.make_graphene_diamond()
    sc = tb.SuperCell(cell, dim=(9, 7, 1), pbc=(True, True, False))
    s = tb.Sample(sc)
    s.init_orb_eng()
    s.orb_eng += rng.uniform(-0.5, 0.5, s.orb_eng.size)
    s.rescale_ham(9.0)
    out["sample/orb_eng"] = s.orb_eng.copy()

    config = tb.Config()
    config.generic["nr_time_steps"] = 48
    config.generic["nr_random_samples"] = 3
    config.generic["wfn_check_steps"] = 16
    config.DC_conductivity["energy_limits"] = (-1.5, 1.5)
    config.dyn_pol["q_points"] = [[1.0, 0.0, 0.0], [0.3, 0.4, 0.0]]
    solver = tb.Solver(s, config, prefix="calls", directory=os.path.join(args.scratch, "calls"))
    solver.calc_corr_dos()
    solver.calc_corr_ac_cond()
    solver.calc_corr_dc_cond()
    solver.calc_corr_dyn_pol()
    psi0 = np.exp(2j * np.pi * rng.random(s.build_ham_csr().shape[0]))
    psi0 /= np.linalg.norm(psi0)
    solver.calc_psi_t(psi0, [0, 5, 17, 48])
    out["calls"] = np.array(calls)
    np.savez_compressed(args.out, **out)
    print(f"wrote {args.out}: {len(calls)} calls ({', '.join(calls)}), "
          f"{os.path.getsize(args.out) / 1024:.1f} KiB")


if __name__ == "__main__":
    main()
