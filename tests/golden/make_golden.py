"""Generate the golden fixtures of tests/golden from the reference TBPLaS.

Run in a container that holds the reference source tree (read-only):

    python tests/golden/make_golden.py --ref <reference tree> --scratch <scratch dir>

The script copies the reference package to a scratch directory, compiles its
Cython extensions there (cythonize -i), and imports it with three shims:
a stub `matplotlib` (imported at module level by the builder), the removed
`scipy.integrate.trapz` aliased to `trapezoid`, and `tbplas.fortran.f2py`
replaced by the CPU oracle of this repository (the reference's Fortran core
cannot be compiled here).  It then records

* Sample outputs of the reference builder (build_ham_csr, build_ham_dxy,
  orb_pos, hop arrays, rescale, energy_range, unit-cell data) for graphene
  supercells with/without disorder, vacancies, magnetic field, open
  boundaries;
* Solver parameter handling (Bessel series, time steps, DC energy grid and
  qe indices, beta/mu rescaling);
* correlation functions produced by the reference Solver driving the oracle
  with injected initial states, and the states themselves;
* Analyzer outputs (calc_dos, calc_ac_cond, calc_dc_cond, calc_diff_coeff) of
  the reference on those correlations.

Everything is written to tests/golden/reference_tbplas.npz.
"""

import argparse
import math
import os
import shutil
import subprocess
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)


def prepare_scratch(ref: str, scratch: str) -> None:
    dst = os.path.join(scratch, "tbplas")
    if not os.path.exists(dst):
        os.makedirs(scratch, exist_ok=True)
        shutil.copytree(os.path.join(ref, "tbplas"), dst)
        for root, dirs, files in os.walk(dst):
            os.chmod(root, 0o755)
            for f in files:
                os.chmod(os.path.join(root, f), 0o644)
    cy = os.path.join(dst, "cython")
    for name in ("primitive", "super", "sample", "lindhard", "atom"):
        if not any(f.startswith(name + ".") and f.endswith(".so") for f in os.listdir(cy)):
            subprocess.run(["cythonize", "-i", "-3", name + ".pyx"], cwd=cy, check=True,
                           stdout=subprocess.DEVNULL)


def install_shims(shim) -> None:
    import scipy.integrate as si
    if not hasattr(si, "trapz"):
        si.trapz = si.trapezoid

    class _Any:
        def __getattr__(self, k):
            return _Any()

        def __call__(self, *a, **k):
            return _Any()

    mpl = types.ModuleType("matplotlib")
    mpl.__path__ = []
    for sub in ("pyplot", "collections"):
        m = types.ModuleType("matplotlib." + sub)
        m.__getattr__ = lambda k: _Any()
        setattr(mpl, sub, m)
        sys.modules["matplotlib." + sub] = m
    sys.modules["matplotlib"] = mpl
    fort = types.ModuleType("tbplas.fortran")
    fort.__path__ = []
    fort.f2py = shim
    sys.modules["tbplas.fortran"] = fort
    sys.modules["tbplas.fortran.f2py"] = shim


def sample_record(tb, out: dict, key: str, sample) -> None:
    h = sample.build_ham_csr()
    out[f"{key}/csr_indptr"] = h.indptr
    out[f"{key}/csr_indices"] = h.indices
    out[f"{key}/csr_data"] = h.data
    ip, ix, hop, dx, dy = sample.build_ham_dxy()
    out[f"{key}/dxy_indptr"] = ip
    out[f"{key}/dxy_indices"] = ix
    out[f"{key}/dxy_hop"] = hop
    out[f"{key}/dxy_dx"] = dx
    out[f"{key}/dxy_dy"] = dy
    sample.init_orb_pos()
    out[f"{key}/orb_pos"] = sample.orb_pos
    out[f"{key}/rescale"] = np.array(sample.rescale)
    out[f"{key}/energy_range"] = np.array(sample.energy_range)
    out[f"{key}/area_unit_cell"] = np.array(sample.area_unit_cell)
    out[f"{key}/volume_unit_cell"] = np.array(sample.volume_unit_cell)
    out[f"{key}/nr_orbitals"] = np.array(sample.nr_orbitals)
    out[f"{key}/extended"] = np.array(sample.extended)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="root of the reference source tree")
    ap.add_argument("--scratch", required=True,
                    help="scratch directory for the cythonized copy of the reference")
    ap.add_argument("--out", default=os.path.join(HERE, "reference_tbplas.npz"))
    args = ap.parse_args()

    from oracle import oracle
    shim_obj = oracle.F2pyShim()
    shim = types.ModuleType("tbplas.fortran.f2py")
    for name in ("tbpm_dos", "tbpm_accond", "tbpm_dccond", "tbpm_psi_t"):
        setattr(shim, name, getattr(shim_obj, name))

    prepare_scratch(args.ref, args.scratch)
    install_shims(shim)
    sys.path.insert(0, args.scratch)
    import tbplas as tb

    out = {}
    rng = np.random.default_rng(20240611)

    # ---- samples ---------------------------------------------------------
    def graphene(dim, pbc=True, vacancies=None, disorder=None, bfield=None, gauge=0,
                 rescale=9.0):
        cell = tb.make_graphene_diamond()
        kw = {} if vacancies is None else {"vacancies": vacancies}
        sc = tb.SuperCell(cell, dim=(dim[0], dim[1], 1), pbc=(pbc, pbc, False), **kw)
        s = tb.Sample(sc)
        if disorder is not None:
            s.init_orb_eng()
            s.orb_eng += disorder
        if bfield is not None:
            s.set_magnetic_field(bfield, gauge=gauge)
        s.rescale_ham(rescale)
        return s

    samples = {}
    samples["g4x3"] = graphene((4, 3))
    dis = rng.uniform(-0.5, 0.5, 7 * 5 * 2)
    out["g7x5_dis/disorder"] = dis
    samples["g7x5_dis"] = graphene((7, 5), disorder=dis)
    vac = [(0, 0, 0, 0), (2, 3, 0, 1), (5, 5, 0, 0), (3, 1, 0, 1)]
    out["g6x6_vac/vacancies"] = np.array(vac)
    samples["g6x6_vac"] = graphene((6, 6), vacancies=vac)
    for g in (0, 1, 2):
        samples[f"g6x5_mag{g}"] = graphene((6, 5), bfield=77.06, gauge=g)
    samples["g5x4_open"] = graphene((5, 4), pbc=False)
    samples["g8x8_r10"] = graphene((8, 8), rescale=10.0)
    for key, s in samples.items():
        sample_record(tb, out, key, s)

    # ---- Solver parameters and correlation functions ------------------------
    s = samples["g7x5_dis"]
    n = s.num_orb_tot if hasattr(s, "num_orb_tot") else s.build_ham_csr().shape[0]
    states = np.exp(2j * np.pi * rng.random((2, n)))
    states /= np.linalg.norm(states, axis=1, keepdims=True)
    out["solver/states"] = states
    shim_obj.states = states
    config = tb.Config()
    config.generic["nr_time_steps"] = 64
    config.generic["nr_random_samples"] = 2
    solver = tb.Solver(s, config, prefix="golden", directory=os.path.join(args.scratch, "sim"))
    t = solver._get_time_step()
    out["solver/time_step"] = np.array(t)
    out["solver/bessel_dos"] = np.array(solver._get_bessel_series(t))
    out["solver/bessel_ac"] = np.array(solver._get_bessel_series(0.5 * t))
    out["solver/beta_mu_re"] = np.array(solver._get_beta_mu_re())
    out["solver/corr_dos"] = solver.calc_corr_dos()
    config.generic["nr_time_steps"] = 32
    out["solver/corr_ac"] = solver.calc_corr_ac_cond()
    corr_dos_dc, corr_dc = solver.calc_corr_dc_cond()
    out["solver/corr_dos_dc"] = corr_dos_dc
    out["solver/corr_dc"] = corr_dc
    shim_obj.states = None
    psi0 = states[0]
    out["solver/psi_t"] = solver.calc_psi_t(psi0, [0, 3, 10, 32, 3])
    tnr = 32
    en_range = s.energy_range
    energies = np.array([0.5 * i * en_range / tnr - en_range / 2. for i in range(tnr * 2)])
    out["solver/dc_energies"] = energies
    out["solver/dc_qe_indices"] = np.where((energies >= -0.5) & (energies <= 0.5))[0]
    g = config.generic
    out["config/generic_values"] = np.array([g['Bessel_max'], g['Bessel_precision'], g['beta'],
                                             g['mu'], g['nr_random_samples'], g['seed'],
                                             g['wfn_check_steps'], g['wfn_check_thr'],
                                             g['nr_Fermi_fft_steps'],
                                             g['Fermi_cheb_precision']], dtype=float)

    # ---- Analyzer ------------------------------------------------------------
    for spin in (False, True):
        cfg = tb.Config()
        cfg.generic["nr_time_steps"] = 64
        cfg.generic["correct_spin"] = spin
        an = tb.Analyzer(s, cfg, dimension=2)
        e, d = an.calc_dos(out["solver/corr_dos"])
        out[f"analyzer/spin{int(spin)}/dos_energies"] = e
        out[f"analyzer/spin{int(spin)}/dos"] = d
        cfg.generic["nr_time_steps"] = 32
        an = tb.Analyzer(s, cfg, dimension=2)
        om, ac = an.calc_ac_cond(out["solver/corr_ac"])
        out[f"analyzer/spin{int(spin)}/ac_omegas"] = om
        out[f"analyzer/spin{int(spin)}/ac"] = ac
        en, dc = an.calc_dc_cond(out["solver/corr_dos_dc"], out["solver/corr_dc"])
        out[f"analyzer/spin{int(spin)}/dc_energies"] = en
        out[f"analyzer/spin{int(spin)}/dc"] = dc
        tm, dcoef = an.calc_diff_coeff(out["solver/corr_dc"])
        out[f"analyzer/spin{int(spin)}/diff_time"] = tm
        out[f"analyzer/spin{int(spin)}/diff_coeff"] = dcoef
    an3 = tb.Analyzer(s, cfg, dimension=3)
    om, ac = an3.calc_ac_cond(out["solver/corr_ac"])
    out["analyzer/dim3/ac"] = ac

    np.savez_compressed(args.out, **out)
    print(f"wrote {args.out}: {len(out)} arrays, "
          f"{os.path.getsize(args.out) / 1024:.1f} KiB")


if __name__ == "__main__":
    main()
