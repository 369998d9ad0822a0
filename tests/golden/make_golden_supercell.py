"""Generate tests/golden/reference_supercell.npz from the reference TBPLaS builder.

Run in a container that holds the reference source tree (read-only):

    python tests/golden/make_golden_supercell.py --ref <reference tree> --scratch <scratch dir>

It compiles the reference's Cython extensions in a scratch copy and imports the
reference package with the shims of make_golden.py.  For a set of primitive
cells (graphene in two settings, a non-orthogonal two-orbital lattice with
complex, second-neighbour and zero hoppings and a shifted origin, simple-cubic
lattices in 3-D) and supercells of them (periodic, open and mixed
boundaries, vacancies, on-site disorder, Peierls fields in the three gauges,
fixed and estimated rescale factors) it records

* the inputs the GPU supercell builder takes: the primitive cell's lattice
  vectors, origin, fractional orbital positions, orbital energies, reduced
  hopping indices and energies, the supercell dimension, boundary conditions,
  the sorted vacancy indices, the per-orbital energies of the Sample before
  rescaling, the field and gauge and the rescale argument;
* the reference outputs: Sample.build_ham_csr (indptr, indices, data),
  Sample.build_ham_dxy with the default "fast" algorithm and its native entry
  order (indptr, indices, hop, dx, dy), Sample.rescale and Sample.orb_pos.
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
    ap.add_argument("--out", default=os.path.join(HERE, "reference_supercell.npz"))
    args = ap.parse_args()

    prepare_scratch(args.ref, args.scratch)
    install_shims(types.ModuleType("tbplas.fortran.f2py"))
    sys.path.insert(0, args.scratch)
    import tbplas as tb

    rng = np.random.default_rng(77060)
    out = {}

    def square2():
        lat = np.array([[0.31, 0.0, 0.0], [0.07, 0.29, 0.0], [0.0, 0.0, 0.5]])
        cell = tb.PrimitiveCell(lat, origin=np.array([0.1, -0.2, 0.05]), unit=1.0)
        cell.add_orbital((0.0, 0.0), energy=0.3)
        cell.add_orbital((0.45, 0.55), energy=0.0)
        cell.add_hopping((0, 0), 0, 1, -1.0 + 0.2j)
        cell.add_hopping((1, 0), 0, 0, -0.7)
        cell.add_hopping((0, 1), 1, 1, -0.5 + 0.1j)
        cell.add_hopping((1, 1), 0, 1, 0.15 - 0.05j)
        cell.add_hopping((1, -1), 1, 0, 0.12)
        cell.add_hopping((2, 0), 0, 0, 0.05)
        cell.add_hopping((0, 1), 0, 1, 0.0)
        return cell

    def cubic(n_orb):
        cell = tb.PrimitiveCell(np.diag([0.3, 0.32, 0.35]), unit=1.0)
        for o in range(n_orb):
            cell.add_orbital((0.5 * o, 0.25 * o, 0.1 * o), energy=0.2 * o)
        for o in range(n_orb):
            for rn, t in (((1, 0, 0), -1.0), ((0, 1, 0), -0.9 + 0.05j), ((0, 0, 1), -0.8)):
                cell.add_hopping(rn, o, o, t)
        if n_orb > 1:
            cell.add_hopping((0, 0, 0), 0, 1, -0.4)
            cell.add_hopping((1, 0, -1), 1, 0, 0.2j)
        return cell

    cases = [
        # key, cell factory, dim, pbc, vacancies, disorder W, field, gauge, rescale
        ("gd_pbc", tb.make_graphene_diamond, (6, 5, 1), (True, True, False), None, 0.0,
         None, 0, 9.0),
        ("gd_vac_dis", tb.make_graphene_diamond, (7, 6, 1), (True, True, False),
         [(0, 0, 0, 0), (2, 3, 0, 1), (6, 5, 0, 0), (3, 1, 0, 1)], 1.0, None, 0, None),
        ("gd_mag0", tb.make_graphene_diamond, (6, 5, 1), (True, True, False), None, 1.0,
         77.06, 0, None),
        ("gd_mag1", tb.make_graphene_diamond, (6, 5, 1), (True, True, False), None, 1.0,
         77.06, 1, None),
        ("gd_mag2", tb.make_graphene_diamond, (6, 5, 1), (True, True, False),
         [(1, 1, 0, 0)], 1.0, 120.0, 2, None),
        ("gd_open_mag", tb.make_graphene_diamond, (5, 4, 1), (False, False, False), None,
         0.0, 40.0, 0, 9.0),
        ("grect", tb.make_graphene_rect, (4, 5, 1), (True, True, False), None, 0.0, None, 0,
         None),
        ("sq2", square2, (6, 5, 1), (True, False, False), [(2, 2, 0, 1), (5, 0, 0, 0)], 0.4,
         None, 0, None),
        ("sq2_pbc_mag", square2, (5, 6, 1), (True, True, False), None, 0.0, 60.0, 2, 6.5),
        ("cubic1", lambda: cubic(1), (4, 3, 5), (True, True, True), None, 0.6, None, 0, 7.0),
        ("cubic2_mixed", lambda: cubic(2), (3, 4, 3), (True, False, True),
         [(0, 0, 0, 1), (2, 3, 2, 0)], 0.3, 25.0, 2, None),
    ]
    keys = []
    for key, make_cell, dim, pbc, vac, w, field, gauge, rescale in cases:
        cell = make_cell()
        kw = {} if vac is None else {"vacancies": vac}
        sc = tb.SuperCell(cell, dim=dim, pbc=pbc, **kw)
        s = tb.Sample(sc)
        s.init_orb_eng()
        if w > 0:
            s.orb_eng += rng.uniform(-0.5 * w, 0.5 * w, s.orb_eng.size)
        out[f"{key}/sc_orb_eng"] = s.orb_eng.copy()
        if field is not None:
            s.set_magnetic_field(field, gauge=gauge)
        s.rescale_ham(rescale)
        out[f"{key}/lat_vec"] = np.array(cell.lat_vec)
        out[f"{key}/origin"] = np.array(cell.origin)
        out[f"{key}/orb_pos"] = np.array(cell.orb_pos)
        out[f"{key}/orb_eng"] = np.array(cell.orb_eng)
        out[f"{key}/hop_ind"] = np.array(cell.hop_ind, dtype=np.int32)
        out[f"{key}/hop_eng"] = np.array(cell.hop_eng, dtype=np.complex128)
        out[f"{key}/dim"] = np.array(sc.dim if hasattr(sc, "dim") else dim, dtype=np.int32)
        out[f"{key}/pbc"] = np.array([1 if p else 0 for p in pbc], dtype=np.int32)
        out[f"{key}/vac_id_sc"] = np.array(sc.sc0._vac_id_sc if hasattr(sc, "sc0")
                                           else sc._vac_id_sc, dtype=np.int64)
        out[f"{key}/field"] = np.array([0.0 if field is None else field, gauge])
        out[f"{key}/rescale_arg"] = np.array(0.0 if rescale is None else rescale)
        h = s.build_ham_csr()
        out[f"{key}/csr_indptr"] = h.indptr
        out[f"{key}/csr_indices"] = h.indices
        out[f"{key}/csr_data"] = h.data
        ip, ix, hop, dx, dy = s.build_ham_dxy()
        out[f"{key}/dxy_indptr"] = ip
        out[f"{key}/dxy_indices"] = ix
        out[f"{key}/dxy_hop"] = hop
        out[f"{key}/dxy_dx"] = dx
        out[f"{key}/dxy_dy"] = dy
        s.init_orb_pos()
        out[f"{key}/sc_orb_pos"] = s.orb_pos
        out[f"{key}/rescale"] = np.array(s.rescale)
        keys.append(key)
    out["cases"] = np.array(keys)
    np.savez_compressed(args.out, **out)
    print(f"wrote {args.out}: {len(keys)} cases, {os.path.getsize(args.out) / 1024:.1f} KiB")


if __name__ == "__main__":
    main()
