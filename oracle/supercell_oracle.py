"""TEST INFRASTRUCTURE ONLY -- numpy restatement of the reference supercell builder.

Restates, for a supercell of any primitive cell, the arrays that the reference
TBPLaS builder hands to the TBPM core:

* orbital positions      -- cython/super.pyx:569-612 build_orb_pos (+ pc_origin,
                            builder/super.py:671-685 get_orb_pos)
* reduced hopping list   -- cython/super.pyx:643-754 build_hop_gen (vacancies),
                            :811-912 build_hop_pbc + :757-808 split_pc_hop
                            (no vacancies), in that list order
                            (builder/super.py:687-790 get_hop)
* Peierls phases         -- cython/sample.pyx:20-74 set_mag_field
* rescale estimate       -- cython/sample.pyx:77-116 get_rescale
* rescaling              -- builder/sample.py:272-299 rescale_ham
* CSR Hamiltonian        -- builder/sample.py:375-391 build_ham_csr (scipy sum
                            of the diagonal, the half matrix and its adjoint)
* conductivity arrays    -- cython/sample.pyx:150-257 build_ham_dxy_fast (entry
                            order: diagonal first, then hopping terms in list
                            order, each term giving the row of its bra and the
                            row of its ket)

It is pinned to the reference itself by tests/golden/reference_supercell.npz
(tests/test_supercell_oracle.py) and is the checker of the GPU supercell
builder at sizes without fixtures.  Only tests/ use it.
"""

import math

import numpy as np
from scipy.sparse import csr_matrix, dia_matrix

PEIERLS_FACTOR = math.pi / 4135.666734  # cython/sample.pyx:48


class SupercellSpec:
    """A periodic supercell of a primitive cell, as the reference SuperCell
    holds it: lattice vectors (rows, nm), origin (nm), fractional orbital
    positions, orbital energies (eV), reduced hopping indices (ra, rb, rc,
    bra, ket) and energies, dimension, boundary conditions and the sorted
    vacancy indices in supercell numbering ((ia*nb + ib)*nc + ic)*n_orb + o."""

    def __init__(self, lat_vec, origin, orb_pos, orb_eng, hop_ind, hop_eng, dim, pbc,
                 vac_id_sc=None):
        self.lat_vec = np.ascontiguousarray(lat_vec, dtype=np.float64).reshape(3, 3)
        self.origin = np.ascontiguousarray(origin, dtype=np.float64).reshape(3)
        self.orb_pos = np.ascontiguousarray(orb_pos, dtype=np.float64).reshape(-1, 3)
        self.orb_eng = np.ascontiguousarray(orb_eng, dtype=np.float64).reshape(-1)
        self.hop_ind = np.ascontiguousarray(hop_ind, dtype=np.int32).reshape(-1, 5)
        self.hop_eng = np.ascontiguousarray(hop_eng, dtype=np.complex128).reshape(-1)
        self.dim = np.array(dim, dtype=np.int64).reshape(3)
        self.pbc = np.array([1 if p else 0 for p in pbc], dtype=np.int64).reshape(3)
        v = np.zeros(0, dtype=np.int64) if vac_id_sc is None else np.asarray(vac_id_sc)
        self.vac_id_sc = np.unique(v.astype(np.int64))

    @property
    def n_orb_pc(self) -> int:
        return self.orb_pos.shape[0]

    @property
    def n_full(self) -> int:
        return int(np.prod(self.dim)) * self.n_orb_pc

    @property
    def sc_lat_vec(self) -> np.ndarray:
        s = self.lat_vec.copy()
        for i in range(3):
            s[i] *= int(self.dim[i])
        return s


def _split_index(spec, g):
    n_orb = spec.n_orb_pc
    nb, nc = spec.dim[1], spec.dim[2]
    cell = g // n_orb
    return cell // (nb * nc), (cell // nc) % nb, cell % nc, g % n_orb


def _wrap(j, n, p):
    """_wrap_pbc (super.pyx:446-493): periodic wrap, or -1 when outside an open
    boundary."""
    if p:
        return j % n
    return np.where((j >= 0) & (j < n), j, -1)


def orbital_positions(spec, g):
    """Cartesian positions of supercell orbitals g (super.pyx:602-611 + origin)."""
    ia, ib, ic, o = _split_index(spec, g)
    ra = spec.orb_pos[o, 0] + ia
    rb = spec.orb_pos[o, 1] + ib
    rc = spec.orb_pos[o, 2] + ic
    lat = spec.lat_vec
    pos = np.empty((np.size(g), 3))
    for k in range(3):
        pos[:, k] = ra * lat[0, k] + rb * lat[1, k] + rc * lat[2, k]
    pos += spec.origin
    return pos


def kept_orbitals(spec):
    """Supercell indices of the orbitals that are not vacancies, and the map
    from supercell index to row (-1 for vacancies)."""
    keep = np.ones(spec.n_full, dtype=bool)
    keep[spec.vac_id_sc] = False
    g = np.nonzero(keep)[0]
    new = np.full(spec.n_full, -1, dtype=np.int64)
    new[g] = np.arange(g.size)
    return g, new


def _terms(spec, g_bra, ih, new):
    """Hopping terms of bras g_bra (full indices) through pc terms ih."""
    ia, ib, ic, _ = _split_index(spec, g_bra)
    r = spec.hop_ind[ih]
    j0 = [ia + r[:, 0], ib + r[:, 1], ic + r[:, 2]]
    j = [_wrap(j0[d], spec.dim[d], spec.pbc[d]) for d in range(3)]
    ok = (j[0] >= 0) & (j[1] >= 0) & (j[2] >= 0)
    n_orb = spec.n_orb_pc
    g_ket = ((j[0] * spec.dim[1] + j[1]) * spec.dim[2] + j[2]) * n_orb + r[:, 4]
    g_ket = np.where(ok, g_ket, 0)
    ok &= new[g_ket] >= 0
    na = [np.floor_divide(j0[d], spec.dim[d]) for d in range(3)]
    return ok, g_ket, na


def build_hop(spec):
    """(hop_i, hop_j, hop_v, dr) in the reference list order (super.py:743-766)."""
    g_rows, new = kept_orbitals(spec)
    n_orb = spec.n_orb_pc
    nh = spec.hop_ind.shape[0]
    parts = []
    if spec.vac_id_sc.size == 0:
        is_pbc = np.all((spec.pbc[None, :] == 1) | (spec.hop_ind[:, :3] == 0), axis=1)
        pbc_ih = np.nonzero(is_pbc)[0]
        free_ih = np.nonzero(~is_pbc)[0]
        n_cells = int(np.prod(spec.dim))
        # build_hop_pbc: cells in order, then pc terms
        if pbc_ih.size:
            cell = np.repeat(np.arange(n_cells), pbc_ih.size)
            ih = np.tile(pbc_ih, n_cells)
            g_bra = cell * n_orb + spec.hop_ind[ih, 3]
            parts.append((g_bra, ih))
        # build_hop_gen on the free terms: orbitals in order, then terms
        if free_ih.size:
            g_bra = np.repeat(g_rows, free_ih.size)
            ih = np.tile(free_ih, g_rows.size)
            m = spec.hop_ind[ih, 3] == g_bra % n_orb
            parts.append((g_bra[m], ih[m]))
    else:
        g_bra = np.repeat(g_rows, nh)
        ih = np.tile(np.arange(nh), g_rows.size)
        m = spec.hop_ind[ih, 3] == g_bra % n_orb
        parts.append((g_bra[m], ih[m]))
    hop_i, hop_j, hop_v, dr = [], [], [], []
    sc_lat = spec.sc_lat_vec
    for g_bra, ih in parts:
        ok, g_ket, na = _terms(spec, g_bra, ih, new)
        g_bra, g_ket, ih = g_bra[ok], g_ket[ok], ih[ok]
        na = [a[ok] for a in na]
        pi = orbital_positions(spec, g_bra)
        pj = orbital_positions(spec, g_ket)
        d = np.empty((g_bra.size, 3))
        for k in range(3):
            d[:, k] = pj[:, k] - pi[:, k] + na[0] * sc_lat[0, k] + na[1] * sc_lat[1, k] \
                + na[2] * sc_lat[2, k]
        hop_i.append(new[g_bra])
        hop_j.append(new[g_ket])
        hop_v.append(spec.hop_eng[ih])
        dr.append(d)
    if not hop_i:
        return (np.zeros(0, np.int64), np.zeros(0, np.int64), np.zeros(0, np.complex128),
                np.zeros((0, 3)))
    return (np.concatenate(hop_i), np.concatenate(hop_j), np.concatenate(hop_v),
            np.concatenate(dr))


class SampleOracle:
    """The TBPM-facing arrays of a reference Sample built on one supercell."""

    def __init__(self, spec: SupercellSpec, sc_orb_eng=None):
        self.spec = spec
        g_rows, _ = kept_orbitals(spec)
        self.orb_pos = orbital_positions(spec, g_rows)
        if sc_orb_eng is None:
            self.orb_eng = spec.orb_eng[g_rows % spec.n_orb_pc].copy()
        else:
            self.orb_eng = np.array(sc_orb_eng, dtype=np.float64).reshape(-1).copy()
            if self.orb_eng.size != g_rows.size:
                raise ValueError("one energy per orbital required")
        self.hop_i, self.hop_j, self.hop_v, self.dr = build_hop(spec)
        self.rescale = 1.0

    @property
    def num_orb(self) -> int:
        return self.orb_eng.size

    def set_magnetic_field(self, intensity: float, gauge: int = 0) -> None:
        """sample.pyx:20-74 (vectorised; same operation order per term)."""
        pi, pj = self.orb_pos[self.hop_i], self.orb_pos[self.hop_j]
        dx, dy = self.dr[:, 0], self.dr[:, 1]
        if gauge == 0:
            phase = PEIERLS_FACTOR * intensity * dx * (pj[:, 1] + pi[:, 1])
        elif gauge == 1:
            phase = -PEIERLS_FACTOR * intensity * dy * (pj[:, 0] + pi[:, 0])
        elif gauge == 2:
            sx = pj[:, 0] + pi[:, 0]
            sy = pj[:, 1] + pi[:, 1]
            phase = PEIERLS_FACTOR * 0.5 * intensity * (dx * sx - dy * sy)
        else:
            raise ValueError(f"Illegal gauge {gauge}")
        c, s = np.cos(phase), np.sin(phase)
        v = self.hop_v
        self.hop_v = (v.real * c - v.imag * s) + 1j * (v.real * s + v.imag * c)

    def get_rescale(self) -> float:
        """sample.pyx:77-116: each term adds |h| to the row of its bra, then to
        the row of its ket, in list order."""
        s = self.orb_eng.copy()
        habs = np.sqrt(self.hop_v.real ** 2 + self.hop_v.imag ** 2)
        rows = np.stack([self.hop_i, self.hop_j], axis=1).reshape(-1)
        np.add.at(s, rows, np.repeat(habs, 2))
        return float(np.max(s))

    def rescale_ham(self, factor: float = None) -> None:
        """builder/sample.py:272-299."""
        if factor is None:
            factor = self.get_rescale()
        self.orb_eng *= (self.rescale / factor)
        self.hop_v *= (self.rescale / factor)
        self.rescale = factor

    def build_ham_csr(self) -> csr_matrix:
        """builder/sample.py:375-391."""
        n = self.num_orb
        ham_dia = dia_matrix((self.orb_eng, 0), shape=(n, n))
        ham_half = csr_matrix((self.hop_v, (self.hop_i, self.hop_j)), shape=(n, n))
        return ham_dia + ham_half + ham_half.getH()

    def build_ham_dxy(self, orb_eng_cutoff: float = 1.0e-5):
        """sample.pyx:150-257 build_ham_dxy_fast, native entry order."""
        n = self.num_orb
        diag = np.nonzero(np.abs(self.orb_eng) >= orb_eng_cutoff)[0]
        nh = self.hop_i.size
        rows = np.concatenate([diag, np.stack([self.hop_i, self.hop_j], 1).reshape(-1)])
        cols = np.concatenate([diag, np.stack([self.hop_j, self.hop_i], 1).reshape(-1)])
        vals = np.concatenate([self.orb_eng[diag].astype(np.complex128),
                               np.stack([self.hop_v, np.conj(self.hop_v)], 1).reshape(-1)])
        dx = np.concatenate([np.zeros(diag.size),
                             np.stack([self.dr[:, 0], -self.dr[:, 0]], 1).reshape(-1)])
        dy = np.concatenate([np.zeros(diag.size),
                             np.stack([self.dr[:, 1], -self.dr[:, 1]], 1).reshape(-1)])
        order = np.argsort(rows, kind="stable")
        indptr = np.zeros(n + 1, dtype=np.int64)
        np.cumsum(np.bincount(rows, minlength=n), out=indptr[1:])
        del nh
        return (indptr, cols[order].astype(np.int64), vals[order], dx[order], dy[order])


def sample_from_golden(z, key: str) -> SampleOracle:
    """Rebuild a recorded case of tests/golden/reference_supercell.npz."""
    spec = SupercellSpec(z[f"{key}/lat_vec"], z[f"{key}/origin"], z[f"{key}/orb_pos"],
                         z[f"{key}/orb_eng"], z[f"{key}/hop_ind"], z[f"{key}/hop_eng"],
                         z[f"{key}/dim"], z[f"{key}/pbc"], z[f"{key}/vac_id_sc"])
    s = SampleOracle(spec, z[f"{key}/sc_orb_eng"])
    field, gauge = z[f"{key}/field"]
    if field != 0.0:
        s.set_magnetic_field(float(field), int(gauge))
    r = float(z[f"{key}/rescale_arg"])
    s.rescale_ham(r if r > 0 else None)
    return s
