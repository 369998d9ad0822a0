"""Graphene samples with the TBPM-facing interface of tbplas.Sample.

The reference builds TBPM inputs with PrimitiveCell -> SuperCell -> Sample
(tbplas/builder, tbplas/cython/super.pyx, tbplas/cython/sample.pyx).  The
B200 path only needs what the Solver reads from a Sample: the CSR Hamiltonian
(`build_ham_csr`, builder/sample.py:375-391), the conductivity arrays
(`build_ham_dxy`, sample.py:417-461), `rescale`, `energy_range`
(sample.py:682-693) and the unit-cell data used by the Analyzer.  This module
produces them for supercells of the graphene primitive cell of
`make_graphene_diamond` (materials/graphene.py:16-31: a = 0.246 nm, lattice
angle 60 deg, orbitals at fractional (0,0) and (1/3,1/3), hopping t between
orbital 0 and orbital 1 at R = (0,0), (-1,0), (0,-1)) with

* periodic or open boundaries,
* vacancies (removed orbitals, SuperCell(vacancies=...)),
* on-site energies (Sample.orb_eng, e.g. Anderson disorder),
* Peierls phases of a perpendicular magnetic field
  (Sample.set_magnetic_field, cython/sample.pyx:20-74),
* rescaling (Sample.rescale_ham, sample.py:272-299),

with the orbital order of the reference supercell: index = (ia*ny + ib)*2 + o
before vacancies are removed, vacancies dropped in place.  Arrays are built
with vectorised numpy, so 4096 x 4096 cells (33.5M orbitals) take seconds.
"""

import math
from typing import Iterable, Optional, Tuple

import numpy as np
from scipy.sparse import csr_matrix

__all__ = ["LatticeSample", "make_graphene_sample", "pack_samples", "PackedSamples"]

_PEIERLS_FACTOR = math.pi / 4135.666734  # cython/sample.pyx:48


class LatticeSample:
    """Graphene supercell of nx x ny primitive cells.

    :param dim: (nx, ny) numbers of primitive cells along a1 and a2
    :param t: hopping integral in eV
    :param a: lattice constant in nm
    :param pbc: periodic boundary conditions along a1 and a2
    :param vacancies: iterable of (ia, ib, orbital) or (ia, ib, 0, orbital)
    :param c: length of the c axis in nm (only enters volume_unit_cell)
    """

    def __init__(self, dim: Tuple[int, int], t: complex = -2.7, a: float = 0.246,
                 pbc: Tuple[bool, bool] = (True, True),
                 vacancies: Optional[Iterable] = None, c: float = 1.0) -> None:
        nx, ny = int(dim[0]), int(dim[1])
        if nx < 1 or ny < 1:
            raise ValueError("dim must be positive")
        self.nx, self.ny = nx, ny
        self.pbc = (bool(pbc[0]), bool(pbc[1]))
        self.a = float(a)
        self.c = float(c)
        self.t = complex(t)
        # lattice vectors as base/lattice.py gen_lattice_vectors(a, a, c, gamma=60)
        gamma = 60 / 180 * math.pi
        self.a1 = np.array([a, 0.0, 0.0])
        self.a2 = np.array([a * math.cos(gamma), a * math.sin(gamma), 0.0])
        self.a2[np.abs(self.a2) < 1.0e-15] = 0.0
        self.frac = np.array([[0.0, 0.0], [1 / 3., 1 / 3.]])
        n_full = nx * ny * 2
        keep = np.ones(n_full, dtype=bool)
        if vacancies is not None:
            for v in vacancies:
                v = tuple(int(x) for x in v)
                ia, ib, o = (v[0], v[1], v[-1])
                if not (0 <= ia < nx and 0 <= ib < ny and o in (0, 1)):
                    raise ValueError(f"illegal vacancy {v}")
                keep[(ia * ny + ib) * 2 + o] = False
        self._keep = keep
        new_index = np.full(n_full, -1, dtype=np.int64)
        new_index[keep] = np.arange(int(keep.sum()), dtype=np.int64)
        self._new_index = new_index
        self.num_orb = int(keep.sum())
        self._build_positions()
        self._build_hoppings()
        self.orb_eng = np.zeros(self.num_orb, dtype=np.float64)
        self._rescale = 1.0

    # -- geometry ------------------------------------------------------------
    def _cart(self, fa, fb):
        # ra*a1 + rb*a2 + 0*a3, summed in the order of super.pyx build_orb_pos
        pos = np.empty((np.size(fa), 3))
        for k in range(3):
            pos[:, k] = (fa * self.a1[k] + fb * self.a2[k]) + 0.0 * (self.c if k == 2 else 0.0)
        return pos

    def _build_positions(self) -> None:
        nx, ny = self.nx, self.ny
        idx = np.nonzero(self._keep)[0]
        cell = idx // 2
        o = idx % 2
        ia = cell // ny
        ib = cell % ny
        fa = ia + self.frac[o, 0]
        fb = ib + self.frac[o, 1]
        self.orb_pos = self._cart(fa, fb)

    def _build_hoppings(self) -> None:
        """Half hopping list (hop_i, hop_j, hop_v, dr) as in Sample.init_hop."""
        nx, ny = self.nx, self.ny
        ia, ib = np.meshgrid(np.arange(nx, dtype=np.int64), np.arange(ny, dtype=np.int64),
                             indexing="ij")
        ia = ia.reshape(-1)
        ib = ib.reshape(-1)
        sc_a1, sc_a2 = nx * self.a1, ny * self.a2

        def pos(ca, cb, o):
            return self._cart(ca + self.frac[o, 0], cb + self.frac[o, 1])

        his, hjs, drs = [], [], []
        # (0,0): orbital 0 -> orbital 1 of the same cell
        his.append((ia * ny + ib) * 2)
        hjs.append((ia * ny + ib) * 2 + 1)
        drs.append(pos(ia, ib, 1) - pos(ia, ib, 0))
        # (1,0) and (0,1): orbital 1 -> orbital 0 of the next cell.  dr as in
        # super.pyx build_hop_pbc: pos_j - pos_i + na*A_sc[0] + nb*A_sc[1]
        for da, db in ((1, 0), (0, 1)):
            ja0, jb0 = ia + da, ib + db
            ok = np.ones(ia.size, dtype=bool)
            if not self.pbc[0]:
                ok &= ja0 < nx
            if not self.pbc[1]:
                ok &= jb0 < ny
            ja, jb = ja0 % nx, jb0 % ny
            na, nb = (ja0 // nx).astype(float), (jb0 // ny).astype(float)
            d = pos(ja, jb, 0) - pos(ia, ib, 1)
            for k in range(3):
                d[:, k] = (d[:, k] + na * sc_a1[k]) + nb * sc_a2[k]
            his.append(((ia * ny + ib) * 2 + 1)[ok])
            hjs.append(((ja * ny + jb) * 2)[ok])
            drs.append(d[ok])
        hi = np.concatenate(his)
        hj = np.concatenate(hjs)
        dr = np.concatenate(drs).astype(np.float64)
        ni, nj = self._new_index[hi], self._new_index[hj]
        ok = (ni >= 0) & (nj >= 0)
        self.hop_i = ni[ok]
        self.hop_j = nj[ok]
        self.dr = np.ascontiguousarray(dr[ok])
        self.hop_v = np.full(self.hop_i.size, self.t, dtype=np.complex128)

    # -- Sample interface -------------------------------------------------------
    @property
    def rescale(self) -> float:
        return self._rescale

    @property
    def energy_range(self) -> float:
        """2 * rescale (builder/sample.py:682-693)."""
        return 2.0 * self._rescale

    @property
    def area_unit_cell(self) -> float:
        return float(np.linalg.norm(np.cross(self.a1, self.a2)))

    @property
    def volume_unit_cell(self) -> float:
        return self.area_unit_cell * self.c

    @property
    def extended(self) -> float:
        return 1.0

    @property
    def nr_orbitals(self) -> int:
        return 2

    @property
    def num_hop(self) -> int:
        return int(self.hop_i.size)

    def get_rescale(self) -> float:
        """max_i (orb_eng_i + sum_j |h_ij|) (cython/sample.pyx:77-116)."""
        s = self.orb_eng.astype(np.float64).copy()
        habs = np.abs(self.hop_v)
        np.add.at(s, self.hop_i, habs)
        np.add.at(s, self.hop_j, habs)
        return float(np.max(s))

    def rescale_ham(self, factor: float = None) -> None:
        """Divide energies and hoppings by factor w.r.t. their unscaled values
        (builder/sample.py:272-299)."""
        if factor is None:
            factor = self.get_rescale() * self._rescale
        self.orb_eng = self.orb_eng * (self._rescale / factor)
        self.hop_v = self.hop_v * (self._rescale / factor)
        self._rescale = float(factor)

    def set_orb_eng(self, energies: np.ndarray) -> None:
        """Set on-site energies in eV (unscaled); rescaling is applied."""
        e = np.asarray(energies, dtype=np.float64).reshape(-1)
        if e.size != self.num_orb:
            raise ValueError("one energy per orbital required")
        self.orb_eng = e / self._rescale

    def set_magnetic_field(self, intensity: float, gauge: int = 0) -> None:
        """Peierls phases of a field along -z in Tesla (cython/sample.pyx:20-74)."""
        if gauge not in (0, 1, 2):
            raise ValueError(f"Illegal gauge {gauge}")
        pi_, pj = self.orb_pos[self.hop_i], self.orb_pos[self.hop_j]
        if gauge == 0:
            phase = _PEIERLS_FACTOR * intensity * self.dr[:, 0] * (pj[:, 1] + pi_[:, 1])
        elif gauge == 1:
            phase = -_PEIERLS_FACTOR * intensity * self.dr[:, 1] * (pj[:, 0] + pi_[:, 0])
        else:
            sx = pj[:, 0] + pi_[:, 0]
            sy = pj[:, 1] + pi_[:, 1]
            phase = _PEIERLS_FACTOR * 0.5 * intensity * (self.dr[:, 0] * sx -
                                                         self.dr[:, 1] * sy)
        self.hop_v = self.hop_v * (np.cos(phase) + 1j * np.sin(phase))

    # -- CSR builders -------------------------------------------------------------
    def _rows(self, with_diag: np.ndarray):
        """Entries of the full Hermitian matrix as (row, col, value, dx, dy)."""
        diag = np.nonzero(with_diag)[0]
        rows = np.concatenate([diag, self.hop_i, self.hop_j])
        cols = np.concatenate([diag, self.hop_j, self.hop_i])
        vals = np.concatenate([self.orb_eng[diag].astype(np.complex128), self.hop_v,
                               np.conj(self.hop_v)])
        dx = np.concatenate([np.zeros(diag.size), self.dr[:, 0], -self.dr[:, 0]])
        dy = np.concatenate([np.zeros(diag.size), self.dr[:, 1], -self.dr[:, 1]])
        return rows, cols, vals, dx, dy

    def _sorted_csr(self, rows, cols, vals, dx, dy, merge: bool):
        n = self.num_orb
        order = np.lexsort((cols, rows))
        rows, cols, vals, dx, dy = rows[order], cols[order], vals[order], dx[order], dy[order]
        if merge and rows.size > 1:
            dup = (rows[1:] == rows[:-1]) & (cols[1:] == cols[:-1])
            if dup.any():
                start = np.concatenate([[True], ~dup])
                seg = np.cumsum(start) - 1
                vals = np.bincount(seg, weights=vals.real) + \
                    1j * np.bincount(seg, weights=vals.imag)
                rows, cols = rows[start], cols[start]
                dx, dy = dx[start], dy[start]
        indptr = np.zeros(n + 1, dtype=np.int64)
        np.cumsum(np.bincount(rows, minlength=n), out=indptr[1:])
        return indptr, cols, vals, dx, dy

    def build_ham_csr(self) -> csr_matrix:
        """Sparse Hamiltonian: diag(orb_eng) + H_half + H_half^H, int32 sorted
        indices, explicit zeros removed (builder/sample.py:375-391)."""
        rows, cols, vals, dx, dy = self._rows(self.orb_eng != 0.0)
        indptr, cols, vals, _, _ = self._sorted_csr(rows, cols, vals, dx, dy, merge=True)
        nz = vals != 0
        if not nz.all():
            rows = np.repeat(np.arange(self.num_orb), np.diff(indptr))[nz]
            cols, vals = cols[nz], vals[nz]
            indptr = np.zeros(self.num_orb + 1, dtype=np.int64)
            np.cumsum(np.bincount(rows, minlength=self.num_orb), out=indptr[1:])
        # scipy's sparse sum stores x + 0, turning the -0.0 of conj() into +0.0
        vals = vals + 0.0
        m = csr_matrix((vals, cols.astype(np.int32), indptr.astype(np.int32)),
                       shape=(self.num_orb, self.num_orb))
        m.has_sorted_indices = True
        return m

    def build_ham_dxy(self, orb_eng_cutoff: float = 1.0e-5, algo: str = "fast",
                      sort_col: bool = False):
        """(indptr, indices, hop, dx, dy) for conductivity calculations
        (builder/sample.py:417-461); on-site terms with |E| < orb_eng_cutoff are
        dropped; columns are sorted within rows (the reference's sort_col=True
        order).  indptr and indices are int64."""
        del algo, sort_col
        rows, cols, vals, dx, dy = self._rows(np.abs(self.orb_eng) >= orb_eng_cutoff)
        indptr, cols, vals, dx, dy = self._sorted_csr(rows, cols, vals, dx, dy, merge=False)
        return (indptr, cols.astype(np.int64), np.ascontiguousarray(vals),
                np.ascontiguousarray(dx), np.ascontiguousarray(dy))


def make_graphene_sample(nx: int, ny: int, t: float = -2.7, rescale: float = 9.0,
                         pbc: bool = True, disorder: float = 0.0, vacancy_rate: float = 0.0,
                         b_field: float = 0.0, seed: int = 1337) -> LatticeSample:
    """Graphene sample of nx x ny cells with Anderson disorder U[-W/2, W/2] eV,
    randomly removed orbitals and an optional magnetic field (Tesla)."""
    rng = np.random.default_rng(seed)
    vac = None
    if vacancy_rate > 0:
        n = nx * ny * 2
        k = int(round(vacancy_rate * n))
        pick = rng.choice(n, size=k, replace=False)
        vac = [((p // 2) // ny, (p // 2) % ny, p % 2) for p in np.sort(pick)]
    s = LatticeSample((nx, ny), t=t, pbc=(pbc, pbc), vacancies=vac)
    if disorder > 0:
        s.set_orb_eng(rng.uniform(-0.5 * disorder, 0.5 * disorder, s.num_orb))
    if b_field:
        s.set_magnetic_field(b_field)
    s.rescale_ham(rescale)
    return s


class PackedSamples:
    """Several samples packed into one block-diagonal CSR (a batch of uneven
    realisations propagated in one launch).  Segment k owns rows
    [offsets[k], offsets[k+1])."""

    def __init__(self, indptr, indices, data, offsets, rescale):
        self.indptr = indptr
        self.indices = indices
        self.data = data
        self.offsets = offsets
        self.rescale = rescale

    @property
    def num_orb(self) -> int:
        return int(self.offsets[-1])

    @property
    def energy_range(self) -> float:
        return 2.0 * self.rescale


def pack_samples(samples, align: int = 1) -> PackedSamples:
    """Pack samples sharing one rescale factor into a block-diagonal CSR; each
    block starts at a multiple of `align` rows (padding rows are empty)."""
    rescales = {round(s.rescale, 12) for s in samples}
    if len(rescales) != 1:
        raise ValueError("packed samples must share one rescale factor")
    ips, ixs, vs, offsets = [], [], [], [0]
    nnz = 0
    for s in samples:
        h = s.build_ham_csr()
        start = offsets[-1]
        n = h.shape[0]
        pad = (-n) % align
        ip = h.indptr.astype(np.int64)
        ips.append((ip[:-1] + nnz))
        if pad:
            ips.append(np.full(pad, ip[-1] + nnz, dtype=np.int64))
        ixs.append(h.indices.astype(np.int64) + start)
        vs.append(h.data)
        nnz += h.nnz
        offsets.append(start + n + pad)
    indptr = np.concatenate(ips + [np.array([nnz], dtype=np.int64)])
    return PackedSamples(indptr.astype(np.int32), np.concatenate(ixs).astype(np.int32),
                         np.concatenate(vs), np.array(offsets, dtype=np.int64),
                         samples[0].rescale)
