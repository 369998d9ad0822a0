"""Supercell samples whose TBPM Hamiltonian is assembled on the GPU.

The reference builds the TBPM input on the host: PrimitiveCell -> SuperCell ->
Sample -> build_ham_csr / build_ham_dxy (tbplas/builder/sample.py:375-461,
tbplas/cython/super.pyx:569-912, tbplas/cython/sample.pyx:20-257).  For a
33.5M-orbital sample that is tens of seconds of host work and a multi-GB CSR
upload.  `DeviceSample` describes the same supercell by its primitive cell and
lets libtbpm_b200 assemble the Hamiltonian directly in HBM
(tbpm_supercell_ham), in the reference's entry order and arithmetic.

It has the TBPM-facing interface of tbplas.Sample, so the Solver and the
Analyzer take it unchanged: `build_ham_csr()` / `build_ham_dxy()` return
handles that the f2py-compatible drivers recognise and turn into a resident
Hamiltonian instead of an upload; `rescale`, `energy_range`,
`area_unit_cell`, `volume_unit_cell`, `extended` and `nr_orbitals` are those
of the reference Sample.  `download_ham_csr()` / `download_ham_dxy()` copy
the device-built arrays to the host (scipy CSR / the five arrays of
build_ham_dxy) for inspection or for other tools.
"""

import ctypes
from typing import Iterable, Optional, Tuple

import numpy as np
from scipy.sparse import csr_matrix

from . import _native as nat

__all__ = ["DeviceSample", "ResidentHam", "make_graphene_device_sample"]


class ResidentHam:
    """Handle of a device-assembled Hamiltonian; passed where the reference
    passes the CSR arrays (the `indptr` argument of the f2py drivers)."""

    def __init__(self, sample: "DeviceSample", layout: int, cutoff: float) -> None:
        self.sample = sample
        self.layout = layout
        self.cutoff = float(cutoff)

    def make_resident(self, ctx: nat.Context) -> Tuple[int, int]:
        """Assemble the Hamiltonian in ctx (in its current precision); returns
        (rows, entries of the full CSR)."""
        return self.sample._assemble(ctx, self.layout, self.cutoff)

    @property
    def shape(self) -> Tuple[int, int]:
        return (self.sample.num_orb, self.sample.num_orb)


class _ResidentCSR:
    """What DeviceSample.build_ham_csr returns: the resident handle in the
    place of indptr, as the Solver reads ham_csr.indptr / .indices / .data."""

    def __init__(self, handle: ResidentHam) -> None:
        self.indptr = handle
        self.indices = None
        self.data = None
        self.shape = handle.shape


class DeviceSample:
    """A periodic supercell of a primitive cell, assembled on the GPU.

    :param lat_vec: (3, 3) lattice vectors of the primitive cell in nm (rows)
    :param origin: (3,) lattice origin in nm
    :param orb_pos: (n_orb, 3) fractional orbital positions (2-D positions are
        padded with 0)
    :param orb_eng: (n_orb,) on-site energies in eV
    :param hop_ind: (n_hop, 5) reduced hopping indices (ra, rb, rc, bra, ket),
        as PrimitiveCell.hop_ind
    :param hop_eng: (n_hop,) hopping energies in eV
    :param dim: supercell dimension (2 or 3 entries)
    :param pbc: periodic boundary conditions (2 or 3 entries)
    :param vac_id_sc: vacancy indices in supercell numbering
        ((ia*nb + ib)*nc + ic)*n_orb + o
    :param orb_eng_sc: optional on-site energies of every supercell orbital
        (eV, unscaled), e.g. Anderson disorder (Sample.orb_eng)
    :param b_field: Peierls field in Tesla (Sample.set_magnetic_field)
    :param gauge: gauge of the field (0, 1, 2)
    :param rescale: Sample.rescale_ham factor; None estimates it on the GPU
        like Sample.get_rescale
    """

    def __init__(self, lat_vec, origin, orb_pos, orb_eng, hop_ind, hop_eng, dim,
                 pbc=(False, False, False), vac_id_sc: Optional[Iterable[int]] = None,
                 orb_eng_sc=None, b_field: float = 0.0, gauge: int = 0,
                 rescale: Optional[float] = None, extended: float = 1.0) -> None:
        self.lat_vec = np.ascontiguousarray(lat_vec, dtype=np.float64).reshape(3, 3)
        self.origin = np.ascontiguousarray(
            np.zeros(3) if origin is None else origin, dtype=np.float64).reshape(3)
        pos = np.atleast_2d(np.asarray(orb_pos, dtype=np.float64))
        if pos.shape[1] == 2:
            pos = np.hstack([pos, np.zeros((pos.shape[0], 1))])
        self.pc_orb_pos = np.ascontiguousarray(pos)
        self.orb_eng = np.ascontiguousarray(orb_eng, dtype=np.float64).reshape(-1)
        if self.orb_eng.size != self.pc_orb_pos.shape[0]:
            raise ValueError("one energy per orbital required")
        self.hop_ind = np.ascontiguousarray(hop_ind, dtype=np.int32).reshape(-1, 5)
        self.hop_eng = np.ascontiguousarray(hop_eng, dtype=np.complex128).reshape(-1)
        if self.hop_eng.size != self.hop_ind.shape[0]:
            raise ValueError("hop_ind and hop_eng must have the same length")
        dim = list(dim) + [1] * (3 - len(dim))
        pbc = list(pbc) + [False] * (3 - len(pbc))
        self.dim = tuple(int(d) for d in dim)
        self.pbc = tuple(bool(p) for p in pbc)
        v = np.zeros(0, dtype=np.int64) if vac_id_sc is None else np.asarray(vac_id_sc)
        self.vac_id_sc = np.ascontiguousarray(np.unique(v.astype(np.int64)))
        n_full = int(np.prod(self.dim)) * self.pc_orb_pos.shape[0]
        self._num_orb = n_full - self.vac_id_sc.size
        self.orb_eng_sc = None
        if orb_eng_sc is not None:
            e = np.ascontiguousarray(orb_eng_sc, dtype=np.float64).reshape(-1)
            if e.size != self._num_orb:
                raise ValueError("orb_eng_sc needs one energy per supercell orbital")
            self.orb_eng_sc = e
        if gauge not in (0, 1, 2):
            raise ValueError(f"Illegal gauge {gauge}")
        self.b_field = float(b_field)
        self.gauge = int(gauge)
        self._rescale_arg = None if rescale is None else float(rescale)
        self._rescale = None
        self._extended = float(extended)

    # -- construction from the reference's objects --------------------------------
    @classmethod
    def from_supercell(cls, sc, **kw) -> "DeviceSample":
        """From a tbplas SuperCell (its primitive cell, dimension, boundary
        conditions and vacancies)."""
        pc = sc.prim_cell
        sc.sync_array()
        return cls(pc.lat_vec, pc.origin, pc.orb_pos, pc.orb_eng, pc.hop_ind, pc.hop_eng,
                   sc.dim, [bool(p) for p in sc.pbc], vac_id_sc=sc.vac_id_sc,
                   extended=getattr(pc, "extended", 1.0), **kw)

    # -- the Sample interface -----------------------------------------------------
    @property
    def num_orb(self) -> int:
        return self._num_orb

    @property
    def rescale(self) -> float:
        """Sample.rescale; estimated on the GPU on first use when not given."""
        if self._rescale is None:
            if self._rescale_arg is not None:
                self._rescale = self._rescale_arg
            else:
                self._rescale = self._query(nat.get_context(), nat.LAYOUT_CSR, 0.0)[2]
        return self._rescale

    @property
    def energy_range(self) -> float:
        """2 * rescale (builder/sample.py:682-693)."""
        return 2.0 * self.rescale

    @property
    def area_unit_cell(self) -> float:
        """|a1 x a2| of the primitive cell (base/lattice.py:181-204)."""
        return float(np.linalg.norm(np.cross(self.lat_vec[0], self.lat_vec[1])))

    @property
    def volume_unit_cell(self) -> float:
        """|(a1 x a2) . a3| (base/lattice.py:207-218)."""
        return float(np.abs(np.dot(np.cross(self.lat_vec[0], self.lat_vec[1]),
                                   self.lat_vec[2])))

    @property
    def extended(self) -> float:
        return self._extended

    @property
    def nr_orbitals(self) -> int:
        return self.pc_orb_pos.shape[0]

    @property
    def orb_pos(self) -> np.ndarray:
        """Cartesian positions (nm) of the supercell orbitals, (num_orb, 3),
        as SuperCell.get_orb_pos computes them (cython/super.pyx:569-612 plus
        the origin, builder/super.py:671-685).  Host arrays; needed by the
        dynamical polarisation (Sample.orb_pos)."""
        n_orb = self.pc_orb_pos.shape[0]
        keep = np.ones(int(np.prod(self.dim)) * n_orb, dtype=bool)
        keep[self.vac_id_sc] = False
        g = np.nonzero(keep)[0]
        cell, o = g // n_orb, g % n_orb
        ia = cell // (self.dim[1] * self.dim[2])
        ib = (cell // self.dim[2]) % self.dim[1]
        ic = cell % self.dim[2]
        ra = self.pc_orb_pos[o, 0] + ia
        rb = self.pc_orb_pos[o, 1] + ib
        rc = self.pc_orb_pos[o, 2] + ic
        pos = np.empty((g.size, 3))
        for k in range(3):
            pos[:, k] = ra * self.lat_vec[0, k] + rb * self.lat_vec[1, k] + \
                rc * self.lat_vec[2, k]
        return pos + self.origin

    def build_ham_csr(self) -> _ResidentCSR:
        """Handle of the build_ham_csr Hamiltonian, assembled on the GPU when a
        driver uses it."""
        return _ResidentCSR(ResidentHam(self, nat.LAYOUT_CSR, 0.0))

    def build_ham_dxy(self, orb_eng_cutoff: float = 1.0e-5, algo: str = "fast",
                      sort_col: bool = False):
        """Handle of the build_ham_dxy arrays (in the place of indptr; the other
        four entries are None), assembled on the GPU when a driver uses it."""
        del algo, sort_col
        return (ResidentHam(self, nat.LAYOUT_DXY, orb_eng_cutoff), None, None, None, None)

    # -- host copies ----------------------------------------------------------------
    def download_ham_csr(self, ctx: Optional[nat.Context] = None) -> csr_matrix:
        """The device-built build_ham_csr matrix as scipy CSR (int32 indices)."""
        ip, ix, hop, _, _ = self._download(ctx, nat.LAYOUT_CSR, 0.0, False)
        m = csr_matrix((hop, ix, ip.astype(np.int32)), shape=(self.num_orb, self.num_orb))
        m.has_sorted_indices = True
        return m

    def download_ham_dxy(self, orb_eng_cutoff: float = 1.0e-5,
                         ctx: Optional[nat.Context] = None):
        """The device-built build_ham_dxy arrays (indptr, indices as int64; hop,
        dx, dy) in the reference's "fast" entry order."""
        ip, ix, hop, dx, dy = self._download(ctx, nat.LAYOUT_DXY, orb_eng_cutoff, True)
        return ip, ix.astype(np.int64), hop, dx, dy

    # -- internals ------------------------------------------------------------------
    def _struct(self) -> nat.Supercell:
        s = nat.Supercell()
        s.lat_vec = nat.ptr(self.lat_vec)
        s.origin = nat.ptr(self.origin)
        s.n_orb = self.pc_orb_pos.shape[0]
        s.orb_pos = nat.ptr(self.pc_orb_pos)
        s.orb_eng = nat.ptr(self.orb_eng)
        s.n_hop = self.hop_ind.shape[0]
        s.hop_ind = nat.ptr(self.hop_ind) if self.hop_ind.size else None
        s.hop_eng = nat.ptr(self.hop_eng) if self.hop_eng.size else None
        for k in range(3):
            s.dim[k] = self.dim[k]
            s.pbc[k] = 1 if self.pbc[k] else 0
        s.vac_id_sc = nat.ptr(self.vac_id_sc) if self.vac_id_sc.size else None
        s.n_vac = self.vac_id_sc.size
        s.sc_orb_eng = nat.ptr(self.orb_eng_sc) if self.orb_eng_sc is not None else None
        s.b_field = self.b_field
        s.gauge = self.gauge
        s.rescale = self._rescale if self._rescale is not None else (
            self._rescale_arg if self._rescale_arg is not None else 0.0)
        return s

    def _query(self, ctx, layout, cutoff):
        n, nnz, r = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_double()
        s = self._struct()
        ctx.call("tbpm_supercell_csr", ctypes.byref(s), int(layout), float(cutoff),
                 ctypes.byref(n), ctypes.byref(nnz), ctypes.byref(r), None, None, None, None,
                 None)
        return int(n.value), int(nnz.value), float(r.value)

    def _assemble(self, ctx, layout, cutoff) -> Tuple[int, int]:
        n, nnz, r = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_double()
        s = self._struct()
        ctx.call("tbpm_supercell_ham", ctypes.byref(s), int(layout), float(cutoff),
                 ctypes.byref(n), ctypes.byref(nnz), ctypes.byref(r))
        self._rescale = float(r.value)
        return int(n.value), int(nnz.value)

    def _download(self, ctx, layout, cutoff, with_dxy):
        ctx = ctx or nat.get_context()
        n, nnz, r = self._query(ctx, layout, cutoff)
        self._rescale = r
        ip = np.zeros(n + 1, dtype=np.int64)
        ix = np.zeros(max(nnz, 1), dtype=np.int32)
        hop = np.zeros(max(nnz, 1), dtype=np.complex128)
        dx = np.zeros(max(nnz, 1)) if with_dxy else None
        dy = np.zeros(max(nnz, 1)) if with_dxy else None
        s = self._struct()
        ctx.call("tbpm_supercell_csr", ctypes.byref(s), int(layout), float(cutoff),
                 ctypes.byref(ctypes.c_int64()), ctypes.byref(ctypes.c_int64()),
                 ctypes.byref(ctypes.c_double()), nat.ptr(ip), nat.ptr(ix), nat.ptr(hop),
                 nat.ptr(dx), nat.ptr(dy))
        return (ip, ix[:nnz], hop[:nnz], None if dx is None else dx[:nnz],
                None if dy is None else dy[:nnz])


_GRAPHENE_LAT = np.array([[0.246, 0.0, 0.0],
                          [0.246 * np.cos(np.pi / 3), 0.246 * np.sin(np.pi / 3), 0.0],
                          [0.0, 0.0, 1.0]])


def make_graphene_device_sample(nx: int, ny: int, t: float = -2.7,
                                rescale: Optional[float] = 9.0, pbc: bool = True,
                                disorder: float = 0.0, vacancy_rate: float = 0.0,
                                b_field: float = 0.0, gauge: int = 0,
                                seed: int = 1337) -> DeviceSample:
    """Graphene (materials/graphene.py:16-31 make_graphene_diamond) supercell of
    nx x ny cells on the GPU, with the disorder and vacancies of
    tbplas_b200.builder.make_graphene_sample drawn from the same seeded
    generator, so both builders describe the same sample."""
    from .builder import LatticeSample
    lat = LatticeSample((1, 1))
    lat_vec = np.vstack([lat.a1, lat.a2, [0.0, 0.0, lat.c]])
    rng = np.random.default_rng(seed)
    vac = None
    n_full = nx * ny * 2
    if vacancy_rate > 0:
        k = int(round(vacancy_rate * n_full))
        vac = np.sort(rng.choice(n_full, size=k, replace=False))
    n = n_full - (0 if vac is None else vac.size)
    eng = None
    if disorder > 0:
        eng = rng.uniform(-0.5 * disorder, 0.5 * disorder, n)
    hop_ind = np.array([[0, 0, 0, 0, 1], [1, 0, 0, 1, 0], [0, 1, 0, 1, 0]], dtype=np.int32)
    return DeviceSample(lat_vec, np.zeros(3), [[0.0, 0.0, 0.0], [1 / 3., 1 / 3., 0.0]],
                        [0.0, 0.0], hop_ind, np.full(3, t, dtype=np.complex128), (nx, ny, 1),
                        (pbc, pbc, False), vac_id_sc=vac, orb_eng_sc=eng, b_field=b_field,
                        gauge=gauge, rescale=rescale)
