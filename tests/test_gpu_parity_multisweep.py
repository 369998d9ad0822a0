"""GPU vs oracle at sizes where every block of the persistent grid sweeps the
rows several times.

The Chebyshev-term, correlation and state kernels launch at most as many
blocks as a B200 holds at once and walk the row tiles grid-stride.  On the
small lattices of the other parity tests each block handles one tile, so the
second and later sweep iterations, the per-thread accumulation of the
correlation and norm across iterations, and the L2 prefetch of the next
iteration's tiles would go unchecked there.  Here every case has more row
tiles than a B200 can hold blocks (148 SMs x 2048 threads), which forces at
least two sweep iterations whatever the occupancy, and is compared with the
oracle on the same inputs: FP64 to a relative 1e-10 (max |diff| / max
|oracle|), FP32 states to the stated bound.
"""

import math

import numpy as np
import pytest

import tbplas_b200 as tb
from tbplas_b200.fortran import f2py
from oracle import oracle

from conftest import bessel_series, rel_err, unit_states

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10
FP32_TOL = 2e-5
SMS = 148
THREADS_PER_SM = 2048


def max_rows_per_sweep(ld, values_per_thread, threads_wanted=128):
    """Rows that one sweep of the largest possible persistent grid covers:
    blocks of rpp rows x tpr threads (the library's block shape), at most
    2048 // threads blocks per SM."""
    tpr = ld // values_per_thread
    rpp = max(1, threads_wanted // tpr)
    threads = rpp * tpr
    return SMS * (THREADS_PER_SM // threads) * rpp


@pytest.fixture(autouse=True)
def _backend():
    f2py.set_backend(precision="fp64", batch=16, device=0, state_kind="exp", use_graphs=True,
                     vector_width=0, threads_per_block=0, rows_per_tile=0)
    yield
    f2py.set_backend(precision="fp64", batch=16, state_kind="exp", use_graphs=True,
                     vector_width=0)


@pytest.fixture(scope="module")
def g256():
    """256 x 256 graphene cells (131,072 orbitals), W = 1 eV."""
    return tb.make_graphene_sample(256, 256, disorder=1.0, rescale=9.0, seed=1337)


@pytest.fixture(scope="module")
def g128():
    """128 x 128 graphene cells (32,768 orbitals), W = 1 eV."""
    return tb.make_graphene_sample(128, 128, disorder=1.0, rescale=9.0, seed=11)


def test_dos_fp64_seeded_16_states_multi_sweep(g256):
    """16 device-generated states as one block (two complex128 per thread: 8
    threads per row, 16 rows per 128-thread block): 8,192 row tiles."""
    h = g256.build_ham_csr()
    n = h.shape[0]
    assert n > 3 * max_rows_per_sweep(16, 2)
    bes = bessel_series(math.pi)
    got = f2py.tbpm_dos(bes, h.indptr, h.indices, h.data, 1337, 32, 16, "unused", 0, 128, 1e-9)
    ref = oracle.tbpm_dos(bes, h.indptr, h.indices, h.data, 32, seed=1337, n_samples=16)
    assert rel_err(got, ref) < FP64_TOL


def test_dos_fp32_16_states_multi_sweep(g256):
    """FP32 states, four complex64 per thread (4 threads per row)."""
    h = g256.build_ham_csr()
    n = h.shape[0]
    assert n > max_rows_per_sweep(16, 4)
    wf0 = unit_states(16, n, seed=5)
    bes = bessel_series(math.pi)
    f2py.set_backend(precision="fp32")
    got = f2py.tbpm_dos_states(bes, h.indptr, h.indices, h.data, wf0, 32, 16, 1e-9)
    ref = oracle.tbpm_dos(bes, h.indptr, h.indices, h.data, 32, wf0=wf0)
    assert rel_err(got, ref) < FP32_TOL


def test_ac_fp64_48_column_block_multi_sweep(g128):
    """16 states: the AC block [J_x psi | J_y psi | psi] has 48 columns (24
    threads per row, 5 rows per 120-thread block: 6,554 row tiles).  The Fermi
    operator is taken at 3000 K, which shortens its expansion; the kernels are
    the same as at 300 K."""
    ip, ix, hv, dx, dy = g128.build_ham_dxy()
    n = ip.size - 1
    assert n > 2 * max_rows_per_sweep(48, 2)
    wf0 = unit_states(16, n, seed=21)
    bes = bessel_series(math.pi / 2)
    beta = g128.rescale / (tb.KB * 3000.0)
    got = f2py.tbpm_accond_states(bes, beta, 0.0, ip, ix, hv, g128.rescale, dx, dy, wf0, 12,
                                  2**15, 1e-12, 128, 1e-9)
    ref = oracle.tbpm_accond(bes, beta, 0.0, ip, ix, hv, g128.rescale, dx, dy, 12, wf0=wf0)
    assert np.all(got[:, 0] == 0)
    assert rel_err(got, ref) < FP64_TOL


def test_dc_fp64_16_states_two_energy_chunks_multi_sweep(g128):
    """16 states (a 32-column +/- block, 8 rows per block) and 44 energies: the
    quasi-eigenstate kernels cover 32 energies x 16 states per block row, so
    each row takes two element chunks."""
    ip, ix, hv, dx, dy = g128.build_ham_dxy()
    n = ip.size - 1
    assert n > max_rows_per_sweep(32, 2)
    tnr = 24
    en_range = g128.energy_range
    energies = np.array([0.5 * i * en_range / tnr - en_range / 2. for i in range(2 * tnr)])
    sel = np.where((energies >= -8.0) & (energies <= 8.0))[0]
    assert sel.size > 32
    wf0 = unit_states(16, n, seed=31)
    bes = bessel_series(math.pi)
    t_step = 2 * math.pi / en_range
    dos, dc = f2py.tbpm_dccond_states(bes, ip, ix, hv, g128.rescale, dx, dy, wf0, tnr, t_step,
                                      energies, sel, 128, 1e-9)
    rdos, rdc = oracle.tbpm_dccond(bes, ip, ix, hv, g128.rescale, dx, dy, tnr, t_step,
                                   energies, sel, wf0=wf0)
    assert rel_err(dos, rdos) < FP64_TOL
    assert rel_err(dc, rdc) < FP64_TOL


def test_psi_t_fp64_one_state_multi_sweep():
    """One state (one thread per row, 128 rows per block) of 512 x 512 graphene
    (524,288 orbitals)."""
    s = tb.make_graphene_sample(512, 512, disorder=1.0, rescale=9.0, seed=41)
    h = s.build_ham_csr()
    n = h.shape[0]
    assert n > max_rows_per_sweep(1, 1)
    psi0 = unit_states(1, n, seed=43)[0]
    bes = bessel_series(math.pi)
    time_log = np.array([0, 1, 7, 12])
    got = f2py.tbpm_psi_t(bes, h.indptr, h.indices, h.data, psi0, time_log, 12, 128, 1e-9)
    ref = oracle.tbpm_psi_t(bes, h.indptr, h.indices, h.data, psi0, time_log, 12)
    assert rel_err(got, ref) < FP64_TOL
    assert np.allclose(np.linalg.norm(got, axis=0), 1.0, atol=1e-12)


def test_cheb_timestep_multi_sweep(g256):
    """The allocating time-step entry point on 16 states, forward then back."""
    from tbplas_b200 import _native as nat
    h = g256.build_ham_csr()
    n = h.shape[0]
    wf = unit_states(16, n, seed=17)
    ctx = f2py._ctx()
    ip32, ix32 = h.indptr.astype(np.int32), h.indices.astype(np.int32)
    hv = np.ascontiguousarray(h.data)
    ctx.call("tbpm_ham_upload", nat.ptr(ip32), nat.ptr(ix32), nat.ptr(hv), n, hv.size, None,
             None, 1.0)
    bes = np.asarray(bessel_series(math.pi))
    got = np.ascontiguousarray(wf.copy())
    ctx.call("tbpm_cheb_timestep", nat.ptr(bes), bes.size, nat.ptr(got), 16, 1)
    ref = np.stack([oracle.cheb_timestep(bes, h.indptr, h.indices, h.data, wf[b])
                    for b in range(16)])
    assert rel_err(got, ref) < 1e-12
    ctx.call("tbpm_cheb_timestep", nat.ptr(bes), bes.size, nat.ptr(got), 16, 0)
    back = np.stack([oracle.cheb_timestep(bes, h.indptr, h.indices, h.data, ref[b],
                                          forward=False) for b in range(16)])
    assert rel_err(got, back) < 1e-12


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_ring_and_grid_stride_term_kernels_agree(g256, prec):
    """The shared-memory ring kernel computes every element in the order of the
    grid-stride kernel: time-stepped states are bit-identical, correlations
    (whose block partials group differently) agree to rounding."""
    h = g256.build_ham_csr()
    n = h.shape[0]
    wf0 = unit_states(16, n, seed=19)
    bes = bessel_series(math.pi)
    out = {}
    for kernel in (1, 2):
        f2py.set_backend(precision=prec, term_kernel=kernel)
        out[kernel] = (f2py.tbpm_dos_states(bes, h.indptr, h.indices, h.data, wf0, 8, 4, 1e-9),
                       f2py.tbpm_psi_t(bes, h.indptr, h.indices, h.data, wf0[3],
                                       np.array([0, 5]), 5, 4, 1e-9))
    f2py.set_backend(term_kernel=0)
    assert np.array_equal(out[1][1], out[2][1])
    assert rel_err(out[2][0], out[1][0]) < (1e-13 if prec == "fp64" else 1e-6)


def test_ring_kernel_with_a_dense_row(graphene_small):
    """One row coupled to 300 others: its tile holds more CSR entries than a
    ring stage, so that tile's entries are read from global memory."""
    h = graphene_small.build_ham_csr()
    n = h.shape[0]
    rows, cols, vals = [], [], []
    for r in range(n):
        a, b = h.indptr[r], h.indptr[r + 1]
        c, v = list(h.indices[a:b]), list(h.data[a:b])
        if r == 5:
            c += list(range(60, 360))
            v += [0.001 * (1 + 0.5j)] * 300
        elif 60 <= r < 360:
            c += [5]
            v += [0.001 * (1 - 0.5j)]
        order = np.argsort(c)
        rows += [r] * len(c)
        cols += list(np.asarray(c)[order])
        vals += list(np.asarray(v)[order])
    ip = np.zeros(n + 1, dtype=np.int32)
    np.cumsum(np.bincount(rows, minlength=n), out=ip[1:])
    ix = np.array(cols, dtype=np.int32)
    hv = np.array(vals, dtype=np.complex128)
    wf0 = unit_states(16, n, seed=8)
    bes = bessel_series(math.pi)
    f2py.set_backend(term_kernel=2)  # the ring kernel at this small size
    got = f2py.tbpm_dos_states(bes, ip, ix, hv, wf0, 12, 128, 1e-9)
    f2py.set_backend(term_kernel=0)
    ref = oracle.tbpm_dos(bes, ip, ix, hv, 12, wf0=wf0)
    assert rel_err(got, ref) < FP64_TOL


@pytest.mark.parametrize("kernel", [0, 2])
@pytest.mark.parametrize("prec,tol", [("fp64", FP64_TOL), ("fp32", FP32_TOL)])
@pytest.mark.parametrize("case", ["dimer", "chain5", "diagonal_only", "one_row"])
def test_tiny_and_degenerate_hamiltonians(prec, tol, case, kernel):
    """Fewer rows than one tile of the ring kernel (60 rows at 16 states), row
    counts that are not multiples of 4 (the widened indptr window), no
    off-diagonal entries at all (no CSR slice to stage), and a single row;
    through the ring kernel (term_kernel 2) and the automatic choice (which
    takes the grid-stride kernel at these sizes)."""
    if case == "dimer":
        n, rows = 2, {0: [(1, -0.4)], 1: [(0, -0.4)]}
    elif case == "chain5":
        n = 5  # Hermitian: H[r][r+1] = -0.3 + 0.05i, H[r+1][r] its conjugate
        rows = {r: [(c, -0.3 + 0.05j if c > r else -0.3 - 0.05j)
                    for c in (r - 1, r + 1) if 0 <= c < n] for r in range(n)}
        rows[2].append((2, 0.1))
    elif case == "diagonal_only":
        n = 7
        rows = {r: [(r, 0.05 * (r - 3))] for r in range(n)}
    else:
        n, rows = 1, {0: [(0, 0.3)]}
    ip = np.zeros(n + 1, dtype=np.int32)
    ix, hv = [], []
    for r in range(n):
        ent = sorted(rows.get(r, []), key=lambda e: e[0])
        ip[r + 1] = ip[r] + len(ent)
        ix += [c for c, _ in ent]
        hv += [v for _, v in ent]
    ix = np.array(ix, dtype=np.int32)
    hv = np.array(hv, dtype=np.complex128)
    wf0 = unit_states(16, n, seed=3)
    bes = bessel_series(math.pi)
    f2py.set_backend(precision=prec, term_kernel=kernel)
    got = f2py.tbpm_dos_states(bes, ip, ix, hv, wf0, 20, 8, 1e-9)
    f2py.set_backend(term_kernel=0)
    ref = oracle.tbpm_dos(bes, ip, ix, hv, 20, wf0=wf0)
    assert rel_err(got, ref) < tol


def _launches():
    return f2py._ctx().last_stats()[0]


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_paired_terms_match_single_terms_bit_for_bit(g256, prec):
    """Two Chebyshev terms per launch (cheb_pair_kernel, term_kernel 3: the
    second term of a tile waits for the first term of every tile it couples
    to, and reads p_k from L2) give the states of one term per launch (the
    ring kernel, term_kernel 2, and the automatic choice 0) bit for bit, in
    fewer launches."""
    h = g256.build_ham_csr()
    n = h.shape[0]
    wf0 = unit_states(16, n, seed=23)
    bes = bessel_series(math.pi)
    out, launches = {}, {}
    for kernel in (2, 0, 3):
        f2py.set_backend(precision=prec, term_kernel=kernel)
        dos = f2py.tbpm_dos_states(bes, h.indptr, h.indices, h.data, wf0, 8, 4, 1e-9)
        launches[kernel] = _launches()
        psi = f2py.tbpm_psi_t(bes, h.indptr, h.indices, h.data, wf0[3], np.array([0, 5]), 5, 4,
                              1e-9)
        out[kernel] = (dos, psi)
    f2py.set_backend(term_kernel=0)
    for kernel in (0, 3):
        assert np.array_equal(out[kernel][0], out[2][0])
        assert np.array_equal(out[kernel][1], out[2][1])
    assert launches[0] == launches[2]
    assert launches[3] < 0.65 * launches[2]


def test_paired_terms_ac_and_dc_bit_for_bit(g128):
    """The AC block (48 columns, Fermi and time expansions) and the DC +/-
    block (32 columns) through paired terms equal the single-term ring."""
    ip, ix, hv, dx, dy = g128.build_ham_dxy()
    n = ip.size - 1
    wf0 = unit_states(16, n, seed=29)
    bes = bessel_series(math.pi / 2)
    beta = g128.rescale / (tb.KB * 3000.0)
    tnr = 12
    en_range = g128.energy_range
    energies = np.array([0.5 * i * en_range / tnr - en_range / 2. for i in range(2 * tnr)])
    sel = np.where((energies >= -8.0) & (energies <= 8.0))[0]
    t_step = 2 * math.pi / en_range
    out = {}
    for kernel in (2, 3):
        f2py.set_backend(term_kernel=kernel)
        ac = f2py.tbpm_accond_states(bes, beta, 0.0, ip, ix, hv, g128.rescale, dx, dy, wf0, tnr,
                                     2**15, 1e-12, 128, 1e-9)
        dos, dc = f2py.tbpm_dccond_states(bes, ip, ix, hv, g128.rescale, dx, dy, wf0[:8], tnr,
                                          t_step, energies, sel, 128, 1e-9)
        out[kernel] = (ac, dos, dc)
    f2py.set_backend(term_kernel=0)
    for a, b in zip(out[3], out[2]):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("prec,tol", [("fp64", FP64_TOL), ("fp32", FP32_TOL)])
def test_paired_terms_with_far_couplings(prec, tol):
    """A ring of 6,000 sites whose every site also couples to the site half
    the ring away: each row tile depends on a tile far down the sequence, so
    most second terms are placed after all first terms and wait on their
    flags (term_kernel 3 pairs them regardless of the L2 window)."""
    n = 6000
    rows = {}
    rng = np.random.default_rng(5)
    for r in range(n):
        ent = {(r + 1) % n: -1.0, (r - 1) % n: -1.0}
        ent[(r + n // 2) % n] = 0.3 + 0.1j if r < n // 2 else 0.3 - 0.1j
        ent[r] = rng.uniform(-0.5, 0.5)
        rows[r] = sorted(ent.items())
    ip = np.zeros(n + 1, dtype=np.int32)
    for r in range(n):
        ip[r + 1] = ip[r] + len(rows[r])
    ix = np.array([c for r in range(n) for c, _ in rows[r]], dtype=np.int32)
    hv = np.array([v for r in range(n) for _, v in rows[r]], dtype=np.complex128) / 3.0
    wf0 = unit_states(16, n, seed=7)
    bes = bessel_series(math.pi)
    f2py.set_backend(precision=prec, term_kernel=3)
    got = f2py.tbpm_dos_states(bes, ip, ix, hv, wf0, 16, 8, 1e-9)
    launches = _launches()
    f2py.set_backend(term_kernel=2)
    single = f2py.tbpm_dos_states(bes, ip, ix, hv, wf0, 16, 8, 1e-9)
    launches_single = _launches()
    f2py.set_backend(term_kernel=0)
    ref = oracle.tbpm_dos(bes, ip, ix, hv, 16, wf0=wf0)
    assert rel_err(got, ref) < tol
    assert np.array_equal(got, single)
    assert launches < 0.65 * launches_single


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_ring_row_windows_match_gathers_bit_for_bit(g256, g128, prec):
    """The ring kernel with row windows (term_kernel 4: each tile's neighbour
    rows staged into shared memory by bulk copies) gives the results of the
    ring kernel that gathers them from global memory (term_kernel 2) bit for
    bit: DOS on 256 x 256 graphene, the AC block and the DC +/- block on
    128 x 128."""
    h = g256.build_ham_csr()
    n = h.shape[0]
    wf0 = unit_states(16, n, seed=37)
    bes = bessel_series(math.pi)
    ip, ix, hv, dx, dy = g128.build_ham_dxy()
    n2 = ip.size - 1
    wf2 = unit_states(16, n2, seed=39)
    bes2 = bessel_series(math.pi / 2)
    beta = g128.rescale / (tb.KB * 3000.0)
    tnr = 12
    en_range = g128.energy_range
    energies = np.array([0.5 * i * en_range / tnr - en_range / 2. for i in range(2 * tnr)])
    sel = np.where((energies >= -8.0) & (energies <= 8.0))[0]
    t_step = 2 * math.pi / en_range
    out = {}
    for kernel in (2, 4):
        f2py.set_backend(precision=prec, term_kernel=kernel)
        dos = f2py.tbpm_dos_states(bes, h.indptr, h.indices, h.data, wf0, 8, 4, 1e-9)
        ac = f2py.tbpm_accond_states(bes2, beta, 0.0, ip, ix, hv, g128.rescale, dx, dy, wf2,
                                     tnr, 2**15, 1e-12, 128, 1e-9)
        dcd, dcc = f2py.tbpm_dccond_states(bes2, ip, ix, hv, g128.rescale, dx, dy, wf2[:8],
                                           tnr, t_step, energies, sel, 128, 1e-9)
        out[kernel] = (dos, ac, dcd, dcc)
    f2py.set_backend(term_kernel=0)
    for a, b in zip(out[4], out[2]):
        assert np.array_equal(a, b)
