"""Known answers for the oracle's restatements of tbpm_dyn_pol, tbpm_eigenstates,
tbpm_kbdc and ldos_haydock (tbplas/fortran/tbpm.f90:355-493, 721-1026,
propagation.f90:85-155, funcs.f90:125-172).

Each driver is checked against a dense evaluation of the same formulas:
propagators and Chebyshev polynomials from the exact eigen-decomposition of
the rescaled Hamiltonian, Fermi operators as the same Chebyshev series
evaluated on the eigenvalues, currents as dense matrices, and the Lanczos
recursion through its moment identity and the closed form of a chain.
"""

import math

import numpy as np
import pytest

import tbplas_b200 as tb
from oracle import oracle

from conftest import bessel_series, unit_states


@pytest.fixture(scope="module")
def small():
    s = tb.make_graphene_sample(6, 5, disorder=1.0, rescale=9.0, seed=11)
    s.set_magnetic_field(40.0)
    return s


def _eig(s):
    h = s.build_ham_csr()
    E, V = np.linalg.eigh(h.toarray())
    return h, E, V


def _apply(E, V, fE, psi):
    return V @ (fE * (V.conj().T @ psi))


def test_oracle_dyn_pol_exact(small):
    h, E, V = _eig(small)
    n = h.shape[0]
    beta = 9.0 / (tb.KB * 300) * 1.0
    mu = 0.1 / 9.0
    cf = oracle.fermi_cheb_coef(2**15, beta, mu, False, 1e-12)
    comf = oracle.fermi_cheb_coef(2**15, beta, mu, True, 1e-12)
    pos = small.orb_pos
    q = np.array([[1.3, 0.4, 0.0], [0.2, 2.0, 0.1]])
    wf = unit_states(2, n, seed=5)
    tnr = 20
    bes = bessel_series(math.pi / 2)
    got = oracle.tbpm_dyn_pol(bes, beta, mu, h.indptr, h.indices, h.data, pos[:, 0],
                              pos[:, 1], pos[:, 2], q, tnr, wf0=wf)
    fE = np.polynomial.chebyshev.chebval(E, cf)
    omfE = np.polynomial.chebyshev.chebval(E, comf)
    exact = np.zeros((2, tnr))
    for iq in range(2):
        ph = pos @ q[iq]
        dq = np.exp(1j * ph)
        for w in wf:
            p1 = _apply(E, V, omfE, np.conj(dq) * w)
            p2 = _apply(E, V, fE, w)
            for t in range(tnr):
                u = np.exp(-1j * E * (math.pi / 2) * t)
                a, b = _apply(E, V, u, p1), _apply(E, V, u, p2)
                exact[iq, t] += np.vdot(b, dq * a).imag / 2
    assert np.max(np.abs(got - exact)) < 1e-12 * max(1.0, np.max(np.abs(exact)))


def test_oracle_eigenstates_exact(small):
    h, E, V = _eig(small)
    n = h.shape[0]
    wf = unit_states(2, n, seed=6)
    tnr = 24
    t_step = 2 * math.pi / small.energy_range
    energies = np.array([-0.4, 0.0, 0.25])
    bes = bessel_series(math.pi)
    got = oracle.tbpm_eigenstates(bes, h.indptr, h.indices, h.data, tnr, t_step, energies,
                                  wf0=wf)
    exact = np.zeros((3, n))
    for w in wf:
        for i, en in enumerate(energies):
            q = w.astype(complex).copy()
            for k in range(1, tnr + 1):
                W = 0.5 * (1 + math.cos(math.pi * k / tnr))
                P = np.exp(1j * en * k * t_step)
                fwd = _apply(E, V, np.exp(-1j * E * math.pi * k), w)
                bwd = _apply(E, V, np.exp(1j * E * math.pi * k), w)
                q += W * (P * fwd + np.conj(P) * bwd)
            q /= np.linalg.norm(q)
            exact[i] += np.abs(q) ** 2 / 2
    assert np.max(np.abs(got - exact)) < 1e-12 * np.max(exact)


def test_oracle_kbdc_exact(small):
    h, E, V = _eig(small)
    n = h.shape[0]
    ip, ix, hop, dx, dy = small.build_ham_dxy()
    from scipy.sparse import csr_matrix
    Hd = csr_matrix((hop, ix, ip), shape=(n, n)).toarray()
    E2, V2 = np.linalg.eigh(Hd)
    jx = csr_matrix((1j * small.rescale * hop * dx, ix, ip), shape=(n, n)).toarray()
    jy = csr_matrix((1j * small.rescale * hop * dy, ix, ip), shape=(n, n)).toarray()
    wf = unit_states(2, n, seed=8)
    nk = 12
    theta = np.arccos(np.clip(E2, -1, 1))
    g = np.array([0.5] + [((nk - k) * math.cos(math.pi / nk * k) +
                          math.sin(math.pi / nk * k) / math.tan(math.pi / nk)) / nk
                          for k in range(1, nk)])
    for direction, ja in ((1, jx), (2, jy)):
        got = oracle.tbpm_kbdc(ip, ix, hop, small.rescale, dx, dy, nk, direction, wf0=wf)
        exact = np.zeros((nk, nk), dtype=complex)
        for w in wf:
            left = [_apply(E2, V2, np.cos(m * theta), jx @ w) for m in range(nk)]
            right = [ja @ _apply(E2, V2, np.cos(m * theta), w) for m in range(nk)]
            for i in range(nk):
                for j in range(nk):
                    exact[i, j] += g[i] * g[j] * np.vdot(left[i], right[j]) / 2
        assert np.max(np.abs(got - exact)) < 1e-11 * np.max(np.abs(exact))


def test_oracle_haydock_chain_closed_form():
    """Ring of 64 sites, hopping t: from one site b = (sqrt(2)|t|, |t|, |t|, ...),
    a = 0, for depths inside the ring."""
    n, t, rescale = 64, -1.3, 3.0
    rows = np.arange(n)
    from scipy.sparse import csr_matrix
    m = csr_matrix((np.full(2 * n, t / rescale, dtype=complex),
                    (np.concatenate([rows, rows]),
                     np.concatenate([(rows + 1) % n, (rows - 1) % n]))), shape=(n, n))
    m.sort_indices()
    a, b = oracle.haydock_coef([5], m.indptr, m.indices, m.data, rescale, 20,
                               wf_sites=np.array([[1.0 + 0j]]))
    assert np.max(np.abs(a)) < 1e-13
    assert abs(b[0] - math.sqrt(2) * abs(t)) < 1e-13
    assert np.max(np.abs(b[1:] - abs(t))) < 1e-12


def test_oracle_haydock_moments(small):
    """Lanczos identity <n1|H^k|n1> = (T^k)_{00} for k < 2*depth."""
    h, E, V = _eig(small)
    n = h.shape[0]
    sites = [3, 17, 40]
    w = unit_states(1, len(sites), seed=9)
    a, b = oracle.haydock_coef(sites, h.indptr, h.indices, h.data, small.rescale, 8,
                               wf_sites=w)
    psi = np.zeros(n, dtype=complex)
    psi[sites] = w[0]
    Hphys = h.toarray() * small.rescale
    T = np.diag(a.real) + np.diag(b[:-1], 1) + np.diag(b[:-1], -1)
    for k in range(1, 12):
        mk = np.vdot(psi, np.linalg.matrix_power(Hphys, k) @ psi).real
        tk = np.linalg.matrix_power(T, k)[0, 0]
        assert abs(mk - tk) < 1e-9 * max(1.0, abs(mk))
    en, ldos = oracle.ldos_haydock(sites, 0.05, small.energy_range, h.indptr, h.indices,
                                   h.data, small.rescale, 1, 8, 200, 1, wf_sites=w)
    assert en.size == 401 and abs(en[0] + small.energy_range / 2) < 1e-12
    assert np.all(ldos > 0)
