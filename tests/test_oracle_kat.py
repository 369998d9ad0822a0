"""Known-answer tests that pin the CPU oracle (no GPU).

The reference Fortran cannot be compiled here, so the oracle is pinned by
mathematics: every driver is checked against an exact-diagonalisation
evaluation of the same formulas (tbpm.f90 semantics: time grids, the t=1 quirk
of tbpm_accond, Hanning-windowed quasi-eigenstates of tbpm_dccond), the
Fermi expansion against direct quadrature, and the random-state generator
against the published Philox4x32-10 known-answer vectors.
"""

import math

import numpy as np
import pytest

import tbplas_b200 as tb
from oracle import oracle

from conftest import bessel_series, rel_err, unit_states


def test_philox_published_vectors():
    # Random123 known-answer vectors for Philox4x32-10
    assert oracle.philox4x32_10([0, 0, 0, 0], [0, 0]).tolist() == \
        [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]
    assert oracle.philox4x32_10([0xffffffff] * 4, [0xffffffff] * 2).tolist() == \
        [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]
    assert oracle.philox4x32_10([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344],
                                [0xa4093822, 0x299f31d0]).tolist() == \
        [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]


def test_random_state_distribution():
    """random.f90:36-69: |z|^2 ~ Exp(1), uniform phase, unit norm."""
    n = 200000
    wf = oracle.random_state(n, 1337 * 49741 // 49741, kind=0)
    assert abs(np.linalg.norm(wf) - 1) < 1e-12
    a2 = np.abs(wf) ** 2 * n
    assert abs(a2.mean() - 1) < 0.01 and abs(a2.var() - 1) < 0.05  # Exp(1)
    ph = np.angle(wf)
    assert abs(np.mean(np.cos(ph))) < 0.01 and abs(np.mean(np.sin(ph))) < 0.01
    u = oracle.random_state(1000, 7, kind=1)
    assert np.allclose(np.abs(u), 1 / math.sqrt(1000), rtol=1e-12)
    assert not np.allclose(oracle.random_state(100, 7), oracle.random_state(100, 8))


def _dense(s):
    h = s.build_ham_csr()
    return h, h.toarray()


def _propagator(Hd, tau):
    E, V = np.linalg.eigh(Hd)
    return lambda psi, m: V @ (np.exp(-1j * E * tau * m) * (V.conj().T @ psi))


@pytest.fixture(scope="module")
def small():
    s = tb.make_graphene_sample(6, 5, disorder=1.0, rescale=9.0, seed=11)
    s.set_magnetic_field(40.0)
    return s


def test_oracle_dos_exact_diagonalisation(small):
    h, Hd = _dense(small)
    bes = bessel_series(math.pi)
    wf = unit_states(2, h.shape[0], seed=2)
    corr = oracle.tbpm_dos(bes, h.indptr, h.indices, h.data, 80, wf0=wf)
    U = _propagator(Hd, math.pi)
    exact = np.array([np.mean([np.vdot(w, U(w, t)) for w in wf]) for t in range(81)])
    assert np.max(np.abs(corr - exact)) < 1e-12


def test_oracle_backward_step_and_psi_t(small):
    h, Hd = _dense(small)
    bes = bessel_series(math.pi)
    psi = unit_states(1, h.shape[0], seed=3)[0]
    U = _propagator(Hd, math.pi)
    back = oracle.cheb_timestep(bes, h.indptr, h.indices, h.data, psi, forward=False)
    assert np.max(np.abs(back - U(psi, -1))) < 1e-13
    tl = [0, 2, 9, 20]
    got = oracle.tbpm_psi_t(bes, h.indptr, h.indices, h.data, psi, tl, 20)
    for j, t in enumerate(tl):
        assert np.max(np.abs(got[:, j] - U(psi, t))) < 1e-12


def _fermi(beta, mu, e):
    return 1.0 / (1.0 + np.exp(beta * (e - mu)))


def test_oracle_fermi_coefficients_quadrature():
    beta = 9.0 / (tb.KB * 300)
    mu = 0.05
    coef = oracle.fermi_cheb_coef(2**15, beta, mu, False, 1e-12)
    n_cheb = 2**14
    theta = np.linspace(0, np.pi, 2**20 + 1)
    f = _fermi(beta, mu, np.cos(theta))
    q = math.pi / n_cheb
    for k in (0, 1, 2, 5, 33, 200):
        g = 0.5 if k == 0 else ((n_cheb - k) * math.cos(q * k) +
                                math.sin(q * k) / math.tan(q)) / n_cheb
        ck = g * 2 / np.pi * np.trapezoid(f * np.cos(k * theta), theta)
        assert abs(coef[k] - ck) < 1e-9
    # truncation rule: the last two kept coefficients are not both below eps
    assert abs(coef[-1]) < 1e-12 or abs(coef[-2]) >= 1e-12
    omf = oracle.fermi_cheb_coef(2**15, beta, mu, True, 1e-12)
    m = min(len(coef), len(omf))
    assert abs(coef[0] + omf[0] - 1.0) < 1e-12
    assert np.max(np.abs(coef[1:m] + omf[1:m])) < 1e-12


def test_oracle_fermi_operator_exact(small):
    h, Hd = _dense(small)
    beta = 9.0 / (tb.KB * 300)
    coef = oracle.fermi_cheb_coef(2**15, beta, 0.0, False, 1e-12)
    psi = unit_states(1, h.shape[0], seed=4)[0]
    got = oracle.fermi(coef, h.indptr, h.indices, h.data, psi)
    E, V = np.linalg.eigh(Hd)
    fE = np.polynomial.chebyshev.chebval(E, coef)
    exact = V @ (fE * (V.conj().T @ psi))
    assert np.max(np.abs(got - exact)) < 1e-11


def _current(s, which):
    ip, ix, hop, dx, dy = s.build_ham_dxy()
    d = dx if which == 0 else dy
    n = ip.size - 1
    J = np.zeros((n, n), dtype=complex)
    rows = np.repeat(np.arange(n), np.diff(ip))
    np.add.at(J, (rows, ix), 1j * s.rescale * hop * d)
    return J


def test_oracle_ac_exact_diagonalisation():
    s = tb.make_graphene_sample(5, 4, disorder=0.5, rescale=9.0, seed=5)
    ip, ix, hop, dx, dy = s.build_ham_dxy()
    n = ip.size - 1
    Hd = np.zeros((n, n), dtype=complex)
    rows = np.repeat(np.arange(n), np.diff(ip))
    np.add.at(Hd, (rows, ix), hop)
    Jx, Jy = _current(s, 0), _current(s, 1)
    assert np.allclose(Jx, Jx.conj().T) and np.allclose(Jy, Jy.conj().T)
    bes = bessel_series(math.pi / 2)
    beta = 9.0 / (tb.KB * 300)
    wf = unit_states(2, n, seed=6)
    T = 12
    corr = oracle.tbpm_accond(bes, beta, 0.0, ip, ix, hop, s.rescale, dx, dy, T, wf0=wf)
    cf = oracle.fermi_cheb_coef(2**15, beta, 0.0, False, 1e-12)
    comf = oracle.fermi_cheb_coef(2**15, beta, 0.0, True, 1e-12)
    E, V = np.linalg.eigh(Hd)
    F = V @ np.diag(np.polynomial.chebyshev.chebval(E, cf)) @ V.conj().T
    OMF = V @ np.diag(np.polynomial.chebyshev.chebval(E, comf)) @ V.conj().T
    U = _propagator(Hd, math.pi / 2)
    exact = np.zeros((4, T), dtype=complex)
    for w in wf:
        p1x, p1y, p2 = OMF @ (Jx @ w), OMF @ (Jy @ w), F @ w
        for t in range(2, T + 1):
            a, b, c = U(p1x, t - 1), U(p1y, t - 1), U(p2, t - 1)
            exact[:, t - 1] += np.array([np.vdot(c, Jx @ a), np.vdot(c, Jy @ a),
                                         np.vdot(c, Jx @ b), np.vdot(c, Jy @ b)]) / len(wf)
    assert np.all(corr[:, 0] == 0)
    assert np.max(np.abs(corr - exact)) < 1e-11 * max(1.0, np.max(np.abs(exact)))


def test_oracle_dc_exact_diagonalisation():
    s = tb.make_graphene_sample(5, 4, disorder=0.5, rescale=9.0, seed=8)
    ip, ix, hop, dx, dy = s.build_ham_dxy()
    n = ip.size - 1
    Hd = np.zeros((n, n), dtype=complex)
    rows = np.repeat(np.arange(n), np.diff(ip))
    np.add.at(Hd, (rows, ix), hop)
    J = [_current(s, 0), _current(s, 1)]
    bes = bessel_series(math.pi)
    T = 10
    en_range = s.energy_range
    energies = np.array([0.5 * i * en_range / T - en_range / 2. for i in range(2 * T)])
    qe = np.where(np.abs(energies) <= 3.0)[0]
    t_step = 2 * math.pi / en_range
    wf = unit_states(1, n, seed=9)
    dos, dc = oracle.tbpm_dccond(bes, ip, ix, hop, s.rescale, dx, dy, T, t_step, energies, qe,
                                 wf0=wf)
    U = _propagator(Hd, math.pi)
    w0 = wf[0]
    exact_dos = np.array([np.vdot(w0, U(w0, t)) for t in range(1, T + 1)])
    assert np.max(np.abs(dos - exact_dos)) < 1e-12
    QE = []
    for i in qe:
        q = w0.copy()
        for t in range(1, T + 1):
            W = 0.5 * (1 + math.cos(math.pi * t / T))
            P = np.exp(1j * energies[i] * t * t_step)
            q = q + P * U(w0, t) * W + np.conj(P) * U(w0, -t) * W
        q = q / np.linalg.norm(q)
        QE.append(q / abs(np.vdot(w0, q)))
    exact = np.zeros((2, energies.size, T), dtype=complex)
    for k in range(2):
        wj = J[k] @ w0
        for t in range(1, T + 1):
            wt = U(wj, t - 1)
            for i, q in enumerate(QE):
                exact[k, i, t - 1] = np.vdot(wt, J[k] @ q)
    assert np.max(np.abs(dc - exact)) < 1e-11 * np.max(np.abs(exact))
    assert np.all(dc[:, qe.size:, :] == 0)


def test_oracle_norm_check_stops():
    s = tb.make_graphene_sample(6, 6, rescale=2.0)
    h = s.build_ham_csr()
    with pytest.raises(oracle.OracleError):
        oracle.tbpm_dos(bessel_series(math.pi), h.indptr, h.indices, h.data, 12,
                        wf0=unit_states(1, h.shape[0]), chk_step=6)


def test_oracle_reproduces_golden_solver_runs():
    """The golden correlations were produced by the reference Solver driving
    the oracle with the stored states: rerun them with this repository's Bessel
    series and CSR builder to pin both against the reference Python layer."""
    import os
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_tbplas.npz"))
    states = g["solver/states"]
    ip, ix, data = g["g7x5_dis/csr_indptr"], g["g7x5_dis/csr_indices"], g["g7x5_dis/csr_data"]
    corr = oracle.tbpm_dos(g["solver/bessel_dos"], ip, ix, data, 64, wf0=states)
    assert rel_err(corr, g["solver/corr_dos"]) < 1e-13
    dip, dix, dhop = g["g7x5_dis/dxy_indptr"], g["g7x5_dis/dxy_indices"], g["g7x5_dis/dxy_hop"]
    dx, dy = g["g7x5_dis/dxy_dx"], g["g7x5_dis/dxy_dy"]
    beta_re, mu_re = g["solver/beta_mu_re"]
    ac = oracle.tbpm_accond(g["solver/bessel_ac"], beta_re, mu_re, dip, dix, dhop, 9.0, dx, dy,
                            32, wf0=states)
    assert rel_err(ac, g["solver/corr_ac"]) < 1e-13
    dos, dc = oracle.tbpm_dccond(g["solver/bessel_dos"], dip, dix, dhop, 9.0, dx, dy, 32,
                                 float(g["solver/time_step"]), g["solver/dc_energies"],
                                 g["solver/dc_qe_indices"], wf0=states)
    assert rel_err(dos, g["solver/corr_dos_dc"]) < 1e-13
    assert rel_err(dc, g["solver/corr_dc"]) < 1e-13
