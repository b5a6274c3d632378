"""The oracle's level-0 loop traces (twAverage with nsub = 0, Q/vevbleft.f90:2541-4704,
restated literally in oracle/loops.cpp) against their closed form, evaluated here in
numpy.  With eta the real part of the noise (twAverage uses only that) and
x' = x - cos(delta) (cos(delta) - sin(delta) i gamma5) eta, per time slice t:

  J_mu(t) = kappa sum_{y in t} [eta(y+mu)^T (1+gamma_mu) U_mu(y)^+ x'(y)
                                - eta(y)^T (1-gamma_mu) U_mu(y) x'(y+mu)]
  psibar psi (t) = sum eta^T x',  psibar gamma5 psi (t) = sum eta^T gamma5 x'

(periodic wrap without the boundary sign; dobndry = 1 drops the time current of the
last slice).  Operator order J4, psibar psi, J1, J2, J3, psibar gamma5 psi.
Tolerance 1e-12 relative to the largest entry (FP64, different summation order)."""
import numpy as np
import pytest

import oracle
from qqtest import GAMMA, GAMMA5, golden_gauge, half_to_lex, random_half

BC = (1, 1, 1, -1)


def closed_form(links, eta, x, kappa, delta, dobndry):
    J5 = 1j * GAMMA5
    sp = lambda M, v: np.einsum("st,...ta->...sa", M, v)  # noqa: E731
    xp = x - np.cos(delta) * (np.cos(delta) * eta - np.sin(delta) * sp(J5, eta))
    nt = x.shape[0]
    out = np.zeros((6, nt), complex)
    axes = {0: 3, 1: 2, 2: 1, 3: 0}
    slot = {3: 0, 0: 2, 1: 3, 2: 4}
    for mu in range(4):
        U = links[mu]
        eta_f = np.roll(eta, -1, axis=axes[mu])
        xp_f = np.roll(xp, -1, axis=axes[mu])
        Udx = np.einsum("...ba,...sb->...sa", np.conj(U), xp)  # U^+ x'(y)
        Ux = np.einsum("...ab,...sb->...sa", U, xp_f)  # U x'(y+mu)
        a = np.einsum("...sa,...sa->...", eta_f, sp(np.eye(4) + GAMMA[mu], Udx))
        b = np.einsum("...sa,...sa->...", eta, sp(np.eye(4) - GAMMA[mu], Ux))
        val = a - b
        if mu == 3 and dobndry == 1:
            val[-1] = 0.0
        out[slot[mu]] = kappa * val.sum(axis=(1, 2, 3))
    out[1] = np.einsum("...sa,...sa->...", eta, xp).sum(axis=(1, 2, 3))
    out[5] = np.einsum("...sa,...sa->...", eta, sp(GAMMA5, xp)).sum(axis=(1, 2, 3))
    return out


@pytest.mark.parametrize("dims", [(4, 4, 4, 8), (8, 4, 4, 4)])
@pytest.mark.parametrize("delta,dobndry", [(0.0, 0), (0.0, 1), (0.37, 0)])
def test_level0_traces_closed_form(dims, delta, dobndry):
    ol = oracle.OracleLattice(*dims, bc=BC)
    links, u = golden_gauge(dims, ol.ntotal, seed=31, eps=0.6)
    ol.set_gauge(u)
    oracle.initlagfib(0, 13)
    be, bo = ol.z4source()
    xe = random_half(ol.ntotal, ol.nvhalf, 32)
    xo = random_half(ol.ntotal, ol.nvhalf, 33)
    kappa = 0.1565
    J = ol.twaverage_level0(be, bo, xe, xo, kappa, delta, dobndry)
    noise = half_to_lex(be, dims, 1) + half_to_lex(bo, dims, 2)
    x = half_to_lex(xe, dims, 1) + half_to_lex(xo, dims, 2)
    want = closed_form(links, noise.real, x, kappa, delta, dobndry)
    got = J[..., 0] + 1j * J[..., 1]
    assert np.abs(got - want).max() < 1e-12 * np.abs(want).max()
    live = np.ones(want.shape, bool)
    if dobndry == 1:
        live[0, -1] = False  # the time current of the last slice is dropped
        assert want[0, -1] == 0 and got[0, -1] == 0
    assert np.abs(want[live]).min() > 0  # every other operator and slice is exercised


def test_level0_uses_only_the_real_part_of_the_noise():
    dims = (4, 4, 4, 8)
    ol = oracle.OracleLattice(*dims, bc=BC)
    _, u = golden_gauge(dims, ol.ntotal, seed=31, eps=0.6)
    ol.set_gauge(u)
    be, bo = random_half(ol.ntotal, ol.nvhalf, 41), random_half(ol.ntotal, ol.nvhalf, 42)
    xe, xo = random_half(ol.ntotal, ol.nvhalf, 43), random_half(ol.ntotal, ol.nvhalf, 44)
    J1 = ol.twaverage_level0(be, bo, xe, xo, 0.15)
    be[..., 1::2] = 7.0
    bo[..., 1::2] = -3.0
    J2 = ol.twaverage_level0(be, bo, xe, xo, 0.15)
    assert np.array_equal(J1, J2)


def closed_form_mom(links, eta, x, kappa, delta, dobndry, io, nmom, r=1):
    """The same per-site values with twAverage's momentum projections (:4434-4503):
    imom 2..5 weight rho, psibar psi and psibar gamma5 psi by ffac(y) and take
    (Im J1 fas3, Im J2 fas1), (Im J3 fas2, Im J1 fas2), (Im J2 fas3, Im J3 fas1) as the
    (real, imaginary) slots of operators 3, 4, 5, each factor at the site y the value
    sits on.  Wilson r enters as (r +- gamma_mu) in place of (1 +- gamma_mu)
    (currentCalc2M differs from currentCalc2P by the sign of the diagonal terms)."""
    import vevref

    J5 = 1j * GAMMA5
    sp = lambda M, v: np.einsum("st,...ta->...sa", M, v)  # noqa: E731
    xp = x - np.cos(delta) * (np.cos(delta) * eta - np.sin(delta) * sp(J5, eta))
    nt, nz, ny, nx = x.shape[:4]
    axes = {0: 3, 1: 2, 2: 1, 3: 0}
    site = {}
    for mu in range(4):
        U = links[mu]
        Udx = np.einsum("...ba,...sb->...sa", np.conj(U), xp)
        Ux = np.einsum("...ab,...sb->...sa", U, np.roll(xp, -1, axis=axes[mu]))
        a = np.einsum("...sa,...sa->...", np.roll(eta, -1, axis=axes[mu]), sp(r * np.eye(4) + GAMMA[mu], Udx))
        b = np.einsum("...sa,...sa->...", eta, sp(r * np.eye(4) - GAMMA[mu], Ux))
        val = kappa * (a - b)
        if mu == 3 and dobndry == 1:
            val[-1] = 0.0
        site[mu] = val
    psi = np.einsum("...sa,...sa->...", eta, xp)
    psu = np.einsum("...sa,...sa->...", eta, sp(GAMMA5, xp))
    mf = vevref.momentum_factors((nx, ny, nz, nt), io)
    fac = np.zeros((4, 5, nz, ny, nx))  # (ffac, fas1, fas2, fas3), k
    for z in range(nz):
        for y in range(ny):
            for xx in range(nx):
                f = mf(xx, y, z)
                for k in range(1, 5):
                    for a_ in range(4):
                        fac[a_, k, z, y, xx] = f[a_][k]
    out = np.zeros((6, nmom, nt), complex)
    S = lambda v, w=1.0: (v * w).sum(axis=(1, 2, 3))  # noqa: E731
    out[:, 0] = [S(site[3]), S(psi), S(site[0]), S(site[1]), S(site[2]), S(psu)]
    for k in range(1, nmom):
        ff, f1, f2, f3 = fac[0, k], fac[1, k], fac[2, k], fac[3, k]
        out[0, k] = S(site[3], ff)
        out[1, k] = S(psi, ff)
        out[2, k] = S(site[0].imag, f3) + 1j * S(site[1].imag, f1)
        out[3, k] = S(site[2].imag, f2) + 1j * S(site[0].imag, f2)
        out[4, k] = S(site[1].imag, f3) + 1j * S(site[2].imag, f1)
        out[5, k] = S(psu, ff)
    return out


@pytest.mark.parametrize("delta,dobndry,io,r", [(0.0, 0, (1, 1, 1), 1), (0.37, 1, (3, 2, 4), 1),
                                                (0.0, 0, (2, 1, 1), -1), (-0.21, 1, (1, 3, 2), -1)])
def test_momentum_traces_closed_form(delta, dobndry, io, r):
    dims = (4, 4, 4, 8)
    ol = oracle.OracleLattice(*dims, bc=BC)
    links, u = golden_gauge(dims, ol.ntotal, seed=35, eps=0.6)
    ol.set_gauge(u)
    oracle.initlagfib(0, 17)
    be, bo = ol.z4source()
    xe = random_half(ol.ntotal, ol.nvhalf, 52)
    xo = random_half(ol.ntotal, ol.nvhalf, 53)
    J = ol.twaverage(be, bo, xe, xo, 0.1565, delta, io=io, dobndry=dobndry, nmom=5, ir=r)
    noise = half_to_lex(be, dims, 1) + half_to_lex(bo, dims, 2)
    x = half_to_lex(xe, dims, 1) + half_to_lex(xo, dims, 2)
    want = closed_form_mom(links, noise.real, x, 0.1565, delta, dobndry, io, 5, r)
    got = J[..., 0] + 1j * J[..., 1]
    assert np.abs(got - want).max() < 1e-12 * np.abs(want).max()
    assert np.abs(want[:, 1:]).max() > 0
    if r == 1:
        J0 = ol.twaverage_level0(be, bo, xe, xo, 0.1565, delta, dobndry)
        assert np.array_equal(J[:, 0], J0)
