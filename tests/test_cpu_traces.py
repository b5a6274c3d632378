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
