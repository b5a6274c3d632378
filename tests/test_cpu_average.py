"""The oracle's restatement of the Wilson driver's loop operators with subtraction
levels (average / loopops / spacesum, Q/disconloops.f90:5343-5733, 7769-7910,
9012-9124; oracle/average.cpp) against an independent numpy statement:

  y = x - sub_k,  sub_1 = 0,  sub_k = sum_{n=0}^{k+1} kappa^n H^n b  (k >= 2),
  J_mu(x)     = conj( y(x+mu)^+ (1 - gamma_mu) U_mu(x)^+ b(x) - y(x)^+ (1 + gamma_mu) U_mu(x) b(x+mu) ),
  J_5(x)      = conj( y^+ b ) + 12 (k >= 2),   J_{5+mu}(x) = conj( y^+ gamma_mu b ),

with H the full-lattice hopping term (qqtest.hop_lex), neighbours across the edge times
bc(mu), time-slice sums, the caller's momentum factors on operators 1..5 in the
reference's slots, and operators 1..4 times kappa.  Random complex noise and solution,
antiperiodic time: 1e-12 relative to the largest entry."""
import numpy as np

import oracle
from qqtest import GAMMA, golden_gauge, half_to_lex, hop_lex, random_half, site_map

DIMS, BC = (4, 4, 4, 8), (1, 1, 1, -1)
AXES = (3, 2, 1, 0)


def closed_form(links, b, x, kappa, nsub, nmom, nop, momfac):
    nt = DIMS[3]
    sm = site_map(DIMS)
    sp = lambda M, v: np.einsum("st,...ta->...sa", M, v)  # noqa: E731
    dot = lambda a, c: np.einsum("...sa,...sa->...", np.conj(a), c)  # noqa: E731
    out = np.zeros((nop, nmom, nsub, nt), complex)
    sub = np.zeros_like(b)
    powers = [b]
    for k in range(1, nsub + 1):
        if k == 2:
            for n in range(1, 4):
                powers.append(hop_lex(links, powers[-1], BC))
            sub = sum(kappa ** n * powers[n] for n in range(4))
        elif k > 2:
            powers.append(hop_lex(links, powers[-1], BC))
            sub = sub + kappa ** (k + 1) * powers[k + 1]
        y = x - sub
        ops = []
        for mu in range(4):
            ax, U = AXES[mu], links[mu]
            n = DIMS[mu]
            sl = [slice(None)] * 4
            sl[ax] = n - 1
            yn = np.roll(y, -1, axis=ax)
            yn[tuple(sl)] *= BC[mu]
            bn = np.roll(b, -1, axis=ax)
            bn[tuple(sl)] *= BC[mu]
            udb = np.einsum("...ba,...sb->...sa", np.conj(U), b)
            ubn = np.einsum("...ab,...sb->...sa", U, bn)
            A = dot(yn, sp(np.eye(4) - GAMMA[mu], udb))
            B = dot(y, -sp(np.eye(4) + GAMMA[mu], ubn))
            ops.append(np.conj(A + B))
        ops.append(np.conj(dot(y, b)) + (12.0 if k >= 2 else 0.0))
        for mu in range(4):
            ops.append(np.conj(dot(y, sp(GAMMA[mu], b))))
        for iop in range(9):
            out[iop, 0, k - 1] = ops[iop].sum(axis=(1, 2, 3))
        for im in range(2, nmom + 1):
            mf = [None] + [momfac[kk - 1, im - 2, sm["ibl"] - 1, sm["ieo"] - 1, sm["isite"] - 1] for kk in range(1, 6)]
            S = lambda v: v.sum(axis=(1, 2, 3))  # noqa: E731
            out[0, im - 1, k - 1] = S(mf[3] * ops[0].imag) + 1j * S(mf[2] * ops[0].imag)
            out[1, im - 1, k - 1] = S(mf[1] * ops[1].imag) + 1j * S(mf[3] * ops[1].imag)
            out[2, im - 1, k - 1] = S(mf[2] * ops[2].imag) + 1j * S(mf[1] * ops[2].imag)
            out[3, im - 1, k - 1] = S(mf[4] * ops[3])
            out[4, im - 1, k - 1] = S(mf[5] * ops[4])
    out[:4] *= kappa
    return out


def test_average_closed_form():
    ol = oracle.OracleLattice(*DIMS, bc=BC)
    links, u = golden_gauge(DIMS, ol.ntotal, seed=37, eps=0.6)
    ol.set_gauge(u)
    be, bo = random_half(ol.ntotal, ol.nvhalf, 71), random_half(ol.ntotal, ol.nvhalf, 72)
    xe, xo = random_half(ol.ntotal, ol.nvhalf, 73), random_half(ol.ntotal, ol.nvhalf, 74)
    nsub, nmom, nop, kappa = 6, 3, 10, 0.153
    rng = np.random.default_rng(75)
    momfac = rng.standard_normal((5, nmom - 1, 16, 2, ol.nvhalf))
    J = ol.average(be, bo, xe, xo, kappa, nsub=nsub, nmom=nmom, nop=nop, momfac=momfac)
    b = half_to_lex(be, DIMS, 1) + half_to_lex(bo, DIMS, 2)
    x = half_to_lex(xe, DIMS, 1) + half_to_lex(xo, DIMS, 2)
    want = closed_form(links, b, x, kappa, nsub, nmom, nop, momfac)
    got = J[..., 0] + 1j * J[..., 1]
    assert np.abs(want).max() > 0 and np.all(got[9:] == 0)
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
    # every level differs (the subtraction is active) and each operator is exercised
    assert np.all(np.abs(np.diff(got[:9, 0], axis=1)).max(axis=(1, 2)) > 0)


def test_momfacs_library_matches_oracle():
    """qq_momfacs (host code of the library) against the oracle's literal restatement
    of momfacs (Q/disconloops.f90:8925-8984): bit for bit, two origins, two shapes."""
    import baylorlqcd_b200 as qq

    for dims, io in [((4, 4, 4, 8), (1, 1, 1)), ((8, 4, 4, 8), (3, 2, 4))]:
        ol = oracle.OracleLattice(*dims, bc=BC)
        assert np.array_equal(qq.momfacs(dims, io), ol.momfacs(io))
        mf = ol.momfacs(io)
        assert np.array_equal(mf[4], mf[3]) and np.abs(mf).max() > 0


def test_generalaverage_styles_1_and_2_are_average_levels():
    """generalaverage (Q/disconloops.f90:119-333) builds its style 1 from nsaverage (the
    operators of the unsubtracted solution with zero momentum factors, :3079-3143) and its
    style 2 as NS - PS, PS = -average of a zero solution.  average is linear in the solution
    apart from the constant on psibar psi of the subtracted levels, which the zero-solution
    run carries too, so NS - PS at level k equals average's level k: checked on the oracle,
    at imom = 1 and zero momentum factors, as generalaverage calls them."""
    ol = oracle.OracleLattice(*DIMS, bc=BC)
    _, u = golden_gauge(DIMS, ol.ntotal, seed=41, eps=0.6)
    ol.set_gauge(u)
    be, bo = random_half(ol.ntotal, ol.nvhalf, 81), random_half(ol.ntotal, ol.nvhalf, 82)
    xe, xo = random_half(ol.ntotal, ol.nvhalf, 83), random_half(ol.ntotal, ol.nvhalf, 84)
    kappa, nsub, nmom, nop = 0.153, 6, 5, 9
    zero = np.zeros((5, nmom - 1, 16, 2, ol.nvhalf))
    J = ol.average(be, bo, xe, xo, kappa, nsub, nmom, nop, zero)
    PS = -ol.average(be, bo, ol.new_half(), ol.new_half(), kappa, nsub, nmom, nop, zero)
    NS = J[:, 0, 0]  # style 1: level 1, imom = 1
    assert np.abs(PS[:, 0, 0]).max() == 0.0  # nothing to subtract at level 1
    for k in range(nsub):
        style2 = NS - PS[:, 0, k]
        np.testing.assert_allclose(style2, J[:, 0, k], rtol=0, atol=1e-12 * np.abs(J).max())
    assert np.abs(J[:, 1:]).max() == 0.0  # zero momentum factors: only imom = 1 survives
