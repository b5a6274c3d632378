"""The oracle's restatement of the eigenmode subtraction of the Wilson loop driver
(oracle/eigen.cpp: eigmodesofM, eigmodesofMprime, xigenerator, eigaverage,
Q/disconloops.f90:1593-1937, 2573-2875, 465-838, 3239-3342) against independent numpy
statements on a 4^4 heatbath configuration:

  * every kept mode of M = 1 - kappa D is an eigenpair, M R = lambda R, computed with the
    numpy hopping term (qqtest.hop_lex), to 1e-8 (the routine's own acceptance bound);
    its left vector satisfies M^H L = conj(lambda) L; <R_i, L_j> = delta_ij; the modes
    come in conjugate pairs and are sorted by |lambda|;
  * every kept mode of M gamma5 is an orthonormal eigenpair with a real eigenvalue;
  * xiinv(isub, j) = <L_j, S_isub R_j> with S_isub = sum_{n <= isub+1} kappa^n H^n in
    numpy (gamma5 S for the M gamma5 modes), to 1e-12;
  * eigaverage equals the prefix sums of s_j <L_j, z> times the level-1 loop operators of
    each mode alone (oq_average, itself checked in test_cpu_average.py), for both the M
    modes (loopops) and the M gamma5 modes (loopops of gamma5 x'), with the eigstart /
    eigstep selection, to 1e-12."""
import numpy as np
import pytest

import oracle
from qqtest import GAMMA, GAMMA5, half_to_lex, hop_lex

DIMS, BC = (4, 4, 4, 4), (1, 1, 1, -1)
KAPPA = (0.15, 0.0)


@pytest.fixture(scope="module")
def lat():
    ol = oracle.OracleLattice(*DIMS, bc=BC)
    u = ol.coldstart()
    oracle.initlagfib(0, 7)
    ol.heatbath(u, 5.8, 20)
    ol.set_gauge(u)
    return ol


def links_of(ol):
    """Links (4, nt, nz, ny, nx, 3, 3) from the oracle's reference-layout field."""
    from qqtest import site_map

    sm = site_map(DIMS)
    u = ol.u  # (16, 2, 4, ntotal, 18)
    out = np.zeros((4,) + tuple(reversed(DIMS)) + (3, 3), complex)
    for mu in range(4):
        v = u[sm["ibl"] - 1, sm["ieo"] - 1, mu, sm["isite"] - 1, :]
        out[mu] = (v[..., 0::2] + 1j * v[..., 1::2]).reshape(v.shape[:-1] + (3, 3))
    return out


def lex(full):
    return half_to_lex(full[0], DIMS, 1) + half_to_lex(full[1], DIMS, 2)


def spin(M, v):
    return np.einsum("st,...ta->...sa", M, v)


@pytest.fixture(scope="module")
def modes(lat):
    ev, R, L, cyc = lat.eigmodes(1, (30, 16), 40, KAPPA)
    return ev, R, L


@pytest.fixture(scope="module")
def modes_p(lat):
    oracle.initlagfib(0, 11)
    se, so = lat.z4source()
    ev, R, L, cyc = lat.eigmodes(2, (30, 16), 40, KAPPA, se, so)
    return ev, R, L


def test_modes_of_m_are_eigenpairs(lat, modes):
    ev, R, L = modes
    assert len(ev) >= 6 and len(ev) % 2 == 0
    links = links_of(lat)
    k = KAPPA[0]
    for j, lam in enumerate(ev):
        r, l_ = lex(R[j]), lex(L[j])
        res = r - k * hop_lex(links, r, BC) - lam * r
        assert np.linalg.norm(res) < 1e-8, j
        resl = l_ - k * hop_lex(links, l_, BC, idag=1) - np.conj(lam) * l_
        assert np.linalg.norm(resl) < 1e-6 * np.linalg.norm(l_), j
    assert np.all(np.diff(np.abs(ev)) >= -1e-14)
    for j in range(0, len(ev), 2):  # pairs lambda, conj(lambda) share |lambda|
        assert np.isclose(abs(ev[j]), abs(ev[j + 1]), rtol=1e-8)
    G = np.array([[np.vdot(lex(R[i]), lex(L[j])) for j in range(len(ev))] for i in range(len(ev))])
    np.testing.assert_allclose(G, np.eye(len(ev)), atol=1e-10)


def test_modes_of_m_gamma5_are_orthonormal_eigenpairs(lat, modes_p):
    ev, R, _ = modes_p
    assert len(ev) >= 4
    assert np.all(ev.imag == 0.0)
    links = links_of(lat)
    k = KAPPA[0]
    for j, lam in enumerate(ev):
        r = lex(R[j])
        g5r = spin(GAMMA5, r)
        res = g5r - k * hop_lex(links, g5r, BC) - lam.real * r
        assert np.linalg.norm(res) < 1e-5, j
    assert np.all(np.diff(np.abs(ev.real)) >= 0)
    G = np.array([[np.vdot(lex(R[i]), lex(R[j])) for j in range(len(ev))] for i in range(len(ev))])
    np.testing.assert_allclose(G, np.eye(len(ev)), atol=1e-8)


@pytest.mark.parametrize("which", ["m", "mprime"])
def test_xigenerator(lat, modes, modes_p, which):
    ev, R, L = modes if which == "m" else modes_p
    gammaid = 1 if which == "m" else 2
    k = KAPPA[0]
    xi = lat.xigenerator(R, L, k, gammaid)
    links = links_of(lat)
    for j in range(len(ev)):
        r, l_ = lex(R[j]), lex(L[j])
        powers = [r]
        for _ in range(7):
            powers.append(hop_lex(links, powers[-1], BC))
        for isub in range(1, 7):
            s = np.zeros_like(r) if isub == 1 else sum(k ** n * powers[n] for n in range(isub + 2))
            if gammaid == 2:
                s = spin(GAMMA5, s)
            want = np.vdot(l_, s)
            assert abs(xi[j, isub - 1] - want) <= 1e-12 * max(1.0, abs(want)), (j, isub)


@pytest.mark.parametrize("which", ["m", "mprime"])
@pytest.mark.parametrize("eigstart,eigstep", [(1, 1), (2, 3)])
def test_eigaverage_is_prefix_sum_of_mode_traces(lat, modes, modes_p, which, eigstart, eigstep):
    ev, R, L = modes if which == "m" else modes_p
    eshfes = 1 if which == "m" else 2
    k = KAPPA[0]
    oracle.initlagfib(0, 5)
    ze, zo = lat.z4source()
    scal = 1.0 / ev
    J = lat.eigaverage(ze, zo, k, R, L, scal, eshfes, eigstart, eigstep)
    n = len(ev)
    acc = np.zeros((9, DIMS[3]), complex)
    for e in range(1, n + 1):
        r = R[e - 1].copy()
        if eshfes == 2:
            r[0] = lat.gam5x(r[0])
            r[1] = lat.gam5x(r[1])
        T = lat.average(ze, zo, r[0], r[1], k, nsub=1, nmom=1, nop=9)[:, 0, 0]  # (9, nt, 2)
        c = (lat.vecdot(L[e - 1][0], ze) + lat.vecdot(L[e - 1][1], zo)) * scal[e - 1]
        acc += c * (T[..., 0] + 1j * T[..., 1])
        got = J[:, e - 1, :, 0] + 1j * J[:, e - 1, :, 1]
        pick = e == eigstart or (e > eigstart and (e - eigstart) % eigstep == 0) or e == n
        if pick:
            np.testing.assert_allclose(got, acc, rtol=0, atol=1e-12 * max(1.0, np.abs(acc).max()))
        else:
            assert np.all(got == 0.0)


# ---- the polynomial estimators (ppaverage*, xipolygenerator, oracle/eigen.cpp) ----
TERMS = {  # (coefficient, power) added at levels 2..6, 1-based (Q/disconloops.f90:5740-7434)
    11: {2: [(1, 1), (2, 2), (3, 3), (4, 4)], 3: [(5, 5)], 4: [(6, 6)], 5: [(7, 7)],
         6: [(8, 8), (9, 9), (10, 10), (11, 11)]},
    8: {2: [(1, 1), (2, 2), (3, 3), (4, 4)], 3: [(5, 5)], 4: [(6, 6)], 5: [(7, 7)], 6: [(8, 8)]},
    5: {2: [(1, 1), (2, 2), (3, 3), (4, 4)], 3: [(5, 5)], 4: [(5, 6)], 5: [(5, 7)], 6: [(5, 8)]},
}


def mpowers(links, b, n):
    out = [b]
    for _ in range(n - 1):
        out.append(out[-1] - KAPPA[0] * hop_lex(links, out[-1], BC))
    return out


@pytest.fixture(scope="module")
def noise(lat):
    oracle.initlagfib(0, 23)
    return lat.z4source()


@pytest.mark.parametrize("p", [5, 8, 11])
def test_ppcoeffs_minimise_the_polynomial_residual(lat, noise, p):
    """The normal-equation fit reaches the least-squares residual of numpy's lstsq on the
    Krylov matrix (the coefficients themselves are ill-conditioned)."""
    ze, zo = noise
    co = lat.ppcoeffs(ze, zo, KAPPA[0], p)
    b = half_to_lex(ze, DIMS, 1) + half_to_lex(zo, DIMS, 2)
    K = np.stack([v.ravel() for v in mpowers(links_of(lat), b, p + 1)[1:]], axis=1)
    best = np.linalg.lstsq(K, b.ravel(), rcond=None)[0]
    r_fit = np.linalg.norm(b.ravel() - K @ co)
    r_best = np.linalg.norm(b.ravel() - K @ best)
    assert r_fit <= r_best * (1 + 1e-5) + 1e-12 * np.linalg.norm(b)
    assert r_fit < np.linalg.norm(b)


@pytest.mark.parametrize("p", [5, 8, 11])
def test_ppaverage_levels(lat, noise, p):
    """Level isub: loop operators of x - sum of the level terms' co_c M^(v-1) b, against
    numpy-built subtractions through the oracle's loop operators."""
    from qqtest import lex_to_half

    ze, zo = noise
    rng = np.random.default_rng(p)
    co = rng.standard_normal(p) + 1j * rng.standard_normal(p)
    xe = lat.new_half()
    xo = lat.new_half()
    xe[:, :, :, :lat.nvhalf] = rng.standard_normal(xe[:, :, :, :lat.nvhalf].shape)
    xo[:, :, :, :lat.nvhalf] = rng.standard_normal(xo[:, :, :, :lat.nvhalf].shape)
    J = lat.ppaverage(p, co, ze, zo, xe, xo, KAPPA[0])
    b = half_to_lex(ze, DIMS, 1) + half_to_lex(zo, DIMS, 2)
    V = mpowers(links_of(lat), b, 12)
    sub = np.zeros_like(b)
    for isub in range(1, 7):
        for c, v in TERMS[p].get(isub, []):
            sub = sub + co[c - 1] * V[v - 1]
        ye = xe - lex_to_half(sub, DIMS, lat.ntotal, 1)
        yo = xo - lex_to_half(sub, DIMS, lat.ntotal, 2)
        want = lat.loop_slices(ze, zo, ye, yo, 0 if isub == 1 else 1, KAPPA[0])
        assert np.abs(J[:, isub - 1] - want).max() <= 1e-11 * np.abs(want).max(), isub


def test_xipolygenerator(lat, modes_p, noise):
    ev, R, _ = modes_p
    ze, zo = noise
    co = lat.ppcoeffs(ze, zo, KAPPA[0], 8)
    xi = lat.xipolygenerator(R, R, KAPPA[0], co)
    links = links_of(lat)
    for j in range(len(ev)):
        r = lex(R[j])
        V = mpowers(links, r, 9)
        sub = np.zeros_like(r)
        for isub in range(1, 7):
            for c, v in TERMS[8].get(isub, []):
                sub = sub + co[c - 1] * V[v - 1]
            want = np.vdot(r, spin(GAMMA5, sub))
            assert abs(xi[j, isub - 1] - want) <= 1e-11 * max(1.0, abs(want)), (j, isub)
