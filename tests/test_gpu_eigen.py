"""GPU parity of the eigenmode subtraction of the Wilson loop driver (qq_eigmodes,
qq_xigenerator, qq_eigaverage: eigmodesofM, eigmodesofMprime, xigenerator, eigaverage,
Q/disconloops.f90:1593-1937, 2573-2875, 465-838, 3239-3342) with the oracle's
restatement (oracle/eigen.cpp, checked against numpy in test_cpu_eigen.py), through the C
ABI, on heatbath configurations made by the oracle and uploaded.

Both sides run the same deflated-restart iteration in a different summation order, so
the kept modes agree up to the phase of each eigenvector.  What is compared is what does
not depend on the phases: the eigenvalues (1e-9), the modes' residuals and left/right
biorthogonality on the GPU's own vectors, xiinv (phase free: <L, S R> with <R, L> = 1,
or <R, gamma5 S R> for unit R) and the eigaverage prefix sums (1e-8 of the largest
entry).  Modes are compared over the leading run whose eigenvalues agree; a pair at the
1e-8 acceptance border may be kept on one side only.  One case uses a 141-vector basis
and 61 restart vectors, which takes the chunked multi-vector kernels (128 vectors per
launch) and the tiled restart combination through more than one chunk."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

BC = (1, 1, 1, -1)
KAPPA = (0.15, 0.0)


def make(dims, seed, sweeps):
    import baylorlqcd_b200 as qq

    ol = oracle.OracleLattice(*dims, bc=BC)
    u = ol.coldstart()
    oracle.initlagfib(0, seed)
    ol.heatbath(u, 5.8, sweeps)
    ol.set_gauge(u)
    lat = qq.Lattice(*dims, bc=BC)
    lat.gauge_upload(u)
    return ol, lat


def pair_order(ev, kind):
    """Index order with each conjugate pair of M's modes sorted by imaginary part.  The
    reference sorts the kept modes by |lambda| alone, so the two members of a pair (equal
    |lambda| up to rounding) come in either order on either side; what is compared is
    therefore per pair, and cumulative quantities only at even mode counts."""
    idx = list(range(len(ev)))
    if kind == 1:
        j = 0
        while j < len(ev) - 1:
            if abs(ev[j] - np.conj(ev[j + 1])) <= 1e-8 * abs(ev[j]):
                if ev[j].imag > ev[j + 1].imag:
                    idx[j], idx[j + 1] = idx[j + 1], idx[j]
                j += 2
            else:
                j += 1
    return idx


def leading_match(a, b, tol=1e-9):
    n = 0
    for x, y in zip(a, b):
        if abs(x - y) > tol * max(1.0, abs(y)):
            break
        n += 1
    return n


def cvec(ol, full):
    nv = ol.nvhalf
    return (full[:, ..., :nv, 0::2] + 1j * full[:, ..., :nv, 1::2]).ravel()


@pytest.fixture(scope="module")
def small():
    ol, lat = make((4, 4, 4, 4), 7, 20)
    yield ol, lat
    lat.close()


@pytest.mark.parametrize("kind,nG,cyc", [(1, (30, 16), 40), (2, (30, 16), 40), (1, (140, 60), 4)])
def test_eigenmodes_match_oracle(small, kind, nG, cyc):
    ol, lat = small
    se = so = None
    if kind == 2:
        oracle.initlagfib(0, 11)
        se, so = ol.z4source()
    ev_o, R_o, L_o, cyc_o = ol.eigmodes(kind, nG, cyc, KAPPA, se, so)
    E = lat.eigenmodes(kind, nG, cyc, KAPPA, se, so)
    assert E.cycles == cyc_o <= cyc
    og, oo = pair_order(E.evals, kind), pair_order(ev_o, kind)
    n = leading_match(E.evals[og], ev_o[oo])
    if kind == 1:
        n -= n % 2  # whole pairs
    assert len(ev_o) >= 4 and n >= min(E.num, len(ev_o)) - 2 and n >= 4, (E.evals, ev_o)
    # the GPU's vectors: eigenpairs of the oracle's operator, biorthonormal
    k = KAPPA[0]
    R = np.stack([E.vector(og[j]) for j in range(n)])
    L = np.stack([E.vector(og[j], left=True) for j in range(n)])
    for j in range(n):
        r = R[j]
        if kind == 1:
            mr0 = r[0] - k * ol.hsingle(r[1], 0, 1)
            mr1 = r[1] - k * ol.hsingle(r[0], 0, 2)
            lam = E.evals[og[j]]
            bound = 1e-8
        else:
            g0, g1 = ol.gam5x(r[0]), ol.gam5x(r[1])
            mr0 = g0 - k * ol.hsingle(g1, 0, 1)
            mr1 = g1 - k * ol.hsingle(g0, 0, 2)
            lam = E.evals[og[j]].real
            bound = 1e-5
        res = np.concatenate([cvec(ol, mr0[None]) - lam * cvec(ol, r[0][None]),
                              cvec(ol, mr1[None]) - lam * cvec(ol, r[1][None])])
        assert np.linalg.norm(res) < bound, (j, np.linalg.norm(res))
    G = np.array([[np.vdot(cvec(ol, R[i]), cvec(ol, L[j])) for j in range(n)] for i in range(n)])
    np.testing.assert_allclose(G, np.eye(n), atol=1e-8)
    # phase-free derived quantities against the oracle's
    xi_g = E.xigenerator(k)[og[:n]]
    xi_o = ol.xigenerator(R_o[:n], L_o[:n], k, kind)[oo[:n]]
    assert np.abs(xi_g - xi_o).max() <= 1e-8 * np.abs(xi_o).max()
    oracle.initlagfib(0, 5)
    ze, zo = ol.z4source()
    scal_o = 1.0 / ev_o[:n]
    scal_g = np.zeros(E.num, complex)
    scal_g[:n] = 1.0 / E.evals[:n]
    for eigstart, eigstep in ((1, 1), (2, 3)):
        J_o = ol.eigaverage(ze, zo, k, R_o[:n], L_o[:n], scal_o, kind, eigstart, eigstep)
        J_g = E.eigaverage(ze, zo, k, scal_g, eigstart, eigstep)
        # the counts both sides evaluate over the common modes: whole pairs for M
        counts = [c for c in range(1, n + 1) if c == eigstart or (c > eigstart and (c - eigstart) % eigstep == 0)]
        if kind == 1:
            counts = [c for c in counts if c % 2 == 0]
        for c in counts:
            assert np.abs(J_g[:, c - 1] - J_o[:, c - 1]).max() <= 1e-8 * np.abs(J_o).max(), c
    E.close()


def test_unit_source_needs_no_start_vector_and_bad_arguments(small):
    import baylorlqcd_b200 as qq

    ol, lat = small
    with pytest.raises(qq.QQError):
        lat.eigenmodes(2, (20, 10), 2, KAPPA)  # kind 2 without a start vector
    with pytest.raises(qq.QQError):
        lat.eigenmodes(1, (20, 20), 2, KAPPA)  # k must be below m
    with pytest.raises(qq.QQError):
        lat.eigenmodes(3, (20, 10), 2, KAPPA)


@pytest.fixture(scope="module")
def noise(small):
    ol, _ = small
    oracle.initlagfib(0, 23)
    return ol.z4source()


@pytest.mark.parametrize("p", [5, 8, 11])
def test_ppcoeffs_and_ppaverage_match_oracle(small, noise, p):
    """The GPU fit reaches the oracle's polynomial residual ||z - sum co_b M^b z|| (the
    coefficients themselves are ill-conditioned); with the same coefficients the levels of
    ppaverage / ppaverage1 / ppaverage2 agree to 1e-10."""
    ol, lat = small
    ze, zo = noise
    co_g = lat.ppcoeffs(ze, zo, KAPPA[0], p)
    co_o = ol.ppcoeffs(ze, zo, KAPPA[0], p)

    def cmul(c, v):
        w = np.zeros_like(v)
        z = c * (v[..., 0::2] + 1j * v[..., 1::2])
        w[..., 0::2], w[..., 1::2] = z.real, z.imag
        return w

    def resid(co):
        ve, vo = ze.copy(), zo.copy()
        re_, ro_ = ze.copy(), zo.copy()
        for c in co:
            ve, vo = ve - KAPPA[0] * ol.hsingle(vo, 0, 1), vo - KAPPA[0] * ol.hsingle(ve, 0, 2)
            re_, ro_ = re_ - cmul(c, ve), ro_ - cmul(c, vo)
        return np.sqrt(ol.vecdot(re_, re_).real + ol.vecdot(ro_, ro_).real)

    r_g, r_o = resid(co_g), resid(co_o)
    assert abs(r_g - r_o) <= 1e-6 * r_o, (r_g, r_o)
    rng = np.random.default_rng(p)
    xe, xo = ol.new_half(), ol.new_half()
    xe[:, :, :, :ol.nvhalf] = rng.standard_normal(xe[:, :, :, :ol.nvhalf].shape)
    xo[:, :, :, :ol.nvhalf] = rng.standard_normal(xo[:, :, :, :ol.nvhalf].shape)
    J_g = lat.ppaverage(p, co_o, ze, zo, xe, xo, KAPPA[0])
    J_o = ol.ppaverage(p, co_o, ze, zo, xe, xo, KAPPA[0])
    assert np.abs(J_g - J_o).max() <= 1e-10 * np.abs(J_o).max()


def test_generalaverage_matches_oracle(small, noise):
    """All ten estimator styles of generalaverage for one noise: the GPU's modes and
    components against the oracle's (same polynomial coefficients, a random solution
    vector; every style is phase free)."""
    ol, lat = small
    ze, zo = noise
    k = KAPPA[0]
    oracle.initlagfib(0, 11)
    se, so = ol.z4source()
    m_o = ol.eigmodes(1, (30, 16), 40, KAPPA)
    mp_o = ol.eigmodes(2, (30, 16), 40, KAPPA, se, so)
    m_g = lat.eigenmodes(1, (30, 16), 40, KAPPA)
    mp_g = lat.eigenmodes(2, (30, 16), 40, KAPPA, se, so)
    assert m_g.num == len(m_o[0]) and mp_g.num == len(mp_o[0])
    np.testing.assert_allclose(m_g.evals[pair_order(m_g.evals, 1)], m_o[0][pair_order(m_o[0], 1)], rtol=1e-9)
    np.testing.assert_allclose(mp_g.evals, mp_o[0], rtol=1e-9)
    co = {p: ol.ppcoeffs(ze, zo, k, p) for p in (5, 8, 11)}
    oracle.initlagfib(0, 31)
    pe, po = ol.z4source()
    copoly = ol.ppcoeffs(pe, po, k, 8)
    xi_g = mp_g.xipolygenerator(k, copoly)
    xi_o = ol.xipolygenerator(mp_o[1], mp_o[1], k, copoly)
    assert np.abs(xi_g - xi_o).max() <= 1e-8 * np.abs(xi_o).max()
    rng = np.random.default_rng(3)
    xe, xo = ol.new_half(), ol.new_half()
    xe[:, :, :, :ol.nvhalf] = rng.standard_normal(xe[:, :, :, :ol.nvhalf].shape)
    xo[:, :, :, :ol.nvhalf] = rng.standard_normal(xo[:, :, :, :ol.nvhalf].shape)
    J_g = lat.generalaverage(m_g, mp_g, ze, zo, xe, xo, k, co[11], co[8], co[5], copoly)
    J_o = ol.generalaverage(m_o[:3], mp_o[:2], ze, zo, xe, xo, k, co[11], co[8], co[5], copoly)
    assert J_g.shape == J_o.shape
    scale = np.abs(J_o).max()
    # styles 3 and 5 carry the M modes: whole pairs only (mode counts 2, 4, ...)
    for sty in range(10):
        e = slice(1, None, 2) if sty in (2, 4) else slice(None)
        assert np.abs(J_g[:, sty, e] - J_o[:, sty, e]).max() <= 1e-8 * scale, sty + 1
    assert np.all(J_g[:, 0, 1:] == 0.0) and np.all(J_g[:, 0, 0, 1:] == 0.0)  # style 1: mode 1, level 1
    m_g.close()
    mp_g.close()
