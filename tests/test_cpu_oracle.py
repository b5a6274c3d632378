"""Pins the oracle (the CPU restatement of the reference in oracle/) without the
reference binary, which cannot be built here (Fortran).  Known answers:

* the hopping term against an independent numpy restatement (qqtest.hop_lex) and,
  on the free field, against the analytic plane-wave eigenvalue
  sum_mu 2 (c1 cos p_mu - i c2 gamma_mu sin p_mu) with antiperiodic time momenta;
* adjointness (idag paths) and gauge covariance;
* the dense 4^4 Schur-complement matrix assembled column by column, its solve and
  its smallest eigenvalues against numpy (GMRES-DR solution and harmonic Ritz values);
* fermprop's full-lattice solution against a dense numpy solve of
  M = (1 + 2 i kappa mu gamma5) - kappa H for every in-scope inverter;
* the restated pseudolapack against numpy LAPACK;
* the Z(2)/Z(4) noise rules and draw order of Q/disconloops.f90:4518-4649.

Floating-point tolerances are stated per test (FP64 throughout)."""
import numpy as np
import pytest

import oracle
from qqtest import (GAMMA, GAMMA5, golden_gauge, half_to_lex, half_to_vec, hop_lex, interior_basis,
                    lex_to_half, random_half, site_map, su3_gram_schmidt, vec_to_half)

BC = (1, 1, 1, -1)


@pytest.fixture(scope="module", params=[(4, 4, 4, 8), (8, 4, 4, 4)], ids=["4x4x4x8", "8x4x4x4"])
def cfg(request):
    dims = request.param
    ol = oracle.OracleLattice(*dims, bc=BC)
    links, u = golden_gauge(dims, ol.ntotal, seed=7, eps=0.6)
    ol.set_gauge(u)
    return ol, links, dims


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def parity_mask(dims, gblclr):
    return site_map(dims)["gblclr"] == gblclr


# ---------------------------------------------------------------- operator
@pytest.mark.parametrize("idag", [0, 1])
@pytest.mark.parametrize("gblclr", [1, 2])
def test_hsingle_matches_numpy(cfg, idag, gblclr):
    """1e-13 relative: same arithmetic, different summation order."""
    ol, links, dims = cfg
    gin = random_half(ol.ntotal, ol.nvhalf, 11 + gblclr)
    out = ol.hsingle(gin, idag, gblclr)
    ref = hop_lex(links, half_to_lex(gin, dims, 3 - gblclr), BC, idag=idag)
    m = parity_mask(dims, gblclr)
    assert rel(half_to_lex(out, dims, gblclr)[m], ref[m]) < 1e-13


def test_hsingle_anisotropic_coefficients(cfg):
    ol, links, dims = cfg
    c1, c2 = (0.9, 1.1, 1.0, 0.7), (1.2, 0.8, 1.0, 1.3)
    ol2 = oracle.OracleLattice(*dims, bc=BC, c1=c1, c2=c2)
    ol2.set_gauge(ol.u)
    gin = random_half(ol.ntotal, ol.nvhalf, 21)
    out = ol2.hsingle(gin, 0, 1)
    ref = hop_lex(links, half_to_lex(gin, dims, 2), BC, c1=c1, c2=c2)
    m = parity_mask(dims, 1)
    assert rel(half_to_lex(out, dims, 1)[m], ref[m]) < 1e-13


def test_free_field_plane_wave():
    """KAT-1: U = 1, psi(x) = exp(i p.x) chi -> (H psi)(x) = sum_mu 2 (c1 cos p_mu -
    i c2 gamma_mu sin p_mu) psi(x); p_t = (2 pi n + pi)/nt for the antiperiodic time."""
    dims = (4, 4, 4, 8)
    ol = oracle.OracleLattice(*dims, bc=BC)
    ol.set_gauge(ol.coldstart())
    rng = np.random.default_rng(3)
    chi = rng.standard_normal((4, 3)) + 1j * rng.standard_normal((4, 3))
    nx, ny, nz, nt = dims
    for n in [(0, 0, 0, 0), (1, 0, 2, 3), (3, 1, 1, 6)]:
        p = [2 * np.pi * n[0] / nx, 2 * np.pi * n[1] / ny, 2 * np.pi * n[2] / nz, (2 * np.pi * n[3] + np.pi) / nt]
        t, z, y, x = np.meshgrid(np.arange(nt), np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        phase = np.exp(1j * (p[0] * x + p[1] * y + p[2] * z + p[3] * t))
        psi = phase[..., None, None] * chi
        K = sum(2 * np.cos(p[mu]) * np.eye(4) - 2j * np.sin(p[mu]) * GAMMA[mu] for mu in range(4))
        want = phase[..., None, None] * (K @ chi)
        out = ol.hsingle(lex_to_half(psi, dims, ol.ntotal, 2), 0, 1)
        m = parity_mask(dims, 1)
        assert rel(half_to_lex(out, dims, 1)[m], want[m]) < 1e-13


def test_hsingle_adjoint(cfg):
    """KAT-3: <y_e, H_eo x_o> = <(H^dagger)_oe y_e, x_o>, H^dagger = the idag = 1 path."""
    ol, _, _ = cfg
    x = random_half(ol.ntotal, ol.nvhalf, 31)
    y = random_half(ol.ntotal, ol.nvhalf, 32)
    lhs = ol.vecdot(y, ol.hsingle(x, 0, 1))
    rhs = np.conj(ol.vecdot(x, ol.hsingle(y, 1, 2)))
    assert abs(lhs - rhs) < 1e-12 * abs(lhs)


def jmul(g, s=1.0):
    """g -> g + s J g per site, J = i gamma5: (s0, s1, s2, s3) -> (s2, s3, -s0, -s1)."""
    out = g.copy()
    out[:, :, 0] += s * g[:, :, 2]
    out[:, :, 1] += s * g[:, :, 3]
    out[:, :, 2] -= s * g[:, :, 0]
    out[:, :, 3] -= s * g[:, :, 1]
    return out


def test_hdbletm_adjoint_wilson(cfg):
    """mu = 0: A^dagger is the idag = 1 path."""
    ol, _, _ = cfg
    x = random_half(ol.ntotal, ol.nvhalf, 41)
    y = random_half(ol.ntotal, ol.nvhalf, 42)
    lhs = ol.vecdot(y, ol.hdbletm(x, 0, (0.13, 0.0)))
    rhs = np.conj(ol.vecdot(x, ol.hdbletm(y, 1, (0.13, 0.0))))
    assert abs(lhs - rhs) < 1e-12 * abs(lhs)


def test_hdbletm_adjoint_twisted(cfg):
    """mu > 0: idag flips only gamma_mu (Q/diracops.f90:483-514), so the adjoint
    (1 - 2 i k mu g5)/k^2 - H+_eo (1 + 2 i k mu g5) H+_oe / (1 + 4 k^2 mu^2) is built
    from Hsingle(idag = 1) and the twist here."""
    ol, _, _ = cfg
    k, mu = 0.13, 0.04
    n = ol.nvhalf
    x = random_half(ol.ntotal, n, 41)
    y = random_half(ol.ntotal, n, 42)
    h = jmul(ol.hsingle(y, 1, 2), 2 * k * mu)
    h[:, :, :, n:] = 0.0
    ady = y / k**2 - (2 * mu / k) * (jmul(y, 1.0) - y) - ol.hsingle(h, 1, 1) / (1 + 4 * k * k * mu * mu)
    lhs = ol.vecdot(y, ol.hdbletm(x, 0, (k, mu)))
    rhs = np.conj(ol.vecdot(x, ady))
    assert abs(lhs - rhs) < 1e-12 * abs(lhs)


def test_hdbletm_negative_mu_is_wilson(cfg):
    """The reference switches to Hdouble whenever kappa(2) < 1e-8
    (Q/diracops.f90:467-477), negative twisted masses included."""
    ol, _, _ = cfg
    g = random_half(ol.ntotal, ol.nvhalf, 44)
    n = ol.nvhalf
    a = ol.hdbletm(g, 0, (0.13, -0.04))
    b = ol.hdouble(g, 0, 0.13)
    assert np.array_equal(a[:, :, :, :n], b[:, :, :, :n])


def test_hdouble_is_wilson_hdbletm(cfg):
    ol, _, _ = cfg
    g = random_half(ol.ntotal, ol.nvhalf, 43)
    a = ol.hdouble(g, 0, 0.13)
    b = ol.hdbletm(g, 0, (0.13, 0.0))
    n = ol.nvhalf
    assert rel(a[:, :, :, :n], b[:, :, :, :n]) < 1e-14


def test_gauge_covariance(cfg):
    """KAT-4: U'_mu(x) = W(x) U_mu(x) W(x+mu)^+, psi' = W psi  =>  H' psi' = W H psi."""
    ol, links, dims = cfg
    from qqtest import gauge_to_ref

    nx, ny, nz, nt = dims
    W = su3_gram_schmidt(nx * ny * nz * nt, np.random.default_rng(5)).reshape(nt, nz, ny, nx, 3, 3)
    axes = {0: 3, 1: 2, 2: 1, 3: 0}
    lp = np.empty_like(links)
    for mu in range(4):
        Wn = np.roll(W, -1, axis=axes[mu])
        lp[mu] = W @ links[mu] @ np.conj(np.swapaxes(Wn, -1, -2))
    olp = oracle.OracleLattice(*dims, bc=BC)
    olp.set_gauge(gauge_to_ref(lp, dims, ol.ntotal))
    psi = half_to_lex(random_half(ol.ntotal, ol.nvhalf, 51), dims, 2)
    psip = np.einsum("...ab,...sb->...sa", W, psi)
    out = half_to_lex(ol.hsingle(lex_to_half(psi, dims, ol.ntotal, 2), 0, 1), dims, 1)
    outp = half_to_lex(olp.hsingle(lex_to_half(psip, dims, ol.ntotal, 2), 0, 1), dims, 1)
    m = parity_mask(dims, 1)
    assert rel(outp[m], np.einsum("...ab,...sb->...sa", W, out)[m]) < 1e-13


def test_twmshift_matches_numpy(cfg):
    """twMshift (Q/diracops.f90:1863-1995, iflag = -1) literally:
    h = g - J g / (2 kappa mu) - J H g / (2 mu) on each half, J = i gamma5, i.e.
    (-J / (2 kappa mu)) (1 + 2 i kappa mu gamma5 + kappa H) -- the shift solvers'
    convention, with the opposite sign of H to fermprop's operator."""
    ol, links, dims = cfg
    k, mu = 0.13, 0.03
    g = np.stack([random_half(ol.ntotal, ol.nvhalf, 61), random_half(ol.ntotal, ol.nvhalf, 62)])
    out = ol.twmshift(g, 0, (k, mu))
    psi = half_to_lex(g[0], dims, 1) + half_to_lex(g[1], dims, 2)
    J = 1j * GAMMA5
    Jm = lambda v: np.einsum("st,...ta->...sa", J, v)
    want = psi - Jm(psi) / (2 * k * mu) - Jm(hop_lex(links, psi, BC)) / (2 * mu)
    got = half_to_lex(out[0], dims, 1) + half_to_lex(out[1], dims, 2)
    assert rel(got, want) < 1e-13


# ---------------------------------------------------------------- dense 4^4
def full_operator_apply(links, psi, kappa):
    k, mu = kappa
    tw = np.einsum("st,...ta->...sa", np.eye(4) + 2j * k * mu * GAMMA5, psi)
    return tw - k * hop_lex(links, psi, BC)


@pytest.fixture(scope="module")
def dense44():
    dims = (4, 4, 4, 4)
    ol = oracle.OracleLattice(*dims, bc=BC)
    links, u = golden_gauge(dims, ol.ntotal, seed=9, eps=0.5)
    ol.set_gauge(u)
    kappa = (0.124, 0.0)
    n = 192 * ol.nvhalf
    basis = interior_basis(ol.nvhalf)
    A = np.zeros((n, n), complex)
    for j in range(n):
        e = np.zeros((8, 2, 4, ol.ntotal, 6))
        e[basis[0][j], basis[1][j], basis[2][j], basis[3][j], basis[4][j]] = 1.0
        A[:, j] = half_to_vec(ol.hdbletm(e, 0, kappa), ol.nvhalf)
    return ol, links, dims, kappa, A


def test_dense_schur_complement_matches_numpy(dense44):
    """KAT-2 (operator): the oracle's columns against (1/kappa^2 - H_eo H_oe) in numpy."""
    ol, links, dims, kappa, A = dense44
    rng = np.random.default_rng(71)
    v = rng.standard_normal(A.shape[0]) + 1j * rng.standard_normal(A.shape[0])
    psi = half_to_lex(vec_to_half(v, ol.ntotal, ol.nvhalf), dims, 1)
    h = hop_lex(links, psi, BC) * parity_mask(dims, 2)[..., None, None]
    want = psi / kappa[0] ** 2 - hop_lex(links, h, BC)
    want_v = half_to_vec(lex_to_half(want, dims, ol.ntotal, 1), ol.nvhalf)
    assert rel(A @ v, want_v) < 1e-13


def test_gmresdr_solution_and_deflation_space(dense44):
    """KAT-2 (solver): GMRES-DR(20,6) solution against numpy.linalg.solve (1e-9
    relative).  Its deflation space obeys the GMRES-DR identity A V_k = V_k+1 Hbar_k
    and V_k+1 is orthonormal (to 1e-5 / 1e-6: single-pass modified Gram-Schmidt, as in
    Q/inverters.f90:3099-3155, loses orthogonality as the residual falls to 1e-12).
    The k harmonic Ritz values it reports are the generalized eigenvalues of
    (Hbar_k^H Hbar_k, H_k^H) (1e-8), and the smallest-magnitude eigenvalue of the dense
    matrix is within 1% of one of them."""
    ol, links, dims, kappa, A = dense44
    b = random_half(ol.ntotal, ol.nvhalf, 81)
    d = ol.deflation(20, 6)
    x, st, log = ol.gmresdr(b, ol.new_half(), (20, 6), 1e-12, kappa=kappa, defl=d)
    assert st == 0
    xs = np.linalg.solve(A, half_to_vec(b, ol.nvhalf))
    assert rel(half_to_vec(x, ol.nvhalf), xs) < 1e-9
    hist, _ = log.history()
    assert hist[-1] < 1e-12 and log.ncycles == len(hist)
    vt, hbar = ol.defl_get(d, 6, 20)
    V = np.stack([half_to_vec(v, ol.nvhalf) for v in vt], axis=1)
    assert np.abs(V.conj().T @ V - np.eye(7)).max() < 1e-6
    assert rel(V @ hbar, A @ V[:, :6]) < 1e-5
    theta = np.linalg.eigvals(np.linalg.solve(hbar[:6].conj().T, hbar.conj().T @ hbar))
    ritz = log.ritz_values()
    for t in theta:
        assert np.min(np.abs(ritz[:6] - t)) < 1e-8 * abs(t)
    ev = np.linalg.eigvals(A)
    lam = ev[np.argmin(np.abs(ev))]
    assert np.min(np.abs(ritz - lam)) < 0.01 * abs(lam)


def test_bicgstab_and_gmresproj_solutions(dense44):
    ol, links, dims, kappa, A = dense44
    b = random_half(ol.ntotal, ol.nvhalf, 82)
    xs = np.linalg.solve(A, half_to_vec(b, ol.nvhalf))
    x, st, log = ol.bicgstab(b, ol.new_half(), 1e-12, kappa=kappa)
    assert rel(half_to_vec(x, ol.nvhalf), xs) < 1e-9
    d = ol.deflation(20, 6)
    b1 = random_half(ol.ntotal, ol.nvhalf, 83)
    ol.psc(b1, ol.new_half(), (20, 6), 1e-12, kappa=kappa, isignal=1, defl=d)
    x, st, log = ol.gmresproject(b, (14, 6), 1e-12, kappa=kappa, isignal=2, defl=d)
    assert rel(half_to_vec(x, ol.nvhalf), xs) < 1e-9


@pytest.mark.parametrize("inverter", [0, 5, 6])
@pytest.mark.parametrize("kappa", [(0.124, 0.0), (0.124, 0.05)])
def test_fermprop_full_lattice(inverter, kappa):
    """fermprop (source preparation, even solve, odd reconstruction) against a dense
    solve of M = (1 + 2 i kappa mu gamma5) - kappa H on the whole 4^4 lattice.  psc
    (inverter 6) stops at the reference's fixed 1e-8 for later right-hand sides, so
    it runs here as the first right-hand side (isignal 1, GMRES-DR)."""
    dims = (4, 4, 4, 4)
    ol = oracle.OracleLattice(*dims, bc=BC)
    links, u = golden_gauge(dims, ol.ntotal, seed=9, eps=0.5)
    ol.set_gauge(u)
    be = random_half(ol.ntotal, ol.nvhalf, 91)
    bo = random_half(ol.ntotal, ol.nvhalf, 92)
    d = ol.deflation(20, 6) if inverter == 6 else None
    xe, xo, st, log = ol.fermprop(be, bo, kappa, inverter=inverter, resmax=1e-12, nGMRES=(20, 6),
                                  isignal=1, defl=d)
    b = half_to_lex(be, dims, 1) + half_to_lex(bo, dims, 2)
    x = half_to_lex(xe, dims, 1) + half_to_lex(xo, dims, 2)
    assert rel(full_operator_apply(links, x, kappa), b) < 1e-9


# ---------------------------------------------------------------- pseudolapack
def test_linearsolver_matches_numpy():
    rng = np.random.default_rng(101)
    for n in (3, 10, 31):
        a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        b = rng.standard_normal((n, 2)) + 1j * rng.standard_normal((n, 2))
        assert rel(oracle.linearsolver(a, b), np.linalg.solve(a, b)) < 1e-12


def test_schur_selected_matches_numpy():
    """gmresdr's restart step: Schur form with the k smallest-|theta| eigenvalues
    leading (hessenberg, qgenerator, evalues, orgschur of Q/pseudolapack.f90)."""
    rng = np.random.default_rng(102)
    n, k = 24, 8
    h = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    T, Z, w, wc = oracle.schur_selected(h, k)
    assert np.abs(Z.conj().T @ Z - np.eye(n)).max() < 1e-12
    assert rel(Z @ T @ Z.conj().T, h) < 1e-12
    assert np.abs(np.tril(T, -1)).max() < 1e-10 * np.abs(h).max()
    ev = np.linalg.eigvals(h)
    want = np.sort_complex(ev[np.argsort(np.abs(ev))[:k]])
    got = np.sort_complex(np.diag(T)[:k])
    assert np.abs(got - want).max() < 1e-10 * np.abs(ev).max()


# ---------------------------------------------------------------- noise
def noise_by_rule(rn, nvhalf, z4):
    """Q/disconloops.f90:4518-4649 restated: draws in the order colour (outer), isite,
    spin, ieo, ibleo (inner); Z(4): rn > 0.75 -> 1, 0.5 < rn < 0.75 -> -1,
    0.25 < rn < 0.5 -> i, otherwise -i; Z(2): rn > 0.5 -> 1 else -1."""
    r = rn.reshape(3, nvhalf, 4, 2, 8)
    if z4:
        v = np.where(r > 0.75, 1.0 + 0j, np.where((r > 0.5) & (r < 0.75), -1.0 + 0j,
                     np.where((r > 0.25) & (r < 0.5), 1j, -1j)))
    else:
        v = np.where(r > 0.5, 1.0 + 0j, -1.0 + 0j)
    return np.transpose(v, (4, 3, 2, 1, 0))  # -> (ibleo, ieo, spin, isite, colour)


@pytest.mark.parametrize("z4", [True, False])
def test_noise_sources_follow_the_reference_rule(z4):
    dims = (4, 4, 4, 8)
    ol = oracle.OracleLattice(*dims, bc=BC)
    n = ol.nvhalf
    oracle.initlagfib(0, 13)
    be, bo = ol.z4source() if z4 else ol.z2source()
    oracle.initlagfib(0, 13)
    rn = oracle.rnds(2 * 192 * n)  # one draw per complex component, be then bo
    for half, part in ((be, rn[: 192 * n]), (bo, rn[192 * n:])):
        got = half[:, :, :, :n, 0::2] + 1j * half[:, :, :, :n, 1::2]
        assert np.array_equal(got, noise_by_rule(part, n, z4))
        assert not half[:, :, :, n:].any()
