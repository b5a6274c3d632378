"""The multi-shift solver's oracle: gamma5mult (Q/diracops.f90:1750-1860) and
gmresdrshift (Q/inverters.f90:6041-7179) restated in oracle/, checked without the
reference (which never assigns its shifts).

gamma5mult is -i gamma5 Hdbletm / (2 kappa mu) in the reference's gamma basis, where
-i gamma5 takes the spins (v1, v2, v3, v4) to (-v3, -v4, v1, v2).  The shifted solver
is checked against numpy.linalg.solve of (A - sigma_s) x = b on the dense 4^4 operator
for every shift, and its recursively updated residuals against the true ones."""
import numpy as np
import pytest

import oracle
from qqtest import golden_gauge, half_to_vec, interior_basis, random_half

BC = (1, 1, 1, -1)
DIMS = (4, 4, 4, 4)


def minus_i_gamma5(h):
    out = np.empty_like(h)
    out[:, :, 0] = -h[:, :, 2]
    out[:, :, 1] = -h[:, :, 3]
    out[:, :, 2] = h[:, :, 0]
    out[:, :, 3] = h[:, :, 1]
    return out


@pytest.fixture(scope="module")
def lat44():
    ol = oracle.OracleLattice(*DIMS, bc=BC)
    _, u = golden_gauge(DIMS, ol.ntotal, seed=9, eps=0.5)
    ol.set_gauge(u)
    return ol


def dense(ol, kappa):
    n = 192 * ol.nvhalf
    basis = interior_basis(ol.nvhalf)
    A = np.zeros((n, n), complex)
    for j in range(n):
        e = np.zeros((8, 2, 4, ol.ntotal, 6))
        e[basis[0][j], basis[1][j], basis[2][j], basis[3][j], basis[4][j]] = 1.0
        A[:, j] = half_to_vec(ol.gamma5mult(e, 0, kappa), ol.nvhalf)
    return A


@pytest.mark.parametrize("kappa", [(0.124, 0.05), (0.15, -0.2)])
@pytest.mark.parametrize("idag", [0, 1])
def test_gamma5mult_is_rotated_hdbletm(lat44, kappa, idag):
    """gamma5mult = -i gamma5 Hdbletm / (2 kappa mu) for mu > 0.  For mu < 0 the
    reference's Hdbletm switches to the Wilson Hdouble (Q/diracops.f90:467), so the
    identity is checked there against the twisted form built from Hsingle."""
    ol = lat44
    g = random_half(ol.ntotal, ol.nvhalf, 5)
    got = half_to_vec(ol.gamma5mult(g, idag, kappa), ol.nvhalf)
    k, mu = kappa
    if mu > 0:
        want = minus_i_gamma5(ol.hdbletm(g, idag, kappa)) / (2 * k * mu)
    else:
        t = 2 * k * mu
        ho = ol.hsingle(g, idag, 2)
        tw = ho.copy()  # (1 - i t gamma5) in the reference's spin basis
        tw[:, :, 0] = ho[:, :, 0] - t * ho[:, :, 2]
        tw[:, :, 1] = ho[:, :, 1] - t * ho[:, :, 3]
        tw[:, :, 2] = ho[:, :, 2] + t * ho[:, :, 0]
        tw[:, :, 3] = ho[:, :, 3] + t * ho[:, :, 1]
        he = ol.hsingle(tw, idag, 1)
        g5g = g.copy()
        g5g[:, :, 0] = g[:, :, 0] + t * g[:, :, 2]
        g5g[:, :, 1] = g[:, :, 1] + t * g[:, :, 3]
        g5g[:, :, 2] = g[:, :, 2] - t * g[:, :, 0]
        g5g[:, :, 3] = g[:, :, 3] - t * g[:, :, 1]
        m = g5g / k**2 - he / (1 + t * t)
        want = minus_i_gamma5(m) / t
    want = half_to_vec(want, ol.nvhalf)
    assert np.linalg.norm(got - want) / np.linalg.norm(want) < 1e-14


@pytest.mark.parametrize(
    "kappa,sig_over_k2",
    [((0.124, 0.05), (0.0, -0.3, -0.5)), ((0.15, 0.2), (0.4, 0.0, -0.5, 0.8)), ((0.124, 0.5), (0.2,))],
    ids=["mu0.05-3shifts", "mu0.2-base-shifted-4shifts", "mu0.5-1shift"],
)
def test_gmresdrshift_solves_every_shift(lat44, kappa, sig_over_k2):
    ol = lat44
    sig = np.array(sig_over_k2) / kappa[0] ** 2
    b = random_half(ol.ntotal, ol.nvhalf, 81)
    x, st, resid, log = ol.gmresdrshift(b, sig, (20, 6), 1e-10, kappa=kappa)
    assert st == 0
    assert resid[0] < 1e-10
    A = dense(ol, kappa)
    bv = half_to_vec(b, ol.nvhalf)
    n = A.shape[0]
    for s in range(len(sig)):
        M = A - sig[s] * np.eye(n)
        xs = np.linalg.solve(M, bv)
        xv = half_to_vec(x[s], ol.nvhalf)
        true = np.linalg.norm(bv - M @ xv)
        assert abs(true - resid[s]) < 1e-12 * np.linalg.norm(bv)
        # the further shifts converge alongside the base (collinear residuals)
        assert true < 1e-8
        assert np.linalg.norm(xv - xs) / np.linalg.norm(xs) < 1e-8 * max(1.0, true / 1e-10)


def test_gmresdrshift_shift_matches_single_solve(lat44):
    """The solution of one further shift equals the base solution of a run whose only
    shift is that one (same Krylov problem, different route), to the solver tolerance."""
    ol = lat44
    kappa = (0.15, 0.2)
    k2 = 1 / kappa[0] ** 2
    b = random_half(ol.ntotal, ol.nvhalf, 17)
    x3, st3, _, _ = ol.gmresdrshift(b, np.array([0.0, 0.5]) * k2, (16, 4), 1e-11, kappa=kappa)
    x1, st1, _, _ = ol.gmresdrshift(b, np.array([0.5]) * k2, (16, 4), 1e-11, kappa=kappa)
    assert st3 == 0 and st1 == 0
    a, c = half_to_vec(x3[1], ol.nvhalf), half_to_vec(x1[0], ol.nvhalf)
    assert np.linalg.norm(a - c) / np.linalg.norm(c) < 1e-9


def test_gmresdrshift_zero_rhs(lat44):
    ol = lat44
    x, st, resid, log = ol.gmresdrshift(ol.new_half(), np.array([0.0, 1.0]), (8, 2), 1e-10, kappa=(0.124, 0.1))
    assert st == 0
    assert not x.any()
    assert not resid.any()
