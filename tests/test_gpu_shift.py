"""GPU parity of the multi-shift solver through the C ABI: qq_gamma5mult
(Q/diracops.f90:1750-1860) and qq_gmresdrshift (Q/inverters.f90:6041-7179) against
the oracle's restatement.

The GPU Arnoldi uses CGS2 where the restatement uses modified Gram-Schmidt, and its
collinear shifted systems are solved by LU with partial pivoting on either side, so the
two agree to rounding: the tests require the same number of cycles (+-1), the base
residual history within 10% per cycle, every shift's solution equal to 1e-7 relative,
and each reported residual equal to the true residual b - (A - sigma_s) x_s computed
by the oracle's operator."""
import numpy as np
import pytest

import oracle
from qqtest import random_gauge, random_half

pytestmark = pytest.mark.gpu

DIMS = (4, 4, 4, 8)
BC = (1, 1, 1, -1)
NV = DIMS[0] * DIMS[1] * DIMS[2] * DIMS[3] // 32


@pytest.fixture(scope="module")
def pair():
    import baylorlqcd_b200 as qq

    ol = oracle.OracleLattice(*DIMS, bc=BC)
    _, u = random_gauge(DIMS, ol.ntotal, seed=3, eps=0.6)
    ol.set_gauge(u)
    lat = qq.Lattice(*DIMS, bc=BC)
    lat.gauge_upload(u, recon=18)
    yield ol, lat
    lat.close()


def interior(a):
    return a[:, :, :, :NV, :]


def relnorm(a, b):
    return np.linalg.norm(interior(a) - interior(b)) / np.linalg.norm(interior(b))


@pytest.mark.parametrize("kappa", [(0.18, 0.03), (0.15, -0.2), (0.124, 1.0)])
@pytest.mark.parametrize("idag", [0, 1])
def test_gamma5mult_matches_oracle(pair, kappa, idag):
    ol, lat = pair
    g = random_half(ol.ntotal, ol.nvhalf, 21)
    want = ol.gamma5mult(g, idag, kappa)
    got = lat.gamma5mult(g, idag, kappa)
    assert relnorm(got, want) < 1e-13


@pytest.mark.parametrize(
    "kappa,sig_over_k2,GMRES",
    [((0.18, 0.03), (0.0, -0.3, 0.5), (24, 8)), ((0.16, 0.2), (0.4, 0.0, -0.5, 0.8), (16, 6))],
    ids=["3shifts", "base-shifted-4shifts"],
)
def test_gmresdrshift_matches_oracle(pair, kappa, sig_over_k2, GMRES):
    ol, lat = pair
    sig = np.array(sig_over_k2) / kappa[0] ** 2
    b = random_half(ol.ntotal, ol.nvhalf, 9)
    xo, st, ro, log = ol.gmresdrshift(b, sig, GMRES, 1e-10, kappa=kappa)
    assert st == 0
    x, resid, info = lat.gmresdrshift(b, sig, GMRES, 1e-10, kappa=kappa)
    assert info.status == 0
    hist_o, _ = log.history()
    assert abs(len(info.hist) - len(hist_o)) <= 1
    n = min(len(info.hist), len(hist_o)) - 1
    np.testing.assert_allclose(info.hist[:n], hist_o[:n], rtol=0.1)
    assert resid[0] < 1e-10
    bn = np.linalg.norm(interior(b))
    for s in range(len(sig)):
        assert relnorm(x[s], xo[s]) < 1e-7
        r = b - ol.gamma5mult(x[s], 0, kappa) + sig[s] * x[s]
        true = np.linalg.norm(interior(r))
        assert abs(true - resid[s]) < 1e-12 * bn
        assert true < 1e-8 * bn


def test_gmresdrshift_argument_checks(pair):
    import baylorlqcd_b200 as qq

    ol, lat = pair
    b = random_half(ol.ntotal, ol.nvhalf, 9)
    with pytest.raises(qq.QQError):
        lat.gmresdrshift(b, np.array([0.0]), (12, 4), 1e-10, kappa=(0.18, 0.0))
    with pytest.raises(qq.QQError):
        lat.gmresdrshift(b, np.array([0.0]), (12, 4), 1e-10, kappa=(0.18, 0.03), iflag=-2)
    with pytest.raises(qq.QQError):
        lat.gmresdrshift(b, np.array([]), (12, 4), 1e-10, kappa=(0.18, 0.03))
    with pytest.raises(qq.QQError):
        lat.gmresdrshift(b, np.array([0.0]), (4, 4), 1e-10, kappa=(0.18, 0.03))
    with pytest.raises(qq.QQError):
        lat.gamma5mult(b, 0, (0.18, 0.0))


def test_gmresdrshift_heatbath_recon12_physical_mass():
    """8^4 heatbath configuration (recon-12 links on the device), the twisted mass of the
    noise-trace workload (kappa 0.1566, mu 0.005) and the shifts of the reference's
    commented variants: every shift's solution equal to the oracle's to 1e-7."""
    import baylorlqcd_b200 as qq

    dims = (8, 8, 8, 8)
    nv = dims[0] * dims[1] * dims[2] * dims[3] // 32
    lat = qq.Lattice(*dims, bc=BC)
    try:
        u, _ = lat.heatbath(6.0, 20, seed=11)
        ol = oracle.OracleLattice(*dims, bc=BC)
        ol.set_gauge(u)
        kappa = (0.1566, 0.005)
        sig = np.array([0.0, -0.099, -0.199, -0.3, -0.5]) / kappa[0] ** 2
        b = random_half(ol.ntotal, ol.nvhalf, 31)
        xo, st, ro, log = ol.gmresdrshift(b, sig, (40, 12), 1e-10, kappa=kappa)
        assert st == 0
        x, resid, info = lat.gmresdrshift(b, sig, (40, 12), 1e-10, kappa=kappa)
        assert info.status == 0
        assert abs(info.ncycles - log.ncycles) <= 1
        for s in range(len(sig)):
            d = x[s][:, :, :, :nv, :] - xo[s][:, :, :, :nv, :]
            assert np.linalg.norm(d) / np.linalg.norm(xo[s][:, :, :, :nv, :]) < 1e-7
        assert resid[0] < 1e-10 and np.all(resid < 1e-9) and np.all(ro < 1e-9)
    finally:
        lat.close()
