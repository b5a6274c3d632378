"""GPU parity of the Dirac operator family (Q/diracops.f90) against the CPU oracle,
through the C ABI.  Floating-point tolerance: 1e-13 relative (FP64; the GPU uses spin
projection and a different summation order than the reference's loops)."""
import numpy as np
import pytest

import oracle
from qqtest import random_gauge, random_half

pytestmark = pytest.mark.gpu

TOL = 1e-13


@pytest.fixture(scope="module", params=[(4, 4, 4, 8), (8, 8, 8, 4)], ids=["4x4x4x8", "8x8x8x4"])
def pair(request):
    import baylorlqcd_b200 as qq

    dims = request.param
    bc = (1, 1, 1, -1)
    ol = oracle.OracleLattice(*dims, bc=bc)
    _, u = random_gauge(dims, ol.ntotal, seed=11)
    ol.set_gauge(u)
    lat = qq.Lattice(*dims, bc=bc)
    lat.gauge_upload(u, recon=18)
    yield ol, lat, u
    lat.close()


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("idag", [0, 1])
@pytest.mark.parametrize("gblclr", [1, 2])
def test_hsingle(pair, idag, gblclr):
    ol, lat, u = pair
    g = random_half(ol.ntotal, ol.nvhalf, 100 + idag + 2 * gblclr)
    ref = ol.hsingle(g, idag, gblclr)
    out = lat.hsingle(g, idag, gblclr)
    assert rel(out, ref) < TOL
    # halo slots of the output are zero, as after the reference's `gout = 0`
    assert np.all(out[:, :, :, ol.nvhalf:, :] == 0.0)


@pytest.mark.parametrize("recon", [12, 18])
def test_hsingle_recon(pair, recon):
    ol, lat, u = pair
    lat.gauge_upload(u, recon=recon)
    g = random_half(ol.ntotal, ol.nvhalf, 7)
    assert rel(lat.hsingle(g, 0, 1), ol.hsingle(g, 0, 1)) < 1e-12
    lat.gauge_upload(u, recon=18)


def test_hsingle_anisotropic(pair):
    ol, lat, u = pair
    c1, c2 = (1.0, 0.9, 1.1, 0.7), (0.8, 1.0, 0.6, 1.3)
    ol.set_coact(c1, c2)
    lat.set_coact(c1, c2)
    try:
        for idag in (0, 1):
            g = random_half(ol.ntotal, ol.nvhalf, 8 + idag)
            assert rel(lat.hsingle(g, idag, 2), ol.hsingle(g, idag, 2)) < TOL
    finally:
        ol.set_coact((1.0,) * 4, (1.0,) * 4)
        lat.set_coact((1.0,) * 4, (1.0,) * 4)


def test_wilson_r_minus_one(pair):
    """fermpropR's r = -1 flips coact(3,1,:) (Q/quark.f90:921-926)."""
    ol, lat, u = pair
    ol.set_coact((-1.0,) * 4, (1.0,) * 4)
    lat.set_coact((-1.0,) * 4, (1.0,) * 4)
    try:
        g = random_half(ol.ntotal, ol.nvhalf, 21)
        assert rel(lat.hsingle(g, 0, 1), ol.hsingle(g, 0, 1)) < TOL
    finally:
        ol.set_coact((1.0,) * 4, (1.0,) * 4)
        lat.set_coact((1.0,) * 4, (1.0,) * 4)


@pytest.mark.parametrize("idag", [0, 1])
def test_hdouble(pair, idag):
    ol, lat, u = pair
    g = random_half(ol.ntotal, ol.nvhalf, 31)
    assert rel(lat.hdouble(g, idag, 0.1565), ol.hdouble(g, idag, 0.1565)) < TOL


@pytest.mark.parametrize("kappa", [(0.1566, 0.005), (0.15, 0.0), (0.15, 1e-9), (0.13, -0.2)])
@pytest.mark.parametrize("idag", [0, 1])
def test_hdbletm(pair, kappa, idag):
    ol, lat, u = pair
    g = random_half(ol.ntotal, ol.nvhalf, 41)
    assert rel(lat.hdbletm(g, idag, kappa), ol.hdbletm(g, idag, kappa)) < TOL


def test_twmshift(pair):
    ol, lat, u = pair
    gw = np.stack([random_half(ol.ntotal, ol.nvhalf, 51), random_half(ol.ntotal, ol.nvhalf, 52)])
    k = (0.1566, 0.005)
    ref = ol.twmshift(gw, 0, k)
    out = lat.twmshift(gw, 0, k)
    assert rel(out, ref) < TOL


def test_vecdot(pair):
    ol, lat, u = pair
    a = random_half(ol.ntotal, ol.nvhalf, 61)
    b = random_half(ol.ntotal, ol.nvhalf, 62)
    ref = ol.vecdot(a, b)
    out = lat.vecdot(a, b)
    assert abs(out - ref) / abs(ref) < 1e-13


def test_device_pointers(pair):
    """Reference-layout arrays already in HBM (torch CUDA tensors) are used in place."""
    import torch

    ol, lat, u = pair
    g = random_half(ol.ntotal, ol.nvhalf, 71)
    gd = torch.from_numpy(g).cuda()
    od = torch.zeros_like(gd)
    lat.hsingle(gd, 0, 1, out=od)
    torch.cuda.synchronize()
    assert rel(od.cpu().numpy(), ol.hsingle(g, 0, 1)) < TOL


def test_bad_arguments(pair):
    import baylorlqcd_b200 as qq

    ol, lat, u = pair
    g = random_half(ol.ntotal, ol.nvhalf, 1)
    with pytest.raises(qq.QQError) as e:
        lat.hsingle(g, 0, 3)
    assert e.value.status == qq.QQ_BAD_ARG
    with pytest.raises(qq.QQError):
        lat.hsingle(g, 2, 1)
    with pytest.raises(qq.QQError):
        lat.hdbletm(g, 0, (0.15, 0.0), iflag=-2)  # clover branch is out of scope
