"""GPU parity of qq_pionrho (pionrho, Q/quark.f90:1033-1212) with the oracle's
restatement: random fields for every source spin, accumulation across calls, and the
12 columns of a point-source propagator.  FP64 sums of squares in a different order:
1e-12 relative."""
import numpy as np
import pytest

import oracle
from qqtest import random_half

pytestmark = pytest.mark.gpu

DIMS, BC = (8, 8, 8, 8), (1, 1, 1, -1)


@pytest.fixture(scope="module")
def pair():
    import baylorlqcd_b200 as qq

    lat = qq.Lattice(*DIMS, bc=BC)
    u, _ = lat.heatbath(6.0, 30, seed=4)
    ol = oracle.OracleLattice(*DIMS, bc=BC)
    ol.set_gauge(u)
    yield lat, ol
    lat.close()


@pytest.mark.parametrize("idsrc", [1, 2, 3, 4])
def test_pionrho_random(pair, idsrc):
    lat, ol = pair
    xe = random_half(ol.ntotal, ol.nvhalf, seed=idsrc)
    xo = random_half(ol.ntotal, ol.nvhalf, seed=20 + idsrc)
    got = lat.pionrho(xe, xo, idsrc)
    ref = ol.pionrho(xe, xo, idsrc)
    for g, r in zip(got, ref):
        assert np.abs(g - r).max() <= 1e-12 * np.abs(r).max()


def test_pionrho_propagator(pair):
    """Accumulated over the 12 spin-colour columns of a point-source propagator."""
    lat, ol = pair
    nt = DIMS[3]
    acc = [np.zeros(nt) for _ in range(3)]
    ref = [np.zeros(nt) for _ in range(3)]
    for ic in (1, 2, 3):
        for idd in (1, 2, 3, 4):
            be, bo = lat.pointsource((1, 1, 1, 1), ic, idd)
            xe, xo, info = lat.fermprop(be, bo, (0.150, 0.0), inverter=5, resmax=1e-11, nGMRES=(16, 6))
            assert info.status == 0
            lat.pionrho(xe, xo, idd, *acc)
            for a, b in zip(ref, ol.pionrho(xe, xo, idd)):
                a += b
    for g, r in zip(acc, ref):
        assert np.abs(g - r).max() <= 1e-12 * np.abs(r).max()
    assert np.all(acc[0] > 0)  # the pion correlator is positive


@pytest.mark.parametrize("recon", [18, 12])
def test_smear_matches_oracle(recon):
    """qq_smear (Q/diracops.f90:712-858) against the oracle: three sweeps, an antiperiodic
    spatial direction, both link storages; FP64 in another order, 1e-13."""
    import baylorlqcd_b200 as qq
    from qqtest import golden_gauge

    dims, bc = (4, 8, 4, 4), (1, -1, 1, -1)
    ol = oracle.OracleLattice(*dims, bc=bc)
    _, u = golden_gauge(dims, ol.ntotal, seed=12, eps=0.6)
    ol.set_gauge(u)
    lat = qq.Lattice(*dims, bc=bc)
    lat.gauge_upload(u, recon=recon)
    ge, go = random_half(ol.ntotal, ol.nvhalf, 31), random_half(ol.ntotal, ol.nvhalf, 32)
    he, ho = lat.smear(ge, go, 0.2, 3)
    he_o, ho_o = ol.smear(ge, go, 0.2, 3)
    nv = ol.nvhalf
    for a, b in ((he, he_o), (ho, ho_o)):
        assert np.abs(a[..., :nv, :] - b[..., :nv, :]).max() <= 1e-13 * np.abs(b).max()
    lat.close()


@pytest.mark.parametrize("channels", [0, 1])
def test_mesoncorr_matches_oracle(channels):
    """qq_mesoncorr (Q/quark.f90:1297-2137) against the oracle's loop-by-loop restatement:
    random propagator columns for q and qbar, an off-origin source, all 729 momenta; the
    reference's three channels or all 28.  FP64 in another order: 1e-11 of the largest."""
    import baylorlqcd_b200 as qq

    dims, src = (4, 4, 4, 8), (3, 1, 2, 5)
    ol = oracle.OracleLattice(*dims)
    lat = qq.Lattice(*dims)
    rng = np.random.default_rng(11)
    q = np.zeros((12, 2) + ol.half_shape)
    qb = np.zeros_like(q)
    q[..., :ol.nvhalf, :] = rng.standard_normal(q[..., :ol.nvhalf, :].shape)
    qb[..., :ol.nvhalf, :] = rng.standard_normal(qb[..., :ol.nvhalf, :].shape)
    re, im = lat.mesoncorr(q, src, qbar=qb, channels=channels)
    re_o, im_o = ol.mesoncorr(q, src, qbar=qb, channels=channels)
    scale = max(np.abs(re_o).max(), np.abs(im_o).max())
    assert np.abs(re - re_o).max() <= 1e-11 * scale and np.abs(im - im_o).max() <= 1e-11 * scale
    re1, _ = lat.mesoncorr(q, src, channels=0)
    re1_o, _ = ol.mesoncorr(q, src, channels=0)
    assert np.abs(re1 - re1_o).max() <= 1e-11 * np.abs(re1_o).max()
    lat.close()
