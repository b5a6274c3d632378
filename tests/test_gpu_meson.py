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
