"""qq_twaverage (twAverage, Q/vevbleft.f90:2541-4704, with momenta) and qq_twistdiscon
(twistdiscon, Q/disconloops.f90:3612-4351, at subtraction levels) through the C ABI,
against the oracle.

qq_twaverage: random noise and solution, every level layout (nsub 0, 4, 6), five
momenta about a moved origin, twist and fixed time boundary: 1e-12 relative.
qq_twistdiscon: the expected Jtotal (and each noise's Jtemp) is assembled here as the
reference does --
numnoises * Jvev (twvev, kappa on operators other than 2 and 6, level 6 += level 4)
plus every noise's kappa-scaled twAverage, over numnoises and nx*ny*nz -- from the
oracle's noise stream, solves (FP64 GMRES-DR to 1e-12), twAverage and twvev.  Both
sides solve to <= 1e-11: 1e-8 relative to the largest entry."""
import json
from pathlib import Path

import numpy as np
import pytest

import oracle
from qqtest import golden_gauge, random_half

pytestmark = pytest.mark.gpu

GOLDEN = json.loads((Path(__file__).resolve().parent / "golden" / "golden.json").read_text())
DIMS = tuple(GOLDEN["dims"])
BC = tuple(GOLDEN["bc"])
LEVELS = {0: [0], 4: [0, 3], 6: [0, 3, 5]}


@pytest.fixture(scope="module")
def pair():
    import baylorlqcd_b200 as qq

    lat = qq.Lattice(*DIMS, bc=BC)
    ol = oracle.OracleLattice(*DIMS, bc=BC)
    _, u = golden_gauge(DIMS, lat.ntotal, GOLDEN["gauge_seed"], GOLDEN["gauge_eps"])
    lat.gauge_upload(u)
    ol.set_gauge(u)
    yield lat, ol
    lat.close()


@pytest.mark.parametrize("nsub,ir", [(0, 1), (4, 1), (6, 1), (6, -1)])
def test_twaverage_matches_oracle(pair, nsub, ir):
    lat, ol = pair
    oracle.initlagfib(0, 9)
    be, bo = ol.z4source()
    xe, xo = random_half(ol.ntotal, ol.nvhalf, 61), random_half(ol.ntotal, ol.nvhalf, 62)
    kw = dict(delta=0.3, io=(2, 1, 3), dobndry=1, ir=ir)
    got = lat.twaverage(be, bo, xe, xo, 0.15, nsub=nsub, nmom=5, nop=7, **kw)
    T = ol.twaverage(be, bo, xe, xo, 1.0, nmom=5, **kw)  # (6, nmom, nt, 2), unscaled
    want = np.zeros_like(got)
    for lv in LEVELS[nsub]:
        want[:6, :, lv] = T
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
    assert np.all(got[6:] == 0)


def expected_twistdiscon(ol, kind, nnoise, kappa, nsub, nmom, nop, io, delta, dobndry, ir=1):
    jv = ol.twvev(kappa[0], delta=delta, io=io, dobndry=dobndry, ir=ir, nsub=nsub, nmom=nmom, nop=nop)
    for iop in range(nop):
        if iop not in (1, 5):
            jv[iop] = kappa[0] * jv[iop]
    if nsub == 6:
        jv[:, :, 5] = jv[:, :, 3] + jv[:, :, 5]
    jt = nnoise * jv
    per = []
    for _ in range(nnoise):
        be, bo = ol.z4source() if kind == 4 else ol.z2source()
        xe, xo, st, _ = ol.fermprop(be, bo, kappa, inverter=5, resmax=1e-12, nGMRES=(30, 10))
        assert st == 0
        T = ol.twaverage(be, bo, xe, xo, kappa[0], delta=delta, io=io, dobndry=dobndry, nmom=nmom, ir=ir)
        one = jv.copy()
        for lv in LEVELS.get(nsub, []):
            jt[:6, :, lv] = jt[:6, :, lv] + T
            one[:6, :, lv] = one[:6, :, lv] + T
        per.append(one / (DIMS[0] * DIMS[1] * DIMS[2]))  # Jtemp, written out times 1/(nx ny nz)
    jt = jt / nnoise
    return jt / (DIMS[0] * DIMS[1] * DIMS[2]), np.array(per)


@pytest.mark.parametrize("kappa,delta,dobndry,nsub,ir", [((0.15, 0.0), 0.0, 0, 6, 1), ((0.15, 0.01), 0.2, 1, 4, 1),
                                                          ((0.15, 0.01), 0.2, 0, 6, -1)])
def test_twistdiscon_matches_oracle(pair, kappa, delta, dobndry, nsub, ir):
    import baylorlqcd_b200 as qq

    lat, ol = pair
    io = (1, 2, 1)
    oracle.initlagfib(0, 5)
    want, want_per = expected_twistdiscon(ol, 4, 2, kappa, nsub, 5, 6, io, delta, dobndry, ir)
    qq.initlagfib(0, 5)
    got, infos, per = lat.twistdiscon(4, 2, kappa, nsub=nsub, nmom=5, nop=6, io=io, delta=delta, dobndry=dobndry,
                                      ir=ir, solver=0, m=30, k=10, tol=1e-11, per_noise=True)
    assert all(i.status == 0 for i in infos)
    assert np.abs(got - want).max() <= 1e-8 * np.abs(want).max()
    assert np.abs(per - want_per).max() <= 1e-8 * np.abs(want_per).max()
    assert np.abs(per.mean(axis=0) - got).max() <= 1e-13 * np.abs(got).max()
    # the perturbative part is there: level 4 differs from level 1 by Jvev
    assert np.abs(got[:, :, 3] - got[:, :, 0]).max() > 1e-6 * np.abs(got).max()
