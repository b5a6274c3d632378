"""GPU parity of qq_twvev (twvev, Q/vevbleft.f90:757-2536) with the oracle's literal
restatement, through the C ABI.

The oracle is checked against an independent full-lattice expansion on CPU
(test_cpu_vev.py).  Here the GPU gather program must reproduce it on lattices where
the reference's shells wrap and meet (4^3 x 8, 8 x 4 x 4 x 4), on 8^4, with both link
storages, both Wilson r, twist, both time boundaries, nsub = 4 and 6 and the momentum
projections.  FP64 sums in another order: 1e-12 relative to the largest entry.
At 16^3 x 32, where the oracle is too slow, size-independent properties: a gauge
transformation leaves Jvev unchanged, and two runs are bitwise equal."""
import numpy as np
import pytest

import oracle
from qqtest import gauge_to_ref, random_gauge
from test_cpu_vev import gauge_transform

pytestmark = pytest.mark.gpu

CASES = [
    dict(kappa=0.14, delta=0.0, dobndry=0, ir=1, nsub=6, nmom=5, nop=6, io=(1, 1, 1)),
    dict(kappa=0.15, delta=0.3, dobndry=1, ir=-1, nsub=6, nmom=5, nop=6, io=(2, 1, 3)),
    dict(kappa=0.13, delta=-0.25, dobndry=0, ir=1, nsub=4, nmom=3, nop=7, io=(1, 4, 2)),
]


def _pair(dims, seed, recon):
    import baylorlqcd_b200 as qq

    ol = oracle.OracleLattice(*dims, bc=(1, 1, 1, 1))
    _, u = random_gauge(dims, ol.ntotal, seed=seed)
    ol.set_gauge(u)
    lat = qq.Lattice(*dims, bc=(1, 1, 1, 1))
    lat.gauge_upload(u, recon=recon)
    return lat, ol


@pytest.mark.parametrize("dims,recon", [((4, 4, 4, 8), 18), ((4, 4, 4, 8), 12), ((8, 4, 4, 4), 18)])
@pytest.mark.parametrize("case", range(len(CASES)))
def test_twvev_matches_oracle(dims, recon, case):
    lat, ol = _pair(dims, 31 + case, recon)
    kw = CASES[case]
    got = lat.twvev(**kw)
    ref = ol.twvev(**kw)
    lat.close()
    assert np.abs(ref).max() > 0
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


def test_twvev_8x4_matches_oracle():
    lat, ol = _pair((8, 8, 8, 8), 41, 12)
    kw = CASES[1]
    got = lat.twvev(**kw)
    ref = ol.twvev(**kw)
    lat.close()
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


def test_twvev_nsub0_is_zero():
    lat, _ = _pair((4, 4, 4, 8), 42, 18)
    J = lat.twvev(0.15, nsub=0)
    lat.close()
    assert np.all(J == 0)


def test_twvev_gauge_invariance_and_determinism_16x32():
    import baylorlqcd_b200 as qq

    dims = (16, 16, 16, 32)
    lat = qq.Lattice(*dims, bc=(1, 1, 1, 1))
    links, u = random_gauge(dims, lat.ntotal, seed=43)
    lat.gauge_upload(u, recon=18)
    kw = dict(kappa=0.156, delta=0.2, dobndry=0, ir=1, nsub=6)
    a = lat.twvev(**kw)
    b = lat.twvev(**kw)
    lat.gauge_upload(gauge_to_ref(gauge_transform(links, 7), dims, lat.ntotal), recon=18)
    c = lat.twvev(**kw)
    lat.close()
    assert np.array_equal(a, b)
    assert np.abs(a).max() > 0
    assert np.abs(a - c).max() <= 1e-11 * np.abs(a).max()
