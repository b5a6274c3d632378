"""CPU checks of the oracle's twvev restatement (oracle/vev.cpp, Q/vevbleft.f90:757-2536).

1. Against an independent statement (vevref.py): the full-lattice hopping expansion
   (D R)^n of each unit source with the operators in closed form.  On an 8^4 lattice no
   two offsets of the reference's shells meet, so both must agree site by site; checked
   to 1e-12 relative for both Wilson r, twist angles, both time boundaries and a moved
   momentum origin, at sites on the first and last time slice.
2. Gauge invariance on a 4^3 x 8 lattice, where the shells wrap and meet: every operator
   is a sum of closed loops, so a random gauge transformation leaves Jvev unchanged
   (1e-12 relative).
3. The layout of Jvev: only levels 4 and 6 are filled, level 6 only for nsub = 6, and
   nothing for other nsub, as in the reference (:2233-2280)."""
import numpy as np
import pytest

import oracle
import vevref
from qqtest import gauge_to_ref, random_gauge, random_su3

AXIS = (3, 2, 1, 0)


def gauge_transform(links, seed):
    rng = np.random.default_rng(seed)
    shape = links.shape[1:5]
    g = random_su3(int(np.prod(shape)), rng).reshape(shape + (3, 3))
    out = np.empty_like(links)
    for mu in range(4):
        gs = np.roll(g, -1, axis=AXIS[mu])
        out[mu] = g @ links[mu] @ np.conj(np.swapaxes(gs, -1, -2))
    return out


@pytest.fixture(scope="module")
def lattice8():
    dims = (8, 8, 8, 8)
    ol = oracle.OracleLattice(*dims, bc=(1, 1, 1, 1))
    links, u = random_gauge(dims, ol.ntotal, seed=13)
    ol.set_gauge(u)
    return dims, ol, links


@pytest.mark.parametrize("opts", [
    dict(delta=0.0, dobndry=0, ir=1),
    dict(delta=0.35, dobndry=1, ir=1, io=(3, 1, 6)),
    dict(delta=-0.2, dobndry=0, ir=-1, io=(2, 5, 4)),
])
def test_oracle_matches_full_lattice_expansion(lattice8, opts):
    dims, ol, links = lattice8
    sites = [1, 8 * 8 * 8 * 7 + 8 * 3 + 6]  # (0,0,0,0) and (5,3,0,7), first and last slice
    io = opts.get("io", (1, 1, 1))
    got = ol.twvev_sites(sites, 0.152, delta=opts["delta"], io=io, dobndry=opts["dobndry"], ir=opts["ir"])
    ref = vevref.twvev_sites(links, dims, sites, 0.152, delta=opts["delta"], io=io, dobndry=opts["dobndry"],
                             r=opts["ir"])
    assert np.abs(ref).max() > 0
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("delta,dobndry,ir", [(0.0, 0, 1), (0.3, 1, -1)])
def test_oracle_gauge_invariance_small_lattice(delta, dobndry, ir):
    dims = (4, 4, 4, 8)
    ol = oracle.OracleLattice(*dims, bc=(1, 1, 1, 1))
    links, u = random_gauge(dims, ol.ntotal, seed=21)
    ol.set_gauge(u)
    a = ol.twvev(0.14, delta=delta, dobndry=dobndry, ir=ir, io=(2, 1, 3))
    ol.set_gauge(gauge_to_ref(gauge_transform(links, 5), dims, ol.ntotal))
    b = ol.twvev(0.14, delta=delta, dobndry=dobndry, ir=ir, io=(2, 1, 3))
    assert np.abs(a).max() > 0
    assert np.abs(a - b).max() <= 1e-12 * np.abs(a).max()


def test_oracle_jvev_levels():
    dims = (4, 4, 4, 8)
    ol = oracle.OracleLattice(*dims, bc=(1, 1, 1, 1))
    _, u = random_gauge(dims, ol.ntotal, seed=22)
    ol.set_gauge(u)
    j6 = ol.twvev(0.13, delta=0.1, nsub=6, nmom=3, nop=7)
    j4 = ol.twvev(0.13, delta=0.1, nsub=4, nmom=3, nop=7)
    j0 = ol.twvev(0.13, delta=0.1, nsub=0, nmom=3, nop=7)
    other = [0, 1, 2, 4]
    assert np.all(j6[:, :, other] == 0) and np.all(j6[6:] == 0)
    assert np.abs(j6[:6, :, 3]).max() > 0 and np.abs(j6[:6, :, 5]).max() > 0
    assert np.array_equal(j4[:, :, 3], j6[:, :, 3]) and np.all(j4[:, :, 5] == 0)
    assert np.all(j0 == 0)
