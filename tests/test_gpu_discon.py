"""Batched disconnected loops (qq_discon_traces, through the C ABI) against the
oracle's restatement of the reference's noise loop (twistdiscon, Q/disconloops.f90
:3612-4170, at the unsubtracted level) and against the golden record of the
reference's own method (psc).  Tolerances relative to the largest entry: 1e-8 when
both sides solve to <= 1e-11 (FP64 GMRES-DR), 1e-7 for the batched FP32 BiCGStab
(solutions to 1e-10), 1e-5 for psc (GMRES-Proj stops at the fixed 1e-8)."""
import json
from pathlib import Path

import numpy as np
import pytest

import oracle
from qqtest import golden_gauge

pytestmark = pytest.mark.gpu

GOLDEN = json.loads((Path(__file__).resolve().parent / "golden" / "golden.json").read_text())
DIMS = tuple(GOLDEN["dims"])
BC = tuple(GOLDEN["bc"])


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


def oracle_loop(ol, kind, nnoise, kappa, delta=0.0, dobndry=0):
    Jsum = np.zeros((6, DIMS[3], 2))
    for _ in range(nnoise):
        be, bo = ol.z4source() if kind == 4 else ol.z2source()
        xe, xo, st, _ = ol.fermprop(be, bo, kappa, inverter=5, resmax=1e-12, nGMRES=(30, 10))
        assert st == 0
        Jsum += ol.twaverage_level0(be, bo, xe, xo, kappa[0], delta, dobndry)
    return Jsum / (nnoise * DIMS[0] * DIMS[1] * DIMS[2])


def close(got, want, rtol):
    return np.abs(got - want).max() <= rtol * np.abs(want).max()


@pytest.mark.parametrize("kind,solver,rtol", [(4, 0, 1e-8), (2, 0, 1e-8), (4, 1, 1e-7)])
def test_discon_vs_oracle_loop(pair, kind, solver, rtol):
    import baylorlqcd_b200 as qq

    lat, ol = pair
    kappa = (0.15, 0.0)
    oracle.initlagfib(0, 5)
    want = oracle_loop(ol, kind, 4, kappa)
    qq.initlagfib(0, 5)
    got, infos = lat.discon_traces(kind, 4, kappa, solver=solver, m=30, k=10, precision=32, rhs_block=3,
                                   tol=1e-11 if solver == 0 else 1e-10)
    assert all(i.status == 0 for i in infos)
    assert close(got, want, rtol)


def test_discon_twisted_mass_fixed_boundary(pair):
    import baylorlqcd_b200 as qq

    lat, ol = pair
    kappa = (0.15, 0.01)
    oracle.initlagfib(0, 6)
    want = oracle_loop(ol, 4, 2, kappa, delta=0.2, dobndry=1)
    qq.initlagfib(0, 6)
    got, _ = lat.discon_traces(4, 2, kappa, solver=0, m=30, k=10, tol=1e-11, delta=0.2, dobndry=1)
    assert close(got, want, 1e-8)


def test_discon_psc_golden(pair):
    """The reference's own method (psc) against the committed record."""
    import baylorlqcd_b200 as qq

    lat, _ = pair
    rec = GOLDEN["discon_z4_psc3"]
    qq.initlagfib(0, rec["iseed"])
    got, infos = lat.discon_traces(4, rec["nnoise"], (rec["kappa"], 0.0), solver=2, m=rec["GMRES"][0],
                                   k=rec["GMRES"][1], tol=rec["resmax"])
    assert infos[0].status == 0
    assert close(got, np.array(rec["J"]), 1e-5)


def test_discon_bad_arguments(pair):
    import baylorlqcd_b200 as qq

    lat, _ = pair
    for kw in (dict(noise_kind=3, nnoise=1), dict(noise_kind=4, nnoise=0)):
        with pytest.raises(qq.QQError) as e:
            lat.discon_traces(kw["noise_kind"], kw["nnoise"], (0.15, 0.0), solver=0)
        assert e.value.status == qq.QQ_BAD_ARG
