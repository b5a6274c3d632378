"""GPU level-0 loop traces (qq_twaverage_level0, through the C ABI) against the
oracle's literal restatement of twAverage at nsub = 0 (Q/vevbleft.f90:2541-4704) and
against the committed golden fixture of the first Z(4) noise.  Tolerance: 1e-12 of
the largest entry on identical inputs (FP64, different summation order); 1e-7 where
the GPU also solved for the propagator (solves to 1e-12)."""
import json
from pathlib import Path

import numpy as np
import pytest

import oracle
from qqtest import golden_gauge, random_half

pytestmark = pytest.mark.gpu

BC = (1, 1, 1, -1)
GOLDEN = json.loads((Path(__file__).resolve().parent / "golden" / "golden.json").read_text())


@pytest.fixture(scope="module", params=[((4, 4, 4, 8), 18), ((8, 4, 4, 4), 12)], ids=["4x4x4x8-r18", "8x4x4x4-r12"])
def pair(request):
    import baylorlqcd_b200 as qq

    dims, recon = request.param
    ol = oracle.OracleLattice(*dims, bc=BC)
    _, u = golden_gauge(dims, ol.ntotal, seed=31, eps=0.6)
    ol.set_gauge(u)
    lat = qq.Lattice(*dims, bc=BC)
    lat.gauge_upload(u, recon=recon)
    yield ol, lat
    lat.close()


def close(got, want, rtol):
    return np.abs(got - want).max() <= rtol * np.abs(want).max()


@pytest.mark.parametrize("delta,dobndry", [(0.0, 0), (0.0, 1), (0.37, 0)])
def test_traces_match_oracle(pair, delta, dobndry):
    ol, lat = pair
    oracle.initlagfib(0, 13)
    be, bo = ol.z4source()
    xe = random_half(ol.ntotal, ol.nvhalf, 32)
    xo = random_half(ol.ntotal, ol.nvhalf, 33)
    want = ol.twaverage_level0(be, bo, xe, xo, 0.1565, delta, dobndry)
    got = lat.twaverage_level0(be, bo, xe, xo, 0.1565, delta, dobndry)
    assert close(got, want, 1e-12)


def test_traces_device_arrays(pair):
    """Noise and solution already in HBM (torch CUDA tensors) give the same traces."""
    import torch

    ol, lat = pair
    oracle.initlagfib(0, 14)
    be, bo = ol.z2source()
    xe = random_half(ol.ntotal, ol.nvhalf, 34)
    xo = random_half(ol.ntotal, ol.nvhalf, 35)
    want = ol.twaverage_level0(be, bo, xe, xo, 0.15)
    t = [torch.from_numpy(a).cuda() for a in (be, bo, xe, xo)]
    got = lat.twaverage_level0(*t, 0.15)
    assert close(got, want, 1e-12)


def test_traces_golden_noise1():
    """KAT-7: first Z(4) noise of the lagged-Fibonacci stream, solved and traced on the
    GPU, against the committed fixture."""
    import baylorlqcd_b200 as qq

    dims = tuple(GOLDEN["dims"])
    rec = GOLDEN["traces_z4_noise1"]
    lat = qq.Lattice(*dims, bc=tuple(GOLDEN["bc"]))
    try:
        _, u = golden_gauge(dims, lat.ntotal, GOLDEN["gauge_seed"], GOLDEN["gauge_eps"])
        lat.gauge_upload(u)
        qq.initlagfib(0, 13)
        ze, zo = lat.z4source()
        xe, xo, info = lat.fermprop(ze, zo, (rec["kappa"], 0.0), inverter=5, resmax=1e-12, nGMRES=(30, 10))
        assert info.status == 0
        got = lat.twaverage_level0(ze, zo, xe, xo, rec["kappa"], rec["delta"], rec["dobndry"])
        assert close(got, np.array(rec["J"]), 1e-7)
    finally:
        lat.close()


def test_traces_reject_bad_boundary_flag(pair):
    import baylorlqcd_b200 as qq

    ol, lat = pair
    z = np.zeros(lat.half_shape)
    with pytest.raises(qq.QQError) as e:
        lat.twaverage_level0(z, z, z, z, 0.15, 0.0, 2)
    assert e.value.status == qq.QQ_BAD_ARG
