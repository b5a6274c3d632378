"""GPU tests of the batched mixed-precision propagator solver (qq_fermprop_batch)
against the CPU oracle's FP64 fermprop (Q/quark.f90:458-842 with GMRES-DR).

Every solution must reach the requested FP64 full-lattice residual and agree with the
oracle's FP64 solution within the accuracy that residual implies (1e-7 relative for
tol = 1e-10 on these well-conditioned small systems)."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

DIMS = (8, 8, 8, 8)
BC = (1, 1, 1, -1)


@pytest.fixture(scope="module")
def setup():
    import baylorlqcd_b200 as qq

    lat = qq.Lattice(*DIMS, bc=BC)
    u, plaq = lat.heatbath(6.0, 50, seed=21)
    ol = oracle.OracleLattice(*DIMS, bc=BC)
    ol.set_gauge(u)
    yield lat, ol, u
    lat.close()


def sources(lat, n):
    be = np.zeros((n,) + lat.half_shape)
    bo = np.zeros((n,) + lat.half_shape)
    for i in range(n):
        be[i], bo[i] = lat.pointsource((1 + i % 2, 1, 2, 1 + i // 2), i % 3 + 1, i % 4 + 1)
    return be, bo


def interior_rel(a, b, nv):
    return np.linalg.norm((a - b)[:, :, :, :nv]) / np.linalg.norm(b[:, :, :, :nv])


@pytest.mark.parametrize("solver,precision,deflate", [(0, 64, 0), (1, 64, 0), (1, 32, 0), (1, 32, 1),
                                                      (1, 16, 1)])
@pytest.mark.parametrize("kappa", [(0.150, 0.0), (0.150, 0.01)])
def test_batch_vs_oracle(setup, solver, precision, deflate, kappa):
    lat, ol, u = setup
    be, bo = sources(lat, 5)
    xe, xo, infos = lat.fermprop_batch(be, bo, kappa, m=16, k=6, precision=precision, rhs_block=4,
                                       tol=1e-10, solver=solver, deflate=deflate)
    for i in range(5):
        assert infos[i].status == 0, (i, infos[i])
        assert infos[i].true_rel <= 1e-10
        if precision == 16 and deflate:
            # FP16 against a deflation space can stall on 8^4 (the projection at every
            # reliable update); the FP32 batched iteration then finishes, never GMRES-DR
            assert infos[i].finished_by in (0, 32), (i, infos[i].fallback, infos[i].finished_by)
        else:
            assert infos[i].fallback == 0 and infos[i].finished_by == 0, (i, infos[i].fallback)
        xe_o, xo_o, st, _ = ol.fermprop(be[i], bo[i], kappa, inverter=5, resmax=1e-12, nGMRES=(16, 6))
        assert st == 0
        assert interior_rel(xe[i], xe_o, ol.nvhalf) < 1e-7
        assert interior_rel(xo[i], xo_o, ol.nvhalf) < 1e-7


@pytest.mark.parametrize("precision", [16, -16])
def test_point_source_breakdowns_restart(setup, precision):
    """A point source makes the textbook shadow residual r0 one spin-colour component at
    one site, so every <rhat, .> is a single component, which 16-bit storage against the
    site's norm rounds to exactly zero within a few iterations.  Each such breakdown
    restarts the right-hand side with its re-inserted FP64 residual as the shadow
    residual: FP16 takes at least one restart.  A 16-bit iteration may still stall on a
    right-hand side -- whether it does depends on the hop shapes the autotuner times
    fastest, which set the rounding -- and is then finished by the batched FP32
    iteration, never by GMRES-DR."""
    lat, ol, u = setup
    be, bo = sources(lat, 4)
    xe, xo, infos = lat.fermprop_batch(be, bo, (0.150, 0.01), m=16, k=6, precision=precision, rhs_block=4,
                                       tol=1e-10, solver=1, deflate=0)
    for i in infos:
        assert i.status == 0 and i.true_rel <= 1e-10
        assert i.finished_by in (0, 32), (i.fallback, i.finished_by, i.restarts)
    if precision == 16:
        assert max(i.restarts for i in infos) >= 1, [i.restarts for i in infos]
    xe_o, xo_o, st, _ = ol.fermprop(be[0], bo[0], (0.150, 0.01), inverter=5, resmax=1e-12, nGMRES=(16, 6))
    assert interior_rel(xe[0], xe_o, ol.nvhalf) < 1e-7


@pytest.mark.parametrize("precision", [32, 16, -16])
def test_graph_and_host_loops_agree(setup, monkeypatch, precision):
    """The graph-driven loop (one CUDA graph with conditional nodes) and the host-driven
    loop run the same per-RHS recurrences with fixed-order reductions: a right-hand side
    that waits for its reliable update does not change its own sequence.  Same iteration
    counts, update histories and solutions.  (No deflation space: with one, both modes
    run the host-synchronised deflated loop.)"""
    lat, ol, u = setup
    be, bo = sources(lat, 6)
    kappa = (0.150, 0.01)
    res = {}
    for mode in ("0", "1"):
        monkeypatch.setenv("QQ_HOST_LOOP", mode)
        res[mode] = lat.fermprop_batch(be, bo, kappa, m=16, k=6, precision=precision, rhs_block=6,
                                       tol=1e-10, solver=1, deflate=0)
    (xg, og, ig), (xh, oh, ih) = res["0"], res["1"]
    for i in range(6):
        assert ig[i].status == 0 and ih[i].status == 0
        assert ig[i].fallback == ih[i].fallback and ig[i].finished_by == ih[i].finished_by
        if precision == 32:
            assert ig[i].fallback == 0
        else:  # a 16-bit iteration may stall (400-iteration window); the FP32 one finishes it
            assert ig[i].finished_by in (0, 32)
        assert ig[i].itercount == ih[i].itercount and ig[i].mvp == ih[i].mvp
        assert len(ig[i].hist) == len(ih[i].hist) > 0
        assert np.array_equal(ig[i].hist, ih[i].hist)
    assert interior_rel(xg, xh, ol.nvhalf) < 1e-14
    assert interior_rel(og, oh, ol.nvhalf) < 1e-14


def test_batch_device_arrays(setup):
    """Inputs and outputs already in HBM (torch CUDA tensors): same answers."""
    import torch

    lat, ol, u = setup
    be, bo = sources(lat, 3)
    xe_h, xo_h, _ = lat.fermprop_batch(be, bo, (0.15, 0.0), m=16, k=6, precision=32, rhs_block=2)
    bed, bod = torch.from_numpy(be).cuda(), torch.from_numpy(bo).cuda()
    xed, xod = torch.zeros_like(bed), torch.zeros_like(bod)
    lat.fermprop_batch(bed, bod, (0.15, 0.0), m=16, k=6, precision=32, rhs_block=2, xe=xed, xo=xod)
    torch.cuda.synchronize()
    assert interior_rel(xed.cpu().numpy(), xe_h, ol.nvhalf) < 1e-9
    assert interior_rel(xod.cpu().numpy(), xo_h, ol.nvhalf) < 1e-9


def test_heatbath_matches_oracle_ensemble():
    """KAT-5 against the GPU heatbath: the oracle's restatement of the reference's
    pseudo-heatbath gives, on 8^4 at beta = 6.0 from a cold start, a plaquette that
    averages 0.5943 over sweeps 101..200 (committed record).  The GPU heatbath draws from
    another generator, so only the ensembles can agree: the mean final plaquette of 8
    GPU streams after 200 sweeps must lie within 4 standard errors (GPU spread over the
    streams and the record's spread over its sweeps) of the record's mean."""
    import json
    from pathlib import Path

    import baylorlqcd_b200 as qq

    rec = json.loads((Path(__file__).resolve().parent / "golden" / "golden.json").read_text())["kat5_heatbath"]
    ref = np.array(rec["plaquette"][100:])
    lat = qq.Lattice(8, 8, 8, 8)
    got = np.array([lat.heatbath(6.0, 200, seed=100 + s)[1] for s in range(8)])
    lat.close()
    err = np.sqrt(got.var(ddof=1) / len(got) + ref.var(ddof=1) / 10)  # the record's sweeps are correlated
    assert abs(got.mean() - ref.mean()) < 4 * err, (got.mean(), ref.mean(), err)


def test_heatbath_plaquette(setup):
    """The GPU heatbath thermalises to the known beta = 6.0 plaquette (about 0.594)."""
    import baylorlqcd_b200 as qq

    lat = qq.Lattice(8, 8, 8, 8)
    u, plaq = lat.heatbath(6.0, 200, seed=1)
    ol = oracle.OracleLattice(8, 8, 8, 8)
    assert abs(ol.aveplaq(u) - plaq) < 1e-12       # GPU plaquette = oracle plaquette of u
    assert 0.585 < plaq < 0.600
    lat.close()


@pytest.mark.parametrize("shape,precision,deflate", [(1, 32, 0), (202, 32, 0), (203, 32, 0), (204, 32, 0),
                                                      (1, 16, 0), (202, 16, 0), (203, 16, 0), (204, 16, 0),
                                                      (301, 32, 0), (302, 32, 0), (303, 32, 0), (301, 32, 1),
                                                      (304, 32, 0), (304, 32, 1), (305, 32, 0),
                                                      (306, 32, 0), (307, 32, 0), (307, 32, 1), (308, 32, 0),
                                                      (309, 32, 0), (310, 32, 1), (311, 32, 0),
                                                      (1, -16, 0), (202, -16, 0), (204, -16, 0)])
def test_block_kernel_shapes(setup, monkeypatch, shape, precision, deflate):
    """Each hopping-kernel shape, forced for the whole solve where the launch supports
    it: one RHS per thread; 2, 3 or 4 RHS per thread sharing links and neighbour
    indices; the packed FP32x2 kernel with 1-3 RHS per thread (with deflate = 1 also on
    the single-RHS FP32 launches of the mixed-precision GMRES-DR).  Same converged
    answers as the oracle."""
    import baylorlqcd_b200 as qq

    _, ol, u = setup
    monkeypatch.setenv("QQ_FORCE_TPS", str(shape))
    lat = qq.Lattice(*DIMS, bc=BC)
    try:
        lat.gauge_upload(u)
        be, bo = sources(lat, 12)
        kappa = (0.150, 0.01)
        xe, xo, infos = lat.fermprop_batch(be, bo, kappa, m=16, k=6, precision=precision, rhs_block=12,
                                           tol=1e-10, solver=1, deflate=deflate)
        for i in range(12):
            assert infos[i].status == 0 and infos[i].true_rel <= 1e-10, (i, infos[i])
            if precision in (16, -16):  # 16 bits may stall; the FP32 iteration then finishes
                assert infos[i].finished_by in (0, 32), (i, infos[i].fallback, infos[i].finished_by)
            else:
                assert infos[i].fallback == 0, (i, infos[i].fallback)
        for i in (0, 7, 11):
            xe_o, xo_o, st, _ = ol.fermprop(be[i], bo[i], kappa, inverter=5, resmax=1e-12, nGMRES=(16, 6))
            assert interior_rel(xe[i], xe_o, ol.nvhalf) < 1e-7
            assert interior_rel(xo[i], xo_o, ol.nvhalf) < 1e-7
    finally:
        lat.close()
