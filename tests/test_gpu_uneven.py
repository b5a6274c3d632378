"""GPU tests of the uneven batch (qq_fermprop_uneven): propagator solves on two lattices
of different size, each with its own heatbath gauge field, at two kappa values and a
twisted mass, point and Z(4) sources mixed, in one call.

Every solution must reach the FP64 full-lattice residual 1e-10 and agree with the CPU
oracle's FP64 fermprop (Q/quark.f90:458-842 with GMRES-DR) to 1e-7 relative, as the
single-lattice batch tests require; the concurrent schedule (one host thread and stream
per lattice) must give the solutions of the sequential one."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

BC = (1, 1, 1, -1)


@pytest.fixture(scope="module")
def lattices():
    import baylorlqcd_b200 as qq

    out = []
    for dims, seed in (((8, 8, 8, 8), 21), ((4, 4, 4, 8), 5)):
        lat = qq.Lattice(*dims, bc=BC)
        u, _ = lat.heatbath(6.0, 50, seed=seed)
        ol = oracle.OracleLattice(*dims, bc=BC)
        ol.set_gauge(u)
        out.append((lat, ol))
    yield out
    for lat, _ in out:
        lat.close()


def mixed_sources(qq, lat, npoint, nz4):
    n = npoint + nz4
    be = np.zeros((n,) + lat.half_shape)
    bo = np.zeros((n,) + lat.half_shape)
    for i in range(npoint):
        be[i], bo[i] = lat.pointsource((1 + i % 2, 1, 1 + i // 2, 1), i % 3 + 1, i % 4 + 1)
    for i in range(npoint, n):
        be[i], bo[i] = lat.z4source()
    return be, bo


def interior_rel(a, b, nv):
    return np.linalg.norm((a - b)[:, :, :, :nv]) / np.linalg.norm(b[:, :, :, :nv])


def make_groups(qq, lattices):
    qq.initlagfib(0, 9)
    spec = [(0, 2, 1, (0.150, 0.0)), (1, 1, 2, (0.150, 0.0)), (0, 1, 1, (0.150, 0.01)), (1, 2, 0, (0.145, 0.0))]
    groups = []
    for li, npoint, nz4, kappa in spec:
        lat = lattices[li][0]
        be, bo = mixed_sources(qq, lat, npoint, nz4)
        groups.append((lat, be, bo, kappa))
    return spec, groups


def test_uneven_matches_oracle_and_sequential(lattices):
    import baylorlqcd_b200 as qq

    spec, groups = make_groups(qq, lattices)
    conc, secs_c = qq.fermprop_uneven(groups, m=16, k=6, precision=32, rhs_block=4, tol=1e-10, concurrent=True)
    seq, secs_s = qq.fermprop_uneven(groups, m=16, k=6, precision=32, rhs_block=4, tol=1e-10, concurrent=False)
    assert secs_c > 0.0 and secs_s > 0.0
    for g, ((li, _, _, kappa), (lat, be, bo, _)) in enumerate(zip(spec, groups)):
        ol = lattices[li][1]
        xe, xo, infos = conc[g]
        xe_s, xo_s, _ = seq[g]
        for i in range(be.shape[0]):
            assert infos[i].status == 0, (g, i, infos[i])
            assert infos[i].true_rel <= 1e-10
            xe_o, xo_o, st, _ = ol.fermprop(be[i], bo[i], kappa, inverter=5, resmax=1e-12, nGMRES=(16, 6))
            assert st == 0
            assert interior_rel(xe[i], xe_o, ol.nvhalf) < 1e-7, (g, i)
            assert interior_rel(xo[i], xo_o, ol.nvhalf) < 1e-7, (g, i)
            assert interior_rel(xe_s[i], xe[i], ol.nvhalf) < 1e-12, (g, i)
            assert interior_rel(xo_s[i], xo[i], ol.nvhalf) < 1e-12, (g, i)


def test_uneven_rejects_bad_group(lattices):
    import baylorlqcd_b200 as qq

    (lat, _), _ = lattices
    be = np.zeros((0,) + lat.half_shape)
    with pytest.raises(qq.QQError):
        qq.fermprop_uneven([(lat, be, be, (0.150, 0.0))])


@pytest.mark.parametrize("precision", [32, 16])
def test_stall_forces_gmresdr_fallback(lattices, precision):
    """The fallback path, triggered on purpose: with a stall window of one iteration no
    right-hand side can show the required 10x fall of its FP64 true residual, so the
    batched BiCGStab stops every one of them after its first iteration (fallback = 3,
    stagnation) -- in FP16 first, then in the FP32 iteration that continues a stopped
    16-bit one -- and plain FP64 GMRES-DR(m, k) finishes it from the BiCGStab's solution.
    Every answer must still reach the FP64 full-lattice residual and agree with the
    oracle's FP64 solve (Q/quark.f90:458-842 with GMRES-DR, Q/inverters.f90:2871-3572)."""
    import baylorlqcd_b200 as qq

    lat, ol = lattices[0]
    qq.initlagfib(0, 9)
    be, bo = mixed_sources(qq, lat, 2, 2)
    kappa = (0.1565, 0.005)
    xe, xo, infos = lat.fermprop_batch(be, bo, kappa, m=16, k=6, precision=precision, rhs_block=4, tol=1e-10,
                                       solver=1, deflate=0, stall_window=1)
    for i in range(be.shape[0]):
        assert infos[i].status == 0, (i, infos[i])
        assert infos[i].fallback == 3 and infos[i].finished_by == 64, (i, infos[i].fallback, infos[i].finished_by)
        assert infos[i].true_rel <= 1e-10
        xe_o, xo_o, st, _ = ol.fermprop(be[i], bo[i], kappa, inverter=5, resmax=1e-12, nGMRES=(16, 6))
        assert st == 0
        assert interior_rel(xe[i], xe_o, ol.nvhalf) < 1e-7, i
        assert interior_rel(xo[i], xo_o, ol.nvhalf) < 1e-7, i


def test_near_critical_default_rules(lattices):
    """Twisted mass at kappa = 0.1565, mu = 0.005 on the 8^4 heatbath configuration,
    where the FP32 batched BiCGStab has broken down (NaN) or stalled on Z(4) sources,
    with the default stall window and iteration limit: whichever way each right-hand
    side ends (converged, or any fallback reason), it must reach the FP64 residual and
    agree with the oracle's FP64 solve, and nothing may run to an unbounded count."""
    import baylorlqcd_b200 as qq

    lat, ol = lattices[0]
    qq.initlagfib(0, 9)
    be, bo = mixed_sources(qq, lat, 1, 1)
    kappa = (0.1565, 0.005)
    xe, xo, infos = lat.fermprop_batch(be, bo, kappa, m=16, k=6, precision=32, rhs_block=4, tol=1e-10,
                                       solver=1, deflate=0)
    for i in range(2):
        assert infos[i].status == 0, (i, infos[i])
        assert infos[i].true_rel <= 1e-10
        assert infos[i].fallback in (0, 1, 2, 3, 4)
        xe_o, xo_o, st, _ = ol.fermprop(be[i], bo[i], kappa, inverter=5, resmax=1e-12, nGMRES=(16, 6))
        assert st == 0
        assert interior_rel(xe[i], xe_o, ol.nvhalf) < 1e-7, i
        assert interior_rel(xo[i], xo_o, ol.nvhalf) < 1e-7, i
