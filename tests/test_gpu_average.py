"""GPU parity of qq_average (average / loopops / spacesum, Q/disconloops.f90:5343-5733,
7769-7910, 9012-9124) with the oracle's restatement, through the C ABI: random complex
noise and solution, six subtraction levels, momenta with random momentum factors,
antiperiodic time, both link storages.  The oracle is checked against an independent
numpy statement in test_cpu_average.py.  FP64 in another order: 1e-11 relative to the
largest entry."""
import numpy as np
import pytest

import oracle
from qqtest import golden_gauge, random_half

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dims,recon", [((4, 4, 4, 8), 18), ((4, 4, 4, 8), 12), ((8, 4, 4, 8), 18)])
def test_average_matches_oracle(dims, recon):
    import baylorlqcd_b200 as qq

    bc = (1, 1, 1, -1)
    ol = oracle.OracleLattice(*dims, bc=bc)
    _, u = golden_gauge(dims, ol.ntotal, seed=38, eps=0.6)
    ol.set_gauge(u)
    lat = qq.Lattice(*dims, bc=bc)
    lat.gauge_upload(u, recon=recon)
    be, bo = random_half(ol.ntotal, ol.nvhalf, 81), random_half(ol.ntotal, ol.nvhalf, 82)
    xe, xo = random_half(ol.ntotal, ol.nvhalf, 83), random_half(ol.ntotal, ol.nvhalf, 84)
    nsub, nmom, nop, kappa = 6, 4, 10, 0.152
    momfac = np.random.default_rng(85).standard_normal((5, nmom - 1, 16, 2, ol.nvhalf))
    got = lat.average(be, bo, xe, xo, kappa, nsub=nsub, nmom=nmom, nop=nop, momfac=momfac)
    want = ol.average(be, bo, xe, xo, kappa, nsub=nsub, nmom=nmom, nop=nop, momfac=momfac)
    lat.close()
    assert np.abs(want).max() > 0
    assert np.abs(got - want).max() <= 1e-11 * np.abs(want).max()
