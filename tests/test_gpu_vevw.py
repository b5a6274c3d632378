"""GPU parity of the Wilson loop driver's vacuum values and of one run of the driver
(qq_vev and qq_discon: vev and discon, Q/disconloops.f90:4653-5339 and 3445-3608)
with the oracle (oracle/vevw.cpp, checked against numpy in test_cpu_vevw.py, and the
oracle's noise loop), through the C ABI, on a heatbath configuration made by the oracle.

vev: Jvev to 1e-12 of its largest entry, plaq and psi to 1e-13, for recon-12 and
recon-18 links and two momentum origins.
discon: Jtotal = (Jvev on levels 2..nsub + the sum over the noises of average(nsub,
nmom, nop) with the momfacs factors about io) / nnoise / (nx ny nz); the oracle solves
each noise with its GMRES-DR to 1e-12 and applies its average restatement with the
reference's own nop = 5; 1e-8 of the largest entry when the GPU solves with FP64
GMRES-DR to 1e-11, 1e-7 with the batched FP32 BiCGStab to 1e-10."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

DIMS = (4, 4, 4, 8)
BC = (1, 1, 1, -1)


@pytest.fixture(scope="module")
def config():
    ol = oracle.OracleLattice(*DIMS, bc=BC)
    u = ol.coldstart()
    oracle.initlagfib(0, 17)
    ol.heatbath(u, 5.8, 15)
    ol.set_gauge(u)
    return ol, u


@pytest.mark.parametrize("recon", [12, 18])
@pytest.mark.parametrize("io", [(1, 1, 1), (3, 2, 4)])
def test_vev_matches_oracle(config, recon, io):
    import baylorlqcd_b200 as qq

    ol, u = config
    lat = qq.Lattice(*DIMS, bc=BC)
    try:
        lat.gauge_upload(u, recon=recon)
        kappa = 0.1565
        J, plaq, psi = lat.vev(kappa, io)
        Jo, plaq_o, psi_o = ol.vev(kappa, io)
        assert np.abs(J - Jo).max() <= 1e-12 * np.abs(Jo).max()
        assert abs(plaq - plaq_o) <= 1e-13 and abs(psi - psi_o) <= 1e-13 * abs(psi_o)
        assert abs(plaq - ol.aveplaq(u)) <= 1e-13
    finally:
        lat.close()


def oracle_discon(ol, noise_kind, nnoise, kappa, nsub, nmom, nop, io):
    nt = DIMS[3]
    Jv, _, _ = ol.vev(kappa, io)
    mf = ol.momfacs(io) if nmom > 1 else None
    J = np.zeros((nop, nmom, nsub, nt, 2))
    n5 = min(nop, 5)
    for isub in range(1, nsub):
        J[:n5, :, isub] = Jv[:n5, :nmom]
    for _ in range(nnoise):
        be, bo = ol.z4source() if noise_kind == 4 else ol.z2source()
        xe, xo, st, _ = ol.fermprop(be, bo, (kappa, 0.0), inverter=5, resmax=1e-12, nGMRES=(30, 10))
        assert st == 0
        J += ol.average(be, bo, xe, xo, kappa, nsub=nsub, nmom=nmom, nop=nop, momfac=mf)
    return J / nnoise / (DIMS[0] * DIMS[1] * DIMS[2])


@pytest.mark.parametrize("noise_kind,nsub,nmom,nop,io,solver,rtol", [(2, 6, 5, 5, (1, 1, 1), 0, 1e-8),
                                                                     (4, 4, 1, 9, (2, 3, 1), 0, 1e-8),
                                                                     (2, 6, 5, 5, (1, 1, 1), 1, 1e-7)])
def test_discon_matches_oracle(config, noise_kind, nsub, nmom, nop, io, solver, rtol):
    import baylorlqcd_b200 as qq

    ol, u = config
    lat = qq.Lattice(*DIMS, bc=BC)
    try:
        lat.gauge_upload(u)
        kappa, nnoise = 0.15, 3
        oracle.initlagfib(0, 9)
        want = oracle_discon(ol, noise_kind, nnoise, kappa, nsub, nmom, nop, io)
        qq.initlagfib(0, 9)
        got, jv, infos = lat.discon(noise_kind, nnoise, kappa, nsub=nsub, nmom=nmom, nop=nop, io=io, solver=solver,
                                    m=30, k=10, tol=1e-11 if solver == 0 else 1e-10, rhs_block=3)
        assert all(i.status == 0 for i in infos)
        assert got.shape == want.shape
        assert np.abs(got - want).max() <= rtol * np.abs(want).max()
        jv_o, _, _ = ol.vev(kappa, io)
        assert np.abs(jv - jv_o).max() <= 1e-12 * np.abs(jv_o).max()
    finally:
        lat.close()


def test_discon_bad_arguments(config):
    import baylorlqcd_b200 as qq

    ol, u = config
    lat = qq.Lattice(*DIMS, bc=BC)
    try:
        lat.gauge_upload(u)
        for kw in ({"nop": 10}, {"nsub": 7}, {"nmom": 6}):
            with pytest.raises(qq.QQError):
                lat.discon(2, 1, 0.15, **kw)
        with pytest.raises(qq.QQError):
            lat.discon(3, 1, 0.15)
        with pytest.raises(qq.QQError):
            lat.discon(2, 0, 0.15)
    finally:
        lat.close()
