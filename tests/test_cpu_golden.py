"""The oracle against the committed golden fixtures (tests/golden/golden.json,
written by tests/golden/make_golden.py).  Random streams and noise codes must match
bit for bit; solver histories, Ritz values and checksums to 1e-10 relative (the oracle
is compiled for baseline x86-64 without FMA contraction, so it reproduces across x86
hosts up to the last bits of libm)."""
import json
from pathlib import Path

import numpy as np
import pytest

import oracle
from qqtest import golden_gauge

GOLDEN = json.loads((Path(__file__).resolve().parent / "golden" / "golden.json").read_text())
DIMS = tuple(GOLDEN["dims"])
BC = tuple(GOLDEN["bc"])
RTOL = 1e-10


@pytest.fixture(scope="module")
def ol():
    o = oracle.OracleLattice(*DIMS, bc=BC)
    _, u = golden_gauge(DIMS, o.ntotal, GOLDEN["gauge_seed"], GOLDEN["gauge_eps"])
    o.set_gauge(u)
    return o


def sources(ol):
    return {"be": ol.pointsource((1, 1, 1, 1), 1, 1), "be2": ol.pointsource((2, 3, 1, 4), 2, 3)}


def codes(half, nvhalf):
    m = {1: "a", -1: "b", 1j: "c", -1j: "d"}
    c = (half[:, :, :, :nvhalf, 0::2] + 1j * half[:, :, :, :nvhalf, 1::2]).ravel()
    return "".join(m[complex(v)] for v in c)


@pytest.mark.parametrize("key", sorted(GOLDEN["lagfib"]))
def test_lagfib_stream(key):
    myid, iseed = (int(v) for v in key.split(","))
    oracle.initlagfib(myid, iseed)
    assert oracle.rnds(32).tolist() == GOLDEN["lagfib"][key]


@pytest.mark.parametrize("kind", ["z4", "z2"])
def test_noise_codes(ol, kind):
    oracle.initlagfib(0, 13)
    be, bo = ol.z4source() if kind == "z4" else ol.z2source()
    assert codes(be, ol.nvhalf) == GOLDEN["noise"][kind]["be"]
    assert codes(bo, ol.nvhalf) == GOLDEN["noise"][kind]["bo"]


def test_plaquette(ol):
    assert abs(ol.aveplaq() - GOLDEN["plaquette"]) < 1e-14


def check_record(rec, x, st, log, b, ol):
    assert st == rec["status"]
    assert log.itercount == rec["itercount"] and log.ncycles == rec["ncycles"]
    hist, _ = log.history()
    np.testing.assert_allclose(hist, rec["hist"], rtol=RTOL, atol=1e-22)
    r = np.array(rec["ritz"]).reshape(-1, 2)
    np.testing.assert_allclose(log.ritz_values(), r[:, 0] + 1j * r[:, 1], rtol=RTOL)
    np.testing.assert_allclose(ol.vecdot(x, x).real, rec["x_norm2"], rtol=RTOL)
    bx = ol.vecdot(b, x)
    np.testing.assert_allclose([bx.real, bx.imag], rec["b_dot_x"], rtol=RTOL)


@pytest.mark.parametrize("name", ["gmresdr_wilson", "gmresdr_tm"])
def test_gmresdr(ol, name):
    rec = GOLDEN["solves"][name]
    b = sources(ol)[rec["src"]][0]
    x, st, log = ol.gmresdr(b, ol.new_half(), tuple(rec["GMRES"]), rec["resmax"], kappa=tuple(rec["kappa"]))
    check_record(rec, x, st, log, b, ol)


def test_bicgstab(ol):
    rec = GOLDEN["solves"]["bicgstab_wilson"]
    b = sources(ol)["be"][0]
    x, st, log = ol.bicgstab(b, ol.new_half(), rec["resmax"], kappa=tuple(rec["kappa"]))
    check_record(rec, x, st, log, b, ol)


def test_psc_second_rhs(ol):
    rec = GOLDEN["solves"]["psc_second_rhs"]
    src = sources(ol)
    k = tuple(rec["kappa"])
    d = ol.deflation(20, 6)
    ol.psc(src["be"][0], ol.new_half(), (20, 6), 1e-10, kappa=k, isignal=1, defl=d)
    x, st, log = ol.psc(src["be2"][0], ol.new_half(), (20, 6), 1e-10, kappa=k, isignal=2, defl=d)
    check_record(rec, x, st, log, src["be2"][0], ol)


def test_fermprop(ol):
    rec = GOLDEN["solves"]["fermprop_wilson"]
    be, bo = sources(ol)["be"]
    xe, xo, st, log = ol.fermprop(be, bo, tuple(rec["kappa"]), inverter=5, resmax=1e-10,
                                  nGMRES=tuple(rec["nGMRES"]))
    assert log.itercount == rec["itercount"]
    np.testing.assert_allclose(ol.vecdot(xe, xe).real, rec["xe_norm2"], rtol=RTOL)
    np.testing.assert_allclose(ol.vecdot(xo, xo).real, rec["xo_norm2"], rtol=RTOL)


def test_traces_z4_noise1(ol):
    rec = GOLDEN["traces_z4_noise1"]
    oracle.initlagfib(0, 13)
    ze, zo = ol.z4source()
    xe, xo, st, log = ol.fermprop(ze, zo, (rec["kappa"], 0.0), inverter=5, resmax=1e-12, nGMRES=(30, 10))
    assert log.itercount == rec["itercount"]
    J = ol.twaverage_level0(ze, zo, xe, xo, rec["kappa"], rec["delta"], rec["dobndry"])
    want = np.array(rec["J"])
    assert np.abs(J - want).max() <= RTOL * np.abs(want).max()


def test_discon_psc3(ol):
    """The reference's noise loop (twistdiscon): 3 Z(4) noises, psc, level-0 traces."""
    rec = GOLDEN["discon_z4_psc3"]
    oracle.initlagfib(0, rec["iseed"])
    d = ol.deflation(*rec["GMRES"])
    Jsum = np.zeros((6, DIMS[3], 2))
    for i in range(rec["nnoise"]):
        ze, zo = ol.z4source()
        xe, xo, st, log = ol.fermprop(ze, zo, (rec["kappa"], 0.0), inverter=6, resmax=rec["resmax"],
                                      nGMRES=tuple(rec["GMRES"]), isignal=1 if i == 0 else 2, defl=d)
        Jsum += ol.twaverage_level0(ze, zo, xe, xo, rec["kappa"], 0.0, 0)
    J = Jsum / (rec["nnoise"] * DIMS[0] * DIMS[1] * DIMS[2])
    want = np.array(rec["J"])
    assert np.abs(J - want).max() <= RTOL * np.abs(want).max()


def test_kat6_c1_reproduces_record():
    """KAT-6 at configuration C1: the oracle's heatbath (8^4, beta = 6.0, cold start,
    lagfib seed (0, 13), 200 sweeps) and its fermprop with GMRES-DR(30,10) to 1e-10 at
    kappa = 0.150 reproduce the committed record: plaquette, cycles, the gmresdr-norm
    history, the harmonic Ritz values and the solution norms."""
    rec = GOLDEN["kat6_c1"]
    c1 = oracle.OracleLattice(*rec["dims"], bc=BC)
    u = c1.coldstart()
    oracle.initlagfib(0, rec["iseed"])
    plaq = c1.heatbath(u, rec["beta"], rec["sweeps"])
    assert plaq[-1] == rec["plaquette"]
    c1.set_gauge(u)
    be, bo = c1.pointsource((1, 1, 1, 1), 1, 1)
    xe, xo, st, log = c1.fermprop(be, bo, tuple(rec["kappa"]), inverter=5, resmax=rec["resmax"],
                                  nGMRES=tuple(rec["nGMRES"]))
    assert st == rec["status"] == 0
    assert log.itercount == rec["itercount"] and log.ncycles == rec["ncycles"]
    hist, _ = log.history()
    np.testing.assert_allclose(hist, rec["hist"], rtol=RTOL, atol=1e-22)
    r = np.array(rec["ritz"]).reshape(-1, 2)
    np.testing.assert_allclose(log.ritz_values(), r[:, 0] + 1j * r[:, 1], rtol=RTOL)
    np.testing.assert_allclose(c1.vecdot(xe, xe).real, rec["xe_norm2"], rtol=RTOL)
    np.testing.assert_allclose(c1.vecdot(xo, xo).real, rec["xo_norm2"], rtol=RTOL)
