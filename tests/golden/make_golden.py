#!/usr/bin/env python
"""Writes tests/golden/golden.json: reference outputs of the oracle (the CPU
restatement of the qqcd hot path in oracle/) on small, seeded, machine-independent
inputs.  The reference ships no golden vectors and its Fortran cannot be built here,
so these pin the oracle against itself over time and give the GPU parity tests
fixed numbers to meet.  Inputs:

* lagged-Fibonacci draws (G/lagfib.f90) for three (myid, iseed) pairs;
* Z(4) / Z(2) noise sources (Q/disconloops.f90:4518-4649) on 4x4x4x8, as code strings;
* GMRES-DR(30,10) (Wilson) and GMRES-DR(20,6) (twisted mass), BiCGStab and
  GMRES-Proj after a deflating first solve (psc), and fermprop with odd
  reconstruction, all on 4x4x4x8 with the Gram-Schmidt gauge field of
  qqtest.golden_gauge(seed 2026, eps 0.25; plaquette 0.52) and point sources;
* level-0 loop traces (Q/vevbleft.f90 twAverage, nsub = 0) of the first Z(4) noise
  after a fermprop solve, and the noise average of three Z(4) noises solved with psc
  as the reference's twistdiscon loop does.
* KAT-5: the oracle's restatement of the reference's pseudo-heatbath (G/heatbath.f90,
  C/cfgsprops.f90 sweep) on 8x8x8x8 at beta = 6.0 from a cold start with lagfib seed
  (0, 7): the plaquette after every sweep of 200 (a reproducible oracle number, not
  a literature value).
* KAT-6 at configuration C1: the same heatbath on 8^4 from a cold start with lagfib seed
  (0, 13), 200 sweeps, then fermprop with GMRES-DR(30,10) to 1e-10 at kappa = 0.150 on
  the point source at site (1,1,1,1): cycle count, the gmresdr-norm history and the
  harmonic Ritz values of the last restart.

Usage: python tests/golden/make_golden.py   (rewrites golden.json)
"""
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))
sys.path.insert(0, str(HERE.parent.parent))

import oracle  # noqa: E402
from qqtest import golden_gauge  # noqa: E402

DIMS = (4, 4, 4, 8)
BC = (1, 1, 1, -1)
GAUGE_SEED, GAUGE_EPS = 2026, 0.25
Z4_CODES = {1: "a", -1: "b", 1j: "c", -1j: "d"}  # +1, -1, +i, -i


def noise_codes(half, nvhalf):
    c = (half[:, :, :, :nvhalf, 0::2] + 1j * half[:, :, :, :nvhalf, 1::2]).ravel()
    return "".join(Z4_CODES[complex(v)] for v in c)


def solve_record(x, st, log, b, ol):
    hist, hmvp = log.history()
    return {"status": int(st), "itercount": int(log.itercount), "ncycles": int(log.ncycles),
            "mvp": int(log.mvp), "hist": [float(h) for h in hist], "hist_mvp": [int(m) for m in hmvp],
            "ritz": [[float(r.real), float(r.imag)] for r in log.ritz_values()],
            "x_norm2": float(ol.vecdot(x, x).real),
            "b_dot_x": [float(ol.vecdot(b, x).real), float(ol.vecdot(b, x).imag)]}


def main():
    out = {"dims": DIMS, "bc": BC, "gauge_seed": GAUGE_SEED, "gauge_eps": GAUGE_EPS}
    out["lagfib"] = {}
    for myid, iseed in [(0, 13), (1, 13), (0, 1)]:
        oracle.initlagfib(myid, iseed)
        out["lagfib"][f"{myid},{iseed}"] = [float(v) for v in oracle.rnds(32)]

    ol = oracle.OracleLattice(*DIMS, bc=BC)
    out["noise"] = {}
    for name, fn in (("z4", ol.z4source), ("z2", ol.z2source)):
        oracle.initlagfib(0, 13)
        be, bo = fn()
        out["noise"][name] = {"be": noise_codes(be, ol.nvhalf), "bo": noise_codes(bo, ol.nvhalf)}

    _, u = golden_gauge(DIMS, ol.ntotal, GAUGE_SEED, GAUGE_EPS)
    ol.set_gauge(u)
    out["plaquette"] = float(ol.aveplaq())
    be, bo = ol.pointsource((1, 1, 1, 1), 1, 1)
    be2, bo2 = ol.pointsource((2, 3, 1, 4), 2, 3)
    solves = {}
    x, st, log = ol.gmresdr(be, ol.new_half(), (30, 10), 1e-10, kappa=(0.15, 0.0))
    solves["gmresdr_wilson"] = dict(kappa=[0.15, 0.0], GMRES=[30, 10], resmax=1e-10, src="be",
                                    **solve_record(x, st, log, be, ol))
    x, st, log = ol.gmresdr(be2, ol.new_half(), (20, 6), 1e-10, kappa=(0.155, 0.01))
    solves["gmresdr_tm"] = dict(kappa=[0.155, 0.01], GMRES=[20, 6], resmax=1e-10, src="be2",
                                **solve_record(x, st, log, be2, ol))
    x, st, log = ol.bicgstab(be, ol.new_half(), 1e-10, kappa=(0.15, 0.0))
    solves["bicgstab_wilson"] = dict(kappa=[0.15, 0.0], resmax=1e-10, src="be",
                                     **solve_record(x, st, log, be, ol))
    d = ol.deflation(20, 6)
    ol.psc(be, ol.new_half(), (20, 6), 1e-10, kappa=(0.15, 0.0), isignal=1, defl=d)
    x, st, log = ol.psc(be2, ol.new_half(), (20, 6), 1e-10, kappa=(0.15, 0.0), isignal=2, defl=d)
    solves["psc_second_rhs"] = dict(kappa=[0.15, 0.0], GMRES=[20, 6], src="be2",
                                    **solve_record(x, st, log, be2, ol))
    xe, xo, st, log = ol.fermprop(be, bo, (0.15, 0.0), inverter=5, resmax=1e-10, nGMRES=(30, 10))
    solves["fermprop_wilson"] = dict(kappa=[0.15, 0.0], nGMRES=[30, 10], inverter=5, src="point 1,1,1,1 c1 s1",
                                     xe_norm2=float(ol.vecdot(xe, xe).real),
                                     xo_norm2=float(ol.vecdot(xo, xo).real),
                                     itercount=int(log.itercount))
    out["solves"] = solves

    # level-0 loop traces of the first Z(4) noise (twAverage, nsub = 0)
    oracle.initlagfib(0, 13)
    ze, zo = ol.z4source()
    xe, xo, st, log = ol.fermprop(ze, zo, (0.15, 0.0), inverter=5, resmax=1e-12, nGMRES=(30, 10))
    J = ol.twaverage_level0(ze, zo, xe, xo, 0.15, 0.0, 0)
    out["traces_z4_noise1"] = {"kappa": 0.15, "delta": 0.0, "dobndry": 0, "solve": "fermprop GMRES-DR(30,10) 1e-12",
                               "itercount": int(log.itercount), "J": J.tolist()}
    # the reference's disconnected-loop method: 3 Z(4) noises through psc (GMRES-DR on
    # the first, GMRES-Proj on the rest), level-0 traces averaged as twistdiscon does
    oracle.initlagfib(0, 21)
    d = ol.deflation(30, 10)
    Jsum = np.zeros((6, DIMS[3], 2))
    for i in range(3):
        ze, zo = ol.z4source()
        xe, xo, st, log = ol.fermprop(ze, zo, (0.15, 0.0), inverter=6, resmax=1e-10, nGMRES=(30, 10),
                                      isignal=1 if i == 0 else 2, defl=d)
        Jsum += ol.twaverage_level0(ze, zo, xe, xo, 0.15, 0.0, 0)
    J = Jsum / (3 * DIMS[0] * DIMS[1] * DIMS[2])
    out["discon_z4_psc3"] = {"kappa": 0.15, "nnoise": 3, "iseed": 21, "GMRES": [30, 10], "resmax": 1e-10,
                             "J": J.tolist()}
    # KAT-5: the oracle heatbath, 8^4 at beta = 6.0, cold start, 200 sweeps
    hb = oracle.OracleLattice(8, 8, 8, 8, bc=BC)
    u = hb.coldstart()
    oracle.initlagfib(0, 7)
    plaq = hb.heatbath(u, 6.0, 200)
    out["kat5_heatbath"] = {"dims": [8, 8, 8, 8], "beta": 6.0, "iseed": 7, "start": "cold",
                            "plaquette": [float(v) for v in plaq]}
    # KAT-6 at configuration C1: the same heatbath with lagfib seed (0, 13), then the
    # reference's fermprop (Q/quark.f90:458-842) with GMRES-DR(30,10) to 1e-10 at
    # kappa = 0.150 on the point source at site (1,1,1,1), colour 1, spin 1
    c1 = oracle.OracleLattice(8, 8, 8, 8, bc=BC)
    u = c1.coldstart()
    oracle.initlagfib(0, 13)
    plaq = c1.heatbath(u, 6.0, 200)
    c1.set_gauge(u)
    be, bo = c1.pointsource((1, 1, 1, 1), 1, 1)
    xe, xo, st, log = c1.fermprop(be, bo, (0.150, 0.0), inverter=5, resmax=1e-10, nGMRES=(30, 10))
    hist, hmvp = log.history()
    out["kat6_c1"] = {"dims": [8, 8, 8, 8], "beta": 6.0, "iseed": 13, "sweeps": 200, "start": "cold",
                      "plaquette": float(plaq[-1]), "kappa": [0.150, 0.0], "nGMRES": [30, 10], "resmax": 1e-10,
                      "src": "point 1,1,1,1 c1 s1", "status": int(st), "itercount": int(log.itercount),
                      "ncycles": int(log.ncycles), "mvp": int(log.mvp), "hist": [float(h) for h in hist],
                      "hist_mvp": [int(m) for m in hmvp],
                      "ritz": [[float(r.real), float(r.imag)] for r in log.ritz_values()],
                      "xe_norm2": float(c1.vecdot(xe, xe).real), "xo_norm2": float(c1.vecdot(xo, xo).real)}
    (HERE / "golden.json").write_text(json.dumps(out, indent=1) + "\n")
    print("wrote", HERE / "golden.json")


if __name__ == "__main__":
    main()
