#!/usr/bin/env python
"""Writes tests/golden/c5_gmresdr_record.json: the oracle's complete plain FP64
GMRES-DR(60,20) solve (Q/inverters.f90:2871-3572 through fermprop, Q/quark.f90:458-842)
at the benchmark configuration -- 24^3x48, twisted mass kappa = 0.1566, mu = 0.0025,
point source at site (1,1,1,1), colour 1, spin 1, even-system tolerance 2.5e-11 (the
full-lattice 1e-10 target) -- on the GPU heatbath configuration (beta = 6.0, cold start,
500 sweeps, seed 13; the counter-based generator makes it the same on every B200).

It records the oracle's iteration and cycle counts, its per-cycle residual history and
its wall time on the host's threads (OpenMP timing build), next to the GPU's FP64
GMRES-DR on the same system.  Needs a GPU (for the configuration) and about 15 minutes
of a 16-core host.

Usage: python tests/golden/make_c5_record.py   (on a GPU box; rewrites the record)
"""
import json
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

import baylorlqcd_b200 as qq  # noqa: E402

DIMS, KAPPA, SWEEPS, SEED, RESMAX, NGMRES = (24, 24, 24, 48), (0.1566, 0.0025), 500, 13, 2.5e-11, (60, 20)


def main():
    lat = qq.Lattice(*DIMS, bc=(1, 1, 1, -1), device=0)
    u, plaq = lat.heatbath(6.0, SWEEPS, seed=SEED)
    be, bo = lat.pointsource((1, 1, 1, 1), 1, 1)
    t = time.perf_counter()
    xe, xo, info = lat.fermprop(be, bo, KAPPA, inverter=5, resmax=RESMAX, nGMRES=NGMRES)
    gpu = {"seconds": time.perf_counter() - t, "iterations": info.itercount, "cycles": info.ncycles,
           "status": info.status, "hist": [float(h) for h in info.hist]}
    lat.close()
    import oracle

    nt = oracle.use_timing_build()
    ol = oracle.OracleLattice(*DIMS, bc=(1, 1, 1, -1))
    ol.set_gauge(u)
    del u
    t = time.perf_counter()
    xe_o, xo_o, st, log = ol.fermprop(be, bo, KAPPA, inverter=5, resmax=RESMAX, nGMRES=NGMRES)
    dt = time.perf_counter() - t
    hist, hmvp = log.history()
    nv = ol.nvhalf
    diff = max(np.linalg.norm((a - b)[:, :, :, :nv]) / np.linalg.norm(b[:, :, :, :nv])
               for a, b in ((xe, xe_o), (xo, xo_o)))
    out = {"dims": list(DIMS), "kappa": list(KAPPA), "beta": 6.0, "sweeps": SWEEPS, "seed": SEED,
           "plaquette": plaq, "src": "point 1,1,1,1 c1 s1", "nGMRES": list(NGMRES), "resmax": RESMAX,
           "oracle": {"status": int(st), "iterations": int(log.itercount), "cycles": int(log.ncycles),
                      "seconds": dt, "threads": nt, "hist": [float(h) for h in hist],
                      "hist_mvp": [int(m) for m in hmvp],
                      "xe_norm2": float(ol.vecdot(xe_o, xe_o).real), "xo_norm2": float(ol.vecdot(xo_o, xo_o).real)},
           "gpu_fp64_gmresdr": gpu, "gpu_vs_oracle_solution": float(diff)}
    (HERE / "c5_gmresdr_record.json").write_text(json.dumps(out, indent=1) + "\n")
    print("wrote", HERE / "c5_gmresdr_record.json", out["oracle"]["iterations"], dt)


if __name__ == "__main__":
    main()
