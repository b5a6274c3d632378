"""Profiling drivers for the hopping kernels and the batched solver.

    python -m baylorlqcd_b200.probe hop   [--dims 16,16,16,32] [--nrhs 12] [--precision 32]
                                          [--shape 0] [--iters 20] [--no-flush]
    python -m baylorlqcd_b200.probe solve [--dims 16,16,16,32] [--nrhs 12] [--precision 32]
                                          [--kappa 0.1565] [--sweeps 500] [--gauge-cache FILE]

    python -m baylorlqcd_b200.probe twvev [--dims 16,16,16,16] [--nsub 6] [--reps 3]
    python -m baylorlqcd_b200.probe discon [--dims 16,16,16,32] [--nnoise 24] [--kappa 0.1565]
                                           [--mu 0.0] [--solver 1] [--nsub 6]
    python -m baylorlqcd_b200.probe shift [--dims 16,16,16,32] [--kappa 0.1566] [--mu 0.005]
                                          [--shifts 0,-0.099,-0.199,-0.3,-0.5] [--m 40] [--k 12]
    python -m baylorlqcd_b200.probe uneven [--sweeps 200] [--precision 32] [--rhs-block 4]

``hop`` times one hopping-kernel shape (qq_bench_hsingle: random fields, L2 flushed
between launches unless --no-flush) and prints its time and algorithmic bandwidth.

``solve`` runs the batched mixed-precision solve of the 12 spin-colour point sources
twice -- the first run tunes every kernel shape -- and wraps the second in the NVTX
range ``solve``, so a profiler can select its launches (ncu --nvtx --nvtx-include
"solve/").  With --gauge-cache the heatbath configuration is written to FILE in the
reference's GFwrite format on the first run and read back on later runs, which keeps
the heatbath's launches out of a profiled run.
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np


def _dims(s: str):
    return tuple(int(x) for x in s.split(","))


def run_hop(a) -> None:
    import baylorlqcd_b200 as qq

    lat = qq.Lattice(*_dims(a.dims))
    lat.heatbath(6.0, 20, seed=13)
    ms, by = lat.bench_hsingle(a.precision, a.nrhs, a.iters, not a.no_flush, a.shape)
    print(f"hop precision {a.precision} nrhs {a.nrhs} shape {a.shape}: {ms * 1e3:.1f} us, "
          f"{by / ms / 1e6:.0f} GB/s algorithmic", flush=True)
    lat.close()


def run_solve(a) -> None:
    import torch

    import baylorlqcd_b200 as qq

    dims = _dims(a.dims)
    lat = qq.Lattice(*dims, bc=(1, 1, 1, -1))
    if a.gauge_cache and os.path.exists(a.gauge_cache):
        u, _ = qq.gfread(a.gauge_cache, lat.nvhalf, lat.ntotal)
        lat.gauge_upload(u)
    else:
        u, _ = lat.heatbath(6.0, a.sweeps, seed=13)
        if a.gauge_cache:
            qq.gfwrite(a.gauge_cache, u, lat.nvhalf, beta=6.0)
    be = np.zeros((a.nrhs,) + lat.half_shape)
    bo = np.zeros_like(be)
    for i in range(a.nrhs):
        be[i], bo[i] = lat.pointsource((1, 1, 1, 1), i % 3 + 1, (i // 3) % 4 + 1)
    bed, bod = torch.from_numpy(be).cuda(), torch.from_numpy(bo).cuda()
    xe, xo = torch.zeros_like(bed), torch.zeros_like(bod)
    kw = dict(precision=a.precision, rhs_block=a.nrhs, tol=1e-10, solver=1, deflate=0, xe=xe, xo=xo)
    lat.fermprop_batch(bed, bod, (a.kappa, 0.0), **kw)
    torch.cuda.synchronize()
    n0 = qq.launch_count()
    torch.cuda.nvtx.range_push("solve")
    _, _, infos = lat.fermprop_batch(bed, bod, (a.kappa, 0.0), **kw)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    print("iterations", [i.itercount for i in infos], "max true_rel", max(i.true_rel for i in infos),
          "library launches", qq.launch_count() - n0, flush=True)
    lat.close()


def run_twvev(a):
    """twvev on a short heatbath configuration: one untimed call, then --reps timed calls
    (wall clock around the whole entry point, host program build included)."""
    import time

    import baylorlqcd_b200 as qq

    dims = _dims(a.dims)
    lat = qq.Lattice(*dims, bc=(1, 1, 1, -1))
    lat.heatbath(6.0, 5, seed=3)
    lat.twvev(0.156, delta=0.2, nsub=a.nsub)
    for _ in range(a.reps):
        t0 = time.perf_counter()
        J = lat.twvev(0.156, delta=0.2, nsub=a.nsub)
        print("twvev", dims, "nsub", a.nsub, "seconds %.4f" % (time.perf_counter() - t0),
              "psibar psi level 4, t = 1: %.10e" % J[1, 0, 3, 0, 0], flush=True)
    lat.close()


def run_discon(a):
    """twistdiscon (qq_twistdiscon) on a heatbath configuration: nnoise Z(4) noises,
    subtraction levels, five momenta.  Prints wall seconds per noise (the twvev part
    included) and the largest true residual of the solves."""
    import time

    import baylorlqcd_b200 as qq

    dims = _dims(a.dims)
    lat = qq.Lattice(*dims, bc=(1, 1, 1, -1))
    lat.heatbath(6.0, a.sweeps, seed=3)
    kw = dict(nsub=a.nsub, nmom=5, nop=6, delta=0.0, dobndry=0, solver=a.solver, m=60, k=20, precision=32,
              rhs_block=12, tol=1e-10)
    qq.initlagfib(0, 5)
    lat.twistdiscon(4, min(a.nnoise, 12), (a.kappa, a.mu), **kw)  # warm-up (tuning, graph capture)
    qq.initlagfib(0, 5)
    t0 = time.perf_counter()
    J, infos = lat.twistdiscon(4, a.nnoise, (a.kappa, a.mu), **kw)
    dt = time.perf_counter() - t0
    print("twistdiscon", dims, "solver", a.solver, "noises", a.nnoise, "seconds %.3f" % dt,
          "per noise %.4f" % (dt / a.nnoise), "max true_rel %.2e" % max(i.true_rel for i in infos),
          "psibar psi level 4, t = 1: %.8e" % J[1, 0, 3, 0, 0], flush=True)
    lat.close()


def run_shift(a):
    """gmresdrshift (qq_gmresdrshift) on a heatbath configuration: one multi-shift solve
    of a unit-norm Z(4) noise for every shift (in units of 1/kappa^2), then each shift
    solved alone, timed with the library's own solve timer.  Prints seconds, operator
    applications and the largest residual of both."""
    import baylorlqcd_b200 as qq

    dims = _dims(a.dims)
    lat = qq.Lattice(*dims, bc=(1, 1, 1, -1))
    lat.heatbath(6.0, a.sweeps, seed=3)
    kappa = (a.kappa, a.mu)
    sig = np.array([float(x) for x in a.shifts.split(",")]) / a.kappa**2
    qq.initlagfib(0, 5)
    be, _ = lat.z4source()
    be /= np.sqrt(lat.vecdot(be, be).real)
    G = (a.m, a.k)
    lat.gmresdrshift(be, sig[:2], (8, 2), 1e-3, kappa=kappa)  # warm-up (tuning)
    x, resid, info = lat.gmresdrshift(be, sig, G, a.tol, kappa=kappa)
    print("gmresdrshift", dims, "kappa", kappa, "GMRES", G, "shifts", len(sig), "seconds %.3f" % info.seconds,
          "mvp", info.mvp, "cycles", info.ncycles, "max resid %.2e" % resid.max(),
          "status", info.status, flush=True)
    tot, mvp, worst = 0.0, 0, 0.0
    for s in range(len(sig)):
        _, r1, i1 = lat.gmresdrshift(be, sig[s:s + 1], G, a.tol, kappa=kappa)
        tot += i1.seconds
        mvp += i1.mvp
        worst = max(worst, r1[0])
        print("  alone: shift %+.3f/kappa^2 seconds %.3f mvp %d status %d" % (sig[s] * a.kappa**2, i1.seconds,
                                                                           i1.mvp, i1.status), flush=True)
    print("separate solves: seconds %.3f mvp %d max resid %.2e; multi-shift speed-up %.2f" %
          (tot, mvp, worst, tot / info.seconds), flush=True)
    lat.close()


UNEVEN_DIMS = ((8, 8, 8, 16), (12, 12, 12, 24), (16, 16, 16, 32), (20, 20, 20, 40))
UNEVEN_KAPPAS = (0.150, 0.155, 0.1565)


def run_uneven(a):
    """Uneven batch (qq_fermprop_uneven): 48 Wilson solves over four heatbath
    configurations (8^3x16, 12^3x24, 16^3x32, 20^3x40 at beta = 6.0), three kappa
    values each, two point and two Z(4) sources per (configuration, kappa), FP32
    BiCGStab inside FP64 reliable updates to the FP64 full-lattice residual 1e-10.
    One untimed call tunes the kernel shapes of every lattice; then the same call runs
    with the lattices side by side (one host thread and stream each) and one after the
    other.  Prints each schedule's wall seconds, aggregate sec/RHS and worst residual."""
    import baylorlqcd_b200 as qq

    lats, groups = [], []
    qq.initlagfib(0, 11)
    for n, dims in enumerate(UNEVEN_DIMS):
        lat = qq.Lattice(*dims, bc=(1, 1, 1, -1))
        _, plaq = lat.heatbath(6.0, a.sweeps, seed=31 + n)
        lats.append(lat)
        print("configuration", dims, "plaquette %.6f" % plaq, flush=True)
        for kappa in UNEVEN_KAPPAS:
            be = np.zeros((4,) + lat.half_shape)
            bo = np.zeros((4,) + lat.half_shape)
            for i in range(2):
                be[i], bo[i] = lat.pointsource((1 + i, 1, 1, 1), i + 1, 2 * i + 1)
            for i in range(2, 4):
                be[i], bo[i] = lat.z4source()
            groups.append((lat, be, bo, (kappa, 0.0)))
    nrhs = sum(g[1].shape[0] for g in groups)
    kw = dict(precision=a.precision, rhs_block=a.rhs_block, tol=1e-10, deflate=0)
    try:
        qq.fermprop_uneven(groups, concurrent=False, **kw)  # tuning
    except qq.QQError as e:
        print("tuning call:", e, flush=True)
    for conc in (True, False):
        try:
            out, secs = qq.fermprop_uneven(groups, concurrent=conc, **kw)
        except qq.QQError as e:
            print("uneven batch, %s: %s" % ("concurrent" if conc else "sequential", e), flush=True)
            continue
        infos = [i for _, _, inf in out for i in inf]
        worst = max(i.true_rel for i in infos)
        bad = sum(i.status != 0 for i in infos)
        fb = sum(i.fallback for i in infos)
        print("uneven batch, %s: %d solves on %d lattices, %.3f s, %.4f s/RHS, max true rel %.2e, %d not converged, "
              "%d by the GMRES-DR fallback" % ("concurrent" if conc else "sequential", nrhs, len(lats), secs,
                                               secs / nrhs, worst, bad, fb), flush=True)
    for lat in lats:
        lat.close()


def main(argv=None) -> int:
    p = argparse.ArgumentParser(prog="python -m baylorlqcd_b200.probe")
    sub = p.add_subparsers(dest="cmd", required=True)
    h = sub.add_parser("hop")
    h.add_argument("--dims", default="16,16,16,32")
    h.add_argument("--nrhs", type=int, default=12)
    h.add_argument("--precision", type=int, default=32)
    h.add_argument("--shape", type=int, default=0)
    h.add_argument("--iters", type=int, default=20)
    h.add_argument("--no-flush", action="store_true")
    s = sub.add_parser("solve")
    s.add_argument("--dims", default="16,16,16,32")
    s.add_argument("--nrhs", type=int, default=12)
    s.add_argument("--precision", type=int, default=32)
    s.add_argument("--kappa", type=float, default=0.1565)
    s.add_argument("--sweeps", type=int, default=500)
    s.add_argument("--gauge-cache", default=None)
    v = sub.add_parser("twvev")
    v.add_argument("--dims", default="16,16,16,16")
    v.add_argument("--nsub", type=int, default=6)
    v.add_argument("--reps", type=int, default=3)
    d = sub.add_parser("discon")
    d.add_argument("--dims", default="16,16,16,32")
    d.add_argument("--nnoise", type=int, default=24)
    d.add_argument("--kappa", type=float, default=0.1565)
    d.add_argument("--mu", type=float, default=0.0)
    d.add_argument("--solver", type=int, default=1)
    d.add_argument("--nsub", type=int, default=6)
    d.add_argument("--sweeps", type=int, default=200)
    f = sub.add_parser("shift")
    f.add_argument("--dims", default="16,16,16,32")
    f.add_argument("--kappa", type=float, default=0.1566)
    f.add_argument("--mu", type=float, default=0.005)
    f.add_argument("--shifts", default="0,-0.099,-0.199,-0.3,-0.5")
    f.add_argument("--m", type=int, default=40)
    f.add_argument("--k", type=int, default=12)
    f.add_argument("--tol", type=float, default=1e-10)
    f.add_argument("--sweeps", type=int, default=200)
    w = sub.add_parser("uneven")
    w.add_argument("--sweeps", type=int, default=200)
    w.add_argument("--precision", type=int, default=32)
    w.add_argument("--rhs-block", type=int, default=4)
    a = p.parse_args(argv)
    {"hop": run_hop, "solve": run_solve, "twvev": run_twvev, "discon": run_discon, "shift": run_shift,
     "uneven": run_uneven}[a.cmd](a)
    return 0


if __name__ == "__main__":
    sys.exit(main())
