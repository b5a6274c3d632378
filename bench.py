#!/usr/bin/env python
"""Benchmark of the qqcd solver hot path on B200.

Workload (configuration C5, the largest single-GPU one): 24^3x48 quenched SU(3) configuration at
beta = 6.0 (cold start + 500 heatbath sweeps on the GPU), twisted-mass operator at
kappa = 0.1566, mu = 0.0025 (near critical), periodic space / antiperiodic time, 12
spin-colour point sources at site (1,1,1,1), every solution to FP64 true full-lattice
relative residual <= 1e-10.

A step solves the 12 right-hand sides once with the accelerated method: all 12 together
in one batched FP32 BiCGStab (multi-RHS Dslash, per-RHS scalars on the device, the whole
iteration one CUDA graph) with FP64 reliable updates and FP64 true residuals; a
right-hand side that breaks down or stalls is finished by plain FP64 GMRES-DR.  The
reference method -- plain FP64 single-RHS GMRES-DR(60,20) -- is timed on the same GPU on
two of the sources, and its solutions give each batched solution's error against the
FP64 solve.

CPU figures come from the oracle (the C++ restatement of the reference's Fortran) in its
OpenMP timing build on the host cores: at this workload a bounded sample (whole
GMRES-DR(60,20) cycles), and at configuration C1 (8^4, Wilson kappa = 0.150,
GMRES-DR(30,10)) complete solves on one core and on all cores.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Multi-GPU: one process per GPU (torchrun); every rank solves its own configuration
(replicas, weak scaling).

Other measurements (one JSON line each, single GPU), the commands behind the design
notes' figures and the ncu captures under profiles/:
  --mode dslash   the hopping kernel alone (qq_bench_hsingle): --dims, --precision,
                  --nrhs, --shape (0: autotuned), --iters; L2 flushed between launches
  --mode c3       disconnected loops (twistdiscon): --nnoise Z(4) noises, --solver
                  (1 batched, 2 the reference's psc sequence), subtraction level --nsub
  --mode c4       the uneven batch: 48 Wilson solves over 8^3x16 .. 20^3x40
  --mode shift    multi-shift GMRES-DR against each shift alone
  --mode twvev    perturbative VEVs of the loop operators
  --mode vevw     the Wilson loop driver's vev against the oracle's restatement
  --mode learned  the learned preconditioner: trained on a training configuration's own
                  GMRES-DR solves (Z(2) sources, FP64 solutions) and deflation vectors,
                  then flexible GMRES-DR with it against plain GMRES-DR on the held-out
                  benchmark configuration, in wall time and operator applications
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "sec/RHS to 1e-10 FP64 true residual, chosen vs plain GMRES-DR; Dslash HBM GB/s"
FALLBACK_HBM = 6650.0
DEFAULT_DIMS = "24,24,24,48"



def ref_full_solves():
    """Complete solves of the reference method, plain FP64 GMRES-DR(m,k), by the oracle
    on the host cores, keyed by (lattice, kappa, mu, m, k, sweeps): the iteration count
    and wall time of the oracle's solve of source 0 (the full-lattice 1e-10 target is an
    even-system 2.5e-11) recorded by tests/golden/make_c5_record.py on a B200 host.  The
    reference arm times whole GMRES-DR cycles, each a separate call that also pays the
    call's set-up (source preparation, first touch of the 61-vector basis), and scales
    the time per iteration to this count; on the recording host that came to 908 s
    against the complete solve's 732 s."""
    out = {}
    f = ROOT / "tests" / "golden" / "c5_gmresdr_record.json"
    if f.exists():
        r = json.loads(f.read_text())
        key = (tuple(r["dims"]), r["kappa"][0], r["kappa"][1], r["nGMRES"][0], r["nGMRES"][1], r["sweeps"])
        o = r["oracle"]
        out[key] = {"iterations": o["iterations"], "seconds": o["seconds"], "threads": o["threads"],
                    "status": o["status"], "where": "a complete solve recorded on a B200 host "
                    "(tests/golden/c5_gmresdr_record.json)"}
    return out


def parse(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--dims", default=DEFAULT_DIMS)
    p.add_argument("--kappa", type=float, default=0.1566)
    p.add_argument("--mu", type=float, default=0.0025, help="twisted mass (0: Wilson)")
    p.add_argument("--nrhs", type=int, default=12)
    p.add_argument("--precision", type=int, default=32, choices=[-16, 16, 32, 64],
                   help="inner solver storage: 64, 32, 16 (FP16) or -16 (BF16)")
    p.add_argument("--rhs-block", type=int, default=12)
    p.add_argument("--deflate", action="store_true",
                   help="project onto GMRES-DR eigenvectors at every reliable update")
    p.add_argument("--defl-tol", type=float, default=1e-5)
    p.add_argument("--m", type=int, default=60)
    p.add_argument("--k", type=int, default=20)
    p.add_argument("--tol", type=float, default=1e-10)
    p.add_argument("--sweeps", type=int, default=500)
    p.add_argument("--plain-rhs", type=int, default=2)
    p.add_argument("--e2e-steps", type=int, default=0, help="end-to-end steps (0: min(steps, 5))")
    p.add_argument("--cpu-threads", type=int, default=0, help="host threads of the CPU legs (0: all)")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--mode", default="solve",
                   choices=["solve", "dslash", "c3", "c4", "shift", "twvev", "vevw", "learned", "eigen"])
    p.add_argument("--train-solves", type=int, default=8, help="--mode learned: training solves")
    p.add_argument("--train-steps", type=int, default=200, help="--mode learned: Adam steps")
    p.add_argument("--channels", default="4,8,8,4", help="--mode learned: channels per layer")
    p.add_argument("--shape", type=int, default=0, help="--mode dslash: kernel shape (0: autotuned)")
    p.add_argument("--iters", type=int, default=20, help="--mode dslash: timed launches")
    p.add_argument("--nnoise", type=int, default=24, help="--mode c3: noises")
    p.add_argument("--solver", type=int, default=1, help="--mode c3: 1 batched, 2 psc")
    p.add_argument("--nsub", type=int, default=6, help="--mode c3 / twvev: subtraction level")
    p.add_argument("--eig", default="200,160,150", help="--mode eigen: m, k and cycles of the eigen-iteration")
    p.add_argument("--cpu-cycles", type=int, default=1, help="--mode eigen: oracle cycles timed (0: none)")
    return p.parse_args(argv)


# ---------------------------------------------------------------------------
def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def max_over_ranks(x: float, world: int) -> float:
    """The largest value of x over all ranks (x itself on one rank): NCCL reduces a
    device tensor, gloo a host tensor."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sec_per_rhs(max_total_ms: float, steps: int, nrhs: int, world: int) -> float:
    """Whole-job throughput: every rank solves nrhs right-hand sides per step (replicas),
    and the job takes as long as its slowest rank."""
    return max_total_ms * 1e-3 / (steps * nrhs * world)


def peaks():
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        d = json.loads(f.read_text())
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM, "fallback"


def dims_label(dims) -> str:
    """16^3x32 style lattice label."""
    nx, ny, nz, nt = dims
    return "%d^3x%d" % (nx, nt) if nx == ny == nz else "%dx%dx%dx%d" % tuple(dims)


def operator_label(mu: float) -> str:
    return "twisted mass mu=%g" % mu if mu else "Wilson"


def shape_name(shape: int) -> str:
    """Kernel behind a hopping-kernel shape code (qq_bench_hsingle)."""
    if shape in (1, 2, 4):
        return "hop_kernel"
    if 32 <= shape <= 128:
        return "hop_staged_kernel"
    if 202 <= shape <= 204:
        return "hop_mrhs_kernel"
    return {301: "hop_f2_kernel", 302: "hop_f2_kernel", 303: "hop_f2_kernel", 304: "hop_f2p_kernel",
            305: "hop_f2s_kernel", 306: "hop_f2a_kernel", 307: "hop_f2a_kernel",
            308: "hop_f2a_kernel", 309: "hop_f2a_kernel", 310: "hop_f2a_kernel",
            311: "hop_f2a_kernel"}.get(shape, "hop kernel")


# DRAM bytes (read + write) of one EPI_STORE launch from an ncu capture, keyed by
# (kernel, precision, RHS, lattice); the capture's summary is the source.  The ring
# depths and register caps of hop_f2a_kernel (shapes 306-310) move the same bytes.
NCU_TRAFFIC = {
    ("hop_f2a_kernel", 32, 12, (16, 16, 16, 32)): (150.6e6, "profiles/hop_f2a_kernel_fp32_blk12_16x16x16x32.md"),
}


class Clocks:
    """nvidia-smi sampler (200 ms) running during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.rows = []
        self.proc = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(device)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, ValueError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 7:
                self.rows.append(parts)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[3 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def point_sources(lat, nrhs):
    be = np.zeros((nrhs,) + lat.half_shape)
    bo = np.zeros((nrhs,) + lat.half_shape)
    for i in range(nrhs):
        ic, idd = i % 3 + 1, (i // 3) % 4 + 1
        e, o = lat.pointsource((1, 1, 1, 1), ic, idd)
        be[i], bo[i] = e, o
    return be, bo


# ---------------------------------------------------------------------------
# CPU legs: the reference algorithm (its C++ restatement, oracle/) on the host cores,
# in the oracle's OpenMP timing build.
def load_timing_oracle(threads: int):
    import oracle

    return oracle, oracle.use_timing_build(threads if threads > 0 else (os.cpu_count() or 1))


def oracle_cycle(oracle, ol, kappa, m, k, src_idx, cycles=1):
    """Wall time of `cycles` GMRES-DR(m,k) cycles of the oracle's fermprop on point
    source src_idx (no convergence inside: resmax 1e-30); returns (seconds, iterations)."""
    ic, idd = src_idx % 3 + 1, (src_idx // 3) % 4 + 1
    be, bo = ol.pointsource((1, 1, 1, 1), ic, idd)
    oracle.set_kcyclim(cycles)
    t = time.perf_counter()
    _, _, _, log = ol.fermprop(be, bo, kappa, inverter=5, resmax=1e-30, nGMRES=(m, k))
    dt = time.perf_counter() - t
    oracle.set_kcyclim(0)
    return dt, log.itercount


def c1_config(oracle):
    """Configuration C1: 8^4 at beta = 6.0 from the oracle's restatement of the
    reference's heatbath (cold start, lagfib seed (0, 13), 200 sweeps)."""
    ol = oracle.OracleLattice(8, 8, 8, 8, bc=(1, 1, 1, -1))
    u = ol.coldstart()
    oracle.initlagfib(0, 13)
    plaq = ol.heatbath(u, 6.0, 200)
    ol.set_gauge(u)
    return ol, u, float(plaq[-1])


def c1_measure(oracle, nthreads, qq=None, device=0):
    """C1 solved completely: the oracle's fermprop with GMRES-DR(30,10) to 1e-10 at
    kappa = 0.150 on one core and on all cores, and (with qq) the same solve on the GPU
    by plain FP64 GMRES-DR and by the batched FP32 method."""
    ol, u, plaq = c1_config(oracle)
    be, bo = ol.pointsource((1, 1, 1, 1), 1, 1)
    kappa = (0.150, 0.0)
    out = {"config": "C1: 8^4 heatbath beta=6.0 (oracle, seed 13, 200 sweeps), Wilson kappa=0.150, "
                     "point source, GMRES-DR(30,10) to 1e-10", "plaquette": plaq}
    for label, nt in (("cpu_1core", 1), ("cpu_allcore", nthreads)):
        oracle.lib().oq_set_threads(nt)
        t = time.perf_counter()
        xe, xo, st, log = ol.fermprop(be, bo, kappa, inverter=5, resmax=1e-10, nGMRES=(30, 10))
        out[label] = {"seconds": time.perf_counter() - t, "cores": nt, "status": int(st),
                      "iterations": int(log.itercount), "cycles": int(log.ncycles)}
    oracle.lib().oq_set_threads(nthreads)
    if qq is not None:
        lat = qq.Lattice(8, 8, 8, 8, bc=(1, 1, 1, -1), device=device)
        lat.gauge_upload(u)
        xg, xog, info = lat.fermprop(be, bo, kappa, inverter=5, resmax=1e-10, nGMRES=(30, 10))  # warm-up
        t = time.perf_counter()
        xg, xog, info = lat.fermprop(be, bo, kappa, inverter=5, resmax=1e-10, nGMRES=(30, 10))
        out["gpu_gmresdr_fp64"] = {"seconds": time.perf_counter() - t, "iterations": info.itercount,
                                   "cycles": info.ncycles, "true_rel": info.true_rel}
        nv = ol.nvhalf
        out["gpu_vs_oracle_solution"] = float(max(
            np.linalg.norm((a - b)[:, :, :, :nv]) / np.linalg.norm(b[:, :, :, :nv]) for a, b in ((xg, xe), (xog, xo))))
        lat.fermprop_batch(be[None], bo[None], kappa, m=30, k=10, precision=32, rhs_block=1, tol=1e-10, solver=1,
                           deflate=0)
        t = time.perf_counter()
        _, _, binfo = lat.fermprop_batch(be[None], bo[None], kappa, m=30, k=10, precision=32, rhs_block=1,
                                         tol=1e-10, solver=1, deflate=0)
        out["gpu_batched_fp32"] = {"seconds": time.perf_counter() - t, "iterations": binfo[0].itercount,
                                   "true_rel": binfo[0].true_rel}
        lat.close()
    return out


# ---------------------------------------------------------------------------
def run_ours(a, rank, world, local):
    import torch

    import baylorlqcd_b200 as qq

    torch.cuda.set_device(local)
    dims = tuple(int(x) for x in a.dims.split(","))
    lat = qq.Lattice(*dims, bc=(1, 1, 1, -1), device=local)
    u, plaq = lat.heatbath(6.0, a.sweeps, seed=13 + rank)
    be, bo = point_sources(lat, a.nrhs)
    kappa = (a.kappa, a.mu)
    stream = torch.cuda.ExternalStream(lat.stream_handle())
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    be_d, bo_d = torch.from_numpy(be).cuda(), torch.from_numpy(bo).cuda()
    xe_d, xo_d = torch.zeros_like(be_d), torch.zeros_like(bo_d)
    meth = dict(m=a.m, k=a.k, precision=a.precision, rhs_block=a.rhs_block, tol=a.tol, solver=1,
                deflate=1 if a.deflate else 0, defl_tol=a.defl_tol)

    def step(be_, bo_, xe_, xo_):
        flush.fill_(rank + 1)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        _, _, infos = lat.fermprop_batch(be_, bo_, kappa, xe=xe_, xo=xo_, **meth)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1), infos

    for _ in range(a.warmup):
        step(be_d, bo_d, xe_d, xo_d)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    n0 = qq.launch_count()
    times, infos = [], None
    torch.cuda.nvtx.range_push("timed")  # ncu --nvtx --nvtx-include "timed/" selects these launches
    for _ in range(a.steps):
        ms, infos = step(be_d, bo_d, xe_d, xo_d)
        times.append(ms)
    torch.cuda.nvtx.range_pop()
    n1 = qq.launch_count()
    torch.cuda.synchronize()
    clk = clocks.stop()
    total_ms = max_over_ranks(sum(times), world)
    if world > 1:
        torch.distributed.barrier()
    spr = sec_per_rhs(total_ms, a.steps, a.nrhs, world)
    converged = all(i.status == 0 and i.true_rel <= a.tol for i in infos)
    xe_b, xo_b = xe_d.cpu().numpy(), xo_d.cpu().numpy()

    # end-to-end through the same entry point with pinned host buffers
    be_h = torch.from_numpy(be).pin_memory().numpy()
    bo_h = torch.from_numpy(bo).pin_memory().numpy()
    xe_h = torch.zeros(be.shape, dtype=torch.float64).pin_memory().numpy()
    xo_h = torch.zeros(bo.shape, dtype=torch.float64).pin_memory().numpy()
    ne2e = a.e2e_steps if a.e2e_steps > 0 else min(a.steps, 5)
    e2e_ms = [step(be_h, bo_h, xe_h, xo_h)[0] for _ in range(ne2e)]
    print("step ms: timed %s; e2e %s" % (["%.0f" % t for t in times], ["%.0f" % t for t in e2e_ms]),
          file=sys.stderr, flush=True)
    e2e = sum(e2e_ms) * 1e-3 / (len(e2e_ms) * a.nrhs)
    half_bytes = int(np.prod(lat.half_shape)) * 8

    # live Dslash roofline: one instrumented step, every hopping launch timed; the
    # dominant kernel is the block hop of the batched solve (precision, rhs_block)
    lat.profile_hop(True)
    step(be_d, bo_d, xe_d, xo_d)
    nlaunch, hop_ms, hop_bytes, hop_flops = lat.profile_hop_select(a.precision, min(a.rhs_block, a.nrhs))
    nall, all_ms, _, _ = lat.profile_hop_select(0, 0)
    lat.profile_hop(False)
    hbm, hbm_kind = peaks()
    achieved = hop_bytes / (hop_ms * 1e-3) / 1e9 if hop_ms > 0 else 0.0
    gflops = hop_flops / (hop_ms * 1e-3) / 1e9 if hop_ms > 0 else 0.0
    shape = lat.hop_tuned_shape(a.precision, a.rhs_block)
    traffic = NCU_TRAFFIC.get((shape_name(shape), a.precision, a.rhs_block, dims))

    # plain FP64 GMRES-DR (the reference method) on the same GPU; its solutions are the
    # FP64 reference solves of the first right-hand sides
    npl = max(1, min(a.plain_rhs, a.nrhs))
    xe_p, xo_p, pinfo = lat.fermprop_batch(be_d[:npl].clone(), bo_d[:npl].clone(), kappa, m=a.m, k=a.k,
                                           precision=64, rhs_block=1, tol=a.tol, solver=0)
    plain = sum(i.seconds for i in pinfo) / npl
    plain_iters = pinfo[0].itercount
    xe_p, xo_p = xe_p.cpu().numpy(), xo_p.cpu().numpy()
    nv = lat.nvhalf

    def rel(x, y):
        return float(np.linalg.norm((x - y)[:, :, :, :nv]) / np.linalg.norm(y[:, :, :, :nv]))

    err64 = max(max(rel(xe_b[i], xe_p[i]), rel(xo_b[i], xo_p[i])) for i in range(npl))

    out = {
        "metric": METRIC,
        "value": spr,
        "unit": "s/RHS",
        "n_gpus": world,
        "steps": a.steps,
        "warmup": a.warmup,
        "ms_per_step": total_ms / a.steps,
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": {-16: "bf16/fp64", 16: "fp16/fp64", 32: "fp32/fp64", 64: "fp64"}[a.precision],
        "data": "synthetic: GPU heatbath configuration (beta=6.0, cold start, %d sweeps), point sources" % a.sweeps,
        "config": {"workload": "%s %s kappa=%.4f, %d point sources, batched FP%d BiCGStab with FP64 "
                               "reliable updates%s, tol %.0e full-lattice FP64; plain = FP64 GMRES-DR(%d,%d)"
                               % (dims_label(dims), operator_label(a.mu), a.kappa, a.nrhs, a.precision,
                                  " + GMRES-DR deflation" if a.deflate else "", a.tol, a.m, a.k),
                   "lattice": list(dims), "kappa": a.kappa, "mu": a.mu, "nrhs": a.nrhs, "precision": a.precision,
                   "rhs_block": a.rhs_block, "parallelism": "replicas x%d" % world,
                   "l2": "512 MiB buffer written before every step; working set > L2",
                   "plaquette": plaq},
        "converged": converged,
        "max_true_rel": max(i.true_rel for i in infos),
        "error_vs_fp64": {"precision": a.precision, "max_rel": err64, "rhs": npl,
                          "what": "||x - x_FP64|| / ||x_FP64|| over both halves, x_FP64 from plain FP64 GMRES-DR"},
        "fallback": [i.fallback for i in infos],
        "finished_by": [i.finished_by for i in infos],
        "iterations": [i.itercount for i in infos],
        "plain_gmresdr_sec_per_rhs": plain,
        "plain_gmresdr_iterations": plain_iters,
        "speedup_vs_plain_gmresdr": plain / (spr * world) if spr > 0 else None,
        "e2e": {"value": e2e, "unit": "s/RHS", "h2d_bytes_per_step": 2 * a.nrhs * half_bytes,
                "d2h_bytes_per_step": 2 * a.nrhs * half_bytes, "steps": ne2e},
        "roofline": {"bound": "hbm", "kernel": "%s (Dslash, %d-bit, shape %d)" % (shape_name(shape), a.precision, shape),
                     "achieved": achieved, "peak": hbm, "peak_kind": hbm_kind, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": traffic[0] if traffic else None,
                     "traffic_source": traffic[1] if traffic else None, "launches_measured": nlaunch,
                     "avg_launch_us": hop_ms * 1e3 / max(nlaunch, 1), "gflops": gflops,
                     "flops_per_site_rhs": 1320,
                     "hop_share_of_step": all_ms / (total_ms / a.steps) if total_ms > 0 else None,
                     "hop_launches_all": nall},
        "gpu_launches": int(n1 - n0),
        "clocks": clk,
    }

    # CPU baseline: the oracle on all host cores, a bounded sample of this workload
    if rank == 0 and world == 1 and not a.no_cpu:
        oracle, nt = load_timing_oracle(a.cpu_threads)
        ol = oracle.OracleLattice(*dims, bc=(1, 1, 1, -1))
        ol.set_gauge(u)
        dt, its = oracle_cycle(oracle, ol, kappa, a.m, a.k, 0)
        out["cpu_baseline"] = {"value": dt / max(its, 1) * plain_iters, "unit": "s/RHS", "cores": nt, "kind": "port",
                               "sample": "one GMRES-DR(%d,%d) cycle (%d iterations, %.1f s) of the oracle's FP64 "
                                         "restatement on source 0, %d threads, scaled to the %d iterations plain FP64 "
                                         "GMRES-DR needed on this system (GPU run above); the cycle also pays the "
                                         "call's set-up" % (a.m, a.k, its, dt, nt, plain_iters)}
        del ol
        out["c1"] = c1_measure(oracle, nt, qq, local)
    lat.close()
    return out


def run_reference(a, rank, world, local):
    """The reference algorithm -- plain FP64 GMRES-DR(m,k), its C++ restatement in
    oracle/ -- on all host cores (OpenMP timing build), on this workload's configuration
    and point sources.  A step is one whole GMRES-DR cycle on the next source; the
    sec/RHS value scales the mean cycle to the iteration count of a complete solve: the
    oracle's own complete solve of this workload (REF_FULL_SOLVES), or, where none is
    recorded, one run here before the timed steps."""
    import baylorlqcd_b200 as qq

    dims = tuple(int(x) for x in a.dims.split(","))
    lat = qq.Lattice(*dims, bc=(1, 1, 1, -1), device=local)   # configuration input only
    u, plaq = lat.heatbath(6.0, a.sweeps, seed=13)
    lat.close()
    oracle, nt = load_timing_oracle(a.cpu_threads)
    ol = oracle.OracleLattice(*dims, bc=(1, 1, 1, -1))
    ol.set_gauge(u)
    del u
    kappa = (a.kappa, a.mu)
    key = (dims, a.kappa, a.mu, a.m, a.k, a.sweeps)
    full = ref_full_solves().get(key)
    if full is None:  # a complete solve of source 0 here, untimed
        be, bo = ol.pointsource((1, 1, 1, 1), 1, 1)
        t = time.perf_counter()
        _, _, st, log = ol.fermprop(be, bo, kappa, inverter=5, resmax=a.tol * 0.25, nGMRES=(a.m, a.k))
        full = {"iterations": int(log.itercount), "seconds": time.perf_counter() - t, "threads": nt,
                "status": int(st), "where": "this run"}
    for _ in range(a.warmup):  # a short cycle per warm-up step (page-in, thread start)
        oracle_cycle(oracle, ol, kappa, 2, 1, 0)
    times, its = [], []
    for i in range(a.steps):
        dt, n = oracle_cycle(oracle, ol, kappa, a.m, a.k, i % a.nrhs)
        times.append(dt)
        its.append(n)
    per_it = sum(times) / max(sum(its), 1)
    value = per_it * full["iterations"]
    return {
        "metric": METRIC, "impl": "reference", "value": value, "unit": "s/RHS", "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": statistics.mean(times) * 1e3, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp64", "data": "same configuration and sources "
        "(GPU heatbath, used as input only)",
        "config": {"workload": "%s %s kappa=%.4f point sources, GMRES-DR(%d,%d), tol %.0e"
                               % (dims_label(dims), operator_label(a.mu), a.kappa, a.m, a.k, a.tol),
                   "lattice": list(dims), "kappa": a.kappa, "mu": a.mu, "plaquette": plaq},
        "cpu_baseline": {"value": value, "unit": "s/RHS", "cores": nt, "kind": "port",
                         "sample": "per step one GMRES-DR(%d,%d) cycle (%d iterations, mean %.1f s) of the oracle on "
                                   "%d threads; sec/RHS = seconds per iteration x the %d iterations of a complete "
                                   "solve of this system by the oracle (%s: %.0f s on %d threads); every sample "
                                   "also pays its call's set-up"
                                   % (a.m, a.k, its[0] if its else 0, statistics.mean(times), nt, full["iterations"],
                                      full["where"], full["seconds"], full["threads"])},
        "full_solve": full,
        "e2e": {"value": value, "unit": "s/RHS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


# ---------------------------------------------------------------------------
# Other measurements (--mode)
def run_dslash(a):
    """The hopping kernel alone on random fields of a heatbath configuration."""
    import baylorlqcd_b200 as qq

    dims = tuple(int(x) for x in a.dims.split(","))
    lat = qq.Lattice(*dims, bc=(1, 1, 1, -1))
    lat.heatbath(6.0, 20, seed=13)
    ms, by = lat.bench_hsingle(a.precision, a.nrhs, a.iters, True, a.shape)
    shape = a.shape
    if not shape:
        try:
            shape = lat.hop_tuned_shape(a.precision, a.nrhs)
        except qq.QQError:
            shape = 0
    hbm, kind = peaks()
    flops = 1320.0 * lat.nvhalf * 16 * a.nrhs
    lat.close()
    return {"mode": "dslash", "kernel": "%s (shape %d)" % (shape_name(shape), shape), "lattice": list(dims),
            "precision": a.precision, "nrhs": a.nrhs, "us_per_launch": ms * 1e3, "bytes_per_launch": by,
            "gbs": by / ms / 1e6, "frac": by / ms / 1e6 / hbm, "peak": hbm, "peak_kind": kind,
            "gflops": flops / ms / 1e6, "l2": "512 MiB written between launches"}


def heatbath_lattice(qq, dims, sweeps, seed):
    lat = qq.Lattice(*dims, bc=(1, 1, 1, -1))
    _, plaq = lat.heatbath(6.0, sweeps, seed=seed)
    return lat, plaq


def run_c3(a):
    """twistdiscon with nnoise Z(4) noises (noise drawing, solves, traces and twvev), wall
    time per noise after one warm-up call."""
    import baylorlqcd_b200 as qq

    dims = tuple(int(x) for x in a.dims.split(","))
    lat, plaq = heatbath_lattice(qq, dims, a.sweeps, 3)
    kw = dict(nsub=a.nsub, nmom=5, nop=6, delta=0.0, dobndry=0, solver=a.solver, m=a.m, k=a.k,
              precision=a.precision, rhs_block=a.rhs_block, tol=a.tol)
    kappa = (a.kappa, a.mu)
    qq.initlagfib(0, 5)
    lat.twistdiscon(4, min(a.nnoise, a.rhs_block), kappa, **kw)
    qq.initlagfib(0, 5)
    t0 = time.perf_counter()
    _, infos = lat.twistdiscon(4, a.nnoise, kappa, **kw)
    dt = time.perf_counter() - t0
    lat.close()
    return {"mode": "c3", "lattice": list(dims), "kappa": a.kappa, "mu": a.mu, "nnoise": a.nnoise,
            "solver": a.solver, "nsub": a.nsub, "plaquette": plaq, "seconds": dt, "sec_per_noise": dt / a.nnoise,
            "max_true_rel": max(i.true_rel for i in infos), "fallback": sum(1 for i in infos if i.fallback)}


def run_c4(a):
    """The uneven batch: 48 Wilson solves over four heatbath configurations, three kappa
    values each, two point and two Z(4) sources per (configuration, kappa); one tuning
    call, then the lattices side by side and one after the other."""
    import baylorlqcd_b200 as qq

    lats, groups = [], []
    qq.initlagfib(0, 11)
    for n, dims in enumerate(((8, 8, 8, 16), (12, 12, 12, 24), (16, 16, 16, 32), (20, 20, 20, 40))):
        lat, _ = heatbath_lattice(qq, dims, a.sweeps, 31 + n)
        lats.append(lat)
        for kappa in (0.150, 0.155, 0.1565):
            be = np.zeros((4,) + lat.half_shape)
            bo = np.zeros((4,) + lat.half_shape)
            for i in range(2):
                be[i], bo[i] = lat.pointsource((1 + i, 1, 1, 1), i + 1, 2 * i + 1)
            for i in range(2, 4):
                be[i], bo[i] = lat.z4source()
            groups.append((lat, be, bo, (kappa, 0.0)))
    nrhs = sum(g[1].shape[0] for g in groups)
    kw = dict(precision=a.precision, rhs_block=4, tol=a.tol, deflate=0)
    qq.fermprop_uneven(groups, concurrent=False, **kw)  # tuning
    out = {"mode": "c4", "solves": nrhs, "lattices": len(lats)}
    for conc in (True, False):
        res, secs = qq.fermprop_uneven(groups, concurrent=conc, **kw)
        infos = [i for _, _, inf in res for i in inf]
        out["concurrent" if conc else "sequential"] = {
            "seconds": secs, "sec_per_rhs": secs / nrhs, "max_true_rel": max(i.true_rel for i in infos),
            "not_converged": sum(i.status != 0 for i in infos), "fallback": sum(1 for i in infos if i.fallback)}
    for lat in lats:
        lat.close()
    return out


def run_shift(a):
    """Multi-shift GMRES-DR of a unit-norm Z(4) noise for five shifts (in units of
    1/kappa^2) against each shift solved alone (the library's own solve timer)."""
    import baylorlqcd_b200 as qq

    dims = tuple(int(x) for x in a.dims.split(","))
    lat, _ = heatbath_lattice(qq, dims, a.sweeps, 3)
    kappa = (a.kappa, a.mu)
    sig = np.array([0.0, -0.099, -0.199, -0.3, -0.5]) / a.kappa**2
    qq.initlagfib(0, 5)
    be, _ = lat.z4source()
    be /= np.sqrt(lat.vecdot(be, be).real)
    lat.gmresdrshift(be, sig[:2], (8, 2), 1e-3, kappa=kappa)  # tuning
    _, resid, info = lat.gmresdrshift(be, sig, (a.m, a.k), a.tol, kappa=kappa)
    alone = [lat.gmresdrshift(be, sig[i:i + 1], (a.m, a.k), a.tol, kappa=kappa) for i in range(len(sig))]
    lat.close()
    return {"mode": "shift", "lattice": list(dims), "kappa": kappa, "GMRES": [a.m, a.k], "shifts": len(sig),
            "multishift": {"seconds": info.seconds, "mvp": info.mvp, "cycles": info.ncycles,
                           "max_resid": float(resid.max())},
            "alone": {"seconds": sum(r[2].seconds for r in alone), "mvp": sum(r[2].mvp for r in alone),
                      "max_resid": float(max(r[1][0] for r in alone))}}


def run_twvev(a):
    """twvev on a short heatbath configuration: one untimed call, then three timed calls
    (wall clock around the entry point, host program build included)."""
    import baylorlqcd_b200 as qq

    dims = tuple(int(x) for x in a.dims.split(","))
    lat, _ = heatbath_lattice(qq, dims, 5, 3)
    lat.twvev(0.156, delta=0.2, nsub=a.nsub)
    ts = []
    for _ in range(3):
        t0 = time.perf_counter()
        lat.twvev(0.156, delta=0.2, nsub=a.nsub)
        ts.append(time.perf_counter() - t0)
    lat.close()
    return {"mode": "twvev", "lattice": list(dims), "nsub": a.nsub, "seconds": ts}


def run_vevw(a):
    """The Wilson loop driver's vev (qq_vev) on a heatbath configuration: wall time of the
    entry point (one untimed call, then five), against the oracle's serial restatement of
    the reference's loops on the same links (the whole computation, timed once), and the
    largest difference of the two Jvev."""
    import baylorlqcd_b200 as qq

    dims = tuple(int(x) for x in a.dims.split(","))
    lat = qq.Lattice(*dims, bc=(1, 1, 1, -1))
    u, plaq = lat.heatbath(6.0, 20, seed=13)
    kappa = a.kappa
    lat.vev(kappa)
    ts = []
    for _ in range(5):
        t0 = time.perf_counter()
        J, plaq_g, psi = lat.vev(kappa)
        ts.append(time.perf_counter() - t0)
    lat.close()
    res = {"mode": "vevw", "lattice": list(dims), "kappa": kappa, "gpu_seconds": ts, "plaquette": plaq_g}
    if not a.no_cpu:
        import oracle

        ol = oracle.OracleLattice(*dims, bc=(1, 1, 1, -1))
        ol.set_gauge(u)
        t0 = time.perf_counter()
        Jo, plaq_o, _ = ol.vev(kappa)
        res["cpu_baseline"] = {"seconds": time.perf_counter() - t0, "cores": 1, "kind": "port",
                               "sample": "the whole vev on the same links, the oracle's serial restatement"}
        res["max_rel_diff"] = float(np.abs(J - Jo).max() / np.abs(Jo).max())
    return res


def run_learned(a):
    """The learned preconditioner on the benchmark operator.  Training configuration
    (heatbath seed 14): --train-solves Z(2) sources solved by plain FP64 GMRES-DR(m,k) to
    the tolerance (the deflation space of the first kept), the pairs (b, x) of those
    solves and (Hdbletm v, v) of its deflation vectors; Adam on them.  Held-out
    configuration (seed 13, the benchmark's): the point source of site (1,1,1,1) solved by
    flexible GMRES-DR(m,k) with the network, without it, and by plain GMRES-DR."""
    import baylorlqcd_b200 as qq

    dims = tuple(int(x) for x in a.dims.split(","))
    kappa = (a.kappa, a.mu)
    G = (a.m, a.k)
    chans = tuple(int(c) for c in a.channels.split(","))
    train, _ = heatbath_lattice(qq, dims, a.sweeps, 14)
    qq.initlagfib(0, 7)
    B, X = [], []
    d = train.deflation(a.m, a.k)
    t0 = time.perf_counter()
    for i in range(a.train_solves):
        b, _ = train.z2source()
        x, _ = train.gmresdr(b, train.new_half(), G, a.tol, kappa=kappa, defl=d if i == 0 else None)
        B.append(b)
        X.append(x)
    for j in range(d.k):
        v = d.vector(j)
        X.append(v)
        B.append(train.hdbletm(v, 0, kappa))
    t_pairs = time.perf_counter() - t0
    net = qq.Net(chans, seed=1, scale=a.kappa**2)
    t0 = time.perf_counter()
    losses = net.train_pairs(train, np.stack(B), np.stack(X), nsteps=a.train_steps, lr=2e-3)
    t_train = time.perf_counter() - t0
    d.close()
    train.close()
    test, _ = heatbath_lattice(qq, dims, a.sweeps, 13)
    b = test.pointsource((1, 1, 1, 1), 1, 1)[0]
    test.fgmres(b, kappa, m=G[0], k=G[1], resmax=1e-3, net=net)  # tuning
    res = {}
    for label, n in (("fgmresdr_net", net), ("fgmresdr_plain", None)):
        _, info = test.fgmres(b, kappa, m=G[0], k=G[1], resmax=a.tol, max_cycles=500, net=n)
        res[label] = {"seconds": info.seconds, "mvp": info.mvp, "status": info.status, "fallback": info.fallback,
                      "true_rel": info.true_rel}
    _, info = test.gmresdr(b, test.new_half(), G, a.tol, kappa=kappa)
    res["gmresdr"] = {"seconds": info.seconds, "mvp": info.mvp, "status": info.status, "true_rel": info.true_rel}
    test.close()
    return {"mode": "learned", "lattice": list(dims), "kappa": kappa, "channels": list(chans), "GMRES": list(G),
            "training": {"solves": a.train_solves, "low_modes": len(B) - a.train_solves, "pairs_seconds": t_pairs,
                         "adam_steps": a.train_steps, "train_seconds": t_train, "loss_first": float(losses[0]),
                         "loss_last": float(losses[-1])},
            "held_out": res,
            "gain_vs_gmresdr": res["gmresdr"]["seconds"] / res["fgmresdr_net"]["seconds"]}


def run_eigen(a):
    """The Wilson loop driver's eigenmode subtraction (testFUNC) on a heatbath
    configuration: the modes of M (kind 1) and of M gamma5 (kind 2) with the
    eigen-iteration's m, k and cycles (the reference's 200, 160, 150 by default), then one
    Z(4) noise: its solve (GMRES-DR(80,40) to 1e-7, the driver's settings), the polynomial
    fits and generalaverage (all ten styles).  Wall time of each call.  Beside it the
    oracle's time for --cpu-cycles cycles of the kind-1 iteration on the same lattice."""
    import baylorlqcd_b200 as qq

    dims = tuple(int(x) for x in a.dims.split(","))
    m, k, cyc = (int(x) for x in a.eig.split(","))
    kappa = (a.kappa, 0.0)
    lat, plaq = heatbath_lattice(qq, dims, a.sweeps, 3)
    out = {"mode": "eigen", "lattice": list(dims), "kappa": a.kappa, "eig_GMRES": [m, k], "cycles": cyc,
           "plaquette": plaq}
    qq.initlagfib(0, 5)
    se, so = lat.z4source()
    t0 = time.perf_counter()
    M = lat.eigenmodes(1, (m, k), cyc, kappa)
    t1 = time.perf_counter()
    Mp = lat.eigenmodes(2, (m, k), cyc, kappa, se, so)
    t2 = time.perf_counter()
    out["modes_of_M"] = {"seconds": t1 - t0, "kept": M.num, "cycles": M.cycles, "mvp": M.mvp,
                         "smallest": [abs(M.evals[0]) if M.num else None]}
    out["modes_of_Mgamma5"] = {"seconds": t2 - t1, "kept": Mp.num, "cycles": Mp.cycles, "mvp": Mp.mvp,
                               "smallest": [abs(Mp.evals[0]) if Mp.num else None]}
    gpu_mvp_m = M.mvp
    ze, zo = lat.z4source()
    t3 = time.perf_counter()
    xe, xo, info = lat.fermprop(ze, zo, kappa, inverter=5, resmax=1e-7, nGMRES=(80, 40))
    t4 = time.perf_counter()
    co = {p: lat.ppcoeffs(ze, zo, a.kappa, p) for p in (5, 8, 11)}
    copoly = lat.ppcoeffs(se, so, a.kappa, 8)
    t5 = time.perf_counter()
    J = lat.generalaverage(M, Mp, ze, zo, xe, xo, a.kappa, co[11], co[8], co[5], copoly)
    t6 = time.perf_counter()
    out["noise"] = {"solve_seconds": t4 - t3, "solve_status": info.status, "fits_seconds": t5 - t4,
                    "generalaverage_seconds": t6 - t5, "finite": bool(np.isfinite(J).all())}
    M.close()
    Mp.close()
    lat.close()
    if a.cpu_cycles > 0 and not a.no_cpu:
        import oracle

        threads = oracle.use_timing_build(a.cpu_threads or None)
        ol = oracle.OracleLattice(*dims, bc=(1, 1, 1, -1))
        g = qq.Lattice(*dims, bc=(1, 1, 1, -1))
        u, _ = g.heatbath(6.0, a.sweeps, seed=3)
        g.close()
        ol.set_gauge(u)
        c0 = time.perf_counter()
        ol.eigmodes(1, (m, k), a.cpu_cycles, kappa)
        c1 = time.perf_counter()
        cpu_mvp = m + (a.cpu_cycles - 1) * (m - k)  # operator applications of the sampled cycles
        out["cpu_baseline"] = {"kind": "port", "cores": threads, "cycles_timed": a.cpu_cycles,
                               "seconds": c1 - c0,
                               "modes_of_M_seconds_scaled": (c1 - c0) / cpu_mvp * gpu_mvp_m,
                               "sample": f"{a.cpu_cycles} cycle(s) of the kind-1 eigen-iteration ({cpu_mvp} operator "
                                         f"applications with their orthogonalisation and restarts), scaled to the "
                                         f"{gpu_mvp_m} of the GPU run"}
    return out


def main(argv=None):
    a = parse(argv)
    if a.mode != "solve":
        fn = {"dslash": run_dslash, "c3": run_c3, "c4": run_c4, "shift": run_shift, "twvev": run_twvev, "vevw": run_vevw,
              "learned": run_learned, "eigen": run_eigen}[a.mode]
        print(json.dumps(fn(a)), flush=True)
        return 0
    rank, world, local = dist_env()
    if a.impl == "reference":
        # the reference's CPU path runs once, on rank 0; other ranks have no work
        if rank == 0:
            print(json.dumps(run_reference(a, rank, world, local)), flush=True)
        return 0
    if world > 1:
        import datetime

        import torch

        torch.cuda.set_device(local)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    out = run_ours(a, rank, world, local)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch

        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
