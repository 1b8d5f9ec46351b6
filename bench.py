#!/usr/bin/env python
"""Benchmark: time-to-k-modes of the B200 normal-mode path.

Workload (default): the 100,000-atom multi-domain assembly (20 touching
globules of 5,000 atoms, seeded synthetic, 300,000 dof, cutoff 8 A, gamma 1,
PlusI 1), lowest 256 non-rigid modes at residual <= 1e-6 * ||H||.

One step = the whole hot path on the GPU from coordinates resident in HBM:
cell-list neighbours -> Cuthill-McKee -> Hessian store (FP64 + FP32) ->
rigid-body deflation basis -> block Chebyshev-filtered subspace iteration with
FP32 SpMM filtering and FP64 Rayleigh-Ritz -> final FP64 Rayleigh-Ritz and
residual certificate -> eigenpairs back in input atom order.

Also reported on the same line:
  plain_f64   the reference's algorithm (Jacobi-Davidson, FP64, single vector)
              from scratch on the same GPU, same input, same residual target
  e2e         the same metric through the public host API (numpy in, numpy out,
              host<->device copies inside the timed region)
  roofline    FP32 SpMM (the dominant kernel) achieved algorithmic GB/s
  cpu_baseline the CPU restatement of the reference path on the host cores
Multi-GPU: the path does not shard (one structure per GPU), so --gpus N runs N
independent replicas ("replicas only"); value is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "time-to-k-modes (s) at resid <=1e-6||H||"
# From the ncu capture of the 128-column FP32 pair-kernel launch on the 100k-atom
# assembly (the file under profiles/ named below holds the command and the figures).
TRAFFIC_B128_BYTES = 566_750_464
TRAFFIC_B128_RATIO = 1.200
TRAFFIC_SOURCE = "profiles/spmm_group_f32_b128_assembly100k.md"
LIMITER_FRAC = 0.868
LIMITER_SOURCE = "profiles/spmm_group_f32_b128_assembly100k.md"
UNIT = "s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="assembly100k")
    ap.add_argument("--k", type=int, default=256)
    ap.add_argument("--tol", type=float, default=1e-6)
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP64 JDM comparison")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-cert", action="store_true", help="skip the accuracy certificates (profiling aid)")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling aid)")
    ap.add_argument("--no-largest", action="store_true",
                    help="skip the single measured solve of the largest configuration (cube2400k)")
    ap.add_argument("--no-largest-plain", action="store_true",
                    help="skip the plain FP64 solve of the largest configuration")
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--kernel-only", default=None, choices=["spmm32", "spmm64"],
                    help="profiling aid: build the workload's store and run only the SpMM")
    ap.add_argument("--b", type=int, default=64, help="columns for --kernel-only")
    ap.add_argument("--reps", type=int, default=5, help="launches for --kernel-only")
    ap.add_argument("--tune", default=None, help="threads,blocks_per_sm for the wide SpMM (--kernel-only)")
    ap.add_argument("--plain-lean", action="store_true", help="cube2400k: also time the FP64 block solve")
    ap.add_argument("--degree", type=int, default=None, help="cube2400k: Chebyshev filter degree (default: the "
                    "solver's size rule)")
    ap.add_argument("--profile", action="store_true", help="cube2400k: CUDA-event phase times of the solver")
    ap.add_argument("--layout", default="groups", choices=["groups", "pairs", "tiles"],
                    help="store layout for --kernel-only (groups: the row-group layout the solvers use for FP32)")
    ap.add_argument("--traversal", type=int, default=None, choices=[0, 1, 2],
                    help="row traversal of the wide pair kernel (--kernel-only)")
    ap.add_argument("--band-panel", type=int, default=None, choices=[64, 128],
                    help="widest FP32 panel of the band-tile product (--kernel-only)")
    return ap.parse_args()


def run_kernel_only(args):
    """Builds the workload's Hessian store and issues --reps SpMM calls on a
    (3N, b) block; prints per-call CUDA-event time and algorithmic GB/s.  Used
    to profile the dominant kernel in isolation (small, self-terminating)."""
    import torch
    from inching_b200 import graph, synth
    from inching_b200.hessian import HessianStore
    from inching_b200 import _native
    if args.tune or args.traversal is not None:
        t, bps = (int(x) for x in (args.tune or "256,5").split(","))
        _native.spmm_tune(t, bps, args.traversal)
    if args.band_panel:
        _native.spmm_band_tune(args.band_panel)
    Xd = torch.from_numpy(synth.workload(args.workload) / 10.0).cuda()
    order, _ = graph.cuthill_mckee(Xd, 8.0)
    prec = 32 if args.kernel_only == "spmm32" else 64
    H = HessianStore(Xd[order], 8.0, 1.0, precisions=("f32",) if prec == 32 else ("f64",),
                     tiles=args.layout == "tiles", groups=2 if args.layout == "groups" else 0)
    dt = torch.float32 if prec == 32 else torch.float64
    g = torch.Generator(device="cuda")
    g.manual_seed(0)
    X = torch.randn((H.shape[0], args.b), generator=g, dtype=torch.float64, device="cuda").to(dt).contiguous()
    Y = torch.empty_like(X)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.reps)]
    for e0, e1 in ev:
        e0.record()
        H.matmul(X, out=Y, prec=prec)
        e1.record()
    torch.cuda.synchronize()
    ms = [e0.elapsed_time(e1) for e0, e1 in ev]
    nbytes = H.store_bytes(prec, args.b) + 2 * X.numel() * X.element_size()
    best = min(ms)
    print(json.dumps({"kernel": args.kernel_only, "b": args.b, "tune": args.tune, "layout": args.layout,
                      "traversal": args.traversal,
                      "band_panel": args.band_panel, "n_atoms": H.n_atoms,
                      "nnz": H.nnz_blocks,
                      "ms": [round(m, 4) for m in ms], "algorithmic_bytes": nbytes,
                      "best_GBps": round(nbytes / best / 1e6, 1)}))


class Clocks:
    """nvidia-smi sampler running while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        import statistics
        mhz, maxmhz, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            p = [x.strip() for x in l.split(",")]
            if len(p) < 9:
                continue
            try:
                mhz.append(float(p[1]))
                maxmhz = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(mhz) if mhz else None, "sm_max_mhz": maxmhz,
                "reasons": sorted(reasons), "samples": len(mhz)}


def flush_l2(buf):
    buf.add_(1.0)


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def _autotune_choices(n_atoms):
    """The autotuner's launch choice and candidate times (ms, fastest of its runs) for
    the store of n_atoms atoms, per (precision, width class)."""
    from inching_b200 import autotune
    out = {}
    for (n, nnz, wc, prec, dev), (best, table) in autotune._cache.items():
        if n == n_atoms:
            out[f"f{prec}_b{wc}"] = {"chosen": "/".join(str(x) for x in best),
                                     "ms": {"/".join(str(x) for x in c): round(t, 4) for c, t in table.items()}}
    return out


def run_ours(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    from inching_b200 import _native, synth
    from inching_b200.hessian import SpmmProbe
    from inching_b200.pipeline import normal_modes, normal_modes_device
    from inching_b200.solvers.chfsi import chfsi

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    from inching_b200 import replicas
    barrier = replicas.barrier

    Xh = synth.workload(args.workload) / 10.0
    Xd = torch.from_numpy(Xh).cuda()
    k, tol = args.k, args.tol
    l2 = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")   # 256 MB > 126 MB L2

    def step():
        return normal_modes_device(Xd, k, solver="chfsi", precision="mixed", tol=tol, warm_start="coarse")

    for _ in range(max(args.warmup, 0)):
        step()
    torch.cuda.synchronize()
    barrier()

    # ---- timed region: device-resident inputs -------------------------------------
    times = []
    launches0 = _native.launches
    with Clocks(local) as clk, SpmmProbe(prec=32) as probe:
        barrier()
        torch.cuda.synchronize()
        for _ in range(args.steps):
            flush_l2(l2)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            evals, modes, info = step()
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1) / 1e3)
        torch.cuda.synchronize()
        barrier()
    launches = _native.launches - launches0
    t_step = replicas.max_over_ranks(sum(times) / len(times))
    sp = probe.summary()
    hbm, peak_kind = peaks()
    achieved = sp["bytes"] / (sp["ms"] / 1e3) / 1e9 if sp["ms"] > 0 else None

    # ---- accuracy and plain FP64 comparison (one GPU only; replicas skip them) -----
    eig_rel, t_f64_tight, plain, cert_jdm = None, None, None, None
    if world == 1 and not args.no_cert:
        from inching_b200 import graph
        from inching_b200.deflation import rigid_body_basis
        from inching_b200.hessian import HessianStore
        order, undo = graph.cuthill_mckee(Xd, 8.0)
        Xr = Xd[order]
        H = HessianStore(Xr, 8.0, 1.0, precisions=("f64", "f32"))
        Q = rigid_body_basis(Xr)
        t0 = time.perf_counter()
        ref_ev, ref_V, ref_info = chfsi(H, k, tol=1e-10, Q=Q, precision="f64", return_info=True)
        torch.cuda.synchronize()
        t_f64_tight = time.perf_counter() - t0
        ev = evals.double().cpu().numpy() + 1.0
        rv = ref_ev.cpu().numpy()
        eig_rel = float(np.max(np.abs(ev - rv) / np.abs(rv)))
        # independent certificate: the reference's own algorithm (single-vector
        # Jacobi-Davidson, FP64, Hotelling deflation) at residual <= 1e-9 ||H||
        from inching_b200.solvers.jdm import jdm
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        cev, _, cinfo = jdm(H, k=k, tol=1e-9 * ref_info["normH"], Q=Q, shift=10.0, maxiter=200000,
                            return_info=True)
        torch.cuda.synchronize()
        t_cert = time.perf_counter() - t0
        cv = cev.cpu().numpy()
        cert_jdm = {"solver": "JDM (reference algorithm), FP64, single-vector, residual <= 1e-9*||H||",
                    "seconds": round(t_cert, 2), "outer_iterations": cinfo["iterations"],
                    "converged": cinfo["converged"],
                    "max_eig_rel_err_ours_vs_this": float(np.max(np.abs(ev - cv) / np.abs(cv))),
                    "max_eig_rel_diff_f64_block_vs_this": float(np.max(np.abs(rv - cv) / np.abs(cv)))}
        if not args.no_plain:
            from inching_b200.solvers.jdm import jdm
            normH = info["normH"]
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            pev, pV, pinfo = jdm(H, k=k, tol=tol * normH, Q=Q, shift=10.0, maxiter=100000, return_info=True)
            torch.cuda.synchronize()
            t_jdm = time.perf_counter() - t0
            # the configuration's own pairing: the same JDM with its correction products on
            # the FP32 store (FP64 Rayleigh-Ritz, orthogonalisation and residuals)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            mev, mV, minfo = jdm(H, k=k, tol=tol * normH, Q=Q, shift=10.0, maxiter=100000, precision="mixed",
                                 return_info=True)
            torch.cuda.synchronize()
            t_jdm_mixed = time.perf_counter() - t0
            t0 = time.perf_counter()
            fev, fV, finfo = chfsi(H, k, tol=tol, Q=Q, precision="f64", return_info=True)
            torch.cuda.synchronize()
            t_f64_block = time.perf_counter() - t0
            plain = {"solver": "JDM (reference algorithm), FP64, single-vector", "seconds": round(t_jdm, 3),
                     "outer_iterations": pinfo["iterations"], "converged": pinfo["converged"],
                     "max_eig_rel_err_vs_f64_certificate": float(np.max(np.abs(pev.cpu().numpy() - rv) / rv)),
                     "f64_block_chfsi_cold_seconds": round(t_f64_block, 3),
                     "jdm_mixed": {"solver": "JDM, correction products on the FP32 store, FP64 Rayleigh-Ritz and "
                                             "orthogonalisation", "seconds": round(t_jdm_mixed, 3),
                                   "outer_iterations": minfo["iterations"], "converged": minfo["converged"],
                                   "speedup_over_f64_jdm": round(t_jdm / t_jdm_mixed, 2),
                                   "max_eig_rel_err_vs_f64_certificate":
                                       float(np.max(np.abs(mev.cpu().numpy() - rv) / rv))}}

    # ---- end to end through the public host API -----------------------------------
    # untimed warm-up in the timed loop's own pattern (the previous result is still held
    # while the next call runs, so the pinned host cache reaches its steady state)
    e2e_times = []
    if not args.no_e2e:
        ev_h, modes_h, info_h = normal_modes(Xh, k, solver="chfsi", precision="mixed", tol=tol,
                                             warm_start="coarse")
        ev_h, modes_h, info_h = normal_modes(Xh, k, solver="chfsi", precision="mixed", tol=tol,
                                             warm_start="coarse")
    for _ in range(0 if args.no_e2e else args.steps):
        flush_l2(l2)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ev_h, modes_h, info_h = normal_modes(Xh, k, solver="chfsi", precision="mixed", tol=tol,
                                             warm_start="coarse")
        e2e_times.append(time.perf_counter() - t0)
    e2e = replicas.max_over_ranks(sum(e2e_times) / len(e2e_times)) if e2e_times else None
    h2d = Xh.size * 8
    d2h = (ev_h.size * 8 + modes_h.size * 8) if e2e_times else None

    # ---- CPU baseline (rank 0, one GPU only) --------------------------------------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu and plain is not None:
        from oracle.baseline import cpu_time_to_modes
        r = cpu_time_to_modes(Xh, k, budget_s=args.cpu_budget, tol_rel=tol,
                              plain_iterations=plain["outer_iterations"])
        cpu = {"value": round(r["projected_s"], 2), "unit": UNIT, "cores": r["cores"], "kind": "port",
               "sample": (f"oracle CPU restatement: cKDTree neighbours + Cuthill-McKee + FP64 Hessian in full "
                          f"({r['preprocess_s']:.1f} s), then {r['sample_iterations']} JDM outer iterations in "
                          f"{r['solve_sample_s']:.1f} s, projected to the {plain['outer_iterations']} iterations "
                          f"the same algorithm needed on the GPU")}

    largest = None
    if world == 1 and not args.no_largest:
        # the largest configuration needs ~160 GB: release the headline's blocks first
        del evals, modes
        import gc
        gc.collect()
        torch.cuda.empty_cache()
        largest = largest_entry(args, plain=not args.no_largest_plain)

    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": round(t_step, 4), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(t_step * 1e3, 2), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 SpMM filter / f64 Rayleigh-Ritz",
        "data": "synthetic (seeded)",
        "config": {"workload": f"{args.workload}: {info['n_atoms']} atoms, {3 * info['n_atoms']} dof, "
                               f"cutoff 8 A, gamma 1, lowest {k} non-rigid modes",
                   "k": k, "solver": "block Chebyshev-filtered subspace iteration, mixed precision, "
                                     "coarse bead-model warm start",
                   "parallelism": "replicas only" if world > 1 else "1 GPU",
                   "l2": "flushed (256 MB write) between timed steps",
                   "mean_degree": round(info["mean_degree"], 2), "nnz_blocks": info["nnz_blocks"]},
        "accuracy": {"max_rel_residual": info["max_rel_residual"], "max_eig_rel_err_vs_f64_certificate": eig_rel,
                     "certificate": None if t_f64_tight is None else
                     f"FP64 block solver at residual 1e-10*||H|| ({t_f64_tight:.2f} s)",
                     "independent_certificate": cert_jdm},
        "plain_f64": plain,
        "e2e": None if e2e is None else {"value": round(e2e, 4), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                                         "d2h_bytes_per_step": int(d2h)},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1) if achieved else None, "peak": hbm,
                     "unit": "GB/s", "frac": round(achieved / hbm, 4) if achieved else None,
                     "peak_kind": peak_kind, "kernel": "FP32 SpMM on the row-group layout (k_spmm_group<2, 128, 4, 16>; pair kernels for "
                               "narrow products)",
                     "spmm_calls": sp["calls"], "spmm_ms": round(sp["ms"], 2),
                     # ncu dram__bytes_read.sum + dram__bytes_write.sum of one 128-column FP32 launch on this
                     # workload: not measured by this run, copied from the profile named in traffic_source
                     "traffic": TRAFFIC_B128_BYTES, "traffic_unit": "bytes per 128-column launch",
                     "traffic_over_algorithmic": TRAFFIC_B128_RATIO, "traffic_source": TRAFFIC_SOURCE,
                     "traffic_measured_in_this_run": False,
                     # what bounds the kernel instead of HBM, from an ncu memory capture of the same
                     # launch; not measured by this run
                     "limiter": {"unit": "L1TEX throughput (X_j gathers through L1, 11.9 % hit rate; L2 at 72 %)",
                                 "throughput_frac": LIMITER_FRAC,
                                 "source": LIMITER_SOURCE, "measured_in_this_run": False}},
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
        "gpu_launches": int(launches),
        "solver_info": {kk: info[kk] for kk in ("iterations", "n_spmm_filter", "n_rr", "block", "degree")},
        "autotune": _autotune_choices(info["n_atoms"]),
        "largest_config": largest,
    }
    print(json.dumps(line))


def run_batched(args):
    """Many-structure workload: 512 globules with sizes log-uniform over 300-20,000
    atoms (seeded), lowest 32 non-rigid modes each; one step = the whole batch.
    Under torchrun each rank solves its size-balanced share (no data-path
    collective); the time is the max over ranks, so the scaling is strong."""
    import torch
    import torch.distributed as dist
    from inching_b200 import replicas, synth
    from inching_b200.batched import sharded_batched_normal_modes
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    sizes = synth.batch_sizes(512, 300, 20000, seed=2)
    structs = [synth.globule(int(n), seed=1000 + i) / 10.0 for i, n in enumerate(sizes)]
    k = 32 if args.k == 256 else args.k
    for _ in range(args.warmup):
        sharded_batched_normal_modes(structs, k=k, tol=args.tol, precision="mixed", gather=False)
    torch.cuda.synchronize()
    replicas.barrier()
    times = []
    info = None
    with Clocks(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        for _ in range(args.steps):
            replicas.barrier()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            res, info = sharded_batched_normal_modes(structs, k=k, tol=args.tol, precision="mixed", gather=False)
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1) / 1e3)
        replicas.barrier()
    t = replicas.max_over_ranks(sum(times) / len(times))
    worst = replicas.max_over_ranks(max([b["max_rel_residual"] for b in info["buckets"]] or [0.0]))
    # the final gather of every structure's modes to rank 0 (untimed: ~1.8 GB of host arrays)
    merged, _ = sharded_batched_normal_modes(structs, k=k, tol=args.tol, precision="mixed", gather=True)
    if rank == 0:
        assert merged is not None and len(merged) == len(structs)
        print(json.dumps({"metric": "time-to-k-modes (s) for a batch of 512 structures", "value": round(t, 3),
                          "unit": "s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                          "higher_is_better": False, "scaling": "strong",
                          "structures_per_s": round(512 / t, 1), "config": {
                              "workload": f"batch512: 512 globules, {int(sizes.sum())} atoms, sizes 300-20000 "
                                          f"log-uniform, {k} lowest non-rigid modes each",
                              "parallelism": f"{world} GPU(s), size-balanced shares, no data-path collective; "
                                             "final gather of the modes to rank 0 not timed",
                              "atoms_this_rank": info["atoms"], "buckets_this_rank": len(info["buckets"])},
                          "max_rel_residual": worst, "clocks": clk.summary()}))
    if world > 1:
        dist.destroy_process_group()


def largest_solve(precision, warm, k, tol, degree=None, profile=False):
    """One solve of the largest configuration (cube2400k: ~2.4M atoms, 300 touching
    globules of 8,000, 7.2M dof) from device-resident coordinates: Cuthill-McKee,
    Hessian store, rigid-body basis, bead warm start (if warm), memory-lean block
    solver.  CUDA-event timed; returns (seconds, eigenvalues, info)."""
    import torch
    from inching_b200 import graph, synth
    from inching_b200.deflation import rigid_body_basis
    from inching_b200.hessian import HessianStore
    from inching_b200.solvers.chfsi import chfsi_lean, default_guard
    from inching_b200.warmstart import coarse_warm_start
    Xd = torch.from_numpy(synth.workload("cube2400k") / 10.0).cuda()
    torch.cuda.synchronize()
    ev_ = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
    ev_[0].record()
    order, undo = graph.cuthill_mckee(Xd, 8.0)
    Xr = Xd[order]
    ev_[1].record()
    H = HessianStore(Xr, 8.0, 1.0, precisions=("f64", "f32") if precision == "mixed" else ("f64",))
    Q = rigid_body_basis(Xr)
    ev_[2].record()
    # all k + guard bead modes converged: with only the k wanted ones (guard left as
    # coarse Ritz vectors) the fine solve took 5 iterations and 96 s instead of 4 and 93 s
    X0 = coarse_warm_start(Xr, k + default_guard(k)) if warm else None
    ev_[3].record()
    ev, V, info = chfsi_lean(H, k, tol=tol, Q=Q, precision=precision, X0=X0, return_info=True, degree=degree,
                             profile=profile)
    del X0
    ev_[4].record()
    torch.cuda.synchronize()
    info["outer_ms"] = {nm: round(ev_[i].elapsed_time(ev_[i + 1]), 1)
                        for i, nm in enumerate(("order", "hessian", "warm_start", "solve"))}
    info["n_atoms"] = int(Xd.shape[0])
    info["nnz_blocks"] = H.nnz_blocks
    del V, H, Q, Xr, Xd
    torch.cuda.empty_cache()
    return ev_[0].elapsed_time(ev_[4]) / 1e3, ev.cpu(), info


def largest_entry(args, plain=True):
    """The largest configuration measured once in this run (mixed precision + bead
    warm start), and the same block algorithm in plain FP64 from a random start on
    the same GPU, with the eigenvalue agreement between them."""
    import numpy as np
    import torch
    k = 1000
    torch.cuda.reset_peak_memory_stats()
    with Clocks(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        t, ev, info = largest_solve("mixed", True, k, args.tol, degree=args.degree, profile=True)
    out = {"workload": "cube2400k: 2,400,000 atoms (300 touching globules of 8,000 in a cube), 7.2M dof, "
                       f"cutoff 8 A, gamma 1, lowest {k} non-rigid modes, residual <= {args.tol:g}*||H||",
           "solver": "memory-lean block Chebyshev-filtered subspace iteration, FP32 SpMM filter, FP64 "
                     "Rayleigh-Ritz, bead-model warm start",
           "seconds": round(t, 2), "timing": "one solve, CUDA events, coordinates resident in HBM",
           "steps": 1, "max_rel_residual": info["max_rel_residual"], "iterations": info["iterations"],
           "degree": info["degree"], "nnz_blocks": info["nnz_blocks"], "phases_ms": info.get("phases_ms"),
           "outer_ms": info.get("outer_ms"), "peak_mem_gb": round(torch.cuda.max_memory_allocated() / 1e9, 1),
           "clocks": clk.summary()}
    if plain:
        with Clocks(int(os.environ.get("LOCAL_RANK", "0"))) as clk2:
            tp, evp, infop = largest_solve("f64", False, k, args.tol)
        a, b = ev.double().numpy(), evp.double().numpy()
        out["plain_f64"] = {"solver": "the same block algorithm in FP64 (FP64 SpMM filter), random start",
                            "seconds": round(tp, 2), "iterations": infop["iterations"],
                            "max_rel_residual": infop["max_rel_residual"],
                            "speedup_mixed_warm_over_plain_f64": round(tp / t, 2),
                            "max_eig_rel_diff_vs_mixed": float(np.max(np.abs(a - b) / np.abs(b))),
                            "clocks": clk2.summary()}
    return out


def run_largest(args):
    """The largest configuration alone: one mixed + warm solve (and with --plain-lean
    the FP64 comparison), printed as its own line."""
    k = 1000 if args.k == 256 else args.k
    with Clocks(0) as clk:
        t, ev, info = largest_solve("mixed", True, k, args.tol, degree=args.degree, profile=args.profile)
    import torch
    line = {"metric": METRIC, "value": round(t, 2), "unit": "s", "n_gpus": 1,
            "steps": 1, "warmup": 0, "higher_is_better": False,
            "config": {"workload": "cube2400k: 2,400,000 atoms (300 touching globules of 8,000), 7.2M dof, "
                                   f"lowest {k} non-rigid modes", "solver": "memory-lean block ChFSI, mixed + warm"},
            "max_rel_residual": info["max_rel_residual"], "iterations": info["iterations"], "degree": info["degree"],
            "phases_ms": info.get("phases_ms"), "outer_ms": info.get("outer_ms"),
            "peak_mem_gb": round(torch.cuda.max_memory_allocated() / 1e9, 1), "clocks": clk.summary()}
    if args.plain_lean:
        tp, evp, infop = largest_solve("f64", False, k, args.tol)
        line["plain_f64_block"] = {"seconds": round(tp, 2), "iterations": infop["iterations"],
                                   "max_rel_residual": infop["max_rel_residual"]}
    print(json.dumps(line))


def run_shell(args):
    """Warm-start comparison on the shell workload: 60 subunits of ~8,300 atoms on a
    250 A sphere (498,000 atoms, 1.49M dof), lowest 1,000 non-rigid modes with the
    memory-lean block solver (mixed precision), from three initial blocks: random,
    the uniform bead model, and the bead model whose spring constants the shipped
    network predicts (with its residual test).  Each start is one CUDA-event timed
    solve including reordering, Hessian assembly and the warm start itself."""
    import torch
    from inching_b200 import graph, synth
    from inching_b200.deflation import rigid_body_basis
    from inching_b200.hessian import HessianStore
    from inching_b200.learned import WarmStartMPNN, learned_warm_start
    from inching_b200.solvers.chfsi import chfsi_lean, default_guard
    from inching_b200.warmstart import coarse_warm_start, galerkin_warm_start
    k = 1000 if args.k == 256 else args.k
    p = k + default_guard(k)
    Xd = torch.from_numpy(synth.workload("shell500k") / 10.0).cuda()
    model = WarmStartMPNN.load()

    def solve(start):
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        order, undo = graph.cuthill_mckee(Xd, 8.0)
        Xr = Xd[order]
        H = HessianStore(Xr, 8.0, 1.0, precisions=("f64", "f32"))
        Q = rigid_body_basis(Xr)
        winfo = None
        X0 = None
        if start == "uniform_beads":
            X0 = coarse_warm_start(Xr, p, wanted=k)
        elif start == "learned_beads":
            X0, winfo = learned_warm_start(Xr, p, model, H.rowptr, H.cols, H=H, Q=Q, k=k, return_info=True)
        elif start == "galerkin_beads":
            X0 = galerkin_warm_start(H, p)
        ev, V, info = chfsi_lean(H, k, tol=args.tol, Q=Q, precision="mixed", X0=X0, return_info=True)
        e1.record()
        torch.cuda.synchronize()
        del X0, V, H
        out = {"seconds": round(e0.elapsed_time(e1) / 1e3, 2), "iterations": info["iterations"],
               "max_rel_residual": info["max_rel_residual"], "lock_restarts": info["lock_restarts"]}
        if winfo:
            out["residual_test"] = {"fallback": winfo["fallback"],
                                    "median_ritz_residual_random": round(winfo["random_median_residual"], 3),
                                    "median_ritz_residual_learned": round(winfo.get("warm_median_residual", -1), 3)}
        return out, ev

    res = {}
    evs = {}
    with Clocks(0) as clk:
        for start in ("random", "uniform_beads", "learned_beads", "galerkin_beads"):
            res[start], evs[start] = solve(start)
            torch.cuda.empty_cache()
    agree = max(float(((evs[s] - evs["random"]).abs() / evs["random"]).max()) for s in evs)
    line = {"metric": "time-to-k-modes (s) at resid <=1e-6||H||", "value": res["learned_beads"]["seconds"],
            "unit": "s", "n_gpus": 1, "steps": 1, "warmup": 0, "higher_is_better": False,
            "config": {"workload": "shell500k: 498,000 atoms (60 subunits of 8,300 on a 250 A sphere), 1.49M dof, "
                                   f"lowest {k} non-rigid modes", "solver": "memory-lean block ChFSI, mixed precision"},
            "starts": res,
            "warm_start_gain_vs_random": round(res["random"]["seconds"] / res["learned_beads"]["seconds"], 2),
            "uniform_bead_gain_vs_random": round(res["random"]["seconds"] / res["uniform_beads"]["seconds"], 2),
            "galerkin_bead_gain_vs_random": round(res["random"]["seconds"] / res["galerkin_beads"]["seconds"], 2),
            "max_eig_rel_diff_between_starts": agree,
            "peak_mem_gb": round(torch.cuda.max_memory_allocated() / 1e9, 1), "clocks": clk.summary()}
    print(json.dumps(line))


# Outer Jacobi-Davidson iterations the reference algorithm (FP64, single vector,
# Hotelling deflation) needs for all k modes at residual <= 1e-6*||H|| on these
# workloads: counted on the B200 by the plain_f64 leg of this benchmark (the GPU run
# of the identical algorithm; 869 on assembly100k with k = 256).  The reference arm
# projects its CPU per-iteration time to this count.
PLAIN_JDM_ITERATIONS = {("assembly100k", 256): 869}


def run_reference(args):
    """Reference arm: the reference path's CPU restatement (the reference's own
    solvers need CuPy and cannot run on the CPU), timed on the host cores on the
    same workload and metric; rank 0 only.  Each step runs the preprocessing in
    full and a bounded Jacobi-Davidson sample; the step's value is the projection
    of the full solve (preprocessing + per-iteration time x the iteration count
    the identical algorithm needs), labelled as such, with the measured lower bound
    beside it."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from inching_b200 import synth
    from oracle.baseline import cpu_time_to_modes
    Xh = synth.workload(args.workload) / 10.0
    iters = PLAIN_JDM_ITERATIONS.get((args.workload, args.k))
    budget = min(args.cpu_budget, 8.0)
    for _ in range(min(args.warmup, 1)):
        cpu_time_to_modes(Xh, args.k, budget_s=1.0, tol_rel=args.tol)
    proj, low = [], []
    r = None
    for _ in range(max(args.steps, 1)):
        r = cpu_time_to_modes(Xh, args.k, budget_s=budget, tol_rel=args.tol, plain_iterations=iters)
        low.append(r["preprocess_s"] + r["solve_sample_s"])
        proj.append(r.get("projected_s", low[-1]))
    v = sum(proj) / len(proj)
    arpack = None
    if Xh.shape[0] <= 20000:
        # the reference's own CPU baseline (ARPACK on the symmetrised Hessian), feasible in
        # full only at this size
        from oracle.baseline import arpack_time_to_modes
        t_arp, _ = arpack_time_to_modes(Xh, args.k)
        arpack = {"seconds": round(t_arp, 3), "call": "scipy.sparse.linalg.eigsh(which='SA'), k + 6 modes, "
                                                      "no deflation, full solve"}
    if iters is not None:
        sample = (f"CPU restatement of the reference path: cKDTree neighbours + sequential Cuthill-McKee + FP64 "
                  f"Hessian in full ({r['preprocess_s']:.1f} s), then {r['sample_iterations']} outer JDM iterations "
                  f"in {r['solve_sample_s']:.1f} s, PROJECTED to the {iters} iterations the identical algorithm "
                  f"needs on this workload")
    else:
        sample = (f"CPU restatement: preprocessing in full + {budget:.0f} s of JDM "
                  f"({r['sample_iterations']} outer iterations); a LOWER BOUND of the full solve")
    line = {"impl": "reference", "metric": METRIC, "value": round(v, 3), "unit": UNIT, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": False,
            "config": {"workload": args.workload, "k": args.k},
            "value_kind": "projection of the full solve" if iters is not None else "lower bound",
            "measured_lower_bound_s": round(sum(low) / len(low), 3),
            "cpu_baseline": {"value": round(v, 3), "unit": UNIT, "cores": r["cores"], "kind": "port",
                             "sample": sample},
            "e2e": {"value": round(v, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if arpack is not None:
        line["arpack"] = arpack
    print(json.dumps(line))


if __name__ == "__main__":
    a = parse()
    if a.kernel_only:
        run_kernel_only(a)
    elif a.workload == "batch512" and a.impl == "ours":
        run_batched(a)
    elif a.workload == "cube2400k" and a.impl == "ours":
        run_largest(a)
    elif a.workload == "shell500k" and a.impl == "ours":
        run_shell(a)
    elif a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)
