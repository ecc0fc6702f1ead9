#!/usr/bin/env python
"""bench.py -- throughput of the periodic pair-count step on B200.

Workload (one "step"): the 2-point periodic-box step of the clustering
pipeline -- DD, RR and DR for both the isotropic and the anisotropic
(|dz|, r_perp) histograms -- on N=32768 Neyman-Scott clustered data (512
parents x 64 Gaussian children, sigma 5, wrapped) plus 32768 uniform
randoms in a box of side 250, weights U(0.5, 1.5), 30 bins per axis,
dmax = 80.  The step grids both catalogs on the device (counting sort) and
runs the six histograms through the library's C ABI.  Before the timed
region the bench picks the step's partition count, whether each catalog
pair's isotropic and anisotropic histograms come from one pass over the
candidate pairs (kind "both") or two, and per histogram class the
privatisation scheme (the library's autotuner); statistics are off inside the
timed region (no per-call host synchronisation).

  value  pairs/s with the catalogs already in HBM (unit: one in-range
         unordered XX pair or one XY pair; the reference counts XX pairs
         twice, the unit does not)
  e2e    the same through the public API from pinned host buffers, with
         the H2D copy of the points and the D2H copy of the histograms
         (one read of all six per step) inside the timed region
  roofline  the pair kernel against the FP32 FMA peak measured in this run
         (8 FP32 flops per in-range pair); the kernel is CUDA-core bound
         (no HBM or tensor-core bound applies: inputs sit in L2)
  cpu_baseline  the reference's own CPU OpenMP engines (oracle/_ref,
         cpp/2PCF{isotropic,anisotropic}/BPC) on the same catalogs

--impl reference times those CPU engines alone (all host threads).
Multi-GPU: one process per GPU (torchrun); every rank runs the same step on
its own GPU (replicas; scaling "weak"); time = max over ranks.
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

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

WORKLOAD = {
    "workload": "2iso+2ani periodic pair counts (DD, RR, DR each): N=32768 Neyman-Scott "
                "clustered data (512x64, sigma 5) + 32768 uniform randoms, box 250, "
                "w~U(0.5,1.5) float32, 30 bins, dmax 80",
    "n_data": 32768, "n_rand": 32768, "box": 250.0, "bins": 30, "dmax": 80.0,
    "bpc": True, "histograms": ["DDiso", "RRiso", "DRiso", "DDani", "RRani", "DRani"],
}
SEED_D, SEED_R = 2001, 2002


def catalogs():
    from desi_b200 import catalog
    D = catalog.neyman_scott(WORKLOAD["n_data"], WORKLOAD["box"], seed=SEED_D, children=64,
                             sigma=5.0, weights="uniform")
    R = catalog.uniform(WORKLOAD["n_rand"], WORKLOAD["box"], seed=SEED_R, weights="uniform")
    return D, R


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def max_over_ranks(x: float, world: int, device=None) -> float:
    """Largest value of x over all ranks (the step time of the slowest GPU)."""
    if world <= 1:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(world: int, units_per_step: float, steps: int, max_total_ms: float) -> float:
    """Whole-job rate: every rank processed units_per_step per step."""
    return world * units_per_step * steps / (max_total_ms * 1e-3)


def tune_step(ctx, D, R, candidates=(8, 9, 10, 11, 12, 13, 14, 16)):
    """Untimed: the partition count of the step (one for all six histograms,
    so the grids are built once per step), whether the isotropic and
    anisotropic histograms of a catalog pair come from one pass (kind
    "both") or two, and per histogram class the privatisation scheme (the
    library's autotuner).  Returns (P, fused, schemes)."""
    W = WORKLOAD
    best = None
    for P in candidates:
        gd, gr = ctx.grid(D, W["box"], partitions=P), ctx.grid(R, W["box"], partitions=P)
        for fused in (False, True):
            kinds = ("both",) if fused else (False, True)
            tot, modes = 0.0, {}
            for ani in kinds:
                for name, (a, b) in (("DD", (gd, None)), ("RR", (gr, None)), ("DR", (gd, gr))):
                    r = ctx.autotune_pairs(a, b, bins=W["bins"], dmax=W["dmax"], ani=ani, bpc=True)
                    tot += r["best_ms"]
                    tag = "both" if ani == "both" else ("ani" if ani else "iso")
                    modes[name + tag] = r["hist_mode"]
            if best is None or tot < best[0]:
                best = (tot, P, fused, modes)
        gd.free()
        gr.free()
    # the tuning table keeps the last candidate's schemes: tune again at the
    # winner.  A both-kinds call tuned to the default rule (-1) runs the two
    # single-kind launches, so it needs their entries too; if every one of
    # the three chose that, the step is the single-kind form.
    _, P, fused, modes = best
    if fused and all(m < 0 for m in modes.values()):
        fused = False
    gd, gr = ctx.grid(D, W["box"], partitions=P), ctx.grid(R, W["box"], partitions=P)
    modes = {}
    for ani in ((False, True, "both") if fused else (False, True)):
        for name, (a, b) in (("DD", (gd, None)), ("RR", (gr, None)), ("DR", (gd, gr))):
            r = ctx.autotune_pairs(a, b, bins=W["bins"], dmax=W["dmax"], ani=ani, bpc=True)
            modes[name + ("both" if ani == "both" else ("ani" if ani else "iso"))] = r["hist_mode"]
    gd.free()
    gr.free()
    return P, fused, modes


HISTS = (("DD", 0), ("RR", 1), ("DR", 2))


def step_calls(ctx, gd, gr, kinds, out_ptrs, with_stats=False):
    """The counting calls of one headline step, each histogram written to
    the device buffer out_ptrs[k] (no host synchronisation unless
    with_stats).  Returns the calls' statistics when with_stats."""
    W = WORKLOAD
    k, st = 0, []
    for ani in kinds:
        for a, b in ((gd, None), (gr, None), (gd, gr)):
            r = ctx.count_pairs(a, b, bins=W["bins"], dmax=W["dmax"], ani=ani, bpc=True,
                                stats=with_stats, out_device_ptr=out_ptrs[k])
            if with_stats:
                st.append(r[1])
            k += 1
    return st


def step_results(outs, kinds):
    """The six histograms of one step as host arrays, from the step's
    device buffers (one row per call; a both-kinds call holds the isotropic
    bins, then the anisotropic ones)."""
    W = WORKLOAD
    b1, b2 = W["bins"], W["bins"] * W["bins"]
    rows = outs.cpu().numpy()
    res = {}
    for name, k in HISTS:
        if kinds == ("both",):
            res[name + "iso"] = rows[k][:b1]
            res[name + "ani"] = rows[k][b1:b1 + b2].reshape(b1, b1)
        else:
            res[name + "iso"] = rows[k][:b1]
            res[name + "ani"] = rows[3 + k][:b2].reshape(b1, b1)
    return res


def oracle_step(D, R):
    """The checker: the six histograms of the step from the FP64 oracle
    (oracle/pcf_oracle.c), computed on the host outside any timed region."""
    import oracle
    W = WORKLOAD
    want = {}
    for ani in (False, True):
        for name, (A, B) in (("DD", (D, None)), ("RR", (R, None)), ("DR", (D, R))):
            want[name + ("ani" if ani else "iso")] = oracle.pairs(
                A, B, box=W["box"], bins=W["bins"], dmax=W["dmax"], ani=ani, bpc=True)
    return want


def mismatches(got, want, rtol=1e-12):
    """Bins per histogram that differ from the oracle: unit weights
    exactly, weighted sums by more than rtol relative (a single pair binned
    differently moves a bin by ~1 in ~1e5, far above rtol)."""
    out = {}
    for k, w in want.items():
        g = np.asarray(got[k], np.float64).reshape(w.shape)
        out[k] = int((np.abs(g - w) > rtol * np.abs(w)).sum())
    return out


def run_ours(args, rank, world, local_rank):
    import torch
    from desi_b200 import api

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    W = WORKLOAD
    D, R = catalogs()
    ctx = api.Context(local_rank)
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
    if args.pair_variant:
        ctx.set_option(api.PCF_OPT_PAIR_VARIANT, args.pair_variant)
    if not args.no_grid_defer:
        # both grids of a step are queued before either is completed, so the
        # host work of one build overlaps the other build on the device
        ctx.set_option(api.PCF_OPT_GRID_DEFER, 1)
    P, fused, tuned = tune_step(ctx, D, R)
    kinds = ("both",) if fused else (False, True)
    # a both-kinds call tuned to the library's default rule (-1) runs as two
    # single-kind launches when the isotropic histogram alone gets
    # lane-private copies (this workload's 30 exact-weight bins)
    one_pass = [k[:2] for k, m in tuned.items() if k.endswith("both") and m >= 0]
    Dt = torch.from_numpy(D).to(dev)
    Rt = torch.from_numpy(R).to(dev)
    outs = torch.zeros((6, W["bins"] + W["bins"] * W["bins"]), dtype=torch.float64, device=dev)
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    # pinned host copies for the end-to-end path
    Dh = torch.from_numpy(D).pin_memory()
    Rh = torch.from_numpy(R).pin_memory()
    torch.cuda.synchronize()

    out_ptrs = [outs[k].data_ptr() for k in range(6)]

    def step_device(collect, with_stats=False):
        # asynchronous: histograms stay in HBM, no per-call host sync
        gd = ctx.grid(None, W["box"], partitions=P, device_ptr=Dt.data_ptr(), n=len(D))
        gr = ctx.grid(None, W["box"], partitions=P, device_ptr=Rt.data_ptr(), n=len(R))
        collect.extend(step_calls(ctx, gd, gr, kinds, out_ptrs, with_stats))
        gd.free()
        gr.free()

    # end to end: points from pinned host memory, histograms into device
    # buffers, one D2H read of all six per step (the public API's
    # device-output form; a per-call host result would wait on every call)
    nbk = (W["bins"] + W["bins"] * W["bins"]) if fused else None
    sizes = [nbk] * 3 if fused else [W["bins"]] * 3 + [W["bins"] * W["bins"]] * 3
    offs = np.concatenate([[0], np.cumsum(sizes)]).astype(int)
    e_out = torch.zeros(int(offs[-1]), dtype=torch.float64, device=dev)
    e_host = torch.zeros(int(offs[-1]), dtype=torch.float64).pin_memory()

    def step_e2e(collect):
        gd = ctx.grid(Dh.numpy(), W["box"], partitions=P)
        gr = ctx.grid(Rh.numpy(), W["box"], partitions=P)
        k = 0
        for ani in kinds:
            for a, b in ((gd, None), (gr, None), (gd, gr)):
                ctx.count_pairs(a, b, bins=W["bins"], dmax=W["dmax"], ani=ani, bpc=True,
                                out_device_ptr=e_out[int(offs[k]):].data_ptr())
                k += 1
        stream.synchronize()
        e_host.copy_(e_out)  # blocking read of this step's histograms
        gd.free()
        gr.free()
        return e_host

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn([])
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        times, stats = [], []
        launches0 = ctx.launches
        ctx.profile(True)
        sampler = ClockSampler(local_rank)
        sampler.start()
        torch.cuda.nvtx.range_push("timed")  # lets ncu --nvtx-include "timed/" skip the tuning
        for _ in range(steps):
            flush.zero_()  # L2 flush between steps (outside the timed region)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn(stats)
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        torch.cuda.nvtx.range_pop()
        clocks = sampler.stop()
        kprof = ctx.profile_read()
        ctx.profile(False)
        torch.cuda.synchronize()
        launches = ctx.launches - launches0
        if world > 1:
            torch.distributed.barrier()
        return times, stats, clocks, launches, kprof

    # pairs per step (deterministic): one untimed pass with counters
    probe = []
    step_device(probe, with_stats=True)
    times, _, clocks, launches, kprof = timed(step_device, args.steps, args.warmup)
    tot_ms = max_over_ranks(sum(times), world, dev)
    # parity of the last timed step's histograms against the FP64 oracle
    # (host, after the timed region)
    ctx.synchronize()
    got = step_results(outs, kinds)
    pairs_step = sum(s["pairs"] for s in probe)
    value = replica_throughput(world, pairs_step, args.steps, tot_ms)

    # end to end through the public API from pinned host buffers
    e_times, e_stats, e_clocks, _, _ = timed(step_e2e, args.steps, max(1, args.warmup // 2))
    e_tot = max_over_ranks(sum(e_times), world, dev)
    e2e_value = replica_throughput(world, pairs_step, args.steps, e_tot)
    h2d = (len(D) + len(R)) * 16
    d2h = int(e_host.numel()) * 8

    # roofline of the pair kernel: 8 FP32 flops per in-range pair
    k_ms, n_launch = kprof  # pair-kernel launches logged over the timed region
    k_pairs = pairs_step * args.steps
    stats = probe
    fp32_peak = ctx.microbench(0)
    smem_peak = ctx.microbench(1)
    achieved = 8.0 * k_pairs / (k_ms * 1e-3) / 1e12
    traffic, inst_per_pair = None, None
    prof = os.path.join(ROOT, "profiles", "k_pairs_c2_traffic.json")
    if os.path.exists(prof):
        try:
            pj = json.load(open(prof))
            traffic = pj.get("dram_bytes_per_launch")
            inst_per_pair = pj.get("thread_inst_per_pair")
        except Exception:
            traffic = None
    roofline = {
        "bound": "fp32", "kernel": "k_pairs",
        "achieved": round(achieved, 4), "peak": round(fp32_peak, 3), "unit": "TFLOP/s",
        "frac": round(achieved / fp32_peak, 5),
        "peak_source": "FP32 FMA-loop microbenchmark of this run (not in MEASURED_PEAKS.json)",
        "traffic": traffic,
        "pairs_per_s_kernel": k_pairs / (k_ms * 1e-3),
        "pairs_bound_per_s": min(fp32_peak * 1e12 / 8.0, smem_peak * 1e9),
        "smem_atomic_gops": round(smem_peak, 1),
        "avg_launch_ms": k_ms / n_launch,
        "algorithmic_flops_per_launch": 8.0 * k_pairs / n_launch,
        "candidates_per_pair": sum(s["candidates"] for s in stats) / max(pairs_step, 1),
        "recheck_fraction": sum(s["rechecks"] for s in stats) / max(pairs_step, 1),
        "kernel_share_of_step": k_ms / tot_ms if world == 1 else None,
    }
    if inst_per_pair:
        # the second ceiling: instruction issue.  Each SM issues one warp
        # instruction per scheduler (4) per clock, 32 threads each; the
        # kernel spends inst_per_pair thread instructions per in-range pair
        # (ncu, profiles/k_pairs_c2.md)
        mhz = clocks.get("sm_mhz") or 1965.0
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        ceil = sms * 4 * 32 * mhz * 1e6 / inst_per_pair
        roofline["issue_bound"] = {"thread_inst_per_pair": inst_per_pair,
                                   "ceiling_pairs_per_s": ceil, "sm_mhz": mhz,
                                   "frac": (k_pairs / (k_ms * 1e-3)) / ceil}
    out = {
        "metric": "pairs/s", "value": value, "unit": "pairs/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded Neyman-Scott data + uniform randoms; no dataset ships with "
                "the workload)",
        "config": dict(W, partitions=P, kinds_in_one_pass=one_pass, schemes=tuned,
                       pair_kernel_variant=args.pair_variant,
                       grid_builds="complete in pcf_grid_build" if args.no_grid_defer else
                       "deferred to first use (PCF_OPT_GRID_DEFER)",
                       parallelism=f"replicas x{world}",
                       l2="flushed between steps (512 MB write)",
                       pairs_per_step=pairs_step),
        "latency_ms": {"p50": statistics.median(times),
                       "p99": float(np.percentile(times, 99))},
        "e2e": {"value": e2e_value, "unit": "pairs/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": e_tot / args.steps},
        "roofline": roofline,
        "clocks": clocks,
        "gpu_launches": int(launches),
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        out["cpu_baseline"] = cpu_baseline(pairs_step)
    if not args.no_parity:
        t0 = time.perf_counter()
        mm = mismatches(got, oracle_step(D, R))
        out["mismatches"] = mm
        out["parity"] = {"checked": "the last timed step's six histograms",
                         "oracle": "FP64 restatement of the reference rules (oracle/pcf_oracle.c), "
                                   "host, outside the timed region",
                         "rtol": 1e-12, "bins_compared": int(sum(v.size for v in got.values())),
                         "mismatched_bins": int(sum(mm.values())),
                         "oracle_s": round(time.perf_counter() - t0, 2)}
    if args.iso_plain:
        out["plain_2iso"] = run_plain_2iso(ctx, torch, stream)
    if not args.no_extras:
        # the grid build, triplets, batched and served forms, measured beside
        # the headline (not the metric)
        out["grid_build"] = run_grid_build(ctx, torch)
        out["triplets"] = run_triplets(ctx, torch, stream)
        out["batched"] = run_batched(ctx, torch, stream)
        if rank == 0:
            out["served"] = run_served_isolated(args.served_requests)
    ctx.close()
    return out


# Algorithmic bytes of the grid build per point: the input point read once
# (16) and the cell-ordered copies written once: SoA planes (16), pair-packed
# blocks (16) and the integer weight (4).  The cell ids, ranks and the
# permutation (28 B per point of scratch traffic) and the O(cells) scan are
# not counted.
GRID_BYTES_PER_POINT = 16 + 16 + 16 + 4


def run_plain_2iso(ctx, torch, stream, reps=5):
    """This library's plain per-call form of the reference's `2iso -bpc` on the
    catalogs of the reference CUDA run (unit weights): DD, RR, DR as three
    calls with the library's default partition choice, device outputs, then
    one D2H read; the grids are built before the timed region, as the
    reference's host grid is built before its timer starts."""
    W = WORKLOAD
    D, R = ref_gpu_catalogs()
    dev = torch.device("cuda", ctx.device)
    out = torch.zeros(3 * W["bins"], dtype=torch.float64, device=dev)
    gd, gr = ctx.grid(D, W["box"]), ctx.grid(R, W["box"])

    def calls():
        for k, (a, b) in enumerate(((gd, None), (gr, None), (gd, gr))):
            ctx.count_pairs(a, b, bins=W["bins"], dmax=W["dmax"], bpc=True,
                            out_device_ptr=out[k * W["bins"]:].data_ptr())
        return out.cpu()

    calls()  # warm: cell structures at the call's partition count
    ms, h = _timed_ms(torch, stream, calls, reps)
    gd.free()
    gr.free()
    h = h.numpy()
    B = W["bins"]
    pairs = float(h[:B].sum()) / 2 + float(h[B:2 * B].sum()) / 2 + float(h[2 * B:].sum())
    return {"workload": "2iso -bpc (DD, RR, DR) of the bench catalogs, unit weights, three plain "
                        "calls", "ms": ms, "pairs": pairs, "pairs_per_s": pairs / (ms * 1e-3),
            "cli": run_cli_2iso(D, R)}


def run_cli_2iso(D, R):
    """This library's PCF.out on the same files and flags as the reference CUDA
    run (`2iso -bpc -f data.dat -r rand.dat -n N -b 30 -d 80 -s 250`, catalogs
    in ../data, histograms to ../results): its printed time and the whole
    process's wall time, the best of two runs."""
    import re
    import subprocess
    import tempfile
    W = WORKLOAD
    exe = os.path.join(ROOT, "desi_b200", "PCF.out")
    best = None
    with tempfile.TemporaryDirectory() as wd:
        for sub in ("data", "results", "run"):
            os.makedirs(os.path.join(wd, sub))
        for name, X in (("data.dat", D), ("rand.dat", R)):
            np.savetxt(os.path.join(wd, "data", name), X.astype(np.float64), fmt="%.9g")
        cmd = [exe, "2iso", "-bpc", "-f", "data.dat", "-r", "rand.dat", "-n", str(len(D)),
               "-b", str(W["bins"]), "-d", repr(W["dmax"]), "-s", repr(W["box"])]
        for _ in range(2):
            t0 = time.perf_counter()
            p = subprocess.run(cmd, cwd=os.path.join(wd, "run"), capture_output=True, text=True,
                               timeout=300)
            wall = time.perf_counter() - t0
            if p.returncode != 0:
                return {"error": p.stdout[-300:] + p.stderr[-300:]}
            m = re.search(r"Spent\s+([0-9.eE+-]+)\s+miliseconds", p.stdout)
            r = {"ms": float(m.group(1)) if m else None, "wall_s": wall}
            if best is None or wall < best["wall_s"]:
                best = r
    return best


def run_grid_build(ctx, torch, n=1 << 25, box=1000.0, partitions=128, reps=3):
    """The GPU counting sort on a catalog far larger than L2: n uniform
    points resident in HBM, gridded into partitions^3 cells; kernel time from
    the library's grid-build log, as HBM GB/s of algorithmic traffic."""
    dev = torch.device("cuda", ctx.device)
    g = torch.Generator(device=dev).manual_seed(9001)
    pts = torch.rand((n, 4), generator=g, device=dev, dtype=torch.float32) * box
    pts[:, 3] = 1.0
    torch.cuda.synchronize()
    ctx.grid(None, box, partitions=partitions, device_ptr=pts.data_ptr(), n=n).free()  # warm
    ctx.profile(True)
    for _ in range(reps):
        ctx.grid(None, box, partitions=partitions, device_ptr=pts.data_ptr(), n=n).free()
    ms, builds, npts = ctx.profile_read_grid()
    ctx.profile(False)
    del pts
    torch.cuda.empty_cache()
    gbs = GRID_BYTES_PER_POINT * npts / (ms * 1e-3) / 1e9
    peak, peak_source = measured_hbm_gbs()
    return {"workload": f"{n} uniform points, box {box}, {partitions}^3 cells", "builds": builds,
            "ms_per_build": ms / max(builds, 1), "bytes_per_point": GRID_BYTES_PER_POINT,
            "achieved_gbs": round(gbs, 1), "peak_gbs": peak,
            "peak_source": peak_source,
            "frac": round(gbs / peak, 4) if peak else None}


def measured_hbm_gbs():
    """(GB/s, source): the driver-measured copy bandwidth when
    MEASURED_PEAKS.json is present, else the pool's earlier copy measurement."""
    try:
        v = float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"])
        return v, "MEASURED_PEAKS.json hbm_gbs (copy, read + write)"
    except Exception:
        return 6650.0, "fallback: 6.65 TB/s, an earlier copy measurement on this pool (MEASURED_PEAKS.json absent)"


def _timed_ms(torch, stream, fn, reps=1):
    ts = []
    for _ in range(reps):
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = fn()
        e1.record(stream)
        e1.synchronize()
        ts.append(e0.elapsed_time(e1))
    return min(ts), r


def run_triplets(ctx, torch, stream, n=32768):
    """Periodic 3iso on n clustered + n uniform points (box 250, 30^3 bins,
    dmax 80, unit weights; n = 32768 in the bench line): DDD, RRR, DDR, DRR,
    and the analytic DDR/RRR path.  Unit: one unordered in-range triangle
    (XXY: one unordered XX pair with one Y point)."""
    from desi_b200 import catalog
    D = catalog.neyman_scott(n, 250.0, seed=3001, weights="unit")
    R = catalog.uniform(n, 250.0, seed=3002, weights="unit")
    gd, gr = ctx.grid(D, 250.0), ctx.grid(R, 250.0)
    kw = dict(bins=30, dmax=80.0, bpc=True, stats=True)
    res = {}

    def four():
        out = {}
        for name, a, b in (("DDD", gd, None), ("RRR", gr, None), ("DDR", gd, gr), ("DRR", gr, gd)):
            _, st = ctx.count_triplets(a, b, **kw)
            out[name] = st
        return out

    sts = four()  # warm-up and the per-histogram counters
    tri = sum(s["pairs"] for s in sts.values())
    dout = torch.zeros((4, 30 ** 3), dtype=torch.float64, device=torch.device("cuda", ctx.device))
    akw = dict(bins=30, dmax=80.0, bpc=True)

    def four_async():
        # device outputs, no host wait between calls (the plain form at its best)
        for k, (a, b) in enumerate(((gd, None), (gr, None), (gd, gr), (gr, gd))):
            ctx.count_triplets(a, b, out_device_ptr=dout[k].data_ptr(), **akw)
        ctx.synchronize()

    four_async()
    ms, _ = _timed_ms(torch, stream, four_async)
    res.update({"workload": f"3iso periodic, {n} Neyman-Scott + {n} uniform, box 250, 30^3 "
                            "bins, dmax 80, unit weights: DDD, RRR, DDR, DRR",
                "ms": ms, "triangles": tri, "value": tri / (ms * 1e-3), "unit": "triplets/s",
                "per_histogram_ms": {k: v["kernel_ms"] for k, v in sts.items()}})
    # the same four histograms as the jobs of one persistent launch
    batched = lambda: ctx.batch_triplets(gd, [gr], **kw)[1]  # noqa: E731
    batched()
    bms, bst = _timed_ms(torch, stream, batched)
    res["batched"] = {"ms": bms, "triangles": bst["pairs"], "value": bst["pairs"] / (bms * 1e-3),
                      "vs_per_call": ms / bms}
    ams, _ = _timed_ms(torch, stream, lambda: ctx.analytic_3iso(gd, bins=30, dmax=80.0,
                                                                 with_ddd=False))
    res["analytic_ddr_rrr_ms"] = ams
    gd.free()
    gr.free()
    res["random_directory"] = run_triplets_rd(ctx, torch, stream)
    return res


def run_triplets_rd(ctx, torch, stream, n_rand=8):
    """The -rd form of 3iso: one clustered data catalog (32768, box 250)
    against n_rand uniform random catalogs of log-uniform sizes 4k-32k,
    periodic, 20^3 bins, dmax 40, unit weights: DDD, RRR_i, DDR_i, DRR_i per
    call (the reference's per-file loop) vs one batched launch."""
    import math
    from desi_b200 import catalog
    rng = np.random.default_rng(3100)
    D = catalog.neyman_scott(32768, 250.0, seed=3101, weights="unit")
    sizes = [int(round(math.exp(rng.uniform(math.log(4096), math.log(32768))))) for _ in range(n_rand)]
    Rs = [catalog.uniform(s, 250.0, seed=3200 + i, weights="unit") for i, s in enumerate(sizes)]
    gd = ctx.grid(D, 250.0)
    grs = [ctx.grid(R, 250.0) for R in Rs]
    kw = dict(bins=20, dmax=40.0, bpc=True)
    calls = [(gd, None)] + [c for g in grs for c in ((g, None), (gd, g), (g, gd))]
    out = torch.zeros((len(calls), 20 ** 3), dtype=torch.float64, device=torch.device("cuda", ctx.device))

    def per_call():
        # device outputs, no host wait between calls (the plain form at its best)
        for k, (x, y) in enumerate(calls):
            ctx.count_triplets(x, y, out_device_ptr=out[k].data_ptr(), **kw)
        ctx.synchronize()

    batched = lambda: ctx.batch_triplets(gd, grs, stats=True, **kw)[1]["pairs"]  # noqa: E731
    per_call()
    btri = batched()
    pms, _ = _timed_ms(torch, stream, per_call, reps=2)
    bms, btri = _timed_ms(torch, stream, batched, reps=2)
    ptri = btri
    for g in grs:
        g.free()
    gd.free()
    return {"workload": f"1 x 32768 Neyman-Scott vs {n_rand} uniform randoms (4k-32k, log-uniform), "
                        "box 250, periodic, 20^3 bins, dmax 40: DDD + RRR/DDR/DRR per random",
            "random_sizes": sizes, "triangles": btri, "per_call_ms": pms, "batched_ms": bms,
            "per_call_triplets_per_s": ptri / (pms * 1e-3),
            "batched_triplets_per_s": btri / (bms * 1e-3), "batched_vs_per_call": pms / bms}


def run_batched(ctx, torch, stream):
    """One clustered data catalog (200k, box 1000) against 32 uniform random
    catalogs of log-uniform sizes 50k-400k, weights U(0.5,1.5), 40 bins,
    dmax 120, iso and ani: per-call loop vs one persistent launch vs the same
    launch replayed from a CUDA graph.  Unit: in-range pairs."""
    import math
    from desi_b200 import catalog
    rng = np.random.default_rng(4000)
    D = catalog.neyman_scott(200_000, 1000.0, seed=4001, weights="uniform")
    sizes = [int(round(math.exp(rng.uniform(math.log(5e4), math.log(4e5))))) for _ in range(32)]
    Rs = [catalog.uniform(n, 1000.0, seed=4100 + i, weights="uniform") for i, n in enumerate(sizes)]
    gd = ctx.grid(D, 1000.0)
    grs = [ctx.grid(R, 1000.0) for R in Rs]
    out = {"workload": "1 x 200k Neyman-Scott vs 32 uniform randoms (50k-400k, log-uniform), "
                       "box 1000, w~U(0.5,1.5), 40 bins, dmax 120, iso + ani",
           "random_sizes": sizes}
    calls = [(gd, None)] + [c for g in grs for c in ((g, None), (gd, g))]
    for ani in (False, True):
        kw = dict(bins=40, dmax=120.0, ani=ani)
        nb = 40 * 40 if ani else 40
        dbuf = torch.zeros((len(calls), nb), dtype=torch.float64, device=torch.device("cuda", ctx.device))

        def per_call():
            # device outputs, no host wait between calls (the plain form at its best)
            for k, (a, b) in enumerate(calls):
                ctx.count_pairs(a, b, out_device_ptr=dbuf[k].data_ptr(), **kw)
            ctx.synchronize()

        def batched(graph):
            return lambda: ctx.batch_pairs(gd, grs, stats=True, graph=graph, **kw)[1]["pairs"]

        per_call()
        ms_plain, _ = _timed_ms(torch, stream, per_call)
        units = batched(False)()
        batched(False)()
        ms_batch, u2 = _timed_ms(torch, stream, batched(False), reps=2)
        batched(True)()  # capture
        ms_graph, u3 = _timed_ms(torch, stream, batched(True), reps=2)
        key = "ani" if ani else "iso"
        out[key] = {"pairs": units, "plain_ms": ms_plain, "batched_ms": ms_batch,
                    "graph_ms": ms_graph, "plain_pairs_per_s": units / (ms_plain * 1e-3),
                    "batched_pairs_per_s": u2 / (ms_batch * 1e-3),
                    "graph_pairs_per_s": u3 / (ms_graph * 1e-3)}
    for g in grs:
        g.free()
    gd.free()
    return out


def run_served_isolated(n_requests=300, timeout=900):
    """run_served in a fresh process, as a request server runs in its own:
    the legs measured before it leave this process with contexts, cached
    device blocks and host threads that slowed the served form (not the plain
    one) by up to a third in earlier runs.  Both forms are measured in the
    child.  If the child fails, the leg runs here instead, and the report
    says so."""
    import subprocess
    code = ("import json, sys; sys.path.insert(0, %r); import bench; "
            "print(json.dumps(bench.run_served(%d)))" % (ROOT, int(n_requests)))
    try:
        p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                           timeout=timeout, cwd=ROOT)
        if p.returncode == 0:
            rep = json.loads(p.stdout.strip().splitlines()[-1])
            rep["process"] = "fresh process (the server's own)"
            return rep
        why = f"child exited {p.returncode}: {p.stderr.strip()[-200:]}"
    except (subprocess.TimeoutExpired, ValueError, IndexError) as e:
        why = f"child failed: {type(e).__name__}"
    rep = run_served(n_requests)
    rep["process"] = "the bench process (" + why + ")"
    return rep


def run_served(n_requests=300, load=0.7):
    """The served stream: a seeded mix of 2iso / 2ani / 3iso requests over a
    shared pool of catalog pairs (N log-uniform 1k-1M, 3iso 1k-65k; bins
    20-50; dmax 40-120; box 250/500/1000, 3iso in the 1000 box; clustered
    or uniform; periodic or not) through the continuous-batching server with
    4 slots, catalogs in page-locked host memory, grids kept resident within
    a pass (dropped before each pass).  Passes over the same requests: a
    warm-up pass (discarded); three closed-loop passes (all submitted at
    once), interleaved with three passes of the plain per-call form (the
    same requests one at a time, each submitted when the previous one
    completed and gridding its catalogs from host memory), the best of each
    kept, the closed loop's measuring capacity in requests/s; then one pass
    with Poisson arrivals at `load` times that capacity (latency p50 / p99
    over all requests).  Reported: pairs/s and triplets/s of the
    served and plain forms (same requests, same kernels)."""
    from desi_b200 import serve

    cats, _ = serve.make_stream_mixed(n_requests, rate_hz=1.0)
    srv = serve.PcfServer(slots=4)
    for k, (p, box) in cats.items():
        srv.register(k, p, box)
    del cats

    def _requests(rate_hz):
        _, reqs = serve.make_stream_mixed(n_requests, rate_hz=rate_hz or 1.0, catalogs=False)
        if rate_hz is None:
            for r in reqs:
                r.arrival = 0.0
        return reqs

    try:
        # warm-up: every request once, so each slot's memory pool and
        # page-locked buffers reach their working size (a first-use
        # cudaMalloc waits for the whole device)
        srv.drop_grids()
        srv.run_stream(_requests(None))
        # served and plain passes interleaved, so a slow spell of the host
        # (the plain form alone varies by up to ~20% between passes on a
        # shared box) falls on both forms alike; the best of each is kept
        passes, plains = [], []
        for _ in range(3):
            srv.drop_grids()
            r = srv.run_stream(_requests(None))
            r.pop("results")
            passes.append(r)
            srv.drop_grids()
            r = srv.run_serial(_requests(None))
            r.pop("results")
            plains.append(r)
        closed = min(passes, key=lambda r: r["wall_s"])
        plain = min(plains, key=lambda r: r["wall_s"])
        capacity = n_requests / closed["wall_s"]
        srv.drop_grids()
        rep = srv.run_stream(_requests(load * capacity))
        rep.pop("results")
    finally:
        srv.close()
    rep["closed_loop"] = {k: closed[k] for k in ("wall_s", "pairs_per_s", "triplets_per_s",
                                                 "overlapping_starts")}
    rep["closed_loop"]["passes_wall_s"] = [r["wall_s"] for r in passes]
    rep["closed_loop"]["passes_allocations"] = [r["allocations"] for r in passes]
    rep["plain_passes_wall_s"] = [r["wall_s"] for r in plains]
    rep["plain_passes_allocations"] = [r["allocations"] for r in plains]
    rep["plain_per_call"] = {k: plain[k] for k in ("wall_s", "pairs_per_s", "triplets_per_s",
                                                   "latency_ms")}
    rep["served_vs_plain"] = {
        "pairs_per_s": closed["pairs_per_s"] / plain["pairs_per_s"] if plain["pairs_per_s"] else None,
        "triplets_per_s": (closed["triplets_per_s"] / plain["triplets_per_s"]
                           if plain["triplets_per_s"] else None),
        "note": "best of three closed-loop served passes vs best of three passes of the same "
                "requests one at a time, the two forms interleaved"}
    rep["capacity_req_per_s"] = capacity
    rep["rate_hz"] = load * capacity
    rep["workload"] = (f"{n_requests} requests, Poisson at {load:.0%} of the closed-loop capacity; "
                       "kinds 2iso/2ani/3iso over a pool of catalog pairs (n_requests/4 per "
                       "pool); N log-uniform 1k-1M (3iso 1k-65k, box 1000); bins 20-50; "
                       "dmax 40-120; box 250/500/1000; 4 slots; resident grids reused")
    return rep


def _ref_engines():
    import oracle
    avail = oracle.available_ref_engines()
    if "2iso_bpc" in avail and "2ani_bpc" in avail:
        return oracle.RefEngine("2iso_bpc"), oracle.RefEngine("2ani_bpc")
    return None


def _cpu_step(engines, D, R, threads, unit=False):
    W = WORKLOAD
    sn = 2.176 * W["box"] / (W["n_data"] ** (1.0 / 3.0))  # the engines' own main() rule
    if unit:
        D = D.copy(); D[:, 3] = 1.0
        R = R.copy(); R[:, 3] = 1.0
    tot = 0.0
    for e in engines:
        e.set_threads(threads)
        a = e.xx(D, box=W["box"], size_node=sn, bins=W["bins"], dmax=W["dmax"])
        b = e.xx(R, box=W["box"], size_node=sn, bins=W["bins"], dmax=W["dmax"])
        c = e.xy(D, R, box=W["box"], size_node=sn, bins=W["bins"], dmax=W["dmax"])
        tot += a.sum() / 2 + b.sum() / 2 + c.sum()
    return tot


def cpu_baseline(pairs_step=None, steps=1):
    """The reference CPU engines on the full step, all host threads."""
    D, R = catalogs()
    threads = os.cpu_count() or 1
    eng = _ref_engines()
    if eng is not None:
        if pairs_step is None:
            pairs_step = _cpu_step(eng, D, R, threads, unit=True)
        t0 = time.perf_counter()
        for _ in range(steps):
            _cpu_step(eng, D, R, threads)
        dt = (time.perf_counter() - t0) / steps
        # as shipped: the engines hard-code num_threads(2) (2PCF.h:163,320)
        t0 = time.perf_counter()
        _cpu_step(eng, D, R, 2)
        dt2 = time.perf_counter() - t0
        return {"value": pairs_step / dt, "unit": "pairs/s", "cores": threads,
                "kind": "reference",
                "sample": "the full step (6 histograms, 32768+32768 points) through the "
                          "reference engines cpp/2PCF{isotropic,anisotropic}/BPC (g++ -O3 -fopenmp), "
                          f"{steps} step(s), {dt:.3f} s per step",
                "seconds_per_step": dt,
                "as_shipped_2_threads": {"value": pairs_step / dt2, "seconds_per_step": dt2},
                "triplets": cpu_triplet_baseline(threads),
                "ingest": ingest_baseline()}
    # fallback: the oracle port (brute force) on a bounded sample
    import oracle
    n = 8192
    Ds, Rs = D[:n], R[:n]
    t0 = time.perf_counter()
    cnt = 0.0
    W = WORKLOAD
    for ani in (False, True):
        for A, B in ((Ds, None), (Rs, None), (Ds, Rs)):
            oracle.pairs(A, B, box=W["box"], bins=W["bins"], dmax=W["dmax"], ani=ani, bpc=True)
    dt = time.perf_counter() - t0
    for ani in (False,):
        for A, B in ((Ds, None), (Rs, None), (Ds, Rs)):
            A1 = A.copy(); A1[:, 3] = 1
            B1 = None if B is None else B.copy()
            if B1 is not None:
                B1[:, 3] = 1
            h = oracle.pairs(A1, B1, box=W["box"], bins=W["bins"], dmax=W["dmax"], bpc=True)
            cnt += h.sum() / (2 if B is None else 1)
    return {"value": 2 * cnt / dt, "unit": "pairs/s", "cores": threads, "kind": "port",
            "sample": f"oracle brute force on the first {n} points of each catalog"}


def ingest_baseline(n=1_000_000):
    """Catalog reading: the reference's open_files (cuda/create_grid.cuh:35-78,
    one thread, ifstream >>) against this library's reader (pcf_read_catalog,
    all host threads) on the same n-row text catalog of 9-digit decimals."""
    import tempfile
    try:
        import oracle
        from desi_b200 import catalog
        rng = np.random.default_rng(77)
        v = rng.uniform(0.0, 1000.0, (n, 4)).astype(np.float32)
        v[:, 3] = rng.uniform(0.5, 1.5, n).astype(np.float32)
        with tempfile.TemporaryDirectory() as d:
            path = os.path.join(d, "catalog.dat")
            np.savetxt(path, v.astype(np.float64), fmt="%.9g")
            mb = os.path.getsize(path) / 1e6
            t0 = time.perf_counter()
            ours, _ = catalog.load(path, n)
            t_ours = time.perf_counter() - t0
            t0 = time.perf_counter()
            ref, _ = oracle.ref_read_catalog(path, n)
            t_ref = time.perf_counter() - t0
        return {"rows": n, "mb": round(mb, 1), "reference_s": t_ref, "reference_mb_per_s": mb / t_ref,
                "ours_s": t_ours, "ours_mb_per_s": mb / t_ours, "ours_threads": os.cpu_count(),
                "identical": bool(np.array_equal(ours.view(np.uint32), ref.view(np.uint32)))}
    except Exception as e:  # the reference reader is built only with the reference tree
        return {"unavailable": str(e)[:200]}


def cpu_triplet_baseline(threads, n=8192):
    """The reference's periodic 3-point CPU engine (cpp/3PCFisotropic/BPC,
    NODE3P::make_histoXXX, compiled in place) on DDD of an n-point
    Neyman-Scott catalog (box 250, 30^3 bins, dmax 80), all host threads.  The
    GPU's triplet workload has 32768 points per catalog; at fixed box the
    work grows as N^3 (N anchors x (N dmax^3/L^3)^2 neighbour pairs), 64x from
    8192 to 32768, so the full-size CPU run is not timed."""
    import oracle
    try:
        e = oracle.Ref3IsoBPC()
    except FileNotFoundError:
        return None
    from desi_b200 import catalog
    D = catalog.neyman_scott(n, 250.0, seed=3001, weights="unit")
    e.set_threads(threads)
    t0 = time.perf_counter()
    h = e.xxx(D, box=250.0, size_node=2.17 * 250.0 / n ** (1.0 / 3.0), bins=30, dmax=80.0)
    dt = time.perf_counter() - t0
    tri = float(h.sum()) / 6.0  # ordered triples -> unordered triangles
    return {"value": tri / dt, "unit": "triplets/s", "cores": threads, "kind": "reference",
            "sample": f"DDD of {n} Neyman-Scott points (box 250, 30^3 bins, dmax 80), periodic, "
                      f"{dt:.2f} s; work scales as N^3 at fixed box",
            "seconds": dt}


def ref_gpu_catalogs():
    """The bench catalogs for the side-by-side 2iso -bpc run against the
    reference's CUDA program: coordinates at least 1e-3 inside the box (its
    host grid does not clamp cell indices) and unit weights, so its
    histograms are pair counts."""
    D, R = catalogs()
    box = WORKLOAD["box"]
    out = []
    for X in (D, R):
        Y = np.array(X, dtype=np.float32, copy=True)
        Y[:, :3] = np.clip(Y[:, :3], 0.0, np.float32(box - 1e-3))
        Y[:, 3] = 1.0
        out.append(Y)
    return out


def run_reference_cuda():
    """The reference's CUDA program (cuda/main.cu, built unmodified for sm_100a
    by oracle/Makefile) on `2iso -bpc`, one random file, the bench catalogs;
    its own event timer (kernels + D2H + histogram files)."""
    import tempfile
    from oracle import ref_cuda
    if not ref_cuda.available():
        return {"unavailable": "oracle/_ref/PCF_ref_cuda.out not built"}
    D, R = ref_gpu_catalogs()
    W = WORKLOAD
    runs = []
    with tempfile.TemporaryDirectory() as wd:
        for _ in range(2):  # the first run also pays module loading on the device
            runs.append(ref_cuda.run_2iso_bpc(D, R, W["box"], W["bins"], W["dmax"], wd))
    best = min(runs, key=lambda r: r["ms"])
    pairs = float(best["DD"].sum()) / 2 + float(best["RR"].sum()) / 2 + float(best["DR"].sum())
    return {"workload": "2iso -bpc (DD, RR, DR) of the bench catalogs, unit weights, default 35 "
                        "partitions, one random file", "ms": best["ms"],
            "ms_runs": [r["ms"] for r in runs], "wall_s": min(r["wall_s"] for r in runs),
            "pairs": pairs,
            "pairs_per_s": pairs / (best["ms"] * 1e-3),
            "timer": "the program's own CUDA events around kernels, D2H copies and file writes"}


def run_reference_cuda_3iso(n=2048, bins=20, dmax=60.0, partitions=20):
    """`3iso -bpc -p 20` of the reference's CUDA program and of this
    library's PCF.out (which counts through the reference kernels' node gates
    by default) on the same files: clustered data and uniform randoms of n
    points in the 250 box, unit weights.  Both programs' own printed times,
    whether every histogram file is equal, and this library's -exact count of
    DDD beside the reference's."""
    import tempfile
    from desi_b200 import catalog
    from oracle import ref_cuda
    if not ref_cuda.available():
        return {"unavailable": "oracle/_ref/PCF_ref_cuda.out not built"}
    box = WORKLOAD["box"]
    D = ref_cuda.inside_box(catalog.neyman_scott(n, box, seed=11), box)
    R = ref_cuda.inside_box(catalog.uniform(n, box, seed=12), box)
    D[:, 3] = 1.0
    R[:, 3] = 1.0
    ours_exe = os.path.join(ROOT, "desi_b200", "PCF.out")
    runs = {}
    for who, exe, extra in (("reference", None, ()), ("ours", ours_exe, ()),
                            ("ours_exact", ours_exe, ("-exact",))):
        best = None
        for _ in range(2):  # the first run also pays module loading
            with tempfile.TemporaryDirectory() as wd:
                r = ref_cuda.run_3pt_bpc("3iso", D, R, box, bins, dmax, partitions, wd, exe=exe,
                                         extra=extra, timeout=600)
            if best is None or r["ms"] < best["ms"]:
                best = r
        runs[who] = best
    hs = ("DDD", "RRR", "DDR", "DRR")
    return {"workload": f"3iso -bpc -p {partitions}, {n} Neyman-Scott + {n} uniform, box {box:g}, "
                        f"{bins}^3 bins, dmax {dmax:g}, unit weights",
            "reference_ms": runs["reference"]["ms"], "ours_ms": runs["ours"]["ms"],
            "ours_exact_ms": runs["ours_exact"]["ms"],
            "files_equal": all(bool(np.array_equal(runs["ours"][h], runs["reference"][h])) for h in hs),
            "ddd_reference": float(runs["reference"]["DDD"].sum()),
            "ddd_exact": float(runs["ours_exact"]["DDD"].sum()),
            "timer": "each program's own printed time (kernels, copies and file writes)"}


def run_reference(args, rank, world):
    if rank != 0:
        return None
    D, R = catalogs()
    threads = os.cpu_count() or 1
    eng = _ref_engines()
    if eng is None:
        return {"impl": "reference",
                "unavailable": "oracle/_ref engines not built (needs the reference tree at "
                               "build time)"}
    pairs_step = _cpu_step(eng, D, R, threads, unit=True)
    for _ in range(args.warmup):
        _cpu_step(eng, D, R, threads)
    # timed steps: as requested, but at most ~90 s of CPU work in total
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        _cpu_step(eng, D, R, threads)
        times.append(time.perf_counter() - t0)
        if sum(times) > 90.0:
            break
    tot = sum(times)
    value = pairs_step * len(times) / tot
    extra = ({"reference_cuda": run_reference_cuda(), "reference_cuda_3iso": run_reference_cuda_3iso()}
             if args.ref_gpu else {})
    return {
        **extra,
        "impl": "reference", "metric": "pairs/s", "value": value, "unit": "pairs/s",
        "n_gpus": world, "steps": len(times), "steps_requested": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * tot / len(times), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded, same catalogs)",
        "config": dict(WORKLOAD, parallelism="reference CPU OpenMP engines"),
        "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": threads,
                         "kind": "reference",
                         "sample": "full step through cpp/2PCF{isotropic,anisotropic}/BPC "
                                   "engines (compiled in place), all host threads"},
        "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "latency_ms": {"p50": 1e3 * statistics.median(times),
                       "p99": 1e3 * float(np.percentile(times, 99))},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--pair-variant", type=int, default=0, choices=[0, 1, 2, 3],
                    help="one-pass pair kernel variant (A/B of shared-memory staging and of "
                         "pair-shared copies; include/pcf_bench.h PCF_OPT_PAIR_VARIANT)")
    ap.add_argument("--no-grid-defer", action="store_true",
                    help="complete each grid build inside pcf_grid_build (PCF_OPT_GRID_DEFER 0)")
    ap.add_argument("--served-requests", type=int, default=300,
                    help="requests of the served stream (the workload's own count: 300)")
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the check of the timed step against the FP64 oracle")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the triplet / batched / served measurements")
    ap.add_argument("--ref-gpu", action="store_true",
                    help="with --impl reference: also run the reference's CUDA program "
                         "(2iso -bpc on the bench catalogs; 3iso -bpc beside this PCF.out on "
                         "2048-point catalogs) and report its times")
    ap.add_argument("--iso-plain", action="store_true",
                    help="with --impl ours: also time this library's plain per-call 2iso -bpc "
                         "(DD, RR, DR) on the catalogs of --ref-gpu")
    ap.add_argument("--triplets-only", type=int, default=0, metavar="N",
                    help="run only the 3iso section on N + N points and print its result "
                         "(a small case for profiling; not the bench line)")
    args = ap.parse_args()
    if args.triplets_only:
        import torch
        from desi_b200 import api
        ctx = api.Context(0)
        stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", 0))
        print(json.dumps(run_triplets(ctx, torch, stream, n=args.triplets_only)))
        ctx.close()
        return
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        out = run_reference(args, rank, world)
        if out is not None:
            print(json.dumps(out))
        return
    if world > 1:
        import datetime

        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                             device_id=torch.device("cuda", local_rank))
    try:
        out = run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))


if __name__ == "__main__":
    main()
