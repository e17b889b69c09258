#!/usr/bin/env python3
"""Benchmark: served scan-to-map registration vs the plain GPU drop-in on one B200.

Workload (seeded, synthetic): 16 sensor streams in one box scene, beam mix
16/32/64/128 (16,384-262,144 rays per scan), 20 scans per stream = 320 requests,
70% CT-ICP with per-point stamps (15 iterations) / 30% rigid ICP (10 iterations).
Each stream's local map starts as 5 static prior scans and is rebuilt on the device
from the stream's last 5 registered scans (deskewed with the estimated velocities).

One step = serving the whole trace with every request arriving at t = 0 (the
saturated trace): moving-tree builds, registrations and map rebuilds, start to
drain.  Metric: alignments/s; beside it p50/p99 request latency under Poisson
arrivals at 10 Hz per stream, and the same trace through the plain drop-in (one
request at a time through kds_tree_build + kds_aligner_compute).

  value   request points resident in HBM when a step starts
  e2e     request points in page-locked host memory, copied inside the step; results
          read back to the host by the server every tick
  --impl reference   the reference's CPU path (oracle/ restatement, MODE_REF32: tree
          build + ICP_CPU_/CTICP_CPU_ with std::async chunks) on the host cores, on a
          bounded sample of the same requests (against the streams' initial maps).

Multi-GPU (torchrun): each rank serves an independent replica of the trace (the path
has no data-path exchange); value = all ranks' requests / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "ICP alignments/s + p50/p99 latency: served vs plain GPU at pose err ≤1e-5"
UNIT = "alignments/s"

TRACE_SEED = 5
STREAMS = 16
SCANS = 20
RATE_HZ = 10.0
TREE = dict(leaf_max_points=16)
ICP = dict(max_error=0.5, max_iterations=10)
CT = dict(max_error=0.5, max_iterations=15, velocity_damping=10.0)
MAP_EVERY = 5
# DRAM bytes per point of a forest build pass: dram__bytes_read.sum + dram__bytes_write.sum
# over all kernels of one ncu-captured pass of the trace's first 80 scans (bench.py
# --forest-only); a step's build traffic scales with its points.  None: not captured.
BUILD_TRAFFIC_PER_POINT = 939.0


def pose_err(A, B):
    A = np.asarray(A).reshape(3, 4)
    B = np.asarray(B).reshape(3, 4)
    dR = A[:, :3].T.astype(np.float64) @ B[:, :3].astype(np.float64)
    # angle from both the skew part (sin) and the trace (cos): arccos alone has a noise
    # floor near 3e-8 rad for identical float matrices
    w = 0.5 * np.array([dR[2, 1] - dR[1, 2], dR[0, 2] - dR[2, 0], dR[1, 0] - dR[0, 1]])
    ang = np.arctan2(np.linalg.norm(w), (np.trace(dR) - 1) / 2)
    return float(np.linalg.norm(A[:, 3].astype(np.float64) - B[:, 3])), float(ang)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 100 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            time.sleep(0.3)  # let the first sample land before the timed region
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx.append(float(p[2]))
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm)}


def max_over_ranks_of(x: float, dist, device: str) -> float:
    """The largest of the ranks' values (every rank gets it); x itself without a process group."""
    if not dist:
        return x
    import torch
    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(world: int, units_per_rank: float, max_seconds: float) -> float:
    """Whole-job throughput of independent replicas: every rank's units over the slowest rank's time."""
    return world * units_per_rank / max_seconds


def make_traces():
    """(saturated trace, Poisson trace): the same scans, guesses and request types."""
    from kd_slam2_b200 import streams
    poi = streams.make_trace(TRACE_SEED, num_streams=STREAMS, scans_per_stream=SCANS, rate_hz=RATE_HZ, threads=16)
    return streams.saturated(poi), poi


def config_block(tr):
    n = [len(r.xyz) for r in tr.requests]
    return {
        "workload": "served registration: %d streams (beams 16/32/64/128, 16k-262k rays), %d scans each "
                    "(%d requests, %d%% CT-ICP / %d%% rigid ICP), per-stream local maps rebuilt every %d scans; "
                    "saturated arrivals" % (STREAMS, SCANS, len(tr.requests),
                                            round(100 * np.mean([r.kind for r in tr.requests])),
                                            round(100 * (1 - np.mean([r.kind for r in tr.requests]))), MAP_EVERY),
        "requests": len(tr.requests), "points_total": int(np.sum(n)), "points_min": int(np.min(n)),
        "points_max": int(np.max(n)), "initial_map_points": [int(len(s.map_xyz)) for s in tr.streams],
        "tree": TREE, "icp": ICP, "ct": CT, "map_every": MAP_EVERY, "trace_seed": TRACE_SEED,
        "l2": "inputs larger than L2: %.0f MB of request points per step plus 16 resident maps" % (
            20 * np.sum(n) / 1e6),
    }


def cpu_sample(tr, max_seconds: float, threads: int, parallel_level: int = -1):
    """The reference CPU path on the requests of the first map window, against each
    stream's initial map, in trace order: per request the tree build with the reference's
    float arithmetic (StableAdder_ sums, closed-form eigen solve, swap partition, std::async
    above parallel_level; -1 = the production default) and ICP_CPU_/CTICP_CPU_ in
    MODE_REF32 with `threads` chunks.  Returns per-request build and align seconds and the
    build seconds of the maps it used (the map rebuilds of the served trace cost the same)."""
    from oracle import orc
    tp = orc.tree_params(**TREE)
    maps, map_s = {}, []
    build_s, align_s = [], []
    t_start = time.perf_counter()
    for r in tr.requests:
        if r.seq >= MAP_EVERY:
            continue
        if r.stream not in maps:
            m = tr.streams[r.stream].map_xyz
            t0 = time.perf_counter()
            maps[r.stream] = orc.OTree.build_ref32(m, np.zeros(len(m)), tp, parallel_level)
            map_s.append(time.perf_counter() - t0)
        t0 = time.perf_counter()
        T = orc.OTree.build_ref32(r.xyz, r.stamps, tp, parallel_level)
        t1 = time.perf_counter()
        if r.kind == 1:
            orc.align(orc.KIND_CT, orc.MODE_REF32, maps[r.stream], T, orc.align_params(**CT), r.X0, v0=r.v0,
                      num_threads=threads)
        else:
            orc.align(orc.KIND_ICP, orc.MODE_REF32, maps[r.stream], T, orc.align_params(**ICP), r.X0,
                      num_threads=threads)
        build_s.append(t1 - t0)
        align_s.append(time.perf_counter() - t1)
        if time.perf_counter() - t_start > max_seconds:
            break
    return {"build_s": build_s, "align_s": align_s, "map_s": map_s}


def map_rebuilds_per_request(tr) -> float:
    """Map rebuilds of the served trace per request: every stream's map is rebuilt after
    each complete window of MAP_EVERY requests except its last."""
    n = 0
    for sid in range(len(tr.streams)):
        k = sum(1 for r in tr.requests if r.stream == sid)
        n += max(0, (k + MAP_EVERY - 1) // MAP_EVERY - 1)
    return n / len(tr.requests)


def cpu_rate(smp, rebuild_rate: float) -> float:
    """Requests per second of the CPU path over a sample: each request's build + align,
    plus its share of map rebuilds at the mean measured map-build time."""
    n = len(smp["build_s"])
    t = float(np.sum(smp["build_s"]) + np.sum(smp["align_s"])) + n * rebuild_rate * float(np.mean(smp["map_s"]))
    return n / t


def cpu_baseline_leg(tr, served, threads: int) -> dict:
    """The CPU baseline leg: the reference's CPU path (the oracle's restatement of its float
    arithmetic) timed on a bounded sample of the trace, build and alignment separately,
    with the production parallel_level (-1) and the demos' (3); and the served results
    checked against the oracle (all-FP64 and the product's semantics)."""
    rr = map_rebuilds_per_request(tr)
    smp = cpu_sample(tr, 12.0, threads, -1)
    smp3 = cpu_sample(tr, 6.0, threads, 3)
    n = len(smp["build_s"])
    return {"value": cpu_rate(smp, rr), "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{n} requests of the first map window in ~12 s, in trace order: tree build with the "
                      f"reference's float arithmetic (parallel_level -1) + ICP_CPU_/CTICP_CPU_ MODE_REF32 "
                      f"with {threads} chunks, against the streams' initial maps; map rebuilds counted at "
                      f"{rr:.3f} per request (the trace's rate) x the mean measured map build",
            "build_ms_mean": 1e3 * float(np.mean(smp["build_s"])),
            "align_ms_mean": 1e3 * float(np.mean(smp["align_s"])),
            "map_build_ms_mean": 1e3 * float(np.mean(smp["map_s"])),
            "parallel_level_3": {"value": cpu_rate(smp3, rr), "requests": len(smp3["build_s"]),
                                 "build_ms_mean": 1e3 * float(np.mean(smp3["build_s"])),
                                 "map_build_ms_mean": 1e3 * float(np.mean(smp3["map_s"])),
                                 "note": "std::async for both children of every node above level 3, as the "
                                         "reference's ICP / CT-ICP demos set it"},
            "served_pose_error_vs_oracle": accuracy_sample(tr, served)}


def accuracy_sample(tr, results, count: int = 6):
    """Pose error of served results against the oracle (FP64 and the product's mixed
    semantics) for requests against the initial maps."""
    from oracle import orc
    tp = orc.tree_params(**TREE)
    out = {"t_vs_fp64_m": [], "r_vs_fp64_rad": [], "t_vs_mixed_m": [], "r_vs_mixed_rad": []}
    same = 0
    maps = {}
    for r, q in zip(tr.requests, results):
        if r.seq != 0 or len(out["t_vs_fp64_m"]) >= count or len(r.xyz) > 70000:
            continue
        if r.stream not in maps:
            m = tr.streams[r.stream].map_xyz
            maps[r.stream] = orc.OTree.build(m, np.zeros(len(m)), tp)
        T = orc.OTree.build(r.xyz, r.stamps, tp)
        kind = orc.KIND_CT if r.kind == 1 else orc.KIND_ICP
        P = orc.align_params(**(CT if r.kind == 1 else ICP))
        v0 = r.v0 if r.kind == 1 else None
        r64 = orc.align(kind, orc.MODE_FP64, maps[r.stream], T, P, r.X0, v0=v0)
        rmx = orc.align(kind, orc.MODE_MIXED, maps[r.stream], T, P, r.X0, v0=v0)
        a, b = pose_err(q["X"], r64["X"])
        c, d = pose_err(q["X"], rmx["X"])
        out["t_vs_fp64_m"].append(a)
        out["r_vs_fp64_rad"].append(b)
        out["t_vs_mixed_m"].append(c)
        out["r_vs_mixed_rad"].append(d)
        same += int(np.array_equal(np.asarray(q["X"], np.float32).ravel(), np.asarray(rmx["X"], np.float32).ravel()))
    return {k: float(np.max(v)) if v else None for k, v in out.items()} | {
        "requests": len(out["t_vs_fp64_m"]), "bit_identical_to_product_semantics_oracle": same}


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    tr, _ = make_traces()
    threads = min(os.cpu_count() or 1, 8)
    rr = map_rebuilds_per_request(tr)
    cpu_sample(tr, 2.0 * max(1, args.warmup) / 3.0, threads)  # warm-up
    step_times = []
    n_total = 0
    for _ in range(max(1, args.steps)):
        smp = cpu_sample(tr, 20.0, threads)
        n = len(smp["build_s"])
        step_times.append(n / cpu_rate(smp, rr))
        n_total += n
    val = n_total / float(np.sum(step_times))
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus,
        "steps": len(step_times), "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(step_times)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": config_block(tr),
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": "each step: up to 20 s of the trace's first-window requests in order "
                                   "(tree build with the reference's float arithmetic, parallel_level -1, + "
                                   f"ICP_CPU_/CTICP_CPU_ MODE_REF32, {threads} chunks) against the streams' "
                                   f"initial maps, plus map rebuilds at the trace's {rr:.3f} per request x the "
                                   "mean measured map build"},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def batched_ba(steps: int):
    """Batched bundle-adjustment pairs: keyframe trees in one forest pass, every pair (rigid
    and CT-ICP) in one graph-captured launch sequence with autotuned launch shape, against
    the plain per-pair kds_aligner_compute on a sample of the same pairs."""
    import torch

    import kd_slam2_b200 as kds
    from kd_slam2_b200 import ba
    wl = ba.make_workload()
    ev = lambda: torch.cuda.Event(enable_timing=True)
    e0, e1 = ev(), ev()
    dev = ba.device_inputs(wl)  # the keyframes resident on the device (untimed)
    trees = ba.build_trees(wl, TREE, inputs=dev)  # warm-up pass
    for t in trees:
        if t is not None:
            t.free()
    torch.cuda.synchronize()
    e0.record()
    trees = ba.build_trees(wl, TREE, inputs=dev)
    e1.record()
    e1.synchronize()
    build_ms = e0.elapsed_time(e1)
    jobs = ba.jobs(wl, trees, ICP, CT)
    b = kds.Batch()
    chosen, tune_ms = b.autotune(jobs)
    res = b.run(jobs)
    res = b.run(jobs)  # the second run of the shape captures the graph that the timed runs replay
    times = []
    for _ in range(max(1, steps)):
        torch.cuda.synchronize()
        e0.record()
        res = b.run(jobs)
        e1.record()
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    batch_ms = float(np.mean(times))
    # plain: one aligner call per pair, on a sample
    sample = list(range(0, len(jobs), max(1, len(jobs) // 200)))
    aligners = {0: kds.ICPB2003D(**ICP), 1: kds.CTICPB2003D(**CT)}
    same = True
    for rep in range(2):  # the first pass grows the aligners' workspaces; the second is timed
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for k in sample:
            p = wl.pairs[k]
            a = aligners[p.kind]
            a.set_fixed(trees[p.i])
            a.set_moving(trees[p.j])
            a.set_x(p.X0)
            if p.kind == 1:
                a.set_fixed_velocities(wl.keyframes[p.i].vel)
                a.set_velocities(wl.keyframes[p.j].vel)
            r = a.compute()
            same = same and r == res[k].result and np.array_equal(np.asarray(a.get_x()).reshape(12),
                                                                  np.array(res[k].X[:]))
        plain_s = (time.perf_counter() - t0) / len(sample)
    # one solver step: every factor linearized at the keyframes' estimates (rigid:
    # buildQuadraticForm, CT: buildQuadraticFormDual), then the factors' block updates
    # assembled on the device (disable_inlier_ratio 0.3, the map's default)
    fjobs, factors, nv = ba.factor_jobs(wl, trees, ICP, CT)
    fb = kds.Batch()
    fb.run(fjobs)
    fb.run(fjobs)  # the second run captures the graph
    lin_t, asm_t = [], []
    for _ in range(max(1, steps)):
        torch.cuda.synchronize()
        e0.record()
        fb.run(fjobs)
        e1.record()
        e1.synchronize()
        lin_t.append(e0.elapsed_time(e1))
        t0 = time.perf_counter()
        brc, _, _, ben = fb.assemble(factors, nv, disable_inlier_ratio=0.3)
        asm_t.append(1e3 * (time.perf_counter() - t0))
    n = [len(k.xyz) for k in wl.keyframes]
    errs = np.array([pose_err(np.array(res[k].X[:]), wl.pairs[k].X_true) for k in range(len(jobs))])
    # pose against the oracle on a sample of jobs (oracle trees from the GPU trees' exports)
    from oracle import orc
    otrees = {}

    def otree(i):
        if i not in otrees:
            e = trees[i].export()
            otrees[i] = orc.OTree.from_nodes(e["mean"], e["dir"], e["dts_mean"], e["left"], e["right"])
        return otrees[i]

    acc = {"t_vs_fp64_m": [], "r_vs_fp64_rad": [], "bit_identical_to_product_semantics_oracle": 0, "jobs": 0}
    for k in list(range(0, len(jobs), max(1, len(jobs) // 8)))[:8]:
        p = wl.pairs[k]
        kind = orc.KIND_CT if p.kind == 1 else orc.KIND_ICP
        P = orc.align_params(**(CT if p.kind == 1 else ICP))
        kw = dict(v0=wl.keyframes[p.j].vel, fixed_v=wl.keyframes[p.i].vel) if p.kind == 1 else {}
        r64 = orc.align(kind, orc.MODE_FP64, otree(p.i), otree(p.j), P, p.X0, **kw)
        rmx = orc.align(kind, orc.MODE_MIXED, otree(p.i), otree(p.j), P, p.X0, **kw)
        X = np.array(res[k].X[:]).reshape(3, 4)
        a_, b_ = pose_err(X, r64["X"])
        acc["t_vs_fp64_m"].append(a_)
        acc["r_vs_fp64_rad"].append(b_)
        acc["bit_identical_to_product_semantics_oracle"] += int(np.array_equal(X, rmx["X"]))
        acc["jobs"] += 1
    ba_pose = {"jobs": acc["jobs"], "bit_identical_to_product_semantics_oracle":
               acc["bit_identical_to_product_semantics_oracle"],
               "t_vs_fp64_m_max": float(np.max(acc["t_vs_fp64_m"])),
               "r_vs_fp64_rad_max": float(np.max(acc["r_vs_fp64_rad"])),
               "t_vs_fp64_m_median": float(np.median(acc["t_vs_fp64_m"])),
               "r_vs_fp64_rad_median": float(np.median(acc["r_vs_fp64_rad"]))}
    return {
        "workload": "200 keyframes on a 2 km loop (%d-%d points, log-uniform), %d pairs within 30 m, each "
                    "aligned rigid (10 it.) and CT-ICP (15 it.) = %d jobs" % (min(n), max(n), len(wl.pairs) // 2,
                                                                             len(jobs)),
        "keyframe_points": int(np.sum(n)), "tree_build_ms": build_ms,
        "tree_build_note": "one forest pass over all keyframes, device-resident inputs",
        "batch_ms": batch_ms,
        "alignments_per_s": len(jobs) / (batch_ms / 1e3), "plain_alignments_per_s": 1.0 / plain_s,
        "batched_over_plain": (len(jobs) / (batch_ms / 1e3)) * plain_s, "plain_sample": len(sample),
        "results_identical_to_plain": bool(same), "autotune_config": int(chosen),
        "autotune_ms": [float(x) for x in tune_ms],
        "autotune_best_ms_by_form": {name: float(np.min(tune_ms[6 * f:6 * f + 6])) for f, name in
                                     enumerate(("launch_per_iteration", "persistent", "two_tiles_per_block"))},
        "autotune_note": "config = staged tree-top nodes index (0, 1023, 2047) + 3 x (larger jobs first) + 6 x form",
        "median_t_err_vs_truth_m": float(np.median(errs[:, 0])), "median_r_err_vs_truth_rad": float(np.median(errs[:, 1])),
        "pose_vs_oracle": ba_pose,
        "factor_step": {"factors": len(factors), "variables": nv, "blocks": int(len(brc)),
                        "enabled": int(np.sum(ben)), "linearize_ms": float(np.mean(lin_t)),
                        "assemble_ms": float(np.mean(asm_t)),
                        "note": "linearize: one graph-replayed batch with results read back; assemble: "
                                "kds_batch_assemble wall time (block layout on the host, sums on the "
                                "device, blocks read back)"},
    }


def single_alignments(steps: int, peak: float, peak_source: str, cpu: bool = True):
    """The plain drop-in on the two single-alignment configurations (kd_slam2_b200/scans.py):
    rigid ICP of a 16 x 1024 scan against a second scan's tree, and CT-ICP of a skewed
    64 x 1024 scan against the 1.2M-surfel tree of 20 prior scans.  Per configuration:
    the map tree build (device-resident points), then per alignment the scan's tree build
    + compute(): with device-resident points (`value`) and with the points in page-locked
    host memory copied inside each alignment (`e2e`), CUDA events around K alignments with
    a device synchronize on both sides.  Beside them: the k_linearize roofline of one
    compute (algorithmic bytes per launch / mean launch time on the aligner's stream), the
    map build's points x levels rate, and the pose against the oracle -- bit-identity with
    the product-semantics run and the distance to the all-FP64 run.  With cpu, the
    reference CPU path (reference-arithmetic tree build + MODE_REF32 compute) on the same
    alignment, host cores."""
    import torch

    import kd_slam2_b200 as kds
    from kd_slam2_b200 import scans
    from oracle import orc
    out = {}
    ev = lambda: torch.cuda.Event(enable_timing=True)
    for name in ("rigid_16x1024", "ct_64x1024_1m_map"):
        wl = getattr(scans, name)()
        ct = wl["kind"] == "ct"
        gen = kds.TreeGeneratorB2003D(**wl["tree"])
        mx = torch.from_numpy(wl["map_xyz"]).cuda()
        M = gen.make_tree(mx, device=True)
        M.free()
        torch.cuda.synchronize()
        e0, e1 = ev(), ev()
        e0.record()
        M = gen.make_tree(mx, device=True)
        torch.cuda.synchronize()
        e1.record()
        e1.synchronize()
        map_ms = e0.elapsed_time(e1)
        sx, ss = torch.from_numpy(wl["xyz"]).cuda(), torch.from_numpy(wl["st"]).cuda()
        hx, hs = torch.from_numpy(wl["xyz"]).pin_memory(), torch.from_numpy(wl["st"]).pin_memory()
        a = kds.CTICPB2003D(**wl["params"]) if ct else kds.ICPB2003D(**wl["params"])
        a.set_fixed(M)
        X0, v0 = wl["X0s"][0], wl["v0"]

        def align(device: bool):
            T = gen.make_tree(sx, ss, device=True) if device else gen.make_tree(hx.numpy(), hs.numpy())
            a.set_moving(T)
            a.set_x(X0)
            if ct:
                a.set_velocities(v0)
            ret = a.compute()
            X = np.array(a.get_x())
            T.free()
            return ret, X

        def timed(device: bool, k: int):
            for _ in range(3):
                align(device)
            torch.cuda.synchronize()
            e0.record()
            for _ in range(k):
                ret, X = align(device)
            torch.cuda.synchronize()
            e1.record()
            e1.synchronize()
            return e0.elapsed_time(e1) / k, ret, X

        k = max(5, 4 * steps)
        ms, ret, X = timed(True, k)
        ms_e2e, ret_h, X_h = timed(False, k)
        # k_linearize roofline of one compute at the initial guess
        T = gen.make_tree(sx, ss, device=True)
        a.set_moving(T)
        a.set_x(X0)
        if ct:
            a.set_velocities(v0)
        touched = a.count_touched_nodes()
        a.set_profiling(True)
        a.compute()
        lin_ms, launches = a.profile()
        a.set_profiling(False)
        leaves = T.num_leaves
        tiles = (leaves + 127) // 128
        D = 12 if ct else 6
        part = (D * (D + 1) // 2 + D + 7) * 8 * 2
        alg = 32.0 * leaves + 32.0 * touched + part * tiles
        lin_ach = alg / (lin_ms * 1e-3) / 1e9 if lin_ms > 0 else None
        # pose against the oracle (trees bit-identical to the GPU's: the map from its export)
        me = M.export()
        Om = orc.OTree.from_nodes(me["mean"], me["dir"], me["dts_mean"], me["left"], me["right"])
        Os = orc.OTree.build(wl["xyz"], wl["st"], orc.tree_params(**wl["tree"]))
        P = orc.align_params(**wl["params"])
        kind = orc.KIND_CT if ct else orc.KIND_ICP
        rm = orc.align(kind, orc.MODE_MIXED, Om, Os, P, X0, v0=v0)
        r64 = orc.align(kind, orc.MODE_FP64, Om, Os, P, X0, v0=v0)
        npts = len(wl["xyz"])
        inf = M.info
        pl = inf.depth * len(wl["map_xyz"])
        map_alg = 48.0 * inf.global_levels * len(wl["map_xyz"]) + (
            32.0 * len(wl["map_xyz"]) if inf.global_levels < inf.depth else 0.0)
        line = {
            "scan_points": npts, "scan_leaves": int(leaves), "map_points": int(len(wl["map_xyz"])),
            "map_leaves": int(M.num_leaves), "map_depth": int(M.info.depth), "iterations": int(wl["params"]["max_iterations"]),
            "ms_per_alignment": ms, "alignments_per_s": 1e3 / ms, "points_per_s": npts * 1e3 / ms,
            "e2e": {"ms_per_alignment": ms_e2e, "alignments_per_s": 1e3 / ms_e2e,
                    "h2d_bytes": int(npts * 20), "note": "scan points and stamps from page-locked host memory"},
            "map_build_ms": map_ms, "map_build_point_levels_per_s": pl / (map_ms * 1e-3),
            "map_levels_level_by_level": int(inf.global_levels),
            "map_build_roofline": {"achieved": map_alg / (map_ms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                                   "frac": map_alg / (map_ms * 1e-3) / 1e9 / peak, "peak_source": peak_source,
                                   "model": "48 B per point per level built level by level + 32 B per point "
                                            "for the shared-memory subtree pass"},
            "roofline_linearize": {"achieved": lin_ach, "peak": peak, "unit": "GB/s",
                                   "frac": lin_ach / peak if lin_ach else None, "peak_source": peak_source,
                                   "mean_launch_ms": lin_ms, "launches": launches, "touched_fixed_nodes": int(touched),
                                   "alg_bytes_per_launch": alg},
            "result": int(ret), "results_identical_host_vs_device": bool(np.array_equal(X, X_h) and ret == ret_h),
            "bit_identical_to_product_semantics_oracle": bool(np.array_equal(X, rm["X"]) and ret == rm["ret"]),
            "pose_error_vs_fp64_oracle": {"t_m": pose_err(X, r64["X"])[0], "r_rad": pose_err(X, r64["X"])[1]},
            "pose_error_vs_truth": {"t_m": pose_err(X, wl["X_true"])[0], "r_rad": pose_err(X, wl["X_true"])[1]},
        }
        if cpu:
            threads = min(os.cpu_count() or 1, 8)
            tp = orc.tree_params(**wl["tree"])
            t0 = time.perf_counter()
            Rm = orc.OTree.build_ref32(wl["map_xyz"], None, tp, -1)
            t1 = time.perf_counter()
            Rs = orc.OTree.build_ref32(wl["xyz"], wl["st"], tp, -1)
            t2 = time.perf_counter()
            orc.align(kind, orc.MODE_REF32, Rm, Rs, P, X0, v0=v0, num_threads=threads)
            t3 = time.perf_counter()
            line["cpu_baseline"] = {"ms_per_alignment": 1e3 * (t3 - t1), "build_ms": 1e3 * (t2 - t1),
                                    "align_ms": 1e3 * (t3 - t2), "map_build_ms": 1e3 * (t1 - t0), "cores": threads,
                                    "kind": "port", "sample": "one alignment: reference-arithmetic scan tree build "
                                    "(parallel_level -1) + MODE_REF32 compute with %d chunks" % threads}
        M.free()
        out[name] = line
    return out


def _precision_worker(args):
    """One perturbation of the precision leg on the oracle: the product-semantics run (recorded),
    its FP64 replay and the free FP64 run (spawned process)."""
    path, X0, v0, params = args
    import sys
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    from oracle import orc
    g = globals()
    if g.get("_prec_path") != path:
        d = np.load(path)
        g["_prec_M"] = orc.OTree.from_nodes(d["mean"], d["dir"], d["dts_mean"], d["left"], d["right"])
        g["_prec_T"] = orc.OTree.build(d["xyz"], d["st"], orc.tree_params(**TREE))
        g["_prec_path"] = path
    P = orc.align_params(**params)
    M, T = g["_prec_M"], g["_prec_T"]
    rec = orc.align_recorded(orc.KIND_CT, M, T, P, X0, v0=v0)
    Xr, _ = orc.align_replay64(orc.KIND_CT, M, T, P, X0, rec["match"], rec["status"], v0=v0)
    r64 = orc.align(orc.KIND_CT, orc.MODE_FP64, M, T, P, X0, v0=v0)
    return rec["X"], Xr, r64["X"]


def precision_leg(steps: int, perturbations: int = 16) -> dict:
    """The precision configuration on a sample: the 128 x 2048 scan against the 4.2M-surfel map,
    seeded perturbations of 0-0.5 m / 0-5 deg aligned in one batch (CUDA events around the
    batch, device-resident trees), each pose against the oracle: bit-identity with the
    product-semantics run, the arithmetic error against the FP64 replay of the same
    correspondences, and the distance to the free all-FP64 run (branch divergence included)."""
    import multiprocessing as mp
    import tempfile

    import torch

    import kd_slam2_b200 as kds
    from kd_slam2_b200 import scans
    from kd_slam2_b200.abi import KDS_CTICP
    wl = scans.ct_128x2048_4m_map(perturbations=perturbations)
    gen = kds.TreeGeneratorB2003D(**wl["tree"])
    M = gen.make_tree(torch.from_numpy(wl["map_xyz"]).cuda(), device=True)
    T = gen.make_tree(wl["xyz"], wl["st"])
    params = kds.aligner_params(**wl["params"])
    jobs = [kds.make_job(KDS_CTICP, M, T, params, X=X0, v=wl["v0"]) for X0 in wl["X0s"]]
    b = kds.Batch()
    b.run(jobs)
    b.run(jobs)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    times = []
    for _ in range(max(1, steps)):
        torch.cuda.synchronize()
        e0.record()
        res = b.run(jobs)
        e1.record()
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    me = M.export()
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "prec.npz")
        np.savez(path, mean=me["mean"], dir=me["dir"], dts_mean=me["dts_mean"], left=me["left"], right=me["right"],
                 xyz=wl["xyz"], st=wl["st"])
        with mp.get_context("spawn").Pool(min(16, os.cpu_count() or 1)) as pool:
            ref = pool.map(_precision_worker, [(path, X0, wl["v0"], wl["params"]) for X0 in wl["X0s"]], chunksize=1)
    same, arith, fp64 = 0, [], []
    for j, (Xm, Xr, X64) in zip(res, ref):
        X = np.array(j.X[:]).reshape(3, 4)
        same += int(np.array_equal(X, Xm))
        arith.append(max(pose_err(X, Xr)))
        fp64.append(max(pose_err(X, X64)))
    arith, fp64 = np.array(arith), np.array(fp64)
    ms = float(np.median(times))
    return {"scan_points": int(len(wl["xyz"])), "scan_leaves": int(T.num_leaves), "map_points": int(len(wl["map_xyz"])),
            "map_leaves": int(M.num_leaves), "perturbations": len(jobs), "batch_ms": ms,
            "alignments_per_s": len(jobs) / (ms / 1e3),
            "bit_identical_to_product_semantics_oracle": same,
            "arithmetic_error_vs_fp64_replay": {"max": float(arith.max()), "median": float(np.median(arith)),
                                                "within_1e-5": int(np.sum(arith <= 1e-5))},
            "vs_free_fp64": {"max": float(fp64.max()), "median": float(np.median(fp64)),
                             "within_1e-5": int(np.sum(fp64 <= 1e-5))},
            "note": "errors are max(translation m, rotation rad) per perturbation"}


def scan_input(steps: int):
    """The scan input stage and the tree wire format on full-size sweeps: toPointsVector +
    Voxelizer_::voxelize on the device (kds_points_voxelize, device-resident inputs) over
    eight 128 x 2048 sweeps, and a KDTree3f round trip (kds_tree_to_msg / from_msg) of the
    tree built from one of them."""
    import torch

    import kd_slam2_b200 as kds
    from kd_slam2_b200 import synth
    boxes = synth.scene(1003)
    scans = []
    for k in range(8):
        X = synth.pose((-4.0 + k, 0.0, 1.8))
        xyz, st = synth.scan(boxes, X, beams=128, cols=2048, elev=(-22.5, 22.5), seed=7000 + k, threads=16)
        scans.append((torch.from_numpy(xyz).cuda(), torch.from_numpy(st).cuda()))
    prm = dict(range_min=1.0, range_max=100.0, space_res=0.1)
    for x, s_ in scans[:2]:
        kds.voxelize(x, s_, **prm)  # warm-up
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    times, kept = [], 0
    for _ in range(max(1, steps)):
        torch.cuda.synchronize()
        e0.record()
        kept = 0
        for x, s_ in scans:
            ox, _ = kds.voxelize(x, s_, **prm)
            kept += len(ox)
        e1.record()
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    pts = sum(len(x) for x, _ in scans)
    ms = float(np.mean(times))
    gx, gs = kds.voxelize(*scans[0], **prm)
    T = kds.TreeGeneratorB2003D(**TREE).make_tree(gx.cpu().numpy(), gs.cpu().numpy())
    t0 = time.perf_counter()
    msg = T.to_msg()
    t1 = time.perf_counter()
    U = kds.Tree.from_msg(msg)
    t2 = time.perf_counter()
    et, eu = T.export(), U.export()
    same = all(np.array_equal(et[k], eu[k]) for k in ("mean", "dir", "dts_mean", "dts_cov", "start", "end", "left",
                                                        "right", "leaves"))
    return {
        "voxelize": {"scans": len(scans), "points": int(pts), "kept_voxels": int(kept), "params": prm,
                     "ms": ms, "points_per_s": pts / (ms / 1e3),
                     "note": "kds_points_voxelize per sweep, device inputs and outputs, CUDA events around the 8 calls"},
        "tree_message": {"nodes": int(T.num_nodes), "bytes": int(msg["nodes"].nbytes), "to_msg_ms": 1e3 * (t1 - t0),
                         "from_msg_ms": 1e3 * (t2 - t1), "round_trip_identical": bool(same)},
    }


def tracker_step(frames: int = 24, cpu_frames: int = 6, cpu: bool = True):
    """The tracker step (kds_tracker_add_frame) on a 64 x 1024 sweep sequence at 10 Hz
    (2 m/s, 0.1 rad/s, in-scan motion): per frame the frame tree is built from host
    points and added to a CT-ICP + constant-velocity tracker (pre-deskew, alignment to
    the keyframe, CT morph, keyframe switch at 0.5 m).  Host-timed per frame (the call
    returns once its results are on the host).  With cpu, beside it the CPU baseline:
    the oracle's restatement of the first frames (tree build + step, the reference's
    FP32 aligner semantics) on one host core, and the largest pose difference between
    the two chains over those frames."""
    import kd_slam2_b200 as kds
    from kd_slam2_b200 import streams, synth
    boxes = synth.scene(1004)
    v = np.array([2.0, 0.1, 0.0, 0.0, 0.0, 0.1])
    P = synth.pose((0.0, 0.0, 1.8))
    M = streams.motion(v, 0.1)
    seq = []
    for k in range(frames + 2):
        xyz, st = synth.scan(boxes, P, vel=v, beams=64, cols=1024, seed=900 + k, t_start=0.1 * k, threads=16)
        seq.append((0.1 * k, xyz, st))
        P = streams.compose(P, M)
    gen = kds.TreeGeneratorB2003D(**TREE)
    kw = dict(max_kf_trans=0.5, min_inlier_frac=0.3)

    def gpu_chain(n):
        trk = kds.Tracker3D(odom_aligner=kds.CTICPB2003D(**CT), motion_model=kds.ConstVelMotionModel3D(), **kw)
        out, ms = [], []
        for ts, xyz, st in seq[:n]:
            t0 = time.perf_counter()
            r = trk.add_frame(gen.make_tree(xyz, st), ts)
            ms.append(1e3 * (time.perf_counter() - t0))
            out.append(r)
        return out, ms

    gpu_chain(2)  # warm-up
    l0 = kds.lib().kds_launch_count()
    res, ms = gpu_chain(frames)
    launches = kds.lib().kds_launch_count() - l0
    steady = ms[1:]
    line = {"frames": frames, "points_per_frame": int(np.mean([len(x) for _, x, _ in seq[:frames]])),
            "keyframes": int(res[-1]["keyframe_count"]),
            "ms_per_frame_p50": float(np.percentile(steady, 50)), "ms_per_frame_max": float(np.max(steady)),
            "frames_per_s": 1e3 / float(np.mean(steady)), "gpu_launches": int(launches),
            "note": "host-timed tree build + add_frame per frame, first frame (keyframe init) excluded"}
    line["many_streams"] = tracker_streams()
    if not cpu:
        return line
    try:
        from oracle import orc
        from oracle.tracker import OTracker
        otrk = OTracker(orc.KIND_CT, orc.align_params(**CT), const_vel=True, mode=orc.MODE_REF32, **kw)
        cms, worst = [], 0.0
        for (ts, xyz, st), rg in zip(seq[:cpu_frames], res):
            t0 = time.perf_counter()
            ro = otrk.add_frame(orc.OTree.build(xyz, st, orc.tree_params(**TREE)), ts)
            cms.append(1e3 * (time.perf_counter() - t0))
            dt, dr = pose_err(rg["pose_in_world"], np.array(ro["pose_in_world"]).reshape(3, 4))
            worst = max(worst, dt, dr)
        line["cpu_baseline"] = {"frames": cpu_frames, "ms_per_frame": float(np.mean(cms[1:])), "cores": 1,
                                "kind": "port", "max_pose_diff_vs_gpu": worst}
    except Exception as e:  # the oracle is the checker; its absence leaves the GPU numbers
        line["cpu_baseline"] = {"unavailable": str(e)[:200]}
    return line


def tracker_streams(num_streams: int = 32, frames: int = 8):
    """Many sensor streams, each with its own tracker (CT-ICP + ConstVel), one frame per
    stream per step: the frames' trees built in one forest pass (kds_tree_build_batch)
    and the steps run as one batched call (kds_tracker_add_frames: one batch of
    alignments), against the same streams stepped one at a time (kds_tree_build +
    kds_tracker_add_frame).  64 x 1024 sweeps in page-locked host memory, copied to the
    device inside each step; host-timed steps after the first (keyframe initialisation);
    the two runs' poses must be identical."""
    import torch

    import kd_slam2_b200 as kds
    from kd_slam2_b200 import streams, synth
    boxes = synth.scene(1005)
    seqs = []
    for i in range(num_streams):
        v = np.array([1.0 + 0.1 * (i % 8), 0.05, 0.0, 0.0, 0.0, 0.02 * ((i % 5) - 2)])
        P = synth.pose((-20.0 + 1.3 * i, -8.0 + 0.5 * (i % 7), 1.8), (0.0, 0.0, 0.2 * i))
        M = streams.motion(v, 0.1)
        fr = []
        for k in range(frames):
            xyz, st = synth.scan(boxes, P, vel=v, beams=64, cols=1024, seed=5000 + 37 * i + k, t_start=0.1 * k,
                                 threads=16)
            # page-locked host buffers, as a sensor driver would fill them
            fr.append((0.1 * k, torch.from_numpy(xyz).pin_memory().numpy(),
                       torch.from_numpy(st).pin_memory().numpy()))
            P = streams.compose(P, M)
        seqs.append(fr)
    gen = kds.TreeGeneratorB2003D(**TREE)
    kw = dict(max_kf_trans=0.5, min_inlier_frac=0.3)

    def trackers():
        return [kds.Tracker3D(odom_aligner=kds.CTICPB2003D(**CT), motion_model=kds.ConstVelMotionModel3D(), **kw)
                for _ in range(num_streams)]

    def one_at_a_time():
        trk, poses, ms = trackers(), [], []
        for k in range(frames):
            t0 = time.perf_counter()
            rs = [trk[i].add_frame(gen.make_tree(seqs[i][k][1], seqs[i][k][2]), seqs[i][k][0])
                  for i in range(num_streams)]
            ms.append(1e3 * (time.perf_counter() - t0))
            poses.append([r["pose_in_world"] for r in rs])
        return poses, ms

    def batched():
        trk, batch, poses, ms = trackers(), kds.Batch(), [], []
        for k in range(frames):
            t0 = time.perf_counter()
            trees = gen.make_trees([(seqs[i][k][1], seqs[i][k][2]) for i in range(num_streams)])
            rs, codes = kds.Tracker3D.add_frames(trk, trees, [seqs[i][k][0] for i in range(num_streams)], batch)
            ms.append(1e3 * (time.perf_counter() - t0))
            assert not np.any(codes)
            poses.append([r["pose_in_world"] for r in rs])
        return poses, ms

    for _ in range(3):  # warm-up (graph capture, pools, clocks)
        batched()
    l0 = kds.lib().kds_launch_count()
    with ClockSampler(torch.cuda.current_device()) as clk:
        pb, mb = batched()
    l1 = kds.lib().kds_launch_count()
    ps, msq = one_at_a_time()
    l2 = kds.lib().kds_launch_count()
    same = all(np.array_equal(a, b) for ra, rb in zip(pb, ps) for a, b in zip(ra, rb))
    fb = num_streams * (frames - 1) / (sum(mb[1:]) / 1e3)
    fs = num_streams * (frames - 1) / (sum(msq[1:]) / 1e3)
    return {"streams": num_streams, "frames": frames,
            "points_per_step": int(sum(len(seqs[i][1][1]) for i in range(num_streams))),
            "batched_frames_per_s": fb, "batched_ms_per_step": float(np.mean(mb[1:])),
            "one_at_a_time_frames_per_s": fs, "one_at_a_time_ms_per_step": float(np.mean(msq[1:])),
            "speedup": fb / fs, "identical_poses": bool(same),
            "batched_ms_all": [float(x) for x in mb], "one_at_a_time_ms_all": [float(x) for x in msq],
            "batched_clocks": clk.summary(),
            "gpu_launches": {"batched": int(l1 - l0), "one_at_a_time": int(l2 - l1)},
            "note": "host-timed steps (one frame of every stream), first step excluded"}


def served_large_maps(steps: int) -> dict:
    """The served configuration with each stream's local map at the configuration's
    ceiling: initial maps of 20 static 128 x 8192 scans (about 14.6M points, 1.2M surfels
    per stream, 16 resident), the same request mix.  Served steps (saturated, device
    inputs) after one warm-up, Poisson latency, and the same step with the admission cap
    (the bytes admitted requests may hold; resident maps are not counted) at a third of
    the uncapped peak, so that admission throttles the build passes."""
    import torch

    import kd_slam2_b200 as kds
    from kd_slam2_b200 import streams
    poi = streams.make_trace(TRACE_SEED, num_streams=STREAMS, scans_per_stream=SCANS, rate_hz=RATE_HZ,
                             map_scans=20, map_layout=(128, 8192, (-22.5, 22.5)), threads=16)
    sat = streams.saturated(poi)
    inputs = [(torch.from_numpy(r.xyz).cuda(), torch.from_numpy(r.stamps).cuda()) for r in sat.requests]

    def step(**kw):
        srv = kds.Server(tree=TREE, icp=ICP, ct=CT, map_every=MAP_EVERY, **kw)
        try:
            for st in sat.streams:
                srv.add_stream(st.map_xyz, st.max_points)
            tickets = [srv.submit(r.stream, r.kind, x, s_, r.X0, r.v0, r.arrival)
                       for r, (x, s_) in zip(sat.requests, inputs)]
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            srv.start()
            srv.drain(900.0)
            torch.cuda.synchronize()
            e1.record()
            e1.synchronize()
            res = [srv.result(t) for t in tickets]
            return e0.elapsed_time(e1), res, srv.stats()
        finally:
            srv.free()

    step()
    times = []
    for _ in range(max(1, min(steps, 3))):
        ms, res, st = step()
        times.append(ms)
    ms = float(np.median(times))
    resident = int(st["peak_reserved"])
    cap = int(resident // 3)
    ms_cap, res_cap, st_cap = step(hbm_cap=cap)
    same = all(np.array_equal(a["X"], b["X"]) for a, b in zip(res, res_cap))
    lat_srv, _, _ = streams.serve(poi, tree=TREE, icp=ICP, ct=CT, map_every=MAP_EVERY, timeout=900.0)
    lat = np.array([1e3 * (q["t_done"] - q["t_arrival"]) for q in lat_srv])
    return {"initial_map_points": [int(len(s_.map_xyz)) for s_ in sat.streams],
            "requests": len(sat.requests), "ms_per_step": ms, "alignments_per_s": len(sat.requests) / (ms / 1e3),
            "latency_ms_poisson": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
            "peak_reserved_bytes": resident, "map_rebuilds": int(st["map_builds"]),
            "capped": {"hbm_cap_bytes": cap, "ms_per_step": ms_cap,
                       "alignments_per_s": len(sat.requests) / (ms_cap / 1e3),
                       "peak_reserved_bytes": int(st_cap["peak_reserved"]), "build_passes": int(st_cap["build_passes"]),
                       "results_identical_to_uncapped": bool(same)}}


def forest_pass(steps: int, scans: int = 5) -> dict:
    """The build workload of the served step on its own: the first `scans` requests of
    every stream of the trace (80 clouds by default) built as one forest pass
    (kds_tree_build_batch, device-resident inputs), CUDA events around each pass."""
    import ctypes as C

    import torch

    import kd_slam2_b200 as kds
    from kd_slam2_b200 import abi, streams
    tr = streams.make_trace(TRACE_SEED, num_streams=STREAMS, scans_per_stream=scans, threads=16)
    clouds = [(r.xyz, r.stamps) for r in tr.requests]
    xyz = torch.from_numpy(np.ascontiguousarray(np.concatenate([c[0] for c in clouds]))).cuda()
    st = torch.from_numpy(np.ascontiguousarray(np.concatenate([c[1] for c in clouds]))).cuda()
    off = np.zeros(len(clouds) + 1, np.int64)
    off[1:] = np.cumsum([len(c[0]) for c in clouds])
    tp = kds.tree_params(**TREE)
    R = len(clouds)
    lib = kds.lib()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    times, depth_pts = [], 0
    for rep in range(3 + max(1, steps)):
        out = (C.c_void_p * R)()
        status = (C.c_int32 * R)()
        torch.cuda.synchronize()
        e0.record()
        rc = lib.kds_tree_build_batch(xyz.data_ptr(), st.data_ptr(), off.ctypes.data, R, abi.KDS_MEM_DEVICE,
                                      C.byref(tp), None, out, status)
        torch.cuda.synchronize()
        e1.record()
        e1.synchronize()
        if rc != abi.KDS_OK:
            raise RuntimeError("kds_tree_build_batch: %d" % rc)
        if rep >= 3:
            times.append(e0.elapsed_time(e1))
        depth = glob = 0
        for i in range(R):
            if out[i]:
                inf = kds.Tree(out[i]).info  # the Tree wrapper frees it
                depth, glob = max(depth, inf.depth), max(glob, inf.global_levels)
        npts = int(off[-1])
    ms = float(np.median(times))
    alg = 48.0 * glob * npts + (32.0 * npts if glob < depth else 0.0)
    return {"clouds": R, "points": npts, "levels": depth, "levels_level_by_level": glob,
            "ms_per_pass_median": ms, "ms_all": times, "point_levels_per_s": depth * npts / (ms * 1e-3),
            "alg_bytes": alg, "alg_gbs": alg / (ms * 1e-3) / 1e9}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="kds", choices=["kds", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain drop-in comparison")
    ap.add_argument("--no-ba", action="store_true", help="skip the batched bundle-adjustment section")
    ap.add_argument("--tracker-only", action="store_true",
                    help="run only the tracker-step leg and print its JSON (for profiling it)")
    ap.add_argument("--forest-only", action="store_true",
                    help="run only the served step's build workload (one forest pass of 80 scans) and print its JSON")
    ap.add_argument("--single-only", action="store_true",
                    help="run only the single-alignment legs (16 x 1024 ICP, 64 x 1024 CT-ICP vs 1.2M surfels)")
    ap.add_argument("--large-maps", action="store_true",
                    help="add the served leg with 1.2M-surfel initial maps per stream (about a minute more)")
    args = ap.parse_args()
    if args.single_only:
        import torch

        import kd_slam2_b200 as kds
        torch.cuda.set_device(0)
        kds.init(0)
        peaks = {}
        try:
            peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        except Exception:
            pass
        print(json.dumps({"single_alignments": single_alignments(
            args.steps, float(peaks.get("hbm_gbs", 6650.0)), "measured" if "hbm_gbs" in peaks else "fallback",
            cpu=not args.no_cpu)}), flush=True)
        return
    if args.forest_only:
        import torch

        import kd_slam2_b200 as kds
        torch.cuda.set_device(0)
        kds.init(0)
        print(json.dumps({"forest_pass": forest_pass(args.steps)}), flush=True)
        return
    if args.tracker_only:
        # the same device setup as the full run before its legs
        import torch

        import kd_slam2_b200 as kds
        torch.cuda.set_device(0)
        kds.init(0)
        print(json.dumps({"tracker_step": tracker_step(cpu=not args.no_cpu)}), flush=True)
        return
    if args.warmup < 3:
        args.warmup = 3

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))

    if args.impl == "reference":
        run_reference_arm(args)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    import kd_slam2_b200 as kds
    from kd_slam2_b200 import streams
    kds.init(local)
    sat, poi = make_traces()
    dev_inputs = [(torch.from_numpy(r.xyz).cuda(), torch.from_numpy(r.stamps).cuda()) for r in sat.requests]
    host_inputs = [(torch.from_numpy(r.xyz).pin_memory(), torch.from_numpy(r.stamps).pin_memory())
                   for r in sat.requests]
    torch.cuda.synchronize()

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    def serve_step(inputs, **kw):
        """One served pass over the saturated trace, timed on the device: events on the
        current stream around start..drain with a device synchronize on both sides."""
        srv = kds.Server(tree=TREE, icp=ICP, ct=CT, map_every=MAP_EVERY, **kw)
        try:
            for st in sat.streams:
                srv.add_stream(st.map_xyz, st.max_points)
            tickets = [srv.submit(r.stream, r.kind, x, s, r.X0, r.v0, r.arrival)
                       for r, (x, s) in zip(sat.requests, inputs)]
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            srv.start()
            srv.drain(600.0)
            torch.cuda.synchronize()
            e1.record()
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            res = [srv.result(t) for t in tickets]
            stats = srv.stats()
        finally:
            srv.free()
        return ms, res, stats

    def max_over_ranks(x: float) -> float:
        return max_over_ranks_of(x, dist, "cuda")

    # warm-up
    for _ in range(args.warmup):
        serve_step(dev_inputs)

    # ---- timed: device-resident inputs
    launches0 = kds.lib().kds_launch_count()
    times, stats_list = [], []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            ms, served, st = serve_step(dev_inputs)
            times.append(ms)
            stats_list.append(st)
    launches = (kds.lib().kds_launch_count() - launches0) // max(1, args.steps)
    n_req = len(sat.requests)
    total_s = max_over_ranks(float(np.sum(times)) / 1e3)
    value = replica_throughput(world, n_req * args.steps, total_s)
    # the other rates of the served step: moving surfels x Gauss-Newton iterations, and
    # scan points registered, per second (rank 0's step, one replica)
    surfel_iters = sum((q["stats"]["num_inliers"] + q["stats"]["num_outliers"] + q["stats"]["num_bad"] +
                        q["stats"]["num_err_normal"] + q["stats"]["num_err_fn"]) * q["iterations"] for q in served)
    scan_points = int(sum(len(r.xyz) for r in sat.requests))
    step_s = float(np.mean(times)) / 1e3
    rates = {"surfel_iterations_per_s": surfel_iters / step_s, "scan_points_per_s": scan_points / step_s,
             "note": "per replica: surfels = moving leaves of each registration (its last iteration's count) "
                     "x its iterations; scan points = the requests' points"}
    ms_step = float(np.mean(times))

    # ---- e2e: page-locked host inputs copied inside the step
    e2e_times, e2e_stats = [], None
    for _ in range(args.steps):
        ms, served_h, e2e_stats = serve_step(host_inputs)
        e2e_times.append(ms)
    e2e_total = max_over_ranks(float(np.sum(e2e_times)) / 1e3)
    e2e_value = replica_throughput(world, n_req * args.steps, e2e_total)
    same_host_dev = all(np.array_equal(a["X"], b["X"]) for a, b in zip(served, served_h))

    # ---- profile pass (untimed): device time and algorithmic bytes of the linearizations
    _, _, pst = serve_step(dev_inputs, profile=1)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    achieved = pst["alg_bytes"] / (pst["lin_ms"] * 1e-3) / 1e9 if pst["lin_ms"] > 0 else None
    # the dominant kernels of the step are the tree-build passes; the linearization launches second
    # per point and level built level by level: a 16 B point record read twice and written once
    # (48 B); the shared-memory subtree pass that finishes the deep levels: 28 B of point record
    # read once + 4 B of point order written (32 B per point)
    deep = pst["build_global_point_levels"] < pst["build_point_levels"]
    build_alg = 48.0 * pst["build_global_point_levels"] + (32.0 * pst["build_points"] if deep else 0.0)
    # the two build threads' passes overlap: the denominator is the time any pass ran
    build_ach = build_alg / (pst["build_busy_ms"] * 1e-3) / 1e9 if pst["build_busy_ms"] > 0 else None
    roofline = {"bound": "hbm", "kernel": "tree-build passes (k_small_part, k_decide, k_big_*, level kernels): "
                                          "forest builds of request and map trees",
                "achieved": build_ach, "peak": peak, "unit": "GB/s",
                "frac": build_ach / peak if build_ach else None,
                "traffic": BUILD_TRAFFIC_PER_POINT * pst["build_points"] if BUILD_TRAFFIC_PER_POINT else None,
                "traffic_source": "DRAM bytes per point of an ncu capture of an 80-scan forest pass (all its "
                                  "kernels), scaled by the step's points",
                "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                "alg_bytes_per_step": build_alg, "build_busy_ms_per_step": pst["build_busy_ms"],
                "build_pass_ms_summed": pst["build_ms"],
                "model": "48 B per point per level built level by level (a 16 B point record read twice and "
                         "written once) + 32 B per point for the shared-memory subtree pass of the deep levels; "
                         "summed over the step's build passes / the time any of them ran",
                "point_levels": pst["build_point_levels"],
                "point_levels_level_by_level": pst["build_global_point_levels"]}
    ticks = max(1, pst["lin_ticks"])
    roofline_lin = {"bound": "hbm", "kernel": "k_linearize<0>/<1> (fused ICP / CT-ICP linearization + GN step)",
                    "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": achieved / peak if achieved else None, "traffic": None,
                    "alg_bytes_per_tick": pst["alg_bytes"] / ticks, "lin_ms_per_tick": pst["lin_ms"] / ticks,
                    "model": "per registration iteration: 32 B x moving surfels + 32 B x distinct fixed nodes "
                             "touched + (M+7) doubles x 2 per tile partial; summed over the run / summed device "
                             "time of the linearization launches",
                    "ticks": pst["lin_ticks"], "mean_registrations_per_tick": pst["mean_active"]}

    # ---- latency under Poisson arrivals (10 Hz per stream)
    lat_srv, _, _ = streams.serve(poi, tree=TREE, icp=ICP, ct=CT, map_every=MAP_EVERY, timeout=600.0)
    lat = np.array([1e3 * (q["t_done"] - q["t_arrival"]) for q in lat_srv])
    lat_sat = np.array([1e3 * (q["t_done"] - q["t_arrival"]) for q in served])

    # ---- the plain drop-in on the same trace
    plain = None
    if not args.no_plain:
        serve_step(dev_inputs, serial=1)  # warm-up: the serial path's aligners grow their workspaces
        p_runs = [serve_step(dev_inputs, serial=1) for _ in range(max(5, args.steps))]
        p_all = [float(r[0]) for r in p_runs]
        p_ms = float(np.median(p_all))
        p_res = p_runs[-1][1]
        p_val = n_req / (p_ms / 1e3)
        same = all(np.array_equal(a["X"], b["X"]) and a["result"] == b["result"] for a, b in zip(served, p_res))
        lat_p, _, _ = streams.serve(poi, serial=True, tree=TREE, icp=ICP, ct=CT, map_every=MAP_EVERY,
                                    timeout=600.0)
        latp = np.array([1e3 * (q["t_done"] - q["t_arrival"]) for q in lat_p])
        plain = {"value": p_val, "unit": UNIT, "ms_per_step": p_ms, "ms_per_step_all": p_all,
                 "reported": "median of %d timed steps after 1 warm-up" % len(p_runs),
                 "spread": {"min_ms": float(np.min(p_all)), "max_ms": float(np.max(p_all))},
                 "served_over_plain": value / world / p_val,
                 "results_identical_to_served": bool(same),
                 "latency_ms_poisson": {"p50": float(np.percentile(latp, 50)), "p99": float(np.percentile(latp, 99))}}

    st0 = stats_list[-1]
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": config_block(sat),
        "latency_ms": {"poisson_10hz_per_stream": {"p50": float(np.percentile(lat, 50)),
                                                    "p99": float(np.percentile(lat, 99))},
                       "saturated": {"p50": float(np.percentile(lat_sat, 50)),
                                     "p99": float(np.percentile(lat_sat, 99))}},
        "plain": plain,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(e2e_stats["h2d_bytes"]),
                "d2h_bytes_per_step": int(e2e_stats["d2h_bytes"]), "results_identical_to_device_inputs":
                    bool(same_host_dev), "ms_per_step_all": [float(x) for x in e2e_times]},
        "gpu_launches": int(launches),
        "served": {"ms_per_step_all": [float(x) for x in times],
                   "ticks": st0["ticks"], "mean_registrations_per_tick": st0["mean_active"],
                   "build_passes": st0["build_passes"], "trees_built": st0["built_trees"],
                   "map_rebuilds": st0["map_builds"], "build_pass_ms": st0["build_ms"],
                   "build_points": st0["build_points"], "peak_reserved_bytes": st0["peak_reserved"],
                   "hbm_cap_bytes": st0["hbm_cap"]},
        "rates": rates,
        "roofline": roofline,
        "roofline_linearize": roofline_lin,
        "clocks": clk.summary(),
    }
    if rank == 0 and not args.no_ba:
        line["single_alignments"] = single_alignments(args.steps, peak, roofline["peak_source"],
                                                      cpu=world == 1 and not args.no_cpu)
        line["batched_ba"] = batched_ba(args.steps)
        line["precision"] = precision_leg(args.steps) if world == 1 and not args.no_cpu else None
        if args.large_maps:
            line["served_large_maps"] = served_large_maps(args.steps)
        line["scan_input"] = scan_input(args.steps)
        line["tracker_step"] = tracker_step(cpu=world == 1 and not args.no_cpu)
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = min(os.cpu_count() or 1, 8)
        line["cpu_baseline"] = cpu_baseline_leg(sat, served, threads)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
