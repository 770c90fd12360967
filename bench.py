"""Benchmark: device ms per mesh for the all-layer analytic depth peel.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config knot-65536]
                    [--impl ours|reference]

One step is one full extraction (projection through world-space triangles)
of the configured synthetic mesh, replayed from one captured CUDA graph.
Under torchrun (N > 1) every rank peels its own replica on its own GPU with no
data-path collective ("replicas only"); the only collectives are the barrier
and the max-over-ranks timing reduction.  Rank 0 prints one JSON line.

``--impl reference`` times the reference's CPU path for the same workload:
the C++ restatement of its fast-bvh-peel (oracle/fast_peel.cpp), all host
threads, on rank 0 only.
"""

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "exact-depth-peeling_b200"))

METRIC = "device ms/mesh for all-layer peel at 64K & 720K faces, ranks exact vs oracle"
UNIT = "ms/mesh"
PEAKS = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0
REFERENCE_BUDGET_S = 60.0  # CPU seconds of timed extractions in the reference arm
DEFAULT_FORM = "filtered64"  # the predicate form of EventPeeler's default


DESCRIPTIONS = {
    "knot-65536": "(3,7) torus-knot tube, 256 rings x 128 segments = 65,536 faces, radius "
                  "0.3 with N(0,0.02) noise (seed 2), pinhole 60 deg at 3x bounding radius",
    "icospheres-2560": "two nested noisy icospheres, 2 x 1,280 faces, orthographic",
    "stack-65536": "65,536 identical-footprint triangles at z = i*1e-3, orthographic",
    "primitives-720k": "40 noisy spheres and tori (radii log-uniform in [0.05, 0.5], seed 7) "
                       "packed disjointly, 720,916 faces, pinhole 60 deg",
    "overlap-720k": "40 noisy spheres and tori (radii log-uniform in [0.05, 0.5], seed 7) "
                    "with centres uniform in the unit box, overlapping, 720,916 faces, "
                    "resolved exactly (peel_b200.resolve) into 1,218,926 faces; pinhole 60 deg",
    "batched-128": "one graph replay of 128 extractions: 64 turntable pinhole views "
                   "(seed 5) of a 16,152-face displaced genus-3 surface plus 64 packed-"
                   "primitive meshes of 1K-32K faces (seed 6)",
}


def workload_config(name, vertices, faces):
    return {"workload": f"{name}: {DESCRIPTIONS.get(name, name)}", "faces": int(len(faces)),
            "vertices": int(len(vertices)),
            "l2": "flushed between timed replays (256 MiB device write)",
            "parallelism": "replicas"}


def algorithmic_bytes(nv, nf, triangles):
    """Compulsory bytes of one mesh: inputs (vertices, faces, camera, settings)
    plus outputs (uv 3x2 f64, world 3x3 f64, source and layer i32 per triangle)."""
    return 24 * nv + 12 * nf + 128 + 48 + 128 * triangles


class ClockSampler:
    """nvidia-smi SM clock / throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, ValueError):
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
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() in ("active", "1"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm)}


def max_over_ranks(value, world, device):
    """The largest of every rank's `value` (a time), through the process
    group (NCCL on GPUs, gloo on CPUs); `value` itself on one rank."""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_ms_per_mesh(max_total_ms, steps, world):
    """Replicas: every rank peels `steps` meshes in the slowest rank's time."""
    return max_total_ms / (steps * world)


def hbm_peak():
    try:
        return float(json.loads(PEAKS.read_text())["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic(config, kernel="k_mesh_polygons"):
    """DRAM bytes (read + write) of one noding stage on this workload (the
    launch of `kernel` plus that of k_mesh_heavy after it), as recorded from an
    ncu capture in profiles/<kernel>_<config>.md, or None."""
    path = ROOT / "profiles" / f"{kernel}_{config}.md"
    try:
        for line in path.read_text().splitlines():
            if line.startswith("| dram bytes per launch |"):
                return int(line.split("|")[2].strip())
    except (OSError, ValueError):
        pass
    return None


# Meshes whose full CPU extraction takes minutes: the CPU legs time the first
# layers only (fast-bvh-peel peels front to back), a lower bound of the full
# extraction's time, so the CPU figure favours the CPU.
CPU_LAYER_SAMPLE = {"overlap-720k": 4}


def cpu_sample_text(config, info):
    cap = CPU_LAYER_SAMPLE.get(config, 0)
    what = (f"the first {cap} layers only ({info['triangles']} triangles; a lower bound of "
            "the full extraction)" if cap else
            f"full extraction of the same mesh, {info['layers']} layers, "
            f"{info['triangles']} triangles")
    return what


def cpu_baseline(arrays, config, budget_s=25.0):
    """The reference's CPU path (fast-bvh-peel, restated) on all host threads;
    a bounded sample: one warm-up extraction plus as many timed ones as fit
    in `budget_s` (at most 4); an extraction longer than the budget is timed
    once, without a warm-up.  CPU_LAYER_SAMPLE meshes peel their first
    layers only."""
    from oracle import fastpeel

    vertices, faces, camera, settings = arrays
    threads = fastpeel.max_threads()
    layers = CPU_LAYER_SAMPLE.get(config, 0)
    first, info = fastpeel.run(vertices, faces, camera, settings, threads=threads, repeat=1,
                               layers=layers)
    if first[0] > budget_s:
        times, warm = first, 0
    else:
        warm = 1
        extra = max(1, min(4, int(budget_s / max(first[0], 1e-3))))
        times, info = fastpeel.run(vertices, faces, camera, settings, threads=threads,
                                   repeat=extra, layers=layers)
    return {
        "value": 1000.0 * statistics.median(times),
        "unit": UNIT,
        "cores": threads,
        "kind": "port",
        "sample": f"{config}: {cpu_sample_text(config, info)}; {warm} warm-up + "
                  f"{len(times)} timed, median; excludes import and projection like the "
                  "reference's algorithm_seconds",
    }


def run_reference(args, rank, world):
    if rank != 0:
        return
    from peel_b200 import scenes
    from oracle import fastpeel

    arrays = scenes.CONFIGS[args.config]()
    threads = fastpeel.max_threads()
    if isinstance(arrays, list):  # a batch: a bounded sample, 4 views and 4 meshes
        sample = arrays[:4] + arrays[len(arrays) // 2:len(arrays) // 2 + 4]
        for v, f, c, st in sample[:1]:
            fastpeel.run(v, f, c, st, threads=threads, repeat=1)
        times, layers, triangles = [], 0, 0
        for v, f, c, st in sample:
            t, info = fastpeel.run(v, f, c, st, threads=threads, repeat=max(1, args.steps // 4))
            times.append(sum(t) / len(t))
            layers, triangles = max(layers, info["layers"]), triangles + info["triangles"]
        ms = 1000.0 * sum(times) / len(times)
        info = {"layers": layers, "triangles": triangles}
        vertices, faces = arrays[0][0], arrays[0][1]
    else:
        vertices, faces, camera, settings = arrays
        cap = CPU_LAYER_SAMPLE.get(args.config, 0)
        first, _ = fastpeel.run(vertices, faces, camera, settings, threads=threads, repeat=1,
                                layers=cap)
        # Bounded: as many of the K steps as fit in REFERENCE_BUDGET_S of CPU time.
        timed = max(1, min(args.steps, int(REFERENCE_BUDGET_S / max(first[0], 1e-3))))
        times, info = fastpeel.run(vertices, faces, camera, settings, threads=threads,
                                   repeat=timed, layers=cap)
        ms = 1000.0 * sum(times) / len(times)
    line = {
        "metric": METRIC, "value": ms, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args.config, vertices, faces), "impl": "reference",
        "cpu_baseline": {"value": ms, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{len(times)} of the {args.steps} steps timed (at most "
                                   f"{REFERENCE_BUDGET_S:.0f} s of extractions) after 1 "
                                   f"warm-up, mean; each {cpu_sample_text(args.config, info)}"},
        "e2e": {"value": ms, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if args.config == "knot-65536":
        second = scenes.CONFIGS[SECOND_CONFIG]()
        t, info = fastpeel.run(*second, threads=threads, repeat=1,
                               layers=CPU_LAYER_SAMPLE.get(SECOND_CONFIG, 0))
        line["configs"] = {SECOND_CONFIG: {
            "value": 1000.0 * t[0], "unit": UNIT,
            "config": workload_config(SECOND_CONFIG, second[0], second[1]),
            "cpu_baseline": {"value": 1000.0 * t[0], "unit": UNIT, "cores": threads,
                             "kind": "port",
                             "sample": f"1 run, no warm-up: "
                                       f"{cpu_sample_text(SECOND_CONFIG, info)}"}}}
    print(json.dumps(line), flush=True)


def run_batched(args, rank, world, local_rank):
    """The batched configuration: every scene of the batch in one graph replay
    per step; value = device ms per mesh (batch time / scenes)."""
    import numpy as np
    import torch
    import torch.distributed as dist

    from peel_b200 import BatchPeeler, _lib, scenes

    device = torch.device("cuda", local_rank)
    torch.cuda.set_device(device)
    host = scenes.CONFIGS[args.config]()
    arrays = [scenes.to_device(h, device) for h in host]
    # Knobs tuned on the batch's first scene, applied to every workspace.
    from peel_b200 import EventPeeler
    from peel_b200.autotune import tune
    from peel_b200.sizing import fit_event_capacities

    _, first_cap = fit_event_capacities(arrays[0])
    knobs, default_ms, tuned_ms, trials = tune(
        lambda: EventPeeler(*arrays[0], capacities=first_cap), replays=5)
    batch = BatchPeeler(arrays, fit=True, tuning=knobs)
    batch.capture()
    meshes = len(batch)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=device)
    for _ in range(args.warmup):
        batch.run()
    batch.read_status()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clocks:
        for k in range(args.steps):
            with torch.cuda.stream(batch.stream):
                flush.zero_()
                starts[k].record(batch.stream)
            batch.run()
            ends[k].record(batch.stream)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    total = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    total = max_over_ranks(total, world, device)
    ms_per_step = total / args.steps
    infos = batch.read_status()
    triangles = sum(i["triangles"] for i in infos)
    polygons = sum(i["polygons"] for i in infos)

    # End to end: every scene's inputs uploaded from pinned host memory, the
    # batch replayed, every status and triangle read back.
    pinned = [[torch.as_tensor(np.ascontiguousarray(a)).pin_memory() for a in h] for h in host]
    e2e_steps = 0 if args.quick else max(1, min(args.steps, 3))
    names = ("triangles_uv", "triangles_world", "triangle_sources", "triangle_layers")
    d2h = [{n: torch.empty(tuple(getattr(p, n)[:i["triangles"]].shape),
                           dtype=getattr(p, n).dtype).pin_memory() for n in names}
           for p, i in zip(batch.peelers, infos)]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        with torch.cuda.stream(batch.stream):
            for dst, src in zip(arrays, pinned):
                for d, s_ in zip(dst, src):
                    d.copy_(s_.reshape(d.shape), non_blocking=True)
        batch.run()
        got = batch.read_status()
        with torch.cuda.stream(batch.stream):
            for p, i, bufs in zip(batch.peelers, got, d2h):
                for n, buf in bufs.items():
                    buf[:i["triangles"]].copy_(getattr(p, n)[:i["triangles"]], non_blocking=True)
        batch.stream.synchronize()
    e2e_ms = 1000.0 * (time.perf_counter() - t0) / max(e2e_steps, 1)
    if rank != 0:
        return
    h2d = sum(a.numel() * a.element_size() for h in pinned for a in h)
    peak, peak_kind = hbm_peak()
    mesh_bytes = sum(algorithmic_bytes(len(h[0]), len(h[1]), i["triangles"])
                     for h, i in zip(host, infos))
    lib = _lib.load()
    launches = 0
    for p, i in zip(batch.peelers, infos):
        outside = np.zeros(2, dtype=np.int64)
        _lib.check(lib.edp_graph_kernels(p._ws.handle, outside.ctypes.data,
                                         outside.ctypes.data + 8), "graph kernels")
        launches += int(outside[0] + outside[1] * i["rounds"])
    cpu = None
    if world == 1 and not args.quick:
        from oracle import fastpeel

        threads = fastpeel.max_threads()
        sample = host[:2] + host[meshes // 2:meshes // 2 + 2]
        times = [fastpeel.run(*h, threads=threads, repeat=1)[0][0] for h in sample]
        cpu = {"value": 1000.0 * sum(times) / len(times), "unit": UNIT, "cores": threads,
               "kind": "port", "sample": "2 views and 2 meshes of the batch, one extraction "
                                         "each, mean per mesh; excludes import and projection"}
    line = {
        "metric": METRIC, "value": whole_job_ms_per_mesh(total, args.steps * meshes, world),
        "unit": UNIT,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_per_step, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{args.config}: {DESCRIPTIONS[args.config]}", "meshes": meshes,
                   "faces": int(sum(len(h[1]) for h in host)),
                   "l2": "flushed between timed replays (256 MiB device write)",
                   "parallelism": "replicas"},
        "roofline": {"bound": "hbm", "kernel": "whole batch graph (compulsory bytes)",
                     "achieved": mesh_bytes / (ms_per_step * 1e-3) / 1e9, "peak": peak,
                     "unit": "GB/s", "frac": mesh_bytes / (ms_per_step * 1e-3) / 1e9 / peak,
                     "traffic": None, "peak_source": f"{peak_kind} copy bandwidth",
                     "algorithmic_bytes": mesh_bytes},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_ms / meshes if e2e_steps else None, "unit": UNIT,
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step":
                    int(sum(64 + 152 + 128 * i["triangles"] for i in infos))},
        "gpu_launches": int(args.steps * launches), "clocks": clocks.summary(),
        "tuning": {"knobs": knobs, "tuned_on": "the batch's first scene",
                   "default_ms": default_ms, "tuned_ms": tuned_ms, "trials": len(trials)},
        "output": {"polygons": polygons, "triangles": triangles,
                   "layers_max": max(i["layers"] for i in infos)},
        "throughput": {"fragments_per_s": polygons / (ms_per_step * 1e-3),
                       "triangles_per_s": triangles / (ms_per_step * 1e-3)},
    }
    print(json.dumps(line), flush=True)


def stage_medians(p, replays, flush):
    """Per-stage device ms from the graph's own timing events (each replay
    records the end of every stage, so the stages sum to the replay): median
    over `replays` L2-flushed replays."""
    import torch

    samples = {}
    for _ in range(replays):
        with torch.cuda.stream(p.stream):
            flush.zero_()
        p.run()
        for name, ms in p.stage_times().items():
            samples.setdefault(name, []).append(ms)
    return {name: statistics.median(v) for name, v in samples.items()}


def time_replays(p, steps, flush):
    """Mean device ms of `steps` replays of p's graph, each after an L2 flush
    (CUDA events on the workspace stream)."""
    import torch

    total = 0.0
    for _ in range(steps):
        with torch.cuda.stream(p.stream):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(p.stream)
        p.run()
        b.record(p.stream)
        b.synchronize()
        total += a.elapsed_time(b)
    return total / max(steps, 1)


def measure_config(config, args, rank, world, local_rank, steps, e2e_steps, cpu_leg,
                   audit_samples, compare_forms=False, compare_pools=False):
    """Time one single-mesh configuration; returns its measurement dict.

    Device time: `steps` replays of the captured extraction after
    args.warmup, each after a 256 MiB L2 flush, CUDA events on the workspace
    stream, max over ranks.  Stages: the graph's own per-stage timing events
    (edp_stage_times), median over further replays.  End to end: inputs
    uploaded from pinned host memory, the replay, status and every triangle
    read back, per step."""
    import numpy as np
    import torch
    import torch.distributed as dist

    from peel_b200 import _lib, scenes
    from peel_b200.sizing import fit_event_capacities

    device = torch.device("cuda", local_rank)
    torch.cuda.set_device(device)
    started = time.perf_counter()
    host = scenes.CONFIGS[config]()
    scene_s = time.perf_counter() - started
    vertices, faces, camera, settings = host
    arrays = scenes.to_device(host, device)
    form = args.predicates
    p, capacities = fit_event_capacities(arrays, predicates=form)
    lib = _lib.load()
    # The autotuner's coordinate search over the work-distribution knobs
    # (same outputs under every choice); the timed replays use its choice.
    from peel_b200 import EventPeeler
    from peel_b200.autotune import SPACE, tune

    if args.quick:  # profiler runs keep the default knobs
        knobs = {k: v for k, v in p.tuning().items() if k in SPACE}
        default_ms = tuned_ms = None
        trials = []
    else:
        knobs, default_ms, tuned_ms, trials = tune(
            lambda: EventPeeler(*arrays, capacities=capacities, predicates=form), replays=5)
    p.set_tuning(**knobs)
    p.capture()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=device)
    for _ in range(args.warmup):
        p.run()
    p.read_status()
    stream = p.stream
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clocks:
        for k in range(steps):
            with torch.cuda.stream(stream):
                flush.zero_()
                starts[k].record(stream)
            p.run()
            ends[k].record(stream)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    total = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    total = max_over_ranks(total, world, device)
    ms_per_mesh = whole_job_ms_per_mesh(total, steps, world)
    check = p.read_status()

    stage_ms = stage_medians(p, max(5, min(steps, 21)), flush)

    pinned = [torch.as_tensor(a).pin_memory() for a in host]
    t_count = check["triangles"]
    d2h = {name: torch.empty(tuple(getattr(p, name)[:t_count].shape),
                             dtype=getattr(p, name).dtype).pin_memory()
           for name in ("triangles_uv", "triangles_world", "triangle_sources", "triangle_layers")}
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        with torch.cuda.stream(stream):
            for dst, src in zip(arrays, pinned):
                dst.copy_(src.reshape(dst.shape), non_blocking=True)
        p.run()
        got = p.read_status()["triangles"]
        with torch.cuda.stream(stream):
            for name, buf in d2h.items():
                buf[:got].copy_(getattr(p, name)[:got], non_blocking=True)
        stream.synchronize()
    e2e_serial_ms = 1000.0 * (time.perf_counter() - t0) / max(e2e_steps, 1)
    outside = np.zeros(2, dtype=np.int64)
    _lib.check(lib.edp_graph_kernels(p._ws.handle, outside.ctypes.data, outside.ctypes.data + 8),
               "graph kernels")
    launches = int(outside[0] + outside[1] * check["rounds"])
    report = None
    if audit_samples and rank == 0:
        from peel_b200.audit import peeler_vertex_audit

        report = peeler_vertex_audit(p, samples=audit_samples)
    # Free this workspace before the stream's two (the 720K pools are large).
    del p
    # The same through peel_b200.pipeline.PeelStream: two workspaces take
    # turns, so mesh i's triangles come back while mesh i + 1 is extracted.
    e2e_ms = None
    if e2e_steps:
        from peel_b200.pipeline import PeelStream

        stream_peeler = PeelStream(arrays, capacities, tuning=knobs, predicates=form)
        pipelined_steps = max(e2e_steps, 4 * e2e_steps)
        stream_peeler.submit(pinned)  # warm-up submission, collected untimed
        stream_peeler.finish()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(pipelined_steps):
            stream_peeler.submit(pinned)
        stream_peeler.finish()
        e2e_ms = 1000.0 * (time.perf_counter() - t0) / pipelined_steps
        del stream_peeler
        e2e_ms = max_over_ranks(e2e_ms, world, device) / world
    e2e_serial_ms = max_over_ranks(e2e_serial_ms, world, device) / world
    h2d = sum(a.numel() * a.element_size() for a in pinned)
    d2h_bytes = 64 + 152 + 128 * t_count
    if rank != 0:
        return None
    peak, peak_kind = hbm_peak()
    mesh_bytes = algorithmic_bytes(len(vertices), len(faces), check["triangles"])
    # Noding / emission kernels: every output triangle written once (128 B),
    # each boundary vertex read once (16 B) and each polygon's header (32 B).
    emit_bytes = 128 * check["triangles"] + 16 * check["boundary_vertices"] + 32 * check["polygons"]
    emit_ms = float(stage_ms["mesh_emit"])
    roofline = {
        "bound": "hbm",
        "kernel": "k_mesh_polygons + k_mesh_heavy (noding, fan emission, world lift)",
        "achieved": emit_bytes / (emit_ms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
        "frac": emit_bytes / (emit_ms * 1e-3) / 1e9 / peak,
        "traffic": ncu_traffic(config),
        "traffic_source": f"ncu capture recorded in profiles/k_mesh_polygons_{config}.md",
        "peak_source": f"{peak_kind} copy bandwidth", "algorithmic_bytes": emit_bytes,
        "launch_ms": emit_ms,
        "pipeline": {"bytes_per_mesh": mesh_bytes,
                     "achieved_gbs": mesh_bytes / (ms_per_mesh * 1e-3) / 1e9,
                     "frac": mesh_bytes / (ms_per_mesh * 1e-3) / 1e9 / peak},
    }
    result = {
        "value": ms_per_mesh, "ms_per_step": total / steps, "steps": steps,
        "config": workload_config(config, vertices, faces),
        "roofline": roofline,
        "cpu_baseline": cpu_baseline(host, config) if cpu_leg else None,
        "e2e": {"value": e2e_ms, "unit": UNIT,
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h_bytes),
                "mode": "peel_b200.pipeline.PeelStream: pinned host inputs uploaded, the "
                        "graph replayed, status and every triangle read back each step; two "
                        "workspaces take turns so a mesh's readback overlaps the next "
                        "extraction",
                "serial_value": e2e_serial_ms if e2e_steps else None},
        "gpu_launches": int(steps * launches),
        "kernels_per_replay": {"outside_loop": int(outside[0]), "per_round": int(outside[1]),
                               "rounds": check["rounds"]},
        "clocks": clocks.summary(),
        "stages_ms": stage_ms,
        "tuning": {"knobs": knobs, "default_ms": default_ms, "tuned_ms": tuned_ms,
                   "trials": len(trials),
                   "search": "coordinate search, median of 5 L2-flushed replays per trial"},
        "stages_sum_ms": sum(stage_ms.values()),
        "output": {k: check[k] for k in ("polygons", "triangles", "layers", "boundary_vertices")},
        "throughput": {"fragments_per_s": check["polygons"] / (ms_per_mesh * 1e-3),
                       "triangles_per_s": check["triangles"] / (ms_per_mesh * 1e-3)},
        "capacities": vars(capacities),
    }
    if report is not None:
        result["vertex_error"] = {k: report[k] for k in (
            "polygons", "vertices_measured", "unexplained_vertices", "max_abs_error",
            "scene_extent", "max_rel_error")}
        result["vertex_error_max"] = report["max_rel_error"]
    if config == "overlap-720k":
        # The scene's exact resolution on the host cores (before any timing).
        parents, summary, raw_vertices, raw_faces = scenes.resolution_info()
        result["resolution"] = dict(summary, input_faces=int(len(raw_faces)),
                                    output_faces=int(len(faces)),
                                    scene_build_seconds=scene_s,
                                    threads=os.cpu_count(),
                                    resolver="peel_b200.resolve (libedp_resolve.so)")
    if compare_pools:
        # Pool sizing: the trained network's pools against the worst-case
        # sizing (EventCapacities.for_mesh) and the fitted pools timed above.
        from peel_b200 import EventCapacities, learned

        sized, learned_cap, fell_back = learned.peel(arrays)
        sized.set_tuning(**knobs)
        sized.capture()
        for _ in range(args.warmup):
            sized.run()
        learned_ms = time_replays(sized, max(5, steps // 4), flush)
        learned_bytes = learned.workspace_bytes(sized)
        same = sized.read_status()["triangles"] == check["triangles"]
        del sized
        worst = EventPeeler(*arrays, capacities=EventCapacities.for_mesh(len(faces)))
        worst_bytes = learned.workspace_bytes(worst)
        del worst
        result["pool_sizing"] = {
            "learned_bytes": learned_bytes, "worst_case_bytes": worst_bytes,
            "learned_over_worst_case": learned_bytes / worst_bytes, "fell_back": fell_back,
            "learned_ms": learned_ms, "same_triangles": bool(same),
            "learned_capacities": vars(learned_cap),
            "network": "16-64-64-3 perceptron, BF16 weights on the tensor cores "
                       "(peel_b200/pool_sizing.json)"}
    if compare_forms:
        # The same extraction under the other predicate forms: the
        # reference's plain binary64 signs (the comparator of the filtered
        # forms) and the other exact form, then one counted extraction for
        # the filters' escalation rates.
        timed = {}
        for other_form in ("binary64", "filtered", "filtered64"):
            if other_form == form:
                continue
            other, _ = fit_event_capacities(arrays, capacities, predicates=other_form)
            other.set_tuning(**knobs)
            other.capture()
            for _ in range(args.warmup):
                other.run()
            ms = time_replays(other, steps, flush)
            info = other.read_status()
            timed[other_form] = {"ms": ms, "output": {k: info[k] for k in ("polygons",
                                                                           "triangles",
                                                                           "layers")},
                           "stages_ms": stage_medians(other, 7, flush)}
            del other
        counted, _ = fit_event_capacities(arrays, capacities, predicates="counted")
        counted.run()
        counts = counted.predicate_counts()
        del counted
        result["predicates"] = {
            "form": form, "ms": ms_per_mesh, "others": timed,
            "binary64_over_default": (timed["binary64"]["ms"] / ms_per_mesh
                                      if "binary64" in timed else 1.0),
            "counts": counts,
            "escalated_share": {c: (v["binary64"] + v["exact"]) / max(1, sum(v.values()))
                                for c, v in counts.items()},
            "exact_share": {c: v["exact"] / max(1, sum(v.values())) for c, v in counts.items()},
        }
    return result


SECOND_CONFIG = "overlap-720k"  # the metric's other mesh (720K faces, overlapping, resolved)


def measure_device_peeler(args, local_rank, config="icospheres-2560", steps=20):
    """The iterative-clipping route (DevicePeeler) on the nested icospheres:
    device ms per mesh, its workspace, and what per-worker pools of the
    reference's defaults would take (workers x pieces_per_worker x 3
    polygons of 32 double2 vertices and a count)."""
    import torch

    from peel_b200 import Capacities, DevicePeeler, learned, scenes

    device = torch.device("cuda", local_rank)
    host = scenes.CONFIGS[config]()
    arrays = scenes.to_device(host, device)
    cap = Capacities.for_mesh(len(host[1]))
    p = DevicePeeler(*arrays, capacities=cap)
    p.capture()
    for _ in range(args.warmup):
        p.run()
    info = p.read_status()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=device)
    ms = time_replays(p, steps, flush)
    return {"config": config, "ms_per_mesh": ms, "steps": steps,
            "output": {k: info[k] for k in ("polygons", "triangles", "layers")},
            "workspace_bytes": learned.workspace_bytes(p),
            "per_worker_pool_bytes_at_reference_defaults":
                cap.workers * cap.pieces_per_worker * 3 * (32 * 16 + 4)}


def run_ours(args, rank, world, local_rank):
    quick = args.quick
    first = measure_config(args.config, args, rank, world, local_rank, args.steps,
                          0 if quick else max(1, min(args.steps, 5)),
                          world == 1 and not quick, 0 if quick else 400,
                          compare_forms=not quick)
    extra = {}
    if args.config == "knot-65536" and not quick:
        second = measure_config(SECOND_CONFIG, args, rank, world, local_rank,
                                max(5, args.steps // 5), 3, world == 1, 300,
                                compare_forms=True, compare_pools=True)
        if second is not None:
            extra[SECOND_CONFIG] = second
    device_peeler = None if quick else measure_device_peeler(args, local_rank)
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": first["value"], "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": first["ms_per_step"],
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
    }
    line.update({k: v for k, v in first.items() if k not in ("value", "ms_per_step", "steps")})
    if extra:
        line["configs"] = extra
    if device_peeler:
        line["device_peeler"] = device_peeler
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--config", default="knot-65536")
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--predicates", default=DEFAULT_FORM,
                    choices=("filtered64", "filtered", "binary64"),
                    help="predicate form of the timed extraction (the EventPeeler default: "
                         "filtered64)")
    ap.add_argument("--quick", action="store_true",
                    help="skip the autotuner, the CPU baseline and the end-to-end leg "
                         "(for profiler runs)")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        if args.config.startswith("batched"):
            run_batched(args, rank, world, local_rank)
        else:
            run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
