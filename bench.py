#!/usr/bin/env python
"""Headline benchmark: BFS GTEPS on the G-Store tile grid of a Graph500
Kronecker graph (scale 26, edgefactor 16, seeds 1/2, undirected, SNB tiles),
on one B200 per rank.

A step is one BFS from a seeded root (splitmix64 stream seeded 1, x mod V,
roots with degree 0 rejected) over the resident tile grid: the per-level
tile sweep of bfs.cpp with its tile-skip rule, done by the sm_100a kernels
of libgstore_cuda.so through its C ABI.  GTEPS = records with both ends
reached / BFS time.

The input is synthetic: the Graph500 generator restated on the device
(byte-identical to the reference's generator) and the "-c 1" converter on
the device; 4.3 GB of records, larger than L2, so no L2 flush is needed
between steps.

Multi-GPU: the path needs no exchange for this workload (each rank holds a
replica and runs its own roots; weak scaling).  Times are device times
(CUDA events on the engine's stream), max over ranks.

Printed JSON keys beyond the base contract: roofline (BFS sweep kernel vs
measured HBM peak), cpu_baseline (the reference built from its own sources,
on this host's cores), e2e (the same metric through the C ABI with host
buffers: graph upload + BFS + depth download per step), secondary (PageRank
edges/s/iteration, WCC, k-core on the same graph).
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

HBM_FALLBACK_GBS = 6650.0
# DRAM bytes (read + write) per algorithmic byte of the BFS sweep kernel,
# from one ncu capture of a full level at scale 22: 275.9 MB / 268.4 MB.
BFS_DRAM_PER_ALG_BYTE = (271.015424 + 4.886016) / (67106947 * 4 / 1e6)


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--scale", type=int, default=26)
    ap.add_argument("--edgefactor", type=int, default=16)
    ap.add_argument("--cpu-scale", type=int, default=24, help="scale of the CPU reference sample")
    ap.add_argument("--no-secondary", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


# ------------------------------------------------------------------ helpers --
def splitmix64_roots(degree: np.ndarray, count: int, seed: int = 1, skip: int = 0):
    """Seeded roots: splitmix64 stream, x mod V, rejecting isolated vertices."""
    V = degree.size
    x = seed & 0xFFFFFFFFFFFFFFFF
    out = []
    n = 0
    while len(out) < count:
        x = (x + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
        z = x
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
        z ^= z >> 31
        v = z % V
        if degree[v] > 0:
            if n >= skip:
                out.append(int(v))
            n += 1
    return out


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return HBM_FALLBACK_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-i", str(self.device), "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in Path(self.path).read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


class Dist:
    def __init__(self, gpus: int):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = False
        if self.world > 1:
            import datetime

            import torch.distributed as td

            td.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
            self.pg = True

    def barrier(self):
        if self.pg:
            import torch
            import torch.distributed as td

            td.barrier(device_ids=[torch.cuda.current_device()])

    def reduce(self, x: float, op: str) -> float:
        if not self.pg:
            return x
        import torch
        import torch.distributed as td

        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        td.all_reduce(t, op=td.ReduceOp.MAX if op == "max" else td.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.pg:
            import torch.distributed as td

            td.destroy_process_group()


# ------------------------------------------------------------ CPU reference --
def reference_sample(scale: int, edgefactor: int, runs: int, log=None):
    """The G-Store reference (compiled from its sources into oracle/_ref) on a
    bounded sample: Graph500 Kron `scale` from the reference generator,
    converted by the reference converter, BFS by its in-memory job -j 20
    (root 1, 32 OpenMP threads, timer excludes loading).  Returns per-run
    seconds and the tile-file prefix."""
    ref = ROOT / "oracle" / "_ref"
    gen, exe = ref / "kron_gen_ref", ref / "gstoreu"
    if not (gen.exists() and exe.exists()):
        return None, "reference binaries absent (oracle/_ref not built)"
    base = Path("/dev/shm") if Path("/dev/shm").is_dir() else Path(tempfile.gettempdir())
    work = Path(tempfile.mkdtemp(prefix="gs_ref_", dir=base))
    V = 1 << scale
    edges = work / "edges.bin"
    prefix = work / "g"
    subprocess.run([str(gen), str(scale), str(edgefactor), str(edges), "1", "2"], check=True,
                   stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    subprocess.run([str(exe), "-v", str(V), "-c", "1", "-i", str(edges), "-o", str(prefix)], check=True,
                   stdout=subprocess.DEVNULL)
    edges.unlink()
    times = []
    for _ in range(runs):
        r = subprocess.run([str(exe), "-v", str(V), "-j", "20", "-i", str(prefix)], check=True,
                           capture_output=True, text=True)
        m = re.search(r"Half BFS time = ([0-9.eE+-]+)", r.stdout)
        times.append(float(m.group(1)))
    return (times, prefix, work), None


def component_edges_root1(prefix: Path, V: int) -> int:
    """GTEPS numerator of the reference sample (records with both ends reached
    from root 1), counted by the engine on the same tile files."""
    import gstore_b200 as gs

    start, grid, _ = gs.read_tile_files(prefix, V, with_degree=False)
    with gs.Context(0) as ctx:
        g = ctx.upload(start, grid, None, V)
        with g.state("bfs", 1) as s:
            s.run()
            e = s.bfs_stats()["edges_in_component"]
        g.free()
    return e


def cpu_baseline(args, steps: int | None = None):
    runs = steps or 3
    res, why = reference_sample(args.cpu_scale, args.edgefactor, runs)
    if res is None:
        return {"unavailable": why}
    times, prefix, work = res
    try:
        E = component_edges_root1(prefix, 1 << args.cpu_scale)
    finally:
        subprocess.run(["rm", "-rf", str(work)])
    t = statistics.median(times)
    return {"value": E / t / 1e9, "unit": "GTEPS", "cores": 32, "kind": "reference",
            "host_cpus": os.cpu_count(),
            "sample": (f"reference gstoreu -j 20 (in-memory BFS, root 1, 32 OpenMP threads, NUM_THDS) on "
                       f"Graph500 Kron {args.cpu_scale} ef{args.edgefactor} from the reference generator and "
                       f"converter; median of {len(times)} runs {['%.3f' % x for x in times]} s; "
                       f"{E} component records"),
            "times_s": times, "edges_in_component": E}


def run_reference_arm(args, dist: Dist):
    if dist.rank != 0:
        return
    base = {"metric": f"GTEPS (BFS, Graph500 Kronecker scale {args.scale}, edgefactor {args.edgefactor})",
            "unit": "GTEPS", "impl": "reference", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u8", "data": "synthetic"}
    cb = cpu_baseline(args, steps=args.steps + args.warmup)
    if "unavailable" in cb:
        print(json.dumps({"impl": "reference", "unavailable": cb["unavailable"]}), flush=True)
        return
    timed = cb["times_s"][args.warmup:] or cb["times_s"]
    t = sum(timed) / len(timed)
    v = cb["edges_in_component"] / t / 1e9
    line = dict(base, value=v, ms_per_step=t * 1e3,
                config={"workload": f"BFS (reference -j 20, root 1) on Kron {args.cpu_scale} ef{args.edgefactor} "
                                    f"as a bounded sample of Kron {args.scale}",
                        "scale": args.cpu_scale, "edgefactor": args.edgefactor},
                cpu_baseline={"value": v, "unit": "GTEPS", "cores": 32, "kind": "reference",
                              "sample": cb["sample"]},
                e2e={"value": v, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0})
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ our arm --
def main():
    args = parse_args()
    dist = Dist(args.gpus)
    if args.impl == "reference":
        run_reference_arm(args, dist)
        dist.close()
        return

    import torch

    import gstore_b200 as gs

    torch.cuda.set_device(dist.local)
    dev = torch.cuda.current_device()
    stream = torch.cuda.Stream()
    ctx = gs.Context(dev)
    ctx.set_stream(stream.cuda_stream)

    scale, ef = args.scale, args.edgefactor
    V = 1 << scale
    M = ef << scale
    # input preparation (untimed): generator + converter on the device
    with torch.cuda.stream(stream):
        d_pairs = torch.empty(2 * M, dtype=torch.int32, device="cuda")
    ctx.kron_generate_device(scale, ef, 1, 2, d_pairs.data_ptr())
    graph = ctx.convert(d_pairs.data_ptr(), V, n_pairs=M)
    del d_pairs
    torch.cuda.empty_cache()
    degree = graph.degree()
    roots = splitmix64_roots(degree, args.warmup + args.steps, seed=1, skip=dist.rank * (args.warmup + args.steps))
    warm, timed_roots = roots[: args.warmup], roots[args.warmup:]

    state = graph.state("bfs", warm[0] if warm else timed_roots[0])
    for r in warm:
        state.reset(r)
        state.run()

    # --------------------------------------------------------- timed region
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ctx.profile(True)
    clocks = ClockSampler(dev)
    dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    launches0 = ctx.launches()
    ev0.record(stream)
    for r in timed_roots:
        state.reset(r)
        state.run()
    ev1.record(stream)
    torch.cuda.synchronize()
    launches = ctx.launches() - launches0
    clk = clocks.stop()
    dist.barrier()
    ms = ev0.elapsed_time(ev1)
    sweep_launches, sweep_ms, _ = ctx.kernel_time(gs.GS_ALGO_BFS)
    ctx.profile(False)

    # statistics of the timed runs (recomputed per root outside the timed region)
    e_comp, swept_records, levels = 0, 0, []
    for r in timed_roots:
        state.reset(r)
        state.run()
        st = state.bfs_stats()
        e_comp += st["edges_in_component"]
        swept_records += int(st["swept"].sum())
        levels.append(int(st["level_counts"].size))
    state.free()
    ms_max = dist.reduce(ms, "max")
    e_total = dist.reduce(float(e_comp), "sum")
    value = e_total / (ms_max / 1e3) / 1e9
    peak, peak_kind = measured_peak()
    achieved = (4.0 * swept_records) / (sweep_ms / 1e3) / 1e9 if sweep_ms > 0 else None
    alg_per_launch = 4.0 * swept_records / max(sweep_launches, 1)
    roofline = {"bound": "hbm", "kernel": "bfs_run_kernel", "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": (achieved / peak) if achieved else None, "peak_source": peak_kind,
                "traffic": BFS_DRAM_PER_ALG_BYTE * alg_per_launch,
                "traffic_note": "bytes per launch: DRAM read+write per algorithmic byte from an ncu capture "
                                "of a full level at scale 22, times this run's algorithmic bytes per launch",
                "algorithmic_bytes": "4 B x records in swept tiles per level",
                "algorithmic_bytes_per_launch": alg_per_launch,
                "launches": sweep_launches, "sweep_ms_total": sweep_ms}

    line = {
        "metric": f"GTEPS (BFS, Graph500 Kronecker scale {scale}, edgefactor {ef})",
        "value": value, "unit": "GTEPS", "n_gpus": dist.world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / max(1, len(timed_roots)), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8",
        "data": "synthetic: Graph500 Kronecker generator (seeds 1,2) restated on the device, -c 1 converter on the device",
        "config": {"workload": f"BFS from seeded roots on the undirected SNB tile grid of Kron {scale} ef{ef}",
                   "scale": scale, "edgefactor": ef, "V": V, "records": graph.n_edges, "tiles": graph.n_tiles,
                   "roots": timed_roots, "levels": levels, "edges_in_component": e_comp,
                   "l2": "inputs larger than L2 (records %.2f GB)" % (graph.n_edges * 4 / 1e9),
                   "parallelism": f"replica x{dist.world}"},
        "roofline": roofline, "gpu_launches": launches, "clocks": clk,
    }

    # ------------------------------------------------------ secondary metrics
    if not args.no_secondary:
        sec = {}
        ctx.profile(True)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with graph.state("pagerank", 5) as s:
            s.run()                      # warm-up
            s.reset(5)
            ctx.profile(True)
            e0.record(stream)
            s.run()
            e1.record(stream)
            torch.cuda.synchronize()
            pr_ms = e0.elapsed_time(e1)
            n, kms, kbytes = ctx.kernel_time(gs.GS_ALGO_PAGERANK)
        sec["pagerank"] = {"metric": "PR edge records/s/iteration", "iterations": 5,
                           "ms_per_iter": pr_ms / 5, "value": graph.n_edges / (pr_ms / 5 / 1e3),
                           "sweep_ms_per_iter": kms / max(n, 1),
                           "sweep_roofline_frac": (kbytes / (kms / 1e3) / 1e9 / peak) if kms else None,
                           "algorithmic_bytes_per_iter": kbytes / max(n, 1)}
        for name, algo, arg in (("wcc", "wcc", 0), ("kcore8", "kcore", 8)):
            with graph.state(algo, arg) as s:
                s.run()
                s.reset(arg)
                e0.record(stream)
                steps = s.run()
                e1.record(stream)
                torch.cuda.synchronize()
                sec[name] = {"ms": e0.elapsed_time(e1), "sweeps": steps, "result": s.count()}
        ctx.profile(False)
        line["secondary"] = sec

    # ----------------------------------------------------------------- e2e
    if not args.no_e2e:
        start_h, grid_h, deg_h = graph.download()
        pin_grid = torch.from_numpy(grid_h.view(np.int32)).pin_memory()
        pin_start = torch.from_numpy(start_h.view(np.int64)).pin_memory()
        pin_deg = torch.from_numpy(deg_h).pin_memory()
        depth_out = torch.empty(V, dtype=torch.uint8).pin_memory()
        del grid_h
        graph.free()
        torch.cuda.empty_cache()

        def e2e_step(root):
            g2 = ctx.upload(pin_start.numpy().view(np.uint64), pin_grid.numpy().view(np.uint32),
                            pin_deg.numpy(), V)
            with g2.state("bfs", root) as s:
                s.run()
                s.download_into(depth_out.numpy())
            g2.free()

        e2e_step(timed_roots[0])
        dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for r in timed_roots:
            e2e_step(r)
        torch.cuda.synchronize()
        e2e_s = dist.reduce(time.perf_counter() - t0, "max")
        line["e2e"] = {"value": e_total / e2e_s / 1e9, "unit": "GTEPS",
                       "h2d_bytes_per_step": int(pin_grid.numel() * 4 + pin_start.numel() * 8 + pin_deg.numel() * 4),
                       "d2h_bytes_per_step": V,
                       "what": "per step: gs_upload_graph from pinned host tile arrays, BFS, depth download"}
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args)
    if dist.rank == 0:
        print(json.dumps(line), flush=True)
    graph.free()
    ctx.close()
    dist.close()


if __name__ == "__main__":
    main()
