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
# from one ncu capture of a full level at scale 25 (536,867,454 records):
# 2,215.8 MB read + 22.4 MB written per 2,147.5 MB of records.
BFS_DRAM_PER_ALG_BYTE = (2215.776 + 22.36288) / (536867454 * 4 / 1e6)


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
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-query measurement")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving-loop measurement")
    ap.add_argument("--no-stream", action="store_true", help="skip the semi-external (streamed) measurement")
    ap.add_argument("--serve-seconds", type=float, default=1.0, help="length of the Poisson arrival trace")
    ap.add_argument("--stream-scale", type=int, default=28)
    ap.add_argument("--stream-budget-gb", type=float, default=4.0)
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
    """One process per GPU (torchrun): rank/world from the environment, a
    process group for the barrier and the max/sum of two scalars per run
    (NCCL on the GPUs; gloo for host-only runs of the same logic)."""

    def __init__(self, gpus: int, backend: str = "nccl"):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.pg = False
        if self.world > 1:
            import datetime

            import torch.distributed as td

            td.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
            self.pg = True

    def _device(self):
        return "cuda" if self.backend == "nccl" else "cpu"

    def barrier(self):
        if self.pg:
            import torch
            import torch.distributed as td

            if self.backend == "nccl":
                td.barrier(device_ids=[torch.cuda.current_device()])
            else:
                td.barrier()

    def reduce(self, x: float, op: str) -> float:
        if not self.pg:
            return x
        import torch
        import torch.distributed as td

        t = torch.tensor([x], dtype=torch.float64, device=self._device())
        td.all_reduce(t, op=td.ReduceOp.MAX if op == "max" else td.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.pg:
            import torch.distributed as td

            td.destroy_process_group()
            self.pg = False


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


# ------------------------------------------------------- workload builders --
def make_graph(ctx, torch, scale: int, ef: int, seed1: int = 1, seed2: int = 2):
    """Graph500 Kronecker graph generated and converted on the device."""
    M = ef << scale
    d_pairs = torch.empty(2 * M, dtype=torch.int32, device="cuda")
    ctx.kron_generate_device(scale, ef, seed1, seed2, d_pairs.data_ptr())
    g = ctx.convert(d_pairs.data_ptr(), 1 << scale, n_pairs=M)
    del d_pairs
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    return g


def bench_batched(ctx, torch, gs):
    """Batched queries: 64 seeded BFS roots on Kron 24 ef16 in one persistent
    multi-source launch vs 64 sequential plain BFS runs; and 16 WCC + 16
    k-core (k uniform 4..32) over 8 graphs of scale 18-22 (seeds 1..8)."""
    out = {}
    g = make_graph(ctx, torch, 24, 16)
    roots = splitmix64_roots(g.degree(), 64, seed=1)
    with g.state("bfs", roots[0]) as s:
        s.run()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        plain = []
        for r in roots:
            s.reset(r)
            s.run()
            plain.append(s.count())
        torch.cuda.synchronize()
        t_plain = time.perf_counter() - t0
    for _ in range(8):                   # the autotuner tries each configuration once
        with gs.Batch(ctx) as b:
            for r in roots:
                b.add(g, "bfs", r)
            b.run()
    with gs.Batch(ctx) as b:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ids = [b.add(g, "bfs", r) for r in roots]
        b.run()
        torch.cuda.synchronize()
        t_batch = time.perf_counter() - t0
        st = b.stats()
        same = all(b.count(q) == plain[i] for i, q in enumerate(ids))
    out["msbfs"] = {"workload": "64 BFS roots (splitmix64 seed 1) on Kron 24 ef16",
                    "plain_queries_per_s": 64 / t_plain, "batched_queries_per_s": 64 / t_batch,
                    "speedup": t_plain / t_batch, "batched_kernel_ms": st["kernel_ms"],
                    "launches": st["launches"], "reached_counts_equal": same,
                    "plain": "gs_state_reset + gs_run per root (per-level sweep + finalize launches)"}
    g.free()
    graphs = [make_graph(ctx, torch, 18 + (i % 5), 16, seed1=i + 1) for i in range(8)]
    rng = np.random.default_rng(1)
    ks = [int(k) for k in rng.integers(4, 33, 16)]
    qs = [(graphs[i % 8], "wcc", 0) for i in range(16)] + [(graphs[i % 8], "kcore", ks[i]) for i in range(16)]

    def plain_pass():
        res = []
        for gg, a, k in qs:
            with gg.state(a, k) as s:
                s.run()
                res.append(s.count())
        torch.cuda.synchronize()
        return res

    def batch_pass():
        with gs.Batch(ctx) as b:
            ids = [b.add(gg, a, k) for gg, a, k in qs]
            b.run()
            torch.cuda.synchronize()
            return b.stats(), [b.count(q) for q in ids]

    # one untimed pass of each (kernel loading, first allocations), then the
    # median of three timed passes of each
    plain = plain_pass()
    batch_pass()
    t_plain, t_batch, kernel_ms, same = [], [], [], True
    for _ in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        plain_pass()
        t_plain.append(time.perf_counter() - t0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        st, counts = batch_pass()
        t_batch.append(time.perf_counter() - t0)
        kernel_ms.append(st["kernel_ms"])
        same = same and counts == plain
    t_plain, t_batch = float(np.median(t_plain)), float(np.median(t_batch))
    st = {"kernel_ms": float(np.median(kernel_ms)), "launches": st["launches"]}
    out["wcc_kcore"] = {"workload": "16 WCC + 16 k-core (k in 4..32, seed 1) over 8 Kron graphs of scale 18-22; "
                                    "one untimed pass each, median of 3 timed passes",
                        "plain_queries_per_s": 32 / t_plain, "batched_queries_per_s": 32 / t_batch,
                        "speedup": t_plain / t_batch, "batched_kernel_ms": st["kernel_ms"],
                        "launches": st["launches"], "result_counts_equal": same}
    for gg in graphs:
        gg.free()
    return out


def poisson_trace(graphs, seconds: float, rate: float, seed: int = 1):
    """Seeded Poisson arrivals: 70% BFS (random non-isolated root), 15%
    k-core (k uniform 4..32), 10% WCC, 5% PageRank (10 iterations)."""
    rng = np.random.default_rng(seed)
    nz = [np.nonzero(g.degree())[0] for g in graphs]
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t > seconds:
            return out
        gi = int(rng.integers(0, len(graphs)))
        u = rng.random()
        if u < 0.70:
            out.append((t, gi, "bfs", int(rng.choice(nz[gi]))))
        elif u < 0.85:
            out.append((t, gi, "kcore", int(rng.integers(4, 33))))
        elif u < 0.95:
            out.append((t, gi, "wcc", 0))
        else:
            out.append((t, gi, "pagerank", 10))


def bench_served(ctx, torch, gs, seconds: float):
    """Serving: Poisson arrivals (2000 req/s, seeded) against 16 resident
    Kronecker graphs of scale 16-24 and edgefactor 8-32 (seeds 1..16); the
    server (continuous batching) vs a one-request-at-a-time plain loop on the
    same trace.  Latency = result on the host - scheduled arrival."""
    graphs = [make_graph(ctx, torch, 16 + (i % 9), (8, 16, 32)[i % 3], seed1=i + 1) for i in range(16)]
    trace = poisson_trace(graphs, seconds, 2000.0)
    res = {"workload": f"{len(trace)} requests, Poisson 2000/s for {seconds:g} s (seed 1), "
                       "70% BFS / 15% k-core / 10% WCC / 5% PageRank(10) over 16 Kron graphs "
                       "(scale 16-24, ef 8/16/32, seeds 1..16)",
           "graphs_records": int(sum(g.n_edges for g in graphs))}

    def summarize(lat, makespan, n):
        lat = np.asarray(lat)
        return {"requests": n, "throughput_req_per_s": n / makespan, "makespan_s": makespan,
                "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
                "mean_ms": float(lat.mean() * 1e3)}

    # server
    with gs.Server(ctx) as srv:
        gids = [srv.add_graph(g) for g in graphs]
        # warm-up: one request of each kind
        for k in ("bfs", "wcc", "kcore", "pagerank"):
            srv.submit(gids[0], k, 1 if k in ("bfs", "pagerank") else 8 if k == "kcore" else 0)
        while srv.step() != (0, 0):
            pass
        torch.cuda.synchronize()
        for rid in srv.completed():
            srv.result(rid, want_data=False)
        base = srv.clock()
        index, i = {}, 0
        lat, results, t_end = [], {}, 0.0

        def collect():
            # the client takes every result as it lands: a view of the
            # server's pinned host buffer (no copy), kept for the sampled
            # checks, then released
            nonlocal t_end
            for rid in srv.completed():
                k = index.pop(rid)
                data, _, t_done, _ = srv.result_view(rid)
                lat.append(t_done - base - trace[k][0])
                t_end = max(t_end, t_done - base)
                if k % 97 == 0:
                    results[k] = data.copy()
                srv.release(rid)

        while True:
            now = srv.clock() - base
            while i < len(trace) and trace[i][0] <= now:
                t, gi, a, arg = trace[i]
                index[srv.submit(gids[gi], a, arg)] = i
                i += 1
            na, nq = srv.step()
            collect()
            if i == len(trace) and na == 0 and nq == 0:
                break
            if na == 0 and nq == 0 and i < len(trace):
                time.sleep(max(0.0, min(0.0005, trace[i][0] - (srv.clock() - base))))
        collect()
        st = srv.stats()
        res["served"] = summarize(lat, t_end, len(lat))
        res["served"].update({"steps": st["steps"], "graph_launches": st["graph_launches"],
                              "kernel_launches": st["kernel_launches"]})
    # plain one-at-a-time loop on the same trace (bounded: at most 120 s)
    lat, t0, n_done, same, checked = [], time.perf_counter(), 0, 0, 0
    for k, (t, gi, a, arg) in enumerate(trace):
        now = time.perf_counter() - t0
        if now < t:
            time.sleep(t - now)
        g = graphs[gi]
        with g.state(a, arg) as s:
            s.run()
            data = s.download(0)
        torch.cuda.synchronize()
        done = time.perf_counter() - t0
        lat.append(done - t)
        n_done += 1
        if k in results:
            checked += 1
            if a == "pagerank":
                ok = np.abs(data.astype(np.float64) - results[k]).sum() <= 1e-6 * np.abs(data.astype(np.float64)).sum()
            else:
                ok = np.array_equal(data, results[k])
            same += int(ok)
        if done > 120.0:
            break
    res["plain"] = summarize(lat, time.perf_counter() - t0, n_done)
    res["plain"]["note"] = "gs_state_create + gs_run + gs_download per request, in arrival order"
    res["throughput_ratio"] = res["served"]["throughput_req_per_s"] / res["plain"]["throughput_req_per_s"]
    res["results_checked_equal"] = f"{same}/{checked}"
    for g in graphs:
        g.free()
    return res


def bench_streamed(args, torch, gs, dev):
    """Semi-external: Kron `stream_scale` ef16 with the HBM tile budget capped
    (default 4 GB: two 2 GB segments); records stream from pinned host memory
    over PCIe, overlapped with the sweeps.  PageRank 10 iterations and one
    BFS; PCIe roofline = copied bytes / time over the measured pinned H2D
    rate."""
    scale = args.stream_scale
    V = 1 << scale
    budget = int(args.stream_budget_gb * (1 << 30))
    ctx = gs.Context(dev)
    g = make_graph(ctx, torch, scale, 16)
    E = g.n_edges
    h_grid = torch.empty(E, dtype=torch.int32, pin_memory=True)
    h_start = np.empty(gs.geometry(V)[2], np.uint64)
    h_deg = np.empty(V, np.int32)
    gs.lib().gs_graph_download(g._h, h_start.ctypes.data, h_grid.data_ptr(), h_deg.ctypes.data)
    g.free()
    ctx.close()
    torch.cuda.empty_cache()
    # measured pinned H2D rate (1 GiB)
    d = torch.empty(min(1 << 28, E), dtype=torch.int32, device="cuda")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    rates = []
    for _ in range(3):
        e0.record()
        d.copy_(h_grid[: d.numel()], non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        rates.append(d.numel() * 4 / (e0.elapsed_time(e1) / 1e3) / 1e9)
    del d
    torch.cuda.empty_cache()
    h2d = max(rates)
    ctx = gs.Context(dev, hbm_budget=budget)
    sg = ctx.upload(h_start, h_grid.numpy().view(np.uint32), h_deg, V)
    out = {"workload": f"Kron {scale} ef16 ({E} records, {E * 4 / 1e9:.1f} GB) with a {args.stream_budget_gb:g} GB "
                       "HBM tile budget (two segments of half the budget), records in pinned host memory",
           "pinned_h2d_GBps": h2d}
    st0 = sg.stream_stats()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    with sg.state("pagerank", 10) as s:
        s.run()
    torch.cuda.synchronize()
    t_pr = time.perf_counter() - t0
    st1 = sg.stream_stats()
    pr_bytes = st1["bytes"] - st0["bytes"]
    out["pagerank"] = {"iterations": 10, "ms_per_iter": t_pr / 10 * 1e3,
                       "edges_per_s_per_iter": E / (t_pr / 10), "pcie_bytes": pr_bytes,
                       "pcie_GBps": pr_bytes / t_pr / 1e9, "pcie_roofline_frac": pr_bytes / t_pr / 1e9 / h2d,
                       "segments": st1["segments"] - st0["segments"], "segments_reused": st1["reused"] - st0["reused"]}
    root = splitmix64_roots(h_deg, 1, seed=1)[0]
    with sg.state("bfs", root) as s:
        s.run()                                     # warm-up of the plan
        s.reset(root)
        st0 = sg.stream_stats()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s.run()
        torch.cuda.synchronize()
        t_bfs = time.perf_counter() - t0
        st1 = sg.stream_stats()
        stats = s.bfs_stats()
    b = st1["bytes"] - st0["bytes"]
    out["bfs"] = {"root": root, "levels": int(stats["level_counts"].size), "ms": t_bfs * 1e3,
                  "gteps": stats["edges_in_component"] / t_bfs / 1e9,
                  "edges_in_component": stats["edges_in_component"], "pcie_bytes": b,
                  "pcie_GBps": b / t_bfs / 1e9, "pcie_roofline_frac": b / t_bfs / 1e9 / h2d}
    sg.free()
    ctx.close()
    del h_grid
    return out


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
                                "of a full level at scale 25, times this run's algorithmic bytes per launch",
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

        parts = {"upload": [], "bfs": [], "download": [], "free": []}

        def e2e_step(root):
            t_a = time.perf_counter()
            g2 = ctx.upload(pin_start.numpy().view(np.uint64), pin_grid.numpy().view(np.uint32),
                            pin_deg.numpy(), V)
            t_b = time.perf_counter()
            with g2.state("bfs", root) as s:
                s.run()
                t_c = time.perf_counter()
                s.download_into(depth_out.numpy())
                t_d = time.perf_counter()
            g2.free()
            t_e = time.perf_counter()
            for k, a, b in (("upload", t_a, t_b), ("bfs", t_b, t_c), ("download", t_c, t_d), ("free", t_d, t_e)):
                parts[k].append((b - a) * 1e3)

        e2e_step(timed_roots[0])
        for v in parts.values():
            v.clear()
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
                       "what": "per step: gs_upload_graph from pinned host tile arrays, BFS, depth download",
                       "ms_per_step_median": {k: float(np.median(v)) for k, v in parts.items()}}
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args)
    # ------------------------------------- batched / served / streamed forms
    if dist.world == 1 and not args.no_secondary:
        graph.free()
        torch.cuda.empty_cache()
        sec = line.setdefault("secondary", {})
        if not args.no_batch:
            sec["batched"] = bench_batched(ctx, torch, gs)
        if not args.no_serve:
            sec["served"] = bench_served(ctx, torch, gs, args.serve_seconds)
        if not args.no_stream:
            ctx.set_stream(None)
            sec["streamed"] = bench_streamed(args, torch, gs, dev)
    if dist.rank == 0:
        print(json.dumps(line), flush=True)
    graph.free()
    ctx.close()
    dist.close()


if __name__ == "__main__":
    main()
