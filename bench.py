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
on this host's cores, on the same graph), e2e (the same metric through the
C ABI with host buffers: graph upload + BFS + depth download per step),
secondary (PageRank on the PageRank workload of Kron 20 and on this graph,
WCC, k-core with their rooflines; batched, served and streamed forms),
dropin (this engine on the reference converter's own tile files) and
parity (results checked against the CPU oracle and the reference's printed
results, outside every timed region).

``--impl reference`` runs the reference's own CPU path instead (the
reference compiled from its sources: its generator, its converter and its
in-memory BFS job) on the same Kron graph; nothing of this engine is loaded.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import shutil
import statistics
import subprocess
import sys
import tempfile
import time
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

HBM_FALLBACK_GBS = 6650.0
# DRAM bytes (read + write) per byte of records read by the BFS sweep kernel,
# from one ncu capture of a full level at scale 25 (536,867,454 records):
# 2,210.0 MB read + 11.7 MB written per 2,147.5 MB of records.
BFS_DRAM_PER_ALG_BYTE = (2210.042 + 11.718) / (536867454 * 4 / 1e6)
PR_TOL = 1e-6      # relative L1 of FP32 PageRank against the FP64 oracle
# pinned host memory a server reserves for results before it takes requests
SERVE_ARENA_BYTES = 4 << 30


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--scale", type=int, default=26)
    ap.add_argument("--edgefactor", type=int, default=16)
    ap.add_argument("--no-secondary", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true",
                    help="skip the reference leg (CPU baseline, drop-in tiles, Kron-scale parity)")
    ap.add_argument("--no-parity", action="store_true", help="skip the oracle checks")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-query measurement")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving-loop measurement")
    ap.add_argument("--no-stream", action="store_true", help="skip the semi-external (streamed) measurement")
    ap.add_argument("--serve-seconds", type=float, default=1.0, help="length of the Poisson arrival trace")
    ap.add_argument("--stream-scale", type=int, default=28)
    ap.add_argument("--stream-budget-gb", type=float, default=4.0)
    ap.add_argument("--case", choices=["bfs", "pagerank", "wcc", "kcore", "msbfs", "wk-mix", "serve"],
                    help="profiling case: build the --scale graph, run this algorithm once (msbfs: 64 seeded "
                         "roots in one batch; wk-mix: the batched WCC / k-core mix; serve: the first 500 "
                         "requests of the serving trace, all at once), print its time, exit")
    ap.add_argument("--case-arg", type=int, default=None,
                    help="the case's argument (PageRank iterations, k of k-core; default 2 and 8)")
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


def host_cpus() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def rel_l1(a, b) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).sum() / np.abs(b).sum())


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
# The G-Store reference compiled from its own sources (oracle/_ref): gstoreu
# (HALF_GRID), its Graph500 generator driver, and build_info.txt (OpenMP
# thread count and flags).  The oracle package is used only as the checker.
REF_BIN = ROOT / "oracle" / "_ref"
_REF_TIME = {20: "Half BFS time", 21: "Page-rank_mmap time", 22: "Kcore time", 23: "WCC time"}


def ref_available() -> bool:
    return (REF_BIN / "gstoreu").exists() and (REF_BIN / "kron_gen_ref").exists()


def ref_build_info() -> dict:
    """OpenMP threads (NUM_THDS, fixed when the reference is compiled) and the
    compiler flags of the reference binaries."""
    info = {"omp_threads": None, "cxxflags": None}
    p = REF_BIN / "build_info.txt"
    if p.exists():
        for line in p.read_text().splitlines():
            k, _, v = line.partition(" ")
            if k == "num_threads" and v.strip().isdigit():
                info["omp_threads"] = int(v)
            elif k == "cxxflags":
                info["cxxflags"] = v.strip()
    return info


def ref_cores() -> dict:
    info = ref_build_info()
    n = host_cpus()
    return {"cores": info["omp_threads"], "host_cpus": n, "cxxflags": info["cxxflags"],
            "threads_note": f"{info['omp_threads']} OpenMP threads (NUM_THDS of gstore.h:72, fixed at compile "
                            f"time) on {n} host CPUs"}


def scratch_dir(need_bytes: int) -> Path:
    """A scratch directory with room for need_bytes: /dev/shm when it has the
    room, else the temporary directory."""
    for base in ("/dev/shm", tempfile.gettempdir()):
        try:
            st = os.statvfs(base)
        except OSError:
            continue
        if st.f_bavail * st.f_frsize >= need_bytes + (2 << 30):
            return Path(tempfile.mkdtemp(prefix="gs_ref_", dir=base))
    raise RuntimeError(f"no scratch space for {need_bytes / 1e9:.1f} GB of tile files")


def ref_geometry(scale: int, job: int | None = None) -> list:
    """The reference CLI's geometry flag for a Kron `scale` graph: -s for
    scale >= 24.  Below 24 -s wraps the group count (gstore.cpp:145-146), so
    -v 2^scale, except for BFS and k-core, which index their state past
    vert_count under -v and run with -s 24 (same tile files)."""
    if scale >= 24:
        return ["-s", str(scale)]
    if job in (0, 10, 20, 2, 12, 22):
        return ["-s", "24"]
    return ["-v", str(1 << scale)]


def ref_make_tiles(scale: int, ef: int, work: Path, edges: np.ndarray | None = None) -> Path:
    """Tile files of Graph500 Kron `scale` edgefactor `ef` (seeds 1, 2)
    written by the reference converter (gstoreu -c 1).  The edge list comes
    from the reference generator, or is given as (M, 2) uint32 pairs."""
    edge_file = work / "edges.bin"
    if edges is None:
        subprocess.run([str(REF_BIN / "kron_gen_ref"), str(scale), str(ef), str(edge_file), "1", "2"],
                       check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    else:
        edges.tofile(edge_file)
    prefix = work / f"kron{scale}"
    subprocess.run([str(REF_BIN / "gstoreu"), *ref_geometry(scale), "-c", "1", "-i", str(edge_file),
                    "-o", str(prefix)], check=True, stdout=subprocess.DEVNULL)
    edge_file.unlink()
    for ext in (".sdegree", ".bdegree"):          # written by the converter, read by nothing here
        Path(str(prefix) + ext).unlink(missing_ok=True)
    return prefix


def ref_job(prefix: Path, scale: int, job: int, arg: int | None = None):
    """One reference job on its tile files: (seconds the job prints, stdout).
    The in-memory jobs' timers exclude reading the files (gstore.cpp:250-333)."""
    cmd = [str(REF_BIN / "gstoreu"), *ref_geometry(scale, job), "-j", str(job), "-i", str(prefix)]
    if arg is not None:
        cmd += ["-a", str(arg)]
    r = subprocess.run(cmd, check=True, capture_output=True, text=True)
    m = re.search(re.escape(_REF_TIME[job]) + r" = ([0-9.eE+-]+)", r.stdout)
    if not m:
        raise RuntimeError(f"reference job {job} printed no time: {r.stdout[-300:]}")
    return float(m.group(1)), r.stdout


def ref_printed_count(stdout: str, job: int) -> int:
    """The result line of -j 22 (k-core, gstore.cpp:2796-2803) or -j 23
    ("WCC count", wcc.cpp:336)."""
    pat = r"vertices count = (\d+)" if job == 22 else r"WCC count = (\d+)"
    return int(re.search(pat, stdout).group(1))


def read_tiles(prefix: Path, V: int, degree: bool = True):
    """<prefix>.start / .grid / .degree as the reference writes them."""
    start = np.fromfile(str(prefix) + ".start", np.uint64)
    grid = np.fromfile(str(prefix) + ".grid", np.uint32)
    deg = np.fromfile(str(prefix) + ".degree", np.int32, count=V) if degree else None
    return start, grid, deg


def ref_pagerank_config1(work: Path, runs: int, edges: np.ndarray | None = None) -> dict:
    """The reference's in-memory PageRank (-j 21 -a 5, d = 0.85 fixed in pr.cpp)
    on Graph500 Kron 20 ef16 tile files of its own converter (-v 2^20)."""
    prefix = ref_make_tiles(20, 16, work, edges=edges)
    E = (Path(str(prefix) + ".grid").stat().st_size) // 4
    times = [ref_job(prefix, 20, 21, 5)[0] for _ in range(runs)]
    t = statistics.median(times)
    return {"prefix": prefix, "records": E, "times_s": times,
            "value": E / (t / 5), "unit": "edge records/s/iteration", "ms_per_iter": t / 5 * 1e3}


def run_reference_arm(args, dist: Dist):
    """--impl reference: the reference's own CPU path on this engine's
    workload -- Graph500 Kron `scale` ef16 from the reference generator, tile
    files from the reference converter (-c 1), its in-memory BFS job -j 20
    (root 1; the timer excludes loading), one job per step.  The GTEPS
    numerator (records with both ends reached from root 1) is counted by
    the CPU oracle on the same files.  Nothing of this engine is loaded."""
    if dist.rank != 0:
        return
    scale, ef = args.scale, args.edgefactor
    V = 1 << scale
    metric = f"GTEPS (BFS, Graph500 Kronecker scale {scale}, edgefactor {ef})"
    if not ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "reference binaries absent (oracle/_ref not built)"}),
              flush=True)
        return
    import oracle

    cores = ref_cores()
    work = scratch_dir((12 * ef) << scale)
    try:
        t0 = time.perf_counter()
        prefix = ref_make_tiles(scale, ef, work)
        prep_s = time.perf_counter() - t0
        runs = [ref_job(prefix, scale, 20)[0] for _ in range(args.warmup + args.steps)]
        timed = runs[args.warmup:] or runs
        start, grid, _ = read_tiles(prefix, V, degree=False)
        p, _, _ = oracle.geometry(V)
        depth, levels, _ = oracle.bfs(start, grid, p, False, V, 1)
        E = oracle.edges_reached(start, grid, p, False, depth)
        n_records = int(grid.size)
        del start, grid, depth
        t = sum(timed) / len(timed)
        v = E / t / 1e9
        sample = (f"reference gstoreu {' '.join(ref_geometry(scale, 20))} -j 20 (in-memory BFS from root 1) on "
                  f"Graph500 Kron {scale} "
                  f"ef{ef} tile files of the reference generator and converter (-c 1); {len(timed)} timed jobs "
                  f"after {args.warmup} warm-up jobs; numerator {E} records with both ends reached (CPU oracle "
                  f"on the same files)")
        line = {"metric": metric, "value": v, "unit": "GTEPS", "impl": "reference", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "u8",
                "data": "synthetic: Graph500 Kronecker generator of the reference (seeds 1,2), its -c 1 converter",
                "config": {"workload": f"BFS from root 1 on the undirected SNB tile grid of Kron {scale} ef{ef}",
                           "scale": scale, "edgefactor": ef, "V": V, "records": n_records,
                           "edges_in_component": E, "levels": int(levels.size),
                           "l2": f"records {n_records * 4 / 1e9:.2f} GB, larger than the caches"},
                "cpu_baseline": dict({"value": v, "unit": "GTEPS", "kind": "reference", "sample": sample,
                                      "times_s": runs}, **cores),
                "e2e": {"value": v, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "prep_s": prep_s}
        if not args.no_secondary:
            sec = {}
            t_pr, _ = ref_job(prefix, scale, 21, 5)
            sec["pagerank"] = {"iterations": 5, "ms_per_iter": t_pr / 5 * 1e3,
                               "value": n_records / (t_pr / 5), "unit": "edge records/s/iteration"}
            t_w, out_w = ref_job(prefix, scale, 23)
            sec["wcc"] = {"ms": t_w * 1e3, "result": ref_printed_count(out_w, 23)}
            t_k, out_k = ref_job(prefix, scale, 22, 8)
            sec["kcore8"] = {"ms": t_k * 1e3, "result": ref_printed_count(out_k, 22)}
            for f in work.iterdir():
                f.unlink()
            pr1 = ref_pagerank_config1(work, 3)
            pr1.pop("prefix")
            sec["pagerank_config1"] = dict(pr1, workload="PageRank 5 iterations, d 0.85, Kron 20 ef16 (-v 1048576)")
            line["secondary"] = sec
    finally:
        shutil.rmtree(work, ignore_errors=True)
    print(json.dumps(line), flush=True)


# --------------------------------------------------------- timing helpers --
class DevTimer:
    """CUDA events on the engine's stream around a callable."""

    def __init__(self, torch, stream):
        self.torch = torch
        self.stream = stream
        self.e0 = torch.cuda.Event(enable_timing=True)
        self.e1 = torch.cuda.Event(enable_timing=True)

    def once(self, fn) -> float:
        self.torch.cuda.synchronize()
        self.e0.record(self.stream)
        fn()
        self.e1.record(self.stream)
        self.torch.cuda.synchronize()
        return self.e0.elapsed_time(self.e1)


def time_bfs_roots(graph, timer, roots, keep: dict | None = None):
    """BFS from each root once (after one untimed run): (ms per root,
    records with both ends reached per root); depths kept in `keep`."""
    ms, edges = [], []
    with graph.state("bfs", roots[0]) as s:
        s.run()
        for r in roots:
            s.reset(r)
            ms.append(timer.once(s.run))
            edges.append(s.bfs_stats()["edges_in_component"])
            if keep is not None:
                keep[r] = s.download()
    return ms, edges


def time_algo(graph, timer, algo, arg, keep: dict | None = None, key=None, what: int = 0, kernel=None):
    """One untimed run, then one timed run of `algo`; returns (ms, sweeps,
    count, kernel).  With kernel = an algorithm id, one more run with the
    engine's kernel timers on (they sync after every sweep launch, so the
    timed run has them off) gives (launches, ms, algorithmic bytes) of the
    sweep kernel."""
    ctx = graph.ctx
    with graph.state(algo, arg) as s:
        s.run()
        s.reset(arg)
        box = {}
        ms = timer.once(lambda: box.__setitem__("n", s.run()))
        if keep is not None:
            keep[key or algo] = s.download(what)
        count = s.count()
        kt = None
        if kernel is not None:
            s.reset(arg)
            ctx.profile(True)
            try:
                s.run()
                kt = ctx.kernel_time(kernel)
            finally:
                ctx.profile(False)
        return ms, box["n"], count, kt


def roofline(peak, peak_kind, kernel, launches, ms, alg_bytes, note):
    achieved = alg_bytes / (ms / 1e3) / 1e9 if ms > 0 else None
    return {"bound": "hbm", "kernel": kernel, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": (achieved / peak) if achieved else None, "peak_source": peak_kind, "traffic": None,
            "algorithmic_bytes": note, "algorithmic_bytes_per_launch": alg_bytes / max(launches, 1),
            "launches": launches, "kernel_ms_total": ms}


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


def bench_pr_config1(args, ctx, torch, gs, timer, peak, peak_kind, checks: bool):
    """PageRank workload: 5 iterations, d = 0.85, FP32, Graph500 Kron 20 ef16
    (seeds 1, 2), undirected, -c 1 tiles.  A step is one 5-iteration
    PageRank; the 67 MB of records fit in L2, so L2 is flushed (a 256 MB
    write on the engine's stream) before each step.  With the reference
    binaries present (rank 0 of a 1-GPU run): the reference's -j 21 -a 5 on
    its own converter's tiles of the same edge list, this engine on those
    tiles, and the FP64 oracle's ranks."""
    scale, ef = 20, 16
    V = 1 << scale
    pairs = ctx.kron_generate(scale, ef)
    g = ctx.convert(pairs, V)
    E = g.n_edges
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    steps = max(args.steps, 5)

    def run_steps(graph):
        with graph.state("pagerank", 5) as s:
            s.run()                               # warm-up (builds the sweep layout)
            ms = []
            for _ in range(steps):
                with torch.cuda.stream(timer.stream):
                    flush.fill_(1)
                s.reset(5)
                ms.append(timer.once(s.run))
            r = s.download(0)
            # one more step with the kernel timers on, for the sweep's roofline
            with torch.cuda.stream(timer.stream):
                flush.fill_(1)
            s.reset(5)
            ctx.profile(True)
            try:
                s.run()
                n, kms, kbytes = ctx.kernel_time(gs.GS_ALGO_PAGERANK)
            finally:
                ctx.profile(False)
        return float(np.median(ms)), n, kms, kbytes, r

    ms, n, kms, kbytes, r = run_steps(g)
    out = {"workload": "PageRank 5 iterations, d 0.85, FP32, Graph500 Kron 20 ef16 (seeds 1,2), undirected, "
                       "-c 1 tiles; L2 flushed before each step",
           "metric": "PR edge records/s/iteration", "unit": "edge records/s/iteration", "records": E,
           "steps": steps, "ms_per_iter": ms / 5, "value": E / (ms / 5 / 1e3),
           "roofline": roofline(peak, peak_kind, "PageRank sweep", n, kms, kbytes,
                                "4E + 12V per iteration (records; x, s, inverse degree)")}
    g.free()
    if checks and ref_available():
        import oracle

        work = scratch_dir(16 << 26)
        try:
            ref = ref_pagerank_config1(work, 3, edges=pairs)
            out["cpu_baseline"] = dict({"value": ref["value"], "unit": ref["unit"], "kind": "reference",
                                        "sample": "reference gstoreu -v 1048576 -j 21 -a 5 (in-memory PageRank) on "
                                                  "the reference converter's tiles of the same edge list; median of 3",
                                        "ms_per_iter": ref["ms_per_iter"], "times_s": ref["times_s"]}, **ref_cores())
            start, grid, degree = read_tiles(ref["prefix"], V)
            gr = ctx.upload(start, grid, degree, V)
            ms_r, _, _, _, r_ref_tiles = run_steps(gr)
            gr.free()
            out["dropin"] = {"ms_per_iter": ms_r / 5, "value": E / (ms_r / 5 / 1e3),
                             "tiles": "reference converter's (records in its thread order)"}
            p, _, _ = oracle.geometry(V)
            r64, _ = oracle.pagerank(start, grid, degree, p, False, V, 5)
            e1, e2 = rel_l1(r, r64), rel_l1(r_ref_tiles, r64)
            out["parity"] = {"rel_l1_vs_fp64_oracle": {"engine_tiles": e1, "reference_tiles": e2},
                             "tolerance": PR_TOL, "within": bool(e1 <= PR_TOL and e2 <= PR_TOL)}
        finally:
            shutil.rmtree(work, ignore_errors=True)
    del flush
    torch.cuda.empty_cache()
    return out


def reference_leg(args, ctx, torch, gs, timer, ours: dict, checks: bool):
    """Rank 0 of a 1-GPU run: the reference's CPU path on the bench graph,
    this engine on the reference's own tile files, and the oracle.

    1. The edge list (the device generator's, byte-identical to the
       reference generator's) goes to the reference converter (-c 1).
    2. cpu_baseline: the reference's -j 20 (root 1) three times; -j 22 -a 8
       and -j 23 once, whose printed results are parity anchors.
    3. dropin: those tile files (records in the converter's thread order)
       through gs_upload_graph; BFS, PageRank, WCC and k-core timed.
    4. parity: the oracle on the reference's files against this engine on
       both tile files (its own converter's and the reference's).

    ours: this engine's results on its own graph -- 'start', 'degree', 'bfs'
    {root: depth}, 'wcc', 'kcore8', 'bfs_roots', 'bfs_ms'."""
    scale, ef = args.scale, args.edgefactor
    V = 1 << scale
    M = ef << scale
    work = scratch_dir(12 * M)
    res = {}
    try:
        d_pairs = torch.empty(2 * M, dtype=torch.int32, device="cuda")
        ctx.kron_generate_device(scale, ef, 1, 2, d_pairs.data_ptr())
        torch.cuda.synchronize()
        edges = d_pairs.cpu().numpy().view(np.uint32)
        del d_pairs
        torch.cuda.empty_cache()
        prefix = ref_make_tiles(scale, ef, work, edges=edges)
        del edges
        bfs_t = [ref_job(prefix, scale, 20)[0] for _ in range(3)]
        t_k, out_k = ref_job(prefix, scale, 22, 8)
        t_w, out_w = ref_job(prefix, scale, 23)
        start, grid, degree = read_tiles(prefix, V)
        # ---- drop-in: this engine on the reference converter's tiles
        theirs = {"bfs": {}}
        roots = ours["bfs_roots"]
        g = ctx.upload(start, grid, degree, V)
        ms_b, e_b = time_bfs_roots(g, timer, roots, theirs["bfs"])
        ms_pr, _, _, _ = time_algo(g, timer, "pagerank", 5, theirs)
        ms_wcc, _, n_wcc, _ = time_algo(g, timer, "wcc", 0, theirs)
        ms_k, _, n_k, _ = time_algo(g, timer, "kcore", 8, theirs, key="kcore8")
        g.free()
        torch.cuda.empty_cache()
        sec = ours.get("secondary", {})
        res["dropin"] = {
            "tiles": "the reference converter's -c 1 files (records in its thread order), gs_upload_graph",
            "bfs": {"roots": roots, "gteps": sum(e_b) / (sum(ms_b) / 1e3) / 1e9,
                    "engine_tiles_gteps": sum(e_b) / (sum(ours["bfs_ms"]) / 1e3) / 1e9},
            "pagerank_ms_per_iter": ms_pr / 5,
            "engine_tiles_pagerank_ms_per_iter": sec.get("pagerank", {}).get("ms_per_iter"),
            "wcc_ms": ms_wcc, "engine_tiles_wcc_ms": sec.get("wcc", {}).get("ms"),
            "kcore8_ms": ms_k, "engine_tiles_kcore8_ms": sec.get("kcore8", {}).get("ms")}
        # ---- parity: the oracle on the reference's tile files
        par = {"graph": f"Kron {scale} ef{ef}: the reference converter's tile files; this engine on them and on "
                        "its own converter's files"}
        par["converter_start_degree_equal"] = bool(np.array_equal(ours["start"], start) and
                                                   np.array_equal(ours["degree"], degree))
        par["wcc_count"] = {"reference_printed": ref_printed_count(out_w, 23), "engine": n_wcc}
        par["kcore8_count"] = {"reference_printed": ref_printed_count(out_k, 22), "engine": n_k}
        if checks:
            import oracle

            p, _, _ = oracle.geometry(V)
            jobs = {("bfs", r): (lambda r=r: oracle.bfs(start, grid, p, False, V, r)[0]) for r in roots}
            jobs["wcc"] = lambda: oracle.wcc(start, grid, p, False, V)[0]
            jobs["kcore8"] = lambda: oracle.kcore(start, grid, degree, p, V, 8)[0]
            jobs["pagerank"] = lambda: oracle.pagerank(start, grid, degree, p, False, V, 5)[0]
            t0 = time.perf_counter()
            with ThreadPoolExecutor(len(jobs)) as ex:          # the oracle's C calls release the GIL
                futs = {k: ex.submit(f) for k, f in jobs.items()}
                orc = {k: f.result() for k, f in futs.items()}
            par["oracle_s"] = time.perf_counter() - t0
            par["bfs_depth_equal"] = {
                "engine_tiles": {str(r): bool(np.array_equal(ours["bfs"][r], orc[("bfs", r)])) for r in roots},
                "reference_tiles": {str(r): bool(np.array_equal(theirs["bfs"][r], orc[("bfs", r)])) for r in roots}}
            par["wcc_partition_equal"] = {"engine_tiles": bool(np.array_equal(ours["wcc"], orc["wcc"])),
                                          "reference_tiles": bool(np.array_equal(theirs["wcc"], orc["wcc"]))}
            par["kcore_deg_equal"] = {"engine_tiles": bool(np.array_equal(ours["kcore8"], orc["kcore8"])),
                                      "reference_tiles": bool(np.array_equal(theirs["kcore8"], orc["kcore8"]))}
            e_own, e_ref = rel_l1(ours["pagerank"], orc["pagerank"]), rel_l1(theirs["pagerank"], orc["pagerank"])
            par["pagerank_rel_l1_vs_fp64_oracle"] = {"engine_tiles": e_own, "reference_tiles": e_ref,
                                                     "iterations": 5, "tolerance": PR_TOL,
                                                     "within": bool(max(e_own, e_ref) <= PR_TOL)}
            E1 = oracle.edges_reached(start, grid, p, False, orc[("bfs", 1)]) if 1 in roots else None
        else:
            E1 = e_b[roots.index(1)] if 1 in roots else None
        # ---- cpu_baseline: the reference's -j 20 from root 1
        t = statistics.median(bfs_t)
        res["cpu_baseline"] = dict({
            "value": E1 / t / 1e9 if E1 else None, "unit": "GTEPS", "kind": "reference",
            "sample": (f"reference gstoreu {' '.join(ref_geometry(scale, 20))} -j 20 (in-memory BFS from root 1) on "
                       f"the reference converter's "
                       f"tile files of this Kron {scale} ef{ef} graph; median of {len(bfs_t)} jobs; numerator "
                       f"{E1} records with both ends reached"),
            "times_s": bfs_t, "kcore8_s": t_k, "wcc_s": t_w}, **ref_cores())
        res["parity"] = par
    finally:
        shutil.rmtree(work, ignore_errors=True)
    return res


def bench_batched(ctx, torch, gs, checks: bool):
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
        for r in roots:
            s.reset(r)
            s.run()
            s.count()
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
        planes = [b.download(q) for q in ids]
    # untimed: each query's depth plane against a plain BFS of its root and,
    # with the checks on, against the oracle's BFS
    plain_equal = all(np.array_equal(planes[i], g.bfs(r)) for i, r in enumerate(roots))
    out["msbfs"] = {"workload": "64 BFS roots (splitmix64 seed 1) on Kron 24 ef16",
                    "plain_queries_per_s": 64 / t_plain, "batched_queries_per_s": 64 / t_batch,
                    "speedup": t_plain / t_batch, "batched_kernel_ms": st["kernel_ms"],
                    "launches": st["launches"], "depth_planes_equal_plain": plain_equal,
                    "plain": "gs_state_reset + gs_run per root (per-level sweep + finalize launches)"}
    if checks:
        import oracle

        start, grid, _ = g.download()
        p, _, _ = oracle.geometry(1 << 24)
        t0 = time.perf_counter()
        with ThreadPoolExecutor(host_cpus()) as ex:
            depths = list(ex.map(lambda r: oracle.bfs(start, grid, p, False, 1 << 24, r)[0], roots))
        out["msbfs"]["depth_planes_equal_oracle"] = f"{sum(np.array_equal(a, b) for a, b in zip(planes, depths))}/64"
        out["msbfs"]["oracle_s"] = time.perf_counter() - t0
        del start, grid, depths
    del planes
    g.free()
    graphs = [make_graph(ctx, torch, 18 + (i % 5), 16, seed1=i + 1) for i in range(8)]
    rng = np.random.default_rng(1)
    ks = [int(k) for k in rng.integers(4, 33, 16)]
    qs = [(graphs[i % 8], "wcc", 0) for i in range(16)] + [(graphs[i % 8], "kcore", ks[i]) for i in range(16)]
    distinct = list({(id(gg), a, k): (gg, a, k) for gg, a, k in qs}.values())

    def plain_pass(queries, keep=None):
        for gg, a, k in queries:
            with gg.state(a, k) as s:
                s.run()
                if keep is not None:
                    keep[(id(gg), a, k)] = s.download()
                else:
                    s.count()
        torch.cuda.synchronize()

    def batch_pass(keep=None):
        with gs.Batch(ctx) as b:
            ids = [b.add(gg, a, k) for gg, a, k in qs]
            b.run()
            torch.cuda.synchronize()
            if keep is not None:
                for (gg, a, k), q in zip(qs, ids):
                    keep.append(((id(gg), a, k), b.download(q)))
            return b.stats()

    # one untimed pass of each (kernel loading, first allocations; results
    # compared array by array), then the median of three timed passes of each
    want, got = {}, []
    plain_pass(distinct, want)
    batch_pass(got)
    same = all(np.array_equal(arr, want[key]) for key, arr in got)
    del want, got
    # each distinct query alone: no batch can finish before its longest
    # query does on the whole GPU, so sum / max bounds the speed-up
    alone = []
    for gg, a, k in distinct:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        plain_pass([(gg, a, k)])
        alone.append(time.perf_counter() - t0)
    t_all, t_dist, t_batch, kernel_ms = [], [], [], []
    for _ in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        plain_pass(qs)
        t_all.append(time.perf_counter() - t0)
        t0 = time.perf_counter()
        plain_pass(distinct)
        t_dist.append(time.perf_counter() - t0)
        t0 = time.perf_counter()
        st = batch_pass()
        t_batch.append(time.perf_counter() - t0)
        kernel_ms.append(st["kernel_ms"])
    t_all, t_dist, t_batch = (float(np.median(x)) for x in (t_all, t_dist, t_batch))
    out["wcc_kcore"] = {"workload": "16 WCC + 16 k-core (k in 4..32, seed 1) over 8 Kron graphs of scale 18-22; "
                                    "one untimed pass each, median of 3 timed passes",
                        "queries": len(qs), "distinct_queries": len(distinct),
                        "plain_queries_per_s": len(qs) / t_all, "batched_queries_per_s": len(qs) / t_batch,
                        "speedup": t_all / t_batch,
                        "plain_distinct_queries_per_s": len(qs) / t_dist,
                        "speedup_without_dedup_credit": t_dist / t_batch,
                        "batched_kernel_ms": float(np.median(kernel_ms)), "launches": st["launches"],
                        "longest_query_alone_ms": max(alone) * 1e3,
                        "speedup_bound_distinct": sum(alone) / max(alone),
                        "results_equal_plain": same,
                        "note": "the batch runs identical queries once; speedup_without_dedup_credit lets the plain "
                                "loop skip them too"}
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
    same trace, and vs the same loop with a cache of earlier identical
    requests' results (no deduplication credit for the server).  Latency =
    result on the host - scheduled arrival."""
    graphs = [make_graph(ctx, torch, 16 + (i % 9), (8, 16, 32)[i % 3], seed1=i + 1) for i in range(16)]
    trace = poisson_trace(graphs, seconds, 2000.0)
    res = {"workload": f"{len(trace)} requests, Poisson 2000/s for {seconds:g} s (seed 1), "
                       "70% BFS / 15% k-core / 10% WCC / 5% PageRank(10) over 16 Kron graphs "
                       "(scale 16-24, ef 8/16/32, seeds 1..16)",
           "graphs_records": int(sum(g.n_edges for g in graphs)),
           "distinct_requests": len({(gi, a, arg) for _, gi, a, arg in trace})}

    def summarize(lat, makespan, n):
        lat = np.asarray(lat)
        return {"requests": n, "throughput_req_per_s": n / makespan, "makespan_s": makespan,
                "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
                "mean_ms": float(lat.mean() * 1e3)}

    def serve_trace(tr, sample: bool):
        """The server on a trace; latency = result on the host - arrival.
        Set-up, before the clock starts: the graphs are registered and the
        server's pinned result arena is reserved (SERVE_ARENA_BYTES; pinning
        pages runs at a few GB/s, so a server pins its result memory when it
        starts, not under the requests)."""
        with gs.Server(ctx) as srv:
            gids = [srv.add_graph(g) for g in graphs]
            t_pin = time.perf_counter()
            srv.reserve_host(SERVE_ARENA_BYTES)
            t_pin = time.perf_counter() - t_pin
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
            lat, kept, t_end = [], {}, 0.0

            def collect():
                # the client takes every result as it lands: a view of the
                # server's pinned host buffer (no copy), kept for the sampled
                # checks, then released
                nonlocal t_end
                for rid in srv.completed():
                    k = index.pop(rid)
                    data, _, t_done, _ = srv.result_view(rid)
                    lat.append(t_done - base - tr[k][0])
                    t_end = max(t_end, t_done - base)
                    if sample and k % 97 == 0:
                        kept[k] = data.copy()
                    srv.release(rid)

            while True:
                now = srv.clock() - base
                while i < len(tr) and tr[i][0] <= now:
                    t, gi, a, arg = tr[i]
                    index[srv.submit(gids[gi], a, arg)] = i
                    i += 1
                na, nq = srv.step()
                collect()
                if i == len(tr) and na == 0 and nq == 0:
                    break
                if na == 0 and nq == 0 and i < len(tr):
                    time.sleep(max(0.0, min(0.0005, tr[i][0] - (srv.clock() - base))))
            collect()
            st = srv.stats()
            out = summarize(lat, t_end, len(lat))
            last_arrival = max(x[0] for x in tr)
            if last_arrival > 0:
                out["offered_req_per_s"] = len(tr) / last_arrival
            out.update({"steps": st["steps"], "graph_launches": st["graph_launches"],
                        "kernel_launches": st["kernel_launches"], "host_phases_s": srv.profile(),
                        "result_arena": {"bytes": SERVE_ARENA_BYTES, "pin_s_at_setup": t_pin}})
        return out, kept

    res["served"], results = serve_trace(trace, True)
    # capacity: the same requests all submitted at t = 0 (the server never
    # waits for an arrival), against the plain loop, which never keeps up
    # with the trace and so runs at its own capacity too
    res["served_saturated"], _ = serve_trace([(0.0, gi, a, arg) for _, gi, a, arg in trace], False)
    res["served_saturated"]["note"] = "the trace's requests all arriving at t = 0"
    res["keeps_up"] = res["served_saturated"]["throughput_req_per_s"] > res["served"].get("offered_req_per_s", 0)

    def plain_loop(cache: bool):
        # one request at a time in arrival order (bounded: at most 120 s);
        # with `cache`, a request identical to an earlier one takes its result
        lat, t0, n_done, same, checked, memo = [], time.perf_counter(), 0, 0, 0, {}
        for k, (t, gi, a, arg) in enumerate(trace):
            now = time.perf_counter() - t0
            if now < t:
                time.sleep(t - now)
            key = (gi, a, arg)
            if cache and key in memo:
                data = memo[key]
            else:
                with graphs[gi].state(a, arg) as s:
                    s.run()
                    data = s.download(0)
                torch.cuda.synchronize()
                if cache:
                    memo[key] = data
            done = time.perf_counter() - t0
            lat.append(done - t)
            n_done += 1
            if k in results:
                checked += 1
                if a == "pagerank":
                    ok = rel_l1(results[k], data) <= PR_TOL
                else:
                    ok = np.array_equal(data, results[k])
                same += int(ok)
            if done > 120.0:
                break
        out = summarize(lat, time.perf_counter() - t0, n_done)
        return out, same, checked

    res["plain"], same, checked = plain_loop(False)
    res["plain"]["note"] = "gs_state_create + gs_run + gs_download per request, in arrival order"
    res["plain_cached"], _, _ = plain_loop(True)
    res["plain_cached"]["note"] = "the same loop reusing the result of an earlier identical request"
    res["throughput_ratio"] = res["served"]["throughput_req_per_s"] / res["plain"]["throughput_req_per_s"]
    res["capacity_ratio"] = res["served_saturated"]["throughput_req_per_s"] / res["plain"]["throughput_req_per_s"]
    res["throughput_ratio_without_dedup_credit"] = (res["served"]["throughput_req_per_s"] /
                                                    res["plain_cached"]["throughput_req_per_s"])
    res["capacity_ratio_without_dedup_credit"] = (res["served_saturated"]["throughput_req_per_s"] /
                                                  res["plain_cached"]["throughput_req_per_s"])
    res["results_checked_equal"] = f"{same}/{checked}"
    for g in graphs:
        g.free()
    return res


def bench_streamed(args, torch, gs, dev, checks: bool = False):
    """Semi-external: Kron `stream_scale` ef16 with the HBM tile budget capped
    (default 4 GB: two 2 GB segments); records stream from pinned host memory
    over PCIe, overlapped with the sweeps.  PageRank 10 iterations and one
    BFS; PCIe roofline = copied bytes / time over the measured pinned H2D
    rate.  Then the same graph resident in HBM (no budget): its BFS depths
    must equal the streamed run's; with the checks on, both runs' ranks are
    compared with the FP64 oracle's (10 iterations)."""
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
        r_streamed = s.download(0)
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
        d_streamed = s.download()
    b = st1["bytes"] - st0["bytes"]
    out["bfs"] = {"root": root, "levels": int(stats["level_counts"].size), "ms": t_bfs * 1e3,
                  "gteps": stats["edges_in_component"] / t_bfs / 1e9,
                  "edges_in_component": stats["edges_in_component"], "pcie_bytes": b,
                  "pcie_GBps": b / t_bfs / 1e9, "pcie_roofline_frac": b / t_bfs / 1e9 / h2d}
    sg.free()
    ctx.close()
    # the same records resident in HBM
    ctx = gs.Context(dev)
    rg = ctx.upload(h_start, h_grid.numpy().view(np.uint32), h_deg, V)
    d_resident = rg.bfs(root)
    r_resident, _ = rg.pagerank(10)
    rg.free()
    ctx.close()
    out["parity"] = {"against": "the same graph resident in HBM",
                     "bfs_depth_equal": bool(np.array_equal(d_streamed, d_resident)),
                     "pagerank_rel_l1_streamed_vs_resident": rel_l1(r_streamed, r_resident), "tolerance": PR_TOL}
    if checks:
        import oracle

        t0 = time.perf_counter()
        p, _, _ = oracle.geometry(V)
        r64, _ = oracle.pagerank(h_start, h_grid.numpy().view(np.uint32), h_deg, p, False, V, 10)
        e_s, e_r = rel_l1(r_streamed, r64), rel_l1(r_resident, r64)
        out["parity"]["pagerank_rel_l1_vs_fp64_oracle"] = {"streamed": e_s, "resident": e_r,
                                                           "within": bool(max(e_s, e_r) <= PR_TOL),
                                                           "oracle_s": time.perf_counter() - t0}
    del h_grid
    torch.cuda.empty_cache()
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
    timer = DevTimer(torch, stream)
    solo = dist.rank == 0 and dist.world == 1
    checks = solo and not args.no_parity

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
    if args.case == "serve":
        graph.free()
        graphs = [make_graph(ctx, torch, 16 + (i % 9), (8, 16, 32)[i % 3], seed1=i + 1) for i in range(16)]
        trace = poisson_trace(graphs, 1.0, 2000.0)[:500]
        t0 = time.perf_counter()
        with gs.Server(ctx) as srv:
            gids = [srv.add_graph(g) for g in graphs]
            srv.reserve_host(SERVE_ARENA_BYTES)
            t0 = time.perf_counter()
            for _, gi, a, arg in trace:
                srv.submit(gids[gi], a, arg)
            n = 0
            while True:
                na, nq = srv.step()
                for rid in srv.completed():
                    srv.result(rid, want_data=False)
                    n += 1
                if na == 0 and nq == 0:
                    break
            st = srv.stats()
        print(json.dumps({"case": "serve", "requests": n, "steps": st["steps"],
                          "ms": (time.perf_counter() - t0) * 1e3}))
        for gg in graphs:
            gg.free()
        ctx.close()
        dist.close()
        return
    if args.case in ("msbfs", "wk-mix"):
        # one batch, for a profiler's capture (not a bench line)
        t0 = time.perf_counter()
        graphs = [graph]
        if args.case == "msbfs":   # the autotuner tries each configuration once first
            for _ in range(8):
                with gs.Batch(ctx) as b:
                    for r in splitmix64_roots(degree, 64, seed=1):
                        b.add(graph, "bfs", r)
                    b.run()
        with gs.Batch(ctx) as b:
            if args.case == "msbfs":
                for r in splitmix64_roots(degree, 64, seed=1):
                    b.add(graph, "bfs", r)
            else:
                graphs = [make_graph(ctx, torch, 18 + (i % 5), 16, seed1=i + 1) for i in range(8)]
                rng = np.random.default_rng(1)
                ks = [int(k) for k in rng.integers(4, 33, 16)]
                for i in range(16):
                    b.add(graphs[i % 8], "wcc", 0)
                for i in range(16):
                    b.add(graphs[i % 8], "kcore", ks[i])
            b.run()
            torch.cuda.synchronize()
            st = b.stats()
        print(json.dumps({"case": args.case, "scale": scale, "batch_kernel_ms": st["kernel_ms"],
                          "ms_incl_setup": (time.perf_counter() - t0) * 1e3}))
        for gg in graphs:
            gg.free()
        ctx.close()
        dist.close()
        return
    if args.case:
        # one query of one algorithm, for a profiler's capture (not a bench line)
        arg = args.case_arg
        if arg is None:
            arg = {"pagerank": 2, "kcore": 8, "wcc": 0}.get(args.case)
        if args.case == "bfs":
            arg = splitmix64_roots(degree, 1, seed=1)[0]
        t0 = time.perf_counter()
        with graph.state(args.case, arg) as s:
            s.run()
        torch.cuda.synchronize()
        print(json.dumps({"case": args.case, "arg": int(arg), "scale": scale,
                          "ms_incl_layout_build": (time.perf_counter() - t0) * 1e3}))
        graph.free()
        ctx.close()
        dist.close()
        return
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
    e_comp, swept_records, read_records, levels = 0, 0, 0, []
    for r in timed_roots:
        state.reset(r)
        state.run()
        st = state.bfs_stats()
        e_comp += st["edges_in_component"]
        swept_records += int(st["swept"].sum())
        read_records += int(st["read"].sum())
        levels.append(int(st["level_counts"].size))
    state.free()
    ms_max = dist.reduce(ms, "max")
    e_total = dist.reduce(float(e_comp), "sum")
    value = e_total / (ms_max / 1e3) / 1e9
    peak, peak_kind = measured_peak()
    # algorithmic bytes: 4 B x the records of the tiles the reference's skip
    # rule sweeps at each level; the kernel reads fewer (it skips chunks
    # whose records all had both ends visited at an earlier level: they can
    # discover nothing), so the line also gives the bandwidth on the bytes
    # it actually read
    achieved = (4.0 * swept_records) / (sweep_ms / 1e3) / 1e9 if sweep_ms > 0 else None
    alg_per_launch = 4.0 * swept_records / max(sweep_launches, 1)
    read_per_launch = 4.0 * read_records / max(sweep_launches, 1)
    achieved_read = read_per_launch * max(sweep_launches, 1) / (sweep_ms / 1e3) / 1e9 if sweep_ms > 0 else None
    rl = {"bound": "hbm", "kernel": "bfs_run_kernel", "achieved": achieved, "peak": peak,
          "unit": "GB/s", "frac": (achieved / peak) if achieved else None, "peak_source": peak_kind,
          "traffic": BFS_DRAM_PER_ALG_BYTE * read_per_launch,
          "traffic_note": "bytes per launch: DRAM read+write per byte of records read, from an ncu capture "
                          "of a full level at scale 25, times this run's records read per launch",
          "algorithmic_bytes": "4 B x records in the tiles the reference's skip rule sweeps per level",
          "algorithmic_bytes_per_launch": alg_per_launch,
          "read_bytes_per_launch": read_per_launch,
          "read_note": "4 B x records the kernel read: the swept tiles less the 256-record chunks whose "
                       "records all had both ends visited at an earlier level",
          "achieved_on_bytes_read": achieved_read,
          "frac_on_bytes_read": (achieved_read / peak) if achieved_read else None,
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
        "roofline": rl, "gpu_launches": launches, "clocks": clk,
    }

    # this engine's results kept for the checks against the oracle and the
    # reference (rank 0 of a 1-GPU run)
    leg = solo and not args.no_cpu_baseline and not args.no_secondary
    ours = {"bfs": {}, "bfs_roots": [1, *timed_roots[:2]]}
    if leg:
        ours["bfs_ms"], _ = time_bfs_roots(graph, timer, ours["bfs_roots"], ours["bfs"])

    # ------------------------------------------------------ secondary metrics
    if not args.no_secondary:
        sec = {}
        pr_ms, _, _, (n, kms, kbytes) = time_algo(graph, timer, "pagerank", 5, ours if leg else None,
                                                  kernel=gs.GS_ALGO_PAGERANK)
        sec["pagerank"] = {"metric": "PR edge records/s/iteration", "iterations": 5,
                           "ms_per_iter": pr_ms / 5, "value": graph.n_edges / (pr_ms / 5 / 1e3),
                           "sweep_ms_per_iter": kms / max(n, 1),
                           "roofline": roofline(peak, peak_kind, "PageRank sweep", n, kms, kbytes,
                                                "4E + 12V per iteration (records; x, s, inverse degree)")}
        keep = ours if leg else None
        for name, algo, arg, gid, kname, note in (
                ("wcc", "wcc", 0, gs.GS_ALGO_WCC, "wcc_hook_runs (sampled pass + full pass)",
                 "4E + 8V per sweep (records; parent read and write); the time covers the sampled "
                 "hooking pass, the largest-tree bitmap and the full pass"),
                ("kcore8", "kcore", 8, gs.GS_ALGO_KCORE, "sweep_runs<KcoreOp>",
                 "4 x records of the tiles with a removed end window + 8V per round")):
            t_ms, steps, count, (n, kms, kbytes) = time_algo(graph, timer, algo, arg, keep, key=name, kernel=gid)
            sec[name] = {"ms": t_ms, "sweeps": steps, "result": count,
                         "roofline": roofline(peak, peak_kind, kname, n, kms, kbytes, note)}
        line["secondary"] = sec
        ours["secondary"] = sec
        if solo:
            sec["pagerank_config1"] = bench_pr_config1(args, ctx, torch, gs, timer, peak, peak_kind, checks)

    # ----------------------------------------------------------------- e2e
    if not args.no_e2e:
        start_h, grid_h, deg_h = graph.download()
        ours["start"], ours["degree"] = start_h, deg_h
        pin_grid = torch.from_numpy(grid_h.view(np.int32)).pin_memory()
        pin_start = torch.from_numpy(start_h.view(np.int64)).pin_memory()
        pin_deg = torch.from_numpy(deg_h).pin_memory()
        depth_out = torch.empty(V, dtype=torch.uint8).pin_memory()
        del grid_h
        graph.free()
        torch.cuda.empty_cache()

        parts = {"upload": [], "bfs": [], "download": [], "state_free": [], "graph_free": [], "step": []}

        def e2e_step(root):
            t_a = time.perf_counter()
            g2 = ctx.upload(pin_start.numpy().view(np.uint64), pin_grid.numpy().view(np.uint32),
                            pin_deg.numpy(), V)
            t_b = time.perf_counter()
            s = g2.state("bfs", root)
            s.run()
            t_c = time.perf_counter()
            s.download_into(depth_out.numpy())
            t_d = time.perf_counter()
            s.free()
            t_e = time.perf_counter()
            g2.free()
            t_f = time.perf_counter()
            for k, a, b in (("upload", t_a, t_b), ("bfs", t_b, t_c), ("download", t_c, t_d), ("state_free", t_d, t_e),
                            ("graph_free", t_e, t_f), ("step", t_a, t_f)):
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
                       "ms_per_step_median": {k: float(np.median(v)) for k, v in parts.items()},
                       "ms_per_step_max": {k: float(np.max(v)) for k, v in parts.items()}}
        del pin_grid
    else:
        ours["start"], _, ours["degree"] = graph.download()
        graph.free()
        torch.cuda.empty_cache()
    # ------------------------------------- the reference on the same graph
    if leg:
        if ref_available():
            res = reference_leg(args, ctx, torch, gs, timer, ours, checks)
            line["cpu_baseline"] = res["cpu_baseline"]
            line["dropin"] = res["dropin"]
            line["parity"] = res["parity"]
        else:
            line["cpu_baseline"] = {"unavailable": "reference binaries absent (oracle/_ref not built)"}
    ours.clear()
    # ------------------------------------- batched / served / streamed forms
    if solo and not args.no_secondary:
        sec = line.setdefault("secondary", {})
        if not args.no_batch:
            sec["batched"] = bench_batched(ctx, torch, gs, checks)
        if not args.no_serve:
            sec["served"] = bench_served(ctx, torch, gs, args.serve_seconds)
        if not args.no_stream:
            ctx.set_stream(None)
            sec["streamed"] = bench_streamed(args, torch, gs, dev, checks)
    if dist.rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    dist.close()


if __name__ == "__main__":
    main()
