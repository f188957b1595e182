"""Benchmark: GRE superstep suite on a seeded RMAT graph, one JSON line.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--scale S]

Workload (ours, per GPU): RMAT scale 26, edge factor 16, symmetrised and de-duplicated
(a/b/c = 0.57/0.19/0.19, seeded), uint32 ids, uint64 offsets, SSSP weights uint32 in
[1, 255]; generated on the device.  One step = the plain suite of the reference's plugins:
PageRank 20 supersteps (FP64, power iteration), direction-optimising BFS from one source,
SSSP from one source and connected components.  Sources are seeded samples of non-isolated
vertices, different every step.

Metric: GTEPS = traversed edges / device time, summed over the suite (PageRank: arcs x
supersteps; BFS/SSSP: undirected edges of the reached component (Graph500); CC: undirected
edges).  Per-algorithm GTEPS and algorithmic HBM GB/s are reported beside it.  `value` uses
device-resident outputs; `e2e` runs the same calls with pinned host outputs, the device->host
copies inside the timed region.  After the timed steps, `batched_vs_plain` reports the batched
forms against their looped plain forms at equal results (256-source BC, 64-source BFS, 128
personalised PageRank vectors, a batch of 32 uneven graphs; scale 20) and the PageRank adjoint
against its forward, plus 1024-source sampled BC in 16 batches of 64 on the scale-26 graph.  `partitioned` times the
1D-partitioned BFS, PageRank, SSSP and CC (gre_part_*, graphine_b200/partition.py) over the
ranks, NCCL exchanges; at one GPU a one-rank communicator, checked equal to the one-GPU calls.

--impl reference runs the reference GRE engine (compiled from its headers into oracle/_ref/)
on the host CPU, each step the same plain suite on a bounded sample of the workload (RMAT scale
--ref-scale, default 18, same generator and seeds; inputs from the oracle's host generator, no
product code loaded), and prints the same line with the same `config`.  Our arm reports the
suite on that sample graph too (`same_scale_as_reference`) and on the reference's stated
configs (`configs`: PageRank-20 on directed RMAT-16, BFS/SSSP/CC on RMAT-22 from 16 sources),
which `--impl reference --configs` runs on the CPU.

`--gpus N` without a launcher starts N ranks itself (torch.distributed.run, one per GPU);
under a launcher (WORLD_SIZE set) each process is one rank.  `--dry-run` exercises the rank
plumbing on the host with gloo.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import shutil
import socket
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "GTEPS & HBM GB/s at RMAT-26 on 1 B200; batched/adjoint vs plain at equal results"
SEED = 26
WSEED = 20240601
PR_ITERS = 20
BC_SOURCES = 1024  # sampled BC sources per rank at the main scale (64 per frontier word)
REF_SCALE = 18  # scale of the reference arm's bounded sample


def env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


# ----------------------------------------------------------------------------------------------
# clocks sampled during the timed region
# ----------------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []  # (arrival time, line)
        self.t0 = self.t1 = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.perf_counter(), line.strip()))

    # the sampler starts before the warm-up (nvidia-smi needs a moment to print its first line);
    # the summary keeps the samples that arrived between these marks
    def mark_start(self):
        self.t0 = time.perf_counter()

    def mark_end(self):
        self.t1 = time.perf_counter()

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        window = "timed"
        lines = [ln for t, ln in self.lines
                 if (self.t0 is None or t >= self.t0) and (self.t1 is None or t <= self.t1 + 0.1)]
        if not lines:  # timed region shorter than the sampling period: warm-up and timed steps
            window, lines = "warmup+timed", [ln for _, ln in self.lines]
        for line in lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for i, nm in enumerate(names):
                if parts[5 + i].lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm), "window": window}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic():
    """DRAM bytes per PageRank superstep from the committed ncu summary, if present."""
    p = os.path.join(ROOT, "profiles", "pagerank_pull_superstep.md")
    try:
        for line in open(p):
            m = re.match(r"\s*traffic_bytes_per_superstep_s26:\s*([0-9.eE+]+)", line)
            if m:
                return float(m.group(1))
    except OSError:
        pass
    return None


# ----------------------------------------------------------------------------------------------
# the workload's identity: one config for both arms (the reference arm times a bounded sample
# of it and says which in cpu_baseline.sample)
# ----------------------------------------------------------------------------------------------
def workload_config(scale: int, gpus: int) -> dict:
    return {"workload": f"GRE plain suite on RMAT scale {scale} EF16 symmetric: PageRank-{PR_ITERS} (power "
                        f"iteration, FP64), DO-BFS 1 src, SSSP 1 src (u32 w in [1,255]), CC",
            "scale": scale, "edgefactor": 16, "graph_seed": SEED, "weight_seed": WSEED,
            "parallelism": f"replica x{gpus}", "l2": "inputs larger than L2 (graph > 126 MB)"}


# ----------------------------------------------------------------------------------------------
# reference arm / CPU baseline: the reference engine on the host (no product code loaded)
# ----------------------------------------------------------------------------------------------
def host_info() -> dict:
    """What the CPU numbers ran on: logical CPUs, the ones this process may use, model, sockets."""
    info = {"nproc": os.cpu_count(), "usable_cpus": len(os.sched_getaffinity(0)), "model": None, "sockets": None,
            "cores_per_socket": None, "threads_per_core": None}
    try:
        out = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=20).stdout
        keys = {"Model name": "model", "Socket(s)": "sockets", "Core(s) per socket": "cores_per_socket",
                "Thread(s) per core": "threads_per_core"}
        for line in out.splitlines():
            k, _, v = line.partition(":")
            if k.strip() in keys and info[keys[k.strip()]] is None:
                v = v.strip()
                info[keys[k.strip()]] = int(v) if v.isdigit() else v
    except Exception:
        pass
    info["mpirun"] = shutil.which("mpirun") or None
    return info


def reference_suite(scale: int, reps: int, workdir: str, only=("pagerank", "bfs", "sssp", "cc")):
    """Runs the reference suite `reps` times on RMAT-`scale` (symmetric); returns per-rep
    (edges, seconds) and the graph's size.  Inputs come from the oracle's own generator and the
    Graph500 numerators from the reference's own BFS levels."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    n, off, col = O.rmat(scale, 16, SEED, True)
    prefix = os.path.join(workdir, f"rmat{scale}")
    O.write_edgelists(prefix, n, off, col, 4)
    roots = O.sample_sources(off, reps, 5)
    O.write_roots(prefix, roots)
    m_arcs = len(col)
    m_und = m_arcs // 2
    t = {k: [0.0] * reps for k in ("pagerank", "bfs", "sssp", "cc")}
    comp = [0] * reps
    if "pagerank" in only:
        _, run = O.run_reference("pagerank", prefix, "iter", PR_ITERS, reps, timeout=7200)
        t["pagerank"] = run.seconds
    if "bfs" in only or "sssp" in only:
        lv, run = O.run_reference("bfs", prefix, reps, timeout=7200)  # the first `reps` roots
        comp = [O.reached_edges(off, lv[i * n:(i + 1) * n]) for i in range(reps)]
        if "bfs" in only:
            t["bfs"] = run.seconds[0::2]  # runs alternate: the BFS plugin, then the Forward levels
    if "sssp" in only:
        _, run = O.run_reference("sssp", prefix, WSEED, reps, timeout=7200)
        t["sssp"] = run.seconds
    if "cc" in only:
        _, run = O.run_reference("cc", prefix, reps, timeout=7200)
        t["cc"] = run.seconds
    per = {k: [(0, 0.0)] * reps for k in t}
    for r in range(reps):
        per["pagerank"][r] = (m_arcs * PR_ITERS, t["pagerank"][r])
        per["bfs"][r] = (comp[r], t["bfs"][r])
        per["sssp"][r] = (comp[r], t["sssp"][r])
        per["cc"][r] = (m_und, t["cc"][r])
    out = [(sum(per[k][r][0] for k in only), sum(per[k][r][1] for k in only)) for r in range(reps)]
    return out, {"n": n, "m": m_arcs, "per": per}


def reference_configs(workdir: str) -> dict:
    """The reference on the stated configs: PageRank-20 on directed RMAT-16 (both plugins, np = 1;
    np = 4 needs MPI), and BFS / SSSP / CC on symmetric RMAT-22 from 16 sources (harmonic mean of
    per-source GTEPS for BFS and SSSP)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    res = {}
    n, off, col = O.rmat(16, 16, 1, False)
    prefix = os.path.join(workdir, "pr16")
    O.write_edgelists(prefix, n, off, col, 4)
    for variant in ("gre", "iter"):
        _, run = O.run_reference("pagerank", prefix, variant, PR_ITERS, 3, timeout=3600)
        s = statistics.median(run.seconds)
        res[f"pagerank_{variant}_s16_dir"] = {"gteps": len(col) * PR_ITERS / s / 1e9, "seconds": s, "np": 1,
                                              "arcs": len(col)}
    res["pagerank_s16_dir_np4"] = "unavailable (no MPI on host)" if not shutil.which("mpirun") else         "not run (MPI present; the harness is built against the single-rank shim)"
    n, off, col = O.rmat(22, 16, 22, True)
    prefix = os.path.join(workdir, "s22")
    O.write_edgelists(prefix, n, off, col, 4)
    roots = O.sample_sources(off, 16, 22)
    O.write_roots(prefix, roots)
    lv, run = O.run_reference("bfs", prefix, 16, timeout=7200)
    comp = [O.reached_edges(off, lv[i * n:(i + 1) * n]) for i in range(16)]
    hm = lambda xs: len(xs) / sum(1.0 / x for x in xs)  # noqa: E731
    res["bfs_s22_16src"] = {"gteps_hmean": hm([c / s / 1e9 for c, s in zip(comp, run.seconds[0::2])]),
                            "seconds_total": sum(run.seconds[0::2])}
    _, run = O.run_reference("sssp", prefix, WSEED, 16, timeout=7200)
    res["sssp_s22_16src"] = {"gteps_hmean": hm([c / s / 1e9 for c, s in zip(comp, run.seconds)]),
                             "seconds_total": sum(run.seconds)}
    _, run = O.run_reference("cc", prefix, 1, timeout=7200)
    res["cc_s22"] = {"gteps": (len(col) // 2) / run.seconds[0] / 1e9, "seconds": run.seconds[0]}
    res["graph_s22"] = {"n": n, "arcs": len(col)}
    return res


REF_THREADS = 12  # the reference engine's fixed worker pool (Engine.hpp:211), plus its master thread


def run_reference_arm(args, rank, world):
    if rank != 0:
        return 0
    t0 = time.perf_counter()
    with tempfile.TemporaryDirectory() as td:
        res, info = reference_suite(args.ref_scale, args.warmup + args.steps, td)
        configs = reference_configs(td) if args.configs else None
    timed = res[args.warmup:]
    edges = sum(e for e, _ in timed)
    secs = sum(s for _, s in timed)
    value = edges / secs / 1e9
    host = host_info()
    sample = (f"each step: the plain suite on RMAT-{args.ref_scale} symmetric EF16 (n={info['n']}, arcs={info['m']}, "
              f"same generator and seeds as the scale-{args.scale} workload; the scale-{args.scale} graph needs "
              f"~40 B/arc of host RAM in the reference loader and hours at -O0), reference GRE engine built -O0 from "
              f"its headers, np=1 (single-rank MPI shim), engine.run timed with MPI_Wtime as usr/test_*.cpp do; "
              f"{REF_THREADS} engine worker threads + master on {host['usable_cpus']} usable of {host['nproc']} "
              f"logical CPUs ({host['model']}, {host['sockets']} socket(s))")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "GTEPS", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64+u32", "data": "synthetic",
        "config": workload_config(args.scale, args.gpus),
        "cpu_baseline": {"value": value, "unit": "GTEPS", "cores": REF_THREADS, "kind": "reference",
                         "sample": sample, "host": host},
        "per_algorithm": {k: {"gteps": sum(e for e, _ in v[args.warmup:]) / max(sum(s for _, s in v[args.warmup:]), 1e-12) / 1e9,
                              "ms_per_step": sum(s for _, s in v[args.warmup:]) / args.steps * 1e3}
                          for k, v in info["per"].items()},
        "e2e": {"value": value, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": time.perf_counter() - t0,
    }
    if configs is not None:
        line["configs"] = configs
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------------------------
# our arm
# ----------------------------------------------------------------------------------------------
def configs_block(G, dev_index: int) -> dict:
    """The GPU on the reference's stated configs (the same graphs and sources as
    `--impl reference --configs`): PageRank-20 on directed RMAT-16 (both plugins), and BFS / SSSP
    / CC on symmetric RMAT-22 from 16 sources (harmonic mean of per-source GTEPS for BFS and
    SSSP, Graph500 numerators).  Device-resident outputs, device time per call."""
    import torch

    dev = torch.device("cuda", dev_index)
    res = {}
    g = G.Graph.rmat(16, 16, 1, False, device=dev_index, reorder=True)
    pr = torch.empty(g.n, dtype=torch.float64, device=dev)
    for variant, name in ((G.PR_REFERENCE, "gre"), (G.PR_ITER, "iter")):
        G.pagerank(g, variant, 0.85, PR_ITERS, out=pr)
        ms = statistics.median(G.pagerank(g, variant, 0.85, PR_ITERS, out=pr)[1].device_ms for _ in range(5))
        res[f"pagerank_{name}_s16_dir"] = {"gteps": g.m * PR_ITERS / (ms * 1e-3) / 1e9, "ms": ms, "arcs": g.m}
    del g
    g = G.Graph.rmat(22, 16, 22, True, device=dev_index, reorder=True)
    g.set_weights_hash(WSEED)
    off, _ = g.csr()
    roots = G.sample_sources(off, 16, 22)
    out = torch.empty(g.n, dtype=torch.int32, device=dev)
    hm = lambda xs: len(xs) / sum(1.0 / x for x in xs)  # noqa: E731
    for name, call in (("bfs", G.bfs), ("sssp", G.sssp)):
        call(g, roots[:1], out=out)
        sts = [call(g, [int(r)], out=out)[1] for r in roots]
        res[f"{name}_s22_16src"] = {"gteps_hmean": hm([s.gteps for s in sts]),
                                    "ms_total": sum(s.device_ms for s in sts)}
    G.cc(g, out=out)
    st = G.cc(g, out=out)[1]
    res["cc_s22"] = {"gteps": st.gteps, "ms": st.device_ms}
    res["graph_s22"] = {"n": g.n, "arcs": g.m}
    return res


def same_scale_block(G, dev_index: int, args) -> dict:
    """The plain suite on the reference arm's sample graph (RMAT-`ref_scale`, same seeds and
    sources), so that both arms can be compared on equal inputs as well."""
    import torch

    dev = torch.device("cuda", dev_index)
    g = G.Graph.rmat(args.ref_scale, 16, SEED, True, device=dev_index, reorder=True)
    g.set_weights_hash(WSEED)
    off, _ = g.csr()
    reps = args.warmup + args.steps
    roots = G.sample_sources(off, reps, 5)
    pr = torch.empty(g.n, dtype=torch.float64, device=dev)
    o32 = torch.empty(g.n, dtype=torch.int32, device=dev)
    edges, ms = 0, 0.0
    for i, r in enumerate(roots):
        sts = [G.pagerank(g, G.PR_ITER, 0.85, PR_ITERS, out=pr)[1], G.bfs(g, [int(r)], out=o32)[1],
               G.sssp(g, [int(r)], out=o32)[1], G.cc(g, out=o32)[1]]
        if i >= args.warmup:
            edges += sum(s.traversed_edges for s in sts)
            ms += sum(s.device_ms for s in sts)
    return {"scale": args.ref_scale, "n": g.n, "arcs": g.m, "steps": args.steps, "gteps": edges / (ms * 1e-3) / 1e9,
            "ms_per_step": ms / args.steps}


def batched_block(G, dev_index: int, scale: int, seed: int):
    """Batched forms vs their looped plain forms at equal results (measured once, untimed for
    `value`): 256-source BC, 64-source BFS, 128 personalised PageRank vectors, a batch of 32
    uneven RMAT graphs, and the PageRank adjoint vs its forward.  Both forms write into device
    buffers, so the comparison is of the device work (a host output would add the same
    device->host copy, 64 levels or 128 vectors per vertex, to both)."""
    import torch

    out = {"scale": scale}
    dev = torch.device("cuda", dev_index)

    def warm(f):  # each form runs once untimed first, so that neither pays first-call allocations
        f()
        return f()

    g = G.Graph.rmat(scale, 16, seed, True, device=dev_index, reorder=True)
    off, _ = g.csr()
    srcs = G.sample_sources(off, 256, 11)
    b_loop, s_loop = warm(lambda: G.bc(g, srcs, batched=False))
    b_bat, s_bat = warm(lambda: G.bc(g, srcs, batched=True))
    out["bc256"] = {"looped_ms": s_loop.device_ms, "batched_ms": s_bat.device_ms,
                    "speedup": s_loop.device_ms / s_bat.device_ms, "identical": bool(np.array_equal(b_loop, b_bat))}
    lv_a = torch.empty(64 * g.n, dtype=torch.int32, device=dev)
    lv_b = torch.empty(64 * g.n, dtype=torch.int32, device=dev)
    _, s_loop = warm(lambda: G.bfs(g, srcs[:64], out=lv_a))
    _, s_bat = warm(lambda: G.msbfs(g, srcs[:64], out=lv_b))
    out["bfs64"] = {"looped_ms": s_loop.device_ms, "batched_ms": s_bat.device_ms,
                    "speedup": s_loop.device_ms / s_bat.device_ms, "identical": bool(torch.equal(lv_a, lv_b))}
    del lv_a, lv_b
    pp_a = torch.empty(128 * g.n, dtype=torch.float64, device=dev)
    pp_b = torch.empty(128 * g.n, dtype=torch.float64, device=dev)
    _, s_loop = warm(lambda: G.ppr(g, srcs[:128], 0.85, PR_ITERS, batched=False, out=pp_a))
    _, s_bat = warm(lambda: G.ppr(g, srcs[:128], 0.85, PR_ITERS, batched=True, out=pp_b))
    out["ppr128"] = {"looped_ms": s_loop.device_ms, "batched_ms": s_bat.device_ms,
                     "speedup": s_loop.device_ms / s_bat.device_ms,
                     "rel_l1": float((pp_a - pp_b).abs().sum() / pp_a.abs().sum())}
    del pp_a, pp_b
    del g
    # 32 RMAT graphs of uneven scales 12..18 in one launch sequence (block-diagonal union)
    rng = np.random.default_rng(seed)
    scales = rng.integers(12, 19, size=32)
    parts = [G.Graph.rmat(int(s), 16, seed + i, True, device=dev_index) for i, s in enumerate(scales)]
    roots = []
    for p in parts:
        o, _ = p.csr()
        roots.append(int(G.sample_sources(o, 1, 3)[0]))
    U, voff = G.Graph.union(parts)
    t_loop, lv_loop = 0.0, []
    for p, r in zip(parts, roots):
        lv, st = warm(lambda: G.bfs(p, [r]))
        t_loop += st.device_ms
        lv_loop.append(lv)
    lv_u, st_u = warm(lambda: G.bfs_multiroot(U, [r + int(voff[i]) for i, r in enumerate(roots)]))
    out["graph_batch32_bfs"] = {"looped_ms": t_loop, "batched_ms": st_u.device_ms, "speedup": t_loop / st_u.device_ms,
                                "identical": bool(np.array_equal(np.concatenate(lv_loop), lv_u)),
                                "scales": [int(s) for s in scales]}
    del parts, U
    # adjoint vs forward (weighted PageRank, lognormal(0,1) weights, row-normalised)
    g = G.Graph.rmat(scale, 16, seed + 7, False, device=dev_index, reorder=True)
    w = np.exp(np.random.default_rng(seed).standard_normal(g.m))
    g.set_weights_f64(w)
    c = np.random.default_rng(seed + 1).standard_normal(g.n)
    r, s_fwd, _ = warm(lambda: G.pagerank_weighted(g, 0.85, None, tol=1e-13, max_iters=2000))
    lam, gp, gw, s_adj, _ = warm(lambda: G.pagerank_adjoint(g, r, c, 0.85, tol=1e-13, max_iters=2000))
    out["pagerank_adjoint"] = {"forward_ms": s_fwd.device_ms, "adjoint_ms": s_adj.device_ms,
                               "adjoint_over_forward": s_adj.device_ms / s_fwd.device_ms,
                               "forward_iters": s_fwd.supersteps, "adjoint_iters": s_adj.supersteps}
    return out


def partitioned_block(G, g, srcs, world: int, rank: int, local_rank: int) -> dict:
    """The 1D-partitioned paths (gre_part_*): this rank's part of the graph, the
    exchanges through the library's own NCCL communicator on the part's stream (over the ranks of
    the default process group; one rank when there is none, where every exchange is a local
    copy).  Device-resident outputs; device time of each call, max over ranks.  At one rank the
    results are compared with the one-GPU calls on the same inputs."""
    import torch
    import torch.distributed as tdist

    from graphine_b200 import partition as PT

    x = PT.NcclExchange()
    try:
        t0 = time.perf_counter()
        part = PT.Part(g, world, rank)
        build_s = time.perf_counter() - t0
        dev = torch.device("cuda", local_rank)
        lv = torch.empty(g.n, dtype=torch.int32, device=dev)
        pr = torch.empty(g.n, dtype=torch.float64, device=dev)
        part.bfs(int(srcs[0]), x, out=lv)  # warm-up (workspace allocation)
        part.pagerank(x, G.PR_ITER, 0.85, 2, out=pr)
        bfs_ms, edges, same_bfs = 0.0, 0, True
        for s in srcs:
            _, st = part.bfs(int(s), x, out=lv)
            bfs_ms += st.device_ms
            edges += st.traversed_edges
            if world == 1:
                one = torch.empty_like(lv)
                G.bfs(g, [int(s)], out=one)
                same_bfs = same_bfs and bool(torch.equal(one, lv))
        _, st = part.pagerank(x, G.PR_ITER, 0.85, PR_ITERS, out=pr)
        pr_ms, pr_bytes = st.device_ms, st.algo_bytes
        same_pr = None
        if world == 1:
            one = torch.empty_like(pr)
            G.pagerank(g, G.PR_ITER, 0.85, PR_ITERS, out=one)
            same_pr = bool(torch.equal(one, pr))
        # SSSP (frontier Bellman-Ford, one all-to-all of offers per superstep) and CC (label
        # propagation, one all-gather per superstep) from the first source
        ds = torch.empty(g.n, dtype=torch.int32, device=dev)
        part.sssp(int(srcs[0]), x, out=ds)
        _, st = part.sssp(int(srcs[0]), x, out=ds)
        sssp_ms, sssp_edges, sssp_steps = st.device_ms, st.traversed_edges, st.supersteps
        cc_l = torch.empty(g.n, dtype=torch.int32, device=dev)
        _, st = part.cc(x, out=cc_l)
        cc_ms, cc_steps = st.device_ms, st.supersteps
        same_sssp = same_cc = None
        if world == 1:
            one = torch.empty_like(ds)
            G.sssp(g, [int(srcs[0])], out=one)
            same_sssp = bool(torch.equal(one, ds))
            G.cc(g, out=one)
            same_cc = bool(torch.equal(one, cc_l))
        if world > 1:
            t = torch.tensor([bfs_ms, pr_ms, sssp_ms, cc_ms], dtype=torch.float64, device=dev)
            tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
            bfs_ms, pr_ms, sssp_ms, cc_ms = (float(v) for v in t)
        info = {"ranks": world, "slots_per_rank": part.slots, "arcs_in_rank0": part.arcs_in, "build_s": build_s,
                "exchange": "library NCCL communicator: all-gather / grouped send-recv on the part's stream",
                "bfs": {"sources": len(srcs), "ms_per_source": bfs_ms / len(srcs),
                        "gteps": edges / (bfs_ms * 1e-3) / 1e9 if bfs_ms else None},
                "pagerank": {"iters": PR_ITERS, "ms_per_iter": pr_ms / PR_ITERS,
                             "hbm_gbs_algorithmic": pr_bytes / (pr_ms * 1e-3) / 1e9 if pr_ms else None},
                "sssp": {"ms": sssp_ms, "supersteps": sssp_steps,
                         "gteps": sssp_edges / (sssp_ms * 1e-3) / 1e9 if sssp_ms else None},
                "cc": {"ms": cc_ms, "supersteps": cc_steps}}
        if world == 1:
            info["identical_to_one_gpu"] = {"bfs": same_bfs, "pagerank": same_pr, "sssp": same_sssp, "cc": same_cc}
        part.free()
        return info
    finally:
        x.free()


def sharded_bc_block(G, g, nz, args, world: int, local_rank: int) -> dict:
    """Sampled betweenness on the main graph: `bc_sources` sources per rank in frontier words of
    64, spread over the ranks by shard.bc (every rank runs the batched kernels on its own graph
    copy, no exchange during the run) and one NCCL sum of the per-rank FP64 vectors (8n bytes).
    Device time of each rank's batches, max over ranks; the sum's time beside it."""
    import torch

    from graphine_b200 import shard

    dev = torch.device("cuda", local_rank)
    k = args.bc_sources * world
    srcs = np.sort(np.random.default_rng(31).choice(nz, size=k, replace=False)).astype(np.uint32)  # same on all ranks
    mine = {"ms": 0.0, "edges": 0}

    def partial(block):
        out, st = G.bc(g, block, batched=True)
        mine["ms"], mine["edges"] = st.device_ms, st.traversed_edges
        return out

    torch.cuda.synchronize()
    t0 = time.perf_counter()
    total = shard.bc(g, srcs, partial=partial)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    t = torch.tensor([mine["ms"], wall], dtype=torch.float64, device=dev)
    e = torch.tensor([float(mine["edges"])], dtype=torch.float64, device=dev)
    if world > 1:
        import torch.distributed as tdist

        tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
        tdist.all_reduce(e, op=tdist.ReduceOp.SUM)
    ms, wall = float(t[0]), float(t[1])
    return {"sources": k, "ranks": world, "ms": ms, "gteps": float(e[0]) / (ms * 1e-3) / 1e9,
            "wall_s_with_sum": wall, "collective": "one all-reduce (sum) of n FP64" if world > 1 else "none (one rank)",
            "checksum": float(np.sum(total))}


def run_ours(args, rank, world, local_rank):
    import torch
    import graphine_b200.gre as G

    dist = world > 1
    if dist:
        import torch.distributed as tdist
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)

    # one-time setup per graph, outside every timed figure (as the reference times engine.run
    # only): generation, relabel + row sort, hash weights, row-schedule tuning, SSSP split
    setup = {}

    def timed(name, f):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = f()
        torch.cuda.synchronize()
        setup[name] = (time.perf_counter() - t0) * 1e3
        return r

    g = timed("generate_ms", lambda: G.Graph.rmat(args.scale, 16, SEED, True, device=local_rank))
    if not args.no_reorder:
        timed("relabel_sort_ms", g.reorder)
    timed("hash_weights_ms", lambda: g.set_weights_hash(WSEED))
    n, m = g.n, g.m
    outdeg = g.getOutdegree()
    nz = np.flatnonzero(outdeg > 0)
    rng = np.random.default_rng(1000 + rank)
    nsteps = args.warmup + args.steps
    one_src = rng.choice(nz, size=nsteps, replace=False).astype(np.uint32)
    timed("tune_ms", lambda: g.row_schedule(True))
    sdist = torch.empty(n, dtype=torch.int32, device=dev)
    timed("first_sssp_ms", lambda: G.sssp(g, one_src[:1], out=sdist))  # builds the light/heavy split
    again = G.sssp(g, one_src[:1], out=sdist)[1]
    setup["sssp_split_ms"] = max(setup.pop("first_sssp_ms") - again.device_ms, 0.0)
    setup["total_ms"] = sum(setup.values())
    del sdist

    # device-resident outputs (value)
    pr_d = torch.empty(n, dtype=torch.float64, device=dev)
    lv_d = torch.empty(n, dtype=torch.int32, device=dev)
    ds_d = torch.empty(n, dtype=torch.int32, device=dev)  # uint32 payload
    cc_d = torch.empty(n, dtype=torch.int32, device=dev)
    names = [k for k in ["pagerank", "bfs", "sssp", "cc"] if not args.only or k in args.only.split(",")]

    def suite(i, outs, src=None):
        pr_o, lv_o, ds_o, cc_o = outs
        s_ = one_src[i:i + 1] if src is None else src
        calls = {"pagerank": lambda: G.pagerank(g, G.PR_ITER, 0.85, PR_ITERS, out=pr_o)[1],
                 "bfs": lambda: G.bfs(g, s_, out=lv_o)[1], "sssp": lambda: G.sssp(g, s_, out=ds_o)[1],
                 "cc": lambda: G.cc(g, out=cc_o)[1]}
        return [calls[k]() for k in names]

    dev_outs = (pr_d, lv_d, ds_d, cc_d)
    sched = dict(zip(("lane_arcs", "cta_min", "hub_chunk", "seg_window"), g.row_schedule(True)))  # tuned above
    per = {k: {"ms": 0.0, "edges": 0, "bytes": 0, "arcs": 0} for k in names}
    with ClockSampler(local_rank) as clk:
        for i in range(args.warmup):
            suite(i, dev_outs)
        torch.cuda.synchronize()
        if dist:
            tdist.barrier()
        torch.cuda.synchronize()
        l0 = G.launch_count()
        clk.mark_start()
        for i in range(args.warmup, nsteps):
            for k, s in zip(names, suite(i, dev_outs)):
                per[k]["ms"] += s.device_ms
                per[k]["edges"] += s.traversed_edges
                per[k]["bytes"] += s.algo_bytes
                per[k]["arcs"] += s.arcs_traversed
        torch.cuda.synchronize()
        clk.mark_end()
        launches = G.launch_count() - l0
    if dist:
        tdist.barrier()
    torch.cuda.synchronize()
    tot_ms = sum(v["ms"] for v in per.values())
    tot_edges = sum(v["edges"] for v in per.values())

    # e2e: the same calls with pinned host buffers; the source id comes from pinned memory and
    # every result is copied device->host inside the timed span
    pin = lambda dt, k: torch.empty(k, dtype=dt, pin_memory=True).numpy()  # noqa: E731
    host_outs = (pin(torch.float64, n), pin(torch.int32, n), pin(torch.int32, n), pin(torch.int32, n))
    src_pinned = pin(torch.int32, 1).view(np.uint32)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e2e_edges = 0
    for i in range(args.warmup, nsteps):
        src_pinned[0] = one_src[i]
        e2e_edges += sum(s.traversed_edges for s in suite(i, host_outs, src_pinned))
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0

    # max over ranks of the time, sum of the work
    if dist:
        t = torch.tensor([tot_ms, e2e_s], dtype=torch.float64, device=dev)
        tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
        w = torch.tensor([float(tot_edges), float(e2e_edges)], dtype=torch.float64, device=dev)
        tdist.all_reduce(w, op=tdist.ReduceOp.SUM)
        max_ms, max_e2e = float(t[0]), float(t[1])
        all_edges, all_e2e_edges = float(w[0]), float(w[1])
    else:
        max_ms, max_e2e, all_edges, all_e2e_edges = tot_ms, e2e_s, float(tot_edges), float(e2e_edges)
    # the partitioned block needs every rank (its collectives); rank 0 reports it
    if world == 1 or args.partitioned:
        psrcs = np.random.default_rng(4242).choice(nz, size=4, replace=False).astype(np.uint32)  # same on all ranks
        part_info = partitioned_block(G, g, psrcs, world, rank, local_rank)
    else:
        part_info = None
    bc_info = None if args.no_batched else sharded_bc_block(G, g, nz, args, world, local_rank)
    if rank != 0:
        return 0

    value = all_edges / (max_ms * 1e-3) / 1e9
    e2e_value = all_e2e_edges / max_e2e / 1e9
    peak, peak_kind = measured_peak()
    pr = per.get("pagerank", {"ms": float("nan")})
    pr_iter_ms = pr["ms"] / (args.steps * PR_ITERS)
    pr_bytes_iter = 8 * (n + 1) + 12 * m + 20 * n
    # bytes no pull superstep can avoid: offsets, a 4-byte column id per arc, one read of the 8n
    # contributions and of the 4n degrees, the 8n rank and 8n contribution writes
    pr_compulsory = 8 * (n + 1) + 4 * m + 28 * n
    achieved = pr_bytes_iter / (pr_iter_ms * 1e-3) / 1e9 if "pagerank" in per else None  # None: not run (--only)
    per_alg = {}
    for k, v in per.items():
        per_alg[k] = {"ms_per_step": v["ms"] / args.steps,
                      "gteps": v["edges"] / (v["ms"] * 1e-3) / 1e9 if v["ms"] else None,
                      "hbm_gbs_algorithmic": v["bytes"] / (v["ms"] * 1e-3) / 1e9 if v["ms"] else None,
                      "share": v["ms"] / tot_ms}
    extra = {}
    if not args.no_batched:
        extra[f"bc{args.bc_sources}_s{args.scale}"] = bc_info
        del g
        torch.cuda.empty_cache()
        extra.update(batched_block(G, local_rank, args.batch_scale, 77))
    if not args.no_batched:
        extra["configs"] = configs_block(G, local_rank)
        extra["same_scale_as_reference"] = same_scale_block(G, local_rank, args)
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        with tempfile.TemporaryDirectory() as td:
            res, info = reference_suite(args.ref_scale, 1, td)
        e, s = res[0]
        host = host_info()
        cpu = {"value": e / s / 1e9, "unit": "GTEPS", "cores": REF_THREADS, "kind": "reference",
               "sample": f"one plain suite on RMAT-{args.ref_scale} symmetric (n={info['n']}, arcs={info['m']}), "
                         f"reference GRE engine -O0 np=1, engine.run timed; {REF_THREADS} engine worker threads + "
                         f"master on {host['usable_cpus']} usable of {host['nproc']} logical CPUs ({host['model']}, "
                         f"{host['sockets']} socket(s))",
               "host": host}
    d2h = n * (8 + 4 + 4 + 4)
    traffic = profiled_traffic() if args.scale == 26 and not args.no_reorder else None
    line = {
        "metric": METRIC, "value": value, "unit": "GTEPS", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": max_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64+u32", "data": "synthetic",
        "config": workload_config(args.scale, world),
        "graph": {"n": n, "arcs": m, "relabelled": not args.no_reorder, "row_schedule": sched},
        "setup_ms": setup,
        "per_algorithm": per_alg,
        "roofline": {"bound": "hbm", "kernel": "PageRank pull superstep (degree-binned row kernels)",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak if achieved else None,
                     "peak_kind": peak_kind, "bytes_per_launch": pr_bytes_iter,
                     "traffic": traffic, "compulsory_bytes": pr_compulsory,
                     "traffic_over_compulsory": traffic / pr_compulsory if traffic else None},
        "batched_vs_plain": extra,
        "partitioned": part_info,
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": "GTEPS", "h2d_bytes_per_step": 4, "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)
    return 0


def free_port() -> int:
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def spawn_ranks(args) -> int:
    """`--gpus N` without a launcher: start N ranks on this node (one per GPU) through
    torch.distributed.run, with this command line, and return the launcher's status."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()), os.path.abspath(__file__)] + sys.argv[1:]
    env = dict(os.environ, OMP_NUM_THREADS=os.environ.get("OMP_NUM_THREADS", "8"))
    try:
        return subprocess.run(cmd, env=env, timeout=args.launch_timeout).returncode
    except subprocess.TimeoutExpired:
        print(json.dumps({"error": f"ranks did not finish within {args.launch_timeout} s"}), flush=True)
        return 1


def run_dry(args, rank, world) -> int:
    """Rank plumbing without a GPU (gloo): every rank times a small host-side step, the time is the
    max over ranks and the work the sum, rank 0 prints the line."""
    import torch
    import torch.distributed as tdist

    if world > 1:
        import datetime

        tdist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        x = np.arange(1 << 16, dtype=np.float64) + rank
        for _ in range(args.warmup):
            float(x.sum())
        if world > 1:
            tdist.barrier()
        t0 = time.perf_counter()
        work = 0
        for _ in range(args.steps):
            work += int(x.size)
            float(np.sqrt(x).sum())
        dt = time.perf_counter() - t0
        t = torch.tensor([dt, float(work), 1.0], dtype=torch.float64)
        if world > 1:
            tmax = t.clone()
            tdist.all_reduce(tmax, op=tdist.ReduceOp.MAX)
            tdist.all_reduce(t, op=tdist.ReduceOp.SUM)
            t[0] = tmax[0]
        if rank == 0:
            print(json.dumps({"dry_run": True, "metric": METRIC, "n_gpus": world, "ranks_reporting": int(t[2]),
                              "steps": args.steps, "warmup": args.warmup, "value": float(t[1]) / max(float(t[0]), 1e-9),
                              "unit": "elements/s (host)", "config": workload_config(args.scale, world)}), flush=True)
        return 0
    finally:
        if world > 1:
            tdist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=int, default=26)
    ap.add_argument("--ref-scale", type=int, default=REF_SCALE,
                    help="scale of the reference arm's bounded sample (and of the CPU baseline)")
    ap.add_argument("--configs", action="store_true",
                    help="reference arm: also run the stated configs (PageRank S16 directed, BFS/SSSP/CC S22 x 16 "
                         "sources); minutes of CPU time")
    ap.add_argument("--batch-scale", type=int, default=20)
    ap.add_argument("--bc-sources", type=int, default=BC_SOURCES, help="sampled BC sources at the main scale")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-reorder", action="store_true", help="keep the generated vertex order")
    ap.add_argument("--only", default="", help="comma-separated subset of the suite (profiling runs)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--partitioned", action="store_true",
                    help="also run the 1D-partitioned BFS/PageRank over the ranks (always at one GPU)")
    ap.add_argument("--dry-run", action="store_true", help="rank plumbing only, on the host (gloo), no GPU")
    ap.add_argument("--launch-timeout", type=int, default=3600)
    args = ap.parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ and args.impl == "ours":
        return spawn_ranks(args)
    rank, world, local_rank = env_int("RANK", 0), env_int("WORLD_SIZE", 1), env_int("LOCAL_RANK", 0)
    if args.dry_run:
        return run_dry(args, rank, world)
    if args.impl == "reference":
        return run_reference_arm(args, rank, world)
    if world > 1:
        import datetime

        import torch.distributed as tdist

        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        return run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as tdist

            tdist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
