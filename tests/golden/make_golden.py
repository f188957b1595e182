"""Generate the golden fixtures of tests/golden/ by running the reference GRE engine.

Run in a checkout that has the reference tree (compiled into oracle/_ref/ by `make -C oracle`):

    python tests/golden/make_golden.py

For each case the input graph is produced by this project's seeded RMAT generator (or written
by hand for the edge cases), stored as CSR so the generator itself is pinned too, and every
output of the reference drivers (oracle/ref_drivers/) is stored next to it together with the
per-superstep active counts the reference engine prints.  The fixtures are small (S8 and S10)
so the CPU test suite can check the oracle restatement against them in seconds.
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import graphine_b200.gre as G  # noqa: E402
import oracle as O  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
WSEED = 20240601
PR_SUPERSTEPS = 20


def _pad(runs):
    k = max((len(r) for r in runs), default=0)
    a = np.full((len(runs), k), -1, dtype=np.int64)
    for i, r in enumerate(runs):
        a[i, : len(r)] = r
    return a


def write_case(name: str, n: int, off: np.ndarray, col: np.ndarray, roots: np.ndarray, symmetric: bool, edge_text=None):
    with tempfile.TemporaryDirectory() as td:
        prefix = os.path.join(td, name)
        if edge_text is None:
            G.write_edgelists(prefix, n, off, col, 4)
        else:
            with open(prefix + ".meta", "w") as f:
                f.write(f"{n} {len(col)}\n")
            for i, text in enumerate(edge_text):
                with open(f"{prefix}.edges.{i}", "w") as f:
                    f.write(text)
        G.write_roots(prefix, roots)
        res = {"n": np.uint64(n), "off": off, "col": col, "roots": roots, "symmetric": np.bool_(symmetric),
               "wseed": np.uint64(WSEED)}
        pr, run = O.run_reference("pagerank", prefix, "gre", 10)
        res["pr_gre10"], res["pr_gre10_active"] = pr, np.array(run.active[0])
        pr, run = O.run_reference("pagerank", prefix, "iter", PR_SUPERSTEPS)
        res["pr_iter20"], res["pr_iter20_active"] = pr, np.array(run.active[0])
        pp, _ = O.run_reference("pagerank", prefix, "ppr", PR_SUPERSTEPS, *[int(r) for r in roots[:2]])
        res["ppr20"] = pp.reshape(-1, n)
        pr, run = O.run_reference("pagerank", prefix, "delta", 1024)
        res["prdelta"], res["prdelta_active"] = pr, np.array(run.active[0])
        if symmetric:
            lv, run = O.run_reference("bfs", prefix)
            assert "GRE_BFS_REACH_MISMATCH" not in run.stdout
            res["bfs_level"] = lv.reshape(-1, n)
            res["bfs_active"] = _pad(run.active[0::2])  # runs alternate: BFS plugin, Forward levels
            dist, run = O.run_reference("sssp", prefix, WSEED)
            res["sssp_dist"], res["sssp_active"] = dist.reshape(-1, n), _pad(run.active)
            raw, run = O.run_reference("sssp1", prefix, WSEED)
            per = 12 * n  # n uint32 distances then n uint64 predecessors per root
            res["sssp1_dist"] = np.stack([raw[i * per:i * per + 4 * n].view(np.uint32) for i in range(len(roots))])
            res["sssp1_pred"] = np.stack([raw[i * per + 4 * n:(i + 1) * per].view(np.uint64) for i in range(len(roots))])
            res["sssp1_active"] = _pad(run.active)
            cnt, run = O.run_reference("countin", prefix)
            res["countin"], res["countin_active"] = cnt, np.array(run.active[0])
            lab, run = O.run_reference("cc", prefix)
            res["cc_label"], res["cc_active"] = lab, np.array(run.active[0])
            b, run = O.run_reference("bc", prefix)
            assert "GRE_BC_OVERFLOW" not in run.stdout
            res["bc"] = b
    np.savez_compressed(os.path.join(OUT, f"{name}.npz"), **res)
    print(f"wrote {name}.npz  n={n} m={len(col)}")


def csr_from_edges(n, edges):
    src = np.array([e[0] for e in edges], dtype=np.uint32)
    dst = np.array([e[1] for e in edges], dtype=np.uint32)
    order = np.argsort(src, kind="stable")
    off = np.zeros(n + 1, dtype=np.uint64)
    np.add.at(off, src.astype(np.int64) + 1, 1)
    return np.cumsum(off).astype(np.uint64), dst[order]


def main():
    if not O.reference_available():
        sys.exit("oracle/_ref binaries missing: run `make -C oracle` where the reference tree exists")
    for scale, sym, seed in [(8, True, 7), (10, True, 7), (10, False, 3)]:
        n, off, col = G.rmat_host(scale, 16, seed, sym)
        roots = G.sample_sources(off, 4, 11)
        write_case(f"rmat_s{scale}_{'sym' if sym else 'dir'}", n, off, col, roots, sym)

    # Edge cases written as text the way a user would: comments, blank lines, a duplicate
    # arc, a self loop, isolated vertices and a second component; files split by source.
    n = 12
    edges = [(0, 1), (1, 0), (1, 2), (2, 1), (2, 3), (3, 2), (0, 3), (3, 0), (3, 3), (4, 5), (5, 4), (0, 1), (1, 0),
             (6, 7), (7, 6), (7, 8), (8, 7)]
    text = ["", "", "", ""]
    for u, v in edges:
        text[u % 4] += f"{u} {v}\n"
    text[0] = "# GRE edge list with comments\n\n" + text[0]
    text[1] = text[1].rstrip("\n")  # last line without newline
    # CSR in the order the reference reads: files 0..3, lines in order
    ordered = []
    for i in range(4):
        for line in text[i].splitlines():
            if line and not line.startswith("#"):
                a, b = line.split()
                ordered.append((int(a), int(b)))
    off, col = csr_from_edges(n, ordered)
    write_case("toy_edge_cases", n, off, col, np.array([0, 4, 6, 9], dtype=np.uint32), True, edge_text=text)


if __name__ == "__main__":
    main()
