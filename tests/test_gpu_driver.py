"""The drop-in driver graphine_b200/drivers/gre_run (the reference's usr/test_*.cpp on this
library, through the C++ mirror include/gre/gre.hpp): run on the golden graphs' text files, its
per-superstep lines must equal the reference engine's active counts."""
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

import graphine_b200.gre as G
import oracle as O

pytestmark = pytest.mark.gpu

DRIVER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "graphine_b200", "drivers", "gre_run")


def run_driver(algo, prefix, env=None):
    p = subprocess.run([DRIVER, algo, prefix, "ascii", "edgelists"], capture_output=True, text=True, timeout=300,
                       env={**os.environ, **(env or {})})
    assert p.returncode == 0, p.stderr
    return [int(x) for x in re.findall(r"Superstep-\d+: Number of active vertices\.\.\.(\d+)", p.stdout)], p.stdout


def strip(a):
    return [int(x) for x in a if x >= 0]


@pytest.mark.parametrize("name", ["rmat_s10_sym", "toy_edge_cases"])
def test_driver_matches_reference_supersteps(golden, name):
    case = golden[name]
    n = int(case["n"])
    with tempfile.TemporaryDirectory() as td:
        prefix = os.path.join(td, "g")
        G.write_edgelists(prefix, n, case["off"], case["col"], 4)
        G.write_roots(prefix, case["roots"])
        env = {"GRE_WSEED": str(int(case["wseed"]))}
        assert run_driver("pagerank", prefix)[0] == list(case["pr_gre10_active"])
        assert run_driver("pagerank_iter", prefix)[0] == list(case["pr_iter20_active"])
        assert run_driver("pagerank_delta", prefix)[0] == list(case["prdelta_active"])
        assert run_driver("bfs", prefix)[0] == strip(case["bfs_active"][0])
        assert run_driver("sssp", prefix, env)[0] == strip(case["sssp_active"][0])
        assert run_driver("sssp1", prefix, env)[0] == strip(case["sssp1_active"][0])
        assert run_driver("cc", prefix)[0] == list(case["cc_active"])
        counts, out = run_driver("cin", prefix)
        assert counts == list(case["countin_active"])
        assert f"Number of in edges: {int(case['countin'].astype(np.int64).sum())}" in out


def test_driver_reports_bad_input_with_status():
    with tempfile.TemporaryDirectory() as td:
        p = subprocess.run([DRIVER, "cc", os.path.join(td, "absent")], capture_output=True, text=True, timeout=60)
        assert p.returncode == G.GRE_IO_ERROR


def test_partitioned_driver_one_rank(golden):
    case = golden["rmat_s10_sym"]
    n = int(case["n"])
    with tempfile.TemporaryDirectory() as td:
        prefix = os.path.join(td, "g")
        G.write_edgelists(prefix, n, case["off"], case["col"], 4)
        G.write_roots(prefix, case["roots"])
        idf = os.path.join(td, "nccl.id")
        args = ["--ranks", "1", "--rank", "0", "--id-file", idf]
        p = subprocess.run([DRIVER, "part_bfs", prefix] + args, capture_output=True, text=True, timeout=300)
        assert p.returncode == 0, p.stderr
        counts = [int(x) for x in re.findall(r"Superstep-\d+: Number of active vertices\.\.\.(\d+)", p.stdout)]
        g = G.Graph.ingress(prefix, dir=G.InOut)
        lv, st = G.bfs(g, [int(case["roots"][0])])
        assert counts == st.active
        assert f"Reached vertices: {int((lv >= 0).sum())}" in p.stdout
        p = subprocess.run([DRIVER, "part_pagerank_iter", prefix] + args, capture_output=True, text=True, timeout=300)
        assert p.returncode == 0, p.stderr
        pr, _ = G.pagerank(G.Graph.ingress(prefix, dir=G.Out), G.PR_ITER, 0.85, 20)
        s = 0.0
        for x in pr:  # the driver's order of summation
            s += float(x)
        assert f"Sum of pr: {s:.15g}" in p.stdout
        wseed = int(case["wseed"])
        p = subprocess.run([DRIVER, "part_sssp", prefix] + args, capture_output=True, text=True, timeout=300,
                           env={**os.environ, "GRE_WSEED": str(wseed)})
        assert p.returncode == 0, p.stderr
        gs = G.Graph.ingress(prefix, dir=G.Out)
        gs.set_weights_hash(wseed)
        d, _ = G.sssp(gs, [int(case["roots"][0])])
        fin = d[d != 0xFFFFFFFF].astype(np.int64)
        assert f"Reached vertices: {len(fin)}" in p.stdout and f"Sum of distances: {int(fin.sum())}" in p.stdout
        p = subprocess.run([DRIVER, "part_cc", prefix] + args, capture_output=True, text=True, timeout=300)
        assert p.returncode == 0, p.stderr
        lab, _ = G.cc(g)
        assert f"Number of components: {int((lab == np.arange(n)).sum())}" in p.stdout


def test_driver_ingress_from_saved_partitions():
    """`gre_run <algo> <prefix> ascii partition P` reads the saved partitions <prefix>.part.P.<r>
    (the reference's ingress method "partition", GraphIngress.hpp:86-96, 1024-1071) instead of the
    edge-list text, and runs as on the same graph loaded from text."""
    n, off, col = G.rmat_host(11, 8, 4, True)
    src = np.repeat(np.arange(n, dtype=np.int64), np.diff(off.astype(np.int64)))
    cut = np.random.default_rng(2).integers(0, 3, len(col))
    with tempfile.TemporaryDirectory() as td:
        prefix = os.path.join(td, "p")
        open(prefix + ".meta", "w").write(f"{n} {len(col)}\n")
        for r in range(3):
            pairs = np.stack([src[cut == r], col[cut == r].astype(np.int64)], axis=1).astype(np.uint64)
            pairs.tofile(prefix + f".part.3.{r}")
        p = subprocess.run([DRIVER, "cc", prefix, "ascii", "partition", "3"], capture_output=True, text=True, timeout=300)
        assert p.returncode == 0, p.stderr
        p2 = subprocess.run([DRIVER, "bfs", prefix, "ascii", "partitions", "3"], capture_output=True, text=True,
                            timeout=300)
        assert p2.returncode != 0  # no .roots file: the reference driver's message and a status
        assert "Err in reading src vertex" in p2.stderr
    lab, _ = O.Restatement.from_csr(n, off, col).cc()
    assert f"Number of components: {int((lab == np.arange(n)).sum())}" in p.stdout
