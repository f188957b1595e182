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
