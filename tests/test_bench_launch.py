"""bench.py's launch paths on the host (no GPU).

* `--gpus N` without a launcher starts N ranks itself; `--dry-run` runs the rank plumbing over
  gloo (barrier, max-over-ranks time, sum of work) and rank 0 reports n_gpus = N.
* `--impl reference` runs the reference engine's binaries on a small sample, reports the same
  `config` as the GPU arm, records the host, and never loads the product library.
"""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BENCH = os.path.join(ROOT, "bench.py")


def last_json(out: str) -> dict:
    lines = [ln for ln in out.splitlines() if ln.startswith("{")]
    assert lines, out
    return json.loads(lines[-1])


@pytest.mark.parametrize("gpus", [1, 2])
def test_gpus_flag_spawns_ranks(gpus):
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    p = subprocess.run([sys.executable, BENCH, "--gpus", str(gpus), "--dry-run", "--steps", "2", "--warmup", "3"],
                       capture_output=True, text=True, timeout=300, env=env, cwd=ROOT)
    assert p.returncode == 0, p.stderr[-3000:]
    line = last_json(p.stdout)
    assert line["dry_run"] and line["n_gpus"] == gpus and line["ranks_reporting"] == gpus
    assert line["config"]["parallelism"] == f"replica x{gpus}"


def test_reference_arm_same_config_and_no_product_library():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    if not O.reference_available():
        pytest.skip("reference binaries not built (oracle/_ref)")
    code = (
        "import sys, runpy\n"
        f"sys.argv = ['bench.py', '--impl', 'reference', '--ref-scale', '10', '--steps', '2', '--warmup', '1']\n"
        "try:\n"
        f"    runpy.run_path({BENCH!r}, run_name='__main__')\n"
        "except SystemExit as e:\n"
        "    assert not e.code, e.code\n"
        "maps = open('/proc/self/maps').read()\n"
        "print('PRODUCT_LOADED', 'libgre_gpu.so' in maps)\n"
    )
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert p.returncode == 0, p.stderr[-3000:]
    assert "PRODUCT_LOADED False" in p.stdout
    line = last_json(p.stdout)
    sys.path.insert(0, ROOT)
    import bench

    assert line["impl"] == "reference" and line["config"] == bench.workload_config(26, 1)
    assert line["value"] > 0 and line["steps"] == 2
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] == bench.REF_THREADS
    assert cb["host"]["nproc"] >= 1 and "RMAT-10" in cb["sample"]
    assert set(line["per_algorithm"]) == {"pagerank", "bfs", "sssp", "cc"}
