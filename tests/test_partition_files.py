"""The offline edge partitioner (gre_partition_edges, host only) against the reference's own
(Graph/GraphIngress.hpp EdgePartition::divideEdges, compiled from the reference's headers into
oracle/_ref/ref_graphpar as usr/debug/test_graphPar.cpp drives it), on the same edge lists:

* <prefix>.part.P.r (the edges of each part, in decision order) and <prefix>.outdegree.P.p equal
  the reference's byte for byte;
* <prefix>.scatterMap.P.p equal it except for the bytes the reference writes from past the end of
  its bitmap allocation (the last count / 8 + 8 - 8 * (count / 64 + 1) bytes of each map);
* the parts together hold every edge of the lists exactly once.
"""
import os
import subprocess

import numpy as np
import pytest

import graphine_b200.gre as G

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "ref_graphpar")


def _edges(prefix, nfiles):
    out = []
    for i in range(nfiles):
        for line in open(f"{prefix}.edges.{i}"):
            if line.strip() and not line.startswith("#"):
                u, v = line.split()[:2]
                out.append((int(u), int(v)))
    return out


def _scatter_defined(data, bits, nmaps):
    """The defined bytes of a scatter-map file: each map's 8-byte count and its whole words."""
    size = bits // 8 + 8
    keep = 8 * (bits // 64 + 1)
    assert len(data) == nmaps * (8 + size)
    return b"".join(data[k * (8 + size):k * (8 + size) + 8 + keep] for k in range(nmaps))


@pytest.mark.parametrize("P", [1, 2, 3, 5, 8])
@pytest.mark.parametrize("sym", [True, False], ids=["sym", "dir"])
def test_partition_files_equal_reference(tmp_path, P, sym):
    if not os.path.exists(REF):
        pytest.skip("reference partitioner not built (no reference tree)")
    n, off, col = G.rmat_host(10, 8, 3 + P, sym)
    ours, ref = tmp_path / "ours", tmp_path / "ref"
    ours.mkdir()
    ref.mkdir()
    for d in (ours, ref):
        G.write_edgelists(str(d / "g"), n, off, col, 4)
    counts = G.partition_edges(str(ours / "g"), P)
    subprocess.run([REF, str(ref / "g"), str(P)], check=True, capture_output=True, timeout=300)
    assert int(counts.sum()) == len(col)
    bits = n // P + (1 if n % P else 0)
    for r in range(P):
        a, b = ours / f"g.part.{P}.{r}", ref / f"g.part.{P}.{r}"
        assert a.exists() == b.exists(), r
        if a.exists():
            assert a.read_bytes() == b.read_bytes(), f"part {r}"
            assert a.stat().st_size == 16 * int(counts[r])
        else:
            assert counts[r] == 0
        assert (ours / f"g.outdegree.{P}.{r}").read_bytes() == (ref / f"g.outdegree.{P}.{r}").read_bytes()
        sa = (ours / f"g.scatterMap.{P}.{r}").read_bytes()
        sb = (ref / f"g.scatterMap.{P}.{r}").read_bytes()
        assert len(sa) == len(sb)
        assert _scatter_defined(sa, bits, P - 1) == _scatter_defined(sb, bits, P - 1), f"scatter map {r}"
    # every edge of the lists in exactly one part
    got = []
    for r in range(P):
        f = ours / f"g.part.{P}.{r}"
        if f.exists():
            got.extend(map(tuple, np.fromfile(f, dtype=np.uint64).reshape(-1, 2).tolist()))
    assert sorted(got) == sorted(_edges(str(ours / "g"), 4))


def test_partition_edges_errors(tmp_path):
    n, off, col = G.rmat_host(6, 4, 1, True)
    G.write_edgelists(str(tmp_path / "g"), n, off, col, 2)
    for bad in (0, 65):
        with pytest.raises(G.GreError) as e:
            G.partition_edges(str(tmp_path / "g"), bad)
        assert e.value.status == G.GRE_INVALID_ARG
    with pytest.raises(G.GreError) as e:
        G.partition_edges(str(tmp_path / "missing"), 2)
    assert e.value.status == G.GRE_IO_ERROR
    with open(tmp_path / "g.edges.0", "a") as f:  # a vertex id past the .meta count
        f.write(f"{n} 0\n")
    with pytest.raises(G.GreError) as e:
        G.partition_edges(str(tmp_path / "g"), 2)
    assert e.value.status == G.GRE_INVALID_ARG


def test_cpp_mirror_drives_the_partitioner(tmp_path):
    """A driver written as usr/debug/test_graphPar.cpp (EdgePartition par; par.divideEdges(prefix,
    n)) compiles against the C++ mirror include/gre/gre.hpp and writes the same parts as
    gre_partition_edges."""
    import shutil

    if not shutil.which("g++"):
        pytest.skip("no host C++ compiler")
    src = tmp_path / "graphpar.cpp"
    src.write_text(
        '#include "gre/gre.hpp"\n#include <cstdlib>\n'
        "int main(int argc, char** argv) {\n"
        "  gre::EdgePartition par;\n"
        "  par.divideEdges(argv[1], atoi(argv[2]));\n"
        "  return 0;\n}\n")
    exe = tmp_path / "graphpar"
    libdir = os.path.join(ROOT, "graphine_b200")
    subprocess.run(["g++", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include", str(src),
                    "-L", libdir, "-lgre_gpu", f"-Wl,-rpath,{libdir}", "-o", str(exe)], check=True, capture_output=True,
                   timeout=300)
    n, off, col = G.rmat_host(9, 8, 11, True)
    a, b = tmp_path / "a", tmp_path / "b"
    a.mkdir()
    b.mkdir()
    for d in (a, b):
        G.write_edgelists(str(d / "g"), n, off, col, 3)
    subprocess.run([str(exe), str(a / "g"), "4"], check=True, capture_output=True, timeout=300)
    G.partition_edges(str(b / "g"), 4)
    for r in range(4):
        assert (a / f"g.part.4.{r}").read_bytes() == (b / f"g.part.4.{r}").read_bytes()
