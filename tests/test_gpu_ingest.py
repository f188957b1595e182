"""Device-side ingress (graphine_b200/csrc/ingest.cu): <prefix>.meta + <prefix>.edges.<i> parsed
on the GPU must give the CSR a line-by-line reader gives (file order within a source, files in
index order) and the same error codes, including when lines straddle the streaming chunks."""
import os
import tempfile

import numpy as np
import pytest

import graphine_b200.gre as G
import oracle as O

pytestmark = pytest.mark.gpu


def reader_csr(n, texts):
    """The loader's rules, line by line: blank and '#' lines skipped, a trailing CR ignored."""
    src, dst = [], []
    for t in texts:
        for line in t.split("\n"):
            line = line[:-1] if line.endswith("\r") else line
            if not line or line[0] == "#":
                continue
            u, v = line.split()
            src.append(int(u))
            dst.append(int(v))
    order = np.argsort(np.array(src, dtype=np.int64), kind="stable")
    off = np.zeros(n + 1, np.uint64)
    np.add.at(off, np.array(src, dtype=np.int64) + 1, 1)
    return np.cumsum(off).astype(np.uint64), np.array(dst, dtype=np.uint32)[order]


def write(td, n, texts):
    p = os.path.join(td, "g")
    open(p + ".meta", "w").write(f"{n} 0\n")
    for i, t in enumerate(texts):
        open(p + f".edges.{i}", "w", newline="").write(t)
    return p


def messy_texts(n, seed):
    rng = np.random.default_rng(seed)
    texts = []
    for f in range(3):
        lines = []
        for _ in range(int(rng.integers(200, 400))):
            r = rng.random()
            if r < 0.05:
                lines.append("# a comment 1 2")
            elif r < 0.08:
                lines.append("")
            else:
                u, v = rng.integers(0, n, 2)
                sep = " " * int(rng.integers(1, 4)) if rng.random() < 0.8 else "\t"
                lead = " " if rng.random() < 0.1 else ""
                tail = "\r" if rng.random() < 0.1 else (" " if rng.random() < 0.1 else "")
                lines.append(f"{lead}{u}{sep}{v}{tail}")
        t = "\n".join(lines)
        texts.append(t if f == 1 else t + "\n")  # file 1 ends without a newline
    return texts


@pytest.mark.parametrize("chunk", [None, "64", "100", "4096"])
def test_device_parse_matches_line_reader(monkeypatch, chunk):
    if chunk:
        monkeypatch.setenv("GRE_INGEST_CHUNK", chunk)
    n = 500
    texts = messy_texts(n, 3)
    with tempfile.TemporaryDirectory() as td:
        g = G.Graph.ingress(write(td, n, texts), G.InOut)
    off, col = g.csr()
    ref_off, ref_col = reader_csr(n, texts)
    np.testing.assert_array_equal(off, ref_off)
    np.testing.assert_array_equal(col, ref_col)


@pytest.mark.parametrize("chunk", [None, "64"])
@pytest.mark.parametrize("text,status", [
    ("0 1\n1 x\n", G.GRE_IO_ERROR),
    ("0 1\n1 9\n", G.GRE_INVALID_ARG),          # vertex 9 >= n = 4
    ("0 1\n1 2 3\n", G.GRE_IO_ERROR),           # a third token
    ("0 1\n  \n", G.GRE_IO_ERROR),              # spaces only
    ("0 1\n 2\n", G.GRE_IO_ERROR),
    ("0 99999999999\n1 x\n", G.GRE_INVALID_ARG),  # the first bad line decides
    ("1 x\n0 99999999999\n", G.GRE_IO_ERROR),
])
def test_bad_lines_rejected_with_loader_codes(monkeypatch, chunk, text, status):
    if chunk:
        monkeypatch.setenv("GRE_INGEST_CHUNK", chunk)
    with tempfile.TemporaryDirectory() as td:
        p = write(td, 4, ["0 1\n" * 50 + text])
        with pytest.raises(G.GreError) as e:
            G.Graph.ingress(p)
        assert e.value.status == status


def test_line_longer_than_a_chunk_is_an_io_error(monkeypatch):
    monkeypatch.setenv("GRE_INGEST_CHUNK", "64")
    with tempfile.TemporaryDirectory() as td:
        p = write(td, 4, ["0 1\n" + "0" * 100 + "1 2\n"])
        with pytest.raises(G.GreError) as e:
            G.Graph.ingress(p)
        assert e.value.status == G.GRE_IO_ERROR


def test_empty_and_comment_only_files():
    with tempfile.TemporaryDirectory() as td:
        g = G.Graph.ingress(write(td, 3, ["", "# nothing\n\n", "2 0"]), G.InOut)
    off, col = g.csr()
    np.testing.assert_array_equal(off, [0, 0, 0, 1])
    np.testing.assert_array_equal(col, [0])


def test_rmat_text_round_trip_relabelled():
    n, off, col = G.rmat_host(14, 16, 21, True)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "r")
        G.write_edgelists(p, n, off, col, 4)
        g = G.Graph.ingress(p, G.InOut, symmetric=True, reorder=True)
    o2, c2 = g.csr()
    np.testing.assert_array_equal(o2, off)
    np.testing.assert_array_equal(c2, col)


def write_parts(td, n, parts):
    p = os.path.join(td, "p")
    open(p + ".meta", "w").write(f"{n} {sum(len(x) for x in parts)}\n")
    for r, pairs in enumerate(parts):
        np.asarray(pairs, dtype=np.uint64).reshape(-1, 2).tofile(p + f".part.{len(parts)}.{r}")
    return p


@pytest.mark.parametrize("chunk", [None, "64"])
def test_saved_partitions_merge_in_rank_order(monkeypatch, chunk):
    if chunk:
        monkeypatch.setenv("GRE_INGEST_CHUNK", chunk)
    n, off, col = G.rmat_host(12, 8, 4, True)
    src = np.repeat(np.arange(n, dtype=np.int64), np.diff(off.astype(np.int64)))
    rank = np.random.default_rng(1).integers(0, 3, len(col))  # an arbitrary edge cut
    parts = [np.stack([src[rank == r], col[rank == r].astype(np.int64)], axis=1) for r in range(3)]
    with tempfile.TemporaryDirectory() as td:
        g = G.Graph.load_parts(write_parts(td, n, parts), 3, G.InOut, symmetric=True)
    allp = np.concatenate(parts)
    order = np.argsort(allp[:, 0], kind="stable")
    o2, c2 = g.csr()
    np.testing.assert_array_equal(o2, off)
    np.testing.assert_array_equal(c2, allp[order, 1].astype(np.uint32))
    R = O.Restatement.from_csr(n, off, col)
    np.testing.assert_array_equal(G.cc(g)[0], R.cc()[0])


def test_saved_partitions_errors():
    with tempfile.TemporaryDirectory() as td:
        p = write_parts(td, 4, [[[0, 1]], [[1, 9]]])  # vertex 9 >= n
        with pytest.raises(G.GreError) as e:
            G.Graph.load_parts(p, 2)
        assert e.value.status == G.GRE_INVALID_ARG
        with pytest.raises(G.GreError) as e:
            G.Graph.load_parts(p, 3)  # p.part.3.* missing
        assert e.value.status == G.GRE_IO_ERROR
        open(p + ".part.2.1", "ab").write(b"\x00" * 8)  # not whole pairs
        with pytest.raises(G.GreError) as e:
            G.Graph.load_parts(p, 2)
        assert e.value.status == G.GRE_IO_ERROR
        with pytest.raises(G.GreError) as e:
            G.Graph.load_parts(p, 0)
        assert e.value.status == G.GRE_INVALID_ARG


@pytest.mark.parametrize("P", [2, 3])
def test_partitioner_output_loads_as_the_graph(P):
    """Edge lists split by gre_partition_edges (the reference's offline partitioner) load back
    through gre_graph_load_parts as the same graph: the merged CSR holds the parts' edges in rank
    order, and BFS / CC on it equal the oracle's on the original edge lists."""
    n, off, col = G.rmat_host(11, 8, 9, True)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "g")
        G.write_edgelists(p, n, off, col, 4)
        counts = G.partition_edges(p, P)
        assert int(counts.sum()) == len(col) and (counts > 0).all()
        parts = [np.fromfile(p + f".part.{P}.{r}", dtype=np.uint64).reshape(-1, 2) for r in range(P)]
        g = G.Graph.load_parts(p, P, G.InOut, symmetric=True)
    allp = np.concatenate(parts).astype(np.int64)
    order = np.argsort(allp[:, 0], kind="stable")
    o2, c2 = g.csr()
    np.testing.assert_array_equal(o2, off)
    np.testing.assert_array_equal(c2, allp[order, 1].astype(np.uint32))
    R = O.Restatement.from_csr(n, off, col)
    roots = G.sample_sources(off, 2, 1)
    np.testing.assert_array_equal(G.bfs(g, roots)[0].reshape(2, n), R.bfs_many(roots))
    np.testing.assert_array_equal(G.cc(g)[0], R.cc()[0])
