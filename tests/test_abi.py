"""The C ABI library: loads, exports every symbol include/gre_gpu.h declares, reports errors
with status codes (never exits), and its host-only utilities work without a GPU."""
import ctypes
import os
import re
import tempfile

import numpy as np
import pytest

import graphine_b200.gre as G
import oracle as O
from conftest import ROOT


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "gre_gpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gre_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_declared_symbols():
    lib = G.lib()
    syms = declared_symbols()
    assert len(syms) >= 30
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_status_strings_mirror_reference_parser():
    # GRE_Status_Parser words (include/Status.hpp:17-30), spelled correctly here
    assert G.status_str(0) == "success"
    assert G.status_str(G.GRE_NOT_IMPLEMENTED) == "not_implemented"
    assert G.status_str(G.GRE_TIMEOUT) == "timeout"
    assert G.status_str(999) == "unknown_status"


def test_missing_files_are_io_errors():
    with tempfile.TemporaryDirectory() as td:
        with pytest.raises(G.GreError) as e:
            G.Graph.ingress(os.path.join(td, "absent"))
        assert e.value.status == G.GRE_IO_ERROR


def test_garbled_meta_rejected_before_any_device_work():
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "bad")
        open(p + ".edges.0", "w").write("0 1\n")
        open(p + ".meta", "w").write("garbage\n")
        with pytest.raises(G.GreError) as e:
            G.Graph.ingress(p)
        assert e.value.status == G.GRE_IO_ERROR
        open(p + ".meta", "w").write("0 1\n")  # no vertices
        with pytest.raises(G.GreError) as e:
            G.Graph.ingress(p)
        assert e.value.status == G.GRE_INVALID_ARG


def test_no_device_is_reported_not_fatal():
    if G.device_count() > 0:
        pytest.skip("a GPU is present")
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "ok")
        open(p + ".meta", "w").write("3 2\n")
        open(p + ".edges.0", "w").write("0 1\n1 2\n")
        with pytest.raises(G.GreError) as e:
            G.Graph.ingress(p)
        assert e.value.status == G.GRE_NO_DEVICE


def test_rmat_host_is_deterministic_and_clean():
    n, off, col = G.rmat_host(9, 16, 5, True)
    n2, off2, col2 = G.rmat_host(9, 16, 5, True)
    np.testing.assert_array_equal(off, off2)
    np.testing.assert_array_equal(col, col2)
    src = np.repeat(np.arange(n, dtype=np.uint64), np.diff(off).astype(np.int64))
    assert np.all(src != col)  # no self loops
    key = src * n + col
    assert np.all(np.diff(key) > 0)  # sorted, no duplicates
    # symmetric: the reverse of every arc is present
    rkey = np.sort(col.astype(np.uint64) * n + src)
    np.testing.assert_array_equal(rkey, key)
    n3, off3, col3 = G.rmat_host(9, 16, 6, True)
    assert not (len(col3) == len(col) and np.array_equal(col3, col))


def test_rmat_directed_has_no_reverse_requirement():
    n, off, col = G.rmat_host(9, 16, 5, False)
    assert off[-1] == len(col) and len(col) <= 16 * n


def test_roots_roundtrip_and_reference_format():
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "g")
        G.write_roots(p, [5, 7, 11])
        assert open(p + ".roots").read().split() == ["3", "5", "7", "11"]
        np.testing.assert_array_equal(G.read_roots(p), [5, 7, 11])


def test_edgelists_split_by_source_modulo():
    n, off, col = G.rmat_host(8, 8, 2, True)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "g")
        G.write_edgelists(p, n, off, col, 4)
        assert open(p + ".meta").read().split() == [str(n), str(len(col))]
        for i in range(4):
            for line in open(f"{p}.edges.{i}"):
                assert int(line.split()[0]) % 4 == i
        R = O.Restatement.load(p)
        o2, c2 = R.csr()
        np.testing.assert_array_equal(o2, off)
        np.testing.assert_array_equal(c2, col)
