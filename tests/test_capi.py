"""CPU tests of the C-ABI boundary: the library loads, exports every entry point that
include/jgpm.h declares, and reports errors as status codes (no compute without a GPU)."""
import ctypes
import os
import re

import numpy as np
import pytest

import jupiter_b200 as J

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\**\s*(jgpm_[A-Za-z0-9_]+)\s*\(",
                             text, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_library_built_in_tree():
    assert os.path.exists(J.library_path())
    assert J.library_path().startswith(os.path.join(ROOT, "jupiter_b200"))


def test_every_declared_symbol_is_exported():
    L = J.lib()
    names = declared_symbols()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_version_and_error_string():
    assert "sm_100a" in J.version()
    assert isinstance(J.lib().jgpm_last_error(), bytes)


def test_status_codes_match_header():
    text = open(os.path.join(ROOT, "include", "jgpm.h")).read()
    for m in re.finditer(r"#define (JGPM_E[A-Z]+|JGPM_OK)\s+\(?(-?\d+)\)?", text):
        assert J.STATUS[int(m.group(2))] == m.group(1)
    for name, val in (("JGPM_OP_INTERSECT", J.OP_INTERSECT), ("JGPM_OP_DIFFERENCE_COUNT",
                                                                J.OP_DIFFERENCE_COUNT),
                      ("JGPM_COUNT_STATS", J.COUNT_STATS), ("JGPM_COUNT_FORCE_ENUM",
                                                             J.COUNT_FORCE_ENUM)):
        assert re.search(rf"#define {name} {val}u?\b", text), name


def test_bad_arguments_are_status_codes():
    L = J.lib()
    assert L.jgpm_graph_get_info(None, None) == -1
    assert L.jgpm_count_ex(None, b"P1", 0, 1, 0, None, None) == -1
    assert L.jgpm_graph_load(None, 0, None) == -1
    n = ctypes.c_int64()
    assert L.jgpm_rmat_edges(1, 10, 0.5, 0.2, 0.2, 1, None, None, ctypes.byref(n)) == -1
    assert L.jgpm_rmat_edges(100, 10, 0.7, 0.2, 0.2, 1, None, None, ctypes.byref(n)) == -1


@pytest.mark.skipif(J.device_count() > 0, reason="checks the no-device path")
def test_no_device_fails_loudly():
    with pytest.raises(J.JgpmError) as e:
        J.Graph.rmat(1024, 4)
    assert e.value.code == -8  # JGPM_ENODEV
    with pytest.raises(J.JgpmError):
        J.setop(J.OP_INTERSECT_COUNT, [1, 2, 3], [2, 3])
    with pytest.raises(J.JgpmError) as e:
        J.setop_split(J.SPLIT_FUSE, [1, 2, 3], [2, 3])
    assert e.value.code == -8


def test_host_rmat_edges_deterministic():
    s1, d1 = J.rmat_edges(5000, 20000, 0.57, 0.19, 0.19, 9)
    s2, d2 = J.rmat_edges(5000, 20000, 0.57, 0.19, 0.19, 9)
    assert (s1 == s2).all() and (d1 == d2).all()
    assert len(s1) == 20000 and s1.max() < 5000 and s1.min() >= 0
    s3, _ = J.rmat_edges(5000, 20000, 0.57, 0.19, 0.19, 10)
    assert not (s1 == s3).all()


def test_split_arguments_checked_before_the_device():
    L = J.lib()
    one = np.zeros(2, dtype=np.int64)
    cnt = np.zeros(1, dtype=np.int32)
    p64 = one.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
    p32 = cnt.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
    assert L.jgpm_setop_split_batch(7, None, p64, None, p64, 1, None, p32, None, None,
                                    None) == -1
    assert L.jgpm_setop_split_batch(J.SPLIT_FUSE, None, None, None, p64, 1, None, p32, None,
                                    None, None) == -1
    assert L.jgpm_setop_split(J.SPLIT_DIF_INT, None, -1, None, 0, 0, None, None, None,
                              p32) == -1
    text = open(os.path.join(ROOT, "include", "jgpm.h")).read()
    assert re.search(rf"#define JGPM_SPLIT_FUSE {J.SPLIT_FUSE}\b", text)
    assert re.search(rf"#define JGPM_SPLIT_DIF_INT {J.SPLIT_DIF_INT}\b", text)


def test_cli_usage_and_loud_failure_without_a_device(tmp_path):
    """The reference CLI's counterpart: usage on no arguments, and a status message with a
    non-zero exit when there is no device (no CPU fallback)."""
    import subprocess
    import sys
    cli = os.path.join(ROOT, "jupiter_b200", "jupiter_gpm")
    assert os.path.exists(cli)
    r = subprocess.run([cli], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "Usage:" in r.stdout and "[pattern(P1)]" in r.stdout
    if J.device_count() > 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_api as O
    g = O.rmat_graph(500, 4, 0.57, 0.19, 0.19, 3)
    prefix = str(tmp_path / "graph")
    O.write_reference_files(g, prefix)
    r = subprocess.run([cli, prefix, "P1"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "status -8" in (r.stdout + r.stderr)
    assert "gpu count" not in r.stdout


def test_every_entry_point_cites_its_reference_interface():
    """Each declaration in include/*.h is preceded by a comment that cites the reference file
    it replaces (path, usually with lines) or says it has no reference counterpart."""
    pat = re.compile(r"(/\*(?:(?!\*/).)*\*/\s*)?((?:#define[^\n]*\n\s*)*)(?:const\s+)?"
                     r"[A-Za-z_][A-Za-z0-9_]*\s*\**\s*(jgpm_[A-Za-z0-9_]+)\s*\(", re.S)
    missing, seen = [], 0
    for h in os.listdir(os.path.join(ROOT, "include")):
        if not h.endswith(".h"):
            continue
        for m in pat.finditer(open(os.path.join(ROOT, "include", h)).read()):
            seen += 1
            c = m.group(1) or ""
            if not (re.search(r"[A-Za-z_/]+\.(cc|cu|cuh|h|mk)\b", c) or "counterpart" in c.lower()):
                missing.append(m.group(3))
    assert seen >= 30 and not missing, missing
