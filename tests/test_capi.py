"""The C-ABI library builds, loads and exports every entry point include/distger.h declares."""
import ctypes
import os
import re

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "distger.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^DG_API\s+[^(]*?\b(dg_[a-z0-9_]+)\s*\(", text, flags=re.M)))


def test_header_declares_the_boundary():
    syms = declared_symbols()
    for must in ["dg_graph_create", "dg_walk_run_round", "dg_paths_write_text", "dg_sgns_create",
                 "dg_sgns_train_paths", "dg_sgns_write_embedding", "dg_last_error"]:
        assert must in syms


def test_library_exports_every_declared_symbol(distger_lib):
    lib = ctypes.CDLL(distger_lib._lib.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_version_and_error_strings(distger_lib):
    L = distger_lib.lib()
    assert L.dg_version().decode().endswith("sm_100a")
    assert isinstance(L.dg_last_error(), bytes)


def test_argument_errors_are_reported_not_fatal(distger_lib, tmp_path):
    """Bad inputs come back as error codes with a message (no exit, no device work)."""
    from distger import DistgerError, Graph
    import pytest
    with pytest.raises(DistgerError) as e:
        Graph(10, graph_path=str(tmp_path / "missing.bin"))
    assert e.value.code == -2
    bad = tmp_path / "bad.bin"
    bad.write_bytes(b"\0" * 13)
    with pytest.raises(DistgerError) as e:
        Graph(10, graph_path=str(bad))
    assert e.value.code == -2
    edges = np.zeros(1, dtype=[("src", "<u4"), ("dst", "<u4"), ("data", "<f4")])
    edges[0] = (3, 12, 0.5)
    with pytest.raises(DistgerError) as e:
        Graph(10, edges=edges)
    assert e.value.code in (-1, -3)  # vertex id >= v_num (or no CUDA device on this host)
