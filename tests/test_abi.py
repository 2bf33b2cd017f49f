"""The C ABI library: loads, exports every function declared in include/*.h,
and reports errors (never aborts) when no GPU is usable.  CPU only."""
import ctypes as C
import inspect
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"\b(gb_[a-z0-9_]+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    from galois_b200 import _lib

    lib = ROOT / "galois_b200" / "libgb.so"
    out = subprocess.run(["nm", "-D", "--defined-only", str(lib)], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r" T (gb_[a-z0-9_]+)$", out, flags=re.M))
    declared = declared_functions()
    assert declared, "no declarations parsed"
    missing = declared - exported
    assert not missing, f"declared but not exported: {sorted(missing)}"
    # and the ctypes layer binds exactly the declared set
    assert set(_lib.SIGNATURES) == declared


def test_version_and_error_string():
    from galois_b200 import _lib

    assert _lib.lib.gb_version() >= 10000
    assert isinstance(_lib.last_error(), str)


def test_null_arguments_return_status_not_crash():
    from galois_b200 import _lib

    lib = _lib.lib
    assert lib.gb_bfs(None, 0, None, None, None) == _lib.GB_ERR_ARG
    assert lib.gb_sssp_delta(None, 0, 13, None, None, None) == _lib.GB_ERR_ARG
    assert lib.gb_cc(None, 0, None, None, None) == _lib.GB_ERR_ARG
    assert lib.gb_graph_info(None, None, None, None) == _lib.GB_ERR_ARG
    assert "null" in _lib.last_error()
    assert lib.gb_gr_read(None, 0, None) == _lib.GB_ERR_ARG


def test_upload_without_gpu_is_an_error_status():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present; the no-GPU error path is not reachable")
    from galois_b200 import _lib

    end = np.array([1, 1], np.uint64)
    col = np.array([1], np.uint32)
    h = C.c_void_p()
    st = _lib.lib.gb_graph_upload(C.c_void_p(end.ctypes.data), C.c_void_p(col.ctypes.data), None, None, 2, 1, 0, 0,
                                  C.byref(h))
    assert st in (_lib.GB_ERR_CUDA, _lib.GB_ERR_ARG)
    assert _lib.last_error()


def test_python_entry_points_mirror_reference_signatures():
    """python/galois: bfs(numThreads, source, filename) (_bfs.pyx:171),
    sssp(numThreads, shift, source, filename) (_sssp.pyx:154),
    pagerank(numThreads, max_iterations, filename) (_pagerank.pyx:157),
    connectedComponents(numThreads, filename) (_connected_components.pyx:87)."""
    from galois_b200.bfs import bfs
    from galois_b200.connected_components import connectedComponents
    from galois_b200.pagerank import pagerank
    from galois_b200.sssp import sssp

    assert list(inspect.signature(bfs).parameters) == ["numThreads", "source", "filename"]
    assert list(inspect.signature(sssp).parameters) == ["numThreads", "shift", "source", "filename"]
    assert list(inspect.signature(pagerank).parameters) == ["numThreads", "max_iterations", "filename"]
    assert list(inspect.signature(connectedComponents).parameters) == ["numThreads", "filename"]
