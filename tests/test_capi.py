"""The C ABI without a GPU: the library loads, exports every function that
include/vcgpu.h declares, validates graphs on the host before touching a
device, and reports a missing device as a status, never by exiting."""
import ctypes

import numpy as np
import pytest

import vcgpu
from vcgpu import workloads as W


def test_library_exports_every_header_function():
    L = vcgpu.lib()
    names = vcgpu.header_functions()
    assert {"vc_solve", "vc_solve_batch", "vc_server_create", "vc_server_submit", "vc_server_poll",
            "vc_server_destroy"} <= set(names)
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_status_strings():
    L = vcgpu.lib()
    assert L.vc_status_string(0) == b"ok"
    assert L.vc_status_string(vcgpu.VC_ERR_INVALID) == b"invalid argument"


def _solve_status(g):
    return vcgpu.solve(g).status


def test_invalid_graphs_rejected_on_host():
    g = W.gnp(20, 0.2, 1)
    bad = W.Graph(g.n, g.row_ptr.copy(), g.col.copy())
    bad.col[0] = bad.n + 5
    assert _solve_status(bad) == vcgpu.VC_ERR_INVALID
    loop = W.Graph(3, np.array([0, 1, 2, 2], np.uint32), np.array([0, 0], np.uint32))
    assert _solve_status(loop) == vcgpu.VC_ERR_INVALID
    asym = W.Graph(3, np.array([0, 1, 1, 1], np.uint32), np.array([1], np.uint32))
    assert _solve_status(asym) == vcgpu.VC_ERR_INVALID
    dup = W.Graph(3, np.array([0, 2, 3, 4], np.uint32), np.array([1, 1, 0, 0], np.uint32))
    assert _solve_status(dup) == vcgpu.VC_ERR_INVALID
    unsorted = W.from_edges(4, np.array([[0, 1], [0, 2], [0, 3]]))
    unsorted.col[:3] = unsorted.col[:3][::-1].copy()
    assert _solve_status(unsorted) == vcgpu.VC_ERR_INVALID


def test_empty_graph_needs_no_device():
    r = vcgpu.solve(W.from_edges(0, np.zeros((0, 2))))
    assert r.status == vcgpu.VC_OK and r.size == 0


def test_null_arguments():
    L = vcgpu.lib()
    assert L.vc_solve(None, None, None) == vcgpu.VC_ERR_INVALID
    assert L.vc_solve_batch(None, None, None) == vcgpu.VC_ERR_INVALID


def test_missing_device_is_a_status():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    r = vcgpu.solve(W.config1_graph())
    assert r.status == vcgpu.VC_ERR_NO_DEVICE
