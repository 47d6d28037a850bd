"""The allocation-free entry point, vc_solve_noalloc, against vc_solve.

vc_solve_noalloc serves callers that may not allocate device memory: they hand
in device buffers for the graph and the result, and the search's scratch lives
in a fixed array inside the library.  This test calls it through the C ABI
twice in a row per graph (the shared array must be fully reset between calls)
and checks every answer against the existing entry point vc_solve: the same
MVC size / PVC decision (integers, exact) and a valid cover of that size.
It is collected last so that a failure here comes after every other test ran.
"""
import ctypes

import numpy as np
import pytest

import vcgpu
from vcgpu import workloads as W

pytestmark = pytest.mark.gpu


def _fn():
    L = vcgpu.lib()
    f = L.vc_solve_noalloc
    f.argtypes = [ctypes.POINTER(vcgpu.Csr), ctypes.POINTER(vcgpu.Request), ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def _run(f, g, d_rp, d_col, instance, k, stream, torch, node_limit=0, want_cover=True):
    res = torch.zeros(8, dtype=torch.int32, device="cuda")
    nw = (g.n + 31) // 32
    cover = torch.zeros(nw, dtype=torch.int32, device="cuda")
    csr = vcgpu.Csr(g.n, g.m, d_rp.data_ptr(), d_col.data_ptr(), None)
    req = vcgpu._request(instance, k, 0, node_limit, 60.0, vcgpu.VC_FLAG_DEVICE_INPUT, -1, stream)
    st = f(ctypes.byref(csr), ctypes.byref(req), res.data_ptr(), cover.data_ptr() if want_cover else None)
    assert st == vcgpu.VC_OK
    torch.cuda.synchronize()
    out = res.cpu().numpy().astype(np.uint32)
    if not want_cover:
        return out, None
    words = cover.cpu().numpy().astype(np.uint32)
    mask = np.array([(words[v >> 5] >> (v & 31)) & 1 for v in range(g.n)], dtype=bool)
    return out, mask


@pytest.mark.parametrize("which", ["gnp60", "batch_n_mid", "batch_n_large"])
def test_noalloc_matches_vc_solve_twice(which):
    torch = pytest.importorskip("torch")
    f = _fn()
    if which == "gnp60":
        g = W.config1_graph()
    elif which == "batch_n_mid":
        g = next(W.batch_instance(i) for i in range(100) if 70 <= W.batch_instance(i).n <= 120 and W.batch_instance(i).m < 400)
    else:
        g = next(W.batch_instance(i) for i in range(200) if W.batch_instance(i).n >= 150 and W.batch_instance(i).m < 420)
    d_rp = torch.from_numpy(g.row_ptr.astype(np.int32)).cuda()
    d_col = torch.from_numpy(g.col.astype(np.int32)).cuda()
    stream = torch.cuda.current_stream().cuda_stream
    ref = vcgpu.solve(g, "mvc", time_limit=60.0)
    assert ref.status == vcgpu.VC_OK
    for _ in range(2):
        out, mask = _run(f, g, d_rp, d_col, "mvc", 0, stream, torch)
        assert out[0] == vcgpu.VC_OK and out[2] == 1 and out[3] == 1
        assert out[1] == ref.size
        assert W.is_cover(g, mask) and int(mask.sum()) == ref.size
        assert (int(out[4]) | (int(out[5]) << 32)) > 0
    for k, expect in ((ref.size, 1), (ref.size - 1, 0)):
        pv = vcgpu.solve(g, "pvc", k=k, time_limit=60.0)
        assert pv.decision == expect
        for _ in range(2):
            out, mask = _run(f, g, d_rp, d_col, "pvc", k, stream, torch)
            assert out[0] == vcgpu.VC_OK and out[2] == expect
            if expect:
                assert W.is_cover(g, mask) and int(mask.sum()) == out[1] <= k


def test_noalloc_rejects_large_graph():
    torch = pytest.importorskip("torch")
    f = _fn()
    g = W.gnp(300, 0.02, 3)
    d_rp = torch.from_numpy(g.row_ptr.astype(np.int32)).cuda()
    d_col = torch.from_numpy(g.col.astype(np.int32)).cuda()
    res = torch.zeros(8, dtype=torch.int32, device="cuda")
    csr = vcgpu.Csr(g.n, g.m, d_rp.data_ptr(), d_col.data_ptr(), None)
    req = vcgpu._request("mvc", 0, 0, 0, 10.0, vcgpu.VC_FLAG_DEVICE_INPUT, -1, 0)
    assert f(ctypes.byref(csr), ctypes.byref(req), res.data_ptr(), None) == vcgpu.VC_ERR_TOO_LARGE


def _hard_small_graph():
    """A batch graph of at most 255 vertices whose search takes many nodes."""
    import json
    import os
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "batch_seed0.jsonl")
    recs = [json.loads(l) for l in open(path) if l.strip()]
    rec = min((r for r in recs if r["status"] == "ok" and 200_000 <= r["nodes"] <= 2_000_000), key=lambda r: r["i"])
    return W.batch_instance(rec["i"]), rec["opt"]


def test_noalloc_early_stop_then_full_call():
    """A call stopped by its node limit reports VC_BUDGET; the next call on the
    same shared array (which still holds the stopped call's state) and a call
    without a cover buffer both give vc_solve's answer."""
    torch = pytest.importorskip("torch")
    f = _fn()
    g, opt = _hard_small_graph()
    d_rp = torch.from_numpy(g.row_ptr.astype(np.int32)).cuda()
    d_col = torch.from_numpy(g.col.astype(np.int32)).cuda()
    stream = torch.cuda.current_stream().cuda_stream
    out, _ = _run(f, g, d_rp, d_col, "mvc", 0, stream, torch, node_limit=1)
    assert out[0] == vcgpu.VC_BUDGET
    ref = vcgpu.solve(g, "mvc", time_limit=60.0)
    assert ref.status == vcgpu.VC_OK and ref.size == opt
    out, mask = _run(f, g, d_rp, d_col, "mvc", 0, stream, torch)
    assert out[0] == vcgpu.VC_OK and out[1] == opt and W.is_cover(g, mask) and int(mask.sum()) == opt
    out, mask = _run(f, g, d_rp, d_col, "mvc", 0, stream, torch, want_cover=False)
    assert out[0] == vcgpu.VC_OK and out[1] == opt and mask is None


def test_noalloc_checks_device_csr():
    """A device-resident graph that breaks the CSR layout (an id out of range) is
    reported VC_ERR_INVALID without being searched; the next call is exact."""
    torch = pytest.importorskip("torch")
    f = _fn()
    g = W.config1_graph()
    col = g.col.astype(np.int64).copy()
    col[0] = g.n + 3
    d_rp = torch.from_numpy(g.row_ptr.astype(np.int32)).cuda()
    d_bad = torch.from_numpy(col.astype(np.int32)).cuda()
    d_col = torch.from_numpy(g.col.astype(np.int32)).cuda()
    stream = torch.cuda.current_stream().cuda_stream
    out, _ = _run(f, g, d_rp, d_bad, "mvc", 0, stream, torch)
    assert out[0] == vcgpu.VC_ERR_INVALID
    ref = vcgpu.solve(g, "mvc", time_limit=60.0)
    out, mask = _run(f, g, d_rp, d_col, "mvc", 0, stream, torch)
    assert out[0] == vcgpu.VC_OK and out[1] == ref.size and W.is_cover(g, mask)
