"""Python access to libvcgpu.so through its C ABI (include/vcgpu.h).

This is the host-side mirror that tests and bench.py use: every call goes
through the same extern "C" entry points a C, C++ or cgo caller would bind.
There is no fallback: if the library is missing the import of `lib()` fails.
"""
from __future__ import annotations

import ctypes
import dataclasses
import os
import re
from typing import List, Optional, Sequence

import numpy as np

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REPO_DIR = os.path.dirname(PKG_DIR)
LIB_PATH = os.path.join(PKG_DIR, "libvcgpu.so")
HEADER = os.path.join(REPO_DIR, "include", "vcgpu.h")

VC_OK, VC_ERR_INVALID, VC_ERR_CUDA, VC_ERR_NOMEM, VC_ERR_TOO_LARGE = 0, 1, 2, 3, 4
VC_TIMEOUT, VC_BUDGET, VC_ERR_INTERNAL, VC_ERR_NO_DEVICE, VC_PENDING = 5, 6, 7, 8, 9
VC_MVC, VC_PVC = 0, 1
VC_FLAG_DEVICE_INPUT, VC_FLAG_NO_VALIDATE = 0x1, 0x2
STATUS_NAMES = {0: "ok", 1: "invalid", 2: "cuda", 3: "nomem", 4: "too_large", 5: "timeout", 6: "budget",
                7: "internal", 8: "no_device", 9: "pending"}

_u32p = ctypes.POINTER(ctypes.c_uint32)
_u64p = ctypes.POINTER(ctypes.c_uint64)


class Csr(ctypes.Structure):
    _fields_ = [("n", ctypes.c_uint32), ("m", ctypes.c_uint32), ("row_ptr", ctypes.c_void_p),
                ("col", ctypes.c_void_p), ("degree", ctypes.c_void_p)]


class CsrArena(ctypes.Structure):
    _fields_ = [("count", ctypes.c_uint32), ("n", ctypes.c_void_p), ("row_off", ctypes.c_void_p),
                ("col_off", ctypes.c_void_p), ("row_ptr", ctypes.c_void_p), ("col", ctypes.c_void_p)]


class Request(ctypes.Structure):
    _fields_ = [("instance", ctypes.c_uint32), ("k", ctypes.c_uint32), ("ub", ctypes.c_uint32),
                ("flags", ctypes.c_uint32), ("node_limit", ctypes.c_uint64), ("time_limit_s", ctypes.c_double),
                ("device", ctypes.c_int32), ("reserved", ctypes.c_uint32), ("stream", ctypes.c_void_p)]


class Result(ctypes.Structure):
    _fields_ = [("size", ctypes.c_uint32), ("decision", ctypes.c_uint32), ("has_cover", ctypes.c_uint32),
                ("status", ctypes.c_int), ("cover_mask", ctypes.c_void_p), ("tree_nodes", ctypes.c_uint64),
                ("kernel_ms", ctypes.c_float), ("total_ms", ctypes.c_float), ("done_ms", ctypes.c_float),
                ("reserved", ctypes.c_uint32)]


@dataclasses.dataclass
class Solution:
    status: int
    size: int
    decision: int
    cover: Optional[np.ndarray]
    tree_nodes: int
    kernel_ms: float
    total_ms: float
    done_ms: float = 0.0

    @property
    def status_name(self) -> str:
        return STATUS_NAMES.get(self.status, str(self.status))


_lib = None


def lib():
    """The loaded libvcgpu.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libvcgpu.so is not built ({LIB_PATH}); run __graft_entry__.build()")
        L = ctypes.CDLL(LIB_PATH)
        L.vc_solve.argtypes = [ctypes.POINTER(Csr), ctypes.POINTER(Request), ctypes.POINTER(Result)]
        L.vc_solve.restype = ctypes.c_int
        L.vc_solve_batch.argtypes = [ctypes.POINTER(CsrArena), ctypes.POINTER(Request), ctypes.POINTER(Result)]
        L.vc_solve_batch.restype = ctypes.c_int
        L.vc_solve_batch_device.argtypes = [ctypes.POINTER(CsrArena), ctypes.c_void_p, ctypes.c_void_p,
                                            ctypes.POINTER(Request), ctypes.POINTER(Result)]
        L.vc_solve_batch_device.restype = ctypes.c_int
        L.vc_kernel_launches.argtypes = []
        L.vc_kernel_launches.restype = ctypes.c_uint64
        L.vc_debug_stats.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_uint32,
                                     ctypes.c_void_p]
        L.vc_debug_stats.restype = ctypes.c_uint32
        L.vc_status_string.argtypes = [ctypes.c_int]
        L.vc_status_string.restype = ctypes.c_char_p
        if hasattr(L, "vc_mcm"):
            L.vc_mcm.argtypes = [ctypes.POINTER(Csr), ctypes.POINTER(Request), ctypes.POINTER(Result)]
            L.vc_mcm.restype = ctypes.c_int
        if hasattr(L, "vc_solve_noalloc"):
            L.vc_solve_noalloc.argtypes = [ctypes.POINTER(Csr), ctypes.POINTER(Request), ctypes.c_void_p,
                                           ctypes.c_void_p]
            L.vc_solve_noalloc.restype = ctypes.c_int
        if hasattr(L, "vc_server_create"):
            L.vc_server_create.argtypes = [ctypes.c_int32, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32,
                                           ctypes.POINTER(ctypes.c_void_p)]
            L.vc_server_create.restype = ctypes.c_int
            L.vc_server_submit.argtypes = [ctypes.c_void_p, ctypes.POINTER(Csr), ctypes.POINTER(Request), _u64p]
            L.vc_server_submit.restype = ctypes.c_int
            L.vc_server_poll.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(Result)]
            L.vc_server_poll.restype = ctypes.c_int
            L.vc_remove_max_ub.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                           ctypes.POINTER(ctypes.c_float)]
            L.vc_remove_max_ub.restype = ctypes.c_int
            L.vc_remove_edge_ub.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int32, ctypes.c_void_p,
                                            ctypes.c_void_p, ctypes.POINTER(ctypes.c_float)]
            L.vc_remove_edge_ub.restype = ctypes.c_int
            L.vc_server_completed.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
                                              ctypes.POINTER(ctypes.c_uint32)]
            L.vc_server_completed.restype = ctypes.c_int
            L.vc_server_shape.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
                                          ctypes.POINTER(ctypes.c_uint32)]
            L.vc_server_shape.restype = ctypes.c_int
            L.vc_server_destroy.argtypes = [ctypes.c_void_p]
            L.vc_server_destroy.restype = ctypes.c_int
        _lib = L
    return _lib


def header_functions() -> List[str]:
    """Names of every function declared in include/vcgpu.h."""
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(vc_[a-z_]+)\s*\(", src)))


def _request(instance: str, k: int, ub: int, node_limit: int, time_limit: float, flags: int,
             device: int, stream: int = 0) -> Request:
    r = Request()
    r.instance = VC_PVC if instance == "pvc" else VC_MVC
    r.k = int(k)
    r.ub = int(ub)
    r.flags = flags
    r.node_limit = int(node_limit)
    r.time_limit_s = float(time_limit)
    r.device = int(device)
    r.stream = stream or None
    return r


def _solution(res: Result, cover: Optional[np.ndarray], n: int) -> Solution:
    return Solution(int(res.status), int(res.size), int(res.decision),
                    cover.astype(bool) if (cover is not None and res.has_cover) else None,
                    int(res.tree_nodes), float(res.kernel_ms), float(res.total_ms), float(res.done_ms))


def solve(g, instance: str = "mvc", k: int = 0, ub: int = 0, node_limit: int = 0, time_limit: float = 0.0,
          want_cover: bool = True, device: int = -1, validate: bool = True) -> Solution:
    """One graph through vc_solve with host buffers (copies inside the call)."""
    rp = np.ascontiguousarray(g.row_ptr, dtype=np.uint32)
    col = np.ascontiguousarray(g.col, dtype=np.uint32)
    c = Csr(g.n, col.shape[0] // 2, rp.ctypes.data, col.ctypes.data if col.size else None, None)
    req = _request(instance, k, ub, node_limit, time_limit, 0 if validate else VC_FLAG_NO_VALIDATE, device)
    res = Result()
    cover = np.zeros(max(g.n, 1), dtype=np.uint8) if want_cover else None
    res.cover_mask = cover.ctypes.data if cover is not None else None
    st = lib().vc_solve(ctypes.byref(c), ctypes.byref(req), ctypes.byref(res))
    if st in (VC_ERR_INVALID, VC_ERR_CUDA, VC_ERR_NOMEM, VC_ERR_TOO_LARGE, VC_ERR_NO_DEVICE):
        return Solution(st, 0, 0, None, 0, 0.0, 0.0)
    return _solution(res, cover[:g.n] if cover is not None else None, g.n)


def mcm(g, node_limit: int = 0, time_limit: float = 0.0, device: int = -1) -> Solution:
    """The MCM mode (vc_mcm): size = 2 * maximum matching + isolated vertices,
    the reference's default build's `maximum`."""
    rp = np.ascontiguousarray(g.row_ptr, dtype=np.uint32)
    col = np.ascontiguousarray(g.col, dtype=np.uint32)
    c = Csr(g.n, col.shape[0] // 2, rp.ctypes.data, col.ctypes.data if col.size else None, None)
    req = _request("mvc", 0, 0, node_limit, time_limit, 0, device)
    res = Result()
    st = lib().vc_mcm(ctypes.byref(c), ctypes.byref(req), ctypes.byref(res))
    if st in (VC_ERR_INVALID, VC_ERR_CUDA, VC_ERR_NOMEM, VC_ERR_TOO_LARGE, VC_ERR_NO_DEVICE):
        return Solution(st, 0, 0, None, 0, 0.0, 0.0)
    return Solution(int(res.status), int(res.size), int(res.decision), None, int(res.tree_nodes),
                    float(res.kernel_ms), float(res.total_ms), 0.0)


def solve_device(n: int, m: int, d_row_ptr: int, d_col: int, instance: str = "mvc", k: int = 0, ub: int = 0,
                 node_limit: int = 0, time_limit: float = 0.0, want_cover: bool = True, device: int = -1,
                 stream: int = 0) -> Solution:
    """One graph whose CSR already lives in device memory (pointers as ints)."""
    c = Csr(n, m, d_row_ptr, d_col, None)
    req = _request(instance, k, ub, node_limit, time_limit, VC_FLAG_DEVICE_INPUT, device, stream)
    res = Result()
    cover = np.zeros(max(n, 1), dtype=np.uint8) if want_cover else None
    res.cover_mask = cover.ctypes.data if cover is not None else None
    st = lib().vc_solve(ctypes.byref(c), ctypes.byref(req), ctypes.byref(res))
    if st in (VC_ERR_INVALID, VC_ERR_CUDA, VC_ERR_NOMEM, VC_ERR_TOO_LARGE, VC_ERR_NO_DEVICE):
        return Solution(st, 0, 0, None, 0, 0.0, 0.0)
    return _solution(res, cover[:n] if cover is not None else None, n)


def _arena_struct(arena) -> CsrArena:
    a = CsrArena()
    a.count = arena.count
    a.n = arena.n.ctypes.data
    a.row_off = arena.row_off.ctypes.data
    a.col_off = arena.col_off.ctypes.data
    a.row_ptr = arena.row_ptr.ctypes.data
    a.col = arena.col.ctypes.data if arena.col.size else None
    return a


def _batch_requests(count: int, instances, ks, ubs, node_limit, time_limit, flags, device, stream=0):
    reqs = (Request * count)()
    for i in range(count):
        inst = instances[i] if isinstance(instances, (list, tuple)) else instances
        reqs[i] = _request(inst, ks[i] if ks is not None else 0, ubs[i] if ubs is not None else 0,
                           node_limit, time_limit, flags, device, stream)
    return reqs


def solve_batch(arena, instances="mvc", ks: Optional[Sequence[int]] = None, ubs: Optional[Sequence[int]] = None,
                node_limit: int = 0, time_limit: float = 0.0, want_cover: bool = True, device: int = -1,
                d_row_ptr: int = 0, d_col: int = 0, validate: bool = True, stream: int = 0):
    """Every graph of a workloads.Arena in one launch (vc_solve_batch, or
    vc_solve_batch_device when d_row_ptr/d_col point at a device copy).
    Returns (call status, [Solution])."""
    count = arena.count
    flags = 0 if validate else VC_FLAG_NO_VALIDATE
    reqs = _batch_requests(count, instances, ks, ubs, node_limit, time_limit, flags, device, stream)
    outs = (Result * count)()
    covers = []
    for i in range(count):
        cv = np.zeros(max(int(arena.n[i]), 1), dtype=np.uint8) if want_cover else None
        covers.append(cv)
        outs[i].cover_mask = cv.ctypes.data if cv is not None else None
    a = _arena_struct(arena)
    if d_row_ptr:
        st = lib().vc_solve_batch_device(ctypes.byref(a), ctypes.c_void_p(d_row_ptr), ctypes.c_void_p(d_col),
                                         reqs, outs)
    else:
        st = lib().vc_solve_batch(ctypes.byref(a), reqs, outs)
    sols = [_solution(outs[i], covers[i][:int(arena.n[i])] if covers[i] is not None else None, int(arena.n[i]))
            for i in range(count)]
    return st, sols


STAT_NAMES = ["nodes", "passes", "donations", "donate_fail", "receives", "roots", "busy_cycles", "idle_cycles",
              "polls", "restored", "smid"]


def debug_stats(enable: Optional[bool] = None, device: int = -1):
    """Enable/disable per-search-unit counters; returns (rows[num_su, 16], launch
    shape (grid, block, smem, num_su, np)) of the last launch."""
    L = lib()
    shape = np.zeros(5, dtype=np.uint32)
    nsu = L.vc_debug_stats(device, -1 if enable is None else int(enable), None, 0, shape.ctypes.data)
    rows = np.zeros((max(nsu, 1), 16), dtype=np.uint64)
    L.vc_debug_stats(device, -1, rows.ctypes.data, nsu, shape.ctypes.data)
    return rows[:nsu], shape


def _ub(kind: str, arena, r: int, device: int):
    if not hasattr(arena, "row_off"):  # one Graph
        from . import workloads
        arena = workloads.pack([arena])
    n = np.ascontiguousarray(arena.n, dtype=np.uint32)
    ro = np.ascontiguousarray(arena.row_off, dtype=np.uint64)
    co = np.ascontiguousarray(arena.col_off, dtype=np.uint64)
    rp = np.ascontiguousarray(arena.row_ptr, dtype=np.uint32)
    col = np.ascontiguousarray(arena.col, dtype=np.uint32)
    a = CsrArena(arena.count, n.ctypes.data, ro.ctypes.data, co.ctypes.data, rp.ctypes.data,
                 col.ctypes.data if col.size else None)
    ub = np.zeros(max(arena.count, 1), dtype=np.uint32)
    cover = np.zeros(max(int(n.sum()), 1), dtype=np.uint8)
    ms = ctypes.c_float(0.0)
    if kind == "max":
        st = lib().vc_remove_max_ub(ctypes.byref(a), device, ub.ctypes.data, cover.ctypes.data, ctypes.byref(ms))
    else:
        st = lib().vc_remove_edge_ub(ctypes.byref(a), r, device, ub.ctypes.data, cover.ctypes.data,
                                     ctypes.byref(ms))
    if st != VC_OK:
        raise RuntimeError(f"vc_remove_{kind}_ub failed: {STATUS_NAMES.get(st, st)}")
    covers, k = [], 0
    for ni in n:
        covers.append(cover[k:k + int(ni)].astype(bool))
        k += int(ni)
    return [int(x) for x in ub[:arena.count]], covers, float(ms.value)


def remove_max_ub(arena, device: int = -1):
    """RemoveMaxApproximateMVC on the GPU for every graph of an Arena (or one
    Graph): (bounds, covers, kernel ms)."""
    return _ub("max", arena, 0, device)


def remove_edge_ub(arena, r: int, device: int = -1):
    """RemoveEdgeApproximateMVC on the GPU with rand() == r: (bounds, covers,
    kernel ms)."""
    return _ub("edge", arena, r, device)


def kernel_launches() -> int:
    return int(lib().vc_kernel_launches())


TUNE_CLASSES = ["dense n<=64", "dense n<=128", "dense n<=255", "wide dense n<=640", "16-bit dense n<=1024", "csr n>1024"]


TUNE_WORDS = 7  # per class


def _unpack_tuning(buf: np.ndarray) -> List[dict]:
    out = []
    for i, name in enumerate(TUNE_CLASSES):
        w = buf[TUNE_WORDS * i:TUNE_WORDS * (i + 1)]
        out.append({"class": name, "set": int(w[0]), "units": "cta" if w[1] else "warp", "warps": int(w[2]),
                    "pool_per_warp": int(w[3]), "ring_bias": int(np.uint32(w[4]).astype(np.int32)),
                    "nodes_per_s": float(np.frombuffer(np.uint32(w[5]).tobytes(), dtype=np.float32)[0]),
                    "ring_first": int(w[6])})
    return out


def autotune(slice_s: float = 0.0, device: int = -1):
    """vc_autotune: measure launch shapes per size class on the device and install
    the fastest.  Returns (status, table words, readable table)."""
    buf = np.zeros(TUNE_WORDS * len(TUNE_CLASSES), dtype=np.uint32)
    L = lib()
    L.vc_autotune.argtypes = [ctypes.c_int32, ctypes.c_double, ctypes.c_void_p, ctypes.c_uint32]
    L.vc_autotune.restype = ctypes.c_int
    st = L.vc_autotune(device, slice_s, buf.ctypes.data, int(buf.size))
    return st, buf, _unpack_tuning(buf)


def set_tuning(table, device: int = -1) -> int:
    """vc_set_tuning: install a table of words from autotune (zeros = built-in rules)."""
    buf = np.ascontiguousarray(np.asarray(table, dtype=np.uint32))
    L = lib()
    L.vc_set_tuning.argtypes = [ctypes.c_int32, ctypes.c_void_p, ctypes.c_uint32]
    L.vc_set_tuning.restype = ctypes.c_int
    return L.vc_set_tuning(device, buf.ctypes.data, int(buf.size))


class Server:
    """A continuous-batching server (vc_server_*): requests are admitted into a
    persistent kernel while others run."""

    def __init__(self, device: int = -1, mem_budget: int = 0, max_requests: int = 0, max_vertices: int = 0):
        self._h = ctypes.c_void_p()
        st = lib().vc_server_create(device, mem_budget, max_requests, max_vertices, ctypes.byref(self._h))
        if st != VC_OK:
            raise RuntimeError(f"vc_server_create failed: {STATUS_NAMES.get(st, st)}")
        self._n = {}

    def submit(self, g, instance: str = "mvc", k: int = 0, ub: int = 0, node_limit: int = 0,
               validate: bool = True) -> int:
        rp = np.ascontiguousarray(g.row_ptr, dtype=np.uint32)
        col = np.ascontiguousarray(g.col, dtype=np.uint32)
        c = Csr(g.n, col.shape[0] // 2, rp.ctypes.data, col.ctypes.data if col.size else None, None)
        req = _request(instance, k, ub, node_limit, 0.0, 0 if validate else VC_FLAG_NO_VALIDATE, -1)
        t = ctypes.c_uint64(0)
        st = lib().vc_server_submit(self._h, ctypes.byref(c), ctypes.byref(req), ctypes.byref(t))
        if st != VC_OK:
            raise RuntimeError(f"vc_server_submit failed: {STATUS_NAMES.get(st, st)}")
        self._n[t.value] = g.n
        return int(t.value)

    def poll(self, ticket: int, want_cover: bool = True) -> Optional[Solution]:
        n = self._n[ticket]
        res = Result()
        cover = np.zeros(max(n, 1), dtype=np.uint8) if want_cover else None
        res.cover_mask = cover.ctypes.data if cover is not None else None
        st = lib().vc_server_poll(self._h, ticket, ctypes.byref(res))
        if st == VC_PENDING:
            return None
        del self._n[ticket]
        if st == VC_ERR_INVALID:
            raise KeyError(ticket)
        return _solution(res, cover[:n] if cover is not None else None, n)

    def completed(self, max_tickets: int = 4096) -> List[int]:
        """Tickets that finished since the last call."""
        buf = np.zeros(max_tickets, dtype=np.uint64)
        cnt = ctypes.c_uint32(0)
        lib().vc_server_completed(self._h, buf.ctypes.data, max_tickets, ctypes.byref(cnt))
        return [int(x) for x in buf[:cnt.value]]

    def shape(self) -> List[dict]:
        """The server's lanes: largest request, grid, block, search units, shared
        memory per CTA and kernel kind."""
        buf = np.zeros(18, dtype=np.uint32)
        cnt = ctypes.c_uint32(0)
        lib().vc_server_shape(self._h, buf.ctypes.data, 3, ctypes.byref(cnt))
        return [{"max_vertices": int(buf[6 * i]), "grid": int(buf[6 * i + 1]), "block": int(buf[6 * i + 2]),
                 "search_units": int(buf[6 * i + 3]), "smem_bytes": int(buf[6 * i + 4]),
                 "kernel": "dense" if buf[6 * i + 5] else "csr"} for i in range(min(int(cnt.value), 3))]

    @staticmethod
    def lane(ticket: int) -> int:
        """The lane a ticket's request runs in (its low two bits)."""
        return int(ticket) & 3

    def wait(self, ticket: int, timeout: float = 120.0, want_cover: bool = True) -> Solution:
        import time
        t0 = time.time()
        while True:
            r = self.poll(ticket, want_cover)
            if r is not None:
                return r
            if time.time() - t0 > timeout:
                raise TimeoutError(ticket)
            time.sleep(0.0005)

    def close(self):
        if self._h:
            lib().vc_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
