"""TEST INFRASTRUCTURE ONLY: ctypes access to the CPU oracle.

Two libraries, both built by oracle/Makefile:
  * ``_build/liboracle.so`` -- this directory's C restatement of the reference's
    sequential solver (vc_oracle.c; Sequential.cpp / SequentialParameterized.cpp);
  * ``_ref/libvcref.so``    -- the reference's own CPU solver compiled from its
    sources with a C-ABI shim (ref_harness.cpp), present where it was built.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
arm use this module, and only as the checker.  The product never imports it.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# Where the reference tree is read from (its graph files, its runGraphs.py, its
# sources for oracle/Makefile): $VC_REFERENCE_ROOT, by default /root/reference.
REFERENCE_ROOT = os.environ.get("VC_REFERENCE_ROOT", "/root/reference")
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libvcref.so")

OK, BUDGET, NOMEM = 0, 1, 2

_u32p = ctypes.POINTER(ctypes.c_uint32)
_u8p = ctypes.POINTER(ctypes.c_uint8)
_lib = None
_ref = None


def _p32(a: np.ndarray):
    return a.ctypes.data_as(_u32p)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"oracle library missing: {LIB_PATH} (run make -C oracle)")
        L = ctypes.CDLL(LIB_PATH)
        L.oracle_mvc.argtypes = [ctypes.c_uint32, _u32p, _u32p, ctypes.c_uint32, _u32p, _u8p,
                                 ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_uint64), ctypes.c_uint64]
        L.oracle_mvc.restype = ctypes.c_int
        L.oracle_pvc.argtypes = [ctypes.c_uint32, _u32p, _u32p, ctypes.c_uint32, _u32p, _u8p,
                                 ctypes.POINTER(ctypes.c_uint64), ctypes.c_uint64]
        L.oracle_pvc.restype = ctypes.c_int
        L.oracle_greedy_ub.argtypes = [ctypes.c_uint32, _u32p, _u32p, _u8p]
        L.oracle_greedy_ub.restype = ctypes.c_uint32
        L.oracle_remove_max_ub.argtypes = [ctypes.c_uint32, _u32p, _u32p, _u8p]
        L.oracle_remove_max_ub.restype = ctypes.c_uint32
        L.oracle_remove_edge_ub.argtypes = [ctypes.c_uint32, _u32p, _u32p, ctypes.c_uint32, _u8p]
        L.oracle_remove_edge_ub.restype = ctypes.c_uint32
        L.oracle_is_cover.argtypes = [ctypes.c_uint32, _u32p, _u32p, _u8p]
        L.oracle_mcm.argtypes = [ctypes.c_uint32, _u32p, _u32p, ctypes.c_uint64, _u32p, ctypes.POINTER(ctypes.c_uint64)]
        L.oracle_mcm.restype = ctypes.c_int
        L.oracle_is_cover.restype = ctypes.c_int
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_PATH)


def ref():
    global _ref
    if _ref is None:
        if not ref_available():
            raise RuntimeError(f"reference CPU solver not built: {REF_PATH}")
        L = ctypes.CDLL(REF_PATH)
        for name in ("ref_mvc", "ref_pvc"):
            fn = getattr(L, name)
            fn.argtypes = [ctypes.c_uint32, _u32p, _u32p, ctypes.c_uint32]
            fn.restype = ctypes.c_uint32
        L.ref_remove_max_ub.argtypes = [ctypes.c_uint32, _u32p, _u32p]
        L.ref_remove_max_ub.restype = ctypes.c_uint32
        L.ref_remove_edge_ub.argtypes = [ctypes.c_uint32, _u32p, _u32p, ctypes.POINTER(ctypes.c_uint32)]
        L.ref_remove_edge_ub.restype = ctypes.c_uint32
        L.ref_load.argtypes = [ctypes.c_char_p, _u32p, _u32p, ctypes.POINTER(_u32p), ctypes.POINTER(_u32p)]
        L.ref_load.restype = ctypes.c_int
        L.ref_free.argtypes = [ctypes.c_void_p]
        _ref = L
    return _ref


def _arrays(g) -> Tuple[np.ndarray, np.ndarray]:
    rp = np.ascontiguousarray(g.row_ptr, dtype=np.uint32)
    col = np.ascontiguousarray(g.col, dtype=np.uint32)
    if col.size == 0:
        col = np.zeros(1, dtype=np.uint32)
    return rp, col


def mvc(g, ub: Optional[int] = None, node_limit: int = 0):
    """Exact MVC by the restatement.  Returns (status, size, cover_mask, nodes).
    With the default ub (greedy) the size is OPT and the mask an optimal cover."""
    rp, col = _arrays(g)
    cover = np.zeros(max(g.n, 1), dtype=np.uint8)
    if ub is None:
        ub = int(lib().oracle_greedy_ub(g.n, _p32(rp), _p32(col), cover.ctypes.data_as(_u8p)))
        ub_cover = cover.copy()
    else:
        ub_cover = None
    size = ctypes.c_uint32(0)
    improved = ctypes.c_int(0)
    nodes = ctypes.c_uint64(0)
    st = lib().oracle_mvc(g.n, _p32(rp), _p32(col), ub, ctypes.byref(size), cover.ctypes.data_as(_u8p),
                          ctypes.byref(improved), ctypes.byref(nodes), node_limit)
    if not improved.value:
        cover = ub_cover
    return st, int(size.value), (cover[:g.n].astype(bool) if cover is not None else None), int(nodes.value)


def mcm(g, node_limit: int = 0):
    """The MCM search of the reference's default build by the restatement.
    Returns (status, maximum, nodes); on a finished tree the maximum is
    2 * maximum matching + isolated vertices."""
    rp, col = _arrays(g)
    best = ctypes.c_uint32(0)
    nodes = ctypes.c_uint64(0)
    st = lib().oracle_mcm(g.n, _p32(rp), _p32(col), node_limit, ctypes.byref(best), ctypes.byref(nodes))
    return st, int(best.value), int(nodes.value)


def pvc(g, k: int, node_limit: int = 0):
    """PVC decision by the restatement.  Returns (status, k_found, cover_mask|None, nodes)."""
    rp, col = _arrays(g)
    cover = np.zeros(max(g.n, 1), dtype=np.uint8)
    found = ctypes.c_uint32(0)
    nodes = ctypes.c_uint64(0)
    st = lib().oracle_pvc(g.n, _p32(rp), _p32(col), k, ctypes.byref(found), cover.ctypes.data_as(_u8p),
                          ctypes.byref(nodes), node_limit)
    return st, int(found.value), (cover[:g.n].astype(bool) if found.value else None), int(nodes.value)


def greedy_ub(g) -> Tuple[int, np.ndarray]:
    rp, col = _arrays(g)
    cover = np.zeros(max(g.n, 1), dtype=np.uint8)
    ub = int(lib().oracle_greedy_ub(g.n, _p32(rp), _p32(col), cover.ctypes.data_as(_u8p)))
    return ub, cover[:g.n].astype(bool)


def is_cover(g, mask) -> bool:
    rp, col = _arrays(g)
    mk = np.ascontiguousarray(np.asarray(mask, dtype=np.uint8))
    if mk.size == 0:
        mk = np.zeros(1, dtype=np.uint8)
    return bool(lib().oracle_is_cover(g.n, _p32(rp), _p32(col), mk.ctypes.data_as(_u8p)))


def ref_mvc(g, ub: Optional[int] = None) -> int:
    """The reference's own Sequential(graph, ub); ub defaults to its
    RemoveMaxApproximateMVC bound."""
    rp, col = _arrays(g)
    if ub is None:
        ub = int(ref().ref_remove_max_ub(g.n, _p32(rp), _p32(col)))
    return int(ref().ref_mvc(g.n, _p32(rp), _p32(col), ub))


def ref_pvc(g, k: int) -> int:
    """The reference's own SequentialParameterized(graph, k+1, k) -> kFound."""
    rp, col = _arrays(g)
    return int(ref().ref_pvc(g.n, _p32(rp), _p32(col), k))


def remove_max_ub(g) -> Tuple[int, np.ndarray]:
    """RemoveMaxApproximateMVC restated exactly (src/auxFunctions.cpp:211-256):
    (cover size, cover mask)."""
    rp = np.ascontiguousarray(g.row_ptr, dtype=np.uint32)
    col = np.ascontiguousarray(g.col, dtype=np.uint32)
    cover = np.zeros(max(g.n, 1), dtype=np.uint8)
    ub = int(lib().oracle_remove_max_ub(g.n, _p32(rp), _p32(col), cover.ctypes.data_as(_u8p)))
    return ub, cover[:g.n].astype(bool)


def remove_edge_ub(g, r: int) -> Tuple[int, np.ndarray]:
    """RemoveEdgeApproximateMVC restated exactly with rand() == r
    (src/auxFunctions.cpp:258-306): (cover size, cover mask)."""
    rp = np.ascontiguousarray(g.row_ptr, dtype=np.uint32)
    col = np.ascontiguousarray(g.col, dtype=np.uint32)
    cover = np.zeros(max(g.n, 1), dtype=np.uint8)
    ub = int(lib().oracle_remove_edge_ub(g.n, _p32(rp), _p32(col), r, cover.ctypes.data_as(_u8p)))
    return ub, cover[:g.n].astype(bool)


def ref_remove_edge_ub_forked(g) -> Optional[Tuple[int, int]]:
    """The reference's own RemoveEdgeApproximateMVC in a forked child: (bound,
    the rand() value its calls used), or None if the run crossed a second
    boundary or the child failed."""
    r, w = os.pipe()
    pid = os.fork()
    if pid == 0:
        os.close(r)
        try:
            rp = np.ascontiguousarray(g.row_ptr, dtype=np.uint32)
            col = np.ascontiguousarray(g.col, dtype=np.uint32)
            ro = ctypes.c_uint32(0)
            v = ref().ref_remove_edge_ub(g.n, _p32(rp), _p32(col), ctypes.byref(ro))
            os.write(w, f"{v} {ro.value}".encode())
        finally:
            os._exit(0)
    os.close(w)
    data = b""
    while True:
        chunk = os.read(r, 64)
        if not chunk:
            break
        data += chunk
    os.close(r)
    _, status = os.waitpid(pid, 0)
    if not data or status != 0:
        return None
    v, rv = (int(x) for x in data.split())
    return None if v == 0xFFFFFFFF else (v, rv)


def ref_remove_max_ub_forked(g) -> Optional[int]:
    """The reference's own RemoveMaxApproximateMVC in a forked child (its binary
    search can read out of bounds on rare inputs); None if the child failed."""
    r, w = os.pipe()
    pid = os.fork()
    if pid == 0:
        os.close(r)
        try:
            v = ref_remove_max_ub(g)
            os.write(w, str(v).encode())
        finally:
            os._exit(0)
    os.close(w)
    data = b""
    while True:
        chunk = os.read(r, 64)
        if not chunk:
            break
        data += chunk
    os.close(r)
    _, status = os.waitpid(pid, 0)
    return int(data) if data and status == 0 else None


def ref_remove_max_ub(g) -> int:
    rp, col = _arrays(g)
    return int(ref().ref_remove_max_ub(g.n, _p32(rp), _p32(col)))


def ref_load(path: str):
    """The reference's own loader (createCSRGraphFromFile) -> (n, row_ptr, col)."""
    n = ctypes.c_uint32(0)
    m = ctypes.c_uint32(0)
    rp = _u32p()
    col = _u32p()
    if ref().ref_load(path.encode(), ctypes.byref(n), ctypes.byref(m), ctypes.byref(rp), ctypes.byref(col)) != 0:
        raise RuntimeError("ref_load failed")
    row_ptr = np.ctypeslib.as_array(rp, shape=(n.value + 1,)).copy()
    cols = np.ctypeslib.as_array(col, shape=(2 * m.value,)).copy() if m.value else np.zeros(0, np.uint32)
    ref().ref_free(rp)
    ref().ref_free(col)
    return int(n.value), row_ptr, cols
