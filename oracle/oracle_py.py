"""ctypes view of the CPU oracle (test infrastructure; see rama_oracle.h).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg import
this module.  It loads oracle/librama_oracle.so (built by oracle/Makefile).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librama_oracle.so")

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_i64 = C.c_int64
_lib = None


class OrcOpts(C.Structure):
    _fields_ = [
        ("max_cycle_length_lb", C.c_int32),
        ("num_dual_itr_lb", C.c_int32),
        ("max_cycle_length_primal", C.c_int32),
        ("num_dual_itr_primal", C.c_int32),
        ("num_outer_itr_dual", C.c_int32),
        ("mean_multiplier_mm", C.c_float),
        ("matching_thresh_crossover_ratio", C.c_float),
        ("tri_memory_factor", C.c_float),
        ("only_compute_lb", C.c_int32),
        ("max_time_sec", C.c_int32),
        ("dump_timeline", C.c_int32),
        ("verbose", C.c_int32),
        ("sanitize_graph", C.c_int32),
        ("woc_pentagons", C.c_int32),
    ]


class OrcStats(C.Structure):
    _fields_ = [
        ("rounds", C.c_int32),
        ("matching_rounds", C.c_int32),
        ("mst_rounds", C.c_int32),
        ("triangles_initial", C.c_int64),
        ("status", C.c_int32),
        ("truncations", C.c_int32),
    ]


class OrcGraph(C.Structure):
    _fields_ = [
        ("n", C.c_int64),
        ("row", C.POINTER(C.c_int32)),
        ("col", C.POINTER(C.c_int32)),
        ("cost", C.POINTER(C.c_float)),
        ("rows", C.c_int32),
        ("cols", C.c_int32),
    ]


_G = C.POINTER(OrcGraph)


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.orc_graph_from_edges.restype = _G
        L.orc_graph_from_edges.argtypes = [_i64, _i32p, _i32p, _f32p]
        L.orc_graph_from_sorted.restype = _G
        L.orc_graph_from_sorted.argtypes = [_i64, _i32p, _i32p, _f32p]
        L.orc_graph_free.argtypes = [_G]
        L.orc_contract.restype = _G
        L.orc_contract.argtypes = [_G, _i32p, _i64]
        L.orc_has_bad_contractions.argtypes = [_G]
        L.orc_remove_diagonal.argtypes = [_G]
        L.orc_compute_offsets.argtypes = [_i32p, _i64, C.c_int32, _i32p]
        L.orc_compress_label_sequence.argtypes = [_i32p, _i64, C.c_int32, _i32p]
        L.orc_cc.argtypes = [C.c_int32, _i32p, _i32p, _i32p]
        L.orc_csum_f32.restype = C.c_double
        L.orc_csum_f32.argtypes = [_f32p, _i64]
        L.orc_rsum_f32.restype = C.c_float
        L.orc_rsum_f32.argtypes = [_f32p, _i64]
        L.orc_matching.argtypes = [_G, C.c_float, _i32p, C.POINTER(_i64), C.POINTER(C.c_int32)]
        L.orc_msf.argtypes = [_i64, _i32p, _i32p, _f32p, _i32p, C.POINTER(_i64)]
        L.orc_woc.argtypes = [_G, _i32p, C.POINTER(_i64), C.POINTER(C.c_int32)]
        L.orc_woc_ex.argtypes = [_G, _i32p, C.POINTER(_i64), C.POINTER(C.c_int32), C.c_int]
        L.orc_conflicted_cycles.argtypes = [_G, C.c_int32, C.c_float, C.c_float, _i32p, _i64, C.POINTER(_i64),
                                            C.POINTER(_i64)]
        L.orc_mp_create.restype = C.c_void_p
        L.orc_mp_create.argtypes = [_G, _i32p, _i32p, _i32p, _i64]
        L.orc_mp_free.argtypes = [C.c_void_p]
        L.orc_mp_lower_bound.restype = C.c_double
        L.orc_mp_lower_bound.argtypes = [C.c_void_p]
        L.orc_mp_send_messages_to_triplets.argtypes = [C.c_void_p]
        L.orc_mp_send_messages_to_edges.argtypes = [C.c_void_p]
        L.orc_mp_iteration.argtypes = [C.c_void_p]
        L.orc_mp_info.argtypes = [C.c_void_p, C.POINTER(_i64), C.POINTER(_i64)]
        L.orc_mp_copy_edges.argtypes = [C.c_void_p, _i32p, _i32p, _f32p, _i32p]
        L.orc_mp_copy_triangles.argtypes = [C.c_void_p] + [_i32p] * 3 + [_f32p] * 3 + [_i32p] * 3
        L.orc_dual_lb_f64.restype = C.c_int
        L.orc_dual_lb_f64.argtypes = [_i64, _i32p, _i32p, _f32p, C.c_int32, C.c_int32, C.c_float, C.c_int32,
                                      C.c_float, C.POINTER(C.c_double)]
        L.orc_dual_solver.restype = C.c_double
        L.orc_dual_solver.argtypes = [C.POINTER(_G), C.c_int32, C.c_int32, C.c_float, C.c_int32, C.c_float,
                                      C.POINTER(_i64)]
        L.orc_opts_init.argtypes = [C.POINTER(OrcOpts), C.c_char_p]
        L.orc_solve.argtypes = [_i64, _i32p, _i32p, _f32p, C.POINTER(OrcOpts), _i32p, _i64, C.POINTER(_i64),
                                C.POINTER(C.c_double), C.POINTER(OrcStats)]
        L.orc_objective.restype = C.c_double
        L.orc_objective.argtypes = [_i64, _i32p, _i32p, _f32p, _i32p]
        L.orc_sanitize.argtypes = [_i64, _i32p, _i32p, _f32p, C.POINTER(_i64), _i32p, _i64, C.POINTER(_i64)]
        L.orc_gaec.argtypes = [_i64, _i32p, _i32p, _f32p, C.c_int32, _i32p]
        _lib = L
    return _lib


def _a32(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.int32))


def _f32(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.float32))


class Graph:
    """Owning handle of an oracle directed graph (row<col, sorted)."""

    def __init__(self, ptr):
        self.ptr = ptr

    @classmethod
    def from_edges(cls, i, j, c):
        i, j, c = _a32(i), _a32(j), _f32(c)
        return cls(lib().orc_graph_from_edges(len(c), i, j, c))

    @classmethod
    def from_sorted(cls, row, col, cost):
        row, col, cost = _a32(row), _a32(col), _f32(cost)
        return cls(lib().orc_graph_from_sorted(len(cost), row, col, cost))

    def __del__(self):
        if getattr(self, "ptr", None) and _lib is not None:
            _lib.orc_graph_free(self.ptr)
            self.ptr = None

    @property
    def n(self):
        return self.ptr.contents.n

    @property
    def dims(self):
        g = self.ptr.contents
        return g.rows, g.cols

    def arrays(self):
        g = self.ptr.contents
        n = g.n
        row = np.ctypeslib.as_array(g.row, shape=(n,)).copy() if n else np.zeros(0, np.int32)
        col = np.ctypeslib.as_array(g.col, shape=(n,)).copy() if n else np.zeros(0, np.int32)
        cost = np.ctypeslib.as_array(g.cost, shape=(n,)).copy() if n else np.zeros(0, np.float32)
        return row, col, cost

    def contract(self, node_map):
        m = _a32(node_map)
        return Graph(lib().orc_contract(self.ptr, m, len(m)))

    def has_bad_contractions(self):
        return bool(lib().orc_has_bad_contractions(self.ptr))

    def remove_diagonal(self):
        lib().orc_remove_diagonal(self.ptr)

    def max_dim(self):
        r, c = self.dims
        return max(r, c)


def compute_offsets(ids, max_value):
    ids = _a32(ids)
    out = np.zeros(max_value + 2, np.int32)
    lib().orc_compute_offsets(ids, len(ids), max_value, out)
    return out


def compress_label_sequence(data, max_label):
    data = _a32(data)
    out = np.zeros(len(data), np.int32)
    lib().orc_compress_label_sequence(data, len(data), max_label, out)
    return out


def connected_components(offsets, cols):
    offsets, cols = _a32(offsets), _a32(cols)
    n = len(offsets) - 1
    out = np.zeros(max(n, 1), np.int32)
    lib().orc_cc(n, offsets, cols, out)
    return out[:n]


def csum(x):
    x = _f32(x)
    return lib().orc_csum_f32(x, len(x))


def rsum(x):
    x = _f32(x)
    return lib().orc_rsum_f32(x, len(x))


def matching(g: Graph, mm=0.05):
    cap = g.max_dim() + 1
    out = np.zeros(cap, np.int32)
    size = _i64(0)
    nr = C.c_int32(0)
    lib().orc_matching(g.ptr, mm, out, C.byref(size), C.byref(nr))
    return out[: size.value].copy(), nr.value


def msf(i, j, w):
    i, j, w = _a32(i), _a32(j), _f32(w)
    out = np.zeros(max(len(w), 1), np.int32)
    k = _i64(0)
    lib().orc_msf(len(w), i, j, w, out, C.byref(k))
    return out[: k.value].copy()


def woc(g: Graph, pentagons=False):
    cap = g.max_dim() + 1
    out = np.zeros(cap, np.int32)
    size = _i64(0)
    nr = C.c_int32(0)
    lib().orc_woc_ex(g.ptr, out, C.byref(size), C.byref(nr), int(bool(pentagons)))
    return out[: size.value].copy(), nr.value


def conflicted_cycles(g: Graph, max_len, tri_factor=2.0, tol=1e-4):
    cap = int(tri_factor * max(g.n, 1)) + 8
    out = np.zeros(3 * cap, np.int32)
    num = _i64(0)
    raw = _i64(0)
    rc = lib().orc_conflicted_cycles(g.ptr, max_len, tri_factor, tol, out, cap, C.byref(num), C.byref(raw))
    if rc != 0:
        raise RuntimeError("max_cycle_length should be <= 5")
    return out[: 3 * num.value].reshape(-1, 3).copy(), raw.value


class MessagePassing:
    def __init__(self, g: Graph, t1, t2, t3):
        t1, t2, t3 = _a32(t1), _a32(t2), _a32(t3)
        self.ptr = lib().orc_mp_create(g.ptr, t1, t2, t3, len(t1))

    def __del__(self):
        if getattr(self, "ptr", None) and _lib is not None:
            _lib.orc_mp_free(self.ptr)
            self.ptr = None

    def lower_bound(self):
        return lib().orc_mp_lower_bound(self.ptr)

    def send_messages_to_triplets(self):
        lib().orc_mp_send_messages_to_triplets(self.ptr)

    def send_messages_to_edges(self):
        lib().orc_mp_send_messages_to_edges(self.ptr)

    def iteration(self):
        lib().orc_mp_iteration(self.ptr)

    def sizes(self):
        e, t = _i64(0), _i64(0)
        lib().orc_mp_info(self.ptr, C.byref(e), C.byref(t))
        return e.value, t.value

    def edges(self):
        E, _ = self.sizes()
        r, c, w, k = (np.zeros(E, np.int32), np.zeros(E, np.int32), np.zeros(E, np.float32), np.zeros(E, np.int32))
        if E:
            lib().orc_mp_copy_edges(self.ptr, r, c, w, k)
        return r, c, w, k

    def triangles(self):
        _, T = self.sizes()
        a = [np.zeros(max(T, 1), np.int32) for _ in range(3)]
        f = [np.zeros(max(T, 1), np.float32) for _ in range(3)]
        e = [np.zeros(max(T, 1), np.int32) for _ in range(3)]
        if T:
            lib().orc_mp_copy_triangles(self.ptr, *a, *f, *e)
        return [x[:T] for x in a], [x[:T] for x in f], [x[:T] for x in e]


def dual_solver(g: Graph, max_len, num_iter, tri_factor=2.0, num_outer=1, tol=1e-4):
    """Runs the dual solver; returns (new Graph, lb, num_triangles_of_last_pass)."""
    ptr = C.pointer(g.ptr.contents)
    holder = _G(g.ptr.contents)
    nt = _i64(0)
    gp = _G()
    gp = g.ptr
    box = C.pointer(gp)
    lb = lib().orc_dual_solver(box, max_len, num_iter, tri_factor, num_outer, tol, C.byref(nt))
    newp = box.contents
    g.ptr = None  # ownership moved (the old graph was freed if replaced)
    del ptr, holder
    return Graph(newp), lb, nt.value


def dual_lb_f64(i, j, c, mode="D", **kw):
    """The bound of the dual phase of `mode` computed by the FP64 oracle: the
    same triangle selection, every cost, message and bound in double."""
    o = opts(mode, **kw)
    i, j, c = _a32(i), _a32(j), _f32(c)
    lb = C.c_double(0)
    rc = lib().orc_dual_lb_f64(len(c), i, j, c, o.max_cycle_length_lb, o.num_dual_itr_lb, o.tri_memory_factor,
                               o.num_outer_itr_dual, 1e-4, C.byref(lb))
    if rc != 0:
        raise RuntimeError(f"FP64 dual oracle failed with status {rc}")
    return lb.value


def opts(mode=None, **kw):
    o = OrcOpts()
    lib().orc_opts_init(C.byref(o), mode.encode() if mode else None)
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def solve(i, j, c, mode="PD", **kw):
    """Full oracle solve: returns (labels, lb, stats)."""
    i, j, c = _a32(i), _a32(j), _f32(c)
    o = opts(mode, **kw)
    cap = int(max(i.max(initial=-1), j.max(initial=-1)) + 1) if len(c) else 1
    out = np.zeros(max(cap, 1), np.int32)
    nl = _i64(0)
    lb = C.c_double(0)
    st = OrcStats()
    rc = lib().orc_solve(len(c), i, j, c, C.byref(o), out, len(out), C.byref(nl), C.byref(lb), C.byref(st))
    if rc != 0:
        raise RuntimeError(f"oracle solve failed with status {rc}")
    return out[: nl.value].copy(), lb.value, st


def objective(i, j, c, labels):
    i, j, c, labels = _a32(i), _a32(j), _f32(c), _a32(labels)
    return lib().orc_objective(len(c), i, j, c, labels)


def sanitize(i, j, c):
    i, j, c = _a32(i).copy(), _a32(j).copy(), _f32(c).copy()
    cap = int(max(i.max(initial=0), j.max(initial=0)) + 1)
    ids = np.zeros(cap, np.int32)
    n = _i64(0)
    sz = _i64(0)
    lib().orc_sanitize(len(c), i, j, c, C.byref(n), ids, cap, C.byref(sz))
    k = n.value
    return i[:k].copy(), j[:k].copy(), c[:k].copy(), ids[: sz.value].copy()


def gaec(i, j, c, num_nodes=None):
    i, j, c = _a32(i), _a32(j), _f32(c)
    if num_nodes is None:
        num_nodes = int(max(i.max(initial=-1), j.max(initial=-1)) + 1)
    out = np.zeros(max(num_nodes, 1), np.int32)
    lib().orc_gaec(len(c), i, j, c, num_nodes, out)
    return out[:num_nodes]
