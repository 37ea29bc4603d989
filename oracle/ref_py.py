"""ctypes view of the reference solver built from source (test infrastructure).

oracle/build_ref.sh compiles the reference's own sources plus
oracle/ref_harness.cu into oracle/_ref/librama_ref.so.  Tests use it as the
parity oracle on the GPU; bench.py --impl reference times ref_rama*.
Everything here needs a CUDA device.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "librama_ref.so")

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_i64 = C.c_int64
_P64 = C.POINTER(C.c_int64)
_PI = C.POINTER(C.c_int)
_PD = C.POINTER(C.c_double)
_lib = None


def available():
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(LIB_PATH)
        L.ref_last_error.restype = C.c_char_p
        L.ref_init.argtypes = [_i64, _i32p, _i32p, _f32p, _P64, _i32p, _i32p, _f32p, _PI, _PI]
        L.ref_contract.argtypes = [_i64, _i32p, _i32p, _f32p, C.c_int, C.c_int, _i32p, _i64, _P64, _i32p, _i32p,
                                   _f32p, _PI, _PI]
        L.ref_matching.argtypes = [_i64, _i32p, _i32p, _f32p, C.c_int, C.c_int, C.c_float, _i32p, _i64, _P64, _PI]
        L.ref_cc.argtypes = [C.c_int, _i32p, _i64, _i32p, _i32p]
        L.ref_msf.argtypes = [_i64, _i32p, _i32p, _f32p, _i32p, _i32p, _f32p, _P64]
        L.ref_conflicted_cycles.argtypes = [_i64, _i32p, _i32p, _f32p, C.c_int, C.c_int, C.c_int, C.c_float,
                                            C.c_float, _i32p, _i64, _P64]
        L.ref_mp.argtypes = [_i64, _i32p, _i32p, _f32p, C.c_int, C.c_int, _i64, _i32p, _i32p, _i32p, C.c_int,
                             C.c_int, _PD, _PD, _P64, _i32p, _i32p, _f32p, _i64]
        L.ref_dual.argtypes = [_i64, _i32p, _i32p, _f32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_int,
                               _PD, _P64, _i32p, _i32p, _f32p, _PI, _PI, _i64]
        L.ref_woc.argtypes = [_i64, _i32p, _i32p, _f32p, C.c_int, C.c_int, _i32p, _i64, _P64, _PI]
        L.ref_woc_pentagons.argtypes = [_i64, _i32p, _i32p, _f32p, C.c_int, C.c_int, _i32p, _i64, _P64, _PI]
        L.ref_rama.argtypes = [_i64, _i32p, _i32p, _f32p, _i32p, _f32p, _i32p, _i64, _P64, _PD, _PI]
        L.ref_rama_device.argtypes = [_i64, C.c_void_p, C.c_void_p, C.c_void_p, _i32p, _f32p, C.c_void_p, _i64,
                                      _P64, _PD]
        _lib = L
    return _lib


def _check(rc):
    if rc != 0:
        raise RuntimeError(f"reference call failed ({rc}): {lib().ref_last_error().decode()}")


def _a32(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.int32))


def _f32(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.float32))


def init(i, j, c):
    i, j, c = _a32(i), _a32(j), _f32(c)
    E = len(c)
    r, co, w = np.zeros(max(E, 1), np.int32), np.zeros(max(E, 1), np.int32), np.zeros(max(E, 1), np.float32)
    n, rows, cols = _i64(0), C.c_int(0), C.c_int(0)
    _check(lib().ref_init(E, i, j, c, C.byref(n), r, co, w, C.byref(rows), C.byref(cols)))
    k = n.value
    return r[:k], co[:k], w[:k], rows.value, cols.value


def contract(row, col, cost, rows, cols, node_map):
    row, col, cost, node_map = _a32(row), _a32(col), _f32(cost), _a32(node_map)
    E = len(cost)
    r, co, w = np.zeros(max(E, 1), np.int32), np.zeros(max(E, 1), np.int32), np.zeros(max(E, 1), np.float32)
    n, ro, cc = _i64(0), C.c_int(0), C.c_int(0)
    _check(lib().ref_contract(E, row, col, cost, rows, cols, node_map, len(node_map), C.byref(n), r, co, w,
                              C.byref(ro), C.byref(cc)))
    k = n.value
    return r[:k], co[:k], w[:k], ro.value, cc.value


def matching(row, col, cost, rows, cols, mm):
    row, col, cost = _a32(row), _a32(col), _f32(cost)
    cap = max(rows, cols) + 2
    out = np.zeros(cap, np.int32)
    sz, nr = _i64(0), C.c_int(0)
    _check(lib().ref_matching(len(cost), row, col, cost, rows, cols, mm, out, cap, C.byref(sz), C.byref(nr)))
    return out[: sz.value], nr.value


def cc(offsets, cols):
    offsets, cols = _a32(offsets), _a32(cols)
    n = len(offsets) - 1
    out = np.zeros(max(n, 1), np.int32)
    _check(lib().ref_cc(n, offsets, len(cols), cols if len(cols) else np.zeros(1, np.int32), out))
    return out[:n]


def msf(i, j, w):
    i, j, w = _a32(i), _a32(j), _f32(w)
    m = len(w)
    a, b, c = np.zeros(max(m, 1), np.int32), np.zeros(max(m, 1), np.int32), np.zeros(max(m, 1), np.float32)
    k = _i64(0)
    _check(lib().ref_msf(m, i, j, w, a, b, c, C.byref(k)))
    return a[: k.value], b[: k.value], c[: k.value]


def conflicted_cycles(row, col, cost, rows, cols, max_len, tri_factor=2.0, tol=1e-4):
    row, col, cost = _a32(row), _a32(col), _f32(cost)
    cap = int(tri_factor * max(len(cost), 1)) * 4 + 64
    out = np.zeros(3 * cap, np.int32)
    n = _i64(0)
    _check(lib().ref_conflicted_cycles(len(cost), row, col, cost, rows, cols, max_len, tri_factor, tol, out, cap,
                                       C.byref(n)))
    return out[: 3 * n.value].reshape(-1, 3)


def mp(row, col, cost, rows, cols, tris, pre_triplets, iters):
    row, col, cost = _a32(row), _a32(col), _f32(cost)
    tris = np.asarray(tris, np.int32).reshape(-1, 3)
    t1, t2, t3 = (np.ascontiguousarray(tris[:, k]) for k in range(3))
    cap = len(cost) + 3 * len(tris) + 1
    r, co, w = np.zeros(cap, np.int32), np.zeros(cap, np.int32), np.zeros(cap, np.float32)
    lb0, lb1, n = C.c_double(0), C.c_double(0), _i64(0)
    _check(lib().ref_mp(len(cost), row, col, cost, rows, cols, len(t1), t1, t2, t3, int(pre_triplets), iters,
                        C.byref(lb0), C.byref(lb1), C.byref(n), r, co, w, cap))
    k = n.value
    return lb0.value, lb1.value, r[:k], co[:k], w[:k]


def dual(row, col, cost, rows, cols, max_len, num_iter, tri_factor=2.0, num_outer=1):
    row, col, cost = _a32(row), _a32(col), _f32(cost)
    cap = int(len(cost) * (1 + 6 * tri_factor)) + 16
    r, co, w = np.zeros(cap, np.int32), np.zeros(cap, np.int32), np.zeros(cap, np.float32)
    lb, n, ro, cc_ = C.c_double(0), _i64(0), C.c_int(0), C.c_int(0)
    _check(lib().ref_dual(len(cost), row, col, cost, rows, cols, max_len, num_iter, tri_factor, num_outer,
                          C.byref(lb), C.byref(n), r, co, w, C.byref(ro), C.byref(cc_), cap))
    k = n.value
    return lb.value, r[:k], co[:k], w[:k], ro.value, cc_.value


def woc(row, col, cost, rows, cols, pentagons=False):
    """The reference's forest contraction; `pentagons` runs it with its
    (otherwise disabled) 5-cycle forest check."""
    row, col, cost = _a32(row), _a32(col), _f32(cost)
    cap = max(rows, cols) + 2
    out = np.zeros(cap, np.int32)
    sz, nr = _i64(0), C.c_int(0)
    f = lib().ref_woc_pentagons if pentagons else lib().ref_woc
    _check(f(len(cost), row, col, cost, rows, cols, out, cap, C.byref(sz), C.byref(nr)))
    return out[: sz.value], nr.value


def opts_arrays(o: dict):
    oi = np.array([o["max_cycle_length_lb"], o["num_dual_itr_lb"], o["max_cycle_length_primal"],
                   o["num_dual_itr_primal"], o["num_outer_itr_dual"], int(o["only_compute_lb"]),
                   o["max_time_sec"], int(o["dump_timeline"]), int(o["sanitize_graph"])], np.int32)
    of = np.array([o["mean_multiplier_mm"], o["matching_thresh_crossover_ratio"], o["tri_memory_factor"]],
                  np.float32)
    return oi, of


MODES = {
    "PD": dict(max_cycle_length_lb=5, num_dual_itr_lb=10, max_cycle_length_primal=3, num_dual_itr_primal=5,
               num_outer_itr_dual=1),
    "P": dict(max_cycle_length_lb=0, num_dual_itr_lb=0, max_cycle_length_primal=0, num_dual_itr_primal=0,
              num_outer_itr_dual=1),
    "PD+": dict(max_cycle_length_lb=5, num_dual_itr_lb=10, max_cycle_length_primal=5, num_dual_itr_primal=10,
                num_outer_itr_dual=1),
    "D": dict(max_cycle_length_lb=5, num_dual_itr_lb=10, max_cycle_length_primal=3, num_dual_itr_primal=5,
              num_outer_itr_dual=5, only_compute_lb=True),
}


def mode_opts(mode="PD", **kw):
    o = dict(mean_multiplier_mm=0.05, matching_thresh_crossover_ratio=0.05, tri_memory_factor=2.0,
             only_compute_lb=False, max_time_sec=-1, dump_timeline=False, sanitize_graph=False)
    o.update(MODES[mode])
    o.update(kw)
    return o


def rama(i, j, c, mode="PD", **kw):
    """reference rama_cuda host overload: returns (labels, lb, solve_ms)."""
    i, j, c = _a32(i), _a32(j), _f32(c)
    oi, of = opts_arrays(mode_opts(mode, **kw))
    cap = int(max(i.max(initial=0), j.max(initial=0))) + 2
    out = np.zeros(cap, np.int32)
    nl, lb, t = _i64(0), C.c_double(0), C.c_int(0)
    _check(lib().ref_rama(len(c), i, j, c, oi, of, out, cap, C.byref(nl), C.byref(lb), C.byref(t)))
    return out[: nl.value], lb.value, t.value


def rama_device(d_i, d_j, d_c, n_edges, d_labels, labels_cap, mode="PD", **kw):
    """reference rama_cuda device overload on raw device pointers; returns (num_labels, lb)."""
    oi, of = opts_arrays(mode_opts(mode, **kw))
    nl, lb = _i64(0), C.c_double(0)
    _check(lib().ref_rama_device(n_edges, d_i, d_j, d_c, oi, of, d_labels, labels_cap, C.byref(nl), C.byref(lb)))
    return nl.value, lb.value
