"""ctypes binding of librama_b200.so (the C ABI in include/rama_b200.h).

The shared library is built in-tree by rama_b200.build (nvcc for sm_100a).
There is no CPU fallback: importing a solver entry point without the built
library raises ImportError.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librama_b200.so")

RAMA_OK = 0
RAMA_ERR_INVALID_ARG = 1
RAMA_ERR_OOM = 2
RAMA_ERR_CUDA = 3
RAMA_ERR_ITER_LIMIT = 4
RAMA_ERR_BAD_CONTRACTION = 5

STEP = dict(INIT=1, CONTRACT=2, MATCHING=3, WOC=4, MSF=5, CC=6, CYCLES=7, MP=8, DUAL=9, CSUM=10, SORT=11,
            COARSEN=12)


class RamaOptions(C.Structure):
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
        ("team", C.c_int32),
        ("woc_pentagons", C.c_int32),
    ]


class RamaStats(C.Structure):
    _fields_ = [
        ("rounds", C.c_int32),
        ("matching_rounds", C.c_int32),
        ("mst_rounds", C.c_int32),
        ("timeline_rounds", C.c_int32),
        ("dual_oom", C.c_int32),
        ("team", C.c_int32),
        ("triangles", C.c_int64),
        ("edges_after_dual", C.c_int64),
        ("workspace_peak", C.c_int64),
        ("device_ms", C.c_double),
        ("alg_bytes", C.c_double),
        ("phase_ms", C.c_double * 32),
        ("phase_bytes", C.c_double * 32),
    ]

class RamaTuning(C.Structure):
    _fields_ = [
        ("grid_ctas_per_sm", C.c_int32),
        ("grid_small_ctas_per_sm", C.c_int32),
        ("grid_small_max", C.c_int64),
        ("cluster_ctas", C.c_int32),
        ("single_cluster_min", C.c_int64),
        ("single_grid_min", C.c_int64),
        ("batch_cluster_min", C.c_int64),
        ("batch_cluster_share", C.c_float),
        ("cta_threads", C.c_int32),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


PHASES = ("init", "cycles", "mp_build", "mp_iter", "dual_commit", "matching", "woc", "contract", "other",
          "match_iter", "csort_big", "csr", "csort_slot", "csort_scatter", "csort_rank", "contract_runs",
          "match_labels", "match_first", "woc_msf", "woc_csr", "woc_checks", "woc_root", "woc_paths",
          "cyc_search", "mp_norm", "mp_chords", "mp_incid", "-", "-", "-", "-", "-")


_P = C.c_void_p


class StepArgs(C.Structure):
    _fields_ = [
        ("op", C.c_int32), ("team", C.c_int32),
        ("row", _P), ("col", _P), ("cost", _P), ("n", C.c_int64), ("rows", C.c_int32), ("cols", C.c_int32),
        ("i", _P), ("j", _P), ("c", _P), ("m", C.c_int64), ("keys", _P), ("key_bits", C.c_int32),
        ("map", _P), ("map_size", C.c_int64),
        ("t1", _P), ("t2", _P), ("t3", _P), ("T", C.c_int64),
        ("offsets", _P), ("adj", _P), ("num_nodes", C.c_int32), ("adj_len", C.c_int64),
        ("max_cycle_length", C.c_int32), ("num_iter", C.c_int32), ("num_outer", C.c_int32),
        ("tri_memory_factor", C.c_float), ("mean_multiplier_mm", C.c_float), ("tol", C.c_float),
        ("out_row", _P), ("out_col", _P), ("out_cost", _P), ("out_cap", C.c_int64),
        ("out_map", _P), ("out_map_cap", C.c_int64),
        ("out_t1", _P), ("out_t2", _P), ("out_t3", _P), ("out_tri_cap", C.c_int64),
        ("out_flags", _P), ("out_keys", _P),
        ("out_n", C.c_int64), ("out_rows", C.c_int32), ("out_cols", C.c_int32),
        ("out_count", C.c_int64), ("out_raw", C.c_int64), ("out_nr", C.c_int32),
        ("out_lb0", C.c_double), ("out_lb1", C.c_double), ("status", C.c_int32),
    ]


# every symbol include/rama_b200.h declares
EXPORTS = ("rama_options_init", "rama_create", "rama_destroy", "rama_solve", "rama_solve_host", "rama_get_timeline",
           "rama_solve_batch", "rama_batch_launch", "rama_batch_poll", "rama_batch_wait", "rama_get_stats",
           "rama_last_error", "rama_objective", "rama_step", "rama_solve_small_static", "rama_parse_multicut",
           "rama_parse_multicut_host", "rama_get_tuning", "rama_set_tuning")

_lib = None
_lock = threading.Lock()


class RamaError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


def load():
    """Loads the in-tree shared library (raises ImportError when it is missing)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is not built; run `python -m rama_b200.build`")
        L = C.CDLL(LIB_PATH)
        i64, i32, P = C.c_int64, C.c_int32, C.c_void_p
        L.rama_options_init.argtypes = [C.POINTER(RamaOptions), C.c_char_p]
        L.rama_create.argtypes = [C.c_int, C.c_uint64, C.POINTER(P)]
        L.rama_destroy.argtypes = [P]
        L.rama_destroy.restype = None
        L.rama_solve.argtypes = [P, P, P, P, i64, C.POINTER(RamaOptions), P, i64, C.POINTER(i64),
                                 C.POINTER(C.c_double), P]
        L.rama_solve_host.argtypes = [P, P, P, P, i64, C.POINTER(RamaOptions), P, i64, C.POINTER(i64),
                                      C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.rama_get_timeline.argtypes = [P, P, i64, C.POINTER(i32), C.POINTER(i64)]
        L.rama_solve_batch.argtypes = [P, P, P, P, P, i32, C.POINTER(RamaOptions), P, P, P, P, P, P]
        L.rama_batch_launch.argtypes = [P, P, P, P, P, i32, P, i32, P, P, P]
        L.rama_batch_poll.argtypes = [P]
        L.rama_batch_wait.argtypes = [P, P, P, P]
        L.rama_get_stats.argtypes = [P, C.POINTER(RamaStats)]
        L.rama_solve_small_static.argtypes = [P, P, P, i64, C.POINTER(RamaOptions), P, i64, C.POINTER(i64),
                                              C.POINTER(C.c_double), P]
        L.rama_parse_multicut.argtypes = [P, P, i64, P, P, P, i64, C.POINTER(i64), P]
        L.rama_parse_multicut_host.argtypes = [P, C.c_char_p, i64, P, P, P, i64, C.POINTER(i64)]
        L.rama_last_error.restype = C.c_char_p
        L.rama_objective.argtypes = [P, P, P, P, i64, P, C.POINTER(C.c_double), P]
        L.rama_step.argtypes = [P, C.POINTER(StepArgs), P]
        L.rama_get_tuning.argtypes = [P, C.POINTER(RamaTuning)]
        L.rama_set_tuning.argtypes = [P, C.POINTER(RamaTuning)]
        _lib = L
        return L


def check(rc):
    if rc != RAMA_OK:
        msg = load().rama_last_error().decode(errors="replace")
        raise RamaError(rc, msg)


def options(mode=None, **kw) -> RamaOptions:
    o = RamaOptions()
    load().rama_options_init(C.byref(o), mode.encode() if mode else None)
    for k, v in kw.items():
        setattr(o, k, v)
    return o


class Handle:
    """Owns one solver context (device workspace) on a device."""

    _per_device: dict = {}

    def __init__(self, device=0, workspace_bytes=0):
        self.device = device
        h = C.c_void_p()
        check(load().rama_create(device, workspace_bytes, C.byref(h)))
        self.h = h

    @classmethod
    def default(cls, device=0):
        key = (device, threading.get_ident())
        if key not in cls._per_device:
            cls._per_device[key] = cls(device)
        return cls._per_device[key]

    def close(self):
        if self.h:
            load().rama_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def tuning(self) -> RamaTuning:
        t = RamaTuning()
        check(load().rama_get_tuning(self.h, C.byref(t)))
        return t

    def set_tuning(self, t: RamaTuning):
        check(load().rama_set_tuning(self.h, C.byref(t)))

    def stats(self) -> RamaStats:
        s = RamaStats()
        check(load().rama_get_stats(self.h, C.byref(s)))
        return s

    def solve_device(self, d_i, d_j, d_c, n, opts, d_labels, cap, stream=None):
        nl = C.c_int64(0)
        lb = C.c_double(0)
        check(load().rama_solve(self.h, d_i, d_j, d_c, n, C.byref(opts), d_labels, cap, C.byref(nl), C.byref(lb),
                                stream))
        return nl.value, lb.value

    def timeline(self):
        r = C.c_int32(0)
        nl = C.c_int64(0)
        check(load().rama_get_timeline(self.h, None, 0, C.byref(r), C.byref(nl)))
        import numpy as np

        out = np.zeros(max(r.value * nl.value, 1), np.int32)
        check(load().rama_get_timeline(self.h, out.ctypes.data, out.size, C.byref(r), C.byref(nl)))
        return out[: r.value * nl.value].reshape(r.value, nl.value)

    def step(self, args: StepArgs, stream=None):
        check(load().rama_step(self.h, C.byref(args), stream))
        return args
