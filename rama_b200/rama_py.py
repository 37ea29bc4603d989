"""Drop-in replacement of the reference's `rama_py` Python module.

Same names, arguments and return values as src/rama_py.cu:21-125 of the
reference (pawelswoboda/RAMA):

* ``multicut_solver_options`` -- ctors ``()``, ``(str)`` and the 11-argument
  form, the 13 read/write fields, ``__repr__``;
* ``rama_cuda(i, j, costs, opts)`` -> ``(labels, lb, solve_ms, timeline)``;
* ``rama_cuda_gpu_pointers(i_ptr, j_ptr, costs_ptr, labels_out_ptr, num_nodes,
  num_edges, device, opts)`` -> ``timeline`` (writes max node id + 1 labels;
  ``num_nodes`` is not used, as in the reference);
* ``rama_torch(i, j, costs, opts)`` -> ``[labels, lb]`` (CUDA int32 labels);
* ``read_multicut_file(path)`` -> ``(i, j, costs)``.

Everything runs through the C ABI of librama_b200.so.  One intentional
difference: ``rama_torch`` returns the lower bound as a float64 tensor (the
reference builds an int32 tensor, src/rama_py.cu:54-56, which truncates it).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib

__all__ = ["multicut_solver_options", "rama_cuda", "rama_cuda_gpu_pointers", "rama_torch", "read_multicut_file"]

_MESSAGES = {
    "PD": "Running solver type PD which offers best compute time versus quality tradeoff.",
    "P": "Running purely primal solver (better runtime, worse quality)",
    "PD+": "Running PD+ solver (worse runtime, better quality)",
    "D": "Running dual solver to compute only the lower bound.",
}


class multicut_solver_options:  # noqa: N801 (reference name)
    """Solver options (reference include/multicut_solver_options.h:4-127)."""

    def __init__(self, *args):
        self.max_cycle_length_lb = 5
        self.num_dual_itr_lb = 10
        self.max_cycle_length_primal = 3
        self.num_dual_itr_primal = 5
        self.num_outer_itr_dual = 1
        self.mean_multiplier_mm = 0.05
        self.matching_thresh_crossover_ratio = 0.05
        self.tri_memory_factor = 2.0
        self.only_compute_lb = False
        self.max_time_sec = -1
        self.dump_timeline = False
        self.verbose = True
        self.sanitize_graph = False
        self.woc_pentagons = False  # not in the reference: see rama_options.woc_pentagons
        if len(args) == 1 and isinstance(args[0], str):
            mode = args[0]
            if mode in _MESSAGES:
                print(_MESSAGES[mode], flush=True)
            o = _lib.options(mode)
            for f in ("max_cycle_length_lb", "num_dual_itr_lb", "max_cycle_length_primal", "num_dual_itr_primal",
                      "num_outer_itr_dual"):
                setattr(self, f, int(getattr(o, f)))
            self.only_compute_lb = bool(o.only_compute_lb)
        elif len(args) == 11:
            (self.max_cycle_length_lb, self.num_dual_itr_lb, self.max_cycle_length_primal, self.num_dual_itr_primal,
             self.num_outer_itr_dual, self.mean_multiplier_mm, self.matching_thresh_crossover_ratio,
             self.tri_memory_factor, self.only_compute_lb, self.max_time_sec, self.dump_timeline) = args
        elif args:
            raise TypeError("multicut_solver_options(): expected (), (str) or 11 arguments")

    def _c(self, team=0) -> _lib.RamaOptions:
        o = _lib.RamaOptions()
        o.max_cycle_length_lb = int(self.max_cycle_length_lb)
        o.num_dual_itr_lb = int(self.num_dual_itr_lb)
        o.max_cycle_length_primal = int(self.max_cycle_length_primal)
        o.num_dual_itr_primal = int(self.num_dual_itr_primal)
        o.num_outer_itr_dual = int(self.num_outer_itr_dual)
        o.mean_multiplier_mm = float(self.mean_multiplier_mm)
        o.matching_thresh_crossover_ratio = float(self.matching_thresh_crossover_ratio)
        o.tri_memory_factor = float(self.tri_memory_factor)
        o.only_compute_lb = int(bool(self.only_compute_lb))
        o.max_time_sec = int(self.max_time_sec)
        o.dump_timeline = int(bool(self.dump_timeline))
        o.verbose = int(bool(self.verbose))
        o.sanitize_graph = int(bool(self.sanitize_graph))
        o.team = int(getattr(self, "team", team))
        o.woc_pentagons = int(bool(self.woc_pentagons))
        return o

    def get_string(self):
        f = "{:.6f}".format
        return ("<multicut_solver_options>:" +
                f"max_cycle_length_lb: {int(self.max_cycle_length_lb)}" +
                f", num_dual_itr_lb: {int(self.num_dual_itr_lb)}" +
                f", num_dual_itr_primal: {int(self.num_dual_itr_primal)}" +
                f", max_cycle_length_primal: {int(self.max_cycle_length_primal)}" +
                f", num_outer_itr_dual: {int(self.num_outer_itr_dual)}" +
                f", mean_multiplier_mm: {f(self.mean_multiplier_mm)}" +
                f", matching_thresh_crossover_ratio: {f(self.matching_thresh_crossover_ratio)}" +
                f", tri_memory_factor: {f(self.tri_memory_factor)}" +
                f", only_compute_lb: {int(bool(self.only_compute_lb))}" +
                f", max_time_sec: {int(self.max_time_sec)}" +
                f", sanitize_graph: {int(bool(self.sanitize_graph))}" +
                f", verbose: {int(bool(self.verbose))}\n")

    def __repr__(self):
        return self.get_string()


def _timeline(h: _lib.Handle, opts):
    if not opts.dump_timeline:
        return []
    return [row.tolist() for row in h.timeline()]


def rama_cuda(i, j, edge_costs, opts: multicut_solver_options):
    """Host-list solve (src/rama_py.cu:105-107 -> src/rama_cuda.cu:166-193)."""
    ii = np.ascontiguousarray(np.asarray(i, dtype=np.int32))
    jj = np.ascontiguousarray(np.asarray(j, dtype=np.int32))
    cc = np.ascontiguousarray(np.asarray(edge_costs, dtype=np.float32))
    if not (len(ii) == len(jj) == len(cc)):
        raise RuntimeError("Input shapes must match")
    n = len(cc)
    cap = int(max(ii.max(initial=-1), jj.max(initial=-1)) + 1)
    labels = np.zeros(max(cap, 1), np.int32)
    h = _lib.Handle.default(0)
    nl = C.c_int64(0)
    lb = C.c_double(0)
    ms = C.c_double(0)
    o = opts._c()
    _lib.check(_lib.load().rama_solve_host(h.h, ii.ctypes.data, jj.ctypes.data, cc.ctypes.data, n, C.byref(o),
                                           labels.ctypes.data, len(labels), C.byref(nl), C.byref(lb), C.byref(ms)))
    return labels[: nl.value].tolist(), lb.value, int(ms.value), _timeline(h, opts)


def rama_cuda_gpu_pointers(i_ptr, j_ptr, edge_costs_ptr, node_labels_out_ptr, num_nodes, num_edges, gpuDeviceID,
                           opts: multicut_solver_options):
    """Device-pointer solve (src/rama_py.cu:61-74, 109-116)."""
    h = _lib.Handle.default(int(gpuDeviceID))
    stream = _current_stream(int(gpuDeviceID))
    cap = 1 << 62  # the reference writes node_mapping.size() labels without a bound
    h.solve_device(C.c_void_p(int(i_ptr)), C.c_void_p(int(j_ptr)), C.c_void_p(int(edge_costs_ptr)), int(num_edges),
                   opts._c(), C.c_void_p(int(node_labels_out_ptr)), cap, stream)
    return _timeline(h, opts)


def _current_stream(device):
    try:
        import torch

        if torch.cuda.is_available():
            return C.c_void_p(torch.cuda.current_stream(device).cuda_stream)
    except Exception:
        pass
    return None


def rama_torch(i, j, costs, opts: multicut_solver_options):
    """torch-tensor solve (src/rama_py.cu:21-58)."""
    import torch

    for name, x in (("_i", i), ("_j", j), ("_costs", costs)):
        if not x.is_cuda:
            raise RuntimeError(f"{name} must be a CUDA tensor")
        if not x.is_contiguous():
            raise RuntimeError(f"{name} must be contiguous")
    if i.size(0) != j.size(0) or i.size(0) != costs.size(0):
        raise RuntimeError("Input shapes must match")
    if i.dtype != j.dtype:
        raise RuntimeError("Node indices i, j should be of same type")
    if i.dim() != 1:
        raise RuntimeError("i should be one-dimensional")
    if j.dim() != 1:
        raise RuntimeError("j should be one-dimensional")
    if costs.dim() != 1:
        raise RuntimeError("costs should be one-dimensional")
    if i.dtype != torch.int32 or costs.dtype != torch.float32:
        raise RuntimeError("i, j must be int32 and costs float32")
    device = costs.device.index
    if device is None or device < 0:
        raise RuntimeError("Invalid device ID")
    n = int(i.numel())
    with torch.cuda.device(device):
        cap = int(torch.maximum(i.max(), j.max()).item()) + 1 if n else 0
        labels = torch.empty(max(cap, 1), dtype=torch.int32, device=costs.device)
        h = _lib.Handle.default(device)
        stream = C.c_void_p(torch.cuda.current_stream(device).cuda_stream)
        nl, lb = h.solve_device(C.c_void_p(i.data_ptr()), C.c_void_p(j.data_ptr()), C.c_void_p(costs.data_ptr()), n,
                                opts._c(), C.c_void_p(labels.data_ptr()), labels.numel(), stream)
        lb_t = torch.full((1,), lb, dtype=torch.float64, device=costs.device)
    return [labels[:nl], lb_t]


def read_multicut_file(filename):
    """MULTICUT text format (src/multicut_text_parser.cpp:6-31)."""
    try:
        f = open(filename, "r")
    except OSError:
        raise RuntimeError("Could not open multicut input file " + str(filename))
    with f:
        first = f.readline().rstrip("\n")
        if first != "MULTICUT":
            raise RuntimeError("first line must be 'MULTICUT'")
        toks = f.read().split()
    i_v, j_v, c_v = [], [], []
    for k in range(0, len(toks) - 2, 3):
        try:
            a, b, c = int(toks[k]), int(toks[k + 1]), float(toks[k + 2])
        except ValueError:
            break
        i_v.append(a)
        j_v.append(b)
        c_v.append(c)
    return i_v, j_v, c_v
