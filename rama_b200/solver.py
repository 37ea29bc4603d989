"""Python access to the solver's C ABI with torch device memory.

``Solver.solve`` / ``Solver.solve_batch`` run whole solves; the ``step_*``
methods run single solver steps (RAMA_STEP_*), which the parity tests compare
with the CPU oracle and the reference.  torch provides device buffers and the
stream only.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib


def _torch():
    import torch

    return torch


def _dev(x, dtype):
    torch = _torch()
    a = np.ascontiguousarray(np.asarray(x, dtype=dtype))
    if a.size == 0:
        a = np.zeros(1, dtype=dtype)
    return torch.from_numpy(a).cuda()


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


class Solver:
    def __init__(self, device=0, workspace_bytes=0):
        self.device = device
        self.handle = _lib.Handle(device, workspace_bytes)

    # ------------------------------------------------------------------ solve
    def solve_device(self, d_i, d_j, d_c, mode="PD", team=0, labels=None, stream=None, **kw):
        """Device tensors in, (labels tensor, lb) out."""
        torch = _torch()
        n = int(d_c.numel())
        o = _lib.options(mode, team=team, **kw)
        if labels is None:
            cap = int(torch.maximum(d_i.max(), d_j.max()).item()) + 1 if n else 1
            labels = torch.empty(cap, dtype=torch.int32, device=d_c.device)
        st = stream if stream is not None else C.c_void_p(torch.cuda.current_stream().cuda_stream)
        nl, lb = self.handle.solve_device(_p(d_i), _p(d_j), _p(d_c), n, o, _p(labels), labels.numel(), st)
        return labels[:nl], lb

    def solve(self, i, j, c, mode="PD", team=0, **kw):
        """numpy in, (labels numpy, lb, stats) out."""
        d_i, d_j, d_c = _dev(i, np.int32), _dev(j, np.int32), _dev(c, np.float32)
        n = len(c)
        if n == 0:
            return np.zeros(0, np.int32), 0.0, self.handle.stats()
        lab, lb = self.solve_device(d_i[:n], d_j[:n], d_c[:n], mode=mode, team=team, **kw)
        _torch().cuda.synchronize()
        return lab.cpu().numpy(), lb, self.handle.stats()

    def solve_batch_device(self, d_i, d_j, d_c, edge_offsets, label_offsets, mode="PD", d_labels=None, stream=None,
                           **kw):
        torch = _torch()
        count = len(edge_offsets) - 1
        eo = np.ascontiguousarray(edge_offsets, dtype=np.int64)
        lo = np.ascontiguousarray(label_offsets, dtype=np.int64)
        if d_labels is None:
            d_labels = torch.empty(max(int(lo[-1]), 1), dtype=torch.int32, device=d_c.device)
        nl = np.zeros(count, np.int64)
        lbs = np.zeros(count, np.float64)
        st_codes = np.zeros(count, np.int32)
        o = _lib.options(mode, **kw)
        st = stream if stream is not None else C.c_void_p(torch.cuda.current_stream().cuda_stream)
        rc = _lib.load().rama_solve_batch(self.handle.h, _p(d_i), _p(d_j), _p(d_c), eo.ctypes.data, count,
                                          C.byref(o), _p(d_labels), lo.ctypes.data, nl.ctypes.data, lbs.ctypes.data,
                                          st_codes.ctypes.data, st)
        return d_labels, nl, lbs, st_codes, rc

    def solve_batch(self, batch, mode="PD", **kw):
        """instances.Batch in; list of (labels numpy, lb) and per-instance status out."""
        d_i, d_j, d_c = _dev(batch.i, np.int32), _dev(batch.j, np.int32), _dev(batch.c, np.float32)
        lo = np.zeros(batch.count + 1, np.int64)
        lo[1:] = np.cumsum(batch.node_counts)
        d_lab, nl, lbs, st, rc = self.solve_batch_device(d_i, d_j, d_c, batch.edge_offsets, lo, mode=mode, **kw)
        _torch().cuda.synchronize()
        lab = d_lab.cpu().numpy()
        out = [(lab[lo[k]:lo[k] + nl[k]].copy(), float(lbs[k])) for k in range(batch.count)]
        return out, st, rc

    def parse_multicut(self, text: bytes, stream=None):
        """MULTICUT text (bytes) parsed on the device: (i, j, costs) as device tensors."""
        torch = _torch()
        n = len(text)
        d_text = torch.frombuffer(bytearray(text), dtype=torch.uint8).cuda() if n else torch.empty(1, dtype=torch.uint8,
                                                                                                   device="cuda")
        cap = (n + 1) // 6 + 1
        d_i = torch.empty(cap, dtype=torch.int32, device="cuda")
        d_j = torch.empty(cap, dtype=torch.int32, device="cuda")
        d_c = torch.empty(cap, dtype=torch.float32, device="cuda")
        ne = C.c_int64(0)
        st = stream if stream is not None else C.c_void_p(torch.cuda.current_stream().cuda_stream)
        _lib.check(_lib.load().rama_parse_multicut(self.handle.h, _p(d_text), n, _p(d_i), _p(d_j), _p(d_c), cap,
                                                   C.byref(ne), st))
        k = ne.value
        return d_i[:k], d_j[:k], d_c[:k]

    def objective(self, d_i, d_j, d_c, d_labels):
        obj = C.c_double(0)
        torch = _torch()
        st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        _lib.check(_lib.load().rama_objective(self.handle.h, _p(d_i), _p(d_j), _p(d_c), int(d_c.numel()),
                                              _p(d_labels), C.byref(obj), st))
        return obj.value

    def stats(self):
        return self.handle.stats()

    # ------------------------------------------------------------------ steps
    def _graph_args(self, a, row, col, cost, rows, cols, keep):
        r, c, w = _dev(row, np.int32), _dev(col, np.int32), _dev(cost, np.float32)
        keep += [r, c, w]
        a.row, a.col, a.cost = _p(r), _p(c), _p(w)
        a.n = len(cost)
        a.rows, a.cols = rows, cols

    def _out_graph(self, a, cap, keep):
        torch = _torch()
        r = torch.empty(max(cap, 1), dtype=torch.int32, device="cuda")
        c = torch.empty(max(cap, 1), dtype=torch.int32, device="cuda")
        w = torch.empty(max(cap, 1), dtype=torch.float32, device="cuda")
        keep += [r, c, w]
        a.out_row, a.out_col, a.out_cost, a.out_cap = _p(r), _p(c), _p(w), cap
        return r, c, w

    def _run(self, a):
        self.handle.step(a, C.c_void_p(_torch().cuda.current_stream().cuda_stream))
        _torch().cuda.synchronize()
        return a

    def step_init(self, i, j, c, team=1):
        a = _lib.StepArgs(op=_lib.STEP["INIT"], team=team)
        keep = []
        di, dj, dc = _dev(i, np.int32), _dev(j, np.int32), _dev(c, np.float32)
        keep += [di, dj, dc]
        a.i, a.j, a.c, a.m = _p(di), _p(dj), _p(dc), len(c)
        r, co, w = self._out_graph(a, len(c), keep)
        self._run(a)
        k = a.out_n
        return r[:k].cpu().numpy(), co[:k].cpu().numpy(), w[:k].cpu().numpy(), a.out_rows, a.out_cols

    def step_contract(self, row, col, cost, rows, cols, node_map, team=1):
        a = _lib.StepArgs(op=_lib.STEP["CONTRACT"], team=team)
        keep = []
        self._graph_args(a, row, col, cost, rows, cols, keep)
        m = _dev(node_map, np.int32)
        keep.append(m)
        a.map, a.map_size = _p(m), len(node_map)
        r, co, w = self._out_graph(a, len(cost), keep)
        self._run(a)
        k = a.out_n
        return r[:k].cpu().numpy(), co[:k].cpu().numpy(), w[:k].cpu().numpy(), a.out_rows, a.out_cols

    def step_coarsen(self, row, col, cost, rows, cols, node_map, team=1):
        """The solver's contraction of a graph by a node map: parallel edges
        summed, self-loops removed (dims taken before, as the reference does);
        returns (row, col, cost, rows, cols, bad)."""
        a = _lib.StepArgs(op=_lib.STEP["COARSEN"], team=team)
        keep = []
        self._graph_args(a, row, col, cost, rows, cols, keep)
        m = _dev(node_map, np.int32)
        keep.append(m)
        a.map, a.map_size = _p(m), len(node_map)
        r, co, w = self._out_graph(a, len(cost), keep)
        self._run(a)
        k = a.out_n
        return (r[:k].cpu().numpy(), co[:k].cpu().numpy(), w[:k].cpu().numpy(), a.out_rows, a.out_cols,
                bool(a.out_nr))

    def _map_step(self, op, row, col, cost, rows, cols, team, mm=0.05, max_cycle_length=0):
        torch = _torch()
        a = _lib.StepArgs(op=_lib.STEP[op], team=team, mean_multiplier_mm=mm, max_cycle_length=max_cycle_length)
        keep = []
        self._graph_args(a, row, col, cost, rows, cols, keep)
        cap = max(rows, cols) + 2
        out = torch.empty(cap, dtype=torch.int32, device="cuda")
        keep.append(out)
        a.out_map, a.out_map_cap = _p(out), cap
        self._run(a)
        return out[: a.out_count].cpu().numpy(), a.out_nr

    def step_matching(self, row, col, cost, rows, cols, mm=0.05, team=1):
        return self._map_step("MATCHING", row, col, cost, rows, cols, team, mm)

    def step_woc(self, row, col, cost, rows, cols, team=1, pentagons=False):
        """Forest contraction map; `pentagons` adds the 5-cycle forest check."""
        return self._map_step("WOC", row, col, cost, rows, cols, team, max_cycle_length=5 if pentagons else 0)

    def step_msf(self, i, j, w, team=1):
        torch = _torch()
        a = _lib.StepArgs(op=_lib.STEP["MSF"], team=team)
        di, dj, dw = _dev(i, np.int32), _dev(j, np.int32), _dev(w, np.float32)
        fl = torch.zeros(max(len(w), 1), dtype=torch.uint8, device="cuda")
        a.i, a.j, a.c, a.m, a.out_flags = _p(di), _p(dj), _p(dw), len(w), _p(fl)
        self._run(a)
        return fl[: len(w)].cpu().numpy().astype(bool)

    def step_cc(self, offsets, adj, team=1):
        torch = _torch()
        a = _lib.StepArgs(op=_lib.STEP["CC"], team=team)
        do, da = _dev(offsets, np.int32), _dev(adj, np.int32)
        n = len(offsets) - 1
        out = torch.empty(max(n, 1), dtype=torch.int32, device="cuda")
        a.offsets, a.adj, a.num_nodes, a.adj_len, a.out_map = _p(do), _p(da), n, len(adj), _p(out)
        self._run(a)
        return out[:n].cpu().numpy()

    def step_cycles(self, row, col, cost, rows, cols, max_len, tri_factor=2.0, tol=1e-4, team=1):
        torch = _torch()
        a = _lib.StepArgs(op=_lib.STEP["CYCLES"], team=team, max_cycle_length=max_len, tri_memory_factor=tri_factor,
                          tol=tol)
        keep = []
        self._graph_args(a, row, col, cost, rows, cols, keep)
        cap = int(tri_factor * max(len(cost), 1)) + 8
        t = [torch.empty(cap, dtype=torch.int32, device="cuda") for _ in range(3)]
        a.out_t1, a.out_t2, a.out_t3, a.out_tri_cap = _p(t[0]), _p(t[1]), _p(t[2]), cap
        self._run(a)
        k = a.out_count
        tri = np.stack([x[:k].cpu().numpy() for x in t], axis=1) if k else np.zeros((0, 3), np.int32)
        return tri, a.out_raw

    def step_mp(self, row, col, cost, rows, cols, tris, iters, team=1):
        tris = np.asarray(tris, np.int32).reshape(-1, 3)
        a = _lib.StepArgs(op=_lib.STEP["MP"], team=team, num_iter=iters)
        keep = []
        self._graph_args(a, row, col, cost, rows, cols, keep)
        t = [_dev(np.ascontiguousarray(tris[:, k]), np.int32) for k in range(3)]
        keep += t
        a.t1, a.t2, a.t3, a.T = _p(t[0]), _p(t[1]), _p(t[2]), len(tris)
        r, co, w = self._out_graph(a, len(cost) + 3 * len(tris), keep)
        self._run(a)
        k = a.out_n
        return a.out_lb0, a.out_lb1, r[:k].cpu().numpy(), co[:k].cpu().numpy(), w[:k].cpu().numpy()

    def step_dual(self, row, col, cost, rows, cols, max_len, num_iter, tri_factor=2.0, num_outer=1, team=1):
        a = _lib.StepArgs(op=_lib.STEP["DUAL"], team=team, max_cycle_length=max_len, num_iter=num_iter,
                          tri_memory_factor=tri_factor, num_outer=num_outer, tol=1e-4)
        keep = []
        self._graph_args(a, row, col, cost, rows, cols, keep)
        cap = int(len(cost) * (1 + 6 * tri_factor)) + 16
        r, co, w = self._out_graph(a, cap, keep)
        self._run(a)
        k = a.out_n
        return a.out_lb0, r[:k].cpu().numpy(), co[:k].cpu().numpy(), w[:k].cpu().numpy(), a.out_rows, a.out_cols

    def step_csum(self, x, team=1):
        a = _lib.StepArgs(op=_lib.STEP["CSUM"], team=team)
        d = _dev(x, np.float32)
        a.c, a.m = _p(d), len(x)
        self._run(a)
        return a.out_lb0

    def step_sort(self, keys, vals, bits, team=1):
        torch = _torch()
        a = _lib.StepArgs(op=_lib.STEP["SORT"], team=team, key_bits=bits)
        k = _dev(np.asarray(keys, np.uint64).view(np.int64), np.int64)
        v = _dev(vals, np.int32)
        ok = torch.empty(max(len(keys), 1), dtype=torch.int64, device="cuda")
        ov = torch.empty(max(len(keys), 1), dtype=torch.int32, device="cuda")
        a.keys, a.i, a.m, a.out_keys, a.out_map = _p(k), _p(v), len(keys), _p(ok), _p(ov)
        self._run(a)
        n = len(keys)
        return ok[:n].cpu().numpy().view(np.uint64), ov[:n].cpu().numpy()
