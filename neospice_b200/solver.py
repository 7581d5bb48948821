"""Python host layer over libnsgpu: topologies (host symbolic phase) and
batches (device refactor / solve / transposed solve).

PyTorch provides device memory and streams only; every numeric step runs in
libnsgpu's CUDA kernels.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib as L


# Engine codes of nsg_topology_order_solver (NSG_SOLVER_*).
SOLVERS = {"markowitz": 0, "amdlu": 1, "auto-amdlu": 2}


def select_solver(num_vars: int, is_linear: bool) -> str:
    """make_solver's engine choice (src/core/make_solver.cpp:156-178), with
    the NEOSPICE_SOLVER / NEOSPICE_FORCE_AMDLU overrides."""
    k = L.lib().nsg_solver_select(int(num_vars), int(bool(is_linear)))
    return {v: n for n, v in SOLVERS.items()}[k]


def amd_order(n, col_ptr, row_idx) -> np.ndarray:
    """amd_ordering (src/core/amd.cpp:14-143): perm[k] = column eliminated at
    step k."""
    cp = np.ascontiguousarray(col_ptr, np.int32)
    ri = np.ascontiguousarray(row_idx, np.int32)
    perm = np.zeros(int(n), np.int32)
    L.check(L.lib().nsg_amd_order(int(n), L.iptr(cp), L.iptr(ri), L.iptr(perm)))
    return perm


class Topology:
    """One factored sparsity structure: pivot sequence + fill pattern.

    ``Topology.order`` runs the Sparse-1.3-compatible Markowitz ordering on
    the host (NeoSolver::symbolic + the first NeoSolver::numeric,
    src/core/neo_solver.cpp:184-245).  ``Topology.import_structure`` takes a
    structure computed by the reference's own NeoSolver instead.
    """

    def __init__(self, handle: ctypes.c_void_p):
        self._h = handle

    @property
    def handle(self):
        return self._h

    @classmethod
    def order(cls, n, col_ptr, row_idx, values, diag_gmin=0.0, solver="markowitz") -> "Topology":
        """Symbolic phase + first numeric().  ``solver``: "markowitz"
        (NeoSolver), "amdlu" (AmdLuSolver) or "auto-amdlu" (make_solver's
        AutoFallbackSolver: AMD-LU, Markowitz if the first factor is
        singular)."""
        cp = np.ascontiguousarray(col_ptr, np.int32)
        ri = np.ascontiguousarray(row_idx, np.int32)
        v = np.ascontiguousarray(values, np.float64)
        h = ctypes.c_void_p()
        L.check(L.lib().nsg_topology_order_solver(int(n), len(ri), L.iptr(cp), L.iptr(ri),
                                                  L.dptr(v), float(diag_gmin), SOLVERS[solver],
                                                  ctypes.byref(h)))
        return cls(h)

    @classmethod
    def order_complex(cls, n, col_ptr, row_idx, ax) -> "Topology":
        """Symbolic phase of an AC sweep (NeoSolver::numeric_complex) on
        complex values ax (complex array of nnz, or 2*nnz interleaved)."""
        cp = np.ascontiguousarray(col_ptr, np.int32)
        ri = np.ascontiguousarray(row_idx, np.int32)
        v = _interleave(ax)
        h = ctypes.c_void_p()
        L.check(L.lib().nsg_topology_order_complex(int(n), len(ri), L.iptr(cp), L.iptr(ri),
                                                   L.dptr(v), ctypes.byref(h)))
        return cls(h)

    @property
    def solver(self) -> str:
        """Engine of the current plan: "markowitz" or "amdlu"."""
        k = L.lib().nsg_topology_solver(self._h)
        return "amdlu" if k == SOLVERS["amdlu"] else "markowitz"

    @classmethod
    def import_structure(cls, n, nnz, int_to_ext_row, int_to_ext_col, elem_row, elem_col,
                         slot_to_elem) -> "Topology":
        arrs = [np.ascontiguousarray(a, np.int32) for a in
                (int_to_ext_row, int_to_ext_col, elem_row, elem_col, slot_to_elem)]
        h = ctypes.c_void_p()
        L.check(L.lib().nsg_topology_import(int(n), int(nnz), L.iptr(arrs[0]), L.iptr(arrs[1]),
                                            len(arrs[2]), L.iptr(arrs[2]), L.iptr(arrs[3]),
                                            L.iptr(arrs[4]), ctypes.byref(h)))
        return cls(h)

    def numeric(self, values, diag_gmin=0.0) -> int:
        """Re-validate pivots on new values (NeoSolver::numeric); returns the
        first re-ordered step (1-based) or 0."""
        v = np.ascontiguousarray(values, np.float64)
        step = ctypes.c_int(0)
        L.check(L.lib().nsg_topology_numeric(self._h, L.dptr(v), float(diag_gmin),
                                             ctypes.byref(step)))
        return step.value

    def info(self) -> dict:
        n, nnz, nlu = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        upd = ctypes.c_longlong()
        cl, fl, bl = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        L.check(L.lib().nsg_topology_info(self._h, ctypes.byref(n), ctypes.byref(nnz),
                                          ctypes.byref(nlu), ctypes.byref(upd), ctypes.byref(cl),
                                          ctypes.byref(fl), ctypes.byref(bl)))
        return dict(n=n.value, nnz=nnz.value, nnz_lu=nlu.value, updates=upd.value,
                    col_levels=cl.value, fwd_levels=fl.value, bwd_levels=bl.value)

    def export(self):
        """(int_to_ext_row, int_to_ext_col, elem_row, elem_col, slot_to_elem),
        1-based, in the reference's export format."""
        i = self.info()
        r = np.zeros(i["n"], np.int32)
        c = np.zeros(i["n"], np.int32)
        er = np.zeros(i["nnz_lu"], np.int32)
        ec = np.zeros(i["nnz_lu"], np.int32)
        se = np.zeros(i["nnz"], np.int32)
        L.check(L.lib().nsg_topology_export(self._h, L.iptr(r), L.iptr(c), L.iptr(er),
                                            L.iptr(ec), L.iptr(se)))
        return r, c, er, ec, se

    def __del__(self):
        if getattr(self, "_h", None) and L._lib is not None:
            L._lib.nsg_topology_free(self._h)
            self._h = None


def _interleave(z) -> np.ndarray:
    """(re, im) pairs of a complex array (or an interleaved float array)."""
    z = np.asarray(z)
    if np.iscomplexobj(z):
        out = np.empty(2 * z.size)
        out[0::2] = z.real
        out[1::2] = z.imag
        return out
    return np.ascontiguousarray(z, np.float64)


def _stream_ptr(stream):
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    return getattr(stream, "cuda_stream", stream)


class Batch:
    """Device batch of instances, instance i factored with topologies[i]."""

    def __init__(self, topologies):
        self.topologies = list(topologies)
        arr = (ctypes.c_void_p * len(self.topologies))(*[t.handle for t in self.topologies])
        h = ctypes.c_void_p()
        L.check(L.lib().nsg_batch_create(len(self.topologies), arr, ctypes.byref(h)))
        self._h = h
        cnt = len(self.topologies) + 1
        self.value_offsets = np.zeros(cnt, np.int64)
        self.vector_offsets = np.zeros(cnt, np.int64)
        self.lu_offsets = np.zeros(cnt, np.int64)
        L.check(L.lib().nsg_batch_layout(self._h, L.llptr(self.value_offsets),
                                         L.llptr(self.vector_offsets), L.llptr(self.lu_offsets)))

    @property
    def count(self):
        return len(self.topologies)

    def set_schedule(self, schedule: int):
        """0 = dataflow refactor (default), 1 = level-synchronous."""
        L.check(L.lib().nsg_batch_set_schedule(self._h, int(schedule)))

    def set_grid_buffer(self, doubles: int):
        """Shared column buffer per warp of the grid-wide refactor (1024,
        2048, 4096; 0 = automatic)."""
        L.check(L.lib().nsg_batch_set_grid_buffer(self._h, int(doubles)))

    def set_grid_tail(self, columns: int):
        """Columns the grid-wide refactor hands to whole CTAs: the last
        `columns`, 0 for none, -1 (default) for the heavy top separators."""
        L.check(L.lib().nsg_batch_set_grid_tail(self._h, int(columns)))

    def refactor(self, d_values, diag_gmin=0.0, check_pivots=False, d_status=None,
                 d_fail_step=None, stream=None):
        """Batched spFactor; returns the device status tensor (int32)."""
        import torch
        if d_status is None:
            d_status = torch.empty(self.count, dtype=torch.int32, device=d_values.device)
        if d_fail_step is None:
            d_fail_step = torch.empty(self.count, dtype=torch.int32, device=d_values.device)
        L.check(L.lib().nsg_batch_refactor(self._h, d_values.data_ptr(), float(diag_gmin),
                                           int(bool(check_pivots)), d_status.data_ptr(),
                                           d_fail_step.data_ptr(), _stream_ptr(stream)))
        return d_status, d_fail_step

    def autotune(self, d_values, d_x, reps=3, stream=None):
        """Time the schedules on this system and keep the fastest:
        (chosen schedule, [ms per refactor+solve for schedules 0, 1, 2])."""
        t = (ctypes.c_float * 3)()
        c = ctypes.c_int(-1)
        L.check(L.lib().nsg_batch_autotune(self._h, d_values.data_ptr(), d_x.data_ptr(), int(reps),
                                           t, ctypes.byref(c), _stream_ptr(stream)))
        return c.value, [float(v) for v in t]

    def solve(self, d_x, stream=None):
        L.check(L.lib().nsg_batch_solve(self._h, d_x.data_ptr(), _stream_ptr(stream)))
        return d_x

    def solve_transposed(self, d_x, stream=None):
        L.check(L.lib().nsg_batch_solve_transposed(self._h, d_x.data_ptr(), _stream_ptr(stream)))
        return d_x

    # --- AC: complex values interleaved (re, im), twice the real offsets ---
    def refactor_complex(self, d_ax, d_lu=None, d_status=None, stream=None):
        """Batched factor_complex with the plans' pivots; returns (complex
        LU device tensor, 2 doubles per LU position; status per instance)."""
        import torch
        if d_lu is None:
            d_lu = torch.empty(2 * int(self.lu_offsets[-1]), dtype=torch.float64,
                               device=d_ax.device)
        if d_status is None:
            d_status = torch.empty(self.count, dtype=torch.int32, device=d_ax.device)
        L.check(L.lib().nsg_batch_refactor_complex(self._h, d_ax.data_ptr(), d_lu.data_ptr(),
                                                   d_status.data_ptr(), _stream_ptr(stream)))
        return d_lu, d_status

    def solve_complex(self, d_lu, d_x, stream=None):
        """Batched solve_complex in place on interleaved d_x."""
        L.check(L.lib().nsg_batch_solve_complex(self._h, d_lu.data_ptr(), d_x.data_ptr(),
                                                _stream_ptr(stream)))
        return d_x

    def lu_values(self):
        """Host copy of the factored LU values of every instance."""
        out = np.zeros(int(self.lu_offsets[-1]))
        L.check(L.lib().nsg_batch_lu_to_host(self._h, L.dptr(out)))
        return out

    def __del__(self):
        if getattr(self, "_h", None) and L._lib is not None:
            L._lib.nsg_batch_free(self._h)
            self._h = None
