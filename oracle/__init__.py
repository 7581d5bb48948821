"""The oracle: test infrastructure, never part of the product.

Two checkers, loaded with ctypes:

* ``port()``  — oracle/_ref/libnsoracle.so, the plain-C restatement of the
  reference's fixed-pivot refactor and solves (ns_oracle.c).
* ``ref()``   — oracle/_ref/libnsref.so, the reference's own C++ sources
  compiled by oracle/Makefile plus the export shim ref_shim.cpp.  Present only
  where the reference sources were available at build time.
* ``seam()``  — oracle/_ref/libnsseam.so, the same plus gpu_seam.cpp: the
  reference's analyses on libnsgpu through its ISolver seam.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use
this package.
"""
from __future__ import annotations

import ctypes
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
OUT = HERE / "_ref"
PORT_SO = OUT / "libnsoracle.so"
REF_SO = OUT / "libnsref.so"
REFERENCE_SRC = pathlib.Path("/root/reference")

_V = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double


def build(reference: bool = True) -> None:
    """Build the C port, and the reference library when its sources exist."""
    targets = ["port"]
    if reference and (REFERENCE_SRC / "src").is_dir():
        targets.append("ref")
        if (HERE.parent / "neospice_b200" / "libnsgpu.so").exists():
            targets.append("seam")
    subprocess.run(["make", "-s", f"-j{8}", *targets], cwd=HERE, check=True)


_port = None
_ref = None


def port() -> ctypes.CDLL:
    global _port
    if _port is None:
        if not PORT_SO.exists():
            build(reference=False)
        lib = ctypes.CDLL(str(PORT_SO))
        lib.nso_refactor.argtypes = [_I, _I, _I, _V, _V, _V, _V, _D, _I, _V, _V]
        lib.nso_solve.argtypes = [_I, _I, _V, _V, _V, _V, _V, _V]
        lib.nso_solve_transposed.argtypes = [_I, _I, _V, _V, _V, _V, _V, _V]
        lib.nso_amd_replay.argtypes = [_I, _V, _V, _V, _V, _V, _V, _V, _V, _V, _D, _V, _V, _V]
        lib.nso_amd_solve.argtypes = [_I] + [_V] * 9
        _port = lib
    return _port


def have_ref() -> bool:
    return REF_SO.exists()


def ref() -> ctypes.CDLL:
    global _ref
    if _ref is None:
        _ref = _bind(ctypes.CDLL(str(REF_SO)))
    return _ref


SEAM_SO = OUT / "libnsseam.so"
_seam = None


def have_seam() -> bool:
    return SEAM_SO.exists()


def seam() -> ctypes.CDLL:
    """oracle/_ref/libnsseam.so: the reference's sources with make_solver
    overridden by oracle/gpu_seam.cpp, so that its analyses can run on
    libnsgpu through the ISolver seam (nsseam_use_gpu).  Same entry points as
    ref()."""
    global _seam
    if _seam is None:
        lib = _bind(ctypes.CDLL(str(SEAM_SO)))
        lib.nsseam_use_gpu.argtypes = [_I]
        lib.nsseam_gpu_solvers.restype = ctypes.c_longlong
        lib.nsseam_ac_sweep.argtypes = [_I, _I, _V, _V, _V, _V, _V, _I, _V, _V, _V]
        lib.nsseam_solve_sequence.argtypes = [_I, _I, _V, _V, _V, _V, _I, _D, _I, _I, _V, _V]
        _seam = lib
    return _seam


def seam_solve_sequence(n, col_ptr, row_idx, values_seq, rhs, gpu: bool, equilibrate=True,
                        diag_gmin=0.0, is_linear=False):
    """numeric() then refactorize() on each value vector of values_seq, each
    followed by solve(rhs), through make_solver's ISolver: the reference's
    (gpu=False) or the GPU adapter (gpu=True).  Returns ((points, n)
    solutions, per-point singular flags)."""
    lib = seam()
    cp = np.ascontiguousarray(col_ptr, np.int32)
    ri = np.ascontiguousarray(row_idx, np.int32)
    vals = np.ascontiguousarray(values_seq, np.float64)
    b = np.ascontiguousarray(rhs, np.float64)
    pts = vals.shape[0]
    out = np.zeros((pts, n))
    sing = np.zeros(pts, np.int32)
    lib.nsseam_use_gpu(1 if gpu else 0)
    try:
        rc = lib.nsseam_solve_sequence(int(n), len(ri), _p(cp), _p(ri), _p(vals), _p(b), pts,
                                       float(diag_gmin), int(bool(equilibrate)),
                                       int(bool(is_linear)), _p(out), _p(sing))
    finally:
        lib.nsseam_use_gpu(0)
    if rc != 0:
        raise RuntimeError("nsseam_solve_sequence: the solver threw")
    return out, sing


def seam_ac_sweep(n, col_ptr, row_idx, g, c, rhs, omegas, gpu: bool):
    """An AC sweep (solve_ac's per-frequency steps) through the ISolver that
    make_solver returns: the reference's NeoSolver (gpu=False) or the GPU
    adapter (gpu=True).  rhs is complex (n,); returns (complex (points, n)
    solutions, per-point singular flags)."""
    lib = seam()
    cp = np.ascontiguousarray(col_ptr, np.int32)
    ri = np.ascontiguousarray(row_idx, np.int32)
    g = np.ascontiguousarray(g, np.float64)
    c = np.ascontiguousarray(c, np.float64)
    z = np.ascontiguousarray(_interleaved(np.asarray(rhs, np.complex128)))
    om = np.ascontiguousarray(omegas, np.float64)
    out = np.zeros((len(om), 2 * n))
    sing = np.zeros(len(om), np.int32)
    lib.nsseam_use_gpu(1 if gpu else 0)
    try:
        rc = lib.nsseam_ac_sweep(int(n), len(ri), _p(cp), _p(ri), _p(g), _p(c), _p(z), len(om),
                                 _p(om), _p(out), _p(sing))
    finally:
        lib.nsseam_use_gpu(0)
    if rc != 0:
        raise RuntimeError("nsseam_ac_sweep: the solver threw")
    return out[:, 0::2] + 1j * out[:, 1::2], sing


def _bind(lib: ctypes.CDLL) -> ctypes.CDLL:
    if True:
        lib.nsref_solver_create.restype = _V
        lib.nsref_solver_create.argtypes = [_I, _I, _V, _V]
        lib.nsref_solver_destroy.argtypes = [_V]
        lib.nsref_solver_numeric.argtypes = [_V, _V, _D]
        lib.nsref_solver_refactor.argtypes = [_V, _V, _D]
        lib.nsref_solver_solve.argtypes = [_V, _V]
        lib.nsref_solver_solve_transposed.argtypes = [_V, _V]
        lib.nsref_solver_element_count.argtypes = [_V]
        lib.nsref_solver_export.argtypes = [_V] * 7
        lib.nsref_mesh_dc.argtypes = [_I, _V, _V, _I, _V, _D, _D, _I, _V, _V, _D, _V, _V, _V]
        lib.nsref_sim_run.restype = _V
        lib.nsref_sim_run.argtypes = [ctypes.c_char_p, _I, _D, _D]
        lib.nsref_sim_info.argtypes = [_V, _V, _V, _V, _V, _V, _V]
        lib.nsref_sim_copy.argtypes = [_V, _V, _V]
        lib.nsref_sim_error.restype = ctypes.c_char_p
        lib.nsref_sim_error.argtypes = [_V]
        lib.nsref_sim_free.argtypes = [_V]
        lib.nsref_sim_initjct.argtypes = [ctypes.c_char_p, _V, _V, _V, _V, _V]
        lib.nsref_sim_eval_seq.argtypes = [ctypes.c_char_p, _I, _V, _V, _V, _V, _V, _V]
        lib.nsref_sim_method.argtypes = [_V]
        lib.nsref_sim_sens.argtypes = [ctypes.c_char_p, _I, _V, _V]
        lib.nsref_step_dc.argtypes = [ctypes.c_char_p, _I, _D, _D, _D, _I, _V, _V, _V]
        lib.nsref_step_tran.argtypes = [ctypes.c_char_p, _I, _D, _D, _D, _D, _D, _I, _I, _V, _V,
                                        _V, _V]
        lib.nsref_mesh_initjct.argtypes = [_I, _V, _V, _I, _V, _D, _D, _I, _V, _V, _D, _V, _V,
                                           _V, _V, _V]
        lib.nsref_amd_order.argtypes = [_I, _V, _V, _V]
        lib.nsref_amdlu_create.restype = _V
        lib.nsref_amdlu_create.argtypes = [_I, _I, _V, _V]
        lib.nsref_amdlu_destroy.argtypes = [_V]
        lib.nsref_amdlu_numeric.argtypes = [_V, _V, _D]
        lib.nsref_amdlu_refactor.argtypes = [_V, _V, _D]
        lib.nsref_amdlu_counts.argtypes = [_V, _V, _V]
        lib.nsref_amdlu_solve.argtypes = [_V, _V]
        lib.nsref_amdlu_sizes.argtypes = [_V, _V, _V]
        lib.nsref_amdlu_export.argtypes = [_V] * 9
        lib.nsref_make_solver_name.argtypes = [_I, _I, ctypes.c_char_p, _I]
        lib.nsref_solver_numeric_complex.argtypes = [_V, _V]
        lib.nsref_solver_refactor_complex.argtypes = [_V, _V]
        lib.nsref_solver_solve_complex.argtypes = [_V, _V]
        lib.nsref_solver_export_imag.argtypes = [_V, _V]
    return lib


def _p(a):
    return a.ctypes.data


class Structure:
    """A factored topology in the reference's export format (1-based)."""

    def __init__(self, n, int_to_ext_row, int_to_ext_col, elem_row, elem_col, slot_to_elem):
        self.n = int(n)
        self.int_to_ext_row = np.ascontiguousarray(int_to_ext_row, np.int32)
        self.int_to_ext_col = np.ascontiguousarray(int_to_ext_col, np.int32)
        self.elem_row = np.ascontiguousarray(elem_row, np.int32)
        self.elem_col = np.ascontiguousarray(elem_col, np.int32)
        self.slot_to_elem = np.ascontiguousarray(slot_to_elem, np.int32)

    @property
    def n_elem(self):
        return len(self.elem_row)

    def same_as(self, other) -> bool:
        return all(np.array_equal(getattr(self, k), getattr(other, k)) for k in
                   ("int_to_ext_row", "int_to_ext_col", "elem_row", "elem_col", "slot_to_elem"))


# --- the C port ------------------------------------------------------------

def port_refactor(st: Structure, a, gmin=0.0, check_pivots=False):
    a = np.ascontiguousarray(a, np.float64)
    lu = np.zeros(st.n_elem)
    step = ctypes.c_int(-1)
    rc = port().nso_refactor(st.n, len(st.slot_to_elem), st.n_elem, _p(st.elem_row),
                             _p(st.elem_col), _p(st.slot_to_elem), _p(a), gmin,
                             int(check_pivots), _p(lu), ctypes.addressof(step))
    return rc, lu, step.value


def port_solve(st: Structure, lu, b, transposed=False):
    x = np.array(b, np.float64, copy=True)
    fn = port().nso_solve_transposed if transposed else port().nso_solve
    rc = fn(st.n, st.n_elem, _p(st.elem_row), _p(st.elem_col), _p(st.int_to_ext_row),
            _p(st.int_to_ext_col), _p(np.ascontiguousarray(lu, np.float64)), _p(x))
    if rc != 0:
        raise RuntimeError(f"oracle solve failed: {rc}")
    return x


def port_amd_replay(f: dict, col_ptr, row_idx, a, gmin=0.0):
    """The C port of AmdLuSolver::refactor_replay_ on the factor structure f
    (RefAmdLu.export format): (rc, Lx, Ux, fail_step)."""
    cp = np.ascontiguousarray(col_ptr, np.int32)
    ri = np.ascontiguousarray(row_idx, np.int32)
    a = np.ascontiguousarray(a, np.float64)
    lx = np.array(f["Lx"], np.float64, copy=True)
    ux = np.array(f["Ux"], np.float64, copy=True)
    step = ctypes.c_int(-1)
    n = len(f["q"])
    rc = port().nso_amd_replay(n, _p(cp), _p(ri), *(_p(np.ascontiguousarray(f[k], np.int32))
                                                    for k in ("q", "pinv", "Lp", "Li", "Up", "Ui")),
                               _p(a), float(gmin), _p(lx), _p(ux), ctypes.addressof(step))
    return rc, lx, ux, step.value


def port_amd_solve(f: dict, lx, ux, b):
    """The C port of AmdLuSolver::solve."""
    x = np.array(b, np.float64, copy=True)
    ints = {k: np.ascontiguousarray(f[k], np.int32) for k in ("q", "pinv", "Lp", "Li", "Up", "Ui")}
    lx = np.ascontiguousarray(lx, np.float64)
    ux = np.ascontiguousarray(ux, np.float64)
    port().nso_amd_solve(len(ints["q"]), _p(ints["q"]), _p(ints["pinv"]), _p(ints["Lp"]),
                         _p(ints["Li"]), _p(lx), _p(ints["Up"]), _p(ints["Ui"]), _p(ux), _p(x))
    return x


# --- the reference itself ----------------------------------------------------

def _interleaved(z) -> np.ndarray:
    """(re, im) pairs of a complex array; an already interleaved float
    array passes through."""
    z = np.asarray(z)
    if np.iscomplexobj(z):
        out = np.empty(2 * z.size)
        out[0::2] = z.real
        out[1::2] = z.imag
        return out
    return np.ascontiguousarray(z, np.float64)


class RefSolver:
    """The reference's NeoSolver on a CSC pattern, through the export shim."""

    def __init__(self, n, col_ptr, row_idx):
        self.n = int(n)
        self.col_ptr = np.ascontiguousarray(col_ptr, np.int32)
        self.row_idx = np.ascontiguousarray(row_idx, np.int32)
        self.h = ref().nsref_solver_create(self.n, len(self.row_idx), _p(self.col_ptr),
                                           _p(self.row_idx))

    def __del__(self):
        if getattr(self, "h", None) and _ref is not None:
            _ref.nsref_solver_destroy(self.h)
            self.h = None

    def numeric(self, values, gmin=0.0) -> int:
        v = np.ascontiguousarray(values, np.float64)
        return ref().nsref_solver_numeric(self.h, _p(v), gmin)

    def refactorize(self, values, gmin=0.0) -> int:
        v = np.ascontiguousarray(values, np.float64)
        return ref().nsref_solver_refactor(self.h, _p(v), gmin)

    def solve(self, b, transposed=False):
        x = np.array(b, np.float64, copy=True)
        fn = ref().nsref_solver_solve_transposed if transposed else ref().nsref_solver_solve
        if fn(self.h, _p(x)) != 0:
            raise RuntimeError("reference solve failed")
        return x

    # --- complex (AC) path: values interleaved (re, im) per slot ---
    def numeric_complex(self, ax) -> int:
        v = _interleaved(ax)
        return ref().nsref_solver_numeric_complex(self.h, _p(v))

    def refactorize_complex(self, ax) -> int:
        v = _interleaved(ax)
        return ref().nsref_solver_refactor_complex(self.h, _p(v))

    def solve_complex(self, b):
        """Complex solve of b (complex array of n); returns a complex array."""
        x = _interleaved(b).copy()
        if ref().nsref_solver_solve_complex(self.h, _p(x)) != 0:
            raise RuntimeError("reference complex solve failed")
        return x[0::2] + 1j * x[1::2]

    def export_complex(self):
        """(Structure, complex element values) after a complex factor."""
        st, re = self.export()
        im = np.zeros(len(re))
        ref().nsref_solver_export_imag(self.h, _p(im))
        return st, re + 1j * im

    def export(self):
        ne = ref().nsref_solver_element_count(self.h)
        n = self.n
        r = np.zeros(n, np.int32)
        c = np.zeros(n, np.int32)
        er = np.zeros(ne, np.int32)
        ec = np.zeros(ne, np.int32)
        ev = np.zeros(ne)
        se = np.zeros(len(self.row_idx), np.int32)
        ref().nsref_solver_export(self.h, _p(r), _p(c), _p(er), _p(ec), _p(ev), _p(se))
        return Structure(n, r, c, er, ec, se), ev


def ref_amd_order(n, col_ptr, row_idx):
    """The reference's amd_ordering (src/core/amd.cpp:14-143)."""
    cp = np.ascontiguousarray(col_ptr, np.int32)
    ri = np.ascontiguousarray(row_idx, np.int32)
    perm = np.zeros(int(n), np.int32)
    ref().nsref_amd_order(int(n), _p(cp), _p(ri), _p(perm))
    return perm


def ref_make_solver_name(num_vars, is_linear) -> str:
    """make_solver(num_vars, is_linear)->name() under the current environment."""
    buf = ctypes.create_string_buffer(64)
    ref().nsref_make_solver_name(int(num_vars), int(bool(is_linear)), buf, 64)
    return buf.value.decode()


class RefAmdLu:
    """The reference's AmdLuSolver on a CSC pattern, through the export shim."""

    def __init__(self, n, col_ptr, row_idx):
        self.n = int(n)
        self.col_ptr = np.ascontiguousarray(col_ptr, np.int32)
        self.row_idx = np.ascontiguousarray(row_idx, np.int32)
        self.h = ref().nsref_amdlu_create(self.n, len(self.row_idx), _p(self.col_ptr),
                                          _p(self.row_idx))

    def __del__(self):
        if getattr(self, "h", None) and _ref is not None:
            _ref.nsref_amdlu_destroy(self.h)
            self.h = None

    def numeric(self, values, gmin=0.0) -> int:
        v = np.ascontiguousarray(values, np.float64)
        return ref().nsref_amdlu_numeric(self.h, _p(v), gmin)

    def refactorize(self, values, gmin=0.0) -> int:
        v = np.ascontiguousarray(values, np.float64)
        return ref().nsref_amdlu_refactor(self.h, _p(v), gmin)

    def counts(self):
        fast, fb = ctypes.c_int(0), ctypes.c_int(0)
        ref().nsref_amdlu_counts(self.h, ctypes.addressof(fast), ctypes.addressof(fb))
        return fast.value, fb.value

    def solve(self, b):
        x = np.array(b, np.float64, copy=True)
        if ref().nsref_amdlu_solve(self.h, _p(x)) != 0:
            raise RuntimeError("reference solve failed")
        return x

    def export(self) -> dict:
        nl, nu = ctypes.c_int(0), ctypes.c_int(0)
        ref().nsref_amdlu_sizes(self.h, ctypes.addressof(nl), ctypes.addressof(nu))
        n = self.n
        f = dict(q=np.zeros(n, np.int32), pinv=np.zeros(n, np.int32),
                 Lp=np.zeros(n + 1, np.int32), Li=np.zeros(nl.value, np.int32),
                 Lx=np.zeros(nl.value), Up=np.zeros(n + 1, np.int32),
                 Ui=np.zeros(nu.value, np.int32), Ux=np.zeros(nu.value))
        ref().nsref_amdlu_export(self.h, *(_p(f[k]) for k in
                                           ("q", "pinv", "Lp", "Li", "Lx", "Up", "Ui", "Ux")))
        return f


# --- the reference on diode meshes (neospice_b200.workloads.DiodeMesh) -------

def _mesh_args(m):
    arrs = dict(r_h=np.ascontiguousarray(m.r_h, np.float64),
                r_v=np.ascontiguousarray(m.r_v, np.float64),
                dn=np.ascontiguousarray(m.diode_nodes, np.int32),
                isn=np.ascontiguousarray(m.isrc_nodes, np.int32),
                ia=np.ascontiguousarray(m.isrc_amps, np.float64))
    args = (m.side, _p(arrs["r_h"]), _p(arrs["r_v"]), len(arrs["dn"]), _p(arrs["dn"]),
            float(m.diode_is), float(m.diode_n), len(arrs["isn"]), _p(arrs["isn"]),
            _p(arrs["ia"]), float(m.v_corner))
    return args, arrs


def ref_mesh_dc(m, lib=None):
    """The reference's DC operating point of a diode mesh: (solution,
    Newton iterations, seconds)."""
    args, keep = _mesh_args(m)
    sol = np.zeros(m.num_vars)
    it = ctypes.c_int(0)
    sec = ctypes.c_double(0.0)
    nv = (lib if lib is not None else ref()).nsref_mesh_dc(*args, _p(sol), ctypes.addressof(it), ctypes.addressof(sec))
    if nv != m.num_vars:
        raise RuntimeError(f"reference DC failed ({nv})")
    return sol, it.value, sec.value


def ref_mesh_initjct(m):
    """The reference's first-iteration matrix: (col_ptr, row_idx, values, rhs)."""
    args, keep = _mesh_args(m)
    nv = ctypes.c_int(0)
    nnz = ref().nsref_mesh_initjct(*args, ctypes.addressof(nv), None, None, None, None)
    cp = np.zeros(nv.value + 1, np.int32)
    ri = np.zeros(nnz, np.int32)
    vals = np.zeros(nnz)
    rhs = np.zeros(nv.value)
    rc = ref().nsref_mesh_initjct(*args, ctypes.addressof(nv), _p(cp), _p(ri), _p(vals), _p(rhs))
    if rc != nnz:
        raise RuntimeError("reference INITJCT evaluation failed")
    return cp, ri, vals, rhs


def ref_sim_initjct(desc: str):
    """The reference's first DC Newton matrix of a described circuit:
    (col_ptr, row_idx, values, rhs)."""
    lib = ref()
    nv = ctypes.c_int(0)
    d = desc.encode()
    nnz = lib.nsref_sim_initjct(d, ctypes.addressof(nv), None, None, None, None)
    if nnz < 0:
        raise RuntimeError("reference INITJCT evaluation failed")
    cp = np.zeros(nv.value + 1, np.int32)
    ri = np.zeros(nnz, np.int32)
    vals = np.zeros(nnz)
    rhs = np.zeros(nv.value)
    if lib.nsref_sim_initjct(d, ctypes.addressof(nv), _p(cp), _p(ri), _p(vals), _p(rhs)) != nnz:
        raise RuntimeError("reference INITJCT evaluation failed")
    return cp, ri, vals, rhs


def ref_sim_eval_seq(desc: str, state_ops, modes, xs, ctx):
    """A sequence of the reference's device evaluations (nsref_sim_eval_seq):
    xs (steps, n) guesses, ctx (steps, 8) integrator fields; returns the
    matrices (steps, nnz) in slot order and the rhs (steps, n)."""
    lib = ref()
    xs = np.ascontiguousarray(xs, np.float64)
    steps, n = xs.shape
    ops = np.ascontiguousarray(state_ops, np.int32)
    md = np.ascontiguousarray(modes, np.int32)
    c = np.ascontiguousarray(ctx, np.float64)
    nv = ctypes.c_int(0)
    nnz = lib.nsref_sim_initjct(desc.encode(), ctypes.addressof(nv), None, None, None, None)
    vals = np.zeros((steps, max(nnz, 0)))
    rhs = np.zeros((steps, n))
    if nnz < 0 or nv.value != n or lib.nsref_sim_eval_seq(
            desc.encode(), steps, _p(ops), _p(md), _p(xs), _p(c), _p(vals), _p(rhs)) != nnz:
        raise RuntimeError("reference evaluation sequence failed")
    return vals, rhs


def ref_step_dc(desc: str, device_line: int, start: float, stop: float, step: float,
                num_nodes: int):
    """The reference's `.op` under `.step <source> start stop step`
    (Simulator::run_step_sweep): the source is line `device_line` of the
    description.  Returns (step values, node voltages [steps x num_nodes],
    Newton iterations per step)."""
    lib = ref()
    d = desc.encode()
    cap = 1 << 12
    vals = np.zeros(cap)
    volts = np.zeros(cap * num_nodes)
    iters = np.zeros(cap, np.int32)
    k = lib.nsref_step_dc(d, int(device_line), float(start), float(stop), float(step), cap,
                          _p(vals), _p(volts), _p(iters))
    if k < 0 or k > cap:
        raise RuntimeError("reference .step run failed")
    return vals[:k].copy(), volts[:k * num_nodes].reshape(k, num_nodes).copy(), iters[:k].copy()


def ref_step_tran(desc: str, device_line: int, start: float, stop: float, step: float,
                  tstep: float, tstop: float, num_nodes: int, cap_points: int = 1 << 18):
    """The reference's `.tran tstep tstop` under `.step <source> start stop
    step`.  Returns a list over steps of (times, node voltages [points x
    num_nodes]) and the Newton iterations per step."""
    lib = ref()
    d = desc.encode()
    cap_steps = 1 << 10
    counts = np.zeros(cap_steps, np.int32)
    iters = np.zeros(cap_steps, np.int32)
    times = np.zeros(cap_points)
    volts = np.zeros(cap_points * num_nodes)
    k = lib.nsref_step_tran(d, int(device_line), float(start), float(stop), float(step),
                            float(tstep), float(tstop), cap_steps, cap_points, _p(counts),
                            _p(times), _p(volts), _p(iters))
    if k < 0 or k > cap_steps or int(counts[:k].sum()) > cap_points:
        raise RuntimeError("reference .step transient failed")
    out, at = [], 0
    for c in counts[:k]:
        out.append((times[at:at + c].copy(), volts[at * num_nodes:(at + c) * num_nodes]
                    .reshape(c, num_nodes).copy()))
        at += c
    return out, iters[:k].copy()


def ref_sim_sens(desc: str, output_node: int):
    """The reference's solve_sens of v(output node): (sensitivities in the
    reference's order -- resistors, voltage sources, current sources, each in
    creation order --, output value)."""
    lib = ref()
    d = desc.encode()
    k = lib.nsref_sim_sens(d, int(output_node), None, None)
    if k < 0:
        raise RuntimeError("reference sensitivity analysis failed")
    out = np.zeros(max(k, 1))
    val = ctypes.c_double()
    lib.nsref_sim_sens(d, int(output_node), _p(out), ctypes.addressof(val))
    return out[:k], val.value


def ref_sim(desc: str, analysis: int = 1, tstep: float = 0.0, tstop: float = 0.0, lib=None):
    """Run a circuit description (see nsref_sim_run in ref_shim.cpp) through
    the reference: analysis 0 = DC operating point, 1 = transient, 2 / 3 / 4
    = the reference's source_stepping / gain_stepping / pseudo_transient
    alone (info["method"] 2, 2, 3 when it converged, -1 when not).  Returns (times, values [npoints x
    width], info dict)."""
    lib = lib if lib is not None else ref()
    h = lib.nsref_sim_run(desc.encode(), int(analysis), float(tstep), float(tstop))
    try:
        nn, nv, npts, it, rej = (ctypes.c_int() for _ in range(5))
        sec = ctypes.c_double()
        rc = lib.nsref_sim_info(h, ctypes.addressof(nn), ctypes.addressof(nv), ctypes.addressof(npts),
                                ctypes.addressof(it), ctypes.addressof(sec), ctypes.addressof(rej))
        if rc != 0:
            raise RuntimeError("reference failed: " + lib.nsref_sim_error(h).decode())
        width = nv.value if analysis in (0, 2, 3, 4) else nn.value
        times = np.zeros(npts.value)
        values = np.zeros((npts.value, width))
        lib.nsref_sim_copy(h, _p(times), _p(values))
        info = dict(num_nodes=nn.value, num_vars=nv.value, points=npts.value,
                    iterations=it.value, seconds=sec.value, rejected=rej.value,
                    method=lib.nsref_sim_method(h))
        return times, values, info
    finally:
        lib.nsref_sim_free(h)
