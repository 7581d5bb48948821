"""ctypes binding of libnsgpu.so (the C ABI in include/nsgpu.h).

The library is loaded from the package directory.  There is no fallback: if
it is missing, importing the solver raises, so a GPU run can never silently
fall back to a CPU path.
"""
from __future__ import annotations

import ctypes
import pathlib

_HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = _HERE / "libnsgpu.so"

c_int = ctypes.c_int
c_ll = ctypes.c_longlong
c_double = ctypes.c_double
c_void_p = ctypes.c_void_p
P = ctypes.POINTER

NSG_OK = 0
NSG_ERR_INVALID = 1
NSG_ERR_CUDA = 2
NSG_ERR_NOMEM = 8
NSG_SINGULAR = 102
NSG_REORDER = 103
NSG_TIMEOUT = 104
NSG_SYMBOLIC_PER_INSTANCE = 0
NSG_SYMBOLIC_PER_PATTERN = 1
NSG_WAVE_DC = 0
NSG_WAVE_PULSE = 1
NSG_WAVE_PWL = 2
NSG_STATIC_SCRATCH_DOUBLES = 1 << 20
NSG_DEFAULT_WAIT_LIMIT = 1 << 22

# name -> (restype, argtypes)
SIGNATURES = {
    "nsg_last_error": (ctypes.c_char_p, []),
    "nsg_set_wait_limit": (c_int, [c_int]),
    "nsg_topology_order": (c_int, [c_int, c_int, P(c_int), P(c_int), P(c_double), c_double,
                                   P(c_void_p)]),
    "nsg_topology_numeric": (c_int, [c_void_p, P(c_double), c_double, P(c_int)]),
    "nsg_topology_order_solver": (c_int, [c_int, c_int, P(c_int), P(c_int), P(c_double),
                                          c_double, c_int, P(c_void_p)]),
    "nsg_solver_select": (c_int, [c_int, c_int]),
    "nsg_topology_solver": (c_int, [c_void_p]),
    "nsg_amd_order": (c_int, [c_int, P(c_int), P(c_int), P(c_int)]),
    "nsg_dc_batch_engines": (c_int, [c_void_p, P(c_int)]),
    "nsg_dc_batch_set_graph": (c_int, [c_void_p, c_int]),
    "nsg_dc_batch_set_row_maps": (c_int, [c_void_p, c_int]),
    "nsg_dc_batch_graph_launches": (c_int, [c_void_p, P(c_ll)]),
    "nsg_batch_autotune": (c_int, [c_void_p, c_void_p, c_void_p, c_int, P(ctypes.c_float),
                                   P(c_int), c_void_p]),
    "nsg_tran_batch_engines": (c_int, [c_void_p, P(c_int), P(c_int)]),
    "nsg_topology_import": (c_int, [c_int, c_int, P(c_int), P(c_int), c_int, P(c_int), P(c_int),
                                    P(c_int), P(c_void_p)]),
    "nsg_topology_info": (c_int, [c_void_p, P(c_int), P(c_int), P(c_int), P(c_ll), P(c_int),
                                  P(c_int), P(c_int)]),
    "nsg_topology_export": (c_int, [c_void_p, P(c_int), P(c_int), P(c_int), P(c_int), P(c_int)]),
    "nsg_topology_free": (None, [c_void_p]),
    "nsg_topology_order_complex": (c_int, [c_int, c_int, P(c_int), P(c_int), P(c_double),
                                           P(c_void_p)]),
    "nsg_batch_refactor_complex": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "nsg_batch_solve_complex": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "nsg_batch_create": (c_int, [c_int, P(c_void_p), P(c_void_p)]),
    "nsg_batch_free": (None, [c_void_p]),
    "nsg_batch_layout": (c_int, [c_void_p, P(c_ll), P(c_ll), P(c_ll)]),
    "nsg_batch_refactor": (c_int, [c_void_p, c_void_p, c_double, c_int, c_void_p, c_void_p,
                                   c_void_p]),
    "nsg_batch_set_schedule": (c_int, [c_void_p, c_int]),
    "nsg_batch_set_grid_buffer": (c_int, [c_void_p, c_int]),
    "nsg_batch_set_grid_tail": (c_int, [c_void_p, c_int]),
    "nsg_set_update_map_limit": (c_int, [c_ll]),
    "nsg_batch_solve": (c_int, [c_void_p, c_void_p, c_void_p]),
    "nsg_batch_solve_transposed": (c_int, [c_void_p, c_void_p, c_void_p]),
    "nsg_batch_solve_static_scratch": (c_int, [c_void_p, c_void_p, c_void_p]),
    "nsg_batch_lu": (c_void_p, [c_void_p]),
    "nsg_batch_lu_to_host": (c_int, [c_void_p, P(c_double)]),
    "nsg_circuit_create": (c_int, [c_int, P(c_void_p)]),
    "nsg_circuit_free": (None, [c_void_p]),
    "nsg_circuit_add_resistor": (c_int, [c_void_p, c_int, c_int, c_double]),
    "nsg_circuit_add_vsource": (c_int, [c_void_p, c_int, c_int, c_double]),
    "nsg_circuit_add_isource": (c_int, [c_void_p, c_int, c_int, c_double]),
    "nsg_circuit_add_diode": (c_int, [c_void_p, c_int, c_int, c_double, c_double]),
    "nsg_circuit_set_temperature": (c_int, [c_void_p, c_double]),
    "nsg_circuit_add_diode_card": (c_int, [c_void_p, c_int, c_int, c_double, c_double, c_double,
                                           c_double, c_double, c_double, c_double]),
    "nsg_diode_param_block": (c_int, [c_double, c_double, c_double, c_double, c_double, c_double,
                                      c_double, c_double, c_double, c_double, c_double,
                                      P(c_double)]),
    "nsg_circuit_add_diode_card_ex": (c_int, [c_void_p, c_int, c_int, c_double, c_double,
                                              c_double, c_double, c_double, c_double, c_double,
                                              c_double, c_double, c_double, c_double]),
    "nsg_circuit_add_resistors": (c_int, [c_void_p, c_int, P(c_int), P(c_int), P(c_double)]),
    "nsg_circuit_add_isources": (c_int, [c_void_p, c_int, P(c_int), P(c_int), P(c_double)]),
    "nsg_circuit_add_diodes": (c_int, [c_void_p, c_int, P(c_int), P(c_int), P(c_double),
                                       P(c_double)]),
    "nsg_circuit_finalize": (c_int, [c_void_p]),
    "nsg_circuit_info": (c_int, [c_void_p, P(c_int), P(c_int), P(c_int), P(c_int)]),
    "nsg_circuit_pattern": (c_int, [c_void_p, P(c_int), P(c_int)]),
    "nsg_circuit_params": (c_int, [c_void_p, P(c_double)]),
    "nsg_circuit_set_param": (c_int, [c_void_p, c_int, c_double]),
    "nsg_circuit_param_count": (c_int, [c_void_p, P(c_int)]),
    "nsg_step_values": (c_int, [c_double, c_double, c_double, c_int, P(c_double), P(c_int)]),
    "nsg_circuit_initial_matrix": (c_int, [c_void_p, c_double, P(c_double), P(c_double)]),
    "nsg_circuit_eval_matrix": (c_int, [c_void_p, c_int, P(c_double), P(c_double), c_int, c_int,
                                        c_double, c_double, c_double, P(c_double), P(c_double),
                                        P(c_double), P(c_double)]),
    "nsg_circuit_state_count": (c_int, [c_void_p]),
    "nsg_dc_batch_create": (c_int, [c_int, P(c_void_p), c_int, c_int, P(c_void_p)]),
    "nsg_dc_batch_free": (None, [c_void_p]),
    "nsg_dc_batch_layout": (c_int, [c_void_p, P(c_ll), P(c_ll)]),
    "nsg_dc_batch_stats": (c_int, [c_void_p, P(c_ll), P(c_ll), P(c_ll), P(c_ll), P(c_int)]),
    "nsg_dc_batch_instance_stats": (c_int, [c_void_p, P(c_ll), P(c_ll), P(c_ll), P(c_ll)]),
    "nsg_dc_batch_set_options": (c_int, [c_void_p, c_double, c_double, c_double, c_double, c_int]),
    "nsg_dc_batch_run": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "nsg_circuit_add_capacitor": (c_int, [c_void_p, c_int, c_int, c_double, c_int, c_double]),
    "nsg_circuit_add_source_wave": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_int,
                                            P(c_double)]),
    "nsg_circuit_add_capacitors": (c_int, [c_void_p, c_int, P(c_int), P(c_int), P(c_double)]),
    "nsg_circuit_add_bsim4_model": (c_int, [c_void_p, c_int, c_int, P(ctypes.c_char_p), P(c_double),
                                             P(c_int)]),
    "nsg_circuit_add_bsim4": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_int, c_double,
                                      c_double, c_double]),
    "nsg_circuit_add_mos1_model": (c_int, [c_void_p, c_int, c_int, P(ctypes.c_char_p), P(c_double),
                                           P(c_int)]),
    "nsg_circuit_add_mosfet": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_int, c_double,
                                       c_double]),
    "nsg_dc_batch_set_reorder": (c_int, [c_void_p, c_int]),
    "nsg_dc_batch_set_first_aid": (c_int, [c_void_p, c_int]),
    "nsg_dc_batch_reorders": (c_int, [c_void_p, P(c_ll)]),
    "nsg_dc_batch_methods": (c_int, [c_void_p, P(c_int), P(c_int)]),
    "nsg_dc_batch_adjoint": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                     c_void_p]),
    "nsg_tran_batch_create": (c_int, [c_int, P(c_void_p), c_double, c_double, c_int, c_int,
                                      P(c_int), c_int, P(c_void_p)]),
    "nsg_tran_batch_free": (None, [c_void_p]),
    "nsg_tran_batch_orderings": (c_int, [c_void_p, P(c_ll)]),
    "nsg_tran_batch_run": (c_int, [c_void_p, c_void_p]),
    "nsg_tran_batch_set_shape": (c_int, [c_void_p, c_int, c_int]),
    "nsg_tran_batch_record": (c_int, [c_void_p, c_int]),
    "nsg_tran_batch_set_adjoint_options": (c_int, [c_void_p, c_double, c_double, c_double, c_int]),
    "nsg_tran_batch_params": (c_int, [c_void_p, P(c_ll), P(c_double), P(c_double)]),
    "nsg_tran_batch_adjoint": (c_int, [c_void_p, P(c_int), c_void_p, c_double, c_int, c_void_p,
                                       c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "nsg_tran_batch_results": (c_int, [c_void_p, P(c_double), P(c_double), P(c_int), P(c_int),
                                       P(c_int)]),
}

_lib = None


def lib() -> ctypes.CDLL:
    """Load libnsgpu.so once; raise if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m neospice_b200.build`")
        handle = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


class NsgError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def check(code: int) -> int:
    if code != NSG_OK:
        raise NsgError(code, lib().nsg_last_error().decode())
    return code


def iptr(a):
    return a.ctypes.data_as(P(c_int))


def dptr(a):
    return a.ctypes.data_as(P(c_double))


def llptr(a):
    return a.ctypes.data_as(P(c_ll))
