"""Batched `.step` sweeps: every value of a stepped parameter solved as one
instance of a single GPU batch, instead of the reference's serial loop of
full re-runs (Simulator::run_step_sweep, src/api/neospice.cpp:228-331).

`.step` of a source (StepCommand::SOURCE) or of any device value: the
parameter is named by its index in Circuit.params() (creation order; see
Circuit.params).  Each step is an independent operating point, as the
reference's loop makes it by clearing the state vectors between steps
(Circuit::reset_state, src/core/circuit.cpp:305-314)."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib as L
from .circuit import Circuit, DcBatch, TranBatch


def step_values(start: float, stop: float, step: float) -> np.ndarray:
    """The values the reference's `.step start stop step` loop visits:
    start, start + step, ... (accumulated) while within stop plus a
    thousandth of |step|."""
    count = ctypes.c_int()
    L.check(L.lib().nsg_step_values(float(start), float(stop), float(step), 0, None,
                                    ctypes.byref(count)))  # the count only
    out = np.zeros(max(count.value, 1), np.float64)
    L.check(L.lib().nsg_step_values(float(start), float(stop), float(step), len(out),
                                    L.dptr(out), ctypes.byref(count)))
    return out[:count.value]


def sweep_dc(circuit: Circuit, param: int, values, symbolic=DcBatch.PER_PATTERN, batch=None):
    """Operating points of `circuit` with parameter `param` set to each of
    `values`, all in one batched launch.  Returns (solutions [len(values), n]
    as a numpy array, status, iterations) per step; `batch` may be a DcBatch
    of len(values) copies of this circuit made by an earlier call, to reuse
    its symbolic phase."""
    import torch

    values = np.asarray(values, np.float64).ravel()
    base = circuit.params()
    if not 0 <= param < len(base):
        raise IndexError(f"parameter {param} out of range (circuit has {len(base)})")
    if batch is None:
        batch = DcBatch([circuit] * len(values), symbolic=symbolic)
    if batch.count != len(values):
        raise ValueError("batch size does not match the number of step values")
    off = batch.param_offsets
    params = np.zeros(int(off[-1]), np.float64)
    for i, v in enumerate(values):
        params[off[i]:off[i + 1]] = base
        params[off[i] + param] = v
    d_params = torch.from_numpy(params).cuda()
    sols, status, iters = batch.run(d_params)
    torch.cuda.synchronize()
    return (np.stack(batch.split(sols)), status.cpu().numpy(), iters.cpu().numpy())


def sweep_transient(build, param: int, values, tstep: float, tstop: float, probes,
                    max_points: int = 100000):
    """Transients of one circuit with parameter `param` set to each of
    `values`, all instances of one TranBatch: `build()` returns a fresh
    finalized Circuit (one per step).  Returns the batch's results() list
    (per step: time, values at the probes, status, counts)."""
    values = np.asarray(values, np.float64).ravel()
    circuits = []
    for v in values:
        c = build()
        c.set_param(param, v)
        circuits.append(c)
    b = TranBatch(circuits, tstep, tstop, np.asarray(probes, np.int32), max_points=max_points)
    b.run()
    return b.results()


def sweep_dc_temperature(build, temps_celsius, symbolic=DcBatch.PER_INSTANCE):
    """`.step TEMP` of an operating point: the reference sets the circuit
    temperature to each step value + 273.15 K and re-runs the analysis
    (src/api/neospice.cpp:255-256), so every step is one instance built by
    `build(kelvin)` (a finalized Circuit with its devices at that
    temperature) of one batched launch.  Returns (solutions
    [len(temps), n], status, iterations) per step."""
    import torch

    temps = np.asarray(temps_celsius, np.float64).ravel()
    batch = DcBatch([build(t + 273.15) for t in temps], symbolic=symbolic)
    sols, status, iters = batch.run()
    torch.cuda.synchronize()
    return (np.stack(batch.split(sols)), status.cpu().numpy(), iters.cpu().numpy())


def sweep_transient_temperature(build, temps_celsius, tstep: float, tstop: float, probes,
                                max_points: int = 100000):
    """`.step TEMP` of a transient: one TranBatch instance per step value,
    built by `build(kelvin)`.  Returns the batch's results() list."""
    temps = np.asarray(temps_celsius, np.float64).ravel()
    b = TranBatch([build(t + 273.15) for t in temps], tstep, tstop,
                  np.asarray(probes, np.int32), max_points=max_points)
    b.run()
    return b.results()


def sweep_dc_multi(circuit: Circuit, params, values, symbolic=DcBatch.PER_PATTERN):
    """`.step PARAM` of an operating point: a `.param` may enter several
    device values, and the reference re-parses the netlist per step value
    (src/api/neospice.cpp:258-290); here the caller gives, per step, the
    values those devices take (`values` [steps x len(params)] for the
    parameter indices `params` of Circuit.params()), and every step is one
    instance of one batched launch.  Returns (solutions [steps, n], status,
    iterations)."""
    import torch

    params = [int(p) for p in params]
    values = np.asarray(values, np.float64).reshape(-1, len(params))
    base = circuit.params()
    for p in params:
        if not 0 <= p < len(base):
            raise IndexError(f"parameter {p} out of range (circuit has {len(base)})")
    batch = DcBatch([circuit] * len(values), symbolic=symbolic)
    off = batch.param_offsets
    flat = np.zeros(int(off[-1]), np.float64)
    for i, row in enumerate(values):
        flat[off[i]:off[i + 1]] = base
        for p, v in zip(params, row):
            flat[off[i] + p] = v
    sols, status, iters = batch.run(torch.from_numpy(flat).cuda())
    torch.cuda.synchronize()
    return (np.stack(batch.split(sols)), status.cpu().numpy(), iters.cpu().numpy())
