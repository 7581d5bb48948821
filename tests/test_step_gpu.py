"""GPU parity of the batched `.step` sweep (every step one instance of one
launch) against the reference's serial Simulator::run_step_sweep
(tests/golden/step_dc.npz): node voltages within 1e-9 relative / 1e-12
absolute and the same Newton iterations at every step."""
import numpy as np
import pytest

import golden_cases
from neospice_b200.circuit import DcBatch
from neospice_b200.step import step_values, sweep_dc

pytestmark = pytest.mark.gpu
CASES = golden_cases.load_steps()


def test_step_sweep_matches_reference():
    for k, g in enumerate(CASES):
        nl = g["netlist"]
        values = step_values(*(float(x) for x in g["sweep"]))
        sols, status, iters = sweep_dc(nl.build(), int(g["param"]), values,
                                       symbolic=DcBatch.PER_INSTANCE)
        assert (status == 0).all(), (k, status)
        np.testing.assert_allclose(sols[:, :nl.num_nodes], g["volts"], rtol=1e-9, atol=1e-12,
                                   err_msg=f"case {k}")
        np.testing.assert_array_equal(iters, g["iterations"], err_msg=f"case {k}")


def test_step_transient_matches_reference():
    """`.tran` under `.step` of a DC supply: each step's timepoints, node
    voltages and Newton iterations as the reference's serial sweep."""
    from neospice_b200.step import sweep_transient
    for k, g in enumerate(golden_cases.load_step_transients()):
        nl = g["netlist"]
        values = step_values(*(float(x) for x in g["sweep"]))
        tstep, tstop = (float(x) for x in g["tran"])
        probes = np.arange(nl.num_nodes, dtype=np.int32)
        res = sweep_transient(nl.build, int(g["param"]), values, tstep, tstop, probes,
                              max_points=max(len(t) for t, _ in g["runs"]) + 8)
        for q, (r, (t, v)) in enumerate(zip(res, g["runs"])):
            assert r["status"] == 0, (k, q, r["status"])
            assert len(r["time"]) == len(t), (k, q, len(r["time"]), len(t))
            np.testing.assert_allclose(r["time"], t, rtol=1e-12, atol=0, err_msg=f"{k}/{q}")
            np.testing.assert_allclose(r["values"], v, rtol=1e-9, atol=1e-12, err_msg=f"{k}/{q}")
            assert r["newton_iters"] == int(g["iterations"][q]), (k, q, r["newton_iters"])
