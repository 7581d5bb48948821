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
