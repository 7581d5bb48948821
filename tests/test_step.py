"""`.step` sweeps on the host: the step values are the reference's own
(tests/golden/step_dc.npz, from Simulator::run_step_sweep), bit for bit —
ascending, descending and with steps that accumulate rounding."""
import numpy as np
import pytest

import golden_cases
from neospice_b200 import _lib as L
from neospice_b200.step import step_values

CASES = golden_cases.load_steps()


def test_step_values_match_reference():
    for g in CASES:
        start, stop, step = (float(x) for x in g["sweep"])
        np.testing.assert_array_equal(step_values(start, stop, step), g["values"])


def test_step_values_edge_cases():
    np.testing.assert_array_equal(step_values(1.0, 1.0, 0.5), [1.0])
    assert len(step_values(1.0, 0.0, 0.5)) == 0
    with pytest.raises(L.NsgError):
        step_values(0.0, 1.0, 0.0)


def test_stepped_parameter_index():
    """The fixture's parameter index addresses the stepped source's value in
    Circuit.params()."""
    for g in CASES:
        nl = g["netlist"]
        c = nl.build()
        dev = [i for i, _ in enumerate(nl.devices)
               if golden_cases.param_starts(nl)[i][1] == int(g["param"])][0]
        assert c.params()[int(g["param"])] == nl.devices[dev][3]


def test_transient_step_values_match_reference():
    for g in golden_cases.load_step_transients():
        start, stop, step = (float(x) for x in g["sweep"])
        assert len(step_values(start, stop, step)) == len(g["runs"])
