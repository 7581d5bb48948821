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


def test_param_step_matches_reference():
    """A `.param` entering two resistors and a diode's IS: every step sets the
    three values at once (sweep_dc_multi); each step's operating point
    equals the reference's on the netlist with those values, to 1e-9 with
    equal iteration counts."""
    import netlists
    import oracle
    from neospice_b200.step import sweep_dc_multi
    from neospice_b200.workloads import Netlist
    if not oracle.have_ref():
        pytest.skip("reference library not built")

    def netlist(r, is_):
        return Netlist(3, [("V", 0, -1, 3.0), ("R", 0, 1, r), ("R", 1, 2, r),
                           ("D", 2, -1, is_, 1.2), ("R", 2, -1, 5e3)], {})

    steps = [(100.0 * (1 + k), 1e-14 * (1 + 3 * k)) for k in range(5)]
    nl = netlist(*steps[0])
    nl.build()
    pidx = nl.param_index
    params = [pidx[1], pidx[2], pidx[3]]  # R1, R2, the diode's IS
    sols, status, iters = sweep_dc_multi(nl.build(), params,
                                         [(r, r, is_) for r, is_ in steps])
    assert (status == 0).all()
    for k, (r, is_) in enumerate(steps):
        _, vals, info = oracle.ref_sim(netlists.ref_desc(netlist(r, is_)), 0)
        np.testing.assert_allclose(sols[k], vals[0], rtol=1e-9, atol=1e-12, err_msg=f"step {k}")
        assert iters[k] == info["iterations"], (k, iters[k], info["iterations"])
