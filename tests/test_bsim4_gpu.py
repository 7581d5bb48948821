"""GPU parity of BSIM4v7 (LEVEL=14) circuits against the reference
(tests/golden/bsim4.npz, made by the reference itself): DC operating points
(the reference unit test's bias point, NMOS / PMOS bias points, inverter
chains with per-device TOXE and DELVTO) within 1e-9 relative / 1e-12
absolute with the same Newton iteration counts and convergence method; and
transients (an inverter chain under a PULSE and Monte Carlo instances of the
200-MOSFET ring-oscillator + NAND-chain circuit) against the reference's
own waveforms.

The transients are held to the Newton tolerances (reltol 1e-3, vntol
1e-6 V), not to 1e-9: the BSIM4v7 load evaluates a few hundred exp / log /
pow per device, and the GPU's versions of those functions round differently
from the host C library in about 2-3 % of the load's outputs (up to 3e-4
relative in terms that are differences of nearly equal capacitances), while
the host load itself is bit-identical to the reference in every mode
(tests/test_bsim4.py).  A Newton solve that stops at |dx| <= vntol returns an
iterate whose distance from the fixed point depends on the Jacobian it used,
so those last-place differences reach the waveform at the size of an
unconverged Newton step, and an iteration count can differ by one now and
then.  The timepoints must still be the same."""
import numpy as np
import pytest
import torch

import golden_cases
from neospice_b200.circuit import DcBatch, TranBatch

pytestmark = pytest.mark.gpu
DC, TRAN = golden_cases.load_bsim4()


@pytest.mark.parametrize("symbolic", [DcBatch.PER_INSTANCE, DcBatch.PER_PATTERN])
def test_bsim4_dc_matches_reference(symbolic):
    batch = DcBatch([g["netlist"].build() for g in DC], symbolic=symbolic)
    sols, status, iters = batch.run()
    torch.cuda.synchronize()
    status = status.cpu().numpy()
    iters = iters.cpu().numpy()
    method, _ = batch.methods()
    for k, (g, s) in enumerate(zip(DC, batch.split(sols))):
        assert status[k] == 0, (k, status[k])
        np.testing.assert_allclose(s, g["solution"], rtol=1e-9, atol=1e-12, err_msg=f"case {k}")
        assert iters[k] == int(g["iterations"]), (k, iters[k], int(g["iterations"]))
        assert method[k] == int(g["method"]), (k, method[k], int(g["method"]))


def test_bsim4_unit_test_drain_current():
    """Id = 5.754970e-05 A at VDS 0.1, VGS 0.8 (ngspice's value, which the
    reference's unit test pins to 1e-3 relative)."""
    batch = DcBatch([DC[0]["netlist"].build()])
    sols, status, _ = batch.run()
    torch.cuda.synchronize()
    assert int(status.cpu()[0]) == 0
    idrain = -float(sols.cpu()[5])
    assert abs(idrain - 5.754970e-05) <= 1e-3 * 5.754970e-05


@pytest.mark.parametrize("group", [[0], [1, 2]])
def test_bsim4_transient_matches_reference(group):
    cases = [TRAN[k] for k in group]
    probes = cases[0]["probes"]
    b = TranBatch([g["netlist"].build() for g in cases], float(cases[0]["tstep"]),
                  float(cases[0]["tstop"]), probes,
                  max_points=max(len(g["times"]) for g in cases) + 8)
    b.run()
    for k, (g, r) in enumerate(zip(cases, b.results())):
        assert r["status"] == 0, (k, r["status"])
        assert len(r["time"]) == len(g["times"]), (k, len(r["time"]), len(g["times"]))
        np.testing.assert_allclose(r["time"], g["times"], rtol=1e-12, atol=0, err_msg=f"case {k}")
        np.testing.assert_allclose(r["values"], g["values"], rtol=1e-3, atol=1e-6,
                                   err_msg=f"case {k}")
        it, it_ref = r["newton_iters"], int(g["iterations"])
        assert abs(it - it_ref) <= max(2, it_ref // 100), (k, it, it_ref)
        assert r["rejected"] == int(g["rejected"]), (k, r["rejected"], int(g["rejected"]))
