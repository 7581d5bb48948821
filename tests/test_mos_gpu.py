"""GPU parity of level-1 MOSFET circuits (MOS1load on the device): DC
operating points of inverter chains and seeded MOS networks against the
reference's solve_dc (tests/golden/mos_dc.npz): solutions within 1e-9
relative / 1e-12 absolute, the same Newton iteration counts and the same
convergence method (direct Newton or gmin stepping)."""
import numpy as np
import pytest
import torch

import golden_cases
from neospice_b200.circuit import DcBatch

pytestmark = pytest.mark.gpu
CASES = golden_cases.load_mos_dc()


@pytest.mark.parametrize("symbolic", [DcBatch.PER_INSTANCE, DcBatch.PER_PATTERN])
def test_mos_dc_matches_reference(symbolic):
    batch = DcBatch([g["netlist"].build() for g in CASES], symbolic=symbolic)
    sols, status, iters = batch.run()
    torch.cuda.synchronize()
    status = status.cpu().numpy()
    iters = iters.cpu().numpy()
    method, _ = batch.methods()
    for k, (g, s) in enumerate(zip(CASES, batch.split(sols))):
        assert status[k] == 0, (k, status[k])
        np.testing.assert_allclose(s, g["solution"], rtol=1e-9, atol=1e-12, err_msg=f"case {k}")
        assert iters[k] == int(g["iterations"]), (k, iters[k], int(g["iterations"]))
        assert method[k] == int(g["method"]), (k, method[k], int(g["method"]))


def test_mos_dc_host_reorder_path():
    """An inverter chain whose pivots fail re-validation during the DC
    Newton solve: without host re-ordering the instance reports 103; with it
    the solve resumes on the device and matches the reference."""
    g = CASES[3]
    batch = DcBatch([g["netlist"].build()], symbolic=DcBatch.PER_INSTANCE)
    batch.set_reorder(False)
    _, status, _ = batch.run()
    torch.cuda.synchronize()
    assert int(status.cpu()[0]) == 103
    batch.set_reorder(True)
    sols, status, iters = batch.run()
    torch.cuda.synchronize()
    assert int(status.cpu()[0]) == 0
    assert batch.reorders() >= 1
    np.testing.assert_allclose(batch.split(sols)[0], g["solution"], rtol=1e-9, atol=1e-12)
    assert int(iters.cpu()[0]) == int(g["iterations"])
