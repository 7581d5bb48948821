"""GPU parity of the operating point's source stepping, gain stepping and
pseudo-transient continuation against the reference's own source_stepping
/ gain_stepping / pseudo_transient run alone (tests/golden/dc_aids.npz):
converged or not as the reference, solutions within 1e-9 relative / 1e-12
absolute, the same Newton iteration count (the aid's total: for source
stepping including the failed solve at zero sources and the diagonal-gmin
ramp that rescues it; for pseudo-transient every step whose pseudo
timestep follows the ratio of Newton residuals, and the probes)."""
import numpy as np
import pytest
import torch

import golden_cases
from neospice_b200.circuit import DcBatch

pytestmark = pytest.mark.gpu
CASES = golden_cases.load_aids()


@pytest.mark.parametrize("aid", ["source", "gain", "ptc"])
def test_aid_matches_reference(aid):
    analysis = {"source": 2, "gain": 3, "ptc": 4}[aid]
    cases = [g for g in CASES if int(g["aid"]) == analysis]
    batch = DcBatch([g["netlist"].build() for g in cases], symbolic=DcBatch.PER_INSTANCE)
    batch.set_first_aid(aid)
    sols, status, iters = batch.run()
    torch.cuda.synchronize()
    status = status.cpu().numpy()
    iters = iters.cpu().numpy()
    method, _ = batch.methods()
    for k, (g, s) in enumerate(zip(cases, batch.split(sols))):
        if int(g["converged"]):
            assert status[k] == 0, (aid, k, status[k])
            # SOURCE_STEPPING (gain stepping reports it too), PSEUDO_TRANSIENT
            assert method[k] == (3 if aid == "ptc" else 2), (aid, k, method[k])
            np.testing.assert_allclose(s, g["solution"], rtol=1e-9, atol=1e-12,
                                       err_msg=f"{aid} case {k}")
        else:
            assert status[k] == 1, (aid, k, status[k])
        assert iters[k] == int(g["iterations"]), (aid, k, iters[k], int(g["iterations"]))


def test_direct_cascade_unchanged_by_aid_option():
    """Back at "direct", a batch gives the cascade's result again (the
    option is per run, and the direct attempt converges on these)."""
    g = [c for c in CASES if int(c["aid"]) == 2][1]
    batch = DcBatch([g["netlist"].build()], symbolic=DcBatch.PER_INSTANCE)
    batch.set_first_aid("source")
    s1, st1, it1 = batch.run()
    batch.set_first_aid("direct")
    s2, st2, it2 = batch.run()
    torch.cuda.synchronize()
    assert int(st1.cpu()[0]) == 0 and int(st2.cpu()[0]) == 0
    assert batch.methods()[0][0] == 0  # DIRECT
    np.testing.assert_allclose(s1.cpu().numpy(), s2.cpu().numpy(), rtol=1e-3, atol=1e-5)
