"""dc_solve_global on one GPU (no process group: the whole batch is this
rank's share): the same solutions, statuses and iteration counts, bit for
bit, as one DcBatch of the same circuits, in the circuits' order."""
import numpy as np
import pytest
import torch

from neospice_b200 import sharding, workloads
from neospice_b200.circuit import DcBatch

pytestmark = pytest.mark.gpu


def test_dc_solve_global_matches_one_batch():
    meshes = workloads.diode_mesh_batch(12, seed=5, side_range=(6, 20))
    out = sharding.dc_solve_global([m.build() for m in meshes])
    batch = DcBatch([m.build() for m in meshes], symbolic=DcBatch.PER_INSTANCE)
    sols, status, iters = batch.run()
    torch.cuda.synchronize()
    st, it = status.cpu().numpy(), iters.cpu().numpy()
    assert len(out) == len(meshes)
    for k, (s, (x, s_k, i_k)) in enumerate(zip(batch.split(sols), out)):
        s = s.cpu().numpy() if hasattr(s, "cpu") else s
        np.testing.assert_array_equal(x, s)
        assert (s_k, i_k) == (int(st[k]), int(it[k])) and s_k == 0
