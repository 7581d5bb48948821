"""Bounded waits give up cleanly.  With nsg_set_wait_limit(0) every
dependency wait that has to poll gives up at once: the dataflow refactor,
the grid-wide refactor and the batched DC Newton kernel report NSG_TIMEOUT
(104) for the instance and return.  With the default limit restored, the
same batches then produce the oracle's values bit for bit, so the context
survived the give-up path."""
import numpy as np
import pytest
import torch

import oracle
from matrices import banded
from neospice_b200 import _lib as L
from neospice_b200 import workloads as W
from neospice_b200.circuit import DcBatch
from neospice_b200.solver import Batch, Topology

pytestmark = pytest.mark.gpu


def _set_limit(polls):
    assert L.lib().nsg_set_wait_limit(polls) == L.NSG_OK, L.lib().nsg_last_error()


@pytest.mark.parametrize("schedule", [0, 2])
def test_zero_wait_limit_reports_timeout_then_refactor_recovers(schedule):
    n, cp, ri, v = banded(3000, 7, seed=11)
    topo = Topology.order(n, cp, ri, v)
    batch = Batch([topo])
    batch.set_schedule(schedule)
    d_a = torch.from_numpy(v).cuda()
    try:
        _set_limit(0)
        st, _ = batch.refactor(d_a)
        torch.cuda.synchronize()
        assert int(st.cpu()[0]) == L.NSG_TIMEOUT
    finally:
        _set_limit(L.NSG_DEFAULT_WAIT_LIMIT)
    st, _ = batch.refactor(d_a)
    torch.cuda.synchronize()
    assert int(st.cpu()[0]) == 0
    s = oracle.Structure(n, *topo.export())
    rc, lu_ref, _ = oracle.port_refactor(s, v)
    assert rc == 0
    np.testing.assert_array_equal(batch.lu_values()[:s.n_elem], lu_ref)


def test_zero_wait_limit_in_the_newton_kernel():
    meshes = W.diode_mesh_batch(2, seed=5, side_range=(40, 48))
    batch = DcBatch([m.build() for m in meshes], symbolic=DcBatch.PER_INSTANCE)
    try:
        _set_limit(0)
        _, status, _ = batch.run()
        torch.cuda.synchronize()
        assert (status.cpu().numpy() == L.NSG_TIMEOUT).all()
    finally:
        _set_limit(L.NSG_DEFAULT_WAIT_LIMIT)
    sols, status, iters = batch.run()
    torch.cuda.synchronize()
    assert int(status.abs().sum()) == 0
    if not oracle.have_ref():
        return
    gpu = batch.split(sols)
    for k, m in enumerate(meshes):
        ref, it, _ = oracle.ref_mesh_dc(m)
        np.testing.assert_allclose(gpu[k], ref, rtol=1e-9, atol=1e-12)
        assert int(iters.cpu()[k]) == it
