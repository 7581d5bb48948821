"""GPU parity of the batched DC operating point: solutions within 1e-9
relative / 1e-12 absolute of the reference's solve_dc, same Newton
iteration counts."""
import numpy as np
import pytest
import torch

import golden_cases
import oracle
from neospice_b200 import workloads
from neospice_b200.circuit import DcBatch

pytestmark = pytest.mark.gpu
MESHES = golden_cases.load_meshes()
RTOL, ATOL = 1e-9, 1e-12


def _check(sol, ref):
    np.testing.assert_allclose(sol, ref, rtol=RTOL, atol=ATOL)


@pytest.mark.parametrize("symbolic", [DcBatch.PER_INSTANCE, DcBatch.PER_PATTERN])
def test_dc_matches_golden(symbolic):
    circuits = [g["mesh"].build() for g in MESHES]
    batch = DcBatch(circuits, symbolic=symbolic)
    sols, status, iters = batch.run()
    torch.cuda.synchronize()
    status = status.cpu().numpy()
    iters = iters.cpu().numpy()
    for k, (g, s) in enumerate(zip(MESHES, batch.split(sols))):
        assert status[k] == 0, (k, status[k])
        assert iters[k] == int(g["iterations"]), (k, iters[k], int(g["iterations"]))
        _check(s, g["solution"])


def test_dc_params_override_and_repeat():
    """Parameters passed on the device replace the circuits' own values;
    repeated runs give identical results."""
    circuits = [g["mesh"].build() for g in MESHES[:4]]
    batch = DcBatch(circuits)
    p = torch.from_numpy(batch.params()).cuda()
    s1, st1, _ = batch.run(d_params=p)
    s2, st2, _ = batch.run(d_params=p)
    torch.cuda.synchronize()
    assert torch.equal(s1, s2)
    assert int(st1.abs().sum()) == 0
    # scale every resistor of instance 0 by 2: its solution must change
    p2 = p.clone()
    m = MESHES[0]["mesh"]
    nr = len(m.r_h) + len(m.r_v)
    p2[:nr] *= 2.0
    s3, st3, _ = batch.run(d_params=p2)
    torch.cuda.synchronize()
    a = batch.split(s1)[0]
    b = batch.split(s3)[0]
    assert not np.allclose(a, b)
    assert np.allclose(batch.split(s1)[1], batch.split(s3)[1])


@pytest.mark.skipif(not oracle.have_ref(), reason="reference library not built here")
def test_dc_mixed_sizes_against_reference():
    meshes = [workloads.diode_mesh(np.random.default_rng([31, k]), side_range=(16, 40))
              for k in range(12)]
    batch = DcBatch([m.build() for m in meshes], symbolic=DcBatch.PER_INSTANCE)
    sols, status, iters = batch.run()
    torch.cuda.synchronize()
    for k, (m, s) in enumerate(zip(meshes, batch.split(sols))):
        ref, ref_it, _ = oracle.ref_mesh_dc(m)
        assert int(status[k]) == 0
        assert int(iters[k]) == ref_it
        _check(s, ref)


def test_dc_graph_replay_matches_plain_launch():
    """Runs replayed from a captured CUDA graph give the plain launch's
    results bit for bit (same buffers every run)."""
    plain = DcBatch([g["mesh"].build() for g in MESHES])
    s0, st0, it0 = plain.run()
    torch.cuda.synchronize()
    batch = DcBatch([g["mesh"].build() for g in MESHES])
    batch.set_graph(True)
    sol = torch.empty_like(s0)
    st = torch.empty_like(st0)
    it = torch.empty_like(it0)
    for _ in range(3):
        sol.zero_()
        batch.run(d_solutions=sol, d_status=st, d_iterations=it)
        torch.cuda.synchronize()
        assert torch.equal(sol, s0) and torch.equal(st, st0) and torch.equal(it, it0)
    assert batch.graph_launches() == 2


def test_dc_row_maps_bitwise():
    """Update destinations from per-warp row maps instead of the plans'
    update maps: identical solutions, statuses and iteration counts on the
    golden meshes, MOS circuits and AMD-LU-sized linear grids, and through a
    captured graph."""
    nets = [g["mesh"].build for g in MESHES] + [g["netlist"].build for g in golden_cases.load_mos_dc()]
    nets += [workloads.power_grid(np.random.default_rng([33, k]), 24, 8, 10).build for k in range(2)]
    base = DcBatch([f() for f in nets])
    s0, st0, it0 = base.run()
    torch.cuda.synchronize()
    rows = DcBatch([f() for f in nets])
    rows.set_row_maps(True)
    for graph in (False, True):
        rows.set_graph(graph)
        for _ in range(2):
            s1, st1, it1 = rows.run()
            torch.cuda.synchronize()
            assert torch.equal(st1, st0) and torch.equal(it1, it0)
            assert torch.equal(s1, s0)
