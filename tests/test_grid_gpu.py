"""The grid-wide schedule (one large instance refactored and swept by every
SM): bit-identical to the one-CTA-per-instance schedules, and to the
reference's AmdLuSolver on a power grid of 10^4 unknowns."""
import numpy as np
import pytest
import torch

import oracle
from neospice_b200 import workloads as W
from neospice_b200.solver import Batch, Topology

pytestmark = pytest.mark.gpu


def grid_matrix(side, pitch, loads, seed):
    c = W.power_grid(np.random.default_rng(seed), side, pitch, loads).build()
    cp, ri = c.pattern()
    vals, _ = c.initial_matrix(0.0)
    return len(cp) - 1, cp, ri, vals


def factor_and_solve(topo, vals, b, schedule, check=False):
    batch = Batch([topo])
    batch.set_schedule(schedule)
    d_a = torch.from_numpy(np.asarray(vals, np.float64)).cuda()
    st, fs = batch.refactor(d_a, 0.0, check_pivots=check)
    d_x = torch.from_numpy(np.asarray(b, np.float64).copy()).cuda()
    batch.solve(d_x)
    torch.cuda.synchronize()
    info = topo.info()
    return int(st.cpu()[0]), batch.lu_values()[:info["nnz_lu"]], d_x.cpu().numpy()


@pytest.mark.parametrize("engine", ["amdlu", "markowitz"])
def test_grid_schedule_matches_cta_schedule(engine):
    rng = np.random.default_rng(3)
    n, cp, ri, vals = grid_matrix(40, 8, 20, 1)
    topo = Topology.order(n, cp, ri, vals, solver=engine)
    vals2 = vals * np.exp(0.01 * rng.standard_normal(len(vals)))
    b = rng.standard_normal(n)
    s0, lu0, x0 = factor_and_solve(topo, vals2, b, 0)
    s2, lu2, x2 = factor_and_solve(topo, vals2, b, 2)
    assert s0 == s2 == 0
    np.testing.assert_array_equal(lu2, lu0)
    np.testing.assert_array_equal(x2, x0)


@pytest.mark.skipif(not oracle.have_ref(), reason="reference library not built")
def test_grid_schedule_power_grid_matches_reference():
    """A 100 x 100 power grid with pads: the reference's AmdLuSolver numeric
    + refactorize + solve, and this library's grid-wide replay, bit for bit."""
    rng = np.random.default_rng(4)
    n, cp, ri, vals = grid_matrix(100, 20, 100, 2)
    ref = oracle.RefAmdLu(n, cp, ri)
    assert ref.numeric(vals) == 0
    topo = Topology.order(n, cp, ri, vals, solver="amdlu")
    vals2 = vals * np.exp(0.02 * rng.standard_normal(len(vals)))
    assert ref.refactorize(vals2) == 0
    b = rng.standard_normal(n)
    x_ref = ref.solve(b)
    s, lu, x = factor_and_solve(topo, vals2, b, 2)
    assert s == 0
    f = ref.export()
    packed = np.concatenate([np.concatenate([f["Ux"][f["Up"][k]:f["Up"][k + 1]],
                                             f["Lx"][f["Lp"][k] + 1:f["Lp"][k + 1]]])
                             for k in range(n)])
    np.testing.assert_array_equal(lu, packed)
    np.testing.assert_array_equal(x, x_ref)


@pytest.mark.parametrize("engine", ["amdlu", "markowitz"])
@pytest.mark.parametrize("colbuf", [0, 1024, 2048, 4096])
def test_plans_without_update_map(engine, colbuf):
    """A factorization too large for an update map (forced here by a zero
    limit) runs on the grid-wide schedule with per-warp row -> position maps:
    factors and solutions bit-identical to the mapped plan's, for every
    column-buffer size; other schedules and circuit batches refuse it."""
    from neospice_b200 import _lib as L
    from neospice_b200.circuit import DcBatch
    rng = np.random.default_rng(11)
    n, cp, ri, vals = grid_matrix(60, 12, 30, 4)
    b = rng.standard_normal(n)
    mapped = Topology.order(n, cp, ri, vals, solver=engine)
    st0, lu0, x0 = factor_and_solve(mapped, vals, b, 2)
    assert L.lib().nsg_set_update_map_limit(0) == L.NSG_OK
    try:
        bare = Topology.order(n, cp, ri, vals, solver=engine)
        batch = Batch([bare])
        with pytest.raises(L.NsgError):
            batch.set_schedule(0)
        batch.set_grid_buffer(colbuf)
        d_a = torch.from_numpy(np.asarray(vals, np.float64)).cuda()
        for _ in range(2):  # the second call reuses the row maps
            st, _ = batch.refactor(d_a)
            d_x = torch.from_numpy(b.copy()).cuda()
            batch.solve(d_x)
            torch.cuda.synchronize()
            assert int(st.cpu()[0]) == st0 == 0
            np.testing.assert_array_equal(batch.lu_values()[:len(lu0)], lu0)
            np.testing.assert_array_equal(d_x.cpu().numpy(), x0)
        with pytest.raises(L.NsgError):
            DcBatch([W.power_grid(np.random.default_rng(1), 12, 6, 4).build()])
    finally:
        assert L.lib().nsg_set_update_map_limit(1 << 30) == L.NSG_OK


@pytest.mark.skipif(not oracle.have_ref(), reason="reference library not built")
@pytest.mark.parametrize("mapped", [True, False])
@pytest.mark.parametrize("colbuf", [2048, 4096])
def test_cta_tail_matches_reference(mapped, colbuf):
    """The grid-wide refactor's CTA-mode tail (columns claimed by whole CTAs,
    L(:, r) staged by cp.async): with the default tail (the columns with at
    least 128 updates), with the last 64 and with every column, mapped and
    map-less plans, refactorize() gives the reference AmdLuSolver's factor
    and solution bit for bit, and numeric() (pivot re-validation on the
    perturbed values) gives the all-warp schedule's verdict and values."""
    from neospice_b200 import _lib as L
    rng = np.random.default_rng(21)
    n, cp, ri, vals = W.power_grid_transient(90)
    ref = oracle.RefAmdLu(n, cp, ri)
    assert ref.numeric(vals) == 0
    vals2 = vals * np.exp(0.02 * rng.standard_normal(len(vals)))
    assert ref.refactorize(vals2) == 0
    b = rng.standard_normal(n)
    x_ref = ref.solve(b)
    f = ref.export()
    packed = np.concatenate([np.concatenate([f["Ux"][f["Up"][k]:f["Up"][k + 1]],
                                             f["Lx"][f["Lp"][k] + 1:f["Lp"][k + 1]]])
                             for k in range(n)])
    if not mapped:
        assert L.lib().nsg_set_update_map_limit(0) == L.NSG_OK
    try:
        topo = Topology.order(n, cp, ri, vals, solver="amdlu")
    finally:
        assert L.lib().nsg_set_update_map_limit(1 << 30) == L.NSG_OK
    d_a = torch.from_numpy(np.asarray(vals2, np.float64)).cuda()

    def run(tail, check):
        batch = Batch([topo])
        batch.set_schedule(2)
        batch.set_grid_buffer(colbuf)
        batch.set_grid_tail(tail)
        st, fs = batch.refactor(d_a, 0.0, check_pivots=check)
        d_x = torch.from_numpy(b.copy()).cuda()
        batch.solve(d_x)
        torch.cuda.synchronize()
        return (int(st.cpu()[0]), int(fs.cpu()[0]), batch.lu_values()[:len(packed)],
                d_x.cpu().numpy())

    numeric0 = run(0, True)
    for tail in (-1, 64, n):
        st, _, lu, x = run(tail, False)
        assert st == 0, tail
        np.testing.assert_array_equal(lu, packed)
        np.testing.assert_array_equal(x, x_ref)
        st, fs, lu, x = run(tail, True)
        assert (st, fs) == numeric0[:2], tail
        if st == 0:
            np.testing.assert_array_equal(lu, numeric0[2])
