"""GPU DC adjoint (transposed solve on the LU at the solution, then the
parameter contraction): against the reference's finite-difference .sens
(tests/golden/sens_dc.npz; its one-sided step of 1e-4 relative limits the
agreement to 1e-3 relative on linear networks and to 5e-3 on MOS networks,
whose second derivatives enter the one-sided difference), and against central finite differences of our own batched
forward solve (h = 1e-6 relative, tight Newton tolerances) to 1e-6 relative,
including MOSFET W, L and VTO; plus the torch.autograd wrapper."""
import numpy as np
import pytest
import torch

import golden_cases
from neospice_b200 import workloads as W
from neospice_b200.autodiff import dc_solve
from neospice_b200.circuit import DcBatch

pytestmark = pytest.mark.gpu
CASES = golden_cases.load_sens()


def _grads(batch, out_nodes, params=None):
    sols, status, _ = batch.run(d_params=params)
    assert int(status.abs().sum()) == 0
    cot = torch.zeros_like(sols)
    off = batch.solution_offsets
    for k, node in enumerate(out_nodes):
        cot[int(off[k]) + node] = 1.0
    g, st = batch.adjoint(sols, cot, d_params=params)
    torch.cuda.synchronize()
    assert int(st.abs().sum()) == 0
    return sols, g.cpu().numpy()


def test_adjoint_matches_reference_sens():
    batch = DcBatch([c["netlist"].build() for c in CASES], symbolic=DcBatch.PER_INSTANCE)
    _, g = _grads(batch, [int(c["output"]) for c in CASES])
    po = batch.param_offsets
    for k, c in enumerate(CASES):
        starts = golden_cases.param_starts(c["netlist"])
        order = ([s for kind, s in starts if kind == "R"] + [s for kind, s in starts if kind == "V"]
                 + [s for kind, s in starts if kind == "I"])
        ours = g[int(po[k]) + np.array(order, dtype=np.int64)]
        ref = c["sens"]
        scale = np.max(np.abs(ref))
        linear = not c["netlist"].models
        np.testing.assert_allclose(ours, ref, rtol=1e-3 if linear else 5e-3, atol=1e-6 * scale,
                                   err_msg=f"case {k}")


def _fd(batch, base, idx, out_global, h_rel=1e-6):
    p_hi, p_lo = base.clone(), base.clone()
    h = abs(float(base[idx])) * h_rel
    p_hi[idx] += h
    p_lo[idx] -= h
    s_hi, st_hi, _ = batch.run(d_params=p_hi)
    x_hi = float(s_hi[out_global])
    s_lo, st_lo, _ = batch.run(d_params=p_lo)
    x_lo = float(s_lo[out_global])
    assert int(st_hi.abs().sum()) == 0 and int(st_lo.abs().sum()) == 0
    return (x_hi - x_lo) / (2 * h)


@pytest.mark.parametrize("k", [0, 4])
def test_adjoint_matches_central_differences(k):
    nl = CASES[k]["netlist"]
    out = int(CASES[k]["output"])
    batch = DcBatch([nl.build()], symbolic=DcBatch.PER_INSTANCE)
    batch.set_options(reltol=1e-12, vntol=1e-15, abstol=1e-18, max_iter=200)
    base = torch.from_numpy(batch.params()).cuda()
    _, g = _grads(batch, [out], base)
    starts = golden_cases.param_starts(nl)
    idx = [s for kind, s in starts if kind in ("R", "V", "I")][:8]
    for kind, s in starts:
        if kind == "M":
            idx += [s + 0, s + 1, s + 2]  # W, L, VTO
    idx = idx[:20]
    for i in idx:
        fd = _fd(batch, base, i, out)
        assert abs(g[i] - fd) <= 1e-6 * max(abs(fd), 1e-12) + 1e-9 * np.max(np.abs(g)), (i, g[i], fd)


def test_autograd_function():
    nls = [W.resistor_network(np.random.default_rng([70, k]), 8) for k in range(3)]
    batch = DcBatch([n.build() for n in nls], symbolic=DcBatch.PER_INSTANCE)
    p = torch.from_numpy(batch.params()).cuda().requires_grad_(True)
    x = dc_solve(batch, p)
    target = torch.zeros_like(x)
    loss = ((x - target) ** 2).sum()
    loss.backward()
    cot = 2 * (x.detach() - target)
    g_ref, _ = batch.adjoint(x.detach(), cot, d_params=p.detach())
    torch.cuda.synchronize()
    assert torch.allclose(p.grad, g_ref, rtol=0, atol=0)
    assert float(p.grad.abs().sum()) > 0


def test_autograd_failed_instance_gets_nan():
    """An instance whose forward solve fails (here: a bounded wait that gives
    up, wait limit 0, on a mesh large enough for the dataflow path) gets NaN
    solutions and NaN gradients; a small instance beside it (warp path, no
    waits) keeps its exact values and gradients."""
    from neospice_b200 import _lib as L
    small = W.resistor_network(np.random.default_rng([71, 0]), 8).build()
    big = W.diode_mesh(np.random.default_rng([71, 1]), side=40).build()
    batch = DcBatch([small, big], symbolic=DcBatch.PER_INSTANCE)
    p = torch.from_numpy(batch.params()).cuda().requires_grad_(True)
    off = batch.solution_offsets
    assert L.lib().nsg_set_wait_limit(0) == L.NSG_OK
    try:  # only the forward solve runs with the zero limit
        x = dc_solve(batch, p)
        torch.cuda.synchronize()
    finally:
        assert L.lib().nsg_set_wait_limit(L.NSG_DEFAULT_WAIT_LIMIT) == L.NSG_OK
    loss = (x[int(off[0]):int(off[1])] ** 2).sum()
    loss.backward()
    torch.cuda.synchronize()
    po = batch.param_offsets
    assert torch.isnan(x[int(off[1]):int(off[2])]).all()
    assert torch.isnan(p.grad[int(po[1]):int(po[2])]).all()
    assert torch.isfinite(p.grad[:int(po[1])]).all()
    assert torch.isfinite(x[:int(off[1])]).all()
