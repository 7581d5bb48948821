"""The allocation-free solve (nsg_batch_solve_static_scratch).

It serves callers that must not allocate device memory when they solve (a
fixed memory budget, another framework's memory pool, or a loop that cannot
absorb cudaMalloc's implicit synchronisation): its sweep workspace is a fixed
array inside the library.  It must give exactly what nsg_batch_solve gives
(the solves here are bit-for-bit, the tolerance all solve tests use), on two
calls in a row, through the C ABI; and it must refuse batches larger than
the array.  This file is collected last so a failure here leaves every other
test already run; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest
import torch

import golden_cases
from matrices import banded
from neospice_b200 import _lib as L
from neospice_b200.solver import Batch, Topology

pytestmark = pytest.mark.gpu


def _packed(batch, per_instance):
    out = np.zeros(int(batch.vector_offsets[-1]))
    for i, v in enumerate(per_instance):
        out[batch.vector_offsets[i]:batch.vector_offsets[i + 1]] = v
    return out


def test_static_scratch_solve_matches_regular_solve_twice():
    cases = golden_cases.load()
    topos = [Topology.order(int(c["n"]), c["col_ptr"], c["row_idx"], c["vals"]) for c in cases]
    batch = Batch(topos)
    a = np.zeros(int(batch.value_offsets[-1]))
    for i, c in enumerate(cases):
        a[batch.value_offsets[i]:batch.value_offsets[i + 1]] = c["vals"]
    status, _ = batch.refactor(torch.from_numpy(a).cuda())
    torch.cuda.synchronize()
    assert int(status.abs().sum()) == 0
    rng = np.random.default_rng(3)
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        b = _packed(batch, [rng.standard_normal(int(c["n"])) for c in cases])
        d_reg = torch.from_numpy(b).cuda()
        d_new = torch.from_numpy(b).cuda()
        batch.solve(d_reg)
        rc = L.lib().nsg_batch_solve_static_scratch(batch._h, d_new.data_ptr(), stream)
        assert rc == L.NSG_OK, L.lib().nsg_last_error()
        torch.cuda.synchronize()
        assert torch.equal(d_reg, d_new), f"call {call}"


def test_static_scratch_rejects_oversized_batch():
    n, cp, ri, v = banded(20000, 7, seed=4)
    topo = Topology.order(n, cp, ri, v)
    count = L.NSG_STATIC_SCRATCH_DOUBLES // n + 1
    batch = Batch([topo] * count)
    assert int(batch.vector_offsets[-1]) > L.NSG_STATIC_SCRATCH_DOUBLES
    d_x = torch.zeros(int(batch.vector_offsets[-1]), dtype=torch.float64, device="cuda")
    rc = L.lib().nsg_batch_solve_static_scratch(batch._h, d_x.data_ptr(),
                                                torch.cuda.current_stream().cuda_stream)
    assert rc == L.NSG_ERR_INVALID
    assert b"static workspace" in L.lib().nsg_last_error()
