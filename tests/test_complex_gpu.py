"""GPU parity of the batched AC path: the pivots of the first frequency
point (NeoSolver::numeric_complex on the host), then every frequency point
of the sweep refactored at once on the GPU (factor_complex with those
pivots) and solved (solve_complex).  Factor values and solutions must equal
the reference's NeoSolver -- numeric_complex at the first point,
refactorize_complex at the others, solve_complex -- bit for bit."""
import numpy as np
import pytest
import torch

import oracle
from matrices import random_matrix
from neospice_b200 import workloads as W
from neospice_b200.solver import Batch, Topology, _interleave

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.have_ref(), reason="reference library not built")]


def _check(n, cp, ri, axs, bs):
    """axs: complex values per frequency point (first one orders); bs: rhs."""
    topo = Topology.order_complex(n, cp, ri, axs[0])
    batch = Batch([topo] * len(axs))
    d_ax = torch.from_numpy(np.concatenate([_interleave(a) for a in axs])).cuda()
    d_lu, st = batch.refactor_complex(d_ax)
    d_x = torch.from_numpy(np.concatenate([_interleave(b) for b in bs])).cuda()
    batch.solve_complex(d_lu, d_x)
    torch.cuda.synchronize()
    assert int(st.abs().sum()) == 0
    lu = d_lu.cpu().numpy()
    x = d_x.cpu().numpy()
    rs = oracle.RefSolver(n, cp, ri)
    for k, (ax, b) in enumerate(zip(axs, bs)):
        rc = rs.numeric_complex(ax) if k == 0 else rs.refactorize_complex(ax)
        assert rc == 0
        _, ref_lu = rs.export_complex()
        o = 2 * int(batch.lu_offsets[k])
        ours = lu[o:o + 2 * len(ref_lu)]
        np.testing.assert_array_equal(ours[0::2], ref_lu.real, err_msg=f"point {k} re")
        np.testing.assert_array_equal(ours[1::2], ref_lu.imag, err_msg=f"point {k} im")
        xr = rs.solve_complex(b)
        v = 2 * int(batch.vector_offsets[k])
        np.testing.assert_array_equal(x[v:v + 2 * n:2], xr.real, err_msg=f"point {k} x re")
        np.testing.assert_array_equal(x[v + 1:v + 2 * n:2], xr.imag, err_msg=f"point {k} x im")


@pytest.mark.parametrize("seed", range(6))
def test_random_complex_sweep_bitwise(seed):
    rng = np.random.default_rng([52, seed])
    n = int(rng.integers(10, 80))
    n_, cp, ri, re = random_matrix(rng, n, 0.12)
    im0 = rng.standard_normal(len(re))
    axs = [re + 1j * im0 * s for s in (1.0, 0.5, 3.0, 10.0)]
    bs = [rng.standard_normal(n_) + 1j * rng.standard_normal(n_) for _ in axs]
    _check(n_, cp, ri, axs, bs)


@pytest.mark.parametrize("kind", ["ladder", "mesh"])
def test_rc_ac_sweep_bitwise(kind):
    nl = W.rc_ladder(np.random.default_rng(5), 40) if kind == "ladder" else \
        W.rc_mesh(np.random.default_rng(6), 12)
    n, cp, ri, g, c, b = W.ac_system(nl)
    freqs = np.logspace(3, 11, 17)
    axs = [g + 1j * (2 * np.pi * f) * c for f in freqs]
    _check(n, cp, ri, axs, [b] * len(axs))
