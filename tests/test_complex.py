"""The AC symbolic phase on the host (NeoSolver::numeric_complex):
Markowitz ordering on complex values with magnitudes |re| + |im| and complex
eliminations must pick exactly the reference's pivots -- checked on seeded
random complex matrices and on G + jwC of RC ladders and meshes."""
import numpy as np
import pytest

import oracle
from matrices import random_matrix
from neospice_b200 import workloads as W
from neospice_b200.solver import Topology

needs_ref = pytest.mark.skipif(not oracle.have_ref(), reason="reference library not built here")


def _same_order(n, cp, ri, ax):
    t = Topology.order_complex(n, cp, ri, ax)
    rs = oracle.RefSolver(n, cp, ri)
    assert rs.numeric_complex(ax) == 0
    st, _ = rs.export_complex()
    assert st.same_as(oracle.Structure(n, *t.export()))


@needs_ref
@pytest.mark.parametrize("seed", range(12))
def test_random_complex_matrices_same_pivots(seed):
    rng = np.random.default_rng([51, seed])
    n = int(rng.integers(5, 60))
    n_, cp, ri, re = random_matrix(rng, n, 0.15, diag_dominant=bool(seed % 2),
                                   zero_diag_frac=0.2 if seed % 3 == 0 else 0.0)
    im = rng.standard_normal(len(re)) * (10.0 ** rng.integers(-3, 3))
    _same_order(n_, cp, ri, re + 1j * im)


@needs_ref
@pytest.mark.parametrize("freq", [1e3, 1e8, 1e11])
def test_rc_circuits_same_pivots(freq):
    for nl in (W.rc_ladder(np.random.default_rng(3), 20), W.rc_mesh(np.random.default_rng(4), 8)):
        n, cp, ri, g, c, _ = W.ac_system(nl)
        _same_order(n, cp, ri, g + 1j * (2 * np.pi * freq) * c)
