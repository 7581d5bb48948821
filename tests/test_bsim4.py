"""BSIM4v7 (LEVEL=14) on the host: the parameter block of the default card
(BSIM4v7setup + BSIM4v7temp) and the device load, checked through the
first DC Newton matrix and rhs (MODEDCOP | MODEINITJCT), which must equal
the reference's bit for bit on every circuit of tests/golden/bsim4.npz and
on nominal and Monte Carlo instances of the 200-MOSFET ring-oscillator +
NAND-chain circuit; unsupported card parameters are refused."""
import numpy as np
import pytest

import golden_cases
import netlists
import oracle
from neospice_b200 import _lib as L
from neospice_b200 import workloads as W
from neospice_b200.circuit import Circuit

DC, TRAN = golden_cases.load_bsim4()
needs_ref = pytest.mark.skipif(not oracle.have_ref(), reason="reference library not built here")


def _check_initjct(nl):
    c = nl.build()
    cp, ri = c.pattern()
    a, rhs = c.initial_matrix(1e-12)
    rcp, rri, ra, rrhs = oracle.ref_sim_initjct(netlists.ref_desc(nl))
    np.testing.assert_array_equal(cp, rcp)
    np.testing.assert_array_equal(ri, rri)
    np.testing.assert_array_equal(a, ra)
    np.testing.assert_array_equal(rhs, rrhs)


@needs_ref
@pytest.mark.parametrize("k", range(len(DC)))
def test_dc_cases_first_matrix_bitwise(k):
    _check_initjct(DC[k]["netlist"])


@needs_ref
@pytest.mark.parametrize("seed", [None, 0, 1, 2])
def test_ring_nand_first_matrix_bitwise(seed):
    rng = None if seed is None else np.random.default_rng([31, seed])
    nl = W.bsim4_ring_nand(rng)
    _check_initjct(nl)
    c = nl.build()
    assert c.info()["num_vars"] == 102
    assert sum(1 for d in nl.devices if d[0] == "M") == 200


def test_golden_operating_point_is_the_unit_tests():
    """The first DC case is the reference unit test's circuit, whose drain
    current the reference pins to ngspice's 5.754970e-05 A (1e-3 relative)."""
    sol = DC[0]["solution"]
    assert abs(-sol[5] - 5.754970e-05) <= 1e-3 * 5.754970e-05


def test_unsupported_card_parameter_is_refused():
    c = Circuit(2)
    with pytest.raises(L.NsgError):
        c.model_bsim4("nmos", K1=0.5)
    m = c.model_bsim4("nmos", TOXE=2.5e-9, VTH0=0.45, U0=0.03)
    with pytest.raises(L.NsgError):
        c.M4(0, 1, -1, -1, m, W=1e-6, L_=-1e-7)
