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


def _eval_sequence(nl, rng, dt=1e-12, temp=None):
    """Ten device evaluations as a DC solve, the transient seeding, backward
    Euler, trapezoidal and Gear-2 steps would run them (INITJCT, INITFLOAT,
    INITTRAN, INITPRED), at random guesses with every terminal bias sign
    (at circuit temperature `temp` kelvin when given); returns (ours,
    reference) lists of (matrix, rhs)."""
    c = nl.build(temp=temp)
    n = c.info()["num_vars"]
    nn = nl.num_nodes

    def guess():
        x = np.zeros(n)
        x[:nn] = rng.uniform(-0.2, 1.3, nn)
        x[nn:] = rng.normal(0.0, 1e-4, n - nn)
        return x

    h0, h1 = dt, 1.5 * dt
    be = [1 / dt, -1 / dt, 0, 0, dt, dt, dt, 1]
    trap = [2 / dt, -2 / dt, 0, 1.0, dt, dt, 2 * dt, 2]
    gear = [(2 * h0 + h1) / (h0 * (h0 + h1)), -(h0 + h1) / (h0 * h1), h0 / (h1 * (h0 + h1)),
            0, h0, h1, 3 * dt, 12]
    dc = [0, 0, 0, 0, 0, 0, 0, 1]
    x2 = guess()
    steps = [(0, 0x210, np.zeros(n), dc), (0, 0x110, guess(), dc), (0, 0x110, x2, dc),
             (2, 0x1001, x2, be), (0, 0x101, guess(), be), (0, 0x101, guess(), be),
             (1, 0x2001, guess(), trap), (0, 0x101, guess(), trap),
             (1, 0x2001, guess(), gear), (0, 0x101, guess(), gear)]
    ops, modes, xs, ctx = (np.array([s[k] for s in steps]) for k in range(4))
    rv, rr = oracle.ref_sim_eval_seq(netlists.ref_desc(nl, None if temp is None else {"temp": temp}),
                                     ops, modes, xs.astype(float),
                                     ctx.astype(float))
    ns = c.state_count()
    st = np.zeros(3 * ns)
    rec = np.zeros(12 * sum(1 for d in nl.devices if d[0] == "M"))
    ours = []
    for s, (op, mode, x, cx) in enumerate(steps):
        if op == 1:  # rotate_state: state2 <- state1 <- copy of state0
            st[2 * ns:] = st[ns:2 * ns]
            st[ns:2 * ns] = st[:ns]
        elif op == 2:  # the transient's seeding from the operating point
            st[ns:2 * ns] = st[:ns]
            st[2 * ns:] = st[:ns]
        ours.append(c.eval_matrix(mode, x, cx[:7], int(cx[7]) % 10, int(cx[7]) // 10, st, rec))
    return ours, list(zip(rv, rr))


@needs_ref
@pytest.mark.parametrize("case", ["chain", "ring0", "ring1"])
def test_transient_mode_loads_bitwise(case):
    """The host load in every transient mode -- charges, NIintegrate, the
    predictor, junction and overlap capacitances, reverse mode, body bias --
    equals the reference's matrix and rhs bit for bit, step after step with
    the state ring carried along."""
    nl = TRAN[0]["netlist"] if case == "chain" else \
        W.bsim4_ring_nand(np.random.default_rng([31, int(case[-1])]))
    ours, ref = _eval_sequence(nl, np.random.default_rng([44, len(case), int(case[-1] == "1")]))
    for s, ((a, r), (ra, rr)) in enumerate(zip(ours, ref)):
        np.testing.assert_array_equal(a, ra, err_msg=f"step {s} matrix")
        np.testing.assert_array_equal(r, rr, err_msg=f"step {s} rhs")


def test_eval_matrix_refuses_diodes():
    c = Circuit(2)
    c.V(0, -1, 1.0)
    c.D(0, 1)
    c.R(1, -1, 1e3)
    c.finalize()
    with pytest.raises(L.NsgError):
        c.eval_matrix(0x210, np.zeros(3), np.zeros(7), 1, 0, np.zeros(3 * c.state_count()),
                      np.zeros(1))
