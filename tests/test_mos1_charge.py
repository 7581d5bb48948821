"""Level-1 MOSFETs with charge on the host: Meyer gate charge (TOX),
gate overlap capacitances and bulk-junction charge (CBD / CBS, with body
effect), through the device load in every transient mode (INITJCT,
INITFLOAT, INITTRAN, INITPRED; backward Euler, trapezoidal and Gear-2
coefficients) with the state ring carried along: matrix and rhs equal the
reference's bit for bit at random guesses with every terminal bias sign."""
import numpy as np
import pytest

import oracle
from neospice_b200 import workloads as W
from test_bsim4 import _eval_sequence

needs_ref = pytest.mark.skipif(not oracle.have_ref(), reason="reference library not built here")

MEYER = {"TOX": 2e-8, "CGSO": 4e-10, "CGDO": 4e-10, "CGBO": 2e-10}
JUNCTION = {"CBD": 5e-15, "CBS": 4e-15, "GAMMA": 0.4}
GRADED = {"CJ": 2e-4, "CJSW": 1e-10, "MJ": 0.4, "MJSW": 0.3, "PB": 0.75, "FC": 0.45}


def _driven(seed, extra):
    nl = W.rc_tree_driven(np.random.default_rng(seed), 6)
    for name in ("nch", "pch"):
        nl.models[name][1].update(extra)
    return nl


@needs_ref
@pytest.mark.parametrize("case", ["meyer", "meyer+junction", "graded", "network"])
def test_mos1_charge_loads_bitwise(case):
    if case == "network":  # mos_network's oxide card plus junction charge everywhere
        nl = W.mos_network(np.random.default_rng(61), 10, pulse=(0.0, 1.8, 0.0, 1e-10, 1e-10,
                                                                  1e-9, 2e-9))
        for _, card in nl.models.values():
            card.update(JUNCTION)
    elif case == "graded":
        nl = _driven(62, {**MEYER, **JUNCTION, **GRADED})
    else:
        nl = _driven(63, dict(MEYER, **(JUNCTION if case == "meyer+junction" else {})))
    ours, ref = _eval_sequence(nl, np.random.default_rng([45, len(case)]))
    for s, ((a, r), (ra, rr)) in enumerate(zip(ours, ref)):
        np.testing.assert_array_equal(a, ra, err_msg=f"{case} step {s} matrix")
        np.testing.assert_array_equal(r, rr, err_msg=f"{case} step {s} rhs")


SERIES = [{"RD": 25.0, "RS": 10.0}, {"RSH": 40.0}, {"RD": 15.0}, {"RS": 30.0, "RSH": 20.0}]


@needs_ref
@pytest.mark.parametrize("k", range(len(SERIES)))
def test_mos1_series_resistance_bitwise(k):
    """Drain / source series resistance (RD, RS, or RSH with one square):
    the internal drain' and source' nodes are numbered as the reference
    numbers them (after the external nodes, in load order, drain' first),
    and the first DC matrix plus the whole transient-mode load sequence,
    charges included, equal the reference's bit for bit."""
    import netlists
    nl = _driven(64 + k, dict(MEYER, **JUNCTION, **SERIES[k]))
    c = nl.build()
    cp, ri = c.pattern()
    a, rhs = c.initial_matrix(1e-12)
    rcp, rri, ra, rrhs = oracle.ref_sim_initjct(netlists.ref_desc(nl))
    np.testing.assert_array_equal(cp, rcp)
    np.testing.assert_array_equal(ri, rri)
    np.testing.assert_array_equal(a, ra)
    np.testing.assert_array_equal(rhs, rrhs)
    assert c.info()["num_nodes"] > nl.num_nodes
    ours, ref = _eval_sequence(nl, np.random.default_rng([46, k]))
    for s, ((a, r), (ra, rr)) in enumerate(zip(ours, ref)):
        np.testing.assert_array_equal(a, ra, err_msg=f"step {s} matrix")
        np.testing.assert_array_equal(r, rr, err_msg=f"step {s} rhs")


def test_mos1_zero_rd_beside_rsh_is_refused():
    from neospice_b200 import _lib as L
    nl = _driven(70, {"RSH": 40.0, "RD": 0.0})
    with pytest.raises(L.NsgError):
        nl.build()
