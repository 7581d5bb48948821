"""Circuits at temperatures other than TNOM (the reference's options.temp,
which `.step TEMP` sets): DIOtemp's saturation current, junction values,
breakdown voltage and vt, and MOS1temp's threshold, transconductance,
junction and saturation values at the device temperature.  The first DC
matrix and rhs, and for level-1 MOSFETs the whole transient-mode load
sequence, equal the reference's bit for bit at -40, 85 and 150 C."""
import numpy as np
import pytest

import netlists
import oracle
from neospice_b200 import _lib as L
from neospice_b200 import workloads as W
from neospice_b200.workloads import Netlist
from test_bsim4 import _eval_sequence

needs_ref = pytest.mark.skipif(not oracle.have_ref(), reason="reference library not built")
TEMPS = [233.15, 358.15, 423.15]
NAN = float("nan")


def diode_net(seed):
    rng = np.random.default_rng(seed)
    devs = [("V", 0, -1, 5.0)]
    for i in range(1, 5):
        devs.append(("R", int(rng.integers(0, i)), i, float(10 ** rng.uniform(1, 4))))
        bv = float(rng.uniform(3, 8)) if i % 2 else NAN
        rs = float(rng.uniform(1, 30)) if i > 2 else 0.0
        devs.append(("D", i, -1, float(10 ** rng.uniform(-15, -12)), float(rng.uniform(1, 1.5)),
                     1e-12, 0.8, 0.4, 0.5, 1e-9, bv, 1e-3, 1.2, rs))
    return Netlist(5, devs, {})


def mos_net(seed):
    nl = W.rc_tree_driven(np.random.default_rng(seed), 6)
    extra = {"TOX": 2e-8, "CGSO": 4e-10, "CGDO": 4e-10, "CBD": 5e-15, "CBS": 4e-15,
             "GAMMA": 0.4, "LAMBDA": 0.02, "RD": 20.0}
    for name in ("nch", "pch"):
        nl.models[name][1].update(extra)
    return nl


def _initjct_equal(nl, temp):
    c = nl.build(temp=temp)
    cp, ri = c.pattern()
    a, rhs = c.initial_matrix(1e-12)
    rcp, rri, ra, rrhs = oracle.ref_sim_initjct(netlists.ref_desc(nl, {"temp": temp}))
    np.testing.assert_array_equal(cp, rcp)
    np.testing.assert_array_equal(ri, rri)
    np.testing.assert_array_equal(a, ra)
    np.testing.assert_array_equal(rhs, rrhs)


@needs_ref
@pytest.mark.parametrize("temp", TEMPS)
def test_diodes_at_temperature_bitwise(temp):
    for seed in (1, 2, 3):
        _initjct_equal(diode_net(seed), temp)


@needs_ref
@pytest.mark.parametrize("temp", TEMPS)
def test_mos1_at_temperature_bitwise(temp):
    nl = mos_net(5)
    _initjct_equal(nl, temp)
    ours, ref = _eval_sequence(nl, np.random.default_rng([47, int(temp)]), temp=temp)
    for s, ((a, r), (ra, rr)) in enumerate(zip(ours, ref)):
        np.testing.assert_array_equal(a, ra, err_msg=f"step {s} matrix")
        np.testing.assert_array_equal(r, rr, err_msg=f"step {s} rhs")


def test_temperature_must_precede_devices_and_bsim4_stays_at_tnom():
    from neospice_b200.circuit import Circuit
    c = Circuit(2)
    c.R(0, 1, 1e3)
    with pytest.raises(L.NsgError):
        c.set_temperature(350.0)
    c2 = Circuit(2)
    with pytest.raises(L.NsgError):
        c2.set_temperature(-5.0)
    c2.set_temperature(350.0)
    m = c2.model_bsim4("nmos")
    with pytest.raises(L.NsgError):
        c2.M4(0, 1, -1, -1, m)
