"""Diodes with reverse breakdown (BV, IBV, NBV) and series resistance (RS,
an internal posPrime node) on the GPU against the reference, run here
through the oracle on the same netlists: seeded Zener clamps and
regulators whose operating points sit below, at and beyond the breakdown
knee, half of them with RS.  DC: solutions to 1e-9 relative (the GPU's exp rounds
differently from the host C library in the last bits) with equal Newton
iteration counts.  Transient (a PULSE swinging the cathode from forward
bias into breakdown, with junction capacitance and transit time):
identical timepoints, node voltages to 1e-9 relative, equal iteration and
rejection counts."""
import numpy as np
import pytest
import torch

import netlists
import oracle
from neospice_b200.circuit import DcBatch, TranBatch
from neospice_b200.workloads import Netlist

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.have_ref(), reason="reference library not built")]
GND = -1


def zener(rng, transient=False, rs=False):
    """Source -> R -> node 1, a diode from ground (anode) to node 1 (cathode,
    reverse biased when node 1 is positive), a load resistor on node 1; with
    rs, the diode has a series resistance."""
    bv = float(rng.uniform(2.5, 12.0))
    n = float(rng.uniform(1.0, 1.5))
    card = [float(10 ** rng.uniform(-15, -12)), n,
            float(rng.uniform(0.5e-12, 5e-12)) if transient else 0.0, 0.8, 0.4, 0.5,
            float(10 ** rng.uniform(-10, -8)) if transient else 0.0,
            bv, float(10 ** rng.uniform(-5, -2)), float(rng.uniform(1.0, 2.0)),
            float(10 ** rng.uniform(0, 2.5)) if rs else 0.0]
    if transient:
        src = ("VPULSE", 0, GND, -2.0, float(rng.uniform(1.2, 2.0)) * bv, 1e-9, 2e-9, 2e-9,
               4e-9, 1e-8)
    else:
        src = ("V", 0, GND, float(rng.uniform(0.2, 2.5)) * bv)
    devs = [src, ("R", 0, 1, float(10 ** rng.uniform(2, 4))),
            ("D", GND, 1, *card), ("R", 1, GND, float(10 ** rng.uniform(3, 5)))]
    return Netlist(2, devs, {})


def test_breakdown_dc_matches_reference():
    nls = [zener(np.random.default_rng([51, k]), rs=k % 2 == 1) for k in range(16)]
    refs = [oracle.ref_sim(netlists.ref_desc(nl), 0) for nl in nls]
    batch = DcBatch([nl.build() for nl in nls], symbolic=DcBatch.PER_INSTANCE)
    sols, status, iters = batch.run()
    torch.cuda.synchronize()
    status = status.cpu().numpy()
    iters = iters.cpu().numpy()
    in_breakdown = 0
    for k, (nl, s, (_, vals, info)) in enumerate(zip(nls, batch.split(sols), refs)):
        assert status[k] == 0, (k, status[k])
        np.testing.assert_allclose(s, vals[0], rtol=1e-9, atol=1e-12, err_msg=f"case {k}")
        assert iters[k] == info["iterations"], (k, iters[k], info["iterations"])
        bv = nl.devices[2][10]
        in_breakdown += int(s[1] > 0.9 * bv)
    assert 3 <= in_breakdown <= 13  # both sides of the knee are exercised


def test_breakdown_transient_matches_reference():
    nls = [zener(np.random.default_rng([52, k]), transient=True, rs=k % 2 == 1)
           for k in range(4)]
    tstep, tstop = 1e-10, 2e-8
    refs = [oracle.ref_sim(netlists.ref_desc(nl), 1, tstep, tstop) for nl in nls]
    b = TranBatch([nl.build() for nl in nls], tstep, tstop, np.array([0, 1], np.int32),
                  max_points=max(len(t) for t, _, _ in refs) + 8)
    b.run()
    reached = 0
    for k, (r, (times, vals, info)) in enumerate(zip(b.results(), refs)):
        assert r["status"] == 0, (k, r["status"])
        assert len(r["time"]) == len(times), (k, len(r["time"]), len(times))
        np.testing.assert_allclose(r["time"], times, rtol=1e-12, atol=0, err_msg=f"case {k}")
        np.testing.assert_allclose(r["values"], vals[:, :2], rtol=1e-9, atol=1e-12,
                                   err_msg=f"case {k}")
        assert r["newton_iters"] == info["iterations"], (k, r["newton_iters"], info["iterations"])
        assert r["rejected"] == info["rejected"], (k, r["rejected"], info["rejected"])
        reached += int(r["values"][:, 1].max() > 0.9 * nls[k].devices[2][10])
    assert reached >= 2  # the cathode reaches the breakdown region during the pulse
