""".step TEMP on the GPU against the reference: the reference's TEMP step
sets the circuit temperature to the step value + 273.15 K and re-runs the
analysis (src/api/neospice.cpp:255-256); here every step value is one
instance of one batch (neospice_b200.step).  Each step's operating point
is compared with the reference run at that temperature (solutions to 1e-9
relative, equal Newton iteration counts), and each step's transient with
identical timepoints, 1e-9 relative voltages and equal counts."""
import numpy as np
import pytest

import netlists
import oracle
from neospice_b200 import workloads as W
from neospice_b200.step import step_values, sweep_dc_temperature, sweep_transient_temperature
from test_temperature import diode_net, mos_net

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.have_ref(), reason="reference library not built")]


@pytest.mark.parametrize("which", ["diodes", "mos"])
def test_step_temp_dc_matches_reference(which):
    nl = diode_net(7) if which == "diodes" else W.mos_network(np.random.default_rng(9), 10)
    temps = step_values(-40.0, 125.0, 55.0)
    sols, status, iters = sweep_dc_temperature(lambda k: nl.build(temp=k), temps)
    assert (status == 0).all(), status
    for i, t in enumerate(temps):
        _, vals, info = oracle.ref_sim(netlists.ref_desc(nl, {"temp": t + 273.15}), 0)
        np.testing.assert_allclose(sols[i], vals[0], rtol=1e-9, atol=1e-12, err_msg=f"T={t}")
        assert iters[i] == info["iterations"], (t, iters[i], info["iterations"])
    assert not np.allclose(sols[0], sols[-1], rtol=1e-6)  # the temperature matters


def test_step_temp_transient_matches_reference():
    nl = mos_net(11)
    for name in ("nch", "pch"):  # moderate gate charge: a full transient in the reference
        nl.models[name][1].update({"TOX": 1e-6, "CGSO": 2e-11, "CGDO": 2e-11})
    temps = step_values(-40.0, 125.0, 82.5)
    tstep, tstop = 1e-12, 2e-10
    refs = [oracle.ref_sim(netlists.ref_desc(nl, {"temp": t + 273.15}), 1, tstep, tstop)
            for t in temps]
    res = sweep_transient_temperature(lambda k: nl.build(temp=k), temps, tstep, tstop,
                                      np.arange(6, dtype=np.int32),
                                      max_points=max(len(r[0]) for r in refs) + 8)
    for i, (r, (times, vals, info)) in enumerate(zip(res, refs)):
        assert r["status"] == 0, (i, r["status"])
        np.testing.assert_allclose(r["time"], times, rtol=1e-12, atol=0, err_msg=f"step {i}")
        np.testing.assert_allclose(r["values"], vals[:, :6], rtol=1e-9, atol=1e-12,
                                   err_msg=f"step {i}")
        assert r["newton_iters"] == info["iterations"], (i, r["newton_iters"], info["iterations"])
        assert r["rejected"] == info["rejected"], (i, r["rejected"], info["rejected"])
