"""Level-1 MOSFETs with drain / source series resistance (RD, RS, RSH: the
internal drain' and source' nodes) on the GPU against the reference, run
here through the oracle on the same netlists: inverter-driven RC trees and
seeded MOS networks.  DC: solutions to 1e-9 relative with equal Newton
iteration counts.  Transient: identical timepoints, node voltages to 1e-9
relative, equal iteration and rejection counts."""
import numpy as np
import pytest
import torch

import netlists
import oracle
from neospice_b200 import workloads as W
from neospice_b200.circuit import DcBatch, TranBatch

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.have_ref(), reason="reference library not built")]

CARDS = [{"RD": 25.0, "RS": 10.0}, {"RSH": 40.0}, {"RD": 150.0, "TOX": 1e-6, "CBD": 5e-15},
         {"RS": 300.0}]


def _networks():
    out = []
    for k, extra in enumerate(CARDS):
        nl = W.mos_network(np.random.default_rng([81, k]), 8)
        for _, card in nl.models.values():
            card.update(extra)
        out.append(nl)
    return out


def test_series_resistance_dc_matches_reference():
    nls = _networks()
    refs = [oracle.ref_sim(netlists.ref_desc(nl), 0) for nl in nls]
    batch = DcBatch([nl.build() for nl in nls], symbolic=DcBatch.PER_INSTANCE)
    sols, status, iters = batch.run()
    torch.cuda.synchronize()
    status = status.cpu().numpy()
    iters = iters.cpu().numpy()
    for k, (s, (_, vals, info)) in enumerate(zip(batch.split(sols), refs)):
        assert status[k] == 0, (k, status[k])
        assert len(s) == vals.shape[1] > nls[k].num_nodes  # internal nodes present
        np.testing.assert_allclose(s, vals[0], rtol=1e-9, atol=1e-12, err_msg=f"case {k}")
        assert iters[k] == info["iterations"], (k, iters[k], info["iterations"])


def test_series_resistance_transient_matches_reference():
    nls = []
    for k, extra in enumerate(CARDS):
        nl = W.rc_tree_driven(np.random.default_rng([82, k]), 8)
        for name in ("nch", "pch"):
            nl.models[name][1].update(extra)
        nls.append(nl)
    tstep, tstop = 1e-12, 3e-10
    refs = [oracle.ref_sim(netlists.ref_desc(nl), 1, tstep, tstop) for nl in nls]
    probes = np.arange(8, dtype=np.int32)
    b = TranBatch([nl.build() for nl in nls], tstep, tstop, probes,
                  max_points=max(len(t) for t, _, _ in refs) + 8)
    b.run()
    for k, (r, (times, vals, info)) in enumerate(zip(b.results(), refs)):
        assert r["status"] == 0, (k, r["status"])
        assert len(r["time"]) == len(times), (k, len(r["time"]), len(times))
        np.testing.assert_allclose(r["time"], times, rtol=1e-12, atol=0, err_msg=f"case {k}")
        np.testing.assert_allclose(r["values"], vals[:, :8], rtol=1e-9, atol=1e-12,
                                   err_msg=f"case {k}")
        assert r["newton_iters"] == info["iterations"], (k, r["newton_iters"], info["iterations"])
        assert r["rejected"] == info["rejected"], (k, r["rejected"], info["rejected"])
