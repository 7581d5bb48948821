"""The transient kernel's launch shapes give the same results.  A batch of a
few hundred instances runs one 512-thread CTA per instance; a larger batch
of small instances (n <= 128) runs 128- or 256-thread CTAs, several per SM.
Every instance of a large batch made of copies of the reference's golden
transients must still match the reference (same timepoints, 1e-9 relative
voltages, same Newton and rejection counts), and a large BSIM4 batch must
equal the same circuit run alone bit for bit."""
import pathlib

import numpy as np
import pytest
import torch

import golden_cases
from neospice_b200.circuit import TranBatch

pytestmark = pytest.mark.gpu


def _large_count():
    return 2 * torch.cuda.get_device_properties(0).multi_processor_count + 8


def _groups(cases):
    groups = {}
    for k, g in enumerate(cases):
        groups.setdefault((float(g["tstep"]), float(g["tstop"])), []).append(k)
    return groups


@pytest.mark.parametrize("which", ["rc_mos", "diode"])
def test_large_batch_matches_reference(which):
    cases = golden_cases.load_transients() if which == "rc_mos" else \
        golden_cases.load_transients(str(pathlib.Path(__file__).resolve().parent / "golden" /
                                         "tran_diode.npz"))
    count = _large_count()
    for (tstep, tstop), ks in _groups(cases).items():
        pick = [ks[i % len(ks)] for i in range(count)]
        nmin = min(cases[k]["netlist"].num_nodes for k in ks)
        b = TranBatch([cases[k]["netlist"].build() for k in pick], tstep, tstop,
                      np.arange(nmin, dtype=np.int32),
                      max_points=max(len(cases[k]["times"]) for k in ks) + 8)
        b.run()
        for i, (k, r) in enumerate(zip(pick, b.results())):
            g = cases[k]
            assert r["status"] == 0, (i, k, r["status"])
            assert len(r["time"]) == len(g["times"]), (i, k)
            np.testing.assert_allclose(r["time"], g["times"], rtol=1e-12, atol=0)
            np.testing.assert_allclose(r["values"], g["values"][:, :nmin], rtol=1e-9, atol=1e-12,
                                       err_msg=f"instance {i} (case {k})")
            assert r["newton_iters"] == int(g["iterations"]), (i, k)
            assert r["rejected"] == int(g["rejected"]), (i, k)


def test_large_bsim4_batch_equals_single_instance():
    _, tran = golden_cases.load_bsim4()
    g = tran[1]
    args = (float(g["tstep"]), float(g["tstop"]), g["probes"])
    one = TranBatch([g["netlist"].build()], *args, max_points=len(g["times"]) + 8)
    one.run()
    r1 = one.results()[0]
    count = _large_count()
    many = TranBatch([g["netlist"].build() for _ in range(count)], *args,
                     max_points=len(g["times"]) + 8)
    many.run()
    for i, r in enumerate(many.results()):
        assert r["status"] == 0, (i, r["status"])
        np.testing.assert_array_equal(r["time"], r1["time"])
        np.testing.assert_array_equal(r["values"], r1["values"])
        assert r["newton_iters"] == r1["newton_iters"]


def test_forced_shapes_identical():
    """nsg_tran_batch_set_shape: every supported shape gives the automatic
    shape's results bit for bit; unsupported shapes are refused."""
    from neospice_b200 import _lib as L
    cases = golden_cases.load_transients()
    (tstep, tstop), ks = next(iter(_groups(cases).items()))
    nmin = min(cases[k]["netlist"].num_nodes for k in ks)
    args = (tstep, tstop, np.arange(nmin, dtype=np.int32))
    mp = max(len(cases[k]["times"]) for k in ks) + 8
    out = []
    for shape in ((0, 0), (128, 8), (256, 4), (512, 2)):
        b = TranBatch([cases[k]["netlist"].build() for k in ks], *args, max_points=mp)
        b.set_shape(*shape)
        b.run()
        out.append([(r["time"], r["values"], r["newton_iters"]) for r in b.results()])
    for other in out[1:]:
        for (t0, v0, i0), (t1, v1, i1) in zip(out[0], other):
            np.testing.assert_array_equal(t1, t0)
            np.testing.assert_array_equal(v1, v0)
            assert i1 == i0
    b = TranBatch([cases[ks[0]]["netlist"].build()], *args, max_points=mp)
    with pytest.raises(L.NsgError):
        b.set_shape(256, 2)
