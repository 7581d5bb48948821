"""GPU parity of the batched transient against the reference's
solve_transient (tests/golden/tran_rc.npz, made by the reference itself):
the same timepoints, node voltages within 1e-9 relative / 1e-12 absolute,
the same Newton iteration and rejected-step counts.  tests/golden/tran_diode.npz
holds the same record for diodes with junction capacitance and transit
time."""
import pathlib

import numpy as np
import pytest

import golden_cases
from neospice_b200.circuit import TranBatch

pytestmark = pytest.mark.gpu
CASES = golden_cases.load_transients()
RTOL, ATOL = 1e-9, 1e-12


def _run(cases):
    out = []
    # circuits sharing (tstep, tstop) run as one batch
    groups = {}
    for k, g in enumerate(cases):
        groups.setdefault((float(g["tstep"]), float(g["tstop"])), []).append(k)
    res = [None] * len(cases)
    for (tstep, tstop), ks in groups.items():
        circuits = [cases[k]["netlist"].build() for k in ks]
        nn = max(cases[k]["netlist"].num_nodes for k in ks)
        # probe every node of the largest circuit; smaller circuits probe
        # their own nodes (probe indices must exist in every circuit)
        nmin = min(cases[k]["netlist"].num_nodes for k in ks)
        probes = np.arange(nmin, dtype=np.int32)
        b = TranBatch(circuits, tstep, tstop, probes, max_points=max(len(cases[k]["times"]) for k in ks) + 8)
        b.run()
        for k, r in zip(ks, b.results()):
            res[k] = (r, nmin)
        del nn
    return res


def _check(cases):
    res = _run(cases)
    for k, (g, (r, nprobe)) in enumerate(zip(cases, res)):
        assert r["status"] == 0, (k, r)
        assert len(r["time"]) == len(g["times"]), (k, len(r["time"]), len(g["times"]))
        np.testing.assert_allclose(r["time"], g["times"], rtol=1e-12, atol=0, err_msg=f"case {k}")
        np.testing.assert_allclose(r["values"], g["values"][:, :nprobe], rtol=RTOL, atol=ATOL,
                                   err_msg=f"case {k}")
        assert r["newton_iters"] == int(g["iterations"]), (k, r["newton_iters"], int(g["iterations"]))
        assert r["rejected"] == int(g["rejected"]), (k, r["rejected"], int(g["rejected"]))


def test_transient_matches_reference():
    _check(CASES)


def test_transient_diodes_match_reference():
    """DIOload's charge storage (depletion below and above the FC*VJ knee,
    diffusion charge TT*Id), its predictor and the truncation error of the
    junction charge: timepoints, waveforms and counts as the reference's."""
    _check(golden_cases.load_transients(
        pathlib.Path(__file__).resolve().parent / "golden" / "tran_diode.npz"))


def test_transient_single_instances_match_batch():
    """Each circuit alone gives the same waveform as inside a batch."""
    g = CASES[4]
    nn = g["netlist"].num_nodes
    probes = np.arange(nn, dtype=np.int32)
    one = TranBatch([g["netlist"].build()], float(g["tstep"]), float(g["tstop"]), probes,
                    max_points=len(g["times"]) + 8)
    one.run()
    r1 = one.results()[0]
    many = TranBatch([c["netlist"].build() for c in [g] * 5], float(g["tstep"]), float(g["tstop"]),
                     probes, max_points=len(g["times"]) + 8)
    many.run()
    for r in many.results():
        np.testing.assert_array_equal(r["time"], r1["time"])
        np.testing.assert_array_equal(r["values"], r1["values"])


def test_transient_max_points_truncates():
    g = CASES[0]
    b = TranBatch([g["netlist"].build()], float(g["tstep"]), float(g["tstop"]),
                  np.arange(2, dtype=np.int32), max_points=10)
    b.run()
    r = b.results()[0]
    assert r["status"] == 0
    assert len(r["time"]) == 10
    np.testing.assert_allclose(r["time"], g["times"][:10], rtol=1e-12)
