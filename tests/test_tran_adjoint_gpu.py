"""GPU transient adjoint: gradients of a squared-error loss on the far-end
voltage of an RC tree driven by a level-1 CMOS inverter, with respect to
every R and C, the DC supply and the drivers' W, L and VTO (also with the
drivers' Meyer gate charge, overlap and junction capacitances; and on
diode-RC transients with diode charge, every R and C), against central finite
differences (h = 1e-6 relative) of the same discrete transient (the recorded
timepoints and integration formulas, Newton to reltol 1e-9) to 1e-6
relative, wherever the difference quotient resolves the gradient: the loss
itself carries a rounding floor of about 5e-12 L (LU rounding of the
perturbed solves), so the quotient's error floor 5e-12 L / (2 h) is allowed
on top; checkpoint spacing does not change the result."""
import numpy as np
import pytest
import torch

from neospice_b200 import _lib as L
from neospice_b200 import workloads as W
from neospice_b200.circuit import TranBatch

pytestmark = pytest.mark.gpu
TIGHT = dict(reltol=1e-9, vntol=1e-12, abstol=1e-15, max_iter=200)


def setup(nodes, seed, tstep=1e-12, tstop=3e-10, count=1, cards=None):
    nls = [W.rc_tree_driven(np.random.default_rng([seed, k]), nodes) for k in range(count)]
    for nl in nls:
        for name, extra in (cards or {}).items():
            nl.models[name][1].update(extra)
    far = nodes - 1
    b = TranBatch([nl.build() for nl in nls], tstep, tstop, np.array([far], np.int32),
                  max_points=20000)
    b.record(True)
    b.run()
    res = b.results()
    assert all(r["status"] == 0 for r in res)
    # a synthetic target: the recorded far-end waveform, scaled and shifted
    tg = np.zeros(count * b.max_points)
    for i, r in enumerate(res):
        v = r["values"][:, 0]
        tg[i * b.max_points:i * b.max_points + len(v)] = 0.97 * v + 0.01
    b.set_adjoint_options(**TIGHT)
    return nls, b, torch.from_numpy(tg).cuda(), [far] * count


def loss_at(b, probes, targets, p_dc, p_tr):
    _, loss, st = b.adjoint(probes, targets, 1.0, 16, p_dc, p_tr)
    torch.cuda.synchronize()
    assert int(st.abs().sum()) == 0
    return loss.cpu().numpy()


def check_against_fd(nls, b, tg, probes, floor_rel=5e-12, h_rel=1e-6, resolved_below=1e-8):
    """Every R and C (first eight of each), the DC sources and each MOSFET's
    W, L and VTO against central differences with step h_rel relative;
    returns the worst relative error among the quotients whose rounding
    floor is below resolved_below |fd|, and their number."""
    off, pdc, ptr = b.params()
    g, loss, st = b.adjoint(probes, tg, 1.0, 16)
    torch.cuda.synchronize()
    assert int(st.abs().sum()) == 0 and float(loss[0]) > 0
    g = g.cpu().numpy()
    nl = nls[0]
    starts, at = [], 0
    sizes = {"R": 1, "C": 2, "V": 1, "I": 1, "VPULSE": 7, "IPULSE": 7, "D": 15, "M": 43}
    for d in nl.devices:
        starts.append((d[0], at))
        at += sizes[d[0]]
    idx = [s for k, s in starts if k == "R"][:8] + [s for k, s in starts if k == "C"][:8]
    idx += [s for k, s in starts if k in ("V", "I")]  # DC sources (VDD)
    for k, s in starts:
        if k == "M":
            idx += [s + 0, s + 1, s + 2]  # W, L, VTO
    worst, resolved = 0.0, 0
    for i in idx:
        h = abs(pdc[i]) * h_rel
        lo_dc, hi_dc, lo_tr, hi_tr = pdc.copy(), pdc.copy(), ptr.copy(), ptr.copy()
        hi_dc[i] += h
        hi_tr[i] += h
        lo_dc[i] -= h
        lo_tr[i] -= h
        dev = lambda a: torch.from_numpy(a).cuda()
        lp = loss_at(b, probes, tg, dev(hi_dc), dev(hi_tr))[0]
        lm = loss_at(b, probes, tg, dev(lo_dc), dev(lo_tr))[0]
        fd = (lp - lm) / (2 * h)
        floor = floor_rel * float(loss[0]) / (2 * h)
        assert abs(g[i] - fd) <= 1e-6 * abs(fd) + floor, (i, g[i], fd, floor)
        if floor < resolved_below * abs(fd):  # well resolved: the adjoint to 1e-6
            worst = max(worst, abs(g[i] - fd) / abs(fd))
            resolved += 1
    return worst, resolved


def test_tran_adjoint_matches_central_differences():
    nls, b, tg, probes = setup(24, 81)
    assert check_against_fd(nls, b, tg, probes)[0] < 1e-6


MEYER = {"TOX": 1e-6, "CGSO": 2e-11, "CGDO": 2e-11, "CGBO": 1e-11}
MEYER_STRONG = {"TOX": 2e-8, "CGSO": 4e-10, "CGDO": 4e-10, "CGBO": 2e-10}
JUNCTION = {"CBD": 5e-15, "CBS": 4e-15, "GAMMA": 0.4}


@pytest.mark.parametrize("extra,min_resolved", [("meyer", 6), ("meyer+junction", 6),
                                                ("strong+junction", 0), ("meyer+series", 6)])
def test_tran_adjoint_with_mos_charge(extra, min_resolved):
    """The drivers carry Meyer gate charge (TOX) with overlap capacitances,
    and bulk-junction charge with body effect: the adjoint's charge units
    and the Meyer terms of the step Jacobian against central differences for
    every R, C, the supply and both drivers' W, L, VTO.  The quotients use
    h = 1e-5 relative: with the Meyer capacitances' kinks the loss curves
    enough that the truncation error is about 2e-6 at h = 1e-4 and falls as
    h^2 (2e-8 at 1e-5), while the rounding floor stays 5e-12 L / 2h.  With
    moderate oxide and overlap capacitance the six W / L / VTO gradients are
    resolved (floor below 1e-7 |fd|) and must be within 1e-6; at TOX = 20 nm
    (the gate-drain charge dominates the output and the loss is small) each
    gradient is checked against its floor only.  With RD / RS the channel
    and the charges sit on the internal drain' and source' nodes."""
    card = dict(MEYER_STRONG if extra.startswith("strong") else MEYER)
    if extra.endswith("junction"):
        card.update(JUNCTION)
    if extra.endswith("series"):  # drain' / source' internal nodes carry the charges
        card.update({"RD": 25.0, "RS": 10.0})
    nls, b, tg, probes = setup(12, 84, cards={"nch": card, "pch": card})
    worst, resolved = check_against_fd(nls, b, tg, probes, h_rel=1e-5, resolved_below=1e-7)
    assert resolved >= min_resolved and worst < 1e-6, (resolved, worst)


def test_tran_adjoint_checkpoint_spacing_and_batching():
    """The same gradients with checkpoints every 1, 7 and 64 steps, and for a
    circuit alone or inside a batch."""
    nls, b, tg, probes = setup(16, 82, count=3)
    outs = []
    for every in (1, 7, 64):
        g, loss, st = b.adjoint(probes, tg, 1.0, every)
        torch.cuda.synchronize()
        assert int(st.abs().sum()) == 0
        outs.append((g.cpu().numpy(), loss.cpu().numpy()))
    for g, l in outs[1:]:
        np.testing.assert_allclose(g, outs[0][0], rtol=1e-12, atol=1e-30)
        np.testing.assert_array_equal(l, outs[0][1])


def test_tran_adjoint_requires_recording_and_rejects_bsim4():
    nl = W.rc_tree_driven(np.random.default_rng(3), 6)
    b = TranBatch([nl.build()], 1e-12, 1e-10, np.array([5], np.int32), max_points=5000)
    b.run()
    tg = torch.zeros(5000, dtype=torch.float64, device="cuda")
    with pytest.raises(L.NsgError):
        b.adjoint([5], tg)
    for name in ("nch", "pch"):  # BSIM4v7 drivers: not covered
        nl.models[name] = (nl.models[name][0], {"LEVEL": 14})
    b2 = TranBatch([nl.build()], 1e-12, 1e-10, np.array([5], np.int32), max_points=5000)
    b2.record(True)
    b2.run()
    assert b2.results()[0]["status"] == 0
    with pytest.raises(L.NsgError, match="BSIM4v7"):
        b2.adjoint([5], tg)


def test_tran_loss_autograd_function():
    """tran_loss's backward is the adjoint's gradient, scaled per instance by
    the incoming gradient of each instance's loss."""
    from neospice_b200.autodiff import tran_loss
    nls, b, tg, probes = setup(16, 83, count=2)
    _, pdc, _ = b.params()
    p = torch.from_numpy(pdc).cuda().requires_grad_(True)
    loss = tran_loss(b, probes, tg, p, every=8)
    (2.0 * loss[0] + 3.0 * loss[1]).backward()
    g, l_ref, st = b.adjoint(probes, tg, 1.0, 8)
    torch.cuda.synchronize()
    assert int(st.abs().sum()) == 0
    assert torch.equal(loss.detach(), l_ref)
    off, _, _ = b.params()
    scale = torch.repeat_interleave(torch.tensor([2.0, 3.0], dtype=torch.float64, device="cuda"),
                                    torch.from_numpy(np.diff(off)).cuda())
    assert torch.equal(p.grad, g * scale)
    assert float(p.grad.abs().sum()) > 0
    assert torch.equal(tran_loss(b, probes, tg, every=8), l_ref)


@pytest.mark.parametrize("case", [0, 2, 3])
def test_tran_adjoint_with_diode_charge(case):
    """Diodes with depletion and transit-time charge (the reference's diode
    transients: a half-wave rectifier into an RC load and seeded diode-RC
    networks across the FC*VJ knee): gradients with respect to every R and C
    against central differences of the same discrete transient, as above.
    The loss of a replay through a strongly conducting diode with 5 ns
    transit time carries the Newton tolerance of the replays (reltol 1e-9)
    rather than only LU rounding: its central quotients move by a few 1e-6
    between h = 1e-5 and 1e-7, so the floor here is 1e-10 L / (2h)."""
    import pathlib
    import golden_cases
    g = golden_cases.load_transients(str(pathlib.Path(__file__).resolve().parent / "golden" /
                                         "tran_diode.npz"))[case]
    nl = g["netlist"]
    probe = nl.num_nodes - 1
    b = TranBatch([nl.build()], float(g["tstep"]), float(g["tstop"]),
                  np.array([probe], np.int32), max_points=20000)
    b.record(True)
    b.run()
    r = b.results()[0]
    assert r["status"] == 0
    tg = np.zeros(b.max_points)
    v = r["values"][:, 0]
    tg[:len(v)] = 0.97 * v + 0.01
    tg = torch.from_numpy(tg).cuda()
    b.set_adjoint_options(**TIGHT)
    _, pdc, ptr = b.params()
    grads, loss, st = b.adjoint([probe], tg, 1.0, 16)
    torch.cuda.synchronize()
    assert int(st.abs().sum()) == 0 and float(loss[0]) > 0
    grads = grads.cpu().numpy()
    sizes = {"R": 1, "C": 2, "V": 1, "I": 1, "VPULSE": 7, "IPULSE": 7, "D": 15, "M": 43}
    idx, at = [], 0
    for d in nl.devices:
        if d[0] in ("R", "C"):
            idx.append(at)
        at += sizes[d[0]]
    dev = lambda a: torch.from_numpy(a).cuda()
    for i in idx:
        h = abs(pdc[i]) * 1e-6
        hi_dc, lo_dc, hi_tr, lo_tr = pdc.copy(), pdc.copy(), ptr.copy(), ptr.copy()
        hi_dc[i] += h
        hi_tr[i] += h
        lo_dc[i] -= h
        lo_tr[i] -= h
        lp = loss_at(b, [probe], tg, dev(hi_dc), dev(hi_tr))[0]
        lm = loss_at(b, [probe], tg, dev(lo_dc), dev(lo_tr))[0]
        fd = (lp - lm) / (2 * h)
        floor = 1e-10 * float(loss[0]) / (2 * h)
        assert abs(grads[i] - fd) <= 1e-6 * abs(fd) + floor, (case, i, grads[i], fd, floor)
