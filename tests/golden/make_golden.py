"""Generate tests/golden/solver_cases.npz from the reference itself.

Runs the reference's own code (oracle/_ref/libnsref.so, built from the
reference sources by oracle/Makefile).

solver_cases.npz: on seeded matrices, per case the CSC pattern and values,
the exported symbolic structure after NeoSolver::numeric (pivot permutations,
LU pattern, slot map), the factored values, the values after
NeoSolver::refactorize on perturbed values, and the solutions of solve and
solve_transposed.

tran_rc.npz: seeded RC netlists, CMOS inverter chains and MOS networks
(neospice_b200.workloads) with PULSE and PWL sources, per case the device
list and model cards (JSON), tstep/tstop, and the
reference's solve_transient output: every timepoint, all node voltages,
total Newton iterations and rejected steps.

tran_diode.npz: the same record for diode circuits with junction capacitance
and transit time (rectifier, reverse recovery, seeded diode-RC networks,
DIOtemp's grading and junction-potential limits).

dc_aids.npz: the reference's source_stepping, gain_stepping and
pseudo_transient run alone (as solve_dc runs them after the earlier aids fail) on inverter chains,
MOS networks, diode-loaded resistor grids and inverter rings; per case the
netlist, the aid, the solution, the Newton iterations and whether it
converged.

step_tran.npz: the same for `.tran` (every step's timepoints and node
voltages) on an RC ladder and a diode with junction charge.

step_dc.npz: the reference's `.op` under `.step` of a source
(Simulator::run_step_sweep) on seeded diode-loaded resistor grids; per case
the netlist, the stepped parameter's index, start/stop/step, the step
values, every step's node voltages and Newton iterations.

mos_dc.npz: CMOS inverter chains and seeded MOS networks, per case the
netlist (JSON) and the reference's solve_dc operating point, Newton
iteration count and convergence method (0 direct, 1 gmin stepping).

sens_dc.npz: seeded resistor and MOS networks, per case the netlist, the
output node and the reference's solve_sens of v(output) (finite-difference
sensitivities to every resistance, voltage source and current source).

mesh_dc.npz: seeded diode-clamped meshes (neospice_b200.workloads), per case
the mesh, the reference's first-iteration matrix and rhs, and its DC
operating point (solve_dc) with the Newton iteration count.

linear_large.npz: linear resistor networks, RC ladders and trees and RC
power grids of 256 or more unknowns (the reference's AMD-LU range), per case
the netlist and the reference's DC operating point or transient output with
its Newton iteration and rejection counts.

amd_cases.npz: the reference's AmdLuSolver (amd_lu_solver.cpp) on the
known-answer matrices of its unit tests (restated from their formulas),
seeded random matrices and resistor meshes with voltage-source branches; per
case the CSC pattern, values and diag_gmin, the factor after numeric() (AMD
order q, row pivots pinv, L and U exactly as the solver stores them), the
factor after refactorize() on second values (with the replay / fallback
counters), a right-hand side and the reference's solution.

bsim4.npz: BSIM4v7 (LEVEL=14) circuits.  DC cases: the reference's own
unit-test operating point (tests/unit/test_bsim4v7_ucb_load.cpp: NMOS
VTH0=0.4 U0=0.04 TOXE=2e-9, W/L = 1u/100n at VDS 0.1, VGS 0.8), NMOS and
PMOS bias points, and inverter / NAND circuits with per-device TOXE and
DELVTO; per case the netlist, solve_dc's solution, Newton iterations and
method.  Transient cases: a BSIM4v7 inverter chain under a PULSE, and
Monte Carlo instances of the 200-MOSFET ring-oscillator + NAND-chain
circuit (neospice_b200.workloads.bsim4_ring_nand) over 1 ns; per case the
timepoints, the voltages at the recorded probe nodes, the Newton
iterations and rejected steps.

Run from the repository root: ``python tests/golden/make_golden.py``.
"""
from __future__ import annotations

import pathlib
import sys

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

import oracle  # noqa: E402
from matrices import banded, mna_mesh, random_matrix  # noqa: E402


def cases():
    rng = np.random.default_rng(20261203)
    out = []
    for k in range(36):
        n = int(rng.integers(2, 48))
        out.append(random_matrix(rng, n, float(rng.uniform(0.05, 0.4)), diag_dominant=(k % 2 == 0),
                                 zero_diag_frac=float(rng.uniform(0.0, 0.4)), integer=(k % 5 == 0)))
    for side, nv in ((3, 1), (6, 2), (9, 3), (12, 1)):
        out.append(mna_mesh(rng, side, nv))
    out.append(banded(100, 7, seed=1))
    return out


def main():
    oracle.build()
    rng = np.random.default_rng(7)
    rec = {}
    kept = 0
    for (n, cp, ri, vals) in cases():
        rs = oracle.RefSolver(n, cp, ri)
        if rs.numeric(vals) != 0:
            continue
        st, lu0 = rs.export()
        vals2 = vals * np.exp(0.05 * rng.standard_normal(len(vals)))
        rc = rs.refactorize(vals2)
        _, lu1 = rs.export()
        b = rng.standard_normal(n)
        x = rs.solve(b)
        xt = rs.solve(b, transposed=True)
        p = f"c{kept:02d}_"
        rec.update({p + "n": np.int32(n), p + "col_ptr": cp, p + "row_idx": ri, p + "vals": vals,
                    p + "vals2": vals2, p + "refactor_rc": np.int32(rc),
                    p + "int_to_ext_row": st.int_to_ext_row, p + "int_to_ext_col": st.int_to_ext_col,
                    p + "elem_row": st.elem_row, p + "elem_col": st.elem_col,
                    p + "slot_to_elem": st.slot_to_elem, p + "lu_numeric": lu0,
                    p + "lu_refactor": lu1, p + "b": b, p + "x": x, p + "xt": xt})
        kept += 1
    rec["count"] = np.int32(kept)
    path = pathlib.Path(__file__).with_name("solver_cases.npz")
    np.savez_compressed(path, **rec)
    print(f"wrote {kept} cases to {path}")


def mesh_main():
    from neospice_b200 import workloads
    rec = {}
    sides = [4, 5, 7, 9, 12, 16, 16, 20]
    for k, side in enumerate(sides):
        m = workloads.diode_mesh(np.random.default_rng([77, k]), side=side)
        cp, ri, vals, rhs = oracle.ref_mesh_initjct(m)
        sol, iters, _ = oracle.ref_mesh_dc(m)
        p = f"m{k:02d}_"
        rec.update({p + "side": np.int32(side), p + "r_h": m.r_h, p + "r_v": m.r_v,
                    p + "diode_nodes": m.diode_nodes, p + "isrc_nodes": m.isrc_nodes,
                    p + "isrc_amps": m.isrc_amps, p + "col_ptr": cp, p + "row_idx": ri,
                    p + "a0": vals, p + "rhs0": rhs, p + "solution": sol,
                    p + "iterations": np.int32(iters)})
    rec["count"] = np.int32(len(sides))
    path = pathlib.Path(__file__).with_name("mesh_dc.npz")
    np.savez_compressed(path, **rec)
    print(f"wrote {len(sides)} meshes to {path}")


def tran_netlists():
    """(netlist, tstep, tstop) cases of tran_rc.npz."""
    from neospice_b200 import workloads as W
    cases = []
    for k, stages in enumerate((1, 2, 3, 5, 8, 13, 20)):
        nl = W.rc_ladder(np.random.default_rng([31, k]), stages)
        cases.append((nl, 1e-11, 4e-9))
    for k, nodes in enumerate((6, 25, 60)):
        cases.append((W.rc_tree(np.random.default_rng([32, k]), nodes), 1e-12, 3e-10))
    # Steps limited by the truncation-error estimate (one with rejections).
    for k, (stages, tstep, tstop) in enumerate(((3, 1e-10, 4e-9), (8, 2e-10, 1e-8),
                                                 (5, 1e-9, 2e-8))):
        cases.append((W.rc_ladder(np.random.default_rng([33, k]), stages), tstep, tstop))
    for k, (nodes, tstep, tstop) in enumerate(((25, 1e-11, 3e-10), (60, 2e-11, 1e-9))):
        cases.append((W.rc_tree(np.random.default_rng([34, k]), nodes), tstep, tstop))
    # CMOS inverter chains and MOS networks driven by a pulse (the 10-stage
    # chain's operating point needs gmin stepping).
    pulse = (0.0, 1.8, 0.0, 1e-10, 1e-10, 1e-9, 2e-9)
    cases.append((W.inverter_chain(3, pulse=pulse), 2e-12, 2e-9))
    cases.append((W.inverter_chain(5, pulse=pulse), 5e-12, 4e-9))
    cases.append((W.inverter_chain(10, pulse=pulse), 1e-11, 2e-9))
    cases.append((W.mos_network(np.random.default_rng([51, 0]), 6, pulse=pulse), 5e-12, 2e-9))
    cases.append((W.mos_network(np.random.default_rng([51, 1]), 9, pulse=pulse), 1e-11, 3e-9))
    # PWL current load into an RC node, a DC source through R, one capacitor
    # with an initial condition, a PULSE with default rise/fall/width/period.
    cases.append((W.Netlist(4, [
        ("V", 0, -1, 1.0), ("R", 0, 1, 100.0), ("C", 1, -1, 1e-12, 0.3),
        ("R", 1, 2, 250.0), ("C", 2, -1, 2e-12),
        ("IPWL", 2, -1, 0.0, 0.0, 1e-10, 1e-3, 3e-10, 1e-3, 3.5e-10, 0.0),
        ("VPULSE", 3, -1, 0.0, 0.5, 2e-10, 0.0, 0.0, 0.0, 0.0), ("R", 3, 2, 500.0),
        ("C", 3, 1, 5e-13)]), 1e-11, 1e-9))
    return cases


def mos_netlists():
    """DC cases of mos_dc.npz: CMOS inverter chains at several input levels
    (the longer ones need gmin stepping) and seeded MOS networks with body
    effect, channel-length modulation and oxide-derived parameters."""
    from neospice_b200 import workloads as W
    cases = []
    for stages, vin in ((1, 0.0), (2, 0.5), (3, 0.9), (4, 0.75), (5, 1.3), (8, 1.8), (12, 0.0)):
        cases.append(W.inverter_chain(stages, vin))
    for k in range(6):
        cases.append(W.mos_network(np.random.default_rng([41, k]), int(4 + 3 * k)))
    return cases


def mos_main():
    import json
    import netlists
    rec = {}
    cases = mos_netlists()
    for k, nl in enumerate(cases):
        _, v, info = oracle.ref_sim(netlists.ref_desc(nl), 0)
        p = f"d{k:02d}_"
        rec.update({p + "netlist": np.array(json.dumps([nl.num_nodes, nl.devices, nl.models])),
                    p + "solution": v[0], p + "iterations": np.int32(info["iterations"]),
                    p + "method": np.int32(info["method"])})
    rec["count"] = np.int32(len(cases))
    path = pathlib.Path(__file__).with_name("mos_dc.npz")
    np.savez_compressed(path, **rec)
    print(f"wrote {len(cases)} MOS operating points to {path}")


def aid_netlists():
    """(netlist, analysis) cases of dc_aids.npz: the reference's
    source_stepping (2), gain_stepping (3) and pseudo_transient (4) run
    alone on inverter chains, seeded MOS networks, diode-loaded resistor
    grids, and inverter rings with channel-length modulation on which the
    aids fail."""
    from neospice_b200 import workloads as W
    nets = [W.inverter_chain(s, v) for s, v in ((1, 0.0), (3, 0.9), (5, 1.3), (9, 0.0), (25, 1.8))]
    nets += [W.mos_network(np.random.default_rng([43, k]), int(5 + 3 * k)) for k in range(4)]
    nets += [W.diode_grid(np.random.default_rng([44, k]), s) for k, s in enumerate((4, 7, 10))]
    nets += [W.inverter_ring(9, 1.8, 0.05), W.inverter_ring(13, 3.3, 0.05)]
    return [(nl, an) for an in (2, 3, 4) for nl in nets]


def aid_main():
    import json
    import netlists
    rec = {}
    cases = aid_netlists()
    for k, (nl, an) in enumerate(cases):
        _, v, info = oracle.ref_sim(netlists.ref_desc(nl), an)
        p = f"a{k:02d}_"
        rec.update({p + "netlist": np.array(json.dumps([nl.num_nodes, nl.devices, nl.models])),
                    p + "aid": np.int32(an), p + "solution": v[0],
                    p + "iterations": np.int32(info["iterations"]),
                    p + "converged": np.int32(info["method"] >= 0)})
    rec["count"] = np.int32(len(cases))
    path = pathlib.Path(__file__).with_name("dc_aids.npz")
    np.savez_compressed(path, **rec)
    print(f"wrote {len(cases)} source / gain stepping and pseudo-transient runs to {path}")


def step_cases():
    """(netlist, device index, start, stop, step) cases of step_dc.npz:
    `.op` under `.step` of the supply or of a current source of seeded
    diode-loaded resistor grids, ascending, descending and with steps that
    accumulate rounding."""
    from neospice_b200 import workloads as W
    out = []
    for k, (side, sweeps) in enumerate(((5, [(0.0, 2.0, 0.25), (1.0, -1.0, -0.3)]),
                                        (8, [(0.0, 1.0, 0.1), (-0.5, 0.5, 0.0999)]),
                                        (12, [(0.2, 3.0, 0.35)]))):
        nl = W.diode_grid(np.random.default_rng([70, k]), side)
        for sw in sweeps:
            out.append((nl, 0) + sw)  # the supply is device 0
        isrc = [i for i, d in enumerate(nl.devices) if d[0] == "I"]
        if isrc:
            out.append((nl, isrc[0], 0.0, 2e-3, 5e-4))
    return out


def step_tran_cases():
    """(netlist, device index, start, stop, step, tstep, tstop) cases of
    step_tran.npz: `.tran` under `.step` of a DC supply — an RC ladder with
    a pulse elsewhere, and a diode with junction charge fed through R from
    the stepped supply and kicked by a current pulse."""
    from neospice_b200 import workloads as W
    ladder = W.Netlist(4, [
        ("V", 0, -1, 1.0), ("R", 0, 1, 500.0), ("C", 1, -1, 1e-12), ("R", 1, 2, 800.0),
        ("C", 2, -1, 2e-12), ("VPULSE", 3, -1, 0.0, 1.0, 2e-10, 1e-10, 1e-10, 5e-10, 2e-9),
        ("R", 3, 2, 1000.0)])
    diode = W.Netlist(2, [
        ("V", 0, -1, 0.5), ("R", 0, 1, 1000.0), ("C", 1, -1, 1e-12),
        ("D", 1, -1, 1e-14, 1.0, 5e-13, 0.8, 0.4, 0.5, 1e-10),
        ("IPULSE", -1, 1, 0.0, 1e-3, 2e-10, 1e-10, 1e-10, 5e-10, 2e-9)])
    return [(ladder, 0, 0.0, 2.0, 0.5, 1e-11, 2e-9), (diode, 0, 0.2, 1.0, 0.2, 1e-11, 2e-9)]


def step_main():
    import json
    import netlists
    import golden_cases
    rec = {}
    cases = step_cases()
    for k, (nl, dev, start, stop, step) in enumerate(cases):
        vals, volts, iters = oracle.ref_step_dc(netlists.ref_desc(nl), dev + 1, start, stop, step,
                                                nl.num_nodes)
        p = f"s{k:02d}_"
        rec.update({p + "netlist": np.array(json.dumps([nl.num_nodes, nl.devices, nl.models])),
                    p + "param": np.int32(golden_cases.param_starts(nl)[dev][1]),
                    p + "sweep": np.array([start, stop, step]), p + "values": vals,
                    p + "volts": volts, p + "iterations": iters})
    rec["count"] = np.int32(len(cases))
    path = pathlib.Path(__file__).with_name("step_dc.npz")
    np.savez_compressed(path, **rec)
    print(f"wrote {len(cases)} .step sweeps to {path}")
    rec = {}
    cases = step_tran_cases()
    for k, (nl, dev, start, stop, step, tstep, tstop) in enumerate(cases):
        runs, iters = oracle.ref_step_tran(netlists.ref_desc(nl), dev + 1, start, stop, step,
                                           tstep, tstop, nl.num_nodes)
        p = f"s{k:02d}_"
        rec.update({p + "netlist": np.array(json.dumps([nl.num_nodes, nl.devices, nl.models])),
                    p + "param": np.int32(golden_cases.param_starts(nl)[dev][1]),
                    p + "sweep": np.array([start, stop, step]),
                    p + "tran": np.array([tstep, tstop]), p + "iterations": iters,
                    p + "nsteps": np.int32(len(runs))})
        for q, (t, v) in enumerate(runs):
            rec[p + f"t{q:02d}"] = t
            rec[p + f"v{q:02d}"] = v
    rec["count"] = np.int32(len(cases))
    path = pathlib.Path(__file__).with_name("step_tran.npz")
    np.savez_compressed(path, **rec)
    print(f"wrote {len(cases)} .step transients to {path}")


def sens_netlists():
    """(netlist, output node) cases of sens_dc.npz: linear resistor networks
    with voltage and current sources, and seeded MOS networks."""
    from neospice_b200 import workloads as W
    cases = []
    for k, nodes in enumerate((6, 12, 25)):
        cases.append((W.resistor_network(np.random.default_rng([61, k]), nodes), nodes - 1))
    for k in range(3):
        nl = W.mos_network(np.random.default_rng([62, k]), 6 + 3 * k)
        cases.append((nl, nl.num_nodes - 1))
    return cases


def sens_main():
    import json
    import netlists
    rec = {}
    cases = sens_netlists()
    for k, (nl, out) in enumerate(cases):
        sens, val = oracle.ref_sim_sens(netlists.ref_desc(nl), out)
        p = f"s{k:02d}_"
        rec.update({p + "netlist": np.array(json.dumps([nl.num_nodes, nl.devices, nl.models])),
                    p + "output": np.int32(out), p + "sens": sens, p + "value": np.float64(val)})
    rec["count"] = np.int32(len(cases))
    path = pathlib.Path(__file__).with_name("sens_dc.npz")
    np.savez_compressed(path, **rec)
    print(f"wrote {len(cases)} sensitivity cases to {path}")


def tran_diode_netlists():
    """(netlist, tstep, tstop) cases of tran_diode.npz: diodes with junction
    capacitance and transit time in the transient — a half-wave rectifier,
    reverse recovery of a clamp, seeded diode-RC networks (forward bias past
    the FC*VJ knee, reverse bias), a charge-free diode, and the grading (M >
    0.9) and junction-potential (FC*VJ > 1) limits of DIOtemp."""
    from neospice_b200 import workloads as W
    cases = []
    cases.append((W.Netlist(3, [
        ("VPULSE", 0, -1, 0.0, 2.0, 1e-9, 1e-9, 1e-9, 5e-9, 12e-9), ("R", 0, 1, 100.0),
        ("D", 1, 2, 1e-14, 1.0, 2e-12, 0.8, 0.4, 0.5, 5e-9),
        ("R", 2, -1, 1000.0), ("C", 2, -1, 1e-11)]), 1e-10, 4e-8))
    cases.append((W.Netlist(2, [
        ("VPULSE", 0, -1, 1.0, -1.0, 5e-9, 1e-10, 1e-10, 20e-9, 40e-9), ("R", 0, 1, 50.0),
        ("D", 1, -1, 1e-14, 1.0, 1e-12, 0.7, 0.5, 0.5, 1e-8)]), 1e-10, 3e-8))
    for k, nodes in enumerate((5, 9)):
        rng = np.random.default_rng([61, k])
        dev = [("VPULSE", 0, -1, -1.0, 1.5, 1e-10, 2e-10, 2e-10, 1e-9, 3e-9)]
        for i in range(1, nodes):
            dev.append(("R", int(rng.integers(0, i)), i, float(rng.lognormal(np.log(200.0), 0.3))))
            dev.append(("C", i, -1, float(rng.lognormal(np.log(1e-13), 0.3))))
            if rng.random() < 0.6:
                a, b = (i, -1) if rng.random() < 0.5 else (-1, i)
                dev.append(("D", a, b, float(10 ** rng.uniform(-15, -13)), float(rng.uniform(1.0, 1.8)),
                            float(rng.lognormal(np.log(5e-13), 0.5)), float(rng.uniform(0.5, 1.0)),
                            float(rng.uniform(0.3, 0.6)), float(rng.uniform(0.3, 0.6)),
                            float(rng.choice([0.0, 1e-10, 1e-9]))))
        cases.append((W.Netlist(nodes, dev), 2e-11, 6e-9))
    cases.append((W.Netlist(3, [
        ("VPULSE", 0, -1, 0.0, 1.2, 0.0, 5e-10, 5e-10, 2e-9, 5e-9), ("R", 0, 1, 300.0),
        ("D", 1, -1, 1e-14, 1.0), ("R", 1, 2, 100.0), ("C", 2, -1, 2e-12)]), 2e-11, 1e-8))
    cases.append((W.Netlist(3, [
        ("VPULSE", 0, -1, -2.0, 1.0, 2e-10, 2e-10, 2e-10, 2e-9, 4e-9), ("R", 0, 1, 200.0),
        ("D", 1, -1, 1e-14, 1.0, 3e-12, 0.9, 0.95, 0.5, 2e-10),
        ("R", 1, 2, 200.0), ("D", 2, -1, 2e-14, 1.2, 1e-12, 2.5, 0.5, 0.5, 0.0),
        ("C", 2, -1, 1e-13)]), 2e-11, 8e-9))
    return cases


def tran_main(which="tran"):
    import json
    import netlists
    rec = {}
    cases = tran_netlists() if which == "tran" else tran_diode_netlists()
    for k, (nl, tstep, tstop) in enumerate(cases):
        t, v, info = oracle.ref_sim(netlists.ref_desc(nl), 1, tstep, tstop)
        p = f"t{k:02d}_"
        rec.update({p + "netlist": np.array(json.dumps([nl.num_nodes, nl.devices, nl.models])),
                    p + "tstep": np.float64(tstep), p + "tstop": np.float64(tstop),
                    p + "times": t, p + "values": v,
                    p + "iterations": np.int32(info["iterations"]),
                    p + "rejected": np.int32(info["rejected"])})
    rec["count"] = np.int32(len(cases))
    path = pathlib.Path(__file__).with_name("tran_rc.npz" if which == "tran" else "tran_diode.npz")
    np.savez_compressed(path, **rec)
    print(f"wrote {len(cases)} transients to {path}")


def linear_netlists():
    """Linear circuits of 256 or more unknowns, which the reference solves
    with its AMD-LU engine: (kind, netlist, tstep, tstop); kind 0 = DC
    operating point, 1 = transient."""
    from neospice_b200 import workloads as W
    cases = [
        (0, W.resistor_network(np.random.default_rng([61, 0]), 300), 0.0, 0.0),
        (0, W.resistor_network(np.random.default_rng([61, 1]), 700), 0.0, 0.0),
        (0, W.power_grid(np.random.default_rng([62, 0]), 20, 10, 30), 0.0, 0.0),
        (1, W.rc_ladder(np.random.default_rng([63, 0]), 300), 1e-11, 2e-9),
        (1, W.rc_tree(np.random.default_rng([64, 0]), 400), 1e-12, 3e-10),
        (1, W.power_grid(np.random.default_rng([65, 0]), 16, 8, 12, t_edge=2e-10), 1e-11, 4e-10),
    ]
    return cases


def linear_main():
    import json
    import netlists
    rec = {}
    cases = linear_netlists()
    for k, (kind, nl, tstep, tstop) in enumerate(cases):
        t, v, info = oracle.ref_sim(netlists.ref_desc(nl), kind, tstep, tstop)
        p = f"l{k:02d}_"
        rec.update({p + "kind": np.int32(kind),
                    p + "netlist": np.array(json.dumps([nl.num_nodes, nl.devices, nl.models])),
                    p + "tstep": np.float64(tstep), p + "tstop": np.float64(tstop),
                    p + "times": t, p + "values": v,
                    p + "num_vars": np.int32(info["num_vars"]),
                    p + "iterations": np.int32(info["iterations"]),
                    p + "rejected": np.int32(info["rejected"])})
        print(k, kind, info["num_vars"], info["points"], info["iterations"], f"{info['seconds']:.2f}s")
    rec["count"] = np.int32(len(cases))
    path = pathlib.Path(__file__).with_name("linear_large.npz")
    np.savez_compressed(path, **rec)
    print(f"wrote {len(cases)} linear circuits to {path}")


def _csc(n, entries):
    """CSC of {(row, col): value}, rows ascending per column."""
    keys = sorted(entries, key=lambda rc: (rc[1], rc[0]))
    cp = np.zeros(n + 1, np.int32)
    for (_, c) in keys:
        cp[c + 1] += 1
    cp = np.cumsum(cp).astype(np.int32)
    ri = np.array([r for (r, _) in keys], np.int32)
    v = np.array([entries[k] for k in keys], np.float64)
    return n, cp, ri, v


def amd_known_answer_cases():
    """The matrices of the reference's AmdLuSolver unit tests
    (tests/unit/test_amd_lu.cpp), rebuilt from their formulas: (name, n,
    entries, second entries or None, gmin, x_true or None, tol)."""
    out = []
    out.append(("dense1x1", 1, {(0, 0): 3.0}, None, 0.0, [7.0], 1e-12))
    out.append(("dense2x2", 2, {(0, 0): 2.0, (1, 0): 1.0, (0, 1): 1.0, (1, 1): 3.0}, None, 0.0,
                [1.6, 1.8], 1e-10))
    out.append(("dense8_diag_dominant", 8,
                {(i, j): (20.0 if i == j else 1.0) for i in range(8) for j in range(8)}, None,
                0.0, [i + 1.0 for i in range(8)], 1e-9))

    def tri(n, d, o):
        e = {}
        for i in range(n):
            e[(i, i)] = d
            if i > 0:
                e[(i, i - 1)] = o
            if i < n - 1:
                e[(i, i + 1)] = o
        return e
    out.append(("tridiagonal60", 60, tri(60, 4.0, -1.0), None, 0.0,
                [(i % 5) + 1.0 for i in range(60)], 1e-9))
    arrow = {(i, i): (100.0 if i == 0 else 5.0) for i in range(16)}
    for i in range(1, 16):
        arrow[(0, i)] = 1.0
        arrow[(i, 0)] = 1.0
    out.append(("arrowhead16", 16, arrow, None, 0.0, [(i % 3) + 0.5 for i in range(16)], 1e-9))
    out.append(("indefinite2x2", 2, {(0, 1): 1.0, (1, 0): 1.0, (1, 1): 1.0}, None, 0.0,
                [1.0, 1.0], 1e-12))
    z = {(0, 2): 1.0, (1, 2): 1.0, (1, 3): 1.0, (2, 0): 1.0, (2, 1): 1.0, (2, 2): 5.0,
         (3, 1): 1.0, (3, 3): 3.0}
    out.append(("zero_diag_block4", 4, z, None, 0.0, [2.0, -1.0, 0.5, 1.5], 1e-9))
    out.append(("diag_gmin2x2", 2, {(0, 0): 0.0, (1, 1): 0.0}, None, 1e-3, None, 1e-9))
    out.append(("refactorize40", 40, tri(40, 4.0, -1.0), tri(40, 8.0, -2.0), 0.0,
                [1.0] * 40, 1e-10))

    def fast(s):
        e = {}
        for i in range(50):
            e[(i, i)] = 10.0 * s + 0.1 * i
            if i > 0:
                e[(i, i - 1)] = -1.0 * s
            if i < 49:
                e[(i, i + 1)] = -1.5 * s
            if i + 2 < 50:
                e[(i, i + 2)] = -0.3 * s
        return e
    out.append(("replay50", 50, fast(1.0), fast(1.7), 0.0,
                [np.sin(0.2 * i) + 1.3 for i in range(50)], 1e-9))
    a0 = [[10, 1, 2], [1, 12, 3], [2, 1, 15]]
    a1 = [[1e-12, 1, 2], [1, 12, 3], [2, 1, 15]]
    out.append(("growth_fallback3", 3, {(i, j): float(a0[i][j]) for i in range(3) for j in range(3)},
                {(i, j): float(a1[i][j]) for i in range(3) for j in range(3)}, 0.0,
                [2.0, -1.0, 0.5], 1e-7))
    out.append(("replay_gmin30", 30, tri(30, 3.0, -1.0), tri(30, 4.2, -1.4), 1e-2, None, 1e-12))
    out.append(("structurally_singular2", 2, {(0, 0): 1.0, (1, 0): 1.0}, None, 0.0, None, 0.0))
    return out


def amd_main():
    oracle.build()
    rng = np.random.default_rng(20261204)
    cases = []
    for (name, n, e, e2, gmin, xt, tol) in amd_known_answer_cases():
        n, cp, ri, v = _csc(n, e)
        v2 = _csc(n, e2)[3] if e2 is not None else v * np.exp(0.05 * rng.standard_normal(len(v)))
        cases.append((name, n, cp, ri, v, v2, gmin, xt, tol))
    for k in range(24):
        n = int(rng.integers(3, 90))
        n, cp, ri, v = random_matrix(rng, n, float(rng.uniform(0.03, 0.3)),
                                     diag_dominant=(k % 2 == 0),
                                     zero_diag_frac=float(rng.uniform(0.0, 0.3)),
                                     integer=(k % 6 == 0))
        v2 = v * np.exp((0.5 if k % 4 == 3 else 0.05) * rng.standard_normal(len(v)))
        cases.append((f"random{k:02d}", n, cp, ri, v, v2, 0.0, None, 0.0))
    for side, nv in ((8, 1), (16, 2), (20, 3), (24, 1)):
        n, cp, ri, v = mna_mesh(rng, side, nv)
        v2 = v * np.exp(0.02 * rng.standard_normal(len(v)))
        cases.append((f"mesh{side}", n, cp, ri, v, v2, 0.0, None, 0.0))
    rec = {}
    for k, (name, n, cp, ri, v, v2, gmin, xt, tol) in enumerate(cases):
        r = oracle.RefAmdLu(n, cp, ri)
        rc = r.numeric(v, gmin)
        p = f"a{k:02d}_"
        rec.update({p + "name": np.array(name), p + "n": np.int32(n), p + "col_ptr": cp,
                    p + "row_idx": ri, p + "vals": v, p + "vals2": v2,
                    p + "gmin": np.float64(gmin), p + "numeric_rc": np.int32(rc),
                    p + "tol": np.float64(tol)})
        if xt is not None:
            rec[p + "x_true"] = np.asarray(xt, np.float64)
        if rc != 0:
            continue
        f1 = r.export()
        rec.update({p + "f1_" + key: val for key, val in f1.items()})
        rc2 = r.refactorize(v2, gmin)
        fast, fallback = r.counts()
        rec.update({p + "refactor_rc": np.int32(rc2), p + "fast": np.int32(fast),
                    p + "fallback": np.int32(fallback)})
        if rc2 != 0:
            continue
        rec.update({p + "f2_" + key: val for key, val in r.export().items()})
        b = rng.standard_normal(n)
        if xt is not None:  # the reference's check_parity: b = A(vals2) * x_true
            a = np.zeros((n, n))
            for j in range(n):
                a[ri[cp[j]:cp[j + 1]], j] = v2[cp[j]:cp[j + 1]]
            b = a @ np.asarray(xt)
        rec.update({p + "b": b, p + "x": r.solve(b)})
    rec["count"] = np.int32(len(cases))
    path = pathlib.Path(__file__).with_name("amd_cases.npz")
    np.savez_compressed(path, **rec)
    print(f"wrote {len(cases)} AMD-LU cases to {path}")


def bsim4_dc_netlists():
    """DC cases of bsim4.npz."""
    from neospice_b200 import workloads as W
    cases = []
    golden = {"LEVEL": 14, "VTH0": 0.4, "U0": 0.04, "TOXE": 2e-9}
    # the reference's unit-test operating point (Id = 5.754970e-05 in ngspice)
    cases.append(W.Netlist(3, [("V", 0, -1, 0.1), ("V", 1, -1, 0.8), ("V", 2, -1, 0.0),
                               ("M", 0, 1, -1, 2, "nmod", 1e-6, 1e-7)], {"nmod": ("nmos", golden)}))
    for vd, vg, vb in ((1.2, 1.2, 0.0), (0.05, 0.3, -0.4), (-0.3, 0.9, 0.0), (0.9, 0.2, 0.3)):
        cases.append(W.Netlist(3, [("V", 0, -1, vd), ("V", 1, -1, vg), ("V", 2, -1, vb),
                                   ("M", 0, 1, -1, 2, "n", 2e-7, 9e-8)],
                               {"n": ("nmos", {"LEVEL": 14})}))
    for vd, vg in ((-1.2, -1.2), (-0.4, -0.9), (0.2, -1.0)):
        cases.append(W.Netlist(3, [("V", 0, -1, vd), ("V", 1, -1, vg), ("V", 2, -1, 0.0),
                                   ("M", 0, 1, -1, 2, "p", 4e-7, 9e-8)],
                               {"p": ("pmos", {"LEVEL": 14, "TOXE": 2.9e-9})}))
    for k, vin in enumerate((0.0, 0.4, 0.6, 1.2)):
        rng = np.random.default_rng([61, k])
        dev = [("V", 0, -1, 1.2), ("V", 1, -1, vin)]
        models = {}
        for st in range(3):
            inp, out = 1 + st, 2 + st
            for kind, d, s_, w in (("n", out, -1, 2e-7), ("p", out, 0, 4e-7)):
                name = f"{kind}{st}"
                models[name] = ("nmos" if kind == "n" else "pmos",
                                {"LEVEL": 14, "TOXE": 3e-9 * (1 + 0.03 * (2 * rng.random() - 1))})
                dev.append(("M", d, inp, s_, s_ if s_ >= 0 else -1, name, w, 9e-8,
                            float(0.03 * rng.standard_normal())))
        cases.append(W.Netlist(5, dev, models))
    return cases


def bsim4_tran_cases():
    """Transient cases of bsim4.npz: (netlist, tstep, tstop, probe nodes)."""
    from neospice_b200 import workloads as W
    chain = W.Netlist(5, [("V", 0, -1, 1.2),
                          ("VPULSE", 1, -1, 0.0, 1.2, 2e-11, 5e-11, 5e-11, 3e-10, 8e-10)] +
                      [x for st in range(3) for x in (
                          ("M", 2 + st, 1 + st, -1, -1, "n", 2e-7, 9e-8),
                          ("M", 2 + st, 1 + st, 0, 0, "p", 4e-7, 9e-8),
                          ("C", 2 + st, -1, 2e-15))],
                      {"n": ("nmos", {"LEVEL": 14}), "p": ("pmos", {"LEVEL": 14})})
    cases = [(chain, 1e-12, 1.6e-9, list(range(5)))]
    for k in range(2):
        nl = W.bsim4_ring_nand(np.random.default_rng([31, k]))
        cases.append((nl, 1e-12, 1e-9, [0, 1, 2, 7, 13, 26, 27, 99, 100]))
    return cases


def bsim4_main():
    import json
    import netlists
    rec = {}
    dc = bsim4_dc_netlists()
    for k, nl in enumerate(dc):
        _, v, info = oracle.ref_sim(netlists.ref_desc(nl), 0)
        p = f"d{k:02d}_"
        rec.update({p + "netlist": np.array(json.dumps([nl.num_nodes, nl.devices, nl.models])),
                    p + "solution": v[0], p + "iterations": np.int32(info["iterations"]),
                    p + "method": np.int32(info["method"])})
    rec["dc_count"] = np.int32(len(dc))
    tr = bsim4_tran_cases()
    for k, (nl, tstep, tstop, probes) in enumerate(tr):
        t, v, info = oracle.ref_sim(netlists.ref_desc(nl), 1, tstep, tstop)
        p = f"t{k:02d}_"
        rec.update({p + "netlist": np.array(json.dumps([nl.num_nodes, nl.devices, nl.models])),
                    p + "tstep": np.float64(tstep), p + "tstop": np.float64(tstop),
                    p + "probes": np.array(probes, np.int32), p + "times": t,
                    p + "values": v[:, probes], p + "iterations": np.int32(info["iterations"]),
                    p + "rejected": np.int32(info["rejected"])})
    rec["tran_count"] = np.int32(len(tr))
    path = pathlib.Path(__file__).with_name("bsim4.npz")
    np.savez_compressed(path, **rec)
    print(f"wrote {len(dc)} BSIM4v7 operating points and {len(tr)} transients to {path}")


if __name__ == "__main__":
    which = sys.argv[1:] or ["solver", "mesh", "tran", "trandiode", "mos", "aids", "step", "sens",
                             "amd", "linear", "bsim4"]
    if "amd" in which:
        amd_main()
    if "linear" in which:
        linear_main()
    if "solver" in which:
        main()
    if "mesh" in which:
        mesh_main()
    if "tran" in which:
        tran_main()
    if "trandiode" in which:
        tran_main("trandiode")
    if "mos" in which:
        mos_main()
    if "aids" in which:
        aid_main()
    if "step" in which:
        step_main()
    if "sens" in which:
        sens_main()
    if "bsim4" in which:
        bsim4_main()
