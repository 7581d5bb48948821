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

mos_dc.npz: CMOS inverter chains and seeded MOS networks, per case the
netlist (JSON) and the reference's solve_dc operating point, Newton
iteration count and convergence method (0 direct, 1 gmin stepping).

sens_dc.npz: seeded resistor and MOS networks, per case the netlist, the
output node and the reference's solve_sens of v(output) (finite-difference
sensitivities to every resistance, voltage source and current source).

mesh_dc.npz: seeded diode-clamped meshes (neospice_b200.workloads), per case
the mesh, the reference's first-iteration matrix and rhs, and its DC
operating point (solve_dc) with the Newton iteration count.

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


def tran_main():
    import json
    import netlists
    rec = {}
    cases = tran_netlists()
    for k, (nl, tstep, tstop) in enumerate(cases):
        t, v, info = oracle.ref_sim(netlists.ref_desc(nl), 1, tstep, tstop)
        p = f"t{k:02d}_"
        rec.update({p + "netlist": np.array(json.dumps([nl.num_nodes, nl.devices, nl.models])),
                    p + "tstep": np.float64(tstep), p + "tstop": np.float64(tstop),
                    p + "times": t, p + "values": v,
                    p + "iterations": np.int32(info["iterations"]),
                    p + "rejected": np.int32(info["rejected"])})
    rec["count"] = np.int32(len(cases))
    path = pathlib.Path(__file__).with_name("tran_rc.npz")
    np.savez_compressed(path, **rec)
    print(f"wrote {len(cases)} transients to {path}")


if __name__ == "__main__":
    which = sys.argv[1:] or ["solver", "mesh", "tran", "mos", "sens"]
    if "solver" in which:
        main()
    if "mesh" in which:
        mesh_main()
    if "tran" in which:
        tran_main()
    if "mos" in which:
        mos_main()
    if "sens" in which:
        sens_main()
