"""Loader for tests/golden/solver_cases.npz (made by the reference itself)."""
import pathlib

import numpy as np

import oracle

PATH = pathlib.Path(__file__).resolve().parent / "golden" / "solver_cases.npz"


def load():
    z = np.load(PATH)
    out = []
    for k in range(int(z["count"])):
        p = f"c{k:02d}_"
        d = {key[len(p):]: z[key] for key in z.files if key.startswith(p)}
        d["structure"] = oracle.Structure(int(d["n"]), d["int_to_ext_row"], d["int_to_ext_col"],
                                          d["elem_row"], d["elem_col"], d["slot_to_elem"])
        out.append(d)
    return out


MESH_PATH = pathlib.Path(__file__).resolve().parent / "golden" / "mesh_dc.npz"


def load_meshes():
    from neospice_b200.workloads import DiodeMesh
    z = np.load(MESH_PATH)
    out = []
    for k in range(int(z["count"])):
        p = f"m{k:02d}_"
        d = {key[len(p):]: z[key] for key in z.files if key.startswith(p)}
        d["mesh"] = DiodeMesh(int(d["side"]), d["r_h"], d["r_v"], d["diode_nodes"],
                              d["isrc_nodes"], d["isrc_amps"])
        out.append(d)
    return out


TRAN_PATH = pathlib.Path(__file__).resolve().parent / "golden" / "tran_rc.npz"


def load_transients(path=None):
    import json
    from neospice_b200.workloads import Netlist
    z = np.load(path or TRAN_PATH)
    out = []
    for k in range(int(z["count"])):
        p = f"t{k:02d}_"
        d = {key[len(p):]: z[key] for key in z.files if key.startswith(p)}
        nn, dev, models = json.loads(str(d["netlist"]))
        d["netlist"] = Netlist(nn, [tuple(x) for x in dev],
                               {k2: (t, p2) for k2, (t, p2) in models.items()})
        out.append(d)
    return out


AIDS_PATH = pathlib.Path(__file__).resolve().parent / "golden" / "dc_aids.npz"


def load_aids():
    """Source / gain stepping and pseudo-transient runs of the reference
    (dc_aids.npz): netlist, aid (2 source, 3 gain, 4 pseudo-transient),
    solution, iterations, converged."""
    import json
    from neospice_b200.workloads import Netlist
    z = np.load(AIDS_PATH)
    out = []
    for k in range(int(z["count"])):
        p = f"a{k:02d}_"
        d = {key[len(p):]: z[key] for key in z.files if key.startswith(p)}
        nn, dev, models = json.loads(str(d["netlist"]))
        d["netlist"] = Netlist(nn, [tuple(x) for x in dev],
                               {k2: (t, p2) for k2, (t, p2) in models.items()})
        out.append(d)
    return out


STEP_PATH = pathlib.Path(__file__).resolve().parent / "golden" / "step_dc.npz"


def load_steps():
    """`.step` sweeps of the reference (step_dc.npz): netlist, param (index
    in Circuit.params()), sweep (start, stop, step), values, volts
    [steps x nodes], iterations."""
    import json
    from neospice_b200.workloads import Netlist
    z = np.load(STEP_PATH)
    out = []
    for k in range(int(z["count"])):
        p = f"s{k:02d}_"
        d = {key[len(p):]: z[key] for key in z.files if key.startswith(p)}
        nn, dev, models = json.loads(str(d["netlist"]))
        d["netlist"] = Netlist(nn, [tuple(x) for x in dev],
                               {k2: (t, p2) for k2, (t, p2) in models.items()})
        out.append(d)
    return out


STEP_TRAN_PATH = pathlib.Path(__file__).resolve().parent / "golden" / "step_tran.npz"


def load_step_transients():
    """`.step` transients of the reference (step_tran.npz): netlist, param,
    sweep, tran (tstep, tstop), iterations per step, runs = [(times, node
    voltages)] per step."""
    import json
    from neospice_b200.workloads import Netlist
    z = np.load(STEP_TRAN_PATH)
    out = []
    for k in range(int(z["count"])):
        p = f"s{k:02d}_"
        d = {key[len(p):]: z[key] for key in z.files if key.startswith(p)}
        nn, dev, models = json.loads(str(d["netlist"]))
        d["netlist"] = Netlist(nn, [tuple(x) for x in dev],
                               {k2: (t, p2) for k2, (t, p2) in models.items()})
        d["runs"] = [(d[f"t{q:02d}"], d[f"v{q:02d}"]) for q in range(int(d["nsteps"]))]
        out.append(d)
    return out


MOS_PATH = pathlib.Path(__file__).resolve().parent / "golden" / "mos_dc.npz"


def load_mos_dc():
    import json
    from neospice_b200.workloads import Netlist
    z = np.load(MOS_PATH)
    out = []
    for k in range(int(z["count"])):
        p = f"d{k:02d}_"
        d = {key[len(p):]: z[key] for key in z.files if key.startswith(p)}
        nn, dev, models = json.loads(str(d["netlist"]))
        d["netlist"] = Netlist(nn, [tuple(x) for x in dev],
                               {k2: (t, p2) for k2, (t, p2) in models.items()})
        out.append(d)
    return out


SENS_PATH = pathlib.Path(__file__).resolve().parent / "golden" / "sens_dc.npz"


def load_sens():
    import json
    from neospice_b200.workloads import Netlist
    z = np.load(SENS_PATH)
    out = []
    for k in range(int(z["count"])):
        p = f"s{k:02d}_"
        d = {key[len(p):]: z[key] for key in z.files if key.startswith(p)}
        nn, dev, models = json.loads(str(d["netlist"]))
        d["netlist"] = Netlist(nn, [tuple(x) for x in dev],
                               {k2: (t, p2) for k2, (t, p2) in models.items()})
        out.append(d)
    return out


def param_starts(netlist):
    """(kind, first parameter index) of every device of a Netlist, in
    creation order (the layout of Circuit.params())."""
    sizes = {"R": 1, "C": 2, "V": 1, "I": 1, "VPULSE": 7, "IPULSE": 7, "D": 15, "M": 43}
    out, at = [], 0
    for d in netlist.devices:
        k = d[0]
        out.append((k, at))
        at += sizes[k] if k in sizes else len(d) - 3
    return out


AMD_PATH = pathlib.Path(__file__).resolve().parent / "golden" / "amd_cases.npz"
_FACTOR_KEYS = ("q", "pinv", "Lp", "Li", "Lx", "Up", "Ui", "Ux")


def load_amd():
    """AMD-LU cases (made by the reference's AmdLuSolver): per case the
    pattern, values, and the factors f1 (after numeric) / f2 (after
    refactorize) as dicts in the reference's storage."""
    z = np.load(AMD_PATH)
    out = []
    for k in range(int(z["count"])):
        p = f"a{k:02d}_"
        d = {key[len(p):]: z[key] for key in z.files if key.startswith(p)}
        d["name"] = str(d["name"])
        for f in ("f1", "f2"):
            if f + "_q" in d:
                d[f] = {key: d.pop(f + "_" + key) for key in _FACTOR_KEYS}
        out.append(d)
    return out


LINEAR_PATH = pathlib.Path(__file__).resolve().parent / "golden" / "linear_large.npz"


def load_linear():
    """Linear circuits of 256+ unknowns (the reference's AMD-LU range)."""
    import json
    from neospice_b200.workloads import Netlist
    z = np.load(LINEAR_PATH)
    out = []
    for k in range(int(z["count"])):
        p = f"l{k:02d}_"
        d = {key[len(p):]: z[key] for key in z.files if key.startswith(p)}
        nn, dev, models = json.loads(str(d["netlist"]))
        d["netlist"] = Netlist(nn, [tuple(x) for x in dev],
                               {k2: (t, p2) for k2, (t, p2) in models.items()})
        out.append(d)
    return out


BSIM4_PATH = pathlib.Path(__file__).resolve().parent / "golden" / "bsim4.npz"


def _netlist_of(d):
    import json
    from neospice_b200.workloads import Netlist
    nn, dev, models = json.loads(str(d["netlist"]))
    return Netlist(nn, [tuple(x) for x in dev], {k: (t, p) for k, (t, p) in models.items()})


def load_bsim4():
    """(dc cases, transient cases) of bsim4.npz, each a dict with the
    netlist rebuilt."""
    z = np.load(BSIM4_PATH)
    out = []
    for pre, count in (("d", int(z["dc_count"])), ("t", int(z["tran_count"]))):
        cases = []
        for k in range(count):
            p = f"{pre}{k:02d}_"
            d = {key[len(p):]: z[key] for key in z.files if key.startswith(p)}
            d["netlist"] = _netlist_of(d)
            cases.append(d)
        out.append(cases)
    return out[0], out[1]
