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
