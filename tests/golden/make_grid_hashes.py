"""Generate tests/golden/grid_full.json: the reference's AmdLuSolver on the
full-size power-grid transient matrix (neospice_b200.workloads.
power_grid_transient, 1000 x 1000 grid, n = 1,000,400), run through the
reference's own code (oracle/_ref/libnsref.so): numeric(), then
refactorize() on the same values, then solve() of a seeded right-hand side.
Records SHA-256 digests of the factor (per column: the U entries in the
reference's stored order, then L below the pivot -- the order of this
project's AMD-LU plans) and of the solution, with the reference's timings on
one core of this host.  The factor is 234 M entries; numeric() takes about
an hour.

    python tests/golden/make_grid_hashes.py [side]
"""
import hashlib
import json
import pathlib
import sys
import time

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))
sys.path.insert(0, str(HERE.parent))

import oracle  # noqa: E402
from neospice_b200 import workloads as W  # noqa: E402


def main(side=1000):
    n, cp, ri, tran = W.power_grid_transient(side)
    ref = oracle.RefAmdLu(n, cp, ri)
    t0 = time.time()
    rc = ref.numeric(tran)
    t1 = time.time()
    rc2 = ref.refactorize(tran)
    t2 = time.time()
    assert rc == 0 and rc2 == 0, (rc, rc2)
    f = ref.export()
    Up, Lp = f["Up"], f["Lp"]
    parts = []
    for k in range(n):
        parts.append(f["Ux"][Up[k]:Up[k + 1]])
        parts.append(f["Lx"][Lp[k] + 1:Lp[k + 1]])
    lu = np.concatenate(parts)
    rhs = np.random.default_rng(5).standard_normal(n)
    t3 = time.time()
    x = ref.solve(rhs)
    t4 = time.time()
    out = {"side": side, "seed": 2026, "n": n, "nnz_lu": int(len(lu)),
           "lu_sha256": hashlib.sha256(lu.tobytes()).hexdigest(),
           "x_sha256": hashlib.sha256(x.tobytes()).hexdigest(),
           "rhs": "numpy default_rng(5).standard_normal(n)",
           "reference_numeric_s": round(t1 - t0, 1),
           "reference_refactorize_s": round(t2 - t1, 1),
           "reference_solve_s": round(t4 - t3, 3)}
    (HERE / "grid_full.json").write_text(json.dumps(out, indent=1) + "\n")
    print(out)


if __name__ == "__main__":
    main(int(sys.argv[1]) if len(sys.argv) > 1 else 1000)
