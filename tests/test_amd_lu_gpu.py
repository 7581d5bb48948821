"""GPU parity of the AMD-LU engine: the batched replay refactor, the
numeric() pivot check and the solves must reproduce the reference's
AmdLuSolver bit for bit (golden fixtures made by the reference itself)."""
import numpy as np
import pytest
import torch

import golden_cases
from matrices import mna_mesh, random_matrix
from neospice_b200 import _lib as L
from neospice_b200.solver import Batch, Topology

pytestmark = pytest.mark.gpu
CASES = golden_cases.load_amd()
FACTORED = [c for c in CASES if int(c["numeric_rc"]) == 0]


def packed_factor(f):
    """The reference's L/U storage in this library's column layout: per
    column the above-diagonal U entries in stored order, the pivot, then
    L(:, k) after its unit diagonal."""
    n = len(f["q"])
    out = []
    for k in range(n):
        out.append(f["Ux"][f["Up"][k]:f["Up"][k + 1]])
        out.append(f["Lx"][f["Lp"][k] + 1:f["Lp"][k + 1]])
    return np.concatenate(out) if out else np.zeros(0)


def same_pivots(f1, f2):
    return all(np.array_equal(f1[k], f2[k]) for k in ("pinv", "Lp", "Li", "Up", "Ui"))


def run(topos, vals, gmins, bs=None, check=False, schedule=0):
    batch = Batch(topos)
    batch.set_schedule(schedule)
    a = np.zeros(int(batch.value_offsets[-1]))
    for i, v in enumerate(vals):
        a[batch.value_offsets[i]:batch.value_offsets[i] + len(v)] = v
    d_a = torch.from_numpy(a).cuda()
    # one diag_gmin per call: group by value
    status = np.zeros(len(topos), np.int32)
    assert len(set(gmins)) == 1
    st, _ = batch.refactor(d_a, gmins[0], check_pivots=check)
    status[:] = st.cpu().numpy()
    lu = batch.lu_values()
    sizes = [t.info()["nnz_lu"] for t in topos]
    lus = [lu[batch.lu_offsets[i]:batch.lu_offsets[i] + sizes[i]] for i in range(len(topos))]
    xs = xts = None
    if bs is not None:
        x = np.zeros(int(batch.vector_offsets[-1]))
        for i, b in enumerate(bs):
            x[batch.vector_offsets[i]:batch.vector_offsets[i] + len(b)] = b
        d_x = torch.from_numpy(x.copy()).cuda()
        d_xt = torch.from_numpy(x.copy()).cuda()
        batch.solve(d_x)
        batch.solve_transposed(d_xt)
        hx, hxt = d_x.cpu().numpy(), d_xt.cpu().numpy()
        ns = [t.info()["n"] for t in topos]
        xs = [hx[batch.vector_offsets[i]:batch.vector_offsets[i] + ns[i]] for i in range(len(topos))]
        xts = [hxt[batch.vector_offsets[i]:batch.vector_offsets[i] + ns[i]]
               for i in range(len(topos))]
    return status, lus, xs, xts


def by_gmin(cases):
    groups = {}
    for c in cases:
        groups.setdefault(float(c["gmin"]), []).append(c)
    return groups.items()


@pytest.mark.parametrize("schedule", [0, 1, 2])
def test_numeric_values_match_reference(schedule):
    """numeric() on the ordering values: the pivot check passes and the
    factor equals AmdLuSolver::factor_'s, bit for bit."""
    for gmin, cases in by_gmin(FACTORED):
        topos = [Topology.order(int(c["n"]), c["col_ptr"], c["row_idx"], c["vals"], gmin,
                                solver="amdlu") for c in cases]
        st, lus, _, _ = run(topos, [c["vals"] for c in cases], [gmin] * len(cases),
                            check=True, schedule=schedule)
        for c, s, lu in zip(cases, st, lus):
            assert s == 0, c["name"]
            np.testing.assert_array_equal(lu, packed_factor(c["f1"]), err_msg=c["name"])


@pytest.mark.parametrize("schedule", [0, 1, 2])
def test_refactorize_and_solve_match_reference(schedule):
    """refactorize() on second values: the replay (or, where its growth test
    fails, the factor_ the reference falls back to) and the solve."""
    for gmin, cases in by_gmin(FACTORED):
        topos = [Topology.order(int(c["n"]), c["col_ptr"], c["row_idx"], c["vals"], gmin,
                                solver="amdlu") for c in cases]
        st, lus, xs, _ = run(topos, [c["vals2"] for c in cases], [gmin] * len(cases),
                             bs=[c["b"] for c in cases], schedule=schedule)
        for k, c in enumerate(cases):
            name = c["name"]
            if int(c["fallback"]) > 0 and not same_pivots(c["f1"], c["f2"]):
                assert st[k] == L.NSG_REORDER, name
                # the host re-factors (AmdLuSolver::factor_) and the device
                # replays the new pivots
                topos[k].numeric(c["vals2"], gmin)
                s2, lu2, x2, _ = run([topos[k]], [c["vals2"]], [gmin], bs=[c["b"]],
                                     schedule=schedule)
                assert s2[0] == 0, name
                np.testing.assert_array_equal(lu2[0], packed_factor(c["f2"]), err_msg=name)
                np.testing.assert_array_equal(x2[0], c["x"], err_msg=name)
                continue
            assert st[k] == 0, name
            np.testing.assert_array_equal(lus[k], packed_factor(c["f2"]), err_msg=name)
            np.testing.assert_array_equal(xs[k], c["x"], err_msg=name)
            if "x_true" in c:
                np.testing.assert_allclose(xs[k], c["x_true"], rtol=0, atol=float(c["tol"]))


def test_numeric_pivot_check_agrees_with_host_factor():
    """numeric() on new values passes on the device exactly when the host
    factor_ would keep the pivots."""
    rng = np.random.default_rng(5)
    topos, vals, expect = [], [], []
    for k in range(60):
        n, cp, ri, v = random_matrix(rng, int(rng.integers(5, 60)), 0.15,
                                     diag_dominant=(k % 3 == 0), zero_diag_frac=0.1)
        try:
            t = Topology.order(n, cp, ri, v, solver="amdlu")
        except L.NsgError:
            continue
        v2 = v * np.exp(rng.uniform(0.0, 1.5) * rng.standard_normal(len(v)))
        try:
            fresh = Topology.order(n, cp, ri, v2, solver="amdlu")
        except L.NsgError:
            continue
        same = all(np.array_equal(a, b) for a, b in zip(t.export(), fresh.export()))
        topos.append(t)
        vals.append(v2)
        expect.append(same)
    st, _, _, _ = run(topos, vals, [0.0] * len(topos), check=True)
    assert any(expect) and not all(expect)
    for s, same in zip(st, expect):
        assert (s == 0) == same
        if not same:
            assert s == L.NSG_REORDER


def test_transposed_solve_and_mixed_engines():
    """One batch holding Markowitz and AMD-LU instances; the transposed
    solve of AMD-LU (no reference counterpart) against numpy."""
    rng = np.random.default_rng(17)
    mats = [mna_mesh(rng, s, 1 + s % 3) for s in (6, 12, 17)]
    mats += [random_matrix(rng, int(rng.integers(10, 80)), 0.05, True, 0.0) for _ in range(6)]
    topos, vals, bs, dense = [], [], [], []
    for k, (n, cp, ri, v) in enumerate(mats):
        topos.append(Topology.order(n, cp, ri, v, solver="amdlu" if k % 2 == 0 else "markowitz"))
        vals.append(v)
        bs.append(rng.standard_normal(n))
        A = np.zeros((n, n))
        for j in range(n):
            A[ri[cp[j]:cp[j + 1]], j] = v[cp[j]:cp[j + 1]]
        dense.append(A)
    st, _, xs, xts = run(topos, vals, [0.0] * len(topos), bs=bs)
    assert np.all(st == 0)
    for A, b, x, xt in zip(dense, bs, xs, xts):
        np.testing.assert_allclose(A @ x, b, rtol=1e-9, atol=1e-9)
        np.testing.assert_allclose(A.T @ xt, b, rtol=1e-9, atol=1e-9)


LINEAR = golden_cases.load_linear()


def test_linear_dc_uses_amdlu_and_matches_reference():
    """Linear circuits of 256+ unknowns: make_solver picks AMD-LU, as the
    reference does, and the operating point is the reference's."""
    from neospice_b200.circuit import DcBatch
    cases = [g for g in LINEAR if int(g["kind"]) == 0]
    batch = DcBatch([g["netlist"].build() for g in cases])
    assert batch.engines() == ["amdlu"] * len(cases)
    sols, status, iters = batch.run()
    torch.cuda.synchronize()
    status, iters = status.cpu().numpy(), iters.cpu().numpy()
    for k, (g, s) in enumerate(zip(cases, batch.split(sols))):
        assert status[k] == 0
        np.testing.assert_array_equal(s, g["values"][0], err_msg=f"case {k}")
        assert iters[k] == int(g["iterations"])


def test_linear_transient_uses_amdlu_and_matches_reference():
    from neospice_b200.circuit import TranBatch
    for g in [g for g in LINEAR if int(g["kind"]) == 1]:
        nn = g["netlist"].num_nodes
        b = TranBatch([g["netlist"].build()], float(g["tstep"]), float(g["tstop"]),
                      np.arange(nn, dtype=np.int32), max_points=len(g["times"]) + 8)
        b.run()
        r = b.results()[0]
        dc, tr = b.engines()
        assert dc == ["amdlu"] and tr == ["amdlu"]
        assert r["status"] == 0
        assert len(r["time"]) == len(g["times"])
        np.testing.assert_allclose(r["time"], g["times"], rtol=1e-12, atol=0)
        np.testing.assert_allclose(r["values"], g["values"], rtol=1e-9, atol=1e-12)
        assert r["newton_iters"] == int(g["iterations"])
        assert r["rejected"] == int(g["rejected"])


def test_forced_markowitz_keeps_linear_results_within_tolerance(monkeypatch):
    """NEOSPICE_SOLVER=markowitz: the other engine, the same operating point
    to 1e-9 (a different pivot order rounds differently)."""
    from neospice_b200.circuit import DcBatch
    monkeypatch.setenv("NEOSPICE_SOLVER", "markowitz")
    cases = [g for g in LINEAR if int(g["kind"]) == 0]
    batch = DcBatch([g["netlist"].build() for g in cases])
    assert batch.engines() == ["markowitz"] * len(cases)
    sols, status, _ = batch.run()
    torch.cuda.synchronize()
    assert np.all(status.cpu().numpy() == 0)
    for g, s in zip(cases, batch.split(sols)):
        np.testing.assert_allclose(s, g["values"][0], rtol=1e-9, atol=1e-12)
