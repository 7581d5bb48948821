"""AMD-LU engine on the host (no GPU): the AMD ordering, the threshold
pivoting factor_ and make_solver's engine choice against the reference's
AmdLuSolver (golden fixtures from tests/golden/make_golden.py, and the
reference library itself where it was built), plus the oracle's C port of
the replay refactor and solve pinned against the same fixtures."""
import os
import pathlib

import numpy as np
import pytest

import golden_cases
import oracle
from neospice_b200 import _lib as L
from neospice_b200.solver import Topology, amd_order, select_solver

CASES = golden_cases.load_amd()
FACTORED = [c for c in CASES if int(c["numeric_rc"]) == 0]


def _grid(side):
    cols = [[] for _ in range(side * side)]
    for y in range(side):
        for x in range(side):
            i = y * side + x
            cols[i] += [i] + ([i - 1] if x else []) + ([i + 1] if x < side - 1 else []) + \
                ([i - side] if y else []) + ([i + side] if y < side - 1 else [])
    cp = np.cumsum([0] + [len(c) for c in cols]).astype(np.int32)
    ri = np.concatenate([sorted(c) for c in cols]).astype(np.int32)
    return side * side, cp, ri


def structure_of(topo):
    """(pinv, q, per-column rows in stored order) of a topology's plan."""
    r, c, er, ec, _ = topo.export()
    n = len(r)
    pinv = np.empty(n, np.int32)
    pinv[r - 1] = np.arange(n)
    cols = [er[ec == k + 1] - 1 for k in range(n)]
    return pinv, c - 1, cols


def reference_columns(f):
    n = len(f["q"])
    return [np.concatenate([f["Ui"][f["Up"][k]:f["Up"][k + 1] - 1], [k],
                            f["Li"][f["Lp"][k] + 1:f["Lp"][k + 1]]]) for k in range(n)]


@pytest.mark.parametrize("case", FACTORED, ids=lambda c: c["name"])
def test_amd_order_matches_reference(case):
    perm = amd_order(int(case["n"]), case["col_ptr"], case["row_idx"])
    np.testing.assert_array_equal(perm, case["f1"]["q"])


@pytest.mark.parametrize("case", CASES, ids=lambda c: c["name"])
def test_host_factor_matches_reference(case):
    """factor_'s pivot sequence, L/U structure and replay order."""
    n = int(case["n"])
    if int(case["numeric_rc"]) != 0:
        with pytest.raises(L.NsgError) as e:
            Topology.order(n, case["col_ptr"], case["row_idx"], case["vals"],
                           float(case["gmin"]), solver="amdlu")
        assert e.value.code == 102
        return
    t = Topology.order(n, case["col_ptr"], case["row_idx"], case["vals"], float(case["gmin"]),
                       solver="amdlu")
    assert t.solver == "amdlu"
    pinv, q, cols = structure_of(t)
    f = case["f1"]
    np.testing.assert_array_equal(q, f["q"])
    np.testing.assert_array_equal(pinv, f["pinv"])
    for got, want in zip(cols, reference_columns(f)):
        np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("case", [c for c in FACTORED if int(c["fallback"]) > 0],
                         ids=lambda c: c["name"])
def test_host_refactor_fallback_matches_reference(case):
    """A replay that fails its growth test falls back to factor_: the host
    numeric() on the second values gives the reference's new factor."""
    n = int(case["n"])
    t = Topology.order(n, case["col_ptr"], case["row_idx"], case["vals"], float(case["gmin"]),
                       solver="amdlu")
    t.numeric(case["vals2"], float(case["gmin"]))
    pinv, q, cols = structure_of(t)
    f = case["f2"]
    np.testing.assert_array_equal(pinv, f["pinv"])
    for got, want in zip(cols, reference_columns(f)):
        np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("case", FACTORED, ids=lambda c: c["name"])
def test_port_replay_and_solve_match_reference(case):
    """The oracle's C port of refactor_replay_ / solve, pinned bit for bit."""
    rc, lx, ux, step = oracle.port_amd_replay(case["f1"], case["col_ptr"], case["row_idx"],
                                              case["vals2"], float(case["gmin"]))
    if int(case["fallback"]) > 0:
        assert rc == 103 and step >= 0
        return
    assert rc == 0
    np.testing.assert_array_equal(lx, case["f2"]["Lx"])
    np.testing.assert_array_equal(ux, case["f2"]["Ux"])
    x = oracle.port_amd_solve(case["f2"], lx, ux, case["b"])
    np.testing.assert_array_equal(x, case["x"])
    if "x_true" in case:
        np.testing.assert_allclose(x, case["x_true"], rtol=0, atol=float(case["tol"]))


def test_port_replay_reproduces_numeric_values():
    """Replaying the numeric() values themselves gives numeric()'s factor,
    unless factor_ accepted a pivot that the replay's stricter growth test
    (|u_kk| >= 1e-3 * the largest |U(:, k)|) rejects -- then the step it
    stops at must be such a pivot."""
    stopped = 0
    for case in FACTORED:
        f = case["f1"]
        rc, lx, ux, step = oracle.port_amd_replay(f, case["col_ptr"], case["row_idx"],
                                                  case["vals"], float(case["gmin"]))
        if rc == 103:
            col = f["Ux"][f["Up"][step]:f["Up"][step + 1]]
            assert abs(col[-1]) < 1e-3 * np.max(np.abs(col)), case["name"]
            stopped += 1
            continue
        assert rc == 0, case["name"]
        np.testing.assert_array_equal(lx, f["Lx"])
        np.testing.assert_array_equal(ux, f["Ux"])
    assert stopped < len(FACTORED) // 2


def test_amd_order_dense_and_grid_patterns():
    # grid: the selection order must not depend on how ties are stored
    n, cp, ri = _grid(12)
    perm = amd_order(n, cp, ri)
    assert sorted(perm) == list(range(n))
    # hub nodes above the dense threshold go last, by ascending degree
    n = 300
    cols = [[j] for j in range(n)]
    for hub, span in ((0, n), (7, 250)):
        for j in range(span):
            if j != hub:
                cols[j].append(hub)
                cols[hub].append(j)
    cp = np.cumsum([0] + [len(set(c)) for c in cols]).astype(np.int32)
    ri = np.concatenate([sorted(set(c)) for c in cols]).astype(np.int32)
    perm = amd_order(n, cp, ri)
    assert list(perm[-2:]) == [7, 0]


@pytest.mark.skipif(not oracle.have_ref(), reason="reference library not built")
@pytest.mark.parametrize("seed", range(6))
def test_amd_order_random_patterns_against_reference(seed):
    rng = np.random.default_rng([91, seed])
    for _ in range(20):
        n = int(rng.integers(1, 200))
        A = rng.random((n, n)) < rng.uniform(0.005, 0.1)
        np.fill_diagonal(A, True)
        if rng.random() < 0.5:
            A |= A.T
        cp = np.concatenate([[0], np.cumsum(A.sum(0))]).astype(np.int32)
        ri = np.concatenate([np.nonzero(A[:, j])[0] for j in range(n)]).astype(np.int32)
        np.testing.assert_array_equal(amd_order(n, cp, ri), oracle.ref_amd_order(n, cp, ri))
    n, cp, ri = _grid(60)
    np.testing.assert_array_equal(amd_order(n, cp, ri), oracle.ref_amd_order(n, cp, ri))


SELECT_ENVS = [
    {}, {"NEOSPICE_SOLVER": "amdlu"}, {"NEOSPICE_SOLVER": "klu"},
    {"NEOSPICE_SOLVER": "markowitz"}, {"NEOSPICE_SOLVER": "sparse"},
    {"NEOSPICE_SOLVER": "auto"}, {"NEOSPICE_FORCE_AMDLU": "1"}, {"NEOSPICE_FORCE_AMDLU": "0"},
    {"NEOSPICE_FORCE_AMDLU": ""}, {"NEOSPICE_SOLVER": "markowitz", "NEOSPICE_FORCE_AMDLU": "1"},
]


@pytest.fixture
def clean_env():
    saved = {k: os.environ.pop(k) for k in ("NEOSPICE_SOLVER", "NEOSPICE_FORCE_AMDLU")
             if k in os.environ}
    yield
    for k in ("NEOSPICE_SOLVER", "NEOSPICE_FORCE_AMDLU"):
        os.environ.pop(k, None)
    os.environ.update(saved)


@pytest.mark.parametrize("env", SELECT_ENVS, ids=lambda e: ",".join(f"{k}={v}" for k, v in e.items()) or "default")
def test_solver_selection_policy(env, clean_env):
    """make_solver's policy (make_solver.cpp:156-178): the reference's own
    choice where its library is built, the stated policy otherwise."""
    os.environ.update(env)
    for n in (1, 191, 255, 256, 257, 5000):
        for lin in (True, False):
            ours = select_solver(n, lin)
            if oracle.have_ref():
                want = oracle.ref_make_solver_name(n, lin)
                assert ours.endswith(want) or (ours == "auto-amdlu" and want == "amdlu"), \
                    (env, n, lin, ours, want)
            if not env or env.get("NEOSPICE_SOLVER") == "auto" or \
                    env.get("NEOSPICE_FORCE_AMDLU") in ("0", ""):
                assert ours == ("auto-amdlu" if (n >= 256 and lin) else "markowitz")


def test_auto_engine_falls_back_to_markowitz_on_singular_first_factor():
    """AutoFallbackSolver: AMD-LU singular at the first factorization ->
    Markowitz for good (here Markowitz also finds it singular, so the
    singular status propagates)."""
    c = next(c for c in CASES if c["name"] == "structurally_singular2")
    with pytest.raises(L.NsgError) as e:
        Topology.order(int(c["n"]), c["col_ptr"], c["row_idx"], c["vals"], solver="auto-amdlu")
    assert e.value.code == 102
    # a matrix AMD-LU factors: the auto engine stays on AMD-LU
    c = next(c for c in CASES if c["name"] == "mesh16")
    t = Topology.order(int(c["n"]), c["col_ptr"], c["row_idx"], c["vals"], solver="auto-amdlu")
    assert t.solver == "amdlu"


def test_update_map_matches_sequential_build(tmp_path):
    """The refactor's update map of a large AMD-LU plan, filled on several
    host threads, equals the one-column-at-a-time map (tests/cpp/
    plan_map_check.cpp, compiled here from the host sources)."""
    import shutil
    import subprocess
    cxx = shutil.which("g++") or shutil.which("c++")
    if not cxx:
        pytest.skip("no host C++ compiler")
    root = pathlib.Path(__file__).resolve().parents[1]
    src = root / "neospice_b200" / "csrc"
    exe = tmp_path / "plan_map_check"
    subprocess.run([cxx, "-std=c++17", "-O2", "-pthread", f"-I{src}",
                    str(root / "tests" / "cpp" / "plan_map_check.cpp"),
                    str(src / "host" / "amd_lu.cpp"), str(src / "host" / "plan.cpp"),
                    str(src / "host" / "sparse_order.cpp"), "-o", str(exe)], check=True)
    res = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "0 failure(s)" in res.stdout
