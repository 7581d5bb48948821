"""Pin the oracle: the C restatement (oracle/ns_oracle.c) must reproduce the
reference's own factor and solve values bit for bit, on the committed golden
cases (generated by the reference) and, where the reference library was
built here, on fresh seeded matrices."""
import numpy as np
import pytest

import golden_cases
import oracle
from matrices import banded, dense_to_csc, mna_mesh, random_matrix

CASES = golden_cases.load()


@pytest.mark.parametrize("k", range(len(CASES)))
def test_port_matches_golden(k):
    c = CASES[k]
    st = c["structure"]
    # order_and_factor and factor share the rounding sequence, so the fixed
    # pivot refactor of the first values reproduces the ordering pass.
    rc, lu, _ = oracle.port_refactor(st, c["vals"])
    assert rc == 0
    np.testing.assert_array_equal(lu, c["lu_numeric"])
    rc, lu, _ = oracle.port_refactor(st, c["vals2"])
    assert rc == int(c["refactor_rc"])
    if rc == 0:
        np.testing.assert_array_equal(lu, c["lu_refactor"])
        np.testing.assert_array_equal(oracle.port_solve(st, lu, c["b"]), c["x"])
        np.testing.assert_array_equal(oracle.port_solve(st, lu, c["b"], transposed=True), c["xt"])


def test_golden_solutions_are_solutions():
    """Sanity of the fixtures: on well-conditioned cases the reference's
    solutions solve A x = b and A^T x = b."""
    from matrices import matvec
    checked = 0
    for c in CASES:
        if int(c["refactor_rc"]) != 0:
            continue
        n, cp, ri, v2 = int(c["n"]), c["col_ptr"], c["row_idx"], c["vals2"]
        dense = np.zeros((n, n))
        for j in range(n):
            dense[ri[cp[j]:cp[j + 1]], j] = v2[cp[j]:cp[j + 1]]
        if np.linalg.cond(dense) > 1e10:
            continue
        checked += 1
        r = matvec(n, cp, ri, v2, c["x"]) - c["b"]
        rt = matvec(n, cp, ri, v2, c["xt"], transposed=True) - c["b"]
        scale = 1 + np.abs(c["b"]).max()
        assert np.abs(r).max() < 1e-6 * scale
        assert np.abs(rt).max() < 1e-6 * scale
    assert checked > 20


# Known-answer systems of the reference's solver tests
# (tests/unit/test_neo_solver.cpp:15-99).
KNOWN = [
    ([[3.0]], [9.0], [3.0]),
    ([[2.0, 1.0], [1.0, 3.0]], [5.0, 7.0], [1.6, 1.8]),
    ([[4.0, 2.0], [1.0, 5.0]], [14.0, 17.0], [2.0, 3.0]),
]


@pytest.mark.skipif(not oracle.have_ref(), reason="reference library not built here")
@pytest.mark.parametrize("A,b,x", KNOWN)
def test_known_answers(A, b, x):
    n, cp, ri, vals = dense_to_csc(A)
    rs = oracle.RefSolver(n, cp, ri)
    assert rs.numeric(vals) == 0
    st, lu = rs.export()
    rc, lu_p, _ = oracle.port_refactor(st, vals)
    assert rc == 0
    np.testing.assert_array_equal(lu_p, lu)
    np.testing.assert_allclose(oracle.port_solve(st, lu_p, b), x, rtol=1e-12)
    np.testing.assert_allclose(rs.solve(b), x, rtol=1e-12)


@pytest.mark.skipif(not oracle.have_ref(), reason="reference library not built here")
def test_port_matches_reference_fresh():
    rng = np.random.default_rng(99)
    mats = [random_matrix(rng, int(rng.integers(2, 60)), 0.15, bool(k % 2), 0.2) for k in range(40)]
    mats += [mna_mesh(rng, 10, 2), banded(300, 7, seed=3)]
    for (n, cp, ri, vals) in mats:
        rs = oracle.RefSolver(n, cp, ri)
        if rs.numeric(vals) != 0:
            continue
        st, lu = rs.export()
        rc, lu_p, _ = oracle.port_refactor(st, vals)
        assert rc == 0
        np.testing.assert_array_equal(lu_p, lu)
        v2 = vals * (1 + 0.1 * rng.standard_normal(len(vals)))
        rc_ref = rs.refactorize(v2)
        _, lu_r = rs.export()
        rc_p, lu_p, _ = oracle.port_refactor(st, v2)
        assert (rc_ref != 0) == (rc_p != 0)
        if rc_ref == 0:
            np.testing.assert_array_equal(lu_p, lu_r)
            b = rng.standard_normal(n)
            np.testing.assert_array_equal(oracle.port_solve(st, lu_p, b), rs.solve(b))
            np.testing.assert_array_equal(oracle.port_solve(st, lu_p, b, True), rs.solve(b, True))


@pytest.mark.skipif(not oracle.have_ref(), reason="reference library not built here")
def test_port_revalidation_flags_like_reference():
    """The check_pivots mode flags exactly the matrices on which a later
    NeoSolver::numeric re-orders."""
    rng = np.random.default_rng(5)
    agree = 0
    for k in range(60):
        n, cp, ri, vals = random_matrix(rng, 20, 0.3, diag_dominant=False, zero_diag_frac=0.1)
        rs = oracle.RefSolver(n, cp, ri)
        if rs.numeric(vals) != 0:
            continue
        st, _ = rs.export()
        v2 = vals * np.exp(rng.standard_normal(len(vals)))
        rc_p, _, step = oracle.port_refactor(st, v2, check_pivots=True)
        rs.numeric(v2)
        st2, _ = rs.export()
        reordered = not st2.same_as(st)
        if rc_p == 0:
            assert not reordered
        agree += 1
    assert agree > 20
