"""The host symbolic phase (neospice_b200 Markowitz ordering) must produce the
reference's pivot sequence, fill pattern and slot map exactly."""
import numpy as np
import pytest

import golden_cases
import oracle
from matrices import mna_mesh, random_matrix
from neospice_b200 import _lib as L
from neospice_b200.solver import Topology

CASES = golden_cases.load()


def _same(topo, st):
    r, c, er, ec, se = topo.export()
    return (np.array_equal(r, st.int_to_ext_row) and np.array_equal(c, st.int_to_ext_col)
            and np.array_equal(er, st.elem_row) and np.array_equal(ec, st.elem_col)
            and np.array_equal(se, st.slot_to_elem))


@pytest.mark.parametrize("k", range(len(CASES)))
def test_order_matches_golden(k):
    c = CASES[k]
    topo = Topology.order(int(c["n"]), c["col_ptr"], c["row_idx"], c["vals"])
    assert _same(topo, c["structure"])


def test_import_roundtrip():
    c = CASES[-1]
    st = c["structure"]
    topo = Topology.import_structure(st.n, len(st.slot_to_elem), st.int_to_ext_row,
                                     st.int_to_ext_col, st.elem_row, st.elem_col, st.slot_to_elem)
    assert _same(topo, st)


def test_import_rejects_unclosed_fill():
    c = CASES[0]
    st = c["structure"]
    # drop one fill-in element (an element no slot maps to), if any
    fills = np.setdiff1d(np.arange(st.n_elem), st.slot_to_elem)
    if len(fills) == 0:
        pytest.skip("case has no fill-in")
    keep = np.setdiff1d(np.arange(st.n_elem), fills[:1])
    remap = -np.ones(st.n_elem, np.int64)
    remap[keep] = np.arange(len(keep))
    with pytest.raises(L.NsgError):
        Topology.import_structure(st.n, len(st.slot_to_elem), st.int_to_ext_row, st.int_to_ext_col,
                                  st.elem_row[keep], st.elem_col[keep], remap[st.slot_to_elem])


def test_order_rejects_bad_pattern():
    with pytest.raises(L.NsgError):
        Topology.order(2, [0, 2, 3], [1, 0, 1], [1.0, 2.0, 3.0])  # rows not ascending


def test_singular_reported():
    # structurally singular: an all-zero column
    with pytest.raises(L.NsgError) as e:
        Topology.order(2, [0, 1, 2], [0, 0], [1.0, 1.0])
    assert e.value.code == L.NSG_SINGULAR


@pytest.mark.skipif(not oracle.have_ref(), reason="reference library not built here")
def test_order_matches_reference_stress():
    rng = np.random.default_rng(1234)
    checked = 0
    for t in range(600):
        kind = t % 3
        if kind == 2:
            n, cp, ri, vals = mna_mesh(rng, int(rng.integers(2, 10)), int(rng.integers(1, 5)))
        else:
            n, cp, ri, vals = random_matrix(rng, int(rng.integers(1, 60)), float(rng.uniform(0.02, 0.5)),
                                            diag_dominant=(kind == 0),
                                            zero_diag_frac=float(rng.uniform(0, 0.5)),
                                            integer=bool(rng.random() < 0.3))
        rs = oracle.RefSolver(n, cp, ri)
        rc = rs.numeric(vals)
        if rc != 0:
            with pytest.raises(L.NsgError):
                Topology.order(n, cp, ri, vals)
            continue
        topo = Topology.order(n, cp, ri, vals)
        st, _ = rs.export()
        assert _same(topo, st), f"case {t}"
        # a later numeric() with new values: re-validation / re-ordering
        v2 = vals * np.exp(0.7 * rng.standard_normal(len(vals)))
        if rs.numeric(v2) != 0:
            continue
        topo.numeric(v2)
        st2, _ = rs.export()
        assert _same(topo, st2), f"case {t} renumeric"
        checked += 1
    assert checked > 300
