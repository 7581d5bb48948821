"""Host circuit layer: pattern, first-iteration matrix and pivot order of
the diode-mesh circuits must equal the reference's, bit for bit."""
import numpy as np
import pytest

import golden_cases
import netlists
import oracle
from neospice_b200 import _lib as L
from neospice_b200 import workloads
from neospice_b200.circuit import GND, Circuit
from neospice_b200.solver import Topology

MESHES = golden_cases.load_meshes()


@pytest.mark.parametrize("k", range(len(MESHES)))
def test_mesh_pattern_and_initial_matrix_match_golden(k):
    g = MESHES[k]
    c = g["mesh"].build()
    cp, ri = c.pattern()
    np.testing.assert_array_equal(cp, g["col_ptr"])
    np.testing.assert_array_equal(ri, g["row_idx"])
    a, r = c.initial_matrix()
    np.testing.assert_array_equal(a, g["a0"])
    np.testing.assert_array_equal(r, g["rhs0"])


@pytest.mark.skipif(not oracle.have_ref(), reason="reference library not built here")
def test_random_meshes_match_reference():
    for k in range(6):
        m = workloads.diode_mesh(np.random.default_rng([5, k]), side_range=(3, 24))
        c = m.build()
        cp, ri = c.pattern()
        a, r = c.initial_matrix()
        rcp, rri, rv, rr = oracle.ref_mesh_initjct(m)
        np.testing.assert_array_equal(cp, rcp)
        np.testing.assert_array_equal(ri, rri)
        np.testing.assert_array_equal(a, rv)
        np.testing.assert_array_equal(r, rr)
        rs = oracle.RefSolver(len(rcp) - 1, rcp, rri)
        assert rs.numeric(rv) == 0
        st, _ = rs.export()
        t = Topology.order(len(cp) - 1, cp, ri, a)
        assert st.same_as(oracle.Structure(st.n, *t.export()))


def test_pivot_order_depends_only_on_pattern_for_meshes():
    """Same-side meshes with different values and diode/source placements
    get the same pivot sequence: the basis of per-pattern symbolic sharing."""
    for side in (6, 11):
        exports = []
        for k in range(4):
            m = workloads.diode_mesh(np.random.default_rng([side, k]), side=side)
            c = m.build()
            cp, ri = c.pattern()
            a, _ = c.initial_matrix()
            exports.append(Topology.order(len(cp) - 1, cp, ri, a).export())
        for e in exports[1:]:
            assert all(np.array_equal(x, y) for x, y in zip(e, exports[0]))


def test_load_order_and_branch_numbering():
    # two sources: the newest is loaded first and gets the first branch index
    c = Circuit(2)
    c.R(0, 1, 1e3)
    c.V(0, GND, 1.0)
    c.V(1, GND, 2.0)
    c.finalize()
    assert c.info()["num_vars"] == 4
    cp, ri = c.pattern()
    # branch 2 belongs to the second source (node 1), branch 3 to the first
    col2 = set(ri[cp[2]:cp[3]])
    col3 = set(ri[cp[3]:cp[4]])
    assert col2 == {1} and col3 == {0}


def test_dead_node_gets_pinned_diagonal():
    c = Circuit(3)
    c.R(0, GND, 1e3)
    c.V(0, GND, 1.0)
    c.I(GND, 1, 0.0)  # node 1: only a current source -> dead
    c.R(2, GND, 10.0)
    c.finalize()
    cp, ri = c.pattern()
    assert 1 in ri[cp[1]:cp[2]]
    a, _ = c.initial_matrix(gmin=1e-12)
    assert a[cp[1]] == 1e-12


def test_circuit_misuse_raises():
    c = Circuit(2)
    with pytest.raises(L.NsgError):
        c.R(0, 5, 1.0)  # node out of range
    with pytest.raises(L.NsgError):
        c.D(0, GND, IS=-1.0)
    c.R(0, 1, 1.0)
    c.R(1, GND, 1.0)
    c.finalize()
    with pytest.raises(L.NsgError):
        c.R(0, 1, 1.0)  # after finalize


def test_capacitor_and_wave_sources_params_order():
    from neospice_b200.circuit import Circuit
    c = Circuit(3)
    c.R(0, 1, 10.0)
    c.C(1, -1, 1e-12, ic=0.25)
    c.VPULSE(0, -1, 0.0, 1.0, 1e-9, 0.0, 0.0, 0.0, 0.0)
    c.IPWL(2, -1, [(0.0, 0.0), (1e-9, 1e-3)])
    c.C(2, 1, 2e-12)
    c.finalize()
    p = c.params()
    np.testing.assert_array_equal(p, [10.0, 1e-12, 0.25, 0.0, 1.0, 1e-9, 0, 0, 0, 0,
                                      0.0, 0.0, 1e-9, 1e-3, 2e-12, 0.0])
    assert c.info()["num_vars"] == 4  # 3 nodes + the V branch


def test_diode_param_block():
    """DIOtemp at the nominal temperature: the junction potential and
    capacitance come back (to rounding) as given, F1..F3 follow their
    definitions, and the grading (M > 0.9) and junction-potential
    (FC*VJ > 1) limits apply."""
    from neospice_b200 import _lib as L
    from neospice_b200.circuit import diode_params
    p = diode_params(1e-14, 1.5, 2e-12, 0.8, 0.4, 0.5, 5e-9)
    assert p[0] == 1e-14 and p[1] == 1.5 and p[9] == 5e-9 and p[8] == 0.4
    np.testing.assert_allclose(p[2], 2e-12, rtol=1e-12)
    np.testing.assert_allclose(p[3], 0.8, rtol=1e-12)
    np.testing.assert_allclose(p[4], 0.4, rtol=1e-12)
    xfc = np.log(1 - 0.5)
    np.testing.assert_allclose(p[5], p[3] * (1 - np.exp((1 - 0.4) * xfc)) / (1 - 0.4), rtol=1e-14)
    np.testing.assert_allclose(p[6], np.exp(1.4 * xfc), rtol=1e-14)
    np.testing.assert_allclose(p[7], 1 - 0.5 * 1.4, rtol=1e-14)
    assert diode_params(M=0.95)[8] == 0.9
    q = diode_params(VJ=2.5, FC=0.5)
    assert q[3] == 2.0 and q[4] == 1.0
    d = diode_params()
    assert d[2] == 0.0 and d[9] == 0.0
    for bad in (dict(CJO=-1e-12), dict(VJ=0.0), dict(M=1.0), dict(FC=1.0), dict(TT=-1e-9),
                dict(IS=0.0), dict(BV=-5.0), dict(BV=5.0, IBV=0.0), dict(BV=5.0, NBV=0.0)):
        with pytest.raises(L.NsgError):
            diode_params(**bad)


def test_diode_breakdown_param_block():
    """DIOtemp's breakdown voltage: without BV the block says so; with BV
    the voltage is where the reverse current matches IBV to the loop's
    exit tolerance (RELTOL 1e-3 of IBV), NBV defaults to N, and an IBV below
    IS*BV/vt keeps BV itself."""
    from neospice_b200.circuit import diode_params
    vt = 1.38064852e-23 / 1.6021766208e-19 * 300.15
    assert diode_params()[10] == 0.0
    p = diode_params(1e-14, 1.2, BV=5.1, IBV=1e-3)
    assert p[10] == 1.0 and p[12] == 1.2
    xbv = p[11]
    assert 4.0 < xbv < 5.1
    xcbv = 1e-14 * (np.exp((5.1 - xbv) / (1.2 * vt)) - 1 + xbv / vt)
    assert abs(xcbv - 1e-3) <= 1e-3 * 1e-3
    q = diode_params(1e-6, 1.0, BV=50.0, IBV=1e-9, NBV=2.0)
    assert q[11] == 50.0 and q[12] == 2.0


def test_tran_batch_rejects_bad_probes():
    """Probe validation (diodes, with or without charge, are accepted)."""
    from neospice_b200 import _lib as L
    from neospice_b200.circuit import Circuit, TranBatch
    c = Circuit(2)
    c.R(0, 1, 10.0)
    c.D(1, -1, 1e-14, 1.0, CJO=1e-12, TT=1e-9)
    c.V(0, -1, 1.0)
    c.finalize()
    with pytest.raises(L.NsgError, match="probe"):
        TranBatch([c], 1e-12, 1e-10, [5])
    d = Circuit(2)
    d.R(0, 1, 10.0)
    d.C(1, -1, 1e-12)
    d.V(0, -1, 1.0)
    d.finalize()
    with pytest.raises(L.NsgError, match="probe"):
        TranBatch([d], 1e-12, 1e-10, [7])


@pytest.mark.skipif(not oracle.have_ref(), reason="reference library not built here")
def test_mos_first_matrix_matches_reference():
    """MOS1load at MODEDCOP | MODEINITJCT on the host: pattern, matrix and
    rhs bit-identical to the reference's first Newton iteration."""
    import netlists
    for g in golden_cases.load_mos_dc():
        nl = g["netlist"]
        cp, ri, a, r = oracle.ref_sim_initjct(netlists.ref_desc(nl))
        c = nl.build()
        cp2, ri2 = c.pattern()
        a2, r2 = c.initial_matrix()
        np.testing.assert_array_equal(cp2, cp)
        np.testing.assert_array_equal(ri2, ri)
        np.testing.assert_array_equal(a2, a)
        np.testing.assert_array_equal(r2, r)


def test_mos_model_card_validation():
    c = Circuit(3)
    with pytest.raises(L.NsgError, match="unknown parameter"):
        c.model_mos1("nmos", VTO=0.7, BOGUS=1.0)
    with pytest.raises(L.NsgError, match="not supported"):
        c.model_mos1("nmos", VTO=0.7, RD=0.0, RSH=10.0)  # node without conductance
    c.model_mos1("nmos", VTO=0.7, RD=10.0)  # series resistance: internal drain' node
    m = c.model_mos1("nmos", VTO=0.7, KP=1e-4, RD=0.0)
    with pytest.raises(L.NsgError, match="W > 0"):
        c.M(0, 1, 2, -1, m, 0.0, 1e-6)


def test_set_param():
    """nsg_circuit_set_param overwrites one entry of the parameter layout and
    rejects indexes outside it."""
    from neospice_b200 import _lib as L
    from neospice_b200.circuit import Circuit
    c = Circuit(2)
    c.R(0, 1, 10.0)
    c.V(0, -1, 1.0)
    c.C(1, -1, 1e-12)
    c.finalize()
    c.set_param(1, 2.5)
    np.testing.assert_array_equal(c.params(), [10.0, 2.5, 1e-12, 0.0])
    for bad in (-1, 4):
        with pytest.raises(L.NsgError):
            c.set_param(bad, 1.0)


def test_device_methods_return_parameter_index():
    """Each device method returns the index of its first parameter in
    params(), so a stepped or swept value can be addressed directly."""
    from neospice_b200.circuit import Circuit
    c = Circuit(3)
    assert c.R(0, 1, 10.0) == 0
    assert c.C(1, -1, 1e-12, ic=0.1) == 1
    assert c.V(0, -1, 1.0) == 3
    assert c.VPULSE(2, -1, 0.0, 1.0, 1e-9) == 4
    assert c.D(2, -1) == 11
    assert c.I(-1, 1, 1e-3) == 26  # a diode holds 15 values
    c.finalize()
    p = c.params()
    assert p[0] == 10.0 and p[1] == 1e-12 and p[3] == 1.0 and p[26] == 1e-3
    assert c.param_count() == len(p) == 27


def _diode_netlists():
    """Diode networks with series resistance (internal posPrime nodes),
    breakdown and plain diodes mixed with sources, resistors and capacitors,
    in varied creation orders."""
    from neospice_b200.workloads import Netlist
    nan = float("nan")
    out = []
    for k in range(6):
        rng = np.random.default_rng([77, k])
        devs = [("V", 0, -1, float(rng.uniform(1, 10)))]
        for i in range(1, 5):
            devs.append(("R", int(rng.integers(0, i)), i, float(10 ** rng.uniform(1, 4))))
            rs = float(10 ** rng.uniform(-1, 2)) if rng.random() < 0.6 else 0.0
            bv = float(rng.uniform(3, 8)) if rng.random() < 0.5 else nan
            a, b = (i, -1) if rng.random() < 0.5 else (-1, i)
            devs.append(("D", a, b, 1e-14, 1.2, 1e-12, 0.8, 0.4, 0.5, 1e-9, bv, 1e-3, 1.3, rs))
            if rng.random() < 0.4:
                devs.append(("C", i, -1, 1e-12))
        out.append(Netlist(5, devs, {}))
    return out


@pytest.mark.skipif(not oracle.have_ref(), reason="reference library not built")
@pytest.mark.parametrize("k", range(6))
def test_diode_series_resistance_first_matrix_bitwise(k):
    """Diodes with RS get the reference's internal node numbering (after the
    external nodes, in load order, before the branch unknowns) and DIOload's
    series-conductance stamps: pattern, first DC matrix and rhs equal the
    reference's bit for bit."""
    nl = _diode_netlists()[k]
    c = nl.build()
    cp, ri = c.pattern()
    a, rhs = c.initial_matrix(1e-12)
    rcp, rri, ra, rrhs = oracle.ref_sim_initjct(netlists.ref_desc(nl))
    np.testing.assert_array_equal(cp, rcp)
    np.testing.assert_array_equal(ri, rri)
    np.testing.assert_array_equal(a, ra)
    np.testing.assert_array_equal(rhs, rrhs)
    n_rs = sum(1 for d in nl.devices if d[0] == "D" and d[13] != 0.0)
    assert c.info()["num_nodes"] == 5 + n_rs


def test_diode_rs_validation():
    from neospice_b200 import _lib as L
    from neospice_b200.circuit import Circuit, diode_params
    assert diode_params(RS=5.0)[13] == 5.0 and diode_params()[13] == 0.0
    c = Circuit(2)
    with pytest.raises(L.NsgError):
        c.D(0, 1, RS=-1.0)
