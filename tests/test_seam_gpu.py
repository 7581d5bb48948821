"""The drop-in claim, end to end: the reference's own analyses -- solve_dc
(src/core/dc.cpp, with its Newton loop and continuation aids) and
solve_transient (src/core/transient.cpp) -- run unmodified with this
repository's GPU solver under them, through the reference's ISolver seam
(oracle/gpu_seam.cpp: GpuNeoSolver, the adapter a maintainer adds, returned
by make_solver).  Every solution, timepoint and iteration count must equal
those of the same analyses on the reference's own NeoSolver / AmdLuSolver,
bit for bit: the GPU factors and solves are bit-identical to the CPU ones,
so the whole Newton sequence is."""
import numpy as np
import pytest

import golden_cases
import netlists
import oracle
from neospice_b200 import workloads as W

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.have_seam(), reason="seam library not built")]


def _both(desc, analysis, tstep=0.0, tstop=0.0):
    lib = oracle.seam()
    out = []
    for on in (0, 1):
        lib.nsseam_use_gpu(on)
        try:
            out.append(oracle.ref_sim(desc, analysis, tstep, tstop, lib=lib))
        finally:
            lib.nsseam_use_gpu(0)
    return out


def test_reference_solve_dc_on_gpu_solver():
    lib = oracle.seam()
    before = lib.nsseam_gpu_solvers()
    nls = [g["netlist"] for g in golden_cases.load_mos_dc()]
    nls += [W.resistor_network(np.random.default_rng([72, k]), 12) for k in range(2)]
    nls.append(W.resistor_network(np.random.default_rng([72, 9]), 300))  # AMD-LU range
    for k, nl in enumerate(nls):
        (_, v_cpu, i_cpu), (_, v_gpu, i_gpu) = _both(netlists.ref_desc(nl), 0)
        np.testing.assert_array_equal(v_gpu, v_cpu, err_msg=f"case {k}")
        assert i_gpu["iterations"] == i_cpu["iterations"], k
        assert i_gpu["method"] == i_cpu["method"], k
    assert lib.nsseam_gpu_solvers() >= before + len(nls)


def test_reference_mesh_dc_on_gpu_solver():
    lib = oracle.seam()
    for k in range(3):
        m = W.diode_mesh(np.random.default_rng([73, k]), side_range=(8, 20))
        lib.nsseam_use_gpu(0)
        s_cpu, it_cpu, _ = oracle.ref_mesh_dc(m, lib=lib)
        lib.nsseam_use_gpu(1)
        try:
            s_gpu, it_gpu, _ = oracle.ref_mesh_dc(m, lib=lib)
        finally:
            lib.nsseam_use_gpu(0)
        np.testing.assert_array_equal(s_gpu, s_cpu)
        assert it_gpu == it_cpu


def test_reference_solve_transient_on_gpu_solver():
    cases = golden_cases.load_transients()
    for k in (0, 1, 2):
        g = cases[k]
        (t_cpu, v_cpu, i_cpu), (t_gpu, v_gpu, i_gpu) = _both(
            netlists.ref_desc(g["netlist"]), 1, float(g["tstep"]), float(g["tstop"]))
        np.testing.assert_array_equal(t_gpu, t_cpu, err_msg=f"case {k}")
        np.testing.assert_array_equal(v_gpu, v_cpu, err_msg=f"case {k}")
        assert i_gpu["iterations"] == i_cpu["iterations"]
        assert i_gpu["rejected"] == i_cpu["rejected"]


@pytest.mark.parametrize("kind", ["ladder", "mesh"])
def test_ac_sweep_through_the_seam(kind):
    """solve_ac's frequency loop (numeric_complex, refactorize_complex,
    solve_complex) on the ISolver adapter: GPU solutions equal NeoSolver's
    bit for bit at every point."""
    nl = W.rc_ladder(np.random.default_rng(15), 40) if kind == "ladder" else \
        W.rc_mesh(np.random.default_rng(16), 10)
    n, cp, ri, g, c, b = W.ac_system(nl)
    omegas = 2 * np.pi * np.logspace(2, 10, 33)
    z_cpu, s_cpu = oracle.seam_ac_sweep(n, cp, ri, g, c, b, omegas, gpu=False)
    z_gpu, s_gpu = oracle.seam_ac_sweep(n, cp, ri, g, c, b, omegas, gpu=True)
    np.testing.assert_array_equal(s_gpu, s_cpu)
    np.testing.assert_array_equal(z_gpu.real, z_cpu.real)
    np.testing.assert_array_equal(z_gpu.imag, z_cpu.imag)


@pytest.mark.parametrize("seed", range(4))
def test_equilibrated_solves_through_the_seam(seed):
    """NeoSolver's row/column equilibration (solve_dc's last aid) on the GPU
    adapter: numeric and refactorize of D_r A D_c, scaled solves -- equal to
    the reference's equilibrated NeoSolver bit for bit, with and without
    diag_gmin, on MNA matrices whose rows span many decades."""
    rng = np.random.default_rng([17, seed])
    m = W.diode_mesh(rng, side_range=(8, 16))
    c = m.build()
    cp, ri = c.pattern()
    a, _ = c.initial_matrix(1e-12)
    n = len(cp) - 1
    rows = 10.0 ** rng.uniform(-6, 6, n)  # badly scaled rows
    seq = np.stack([a * rows[ri] * np.exp(0.05 * rng.standard_normal(len(a))) for _ in range(4)])
    b = rng.standard_normal(n)
    for gmin in (0.0, 1e-9):
        x_cpu, s_cpu = oracle.seam_solve_sequence(n, cp, ri, seq, b, gpu=False, diag_gmin=gmin)
        x_gpu, s_gpu = oracle.seam_solve_sequence(n, cp, ri, seq, b, gpu=True, diag_gmin=gmin)
        np.testing.assert_array_equal(s_gpu, s_cpu)
        np.testing.assert_array_equal(x_gpu, x_cpu)
