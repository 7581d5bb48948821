"""Circuits, batched DC operating points and batched transients on the GPU.

``Circuit`` mirrors the reference's typed Circuit API (src/core/circuit.hpp:
179-237) for resistors, capacitors, DC / PULSE / PWL voltage and current
sources, level-1 diodes and level-1 MOSFETs; nodes are integers and ``GND`` (-1) is ground.
``DcBatch`` runs the direct Newton attempt of Simulator::run_dc
(src/core/dc.cpp:53-118) for many circuits in one kernel launch;
``TranBatch`` runs solve_transient (src/core/transient.cpp:694-1067) for many
circuits in one launch, each with its own adaptive timestep.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib as L

# NSG_SOLVER_* engine codes of a plan.
ENGINE_NAMES = {0: "markowitz", 1: "amdlu"}

GND = -1



# Operating-point aids a DC batch may start at (nsg_dc_batch_set_first_aid).
AIDS = {"direct": 0, "source": 1, "gain": 2, "ptc": 3}

def diode_params(IS: float = 1e-14, N: float = 1.0, CJO: float = 0.0, VJ: float = 1.0,
                 M: float = 0.5, FC: float = 0.5, TT: float = 0.0, BV: float | None = None,
                 IBV: float = 1e-3, NBV: float | None = None, RS: float = 0.0) -> np.ndarray:
    """The 15-value parameter block a diode with this card holds in
    Circuit.params() at the nominal temperature: IS, N, then the junction
    values, then the breakdown flag, DIOtemp's breakdown voltage, NBV, RS
    and vt (nsg_diode_param_block)."""
    out = np.zeros(15, np.float64)
    L.check(L.lib().nsg_diode_param_block(float(IS), float(N), float(CJO), float(VJ), float(M),
                                          float(FC), float(TT),
                                          float("nan") if BV is None else float(BV), float(IBV),
                                          float("nan") if NBV is None else float(NBV), float(RS),
                                          L.dptr(out)))
    return out

class Circuit:
    def __init__(self, num_nodes: int):
        h = ctypes.c_void_p()
        L.check(L.lib().nsg_circuit_create(int(num_nodes), ctypes.byref(h)))
        self._h = h
        self.num_nodes = int(num_nodes)
        self._final = False

    @property
    def handle(self):
        return self._h

    def param_count(self) -> int:
        """Parameters held so far: the device methods below return the index
        of the first parameter of the device they add (for set_param, the
        batches' parameter arrays and `.step` sweeps)."""
        n = ctypes.c_int()
        L.check(L.lib().nsg_circuit_param_count(self._h, ctypes.byref(n)))
        return n.value

    def R(self, a: int, b: int, ohms: float):
        first = self.param_count()
        L.check(L.lib().nsg_circuit_add_resistor(self._h, int(a), int(b), float(ohms)))
        return first

    def V(self, p: int, n: int, volts: float):
        first = self.param_count()
        L.check(L.lib().nsg_circuit_add_vsource(self._h, int(p), int(n), float(volts)))
        return first

    def I(self, p: int, n: int, amps: float):  # noqa: E743 - the reference's name
        first = self.param_count()
        L.check(L.lib().nsg_circuit_add_isource(self._h, int(p), int(n), float(amps)))
        return first

    def set_temperature(self, kelvin: float):
        """The circuit temperature (the reference's options.temp, default
        300.15 K); set it before adding devices."""
        L.check(L.lib().nsg_circuit_set_temperature(self._h, float(kelvin)))

    def D(self, anode: int, cathode: int, IS: float = 1e-14, N: float = 1.0, CJO: float = 0.0,
          VJ: float = 1.0, M: float = 0.5, FC: float = 0.5, TT: float = 0.0,
          BV: float | None = None, IBV: float = 1e-3, NBV: float | None = None,
          RS: float = 0.0):
        """Level-1 diode with the card D(IS N CJO VJ M FC TT [BV IBV NBV]
        [RS]); the junction capacitance and transit time act in the
        transient, BV (when given) adds the reverse breakdown region, RS > 0
        a series resistance through an internal node."""
        first = self.param_count()
        if BV is None and RS == 0.0:
            L.check(L.lib().nsg_circuit_add_diode_card(self._h, int(anode), int(cathode),
                                                       float(IS), float(N), float(CJO), float(VJ),
                                                       float(M), float(FC), float(TT)))
        else:
            nan = float("nan")
            L.check(L.lib().nsg_circuit_add_diode_card_ex(
                self._h, int(anode), int(cathode), float(IS), float(N), float(CJO), float(VJ),
                float(M), float(FC), float(TT), nan if BV is None else float(BV), float(IBV),
                nan if NBV is None else float(NBV), float(RS)))
        return first

    def C(self, a: int, b: int, farads: float, ic: float | None = None):
        first = self.param_count()
        L.check(L.lib().nsg_circuit_add_capacitor(self._h, int(a), int(b), float(farads),
                                                  int(ic is not None),
                                                  0.0 if ic is None else float(ic)))
        return first

    def _wave(self, is_v: bool, p: int, n: int, wave: int, values):
        v = np.ascontiguousarray(values, np.float64)
        first = self.param_count()
        L.check(L.lib().nsg_circuit_add_source_wave(self._h, int(is_v), int(p), int(n), int(wave),
                                                    len(v), L.dptr(v)))
        return first

    def VPULSE(self, p: int, n: int, v1, v2, td=0.0, tr=0.0, tf=0.0, pw=0.0, per=0.0):
        """V source with PULSE(v1 v2 td tr tf pw per) (VSource::set_pulse)."""
        return self._wave(True, p, n, L.NSG_WAVE_PULSE, [v1, v2, td, tr, tf, pw, per])

    def IPULSE(self, p: int, n: int, v1, v2, td=0.0, tr=0.0, tf=0.0, pw=0.0, per=0.0):
        return self._wave(False, p, n, L.NSG_WAVE_PULSE, [v1, v2, td, tr, tf, pw, per])

    def VPWL(self, p: int, n: int, points):
        """V source with PWL(t0 v0 t1 v1 ...) (VSource::set_pwl)."""
        return self._wave(True, p, n, L.NSG_WAVE_PWL, np.asarray(points, np.float64).ravel())

    def IPWL(self, p: int, n: int, points):
        return self._wave(False, p, n, L.NSG_WAVE_PWL, np.asarray(points, np.float64).ravel())

    def model_mos1(self, mtype: str, **params) -> int:
        """A level-1 MOSFET model card, e.g. model_mos1("nmos", VTO=0.7,
        KP=110e-6); returns the model index for M()."""
        t = {"nmos": 1, "pmos": -1}[mtype.lower()]
        keys = (ctypes.c_char_p * max(1, len(params)))(*[k.encode() for k in params])
        vals = np.ascontiguousarray([float(v) for v in params.values()] or [0.0], np.float64)
        out = ctypes.c_int()
        L.check(L.lib().nsg_circuit_add_mos1_model(self._h, t, len(params), keys, L.dptr(vals),
                                                   ctypes.byref(out)))
        return out.value

    def model_bsim4(self, mtype: str, **params) -> int:
        """A BSIM4v7 (LEVEL=14) model card: the default card with TOXE, VTH0
        and U0 optionally given, e.g. model_bsim4("nmos", TOXE=2e-9);
        returns the model index for M4()."""
        t = {"nmos": 1, "pmos": -1}[mtype.lower()]
        params = {k: v for k, v in params.items() if k.lower() != "level"}
        keys = (ctypes.c_char_p * max(1, len(params)))(*[k.encode() for k in params])
        vals = np.ascontiguousarray([float(v) for v in params.values()] or [0.0], np.float64)
        out = ctypes.c_int()
        L.check(L.lib().nsg_circuit_add_bsim4_model(self._h, t, len(params), keys, L.dptr(vals),
                                                    ctypes.byref(out)))
        return out.value

    def M4(self, d: int, g: int, s: int, b: int, model: int, W: float = 1e-6, L_: float = 1e-7,
           delvto: float = 0.0):
        """A BSIM4v7 instance (Circuit::M on a LEVEL=14 model, with the DELVTO
        instance parameter)."""
        first = self.param_count()
        L.check(L.lib().nsg_circuit_add_bsim4(self._h, int(d), int(g), int(s), int(b), int(model),
                                              float(W), float(L_), float(delvto)))
        return first

    def M(self, d: int, g: int, s: int, b: int, model: int, W: float = 1e-6, L_: float = 1e-7):
        """Circuit::M(name, d, g, s, b, model, w, l)."""
        first = self.param_count()
        L.check(L.lib().nsg_circuit_add_mosfet(self._h, int(d), int(g), int(s), int(b), int(model),
                                               float(W), float(L_)))
        return first

    def add_capacitors(self, a, b, farads):
        a, b = np.ascontiguousarray(a, np.int32), np.ascontiguousarray(b, np.int32)
        f = np.ascontiguousarray(np.broadcast_to(farads, a.shape), np.float64)
        L.check(L.lib().nsg_circuit_add_capacitors(self._h, len(a), L.iptr(a), L.iptr(b),
                                                   L.dptr(f)))

    def add_resistors(self, a, b, ohms):
        a, b = np.ascontiguousarray(a, np.int32), np.ascontiguousarray(b, np.int32)
        ohms = np.ascontiguousarray(ohms, np.float64)
        L.check(L.lib().nsg_circuit_add_resistors(self._h, len(a), L.iptr(a), L.iptr(b),
                                                  L.dptr(ohms)))

    def add_isources(self, p, n, amps):
        p, n = np.ascontiguousarray(p, np.int32), np.ascontiguousarray(n, np.int32)
        amps = np.ascontiguousarray(amps, np.float64)
        L.check(L.lib().nsg_circuit_add_isources(self._h, len(p), L.iptr(p), L.iptr(n),
                                                 L.dptr(amps)))

    def add_diodes(self, anode, cathode, IS, N):
        a, k = np.ascontiguousarray(anode, np.int32), np.ascontiguousarray(cathode, np.int32)
        IS = np.ascontiguousarray(np.broadcast_to(IS, a.shape), np.float64)
        N = np.ascontiguousarray(np.broadcast_to(N, a.shape), np.float64)
        L.check(L.lib().nsg_circuit_add_diodes(self._h, len(a), L.iptr(a), L.iptr(k), L.dptr(IS),
                                               L.dptr(N)))

    def finalize(self):
        L.check(L.lib().nsg_circuit_finalize(self._h))
        self._final = True
        return self

    def set_param(self, index: int, value: float):
        """Overwrite parameter `index` of params() (a resistance,
        capacitance, DC source value, MOSFET W / L / VTO)."""
        L.check(L.lib().nsg_circuit_set_param(self._h, int(index), float(value)))

    def info(self) -> dict:
        nv, nn, nnz, npar = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        L.check(L.lib().nsg_circuit_info(self._h, ctypes.byref(nv), ctypes.byref(nn),
                                         ctypes.byref(nnz), ctypes.byref(npar)))
        return dict(num_vars=nv.value, num_nodes=nn.value, nnz=nnz.value, num_params=npar.value)

    def pattern(self):
        i = self.info()
        cp = np.zeros(i["num_vars"] + 1, np.int32)
        ri = np.zeros(i["nnz"], np.int32)
        L.check(L.lib().nsg_circuit_pattern(self._h, L.iptr(cp), L.iptr(ri)))
        return cp, ri

    def params(self):
        p = np.zeros(self.info()["num_params"])
        L.check(L.lib().nsg_circuit_params(self._h, L.dptr(p)))
        return p

    def initial_matrix(self, gmin=1e-12):
        i = self.info()
        a = np.zeros(i["nnz"])
        r = np.zeros(i["num_vars"])
        L.check(L.lib().nsg_circuit_initial_matrix(self._h, float(gmin), L.dptr(a), L.dptr(r)))
        return a, r

    def state_count(self) -> int:
        n = L.lib().nsg_circuit_state_count(self._h)
        if n < 0:
            L.check(n)
        return n

    def eval_matrix(self, mode, x, ctx, order, method, states, mos_rec, gmin=1e-12,
                    reltol=1e-3, abstol=1e-12):
        """One Newton iteration's matrix and rhs evaluated on the host
        (nsg_circuit_eval_matrix).  ctx = (ag0, ag1, ag2, xmu_ratio, delta,
        delta_old1, time); states (3 * state_count()) and mos_rec (12 per
        MOSFET) are float64 arrays updated in place."""
        i = self.info()
        a = np.zeros(i["nnz"])
        r = np.zeros(i["num_vars"])
        x = np.ascontiguousarray(x, np.float64)
        c = np.ascontiguousarray(ctx, np.float64)
        assert states.dtype == np.float64 and states.flags.c_contiguous
        assert mos_rec.dtype == np.float64 and mos_rec.flags.c_contiguous
        L.check(L.lib().nsg_circuit_eval_matrix(self._h, int(mode), L.dptr(x), L.dptr(c),
                                                int(order), int(method), float(gmin),
                                                float(reltol), float(abstol), L.dptr(states),
                                                L.dptr(mos_rec), L.dptr(a), L.dptr(r)))
        return a, r

    def __del__(self):
        if getattr(self, "_h", None) and L._lib is not None:
            L._lib.nsg_circuit_free(self._h)
            self._h = None


class DcBatch:
    """Batched DC operating point of finalized circuits (one CTA each)."""

    PER_INSTANCE = L.NSG_SYMBOLIC_PER_INSTANCE
    PER_PATTERN = L.NSG_SYMBOLIC_PER_PATTERN

    def __init__(self, circuits, symbolic=PER_PATTERN, threads=0):
        self.circuits = list(circuits)
        arr = (ctypes.c_void_p * len(self.circuits))(*[c.handle for c in self.circuits])
        h = ctypes.c_void_p()
        L.check(L.lib().nsg_dc_batch_create(len(self.circuits), arr, int(symbolic), int(threads),
                                            ctypes.byref(h)))
        self._h = h
        cnt = len(self.circuits) + 1
        self.param_offsets = np.zeros(cnt, np.int64)
        self.solution_offsets = np.zeros(cnt, np.int64)
        L.check(L.lib().nsg_dc_batch_layout(self._h, L.llptr(self.param_offsets),
                                            L.llptr(self.solution_offsets)))

    @property
    def count(self):
        return len(self.circuits)

    def stats(self) -> dict:
        n, nnz, nlu, upd = (ctypes.c_longlong() for _ in range(4))
        topo = ctypes.c_int()
        L.check(L.lib().nsg_dc_batch_stats(self._h, ctypes.byref(n), ctypes.byref(nnz),
                                           ctypes.byref(nlu), ctypes.byref(upd),
                                           ctypes.byref(topo)))
        return dict(n=n.value, nnz=nnz.value, nnz_lu=nlu.value, updates=upd.value,
                    topologies=topo.value)

    def instance_stats(self) -> dict:
        arrs = {k: np.zeros(self.count, np.int64) for k in ("n", "nnz", "nnz_lu", "updates")}
        L.check(L.lib().nsg_dc_batch_instance_stats(self._h, L.llptr(arrs["n"]),
                                                    L.llptr(arrs["nnz"]), L.llptr(arrs["nnz_lu"]),
                                                    L.llptr(arrs["updates"])))
        return arrs

    def set_options(self, reltol=1e-3, vntol=1e-6, abstol=1e-12, gmin=1e-12, max_iter=100):
        L.check(L.lib().nsg_dc_batch_set_options(self._h, reltol, vntol, abstol, gmin,
                                                 int(max_iter)))

    def set_reorder(self, enable: bool):
        L.check(L.lib().nsg_dc_batch_set_reorder(self._h, int(bool(enable))))

    def set_first_aid(self, aid: str):
        """Run every operating point through "direct" (the whole cascade of
        aids), or "source" / "gain" / "ptc" (source stepping, gain stepping or
        pseudo-transient continuation alone)."""
        L.check(L.lib().nsg_dc_batch_set_first_aid(self._h, AIDS[aid]))

    def reorders(self) -> int:
        n = ctypes.c_longlong()
        L.check(L.lib().nsg_dc_batch_reorders(self._h, ctypes.byref(n)))
        return n.value

    def set_graph(self, enable: bool = True):
        """Replay run()'s launch from a captured CUDA graph (see
        nsg_dc_batch_set_graph)."""
        L.check(L.lib().nsg_dc_batch_set_graph(self._h, int(bool(enable))))

    def set_row_maps(self, enable: bool = True):
        """Update destinations of the refactor from per-warp row maps
        instead of the plans' update maps (nsg_dc_batch_set_row_maps)."""
        L.check(L.lib().nsg_dc_batch_set_row_maps(self._h, int(bool(enable))))

    def graph_launches(self) -> int:
        n = ctypes.c_longlong()
        L.check(L.lib().nsg_dc_batch_graph_launches(self._h, ctypes.byref(n)))
        return n.value

    def engines(self) -> list:
        """Factorization engine of each instance: "markowitz" or "amdlu"
        (make_solver's choice for the circuit)."""
        out = np.zeros(self.count, np.int32)
        L.check(L.lib().nsg_dc_batch_engines(self._h, L.iptr(out)))
        return [ENGINE_NAMES.get(int(k)) for k in out]

    def methods(self):
        """(method, solves) per instance after a run: 0 direct Newton, 1 gmin
        stepping; Newton solves taken."""
        m = np.zeros(self.count, np.int32)
        n = np.zeros(self.count, np.int32)
        L.check(L.lib().nsg_dc_batch_methods(self._h, L.iptr(m), L.iptr(n)))
        return m, n

    def params(self):
        """Packed default parameters of all circuits (host)."""
        return np.concatenate([c.params() for c in self.circuits])

    def run(self, d_params=None, d_solutions=None, d_status=None, d_iterations=None,
            stream=None):
        """Launch the batched Newton solve; returns device tensors
        (solutions, status, iterations)."""
        import torch
        dev = torch.device("cuda")
        if d_solutions is None:
            d_solutions = torch.empty(int(self.solution_offsets[-1]), dtype=torch.float64, device=dev)
        if d_status is None:
            d_status = torch.empty(self.count, dtype=torch.int32, device=dev)
        if d_iterations is None:
            d_iterations = torch.empty(self.count, dtype=torch.int32, device=dev)
        sp = torch.cuda.current_stream().cuda_stream if stream is None else \
            getattr(stream, "cuda_stream", stream)
        L.check(L.lib().nsg_dc_batch_run(self._h, None if d_params is None else d_params.data_ptr(),
                                         d_solutions.data_ptr(), d_status.data_ptr(),
                                         d_iterations.data_ptr(), sp))
        return d_solutions, d_status, d_iterations

    def adjoint(self, d_solutions, d_cotangent, d_params=None, stream=None):
        """dL/dparams (device tensor, packed like params()) for cotangents
        dL/dx at the run's solutions; status per instance (0, or 102)."""
        import torch
        grads = torch.empty(int(self.param_offsets[-1]), dtype=torch.float64, device="cuda")
        status = torch.empty(self.count, dtype=torch.int32, device="cuda")
        sp = torch.cuda.current_stream().cuda_stream if stream is None else \
            getattr(stream, "cuda_stream", stream)
        L.check(L.lib().nsg_dc_batch_adjoint(
            self._h, None if d_params is None else d_params.data_ptr(), d_solutions.data_ptr(),
            d_cotangent.contiguous().data_ptr(), grads.data_ptr(), status.data_ptr(), sp))
        return grads, status

    def split(self, packed):
        arr = packed.cpu().numpy() if hasattr(packed, "cpu") else np.asarray(packed)
        o = self.solution_offsets
        return [arr[o[i]:o[i + 1]] for i in range(self.count)]

    def __del__(self):
        if getattr(self, "_h", None) and L._lib is not None:
            L._lib.nsg_dc_batch_free(self._h)
            self._h = None


class TranBatch:
    """Batched transient analysis of finalized circuits (one CTA each).

    ``probes`` are unknown indices (node voltages first, then branch
    currents) recorded at t = 0 and every accepted timepoint, at most
    ``max_points`` per circuit."""

    def __init__(self, circuits, tstep, tstop, probes, max_points=4096, threads=0):
        self.circuits = list(circuits)
        self.probes = np.ascontiguousarray(probes, np.int32)
        self.max_points = int(max_points)
        arr = (ctypes.c_void_p * len(self.circuits))(*[c.handle for c in self.circuits])
        h = ctypes.c_void_p()
        L.check(L.lib().nsg_tran_batch_create(len(self.circuits), arr, float(tstep), float(tstop),
                                              self.max_points, len(self.probes),
                                              L.iptr(self.probes), int(threads), ctypes.byref(h)))
        self._h = h

    @property
    def count(self):
        return len(self.circuits)

    def set_shape(self, threads: int = 0, blocks_per_sm: int = 0):
        """Launch shape of the transient kernel (nsg_tran_batch_set_shape;
        0, 0: automatic)."""
        L.check(L.lib().nsg_tran_batch_set_shape(self._h, int(threads), int(blocks_per_sm)))

    def run(self, stream=None):
        import torch
        sp = torch.cuda.current_stream().cuda_stream if stream is None else \
            getattr(stream, "cuda_stream", stream)
        L.check(L.lib().nsg_tran_batch_run(self._h, sp))

    def orderings(self) -> int:
        n = ctypes.c_longlong()
        L.check(L.lib().nsg_tran_batch_orderings(self._h, ctypes.byref(n)))
        return n.value

    # --- adjoint -------------------------------------------------------------
    def record(self, enable: bool = True):
        """Record each accepted step's integration formula and the operating
        point during the next run(), for adjoint()."""
        L.check(L.lib().nsg_tran_batch_record(self._h, int(bool(enable))))

    def set_adjoint_options(self, reltol=1e-3, vntol=1e-6, abstol=1e-12, max_iter=100):
        """Newton tolerances of the adjoint's re-solves of the recorded steps."""
        L.check(L.lib().nsg_tran_batch_set_adjoint_options(self._h, float(reltol), float(vntol),
                                                           float(abstol), int(max_iter)))

    def params(self):
        """(offsets [count+1], DC parameter vector, transient parameter
        vector): the packed circuit parameters (PULSE defaults resolved in
        the transient one)."""
        off = np.zeros(self.count + 1, np.int64)
        L.check(L.lib().nsg_tran_batch_params(self._h, L.llptr(off), None, None))
        dc = np.zeros(int(off[-1]))
        tr = np.zeros(int(off[-1]))
        L.check(L.lib().nsg_tran_batch_params(self._h, L.llptr(off), L.dptr(dc), L.dptr(tr)))
        return off, dc, tr

    def adjoint(self, probes, d_targets, weight=1.0, every=32, d_params_dc=None,
                d_params_tran=None, stream=None):
        """Loss w * sum_n (x_n[probe] - target_n)^2 over the recorded run's
        timepoints (targets packed like the output points: max_points per
        circuit) and its gradient with respect to the parameters (R, C,
        MOSFET W / L / VTO; others zero), by the discrete adjoint with a
        checkpoint every `every` steps.  Returns device tensors (grads packed
        like params(), loss per circuit, status per circuit)."""
        import torch
        off = np.zeros(self.count + 1, np.int64)
        L.check(L.lib().nsg_tran_batch_params(self._h, L.llptr(off), None, None))
        grads = torch.empty(int(off[-1]), dtype=torch.float64, device="cuda")
        loss = torch.empty(self.count, dtype=torch.float64, device="cuda")
        status = torch.empty(self.count, dtype=torch.int32, device="cuda")
        pr = np.ascontiguousarray(probes, np.int32)
        sp = torch.cuda.current_stream().cuda_stream if stream is None else \
            getattr(stream, "cuda_stream", stream)
        L.check(L.lib().nsg_tran_batch_adjoint(
            self._h, L.iptr(pr), d_targets.contiguous().data_ptr(), float(weight), int(every),
            None if d_params_dc is None else d_params_dc.data_ptr(),
            None if d_params_tran is None else d_params_tran.data_ptr(),
            grads.data_ptr(), loss.data_ptr(), status.data_ptr(), sp))
        return grads, loss, status

    def engines(self):
        """(DC engines, transient engines) per circuit: "markowitz",
        "amdlu", or None for a solver not ordered yet."""
        dc = np.zeros(self.count, np.int32)
        tr = np.zeros(self.count, np.int32)
        L.check(L.lib().nsg_tran_batch_engines(self._h, L.iptr(dc), L.iptr(tr)))
        return ([ENGINE_NAMES.get(int(k)) for k in dc], [ENGINE_NAMES.get(int(k)) for k in tr])

    def results(self):
        """Per circuit: dict(time, values [points x probes], status, steps,
        rejected, newton_iters)."""
        c, m, k = self.count, self.max_points, len(self.probes)
        t = np.zeros(c * m)
        v = np.zeros(c * m * k)
        npts = np.zeros(c, np.int32)
        st = np.zeros(c, np.int32)
        stats = np.zeros(4 * c, np.int32)
        L.check(L.lib().nsg_tran_batch_results(self._h, L.dptr(t), L.dptr(v), L.iptr(npts),
                                               L.iptr(st), L.iptr(stats)))
        out = []
        for i in range(c):
            p = int(npts[i])
            out.append(dict(time=t[i * m:i * m + p].copy(),
                            values=v[i * m * k:(i * m + p) * k].reshape(p, k).copy(),
                            status=int(st[i]), steps=int(stats[4 * i]),
                            rejected=int(stats[4 * i + 1]), newton_iters=int(stats[4 * i + 2]),
                            dc_code=int(stats[4 * i + 3])))
        return out

    def __del__(self):
        if getattr(self, "_h", None) and L._lib is not None:
            L._lib.nsg_tran_batch_free(self._h)
            self._h = None
