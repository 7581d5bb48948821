"""Seeded synthetic workloads.

Diode-clamped resistor mesh (the batched DC operating-point workload): a
side x side grid of nodes, node (x, y) numbered y*side + x; resistors between
horizontal and vertical neighbours, lognormal around 1 kOhm (sigma 0.1);
level-1 diodes (IS = 1e-14, N = 1) from a seeded 5% of the nodes to ground
(never at the source corner, whose 1 V source would otherwise drive the diode
at hundreds of amperes); DC current sources of U(0, 1 mA) into a seeded 2% of
the nodes; a 1 V source from node 0 to ground.  Devices are created
resistors (horizontal rows, then vertical), diodes, current sources, source.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from .circuit import GND, Circuit, diode_params


@dataclasses.dataclass
class DiodeMesh:
    side: int
    r_h: np.ndarray        # (side-1)*side horizontal resistors, row by row
    r_v: np.ndarray        # side*(side-1) vertical resistors
    diode_nodes: np.ndarray
    isrc_nodes: np.ndarray
    isrc_amps: np.ndarray
    v_corner: float = 1.0
    diode_is: float = 1e-14
    diode_n: float = 1.0

    @property
    def num_nodes(self):
        return self.side * self.side

    @property
    def num_vars(self):
        return self.num_nodes + 1

    def build(self) -> Circuit:
        s = self.side
        c = Circuit(s * s)
        grid = np.arange(s * s, dtype=np.int32).reshape(s, s)   # [y, x]
        c.add_resistors(grid[:, :-1].ravel(), grid[:, 1:].ravel(), self.r_h)
        c.add_resistors(grid[:-1, :].ravel(), grid[1:, :].ravel(), self.r_v)
        nd = len(self.diode_nodes)
        c.add_diodes(self.diode_nodes, np.full(nd, GND, np.int32), self.diode_is, self.diode_n)
        ni = len(self.isrc_nodes)
        c.add_isources(np.full(ni, GND, np.int32), self.isrc_nodes, self.isrc_amps)
        c.V(0, GND, self.v_corner)
        return c.finalize()

    def params(self) -> np.ndarray:
        """Parameters in the circuit's creation order."""
        block = diode_params(self.diode_is, self.diode_n)
        dio = np.repeat(block[None, :], len(self.diode_nodes), axis=0).ravel()
        return np.concatenate([self.r_h, self.r_v, dio, self.isrc_amps, [self.v_corner]])


def diode_mesh(rng: np.random.Generator, side: int | None = None, side_range=(16, 96)) -> DiodeMesh:
    if side is None:
        side = int(rng.integers(side_range[0], side_range[1] + 1))
    n = side * side
    r_h = 1000.0 * np.exp(0.1 * rng.standard_normal((side - 1) * side))
    r_v = 1000.0 * np.exp(0.1 * rng.standard_normal(side * (side - 1)))
    dmask = rng.random(n) < 0.05
    dmask[0] = False
    imask = rng.random(n) < 0.02
    isrc = np.nonzero(imask)[0].astype(np.int32)
    amps = rng.uniform(0.0, 1e-3, len(isrc))
    return DiodeMesh(side, r_h, r_v, np.nonzero(dmask)[0].astype(np.int32), isrc, amps)


def diode_mesh_batch(count: int, seed: int = 0, side_range=(16, 96)):
    """`count` independent meshes; instance i uses the seed sequence (seed, i)."""
    return [diode_mesh(np.random.default_rng([seed, i]), side_range=side_range)
            for i in range(count)]


@dataclasses.dataclass
class Netlist:
    """A circuit as an ordered device list, built through the typed API in
    list order (so node numbering and device load order are fixed).  Devices:
    ("R", a, b, ohms), ("C", a, b, farads), ("V", p, n, volts),
    ("I", p, n, amps), ("VPULSE"|"IPULSE", p, n, v1, v2, td, tr, tf, pw, per),
    ("VPWL"|"IPWL", p, n, t0, v0, t1, v1, ...), ("D", anode, cathode, IS, N) or
    ("D", anode, cathode, IS, N, CJO, VJ, M, FC, TT).
    ("M", d, g, s, b, model_name, W, L[, delvto]) with models[model_name] =
    ("nmos"|"pmos", {param: value}): a level-1 card, or a BSIM4v7 card when
    its parameters hold LEVEL=14 (DELVTO only on BSIM4v7 instances).  Node
    -1 is ground."""
    num_nodes: int
    devices: list
    models: dict = dataclasses.field(default_factory=dict)

    def build(self, temp: float | None = None) -> Circuit:
        """The finalized circuit (at `temp` kelvin when given: the circuit
        temperature DIOtemp / MOS1temp apply); ``self.param_index`` receives
        the index of each device's first parameter (creation order), the
        layout of Circuit.params()."""
        c = Circuit(self.num_nodes)
        if temp is not None:
            c.set_temperature(temp)
        mid, b4 = {}, set()
        for name, (t, p) in self.models.items():
            if int(p.get("LEVEL", 1)) == 14:
                mid[name] = c.model_bsim4(t, **p)
                b4.add(name)
            else:
                mid[name] = c.model_mos1(t, **p)
        first = []
        for d in self.devices:
            kind, a, b, vals = d[0], d[1], d[2], d[3:]
            if kind == "M" and vals[2] in b4:
                k = c.M4(a, b, vals[0], vals[1], mid[vals[2]], vals[3], vals[4],
                         vals[5] if len(vals) > 5 else 0.0)
            elif kind == "M":
                k = c.M(a, b, vals[0], vals[1], mid[vals[2]], vals[3], vals[4])
            elif kind == "R":
                k = c.R(a, b, vals[0])
            elif kind == "C":
                k = c.C(a, b, vals[0], vals[1] if len(vals) > 1 else None)
            elif kind == "V":
                k = c.V(a, b, vals[0])
            elif kind == "I":
                k = c.I(a, b, vals[0])
            elif kind in ("VPULSE", "IPULSE"):
                k = (c.VPULSE if kind[0] == "V" else c.IPULSE)(a, b, *vals)
            elif kind in ("VPWL", "IPWL"):
                pts = np.asarray(vals, np.float64).reshape(-1, 2)
                k = (c.VPWL if kind[0] == "V" else c.IPWL)(a, b, pts)
            elif kind == "D":
                k = c.D(a, b, *vals)
            else:
                raise ValueError(f"unknown device kind {kind!r}")
            first.append(k)
        self.param_index = first
        return c.finalize()


def rc_ladder(rng: np.random.Generator, stages: int, r_ohm=1e3, c_farad=1e-12, sigma=0.2,
              period=2e-9) -> Netlist:
    """A PULSE(0 1 0 100p 100p period/2-100p period) source at node 0 driving
    an RC ladder of `stages` sections: R (lognormal around r_ohm) from node
    i to node i+1, C (lognormal around c_farad) from node i+1 to ground."""
    dev = [("VPULSE", 0, GND, 0.0, 1.0, 0.0, 1e-10, 1e-10, period / 2 - 1e-10, period)]
    r = r_ohm * np.exp(sigma * rng.standard_normal(stages))
    cc = c_farad * np.exp(sigma * rng.standard_normal(stages))
    for i in range(stages):
        dev.append(("R", i, i + 1, float(r[i])))
        dev.append(("C", i + 1, GND, float(cc[i])))
    return Netlist(stages + 1, dev)


def rc_tree(rng: np.random.Generator, nodes: int, r_ohm=50.0, c_farad=2e-15, sigma=0.2,
            r_drive=1e3) -> Netlist:
    """A random RC interconnect tree: node 0 is the driver node (a 0 -> 1 V
    PULSE through r_drive), each node k >= 1 hangs from a uniformly drawn
    earlier node by a resistor (lognormal around r_ohm) and has a capacitor
    to ground (lognormal around c_farad).  The last node is the far end."""
    dev = [("VPULSE", nodes, GND, 0.0, 1.0, 1e-11, 5e-11, 5e-11, 1e-9, 2e-9),
           ("R", nodes, 0, r_drive)]
    r = r_ohm * np.exp(sigma * rng.standard_normal(nodes))
    cc = c_farad * np.exp(sigma * rng.standard_normal(nodes))
    parent = [0] + [int(rng.integers(0, k)) for k in range(1, nodes)]
    for k in range(1, nodes):
        dev.append(("R", parent[k], k, float(r[k])))
    for k in range(nodes):
        dev.append(("C", k, GND, float(cc[k])))
    return Netlist(nodes + 1, dev)


def inverter_chain(stages: int, vin=0.0, vdd=1.8, c_load=10e-15, pulse=None) -> Netlist:
    """A chain of `stages` CMOS inverters (level-1: NMOS VTO=0.7 KP=110u
    W/L=2u/1u, PMOS VTO=-0.7 KP=50u W/L=4u/1u), a load capacitor per stage
    output, VDD on node 0, the input on node 1 (a DC value, or
    pulse=(v1, v2, td, tr, tf, pw, per)), stage k's output on node k+2."""
    models = {"nch": ("nmos", {"VTO": 0.7, "KP": 110e-6}),
              "pch": ("pmos", {"VTO": -0.7, "KP": 50e-6})}
    dev = [("V", 0, GND, vdd)]
    dev.append(("VPULSE", 1, GND, *pulse) if pulse is not None else ("V", 1, GND, vin))
    for k in range(stages):
        i, o = k + 1, k + 2
        dev.append(("M", o, i, GND, GND, "nch", 2e-6, 1e-6))
        dev.append(("M", o, i, 0, 0, "pch", 4e-6, 1e-6))
        dev.append(("C", o, GND, c_load))
    return Netlist(stages + 2, dev, models)


def inverter_ring(stages: int, vdd=1.8, lam=0.0, c_load=10e-15) -> Netlist:
    """A ring of `stages` CMOS inverters (level-1 cards of inverter_chain,
    optional channel-length modulation), each output loaded by c_load; node
    0 is VDD, node i the output of stage i (driven by stage i-1)."""
    dev = [("V", 0, GND, vdd)]
    for i in range(stages):
        inp, out = 1 + (i - 1) % stages, 1 + i
        dev += [("M", out, inp, GND, GND, "nch", 2e-6, 1e-6), ("M", out, inp, 0, 0, "pch", 4e-6, 1e-6),
                ("C", out, GND, c_load)]
    pn, pp = {"VTO": 0.7, "KP": 1.1e-4}, {"VTO": -0.7, "KP": 5e-5}
    if lam:
        pn["LAMBDA"] = pp["LAMBDA"] = lam
    return Netlist(stages + 1, dev, {"nch": ("nmos", pn), "pch": ("pmos", pp)})


def diode_grid(rng: np.random.Generator, side: int, vdd=1.0) -> Netlist:
    """A side x side resistor grid as a Netlist: R ~ lognormal(ln 1k, 0.1),
    diodes (IS 1e-14, N 1) from a seeded 10% of the nodes to ground, 0-1 mA
    current sources into 5%, a source of vdd at node 0."""
    n = side * side
    dev = [("V", 0, GND, vdd)]
    for y in range(side):
        for x in range(side):
            k = y * side + x
            if x + 1 < side:
                dev.append(("R", k, k + 1, float(rng.lognormal(np.log(1e3), 0.1))))
            if y + 1 < side:
                dev.append(("R", k, k + side, float(rng.lognormal(np.log(1e3), 0.1))))
    for k in range(1, n):
        u = rng.random()
        if u < 0.10:
            dev.append(("D", k, GND, 1e-14, 1.0))
        elif u < 0.15:
            dev.append(("I", GND, k, float(rng.uniform(0.0, 1e-3))))
    return Netlist(n, dev)


def mos_network(rng: np.random.Generator, nodes: int, vdd=1.8, pulse=None) -> Netlist:
    """A seeded MOS network: VDD on node 0, an input on node 1 (a random DC
    level, or a PULSE), and for every further node an NMOS pull-down and a
    PMOS pull-up whose gates hang from random earlier nodes, a resistor to a
    random earlier node and a capacitor to ground.  The cards exercise body
    effect, channel-length modulation, lateral diffusion and oxide-derived
    parameters."""
    models = {
        "n1": ("nmos", {"VTO": 0.6, "KP": 120e-6, "GAMMA": 0.4, "PHI": 0.7, "LAMBDA": 0.05,
                        "LD": 5e-8}),
        "p1": ("pmos", {"VTO": -0.65, "KP": 45e-6, "GAMMA": 0.5, "LAMBDA": 0.08}),
        "n2": ("nmos", {"TOX": 2e-8, "NSUB": 1e16, "U0": 500, "LAMBDA": 0.02}),
    }
    vin = float(rng.uniform(0, vdd))
    dev = [("V", 0, GND, vdd),
           ("VPULSE", 1, GND, *pulse) if pulse is not None else ("V", 1, GND, vin)]
    for k in range(2, nodes):
        g1, g2 = int(rng.integers(1, k)), int(rng.integers(1, k))
        nm = "n1" if rng.random() < 0.6 else "n2"
        dev.append(("M", k, g1, GND, GND, nm, float(rng.uniform(1e-6, 4e-6)), 1e-6))
        dev.append(("M", k, g2, 0, 0, "p1", float(rng.uniform(2e-6, 8e-6)), 1e-6))
        dev.append(("R", k, int(rng.integers(1, k)),
                    float(np.exp(rng.uniform(np.log(1e3), np.log(1e6))))))
        dev.append(("C", k, GND, 1e-14))
    return Netlist(nodes, dev, models)


def inverter_chain_mc(rng: np.random.Generator, stages: int = 32, sigma_vto=0.03,
                      sigma_kp=0.05, pulse=(0.0, 1.8, 0.0, 1e-10, 1e-10, 1e-9, 2e-9)) -> Netlist:
    """A Monte Carlo variant of inverter_chain: the NMOS and PMOS threshold
    voltages drawn with a Gaussian sigma_vto (V) and the transconductances
    with a relative Gaussian sigma_kp, per instance, from rng."""
    nl = inverter_chain(stages, pulse=pulse)
    dv = sigma_vto * rng.standard_normal(2)
    dk = 1.0 + sigma_kp * rng.standard_normal(2)
    nl.models = {"nch": ("nmos", {"VTO": 0.7 + dv[0], "KP": 110e-6 * dk[0]}),
                 "pch": ("pmos", {"VTO": -0.7 + dv[1], "KP": 50e-6 * dk[1]})}
    return nl


def resistor_network(rng: np.random.Generator, nodes: int) -> Netlist:
    """A seeded linear resistor network: a 1 V source on node 0, every further
    node tied to a random earlier node and to ground by resistors (lognormal
    around 1 kOhm), current sources of U(0, 1 mA) into a third of the nodes."""
    dev = [("V", 0, GND, 1.0)]
    for k in range(1, nodes):
        dev.append(("R", int(rng.integers(0, k)), k, float(1e3 * np.exp(0.3 * rng.standard_normal()))))
        dev.append(("R", k, GND, float(1e3 * np.exp(0.3 * rng.standard_normal()))))
        if rng.random() < 1 / 3:
            dev.append(("I", GND, k, float(rng.uniform(0, 1e-3))))
    return Netlist(nodes, dev)


def power_grid(rng: np.random.Generator, side: int, pad_pitch: int, n_loads: int,
               r_ohm=0.1, r_sigma=0.05, c_farad=1e-12, i_max=5e-3, t_edge=1e-9,
               t_rise=5e-11, vdd=1.0) -> Netlist:
    """An on-chip power grid: a side x side mesh of resistors (lognormal
    around r_ohm) with a decoupling capacitor c_farad from every node to
    ground, vdd pads (DC voltage sources to ground) on a lattice of pitch
    pad_pitch starting at (pitch/2, pitch/2), and n_loads PWL current loads
    to ground at random nodes, each stepping from 0 to U(0, i_max) over
    t_rise at a random time in [0, t_edge].  Node (x, y) is y*side + x."""
    dev = []
    n = side * side
    r = r_ohm * np.exp(r_sigma * rng.standard_normal(2 * side * (side - 1)))
    k = 0
    for y in range(side):
        for x in range(side - 1):
            dev.append(("R", y * side + x, y * side + x + 1, float(r[k])))
            k += 1
    for y in range(side - 1):
        for x in range(side):
            dev.append(("R", y * side + x, (y + 1) * side + x, float(r[k])))
            k += 1
    for i in range(n):
        dev.append(("C", i, GND, float(c_farad)))
    h = pad_pitch // 2
    for y in range(h, side, pad_pitch):
        for x in range(h, side, pad_pitch):
            dev.append(("V", y * side + x, GND, float(vdd)))
    nodes = rng.choice(n, size=n_loads, replace=n_loads > n)
    amps = rng.uniform(0.0, i_max, n_loads)
    edges = rng.uniform(0.0, t_edge, n_loads)
    for node, a, t0 in zip(nodes, amps, edges):
        dev.append(("IPWL", int(node), GND, 0.0, 0.0, float(t0), 0.0, float(t0 + t_rise),
                    float(a)))
    return Netlist(n, dev)


def rc_tree_driven(rng: np.random.Generator, nodes: int, r_ohm=50.0, c_farad=2e-15, sigma=0.2,
                   vdd=1.8, w_n=20e-6, w_p=40e-6, l=1e-6,
                   pulse=(0.0, 1.8, 1e-11, 5e-11, 5e-11, 1e-9, 2e-9)) -> Netlist:
    """A random RC interconnect tree (as rc_tree: node k >= 1 hangs from a
    uniformly drawn earlier node by a lognormal resistor, a lognormal
    capacitor from every node to ground) driven at node 0 by a level-1 CMOS
    inverter (NMOS VTO=0.7 KP=110u W=w_n, PMOS VTO=-0.7 KP=50u W=w_p, L=l)
    whose gate (node nodes) carries a PULSE; VDD on node nodes+1.  The last
    tree node is the far end."""
    models = {"nch": ("nmos", {"VTO": 0.7, "KP": 110e-6}),
              "pch": ("pmos", {"VTO": -0.7, "KP": 50e-6})}
    gate, vddn = nodes, nodes + 1
    dev = [("V", vddn, GND, vdd), ("VPULSE", gate, GND, *pulse),
           ("M", 0, gate, GND, GND, "nch", w_n, l), ("M", 0, gate, vddn, vddn, "pch", w_p, l)]
    r = r_ohm * np.exp(sigma * rng.standard_normal(nodes))
    cc = c_farad * np.exp(sigma * rng.standard_normal(nodes))
    parent = [0] + [int(rng.integers(0, k)) for k in range(1, nodes)]
    for k in range(1, nodes):
        dev.append(("R", parent[k], k, float(r[k])))
    for k in range(nodes):
        dev.append(("C", k, GND, float(cc[k])))
    return Netlist(nodes + 2, dev, models)


def bsim4_ring_nand(rng: np.random.Generator | None = None, stages: int = 25, vdd: float = 1.2,
                    l: float = 90e-9, w_n: float = 200e-9, w_p: float = 400e-9,
                    sigma_vth0: float = 0.030, toxe_spread: float = 0.03,
                    ramp: float = 50e-12) -> Netlist:
    """BSIM4v7 Monte Carlo circuit of 200 MOSFETs: a `stages`-stage inverter
    ring oscillator (ring node i driven by stage i-1), and a chain of
    `stages` two-input NAND gates, each followed by an inverter: NAND k takes
    ring node k and the previous AND output (VDD for the first), so the chain
    ANDs the ring's taps.  Default BSIM4v7 cards (LEVEL=14), L = 90n,
    W_n = 200n, W_p = 400n.  With `rng`, every MOSFET gets its own card with
    TOXE uniform within +-toxe_spread of the default 3 nm and a DELVTO drawn
    Gaussian with sigma_vth0 (the per-device VTH0 variation); without it,
    the nominal circuit (two shared cards).  VDD ramps 0 -> vdd in `ramp`
    (PWL), the ring's start-up kick.  Nodes: 0 VDD, 1..S ring, then per
    stage the NAND output, the NAND's series node and the AND output."""
    S = stages
    vddn = 0
    ring = [1 + i for i in range(S)]
    nand_out = [1 + S + 3 * k for k in range(S)]
    nand_mid = [2 + S + 3 * k for k in range(S)]
    and_out = [3 + S + 3 * k for k in range(S)]
    models = {}
    dev = [("VPWL", vddn, GND, 0.0, 0.0, ramp, vdd)]
    count = [0]

    def fet(kind, d, g, s, b, w):
        count[0] += 1
        if rng is None:
            name = "nch" if kind == "n" else "pch"
            if name not in models:
                models[name] = ("nmos" if kind == "n" else "pmos", {"LEVEL": 14})
            dev.append(("M", d, g, s, b, name, w, l))
            return
        name = f"{kind}{count[0]}"
        toxe = 3.0e-9 * (1.0 + toxe_spread * (2.0 * rng.random() - 1.0))
        models[name] = ("nmos" if kind == "n" else "pmos", {"LEVEL": 14, "TOXE": toxe})
        dev.append(("M", d, g, s, b, name, w, l, float(sigma_vth0 * rng.standard_normal())))

    for i in range(S):
        inp, out = ring[(i - 1) % S], ring[i]
        fet("n", out, inp, GND, GND, w_n)
        fet("p", out, inp, vddn, vddn, w_p)
    for k in range(S):
        a = ring[k]
        b = vddn if k == 0 else and_out[k - 1]
        o, m = nand_out[k], nand_mid[k]
        fet("n", o, a, m, GND, w_n)      # series pull-down
        fet("n", m, b, GND, GND, w_n)
        fet("p", o, a, vddn, vddn, w_p)  # parallel pull-up
        fet("p", o, b, vddn, vddn, w_p)
        fet("n", and_out[k], o, GND, GND, w_n)
        fet("p", and_out[k], o, vddn, vddn, w_p)
    return Netlist(1 + S + 3 * S, dev, models)


def ac_system(netlist: Netlist):
    """The small-signal system of a linear R / C / V netlist for an AC sweep
    (the matrices the reference's solve_ac builds, src/core/ac.cpp:113-140):
    (n, col_ptr, row_idx, g, c, b) with G the conductance and source-incidence
    values at the circuit's pattern slots, C the capacitor stamps (+C on the
    diagonal slots of both terminals, -C on the two coupling slots) and b the
    excitation: 1 V AC on the first voltage source's branch.  The matrix at
    angular frequency w is G + jwC (ax = (g, w*c) per slot)."""
    circ = netlist.build()
    cp, ri = circ.pattern()
    g, _ = circ.initial_matrix(0.0)
    n = len(cp) - 1
    c = np.zeros(len(ri))

    def slot(r, col):
        lo, hi = cp[col], cp[col + 1]
        k = lo + int(np.searchsorted(ri[lo:hi], r))
        assert k < hi and ri[k] == r
        return k

    for d in netlist.devices:
        if d[0] != "C":
            continue
        a, b_, farads = d[1], d[2], d[3]
        if a >= 0:
            c[slot(a, a)] += farads
        if b_ >= 0:
            c[slot(b_, b_)] += farads
        if a >= 0 and b_ >= 0:
            c[slot(a, b_)] -= farads
            c[slot(b_, a)] -= farads
    b = np.zeros(n, dtype=complex)
    branch = netlist.num_nodes  # branches follow the nodes; the first V source's
    b[branch] = 1.0             # branch is the first branch unknown when it is the only one
    return n, cp, ri, g, c, b


def rc_mesh(rng: np.random.Generator, side: int, r_ohm=10.0, c_farad=1e-13,
            sigma=0.1) -> Netlist:
    """An RC mesh for AC sweeps: side x side nodes, lognormal resistors to
    the four neighbours, a lognormal capacitor from every node to ground, a
    source resistor from the 1 V (AC) source at node 0 into the corner."""
    n = side * side
    src = n
    dev = [("V", src, GND, 1.0), ("R", src, 0, 50.0)]
    for y in range(side):
        for x in range(side):
            k = y * side + x
            if x + 1 < side:
                dev.append(("R", k, k + 1, float(r_ohm * np.exp(sigma * rng.standard_normal()))))
            if y + 1 < side:
                dev.append(("R", k, k + side, float(r_ohm * np.exp(sigma * rng.standard_normal()))))
            dev.append(("C", k, GND, float(c_farad * np.exp(sigma * rng.standard_normal()))))
    return Netlist(n + 1, dev)


def power_grid_transient(side: int, seed: int = 2026):
    """The transient companion matrix of the seeded side x side power grid
    (power_grid with VDD pads on a pitch-50 lattice and side^2/100 loads):
    conductances plus C/h on every capacitor node's diagonal (1 pF, h =
    10 ps).  Returns (n, col_ptr, row_idx, values) of the CSC pattern."""
    nl = power_grid(np.random.default_rng(seed), side, 50, max(1, side * side // 100))
    c = nl.build()
    cp, ri = c.pattern()
    g, _ = c.initial_matrix(0.0)
    n = len(cp) - 1
    cols = np.repeat(np.arange(n), np.diff(cp))
    capn = np.zeros(n, bool)
    capn[[d[1] for d in nl.devices if d[0] == "C"]] = True
    tran = g.copy()
    tran[(ri == cols) & capn[cols]] += 1e-12 / 1e-11
    return n, cp, ri, tran
