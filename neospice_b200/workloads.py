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

from .circuit import GND, Circuit


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
        dio = np.repeat([[self.diode_is, self.diode_n]], len(self.diode_nodes), axis=0).ravel()
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
