"""Discrete velocity sets, in the direction order of the reference's input decks.

The reference reads the lattice from its input deck (``lbm2d|lbm3d.{ndir, wis,
wim, dirx, diry, dirz}``, Source/Core/AmrCoreLBM.cpp:1212-1236) and computes
``w_q = wis_q / wim_q`` in floating point.  The CUDA kernels bake these three
orderings in as compile-time tables, so a deck must use one of them:

* D2Q9  -- Examples/Cylinder_flow/inputs:35-40
* D3Q19 -- Examples/SquareDuct_flow/inputs:36-41
* D3Q27 -- Examples/Sphere_flow/inputs:34-39
"""
from __future__ import annotations

from dataclasses import dataclass


@dataclass(frozen=True)
class Lattice:
    name: str
    dim: int
    c: tuple  # ((cx, cy, cz), ...) in deck order
    wis: tuple
    wim: tuple

    @property
    def q(self) -> int:
        return len(self.c)

    @property
    def w(self) -> tuple:
        return tuple(a / b for a, b in zip(self.wis, self.wim))

    def opposite(self, q: int) -> int:
        cx, cy, cz = self.c[q]
        for p, (ax, ay, az) in enumerate(self.c):
            if (ax, ay, az) == (-cx, -cy, -cz):
                return p
        raise ValueError("lattice without opposite direction")


def _mk(name, dim, dirx, diry, dirz, wis, wim):
    c = tuple((float(a), float(b), float(z)) for a, b, z in zip(dirx, diry, dirz))
    return Lattice(name, dim, c, tuple(float(x) for x in wis), tuple(float(x) for x in wim))


D2Q9 = _mk(
    "D2Q9", 2,
    [0, 1, 0, -1, 0, 1, -1, -1, 1],
    [0, 0, 1, 0, -1, 1, 1, -1, -1],
    [0] * 9,
    [4, 1, 1, 1, 1, 1, 1, 1, 1],
    [9, 9, 9, 9, 9, 36, 36, 36, 36],
)

D3Q19 = _mk(
    "D3Q19", 3,
    [0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0],
    [0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1],
    [0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1],
    [12, 2, 2, 2, 2, 2, 2, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1],
    [36] * 19,
)

D3Q27 = _mk(
    "D3Q27", 3,
    [0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1],
    [0, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1],
    [0, 0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1],
    [8, 2, 2, 2, 2, 2, 2, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1],
    [27, 27, 27, 27, 27, 27, 27, 54, 54, 54, 54, 54, 54, 54, 54, 54, 54, 54, 54,
     216, 216, 216, 216, 216, 216, 216, 216],
)

LATTICES = {"D2Q9": D2Q9, "D3Q19": D3Q19, "D3Q27": D3Q27}
LATTICE_ID = {"D2Q9": 0, "D3Q19": 1, "D3Q27": 2}
