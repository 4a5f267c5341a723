"""Reader of AMReX plotfiles ("HyperCLaw-V1.1" Header, VisMF MultiFab
headers, FAB data files), for the single-level files that
``LevelSolver.write_plotfile`` / ``ilbm_plotfile_write`` produce and the
reference's ``AmrCoreLBM::WritePlotFile`` (Source/Core/AmrCoreLBM.cpp:1908-1930
via AMReX's WriteMultiLevelPlotfile) writes for one level.

The layout read here is AMReX's published plotfile format:

* ``Header``: version line, component count and names, dimension, time,
  finest level, prob_lo, prob_hi, refinement ratios, per-level domain boxes,
  level steps and cell sizes, coordinate system, boundary width, then per
  level ``level ngrids time`` / ``step`` / one ``lo hi`` line per dimension per
  grid / the MultiFab path (``Level_0/Cell``);
* ``Level_0/Cell_H``: version, how, ncomp, ngrow, the BoxArray, the FabOnDisk
  list (file name, byte offset) and per-FAB component minima and maxima;
* ``Cell_D_*``: per FAB a text line ``FAB ((8, (...)),(8, (byte order)))``
  with the box and ncomp, then ncomp planes of doubles, i fastest.
"""
from __future__ import annotations

import re
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

_BOX = re.compile(r"\(\(([-\d,]+)\)\s*\(([-\d,]+)\)\s*\(([-\d,]+)\)\)")


def _box(text: str):
    m = _BOX.search(text)
    if not m:
        raise ValueError(f"no box in {text!r}")
    lo = tuple(int(v) for v in m.group(1).split(","))
    hi = tuple(int(v) for v in m.group(2).split(","))
    return lo, hi, m.end()


@dataclass
class Plotfile:
    names: list
    dim: int
    time: float
    finest_level: int
    prob_lo: tuple
    prob_hi: tuple
    domain: tuple            # (lo, hi) of level 0
    level_steps: list
    dx: tuple                # level 0 cell sizes
    grids: list              # level 0 grids in physical coordinates: [(lo[d], hi[d]) ...]
    cell_min: np.ndarray     # from Cell_H, per component
    cell_max: np.ndarray
    data: dict = field(default_factory=dict)  # name -> [nz, ny, nx] (nz = 1 in 2D)


def read_plotfile(path) -> Plotfile:
    """Reads a single-level plotfile with one grid (one FAB) on level 0."""
    root = Path(path)
    lines = (root / "Header").read_text().splitlines()
    it = iter(lines)
    version = next(it).strip()
    if not version.startswith("HyperCLaw"):
        raise ValueError(f"not an AMReX plotfile header: {version!r}")
    ncomp = int(next(it))
    names = [next(it).strip() for _ in range(ncomp)]
    dim = int(next(it))
    time = float(next(it))
    finest = int(next(it))
    prob_lo = tuple(float(v) for v in next(it).split())
    prob_hi = tuple(float(v) for v in next(it).split())
    next(it)  # refinement ratios (empty for one level)
    dom_lo, dom_hi, _ = _box(next(it))
    steps = [int(v) for v in next(it).split()]
    dx = tuple(float(v) for v in next(it).split())
    for _ in range(finest):
        next(it)
    next(it)  # coordinate system
    next(it)  # boundary width
    lev, ngrids, _t = next(it).split()
    next(it)  # level step
    grids = []
    for _ in range(int(ngrids)):
        grids.append([tuple(float(v) for v in next(it).split()) for _ in range(dim)])
    mf_path = next(it).strip()

    ch = (root / (mf_path + "_H")).read_text().splitlines()
    # version, how, ncomp, ngrow, "(nboxes 0", boxes..., ")", nfabs, FabOnDisk lines
    ncomp_h = int(ch[2])
    if ncomp_h != ncomp:
        raise ValueError("Cell_H component count differs from Header")
    nbox = int(ch[4].lstrip("(").split()[0])
    pos = 5 + nbox + 1
    nfab = int(ch[pos])
    fods = []
    for n in range(nfab):
        parts = ch[pos + 1 + n].split()
        fods.append((parts[1], int(parts[2])))
    rest = [l for l in ch[pos + 1 + nfab:] if l.strip()]
    cmin = np.array([float(v) for v in rest[1].rstrip(",").split(",")])
    cmax = np.array([float(v) for v in rest[3].rstrip(",").split(",")])
    if nfab != 1:
        raise ValueError("this reader takes one FAB per level")
    fname, off = fods[0]
    raw = (root / Path(mf_path).parent / fname).read_bytes()
    nl = raw.index(b"\n", off)
    head = raw[off:nl].decode()
    if not head.startswith("FAB "):
        raise ValueError(f"bad FAB header {head!r}")
    order = re.findall(r"\(8, \(([\d ]+)\)\)", head)
    if not order or order[-1].split()[0] not in ("8", "1"):
        raise ValueError(f"unsupported real descriptor in {head!r}")
    dt = np.dtype("<f8") if order[-1].split()[0] == "8" else np.dtype(">f8")
    blo, bhi, end = _box(head[head.index(")))") + 3:])
    nc = int(head[head.index(")))") + 3:][end:].split()[0])
    shape = [h - l + 1 for l, h in zip(blo, bhi)]
    n = int(np.prod(shape))
    vals = np.frombuffer(raw, dtype=dt, count=nc * n, offset=nl + 1).astype(np.float64)
    nx, ny = shape[0], shape[1]
    nz = shape[2] if dim == 3 else 1
    arr = vals.reshape(nc, nz, ny, nx)
    pf = Plotfile(names, dim, time, finest, prob_lo, prob_hi, (dom_lo, dom_hi), steps, dx, grids,
                  cmin, cmax)
    pf.data = {name: arr[c] for c, name in enumerate(names)}
    return pf


def plotfile_name(prefix: str, istep: int) -> str:
    """amrex::Concatenate(prefix, istep, 5), as PlotFileName builds it
    (Source/Core/AmrCoreLBM.cpp:1756-1758)."""
    return f"{prefix}{istep:05d}"
