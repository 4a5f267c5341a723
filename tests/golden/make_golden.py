"""Generates the golden fixtures in this directory from the reference's own
code (oracle/_ref: Source/LBM, Source/BC, Source/IBM compiled in place against
oracle/amrex_shim by ``make -C oracle ref REF=<reference tree>``).  Run from
the repository root:  python tests/golden/make_golden.py [name ...]
(no names: every case of golden_cases.GOLDEN_CASES).

Each fixture stores the step count and the reference's macro fields, force
field, per-direction population sums, the populations themselves for the
smaller cases and (for IB cases) the force record after the steps; inputs are regenerated from the
case builders in ilbmrex_b200.cases.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle.checker import CpuLevel  # noqa: E402
from tests.golden.golden_cases import GOLDEN_CASES  # noqa: E402


def main():
    out = Path(__file__).resolve().parent
    names = sys.argv[1:] or list(GOLDEN_CASES)
    for name in names:
        builder, steps = GOLDEN_CASES[name]
        case, init, ib = builder()
        L = CpuLevel(case, "ref")
        L.set_macro(*init())
        L.init_equilibrium()
        if ib is not None:
            L.ib_create(ib)
        L.step(steps)
        f = L.get_f()
        data = dict(macro=L.get_macro(), force=L.get_force(), steps=steps,
                    f_sum=f.reshape(f.shape[0], -1).sum(axis=1))
        if f.size <= 200_000:  # keep the committed fixtures small
            data["f"] = f
        if ib is not None:
            data["rec"] = L.force_record()
            data["fsum"] = L.marker_force_sum()
            data["nmark"] = L.num_markers()
        np.savez_compressed(out / f"{name}.npz", **data)
        print(f"wrote {name}.npz")


if __name__ == "__main__":
    main()
