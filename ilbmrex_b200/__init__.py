"""B200-native (sm_100a) per-level hot path of iLBMReX.

The CUDA kernels and the C ABI live in ``csrc/`` and ``lib/libilbm_b200.so``
(declared in ``include/ilbm_b200.h``).  This package holds the host-side
mirror of the reference's per-level interface:

* :mod:`ilbmrex_b200.capi`    -- ctypes binding of the C ABI;
* :mod:`ilbmrex_b200.lattice` -- D2Q9 / D3Q19 / D3Q27 in the reference deck order;
* :mod:`ilbmrex_b200.cases`   -- level / marker-IB case descriptions and the
  synthetic workloads;
* :mod:`ilbmrex_b200.level`   -- ``LevelSolver``: AdvancePhiAtLevel /
  update_forcing / ComputeIBForce for one level on one GPU.

There is no CPU fallback: without the built library every call raises.
"""
from . import capi, cases, lattice  # noqa: F401

__all__ = ["capi", "cases", "lattice", "LevelSolver", "Context"]


def __getattr__(name):
    if name in ("LevelSolver", "Context"):
        from . import level
        return getattr(level, name)
    raise AttributeError(name)
