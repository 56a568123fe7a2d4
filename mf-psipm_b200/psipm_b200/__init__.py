"""psipm_b200 — B200-native normal-equations inner solve for MF-PSIPM.

Host-side mirror of the reference's KKT solver interfaces; all arithmetic
proportional to the LP runs in libpsipm_b200.so (CUDA, sm_100a).

* :mod:`psipm_b200.kkt`        drop-in KKT solvers (PS-IPM and HSD protocols)
* :mod:`psipm_b200.hsd`        reduced HSD Newton system over the device solve
* :mod:`psipm_b200.device`     one LP's device state (C-ABI handle)
* :mod:`psipm_b200.synthetic`  seeded synthetic LPs
"""

from ._lib import GpuUnavailable, load as load_library  # noqa: F401
from .synthetic import StandardLP  # noqa: F401

__all__ = ["GpuUnavailable", "load_library", "StandardLP"]
