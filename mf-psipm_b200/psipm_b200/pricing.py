"""Pricing rounds of the V3.1 HSD loop on the device.

After the natural-residual test accepts a restricted proximal subproblem, the
reference prices every column of the full LP (psipm_v3_1_hsd.py:2101-2158):

    hsd_violation = A' y - c tau
    candidate     = inactive columns with hsd_violation > pricing_tolerance * max(tau, 1e-12),
                    at most pricing_batch of them (the largest violations)

With ``n`` in the millions this is one full sparse product and a selection
per round.  :class:`DevicePricing` keeps ``A`` and ``c`` on the device and
returns the same ``hsd_violation`` (bit-identical) and candidate set (ties at
the batch cut by ascending index; the reference's ``argpartition`` leaves
that choice to NumPy's build).  The caller keeps the rest of the round
(metrics, certificates, column elimination, pool update) as it is.
"""

from __future__ import annotations

import numpy as np

from .device import NormalEquationsDevice


class DevicePricing:
    """Device pricing for one LP (``A`` m x n, costs ``c``)."""

    def __init__(self, A, c, device: int = 0, dev: NormalEquationsDevice = None):
        self.dev = dev if dev is not None else NormalEquationsDevice(A, device=device)
        self.dev.price_load(np.asarray(c, dtype=np.float64))
        self.rounds = 0

    def price(self, y, tau: float, active: np.ndarray, pricing_tolerance: float, pricing_batch: int):
        """One round: returns ``(hsd_violation, candidate)`` with ``candidate``
        ascending column indices."""
        tau_scale = max(float(tau), 1.0e-12)
        violation, candidate = self.dev.price(y, float(tau), np.asarray(active, dtype=bool),
                                              float(pricing_tolerance) * tau_scale, int(pricing_batch))
        self.rounds += 1
        return violation, candidate

    def close(self) -> None:
        self.dev.close()
