"""Roberts low-discrepancy spread of initial candidates (opt/sampler.py:246-384).

The R_d sequence of M. Roberts ("The unreasonable effectiveness of
quasirandom sequences", 2018): with phi_d the real root of x^(d+1) = x + 1,
point n has coordinates frac(n * a_i), a_i = 1 - phi_d^-(i+1).  robokit
offsets the points to [-0.5, 0.5) and scales them per tangent column; with
`keep_first`, candidate 0 gets zero noise and sits on the seed.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Optional, Sequence, Union

import numpy as np


def roberts_samples(num_points: int, dim: int, offset: int = 0) -> np.ndarray:
    """Low-discrepancy points in [0, 1), shape (num_points, dim)."""
    x = 1.0
    for _ in range(10000):  # Newton on x^(d+1) - x - 1
        f = x ** (dim + 1) - x - 1.0
        x -= f / ((dim + 1) * x ** dim - 1.0)
        if abs(f) < 1e-10:
            break
    alpha = 1.0 - x ** -(1.0 + np.arange(dim))
    n = np.arange(num_points, dtype=np.float64) + offset
    return np.modf(n[:, None] * alpha[None, :])[0]


@dataclass(frozen=True)
class RobertsSamplerConfig:
    """Spread settings: `scale` is the half-width per tangent column (IK helpers scale it by joint range)."""

    scale: Union[float, Sequence[float]] = 0.2
    seed: Optional[int] = None
    keep_first: bool = False
    num_draws: int = 1


class RobertsSampler:
    """Candidate c of every instance gets offset row c (instance-major batches)."""

    def __init__(self, num_candidates: int, tangent_dim: int, seed: Optional[int] = None, keep_first: bool = False):
        off = roberts_samples(num_candidates, tangent_dim, (seed % 10000) if seed is not None else 0) - 0.5
        if keep_first:
            off = np.vstack([np.zeros_like(off[:1]), off[:-1]])
        self.num_candidates = num_candidates
        self.offsets = off.astype(np.float32)

    def tangent(self, batch: int, scale: np.ndarray) -> np.ndarray:
        """Noise for `batch` instances x num_candidates, [batch * num_candidates, tangent_dim]."""
        return np.ascontiguousarray(np.tile(self.offsets * np.asarray(scale, np.float32)[None, :], (batch, 1)))
