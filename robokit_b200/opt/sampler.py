"""Roberts low-discrepancy spread of initial candidates (opt/sampler.py:246-384).

The R_d sequence of M. Roberts ("The unreasonable effectiveness of
quasirandom sequences", 2018): with phi_d the real root of x^(d+1) = x + 1,
point n has coordinates frac(n * a_i), a_i = 1 - phi_d^-(i+1).  robokit
offsets the points to [-0.5, 0.5) and scales them per tangent column; with
`keep_first`, candidate 0 gets zero noise and sits on the seed.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Any, Optional, Sequence, Union

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


class _Scale:
    """Per-column half-width of a sampler; `assign` replaces it between solves (opt/sampler.py:330-333)."""

    def __init__(self, values: np.ndarray):
        self._v = np.asarray(values, np.float32).reshape(-1).copy()

    def assign(self, values: Any) -> "_Scale":
        v = values.numpy() if hasattr(values, "numpy") else np.asarray(values, np.float32)
        v = np.asarray(v, np.float32).reshape(-1)
        if v.shape != self._v.shape:
            raise ValueError(f"scale of {v.size} columns for a sampler of {self._v.size}")
        self._v[:] = v
        return self

    def numpy(self) -> np.ndarray:
        return self._v.copy()

    @property
    def shape(self):
        return self._v.shape


@dataclass(frozen=True)
class RobertsSamplerConfig:
    """Spread settings: `scale` is the half-width per tangent column (IK helpers scale it by joint range)
    (opt/sampler.py:296-316)."""

    scale: Union[float, Sequence[float]] = 0.2
    seed: Optional[int] = None
    keep_first: bool = False
    var_key: Any = None
    num_draws: int = 1

    def build(self, var: Any, num_candidates: int, active_dof_mask: Any = None) -> "RobertsSampler":
        """A sampler for the variables `var` (VarValues) with `num_candidates` per instance."""
        from .var_values import VarKey

        key = self.var_key if self.var_key is not None else VarKey.ROBOT
        width = var.get(key).tangent_dim
        scale = np.broadcast_to(np.asarray(self.scale, np.float32), (width,)).copy()
        if active_dof_mask is not None:
            m = active_dof_mask.numpy() if hasattr(active_dof_mask, "numpy") else np.asarray(active_dof_mask)
            off = var.tangent_offset(key)
            scale *= np.asarray(m, np.float32).reshape(-1)[off:off + width]
        return RobertsSampler(num_candidates, scale, self.seed, self.keep_first, var_key=key)


class RobertsSampler:
    """Seed candidates once with a Roberts low-discrepancy sequence (opt/sampler.py:319-384): candidate c of
    every instance gets offset row c scaled per tangent column (instance-major batches); with `keep_first`
    candidate 0 gets zero noise and sits on the seed."""

    num_draws = 1

    def __init__(self, num_candidates: int, scale: Sequence[float], seed: Optional[int] = None,
                 keep_first: bool = False, device: Any = "cuda", var_key: Any = None):
        sc = np.asarray(scale, np.float32).reshape(-1)
        off = roberts_samples(num_candidates, sc.size, (seed % 10000) if seed is not None else 0) - 0.5
        if keep_first:
            off = np.vstack([np.zeros_like(off[:1]), off[:-1]])
        self.num_candidates = num_candidates
        self.tangent_dim = sc.size
        self.var_key = var_key
        self.offsets = off.astype(np.float32)
        self.scale = _Scale(sc)

    def tangent(self, batch: int, scale: Optional[np.ndarray] = None) -> np.ndarray:
        """Host noise for `batch` instances x num_candidates, [batch * num_candidates, tangent_dim]."""
        s = self.scale.numpy() if scale is None else np.asarray(scale, np.float32)
        return np.ascontiguousarray(np.tile(self.offsets * s[None, :], (batch, 1)))

    def reset(self) -> None:
        """A Roberts spread is fixed."""

    def fill(self, out_tangent: Any, iteration: int = 0) -> None:
        """Write the spread into a device tangent array [rows, tangent_dim] (rows = instances x candidates)."""
        from .. import _native as N

        out = N.as_device(out_tangent, np.float32)
        if out.ndim != 2 or out.shape[1] != self.tangent_dim:
            raise ValueError(f"expected tangent_dim {self.tangent_dim}, got {out.shape[1] if out.ndim == 2 else out.shape}")
        rows = out.shape[0]
        reps = -(-rows // self.num_candidates)
        out.copy_from_numpy(self.tangent(reps)[:rows])

    def sample(self, var_values: Any, scores: Any = None) -> Any:
        """Spread the candidates of `var_values` in place (scores tell a fixed spread nothing)."""
        from .. import _native as N
        from .var_values import VarKey

        var = var_values.get(self.var_key if self.var_key is not None else VarKey.ROBOT)
        noise = N.DeviceArray.zeros((var.batch_size, var.tangent_dim))
        if var.tangent_dim != self.tangent_dim:
            raise ValueError(f"expected tangent_dim {self.tangent_dim}, got {var.tangent_dim}")
        self.fill(noise)
        var.integrate(noise, out=var)
        return var_values
