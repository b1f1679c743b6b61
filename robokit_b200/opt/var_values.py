"""Optimisation variables (robokit opt/var_values.py:24-217)."""

from __future__ import annotations

import abc
from enum import Enum
from typing import Dict, Mapping


class Var(abc.ABC):
    """Protocol of an optimisation variable (opt/var_values.py:24-70)."""

    @property
    @abc.abstractmethod
    def tangent_dim(self) -> int: ...

    @property
    @abc.abstractmethod
    def batch_size(self) -> int: ...

    @abc.abstractmethod
    def clone(self) -> "Var": ...

    @abc.abstractmethod
    def view(self, batch_size: int, offset: int = 0) -> "Var": ...

    @abc.abstractmethod
    def integrate(self, velocity, out=None, tangent_mask=None, weight_decay: float = 0.0, out_velocity=None) -> "Var":
        ...

    @abc.abstractmethod
    def accept(self, accept_mask, proposed) -> "Var": ...

    def invalidate(self) -> None:
        pass


class VarKey(Enum):
    """Keys of the variables robokit's tasks read (opt/var_values.py:73-82)."""

    ROBOT = 0
    TIMING = 1
    ACTION = 2
    SEGMENT_STEP = 7


class VarValues(Var):
    """Variables concatenated into tangent-column blocks in insertion order (opt/var_values.py:94-217)."""

    def __init__(self, named_vars: Mapping[Enum, Var]):
        if not named_vars:
            raise ValueError("VarValues requires at least one variable")
        self._vars: Dict[Enum, Var] = dict(named_vars)
        self._offsets: Dict[Enum, int] = {}
        off = 0
        for k, v in self._vars.items():
            self._offsets[k] = off
            off += v.tangent_dim
        self._tangent_dim = off
        first = next(iter(self._vars.values()))
        self._batch_size = first.batch_size

    @classmethod
    def from_var(cls, var: Var, key: Enum) -> "VarValues":
        return cls({key: var})

    def get(self, key: Enum) -> Var:
        return self._vars[key]

    def __contains__(self, key: Enum) -> bool:
        return key in self._vars

    def keys(self):
        return self._vars.keys()

    def values(self):
        return self._vars.values()

    def items(self):
        return self._vars.items()

    def tangent_offset(self, key: Enum) -> int:
        return self._offsets[key]

    @property
    def tangent_dim(self) -> int:
        return self._tangent_dim

    @property
    def batch_size(self) -> int:
        return self._batch_size

    @property
    def device(self) -> str:
        return "cuda:0"

    def clone(self) -> "VarValues":
        return VarValues({k: v.clone() for k, v in self._vars.items()})

    def view(self, batch_size: int, offset: int = 0) -> "VarValues":
        return VarValues({k: v.view(batch_size, offset) for k, v in self._vars.items()})

    def integrate(self, velocity, out=None, tangent_mask=None, weight_decay: float = 0.0, out_velocity=None):
        if len(self._vars) != 1:
            raise NotImplementedError("integrate over several variables is not on the IK path")
        (k, v), = self._vars.items()
        o = v.integrate(velocity, out=None if out is None else out.get(k), tangent_mask=tangent_mask)
        return VarValues({k: o}) if out is None else out

    def accept(self, accept_mask, proposed: "VarValues") -> "VarValues":
        for k, v in self._vars.items():
            v.accept(accept_mask, proposed.get(k))
        return self

    def invalidate(self) -> None:
        for v in self._vars.values():
            v.invalidate()
