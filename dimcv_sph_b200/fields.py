"""Particle field storage on the device.

Each field is one torch tensor allocated at capacity (the reference's
`particle_max_num`); vector fields are stored with the padded stride of the
C ABI (2 floats per particle in 2D, 4 in 3D; 3-vectors always 4), so a
(capacity, dim) view is what the Python surface shows.
"""
from __future__ import annotations

import torch

from ._abi import PARTICLE_FIELDS, SOLVER_FIELDS, DvFields, DvSolverFields, components, make_struct

_DT = {"f32": torch.float32, "i32": torch.int32, "u8": torch.uint8}


class FieldSet:
    """A set of per-particle tensors with a cached C struct of their pointers."""

    def __init__(self, spec: dict, struct_cls, capacity: int, dim: int, device, fill: dict | None = None):
        self.capacity = capacity
        self.dim = dim
        self.device = device
        self.t: dict[str, torch.Tensor] = {}
        for name, (dt, comp) in spec.items():
            k = components(comp, dim)
            shape = (capacity,) if k == 1 else (capacity, k)
            self.t[name] = torch.zeros(shape, dtype=_DT[dt], device=device)
        for name, val in (fill or {}).items():
            self.t[name].fill_(val)
        self.struct = make_struct(struct_cls, {n: t.data_ptr() for n, t in self.t.items()})

    def __getitem__(self, name: str) -> torch.Tensor:
        return self.t[name]

    def nbytes(self) -> int:
        return sum(t.numel() * t.element_size() for t in self.t.values())


def particle_fields(capacity: int, dim: int, device) -> FieldSet:
    return FieldSet(PARTICLE_FIELDS, DvFields, capacity, dim, device)


def solver_fields(capacity: int, dim: int, device) -> FieldSet:
    return FieldSet(SOLVER_FIELDS, DvSolverFields, capacity, dim, device)
