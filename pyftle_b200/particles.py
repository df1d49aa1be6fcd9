"""Neighbour-particle groups on the device (mirror of pyFTLE's ``particles.py``).

``NeighboringParticles(positions)`` keeps the same contract as the reference
(``particles.py:8-150``): ``positions`` is ``(K*N, dim)`` float64 with
role-blocked rows ``[left; right; top; bottom (; front; back)]`` (``np.split``
into K equal blocks, ``particles.py:153-237``), K = 2*dim.  The initial
separations and centroid are taken once at construction; the ``delta_*`` and
``centroid`` properties follow the current positions.

Differences from the reference: ``positions`` lives on the GPU as a torch
float64 tensor (``positions_host()`` copies it back), and the group size is
checked as ``2*dim`` instead of "a multiple of 4 or 6".
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import torch

from pyftle_b200._device import as_device_f64, to_host


def _split(positions: torch.Tensor, num_neighbors: int):
    n = positions.shape[0] // num_neighbors
    return [positions[r * n:(r + 1) * n] for r in range(num_neighbors)]


def compute_delta_right_left(positions, num_neighbors):
    left, right, *_ = _split(positions, num_neighbors)
    return right - left


def compute_delta_top_bottom(positions, num_neighbors):
    _, _, top, bottom, *_ = _split(positions, num_neighbors)
    return top - bottom


def compute_delta_front_back(positions, num_neighbors):
    *_, front, back = _split(positions, num_neighbors)
    return front - back


def compute_centroid(positions, num_neighbors):
    """Mean of the K neighbours, summed in role order then divided by K."""
    parts = _split(positions, num_neighbors)
    s = parts[0].clone()
    for p in parts[1:]:
        s = s + p
    return s / float(num_neighbors)


@dataclass
class NeighboringParticles:
    positions: torch.Tensor
    initial_delta_top_bottom: torch.Tensor = field(init=False)
    initial_delta_right_left: torch.Tensor = field(init=False)
    initial_delta_front_back: torch.Tensor = field(init=False)
    initial_centroid: torch.Tensor = field(init=False)
    num_neighbors: int = field(init=False)

    def __post_init__(self) -> None:
        self.positions = as_device_f64(self.positions, copy=True)
        if self.positions.ndim != 2 or self.positions.shape[1] not in (2, 3):
            raise ValueError("positions must have shape (K*N, 2) or (K*N, 3)")
        self.num_neighbors = self.positions.shape[1] * 2
        assert self.positions.shape[0] % self.num_neighbors == 0, (
            f"positions.shape[0] must be a multiple of {self.num_neighbors}")
        self.initial_delta_top_bottom = compute_delta_top_bottom(self.positions, self.num_neighbors)
        self.initial_delta_right_left = compute_delta_right_left(self.positions, self.num_neighbors)
        if self.positions.shape[1] == 3:
            self.initial_delta_front_back = compute_delta_front_back(self.positions,
                                                                     self.num_neighbors)
        else:
            self.initial_delta_front_back = torch.zeros(0, dtype=torch.float64,
                                                        device=self.positions.device)
        self.initial_centroid = compute_centroid(self.positions, self.num_neighbors)

    def __len__(self) -> int:
        return self.positions.shape[0] // self.num_neighbors

    @property
    def dim(self) -> int:
        return self.positions.shape[1]

    @property
    def delta_top_bottom(self):
        return compute_delta_top_bottom(self.positions, self.num_neighbors)

    @property
    def delta_right_left(self):
        return compute_delta_right_left(self.positions, self.num_neighbors)

    @property
    def delta_front_back(self):
        return compute_delta_front_back(self.positions, self.num_neighbors)

    @property
    def centroid(self):
        return compute_centroid(self.positions, self.num_neighbors)

    def initial_deltas(self) -> torch.Tensor:
        """(dim, N, dim) stack [right-left; top-bottom (; front-back)] at t0 (C-ABI layout)."""
        parts = [self.initial_delta_right_left, self.initial_delta_top_bottom]
        if self.dim == 3:
            parts.append(self.initial_delta_front_back)
        return torch.stack(parts).contiguous()

    def positions_host(self) -> np.ndarray:
        return to_host(self.positions)
