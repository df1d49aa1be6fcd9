"""FTLE building blocks on the GPU (mirror of pyFTLE's ``ftle.py`` and ``cauchy_green.py``).

Same names and meaning as the reference; arrays are device tensors (numpy
inputs are uploaded):

* ``compute_flow_map_jacobian_2x2/3x3(particles)`` -> (N, d, d)
  ``J[:, i, j] = dx_pair_j[i] / dX0_pair_j[j]`` (cauchy_green.py:15-153);
* ``compute_cauchy_green_2x2`` (C = F^T F, ftle.py:9-69) and
  ``compute_cauchy_green_3x3`` (C = F F^T, ftle.py:72-96);
* ``max_eigenvalue_2x2`` (closed form, ftle.py:122-163) and
  ``max_eigenvalue_3x3`` (symmetric Jacobi; the reference calls
  ``np.linalg.eigvals``, ftle.py:99-119);
* ``compute_ftle_2x2/3x3(J, T)`` = ``(1/T) log(sqrt(lambda_max))``
  (ftle.py:166-233);
* ``compute_ftle_from_positions(particles, T)`` fuses Jacobian -> C ->
  lambda_max -> FTLE in one launch (ftle_solver.py:151-161).
"""

from __future__ import annotations

import torch

from pyftle_b200 import _lib
from pyftle_b200._device import as_device_f64, ptr, stream_ptr
from pyftle_b200.particles import NeighboringParticles


def _check_stack(J: torch.Tensor, d: int) -> torch.Tensor:
    J = as_device_f64(J)
    if J.ndim != 3 or J.shape[1:] != (d, d):
        raise ValueError(f"expected an (N, {d}, {d}) array")
    return J


def _jacobian(particles: NeighboringParticles, d: int) -> torch.Tensor:
    if particles.dim != d:
        raise ValueError(f"expected {d}D particles")
    n = len(particles)
    J = torch.empty((n, d, d), dtype=torch.float64, device=particles.positions.device)
    _lib.call("ftle_flow_map_jacobian", d, ptr(particles.positions),
              ptr(particles.initial_deltas()), n, ptr(J), stream_ptr())
    return J


def compute_flow_map_jacobian_2x2(particles: NeighboringParticles) -> torch.Tensor:
    return _jacobian(particles, 2)


def compute_flow_map_jacobian_3x3(particles: NeighboringParticles) -> torch.Tensor:
    return _jacobian(particles, 3)


def _cg(J, d):
    J = _check_stack(J, d)
    C = torch.empty_like(J)
    _lib.call("ftle_cauchy_green", d, ptr(J), J.shape[0], ptr(C), stream_ptr())
    return C


def compute_cauchy_green_2x2(flow_map_jacobian) -> torch.Tensor:
    return _cg(flow_map_jacobian, 2)


def compute_cauchy_green_3x3(flow_map_jacobian) -> torch.Tensor:
    return _cg(flow_map_jacobian, 3)


def _lmax(C, d):
    C = _check_stack(C, d)
    out = torch.empty(C.shape[0], dtype=torch.float64, device=C.device)
    _lib.call("ftle_max_eigenvalue", d, ptr(C), C.shape[0], ptr(out), stream_ptr())
    return out


def max_eigenvalue_2x2(cauchy_green_tensor) -> torch.Tensor:
    return _lmax(cauchy_green_tensor, 2)


def max_eigenvalue_3x3(cauchy_green_tensor) -> torch.Tensor:
    return _lmax(cauchy_green_tensor, 3)


def _ftle(J, map_period, d):
    J = _check_stack(J, d)
    out = torch.empty(J.shape[0], dtype=torch.float64, device=J.device)
    _lib.call("ftle_from_jacobian", d, ptr(J), J.shape[0], float(map_period), ptr(out),
              stream_ptr())
    return out


def compute_ftle_2x2(flow_map_jacobian, map_period: float) -> torch.Tensor:
    return _ftle(flow_map_jacobian, map_period, 2)


def compute_ftle_3x3(flow_map_jacobian, map_period: float) -> torch.Tensor:
    return _ftle(flow_map_jacobian, map_period, 3)


def compute_ftle_from_positions(particles: NeighboringParticles, map_period: float,
                                out: torch.Tensor | None = None) -> torch.Tensor:
    n = len(particles)
    if out is None:
        out = torch.empty(n, dtype=torch.float64, device=particles.positions.device)
    _lib.call("ftle_from_positions", particles.dim, ptr(particles.positions),
              ptr(particles.initial_deltas()), n, float(map_period), ptr(out), stream_ptr())
    return out
