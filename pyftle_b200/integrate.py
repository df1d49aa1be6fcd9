"""Integrators (mirror of pyFTLE's ``integrate.py``).

``create_integrator(name, interpolator)`` with keys ``"euler"``, ``"ab2"``,
``"rk4"`` (case-insensitive, ``ValueError`` otherwise; ``integrate.py:350-387``).
``integrate(h, particles)`` advances ``particles.positions`` in place by one
step of size h (negative for backward time):

* with the GPU "grid" interpolator the whole step -- every stage, gather and
  update -- is one CUDA launch (``ftle_grid_step``);
* with any other interpolator the velocities come from its ``interpolate``
  and the stage/update arithmetic runs in the CUDA update kernels
  (``ftle_axpy`` / ``ftle_ab2_update`` / ``ftle_rk4_update``), bit-exact with
  the reference's numpy/numba expressions (``integrate.py:16-109``).

As in the reference, RK4 holds the interpolator's current snapshot frozen for
all four stages, and AB2 starts with one Euler step and keeps its velocity
history on the integrator instance.
"""

from __future__ import annotations

from abc import ABC, abstractmethod
from typing import Optional

import torch

from pyftle_b200 import _lib
from pyftle_b200._device import as_device_f64, ptr, stream_ptr
from pyftle_b200.interpolate import HighPerfInterpolator, Interpolator
from pyftle_b200.particles import NeighboringParticles


def _velocity(interpolator: Interpolator, points: torch.Tensor) -> torch.Tensor:
    v = interpolator.interpolate(points)
    v = as_device_f64(v)
    if v.shape != points.shape:
        raise ValueError(f"interpolator returned shape {tuple(v.shape)}, "
                         f"expected {tuple(points.shape)}")
    return v


class Integrator(ABC):
    name = ""

    def __init__(self, interpolator: Interpolator, **kwargs) -> None:  # noqa: ARG002
        self.interpolator = interpolator

    @abstractmethod
    def integrate(self, h: float, particles: NeighboringParticles) -> None:
        ...

    def reset(self) -> None:
        """Forget any multistep history (start of a new window)."""

    def _grid_step(self, code: int, h: float, particles: NeighboringParticles,
                   history: Optional[torch.Tensor] = None, history_valid: bool = False) -> bool:
        it = self.interpolator
        if not isinstance(it, HighPerfInterpolator):
            return False
        if it.grid is None or it.snapshot is None:
            raise AssertionError("interpolator was not initialised with update(velocities, points)")
        pos = particles.positions
        _lib.call("ftle_grid_step", it.grid.to_abi(), ptr(it.snapshot), code, float(h), ptr(pos),
                  pos.shape[0], ptr(history), int(history_valid), stream_ptr())
        return True


class EulerIntegrator(Integrator):
    """x_{n+1} = x_n + h v(x_n)  (integrate.py:161-196)."""

    name = "euler"

    def integrate(self, h: float, particles: NeighboringParticles) -> None:
        if self._grid_step(_lib.EULER, h, particles):
            return
        pos = particles.positions
        v = _velocity(self.interpolator, pos)
        _lib.call("ftle_axpy", ptr(pos), ptr(pos), float(h), ptr(v), pos.numel(), stream_ptr())


class AdamsBashforth2Integrator(Integrator):
    """x_{n+1} = x_n + h (1.5 v_n - 0.5 v_{n-1}); Euler on the first call (integrate.py:204-257)."""

    name = "ab2"

    def __init__(self, interpolator: Interpolator, **kwargs) -> None:
        super().__init__(interpolator, **kwargs)
        self.previous_velocity: Optional[torch.Tensor] = None
        self._have_previous = False

    def reset(self) -> None:
        self.previous_velocity = None
        self._have_previous = False

    def integrate(self, h: float, particles: NeighboringParticles) -> None:
        pos = particles.positions
        if self.previous_velocity is None or self.previous_velocity.shape != pos.shape:
            self.previous_velocity = torch.empty_like(pos)
            self._have_previous = False
        if self._grid_step(_lib.AB2, h, particles, self.previous_velocity, self._have_previous):
            self._have_previous = True
            return
        v = _velocity(self.interpolator, pos)
        if not self._have_previous:
            _lib.call("ftle_axpy", ptr(pos), ptr(pos), float(h), ptr(v), pos.numel(), stream_ptr())
        else:
            _lib.call("ftle_ab2_update", ptr(pos), float(h), ptr(v), ptr(self.previous_velocity),
                      pos.numel(), stream_ptr())
        self.previous_velocity.copy_(v)
        self._have_previous = True


class RungeKutta4Integrator(Integrator):
    """Classical RK4 on the current snapshot (integrate.py:265-342)."""

    name = "rk4"

    def integrate(self, h: float, particles: NeighboringParticles) -> None:
        if self._grid_step(_lib.RK4, h, particles):
            return
        pos = particles.positions
        n = pos.numel()
        s = stream_ptr()
        tmp = torch.empty_like(pos)
        k1 = _velocity(self.interpolator, pos)
        _lib.call("ftle_axpy", ptr(tmp), ptr(pos), 0.5 * h, ptr(k1), n, s)
        k2 = _velocity(self.interpolator, tmp)
        _lib.call("ftle_axpy", ptr(tmp), ptr(pos), 0.5 * h, ptr(k2), n, s)
        k3 = _velocity(self.interpolator, tmp)
        _lib.call("ftle_axpy", ptr(tmp), ptr(pos), float(h), ptr(k3), n, s)
        k4 = _velocity(self.interpolator, tmp)
        _lib.call("ftle_rk4_update", ptr(pos), float(h), ptr(k1), ptr(k2), ptr(k3), ptr(k4), n, s)


def create_integrator(integrator_name: str, interpolator: Interpolator) -> Integrator:
    integrator_name = integrator_name.lower()
    integrator_map = {
        "ab2": AdamsBashforth2Integrator,
        "euler": EulerIntegrator,
        "rk4": RungeKutta4Integrator,
    }
    if integrator_name not in integrator_map:
        raise ValueError(
            f"Invalid integrator name '{integrator_name}'. "
            f"Choose from {list(integrator_map.keys())}.")
    return integrator_map[integrator_name](interpolator)
