"""Closed-form velocity fields and ``AnalyticalSolver`` (mirror of pyFTLE's ``api.py``).

``AnalyticalSolver(velocity_fn, particles, timestep, flow_map_period, num_ftles,
integrator_name)`` computes ``num_ftles`` FTLE fields whose windows start at
``i * timestep`` and take p = int(T/|timestep|) + 1 steps of size ``timestep``,
normalised by (p - 1)|timestep| (api.py:86-224 with ftle_solver.py:151-161).
``run()`` returns ``(num_ftles, N)`` (or ``(N,)`` for one field), or writes
``ftle_<t0>`` files when ``save_output`` is set.

* ``velocity_fn`` a ``DoubleGyre`` / ``ABCFlow``: every window is one CUDA launch
  evaluating the closed-form field inside the kernel (``ftle_analytic_window_run``).
* any other callable ``velocity_fn(t, points) -> velocities`` (numpy in/out, as in
  the reference's notebooks; device tensors with ``velocity_on_host=False``): the
  integrator stages run in the CUDA update kernels around the callable.

Time: pyFTLE's ``AnalyticalInterpolator`` never advances its time (it stays 0.0,
interpolate.py:788,812; the source's ``update_interpolator`` is a no-op,
data_source.py:274-285), so all of its windows evaluate the t = 0 field.  By
default this solver uses the true stage times t0 + i*h (+ h/2, + h);
``freeze_time=True`` reproduces the reference's t = 0 evaluation exactly.
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from datetime import datetime
from typing import Callable, Optional, Union

import numpy as np
import torch

from pyftle_b200 import _lib, flows
from pyftle_b200._device import as_device_f64, ptr, stream_ptr
from pyftle_b200.ftle import compute_ftle_from_positions
from pyftle_b200.particles import NeighboringParticles


@dataclass(frozen=True)
class DoubleGyre:
    """u = -pi A sin(pi f) cos(pi y), v = pi A cos(pi f) sin(pi y) df/dx,
    f = eps sin(omega t) x^2 + (1 - 2 eps sin(omega t)) x."""

    A: float = 0.1
    eps: float = 0.25
    omega: float = 2.0 * math.pi / 10.0
    dim = 2

    def abi(self) -> _lib.FtleFlow:
        f = _lib.FtleFlow()
        f.kind = _lib.FLOW_DOUBLE_GYRE
        f.params[0], f.params[1], f.params[2] = self.A, self.eps, self.omega
        return f

    def __call__(self, t, points):
        return flows.double_gyre_velocity(t, np.asarray(points), self.A, self.eps, self.omega)


@dataclass(frozen=True)
class ABCFlow:
    """A(t) = A + a sin(w t); u = A(t) sin z + C cos y, v = B sin x + A(t) cos z,
    w = C sin y + B cos x."""

    A: float = math.sqrt(3.0)
    B: float = math.sqrt(2.0)
    C: float = 1.0
    a: float = 0.1
    w: float = 1.0
    dim = 3

    def abi(self) -> _lib.FtleFlow:
        f = _lib.FtleFlow()
        f.kind = _lib.FLOW_ABC
        for i, v in enumerate((self.A, self.B, self.C, self.a, self.w)):
            f.params[i] = v
        return f

    def __call__(self, t, points):
        p = np.asarray(points)
        At = self.A + self.a * math.sin(self.w * t)
        out = np.empty_like(p, dtype=np.float64)
        out[:, 0] = At * np.sin(p[:, 2]) + self.C * np.cos(p[:, 1])
        out[:, 1] = self.B * np.sin(p[:, 0]) + At * np.cos(p[:, 2])
        out[:, 2] = self.C * np.sin(p[:, 1]) + self.B * np.cos(p[:, 0])
        return out


DeviceFlow = Union[DoubleGyre, ABCFlow]


def advect_analytic(flow: DeviceFlow, particles: NeighboringParticles, *, t0: float, h: float,
                    num_steps: int, integrator: str = "rk4", map_period: Optional[float] = None,
                    freeze_time: bool = False) -> torch.Tensor:
    """One window of a closed-form field in one launch; returns the FTLE field."""
    if particles.dim != flow.dim:
        raise ValueError(f"{type(flow).__name__} is {flow.dim}D, particles are {particles.dim}D")
    n = len(particles)
    ftle = torch.empty(n, dtype=torch.float64, device=particles.positions.device)
    mp = map_period if map_period is not None else (num_steps - 1) * abs(h)
    _lib.call("ftle_analytic_window_run", flow.abi(), _lib.INTEGRATOR_CODES[integrator.lower()],
              float(t0), float(h), int(num_steps), int(freeze_time), ptr(particles.positions), n,
              float(mp), ptr(ftle), stream_ptr())
    return ftle


def advect_callable(velocity_fn: Callable, particles: NeighboringParticles, *, t0: float,
                    h: float, num_steps: int, integrator: str = "rk4",
                    freeze_time: bool = False, velocity_on_host: bool = True) -> None:
    """Advect with any velocity callable; stage arithmetic in the CUDA update kernels."""
    pos = particles.positions
    n = pos.numel()
    s = stream_ptr()

    def vel(t, x):
        tt = 0.0 if freeze_time else t
        if velocity_on_host:
            v = as_device_f64(velocity_fn(tt, x.cpu().numpy()))
        else:
            v = as_device_f64(velocity_fn(tt, x))
        if v.shape != x.shape:
            raise ValueError(f"velocity_fn returned shape {tuple(v.shape)}")
        return v

    name = integrator.lower()
    prev = None
    tmp = torch.empty_like(pos)
    for i in range(num_steps):
        t = t0 + i * h
        if name == "euler":
            v = vel(t, pos)
            _lib.call("ftle_axpy", ptr(pos), ptr(pos), float(h), ptr(v), n, s)
        elif name == "ab2":
            v = vel(t, pos)
            if prev is None:
                _lib.call("ftle_axpy", ptr(pos), ptr(pos), float(h), ptr(v), n, s)
            else:
                _lib.call("ftle_ab2_update", ptr(pos), float(h), ptr(v), ptr(prev), n, s)
            prev = v.clone()
        elif name == "rk4":
            k1 = vel(t, pos)
            _lib.call("ftle_axpy", ptr(tmp), ptr(pos), 0.5 * h, ptr(k1), n, s)
            k2 = vel(t + 0.5 * h, tmp)
            _lib.call("ftle_axpy", ptr(tmp), ptr(pos), 0.5 * h, ptr(k2), n, s)
            k3 = vel(t + 0.5 * h, tmp)
            _lib.call("ftle_axpy", ptr(tmp), ptr(pos), float(h), ptr(k3), n, s)
            k4 = vel(t + h, tmp)
            _lib.call("ftle_rk4_update", ptr(pos), float(h), ptr(k1), ptr(k2), ptr(k3), ptr(k4),
                      n, s)
        else:
            raise ValueError(f"Invalid integrator name '{integrator}'. "
                             "Choose from ['ab2', 'euler', 'rk4'].")


class AnalyticalSolver:
    def __init__(self, velocity_fn: Callable, particles: NeighboringParticles, timestep: float,
                 flow_map_period: float, num_ftles: int, integrator_name: str,
                 num_processes: int = 1, save_output: bool = False,
                 output_format: str = "vtk", output_dir_name: Optional[str] = None, *,
                 freeze_time: bool = False, velocity_on_host: bool = True):
        self.velocity_fn = velocity_fn
        self.particles = particles
        self.timestep = float(timestep)
        self.flow_map_period = float(flow_map_period)
        self.num_ftles = int(num_ftles)
        self.num_snapshots = int(flow_map_period / abs(timestep)) + 1
        self.integrator_name = integrator_name.lower()
        if self.integrator_name not in _lib.INTEGRATOR_CODES:
            raise ValueError(f"Invalid integrator name '{integrator_name}'. "
                             "Choose from ['ab2', 'euler', 'rk4'].")
        self.freeze_time = freeze_time
        self.velocity_on_host = velocity_on_host
        self.writer = None
        if save_output:
            from pyftle_b200.io import create_writer

            if output_dir_name is None:
                output_dir_name = datetime.now().strftime("run-%Y-%m-%d-%Hh-%Mm-%Ss")
            self.writer = create_writer(output_format, output_dir_name)

    def start_times(self) -> np.ndarray:
        return np.arange(self.num_ftles) * self.timestep  # api.py:137-146

    def run_device(self) -> torch.Tensor:
        p = self.num_snapshots
        h = self.timestep
        T = (p - 1) * abs(h)
        fields = []
        for t0 in self.start_times():
            part = NeighboringParticles(positions=self.particles.positions)
            if isinstance(self.velocity_fn, (DoubleGyre, ABCFlow)):
                f = advect_analytic(self.velocity_fn, part, t0=float(t0), h=h, num_steps=p,
                                    integrator=self.integrator_name, map_period=T,
                                    freeze_time=self.freeze_time)
            else:
                advect_callable(self.velocity_fn, part, t0=float(t0), h=h, num_steps=p,
                                integrator=self.integrator_name, freeze_time=self.freeze_time,
                                velocity_on_host=self.velocity_on_host)
                f = compute_ftle_from_positions(part, T)
            if self.writer is not None:
                self.writer.write(f"ftle_{float(t0):06f}", f.cpu().numpy(),
                                  part.initial_centroid.cpu().numpy())
            fields.append(f)
        return torch.stack(fields)

    def run(self):
        fields = self.run_device()
        if self.writer is not None:
            return None
        out = fields.cpu().numpy()
        return out[0] if self.num_ftles == 1 else out
