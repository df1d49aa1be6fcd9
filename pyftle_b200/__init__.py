"""pyftle_b200 -- B200-native (sm_100a) engine for pyFTLE's FTLE hot path.

Public API mirrors pyFTLE's plugin interface for the path:
``create_integrator``, ``create_interpolator("grid", ...)``,
``NeighboringParticles``, ``FTLESolver`` and the ``BatchSource`` protocol,
plus the fused-window layer (``SnapshotSeries``, ``run_window``).
All arithmetic runs in ``libpyftle_b200.so``; there is no CPU fallback.
"""

from pyftle_b200.data_source import BatchSource, BlendedSnapshotSource, MemoryBatchSource
from pyftle_b200.ftle_solver import FTLESolver
from pyftle_b200.integrate import (
    AdamsBashforth2Integrator,
    EulerIntegrator,
    Integrator,
    RungeKutta4Integrator,
    create_integrator,
)
from pyftle_b200.interpolate import (
    GridSpec,
    HighPerfInterpolator,
    Interpolator,
    create_interpolator,
)
from pyftle_b200.particles import NeighboringParticles
from pyftle_b200.window import EngineOptions, SnapshotSeries, run_window

__all__ = [
    "AdamsBashforth2Integrator", "BatchSource", "BlendedSnapshotSource", "EngineOptions",
    "EulerIntegrator", "FTLESolver", "GridSpec", "HighPerfInterpolator", "Integrator",
    "Interpolator", "MemoryBatchSource", "NeighboringParticles", "RungeKutta4Integrator",
    "SnapshotSeries", "create_integrator", "create_interpolator", "run_window",
]
