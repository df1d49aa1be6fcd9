"""Synthetic velocity fields and seed-particle layouts (host-side input builders).

These build inputs in exactly the layouts pyFTLE consumes, so the same arrays
drive the reference, the oracle and the CUDA engine:

* a snapshot is ``(dim, nodes)`` float64 (``data_source.py`` / ``file_readers.py``);
  2D node ``(i, j)`` is flattened as ``j*nx + i`` and 3D node ``(i, j, k)`` as
  ``(j*nx + i)*nz + k`` -- numpy ``meshgrid(x, y[, z])`` ("xy" indexing)
  followed by C-order ``ravel``, which is what ``interpolate.py:359-401``
  un-flattens;
* grid coordinates are the matching ``(dim, nodes)`` array;
* neighbour particles are role-blocked ``(K*N, dim)`` rows
  ``[left; right; top; bottom (; front; back)]`` (``particles.py:153-237``,
  ``file_readers.py:175-180``).

Flow formulas:

* double gyre (``examples/01_Closed-form_velocity.ipynb`` of pyFTLE):
  ``f = eps sin(wt) x^2 + (1 - 2 eps sin(wt)) x``,
  ``u = -pi A sin(pi f) cos(pi y)``, ``v = pi A cos(pi f) sin(pi y) df/dx``;
* time-periodic ABC: ``A(t) = A + 0.1 sin t``,
  ``u = A(t) sin z + C cos y``, ``v = B sin x + A(t) cos z``,
  ``w = C sin y + B cos x``;
* 2D random-Fourier turbulence (divergence-free through a stream function,
  energy spectrum ``E(k) ~ k^(-5/3)`` on ``4 <= |k| <= kmax``, seeded phases,
  each mode with its own frequency).
"""

from __future__ import annotations

import math

import numpy as np

# ----------------------------------------------------------------------------
# grids and seeds
# ----------------------------------------------------------------------------


def grid_points_2d(nx: int, ny: int, xlim=(0.0, 2.0), ylim=(0.0, 1.0)) -> np.ndarray:
    """(2, nx*ny) node coordinates, meshgrid 'xy' flattening (inclusive axes)."""
    x = np.linspace(xlim[0], xlim[1], nx)
    y = np.linspace(ylim[0], ylim[1], ny)
    X, Y = np.meshgrid(x, y)
    return np.stack((X.ravel(), Y.ravel()))


def periodic_axis(n: int, length: float = 2.0 * math.pi) -> np.ndarray:
    """n nodes of a periodic axis ``[0, length)`` (the endpoint is node 0 again)."""
    return np.arange(n) * (length / n)


def grid_points_3d(x: np.ndarray, y: np.ndarray, z: np.ndarray) -> np.ndarray:
    """(3, nx*ny*nz) node coordinates, meshgrid 'xy' flattening."""
    X, Y, Z = np.meshgrid(x, y, z)
    return np.stack((X.ravel(), Y.ravel(), Z.ravel()))


def seeds_2d(centroids: np.ndarray, delta: float) -> np.ndarray:
    """Role-blocked (4N, 2) neighbours [L; R; T; B] around (N, 2) centroids."""
    c = np.asarray(centroids, dtype=np.float64)
    ex = np.array([delta, 0.0])
    ey = np.array([0.0, delta])
    return np.concatenate((c - ex, c + ex, c + ey, c - ey), axis=0)


def seeds_2d_device(centroids, delta: float):
    """seeds_2d for a (N, 2) float64 device tensor of centroids (stays on the device)."""
    import torch

    c = centroids
    ex = torch.tensor([delta, 0.0], dtype=torch.float64, device=c.device)
    ey = torch.tensor([0.0, delta], dtype=torch.float64, device=c.device)
    return torch.cat((c - ex, c + ex, c + ey, c - ey), dim=0).contiguous()


def seeds_3d_device(centroids, delta: float):
    """seeds_3d for a (N, 3) float64 device tensor of centroids (stays on the device)."""
    import torch

    c = centroids
    e = [torch.zeros(3, dtype=torch.float64, device=c.device) for _ in range(3)]
    for a in range(3):
        e[a][a] = delta
    return torch.cat((c - e[0], c + e[0], c + e[1], c - e[1], c + e[2], c - e[2]),
                     dim=0).contiguous()


def seeds_3d(centroids: np.ndarray, delta: float) -> np.ndarray:
    """Role-blocked (6N, 3) neighbours [L; R; T; B; F; Bk] around (N, 3) centroids."""
    c = np.asarray(centroids, dtype=np.float64)
    ex = np.array([delta, 0.0, 0.0])
    ey = np.array([0.0, delta, 0.0])
    ez = np.array([0.0, 0.0, delta])
    return np.concatenate((c - ex, c + ex, c + ey, c - ey, c + ez, c - ez), axis=0)


def centroid_grid_2d(ncx: int, ncy: int, xlim, ylim) -> np.ndarray:
    """(N, 2) centroids on linspace axes, meshgrid 'xy' order."""
    X, Y = np.meshgrid(np.linspace(*xlim, ncx), np.linspace(*ylim, ncy))
    return np.column_stack((X.ravel(), Y.ravel()))


def centroid_grid_3d(ncx: int, ncy: int, ncz: int, lo, hi) -> np.ndarray:
    """(N, 3) centroids on linspace axes between lo and hi, meshgrid 'xy' order."""
    X, Y, Z = np.meshgrid(np.linspace(lo[0], hi[0], ncx), np.linspace(lo[1], hi[1], ncy),
                          np.linspace(lo[2], hi[2], ncz))
    return np.column_stack((X.ravel(), Y.ravel(), Z.ravel()))


# ----------------------------------------------------------------------------
# double gyre
# ----------------------------------------------------------------------------


def double_gyre_velocity(t: float, pts: np.ndarray, A=0.1, eps=0.25, omega=2.0 * math.pi / 10.0):
    """Velocity at (N, 2) points; same expression as pyFTLE's example notebook."""
    x = pts[:, 0]
    y = pts[:, 1]
    s = math.sin(omega * t)
    f = eps * s * x**2 + (1.0 - 2.0 * eps * s) * x
    dfdx = 2 * eps * s * x + (1.0 - 2.0 * eps * s)
    out = np.empty_like(pts, dtype=np.float64)
    out[:, 0] = -np.pi * A * np.sin(np.pi * f) * np.cos(np.pi * y)
    out[:, 1] = np.pi * A * np.cos(np.pi * f) * np.sin(np.pi * y) * dfdx
    return out


def double_gyre_snapshots(points: np.ndarray, times, **kw) -> np.ndarray:
    """(S, 2, nodes) snapshots of the double gyre at ``times`` on grid ``points``."""
    P = np.ascontiguousarray(points.T)
    return np.stack([double_gyre_velocity(float(t), P, **kw).T.copy() for t in times])


# ----------------------------------------------------------------------------
# time-periodic ABC flow
# ----------------------------------------------------------------------------

ABC_A = math.sqrt(3.0)
ABC_B = math.sqrt(2.0)
ABC_C = 1.0


def abc_velocity(t: float, pts: np.ndarray, A=ABC_A, B=ABC_B, C=ABC_C) -> np.ndarray:
    At = A + 0.1 * math.sin(t)
    x, y, z = pts[:, 0], pts[:, 1], pts[:, 2]
    out = np.empty_like(pts, dtype=np.float64)
    out[:, 0] = At * np.sin(z) + C * np.cos(y)
    out[:, 1] = B * np.sin(x) + At * np.cos(z)
    out[:, 2] = C * np.sin(y) + B * np.cos(x)
    return out


def abc_snapshots(x: np.ndarray, y: np.ndarray, z: np.ndarray, times, A=ABC_A, B=ABC_B,
                  C=ABC_C, dtype=np.float64) -> np.ndarray:
    """(S, 3, nx*ny*nz) ABC snapshots on the tensor grid x, y, z (separable build).

    Node (i, j, k) sits at flat index (j*nx + i)*nz + k.
    """
    nx, ny, nz = len(x), len(y), len(z)
    S = len(times)
    out = np.empty((S, 3, ny, nx, nz), dtype=dtype)
    sx, cx = np.sin(x), np.cos(x)
    sy, cy = np.sin(y), np.cos(y)
    sz, cz = np.sin(z), np.cos(z)
    for s, t in enumerate(times):
        At = A + 0.1 * math.sin(float(t))
        out[s, 0] = (At * sz)[None, None, :] + (C * cy)[:, None, None]
        out[s, 1] = (B * sx)[None, :, None] + (At * cz)[None, None, :]
        out[s, 2] = (C * sy)[:, None, None] + (B * cx)[None, :, None]
    return out.reshape(S, 3, nx * ny * nz)


def abc_snapshots_device(x, y, z, times, A=ABC_A, B=ABC_B, C=ABC_C, device="cuda"):
    """``abc_snapshots`` built on the device as a (S, 3, nx*ny*nz) float64 tensor."""
    import torch

    tx = torch.as_tensor(np.asarray(x), dtype=torch.float64, device=device)
    ty = torch.as_tensor(np.asarray(y), dtype=torch.float64, device=device)
    tz = torch.as_tensor(np.asarray(z), dtype=torch.float64, device=device)
    nx, ny, nz = len(tx), len(ty), len(tz)
    out = torch.empty((len(times), 3, ny, nx, nz), dtype=torch.float64, device=device)
    for s, t in enumerate(times):
        At = A + 0.1 * math.sin(float(t))
        out[s, 0] = (At * torch.sin(tz))[None, None, :] + (C * torch.cos(ty))[:, None, None]
        out[s, 1] = (B * torch.sin(tx))[None, :, None] + (At * torch.cos(tz))[None, None, :]
        out[s, 2] = (C * torch.sin(ty))[:, None, None] + (B * torch.cos(tx))[None, :, None]
    return out.reshape(len(times), 3, nx * ny * nz)


# ----------------------------------------------------------------------------
# 2D random-Fourier turbulence
# ----------------------------------------------------------------------------


class FourierTurbulence2D:
    """Divergence-free 2D random-mode field on the periodic box [0, L)^2.

    psi(x, t) = sum_m a_m cos(k_m . x + phi_m + w_m t); u = dpsi/dy, v = -dpsi/dx.
    Wavenumbers are integer pairs with kmin <= |k| <= kmax (drawn log-uniformly in |k|,
    uniformly in angle); amplitudes follow E(k) ~ k^(-5/3); seeded phases and
    frequencies.  The field is normalised to rms speed ``urms``.  Snapshots on an n x n
    grid (n > 2*kmax) are exact sums of the modes, evaluated by one inverse FFT of the
    sparse spectrum per component.
    """

    def __init__(self, seed: int = 0, num_modes: int = 256, kmin: float = 4.0,
                 kmax: float = 128.0, length: float = 2.0 * math.pi, omega_scale: float = 1.0,
                 urms: float = 1.0):
        rng = np.random.default_rng(seed)
        self.length = length
        kk = np.exp(rng.uniform(math.log(kmin), math.log(kmax), num_modes))
        theta = rng.uniform(0.0, 2.0 * math.pi, num_modes)
        kx = np.round(kk * np.cos(theta)).astype(np.int64)
        ky = np.round(kk * np.sin(theta)).astype(np.int64)
        bad = (kx == 0) & (ky == 0)
        kx[bad] = int(kmin)
        self.ikx, self.iky = kx, ky
        kmag = np.hypot(kx, ky)
        # log-uniform |k| has density ~1/k; E(k) ~ k^-5/3 then needs |u_k|^2 ~ k^-5/3 * k,
        # i.e. psi amplitude ~ k^(-1/3) / k
        amp = kmag ** (-1.0 / 3.0) / kmag
        k0 = 2.0 * math.pi / length
        self.kx = kx * k0
        self.ky = ky * k0
        self.phase = rng.uniform(0.0, 2.0 * math.pi, num_modes)
        self.omega = omega_scale * rng.standard_normal(num_modes)
        speed2 = 0.5 * np.sum((amp * self.kx) ** 2 + (amp * self.ky) ** 2)
        self.amp = urms * amp / math.sqrt(speed2)

    def velocity(self, t: float, pts: np.ndarray) -> np.ndarray:
        """Closed-form velocity at (M, 2) points (direct mode sum; for checks)."""
        th = np.outer(pts[:, 0], self.kx) + np.outer(pts[:, 1], self.ky) + (
            self.phase + self.omega * t)
        s = np.sin(th)
        out = np.empty((pts.shape[0], 2))
        out[:, 0] = s @ (self.amp * -self.ky)
        out[:, 1] = s @ (self.amp * self.kx)
        return out

    def snapshot(self, n: int, t: float) -> np.ndarray:
        """(2, n*n) velocity on the n x n periodic grid (node (i, j) at j*n + i)."""
        if n <= 2 * int(np.max(np.abs(np.concatenate([self.ikx, self.iky])))):
            raise ValueError("grid too coarse for the mode set")
        ph = self.phase + self.omega * t
        out = np.empty((2, n * n))
        for comp, coef in ((0, self.amp * -self.ky), (1, self.amp * self.kx)):
            # component = sum_m coef_m sin(kx x + ky y + ph_m); with spectrum S[ky, kx],
            # f(x) = sum S e^{i k.x} and sin th = (e^{i th} - e^{-i th}) / (2i)
            spec = np.zeros((n, n), dtype=np.complex128)
            c = coef * np.exp(1j * ph) / 2j
            np.add.at(spec, (self.iky % n, self.ikx % n), c)
            np.add.at(spec, ((-self.iky) % n, (-self.ikx) % n), np.conj(c))
            f = np.fft.ifft2(spec) * (n * n)  # rows: y (j), columns: x (i)
            out[comp] = f.real.ravel()
        return out

    def snapshots(self, n: int, times) -> np.ndarray:
        return np.stack([self.snapshot(n, float(t)) for t in times])

    def snapshots_device(self, n: int, times, device="cuda"):
        """(S, 2, n*n) float64 torch tensor built on the device (same values as
        ``snapshots``; input generation only)."""
        import torch

        if n <= 2 * int(np.max(np.abs(np.concatenate([self.ikx, self.iky])))):
            raise ValueError("grid too coarse for the mode set")
        iy = torch.as_tensor(self.iky % n, device=device)
        ix = torch.as_tensor(self.ikx % n, device=device)
        iyc = torch.as_tensor((-self.iky) % n, device=device)
        ixc = torch.as_tensor((-self.ikx) % n, device=device)
        coefs = [torch.as_tensor(self.amp * -self.ky, device=device),
                 torch.as_tensor(self.amp * self.kx, device=device)]
        phase = torch.as_tensor(self.phase, device=device)
        omega = torch.as_tensor(self.omega, device=device)
        out = torch.empty((len(times), 2, n * n), dtype=torch.float64, device=device)
        spec = torch.zeros((n, n), dtype=torch.complex128, device=device)
        for si, t in enumerate(times):
            ph = phase + omega * float(t)
            for comp in range(2):
                c = coefs[comp] * torch.exp(1j * ph) / 2j
                spec.zero_()
                spec.index_put_((iy, ix), c, accumulate=True)
                spec.index_put_((iyc, ixc), torch.conj(c), accumulate=True)
                out[si, comp] = (torch.fft.ifft2(spec) * (n * n)).real.reshape(-1)
        return out
