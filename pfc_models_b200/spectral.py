"""Periodic 2-D spectral substrate on the host: geometry, k-space symbols and
ETD1 coefficients, in FP64 NumPy.

Same names and attribute contract as the reference substrate
(discretization/spectral/geometry_2d.py:1-22 and :70-88, kernels.py:38-71), so
models and user code written against it run unchanged. These tables are built
once per simulation; the device plan rebuilds the coefficients it uses from
the same formulas in C++ (pfc_models_b200/csrc/pfc_plan.cu).
"""
from __future__ import annotations

import numpy as np

npFloatType = np.float64
npComplexType = np.complex128


class Geometry:
    """Geometry contract: Nx, Ny, Lx, Ly, dx, dy, x, y, X, Y, kx, ky, KX, KY, K2,
    plus the coordinate/index conversions (geometry_2d.py:38-67)."""

    def __init__(self):
        self.Nx = self.Ny = None
        self.Lx = self.Ly = None
        self.dx = self.dy = None
        self.x = self.y = self.X = self.Y = None

    def px_to_x(self, px):
        return px * self.dx

    def py_to_y(self, py):
        return py * self.dy

    def x_to_px(self, x):
        return x / self.dx

    def y_to_py(self, y):
        return y / self.dy

    def x_to_ix(self, x):
        return int(x / self.dx)

    def y_to_iy(self, y):
        return int(y / self.dy)

    @property
    def periodic(self):
        return (True, True)


def Build2DGeometry(Nx, Ny, Lx, Ly) -> Geometry:
    """Uniform periodic grid of Nx x Ny points on [0, Lx) x [0, Ly); real-space
    arrays have shape (Ny, Nx), half-spectrum arrays (Ny, Nx//2 + 1) with
    kx = 2 pi rfftfreq(Nx, dx) and ky = 2 pi fftfreq(Ny, dy) (geometry_2d.py:70-88)."""
    g = Geometry()
    g.Nx, g.Ny, g.Lx, g.Ly = Nx, Ny, Lx, Ly
    g.dx = g.Lx / g.Nx
    g.dy = g.Ly / g.Ny
    g.x = np.linspace(0, g.Lx, g.Nx, endpoint=False, dtype=npFloatType)
    g.y = np.linspace(0, g.Ly, g.Ny, endpoint=False, dtype=npFloatType)
    g.X, g.Y = np.meshgrid(g.x, g.y)
    g.kx = 2 * np.pi * np.fft.rfftfreq(g.Nx, d=g.dx).astype(npFloatType)
    g.ky = 2 * np.pi * np.fft.fftfreq(g.Ny, d=g.dy).astype(npFloatType)
    g.KX, g.KY = np.meshgrid(g.kx, g.ky)
    g.K2 = g.KX**2 + g.KY**2
    return g


class _DerivativeKernels:
    pass


def BuildDerivativeKernels(geometry):
    """Spectral derivative symbols i kx, i ky (complex), -kx^2, -ky^2 and the
    Laplacian -(kx^2 + ky^2) (real), as in kernels.py:38-46."""
    dk = _DerivativeKernels()
    dk.Geometry = geometry
    dk.d_dx = 1j * geometry.KX
    dk.d_dy = 1j * geometry.KY
    dk.d2_dx2 = -geometry.KX**2
    dk.d2_dy2 = -geometry.KY**2
    dk.d2_dlap = -(geometry.KX**2 + geometry.KY**2)
    return dk


def kernel_local(geometry, w):
    """Gaussian low-pass exp(-|k|^2 w^2 / 2) used for the local (coarse) fields
    (kernels.py:49-52)."""
    return np.exp(-((geometry.KX) ** 2 + (geometry.KY) ** 2) * w**2 / 2)


def kernel_etd(kLinear, dt, *, small_z_tol=2e-5):
    """ETD1 coefficients for the linear symbol L: A = exp(L dt) and
    B = (A - 1)/L, replaced by dt (1 + z/2 + z^2/6), z = L dt, where |z| <= tol
    (the removable singularity; kernels.py:55-71)."""
    z = kLinear * dt
    A = np.exp(z)
    with np.errstate(divide="ignore", invalid="ignore"):
        B = np.where(np.abs(z) > small_z_tol, (A - 1) / kLinear, dt * (1 + z / 2 + z**2 / 6))
    return A, B


def linear_kernel_mu(beta, q0, epsilon, lap):
    """beta (q0^2 + lap)^2 + epsilon (models/stdpfc/simulation.py:83-90)."""
    return beta * (q0**2 + lap) ** 2 + epsilon


def linear_kernel_n(Gamma, beta, q0, epsilon, lap):
    """Gamma lap (beta (q0^2 + lap)^2 + epsilon) (models/stdpfc/simulation.py:92-96)."""
    return Gamma * lap * linear_kernel_mu(beta, q0, epsilon, lap)
