"""Log PFC with an external potential on B200: the entry points of the reference's
models/logpfc_extv/simulation.py and external_potentials.py over the sm_100a stepper.

Every TimeStep does what the reference's does (simulation.py:301-330): ValidatePhiRange
re-optimises the linear shift M when the field leaves its last optimised range
(OptimizeM and ValidatePhiRange, :332-405), the nonlinearity is the clamped log minus
M phi (:524-539) and the update adds the external potential's force B lap V_hat with the
k = 0 mode kept (:557-577). The decision, M and the rebuilt ETD1 coefficients live on the
device (plans created with PFC_FLAG_EXTV, FP64 plain); `State.M`, `State.phi_min` and
`State.phi_max` read them back. The external potential's shapes are built on the host in
FP64 (NumPy) and uploaded once per change, as the reference builds them once on the device.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .simulation import ModelParameters, Simulation as _Simulation, _SimulationState
from .spectral import Build2DGeometry, BuildDerivativeKernels, Geometry, kernel_etd, kernel_local  # noqa: F401


def BuildLogPFCModel_withVacancyForce_Parameters(Gamma=1.0, beta=1.0, q0=1.0, epsilon=1.0, g=1.0, dt=0.01,
                                                 minPhi=1e-6, meanDensity=None, smallZTol=1e-8, V0=None,
                                                 potWidth=None):
    """models/logpfc_extv/simulation.py:69-97 (smallZTol defaults to this model's 1e-8)."""
    model = ModelParameters()
    model.Gamma = Gamma
    model.beta = beta
    model.q0 = q0
    model.epsilon = epsilon
    model.g = g
    model.dt = dt
    model.minPhi = minPhi
    model.meanDensity = meanDensity
    model.smallZTol = smallZTol
    model.V0 = V0
    model.potWidth = potWidth
    model.minLog = np.log(minPhi)
    return model


def GetLinearKernel_mu(modelParameters, DerivativeKernels, M=0):
    """models/logpfc_extv/simulation.py:100-107: beta (q0^2 + lap)^2 + eps + M."""
    p = modelParameters
    return p.beta * (p.q0**2 + DerivativeKernels.d2_dlap) ** 2 + p.epsilon + M


def GetLinearKernel_phi(modelParameters, DerivativeKernels, M=0):
    """models/logpfc_extv/simulation.py:110-116."""
    return modelParameters.Gamma * DerivativeKernels.d2_dlap * GetLinearKernel_mu(modelParameters, DerivativeKernels,
                                                                                   M=M)


def BuildGeometry(Nx, Ny, Lx, Ly):
    """models/logpfc_extv/simulation.py:487-497: Build2DGeometry plus the triangular lattice
    constants a = 4 pi / sqrt3 and h = 4 pi that this model reads."""
    geometry = Build2DGeometry(Nx, Ny, Lx, Ly)
    geometry.a = 4 * np.pi / 3**0.5
    geometry.h = 4 * np.pi
    return geometry


class _ExternalPotential:
    """The potential shapes of external_potentials.py:47-131, built in FP64 on the host and
    handed to the plan (pfc_set_potential); `V` is the last potential set."""

    def __init__(self, sim, geometry):
        self._sim = sim
        self.Geometry = geometry
        self.V = np.zeros(geometry.X.shape)
        self.X = np.asarray(geometry.X)
        self.Y = np.asarray(geometry.Y)

    def _upload(self, V):
        self.V = np.ascontiguousarray(V, dtype=np.float64)
        plan = self._sim.plan
        t = plan.torch
        dv = t.as_tensor(self.V, dtype=t.float64, device=plan.device).contiguous()
        _lib.check(plan.lib.pfc_set_potential(plan.handle, ctypes.c_void_p(dv.data_ptr()), plan._s()))
        t.cuda.current_stream(plan.device).synchronize()

    @property
    def V_hat(self):
        return np.fft.rfft2(self.V)

    def SetGaussianDipolePotential(self, V0, X0, X1, sigma):
        """external_potentials.py:109-119."""
        x0, y0 = X0
        x1, y1 = X1
        self._upload(V0 * (np.exp(-((self.X - x0) ** 2 + (self.Y - y0) ** 2) / (2 * sigma**2))
                           - np.exp(-((self.X - x1) ** 2 + (self.Y - y1) ** 2) / (2 * sigma**2))))

    def SetPotential(self, V0, V_func):
        """external_potentials.py:121-123."""
        self._upload(V0 * np.asarray(V_func))

    def SetPotential_alongX(self, V0, width, x1, x2):
        """external_potentials.py:125-127."""
        self._upload(V0 * np.tanh((np.abs(self.X - (x1 + x2) / 2) - (x2 - x1) / 2) / width))

    def SetDoubleVacancyAlongX_TanhPotential(self, x1, x2, y1, y2, width_x, width_y, V0):
        """external_potentials.py:129-131."""
        self._upload(V0 * (np.tanh((np.abs(self.X - (x1 + x2) / 2) - (x2 - x1) / 2) / width_x) - 1) / 2
                     * (1 - np.tanh((np.abs(self.Y - (y1 + y2) / 2) - (y2 - y1) / 2) / width_y)) / 2 + 1)


class _ExtvState(_SimulationState):
    """The reference's _SimulationState (simulation.py:119-223) with its M-shift attributes
    (:130-144) read from the plan's device state."""

    phi_floor_tol = 0.1
    phi_ceiling_tol = 0.1

    def _read(self):
        o = (ctypes.c_double * 6)()
        plan = self._sim.plan
        _lib.check(plan.lib.pfc_extv_state(plan.handle, o))
        return list(o)

    @property
    def M(self):
        return self._read()[0]

    @property
    def phi_min(self):
        v = self._read()[1]
        return None if np.isnan(v) else v

    @property
    def phi_max(self):
        v = self._read()[2]
        return None if np.isnan(v) else v

    @property
    def optimizations(self):
        return int(self._read()[5])


class Simulation(_Simulation):
    """The reference's logpfc_extv Simulation (simulation.py:226-484) on a B200 plan."""

    def __init__(self, modelParameters, geometry, device=None, graphs=True):
        super().__init__("log", modelParameters, geometry, precision="fp64", clamp_log=True, device=device,
                         kernels="generic", graphs=graphs, one_cta=False, _flags=_lib.FLAG_EXTV,
                         _state_cls=_ExtvState)
        self._externalV = _ExternalPotential(self, geometry)

    def SetTolerances(self, phi_floor_tol, phi_ceiling_tol):
        """Sets State.phi_floor_tol / State.phi_ceiling_tol (simulation.py:143-144) on the plan."""
        _lib.check(self.plan.lib.pfc_extv_set_tolerances(self.plan.handle, float(phi_floor_tol),
                                                         float(phi_ceiling_tol)))
        self.State.phi_floor_tol, self.State.phi_ceiling_tol = float(phi_floor_tol), float(phi_ceiling_tol)

    def Get_local_phi(self):
        """Gaussian-coarsened phi (simulation.py:407-417)."""
        return self._get_local()

    def GetForce(self):
        """-grad V (simulation.py:453-466), from the potential last set (host FP64)."""
        g = self.Geometry
        vh = np.fft.rfft2(self._externalV.V)
        gx = np.fft.irfft2(1j * g.KX * vh, s=g.X.shape)
        gy = np.fft.irfft2(1j * g.KY * vh, s=g.X.shape)
        return -np.stack((gx, gy))


def BuildB200_Simulation(modelParameters, geometry, device=None, graphs=True):
    return Simulation(modelParameters, geometry, device=device, graphs=graphs)


def BuildCupyGPU_Simulation(modelParameters, geometry):
    """Drop-in name of models/logpfc_extv/simulation.py:500-521."""
    return Simulation(modelParameters, geometry)
