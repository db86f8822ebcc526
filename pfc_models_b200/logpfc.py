"""Log PFC on B200: the entry points of models/logpfc/simulation.py (and
models/logpfc_cpu/simulation.py) over the sm_100a stepper. The density field
is `phi` and the nonlinear chemical potential ln(phi) + g phi^2 + phi^3 is
unclamped by default, as in the reference (logpfc/simulation.py:293-296);
`clamp_log=True` selects the commented-out clamp at minPhi.
"""
from __future__ import annotations

import numpy as np

from .simulation import ModelParameters, Simulation as _Simulation
from .spectral import Build2DGeometry, BuildDerivativeKernels, Geometry, kernel_etd, kernel_local  # noqa: F401


def BuildLogPFCModelParameters(Gamma=1.0, beta=1.0, q0=1.0, epsilon=1.0, g=1.0, dt=0.01, minPhi=1e-6,
                               meanDensity=None, smallZTol=2e-5):
    """models/logpfc/simulation.py:51-75."""
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
    model.minLog = np.log(minPhi)
    return model


def GetLinearKernel_mu(modelParameters, DerivativeKernels):
    p = modelParameters
    return p.beta * (p.q0**2 + DerivativeKernels.d2_dlap) ** 2 + p.epsilon


def GetLinearKernel_phi(modelParameters, DerivativeKernels):
    """models/logpfc/simulation.py:87-91."""
    return modelParameters.Gamma * DerivativeKernels.d2_dlap * GetLinearKernel_mu(modelParameters, DerivativeKernels)


class Simulation(_Simulation):
    def __init__(self, modelParameters, geometry, precision="fp64", clamp_log=False, device=None, kernels="auto",
                 graphs=True, pdl=None, one_cta=True):
        super().__init__("log", modelParameters, geometry, precision=precision, clamp_log=clamp_log, device=device,
                         kernels=kernels, graphs=graphs, pdl=pdl, one_cta=one_cta)

    def Get_local_phi(self):
        """Gaussian-coarsened phi (models/logpfc/simulation.py:232-242)."""
        return self._get_local()


def BuildB200_Simulation(modelParameters, geometry, precision="fp64", clamp_log=False, device=None, kernels="auto",
                         graphs=True, pdl=None, one_cta=True):
    return Simulation(modelParameters, geometry, precision=precision, clamp_log=clamp_log, device=device,
                      kernels=kernels, graphs=graphs, pdl=pdl, one_cta=one_cta)


def BuildCupyGPU_Simulation(modelParameters, geometry, *_, precision="fp64", **__):
    """Drop-in name of models/logpfc/simulation.py:265 and of the CPU builder that
    carries the same name (models/logpfc_cpu/simulation.py:285, which takes nThreads)."""
    return Simulation(modelParameters, geometry, precision=precision)
