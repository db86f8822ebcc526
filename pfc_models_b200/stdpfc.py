"""Standard PFC on B200: the entry points of models/stdpfc/simulation.py
(and the CPU twin models/stdpfc_cpu/simulation.py) over the sm_100a stepper.

    geometry = Build2DGeometry(Nx, Ny, Lx, Ly)
    params = BuildStdPFCModelParameters(Gamma=1, beta=..., q0=1, epsilon=..., g=..., dt=...)
    sim = BuildB200_Simulation(params, geometry, precision="fp64")   # or "fp32" (mixed)
    sim.State.n[...] = n0
    for _ in range(steps): sim.TimeStep()
    f = sim.CalculateFreeEnergy()

`BuildCupyGPU_Simulation` and `BuildNumpyCPU_Simulation` are accepted as drop-in
names for the reference's builders; both return the FP64 plain form on the GPU.
"""
from __future__ import annotations

from .simulation import ModelParameters, Simulation as _Simulation
from .spectral import Build2DGeometry, BuildDerivativeKernels, Geometry, kernel_etd, kernel_local  # noqa: F401


def BuildStdPFCModelParameters(Gamma=1.0, beta=1.0, q0=1.0, epsilon=1.0, g=1.0, dt=0.01, meanDensity=None,
                               smallZTol=2e-5):
    """models/stdpfc/simulation.py:60-80."""
    model = ModelParameters()
    model.Gamma = Gamma
    model.beta = beta
    model.q0 = q0
    model.epsilon = epsilon
    model.g = g
    model.dt = dt
    model.meanDensity = meanDensity
    model.smallZTol = smallZTol
    return model


def GetLinearKernel_mu(modelParameters, DerivativeKernels):
    """beta (q0^2 + lap)^2 + epsilon (models/stdpfc/simulation.py:83-90)."""
    p = modelParameters
    return p.beta * (p.q0**2 + DerivativeKernels.d2_dlap) ** 2 + p.epsilon


def GetLinearKernel_n(modelParameters, DerivativeKernels):
    """Gamma lap L_mu (models/stdpfc/simulation.py:92-96)."""
    return modelParameters.Gamma * DerivativeKernels.d2_dlap * GetLinearKernel_mu(modelParameters, DerivativeKernels)


class Simulation(_Simulation):
    def __init__(self, modelParameters, geometry, precision="fp64", device=None, kernels="auto", graphs=True,
                 pdl=None, one_cta=True):
        super().__init__("std", modelParameters, geometry, precision=precision, device=device, kernels=kernels,
                         graphs=graphs, pdl=pdl, one_cta=one_cta)

    def Get_local_n(self):
        """Gaussian-coarsened n of the state at the start of the last step, on the host
        (models/stdpfc/simulation.py:237-247)."""
        return self._get_local()


def BuildB200_Simulation(modelParameters, geometry, precision="fp64", device=None, kernels="auto", graphs=True,
                         pdl=None, one_cta=True):
    """precision: "fp64" (plain) or "fp32" (mixed); kernels: "auto" (power-of-two step
    kernels where the grid allows) or "generic" (mixed-radix kernels everywhere);
    graphs: replay steps from recorded CUDA graphs (blocks of 16 and single steps);
    pdl: let each power-of-two step kernel start while the one before it drains (None:
    as the tuned variant says)."""
    return Simulation(modelParameters, geometry, precision=precision, device=device, kernels=kernels, graphs=graphs,
                      pdl=pdl, one_cta=one_cta)


def BuildCupyGPU_Simulation(modelParameters, geometry, *_, precision="fp64", **__):
    """Drop-in name of models/stdpfc/simulation.py:270."""
    return Simulation(modelParameters, geometry, precision=precision)


def BuildNumpyCPU_Simulation(modelParameters, geometry, nThreads=2, precision="fp64"):
    """Drop-in name of models/stdpfc_cpu/simulation.py:287 (runs on the GPU; nThreads is ignored)."""
    return Simulation(modelParameters, geometry, precision=precision)
