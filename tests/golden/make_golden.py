"""Generate the golden fixtures in this directory from the unmodified reference.

Run in a container where the reference checkout exists (it is not needed, and
not present, where the tests run):

    NUMBA_CACHE_DIR=<scratch dir> PYTHONPYCACHEPREFIX=<scratch dir> \
        python tests/golden/make_golden.py <reference checkout>

The reference's CPU models (``pfc_models.models.stdpfc_cpu`` and
``logpfc_cpu``) import pyFFTW, which is absent here; ``pyfftw_standin/`` puts a
NumPy-backed module of that name on ``sys.path`` (forward r2c unnormalised,
backward c2r normalised by 1/N, as pyFFTW's defaults). With it the reference's
own pinned regressions reproduce to about 1e-16 relative, so the fixtures carry
the reference's arithmetic up to FFT round-off.

Every case below is written to one ``.npz`` file; ``manifest.json`` lists the
cases, their configuration and the library versions that produced them.
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

# ---------------------------------------------------------------- configurations
A_LAT = 4 * np.pi / 3**0.5      # triangular lattice spacing at q0 = 1
H_LAT = 4 * np.pi               # row spacing at q0 = 1
C12, C34, C14 = (3 / 4) ** 0.5, (3 / 4) ** 0.75, (3 / 4) ** 0.25

# stdpfc_cpu/test_regression.py:64-82 (132^2, 200 steps, vacancy crystal)
STD_REG = dict(Nx=132, Ny=132, Lx=14 * A_LAT, Ly=8 * H_LAT, Gamma=1.0, beta=C12 * 0.5, q0=1.0,
               epsilon=C12 * (-0.9 + 2 * (-2.0) + 4), g=C34 * (-2.0 + 2.5), dt=0.1,
               mean_solid=C14 * (0.55 - 1), mean_vacancy=C14 * (0.30 - 1), A0=C14 * 0.19,
               steps=200, record_every=50)

# logpfc_cpu/test_regression.py:28-55 (28x24, seeded noise, steps 10/100/1000)
LOG_Q = 0.9648639799649456
LOG_REG = dict(Nx=28, Ny=24, Lx=2 * 4 * np.pi / (np.sqrt(3) * LOG_Q), Ly=4 * np.pi / LOG_Q,
               Gamma=1.0, beta=0.5, q0=1.0, epsilon=-0.9, g=-2.0, dt=0.1, mean=0.6326,
               steps=(10, 100, 1000))

# stdPFC config 1: 256^2, dx = pi/4, dt = 0.5, r = -0.25, psi = -0.25 + U[-0.01, 0.01] (seed 0)
CONFIG1 = dict(Nx=256, Ny=256, Lx=256 * np.pi / 4, Ly=256 * np.pi / 4, Gamma=1.0, beta=1.0, q0=1.0,
               epsilon=-0.25, g=0.0, dt=0.5, mean=-0.25, noise=0.01, seed=0,
               steps=1000, record_every=100)

# tests/test_smoke_models.py:60-72, 217-223 (264^2, vacancy crystal, 100 steps, F every step)
SMOKE = dict(Nx=264, Ny=264, Lx=7 * 4 * A_LAT, Ly=4 * 4 * H_LAT, dt=0.1, steps=100)
SMOKE_LOG = dict(beta=0.5, epsilon=-0.9, g=-2.0, mean_solid=0.55, mean_vacancy=0.3, A0=0.15)
SMOKE_STD = dict(beta=C12 * 0.5, epsilon=C12 * (-0.9 + 2 * (-2.0) + 4), g=C34 * (-2.0 + 2.5),
                 mean_solid=C14 * (0.55 - 1), mean_vacancy=C14 * (0.30 - 1), A0=C14 * 0.15)

# logPFC, the example-notebook parameter set on a 128^2 cut of config 3's resolution
LOG_NOISE = dict(Nx=128, Ny=128, Lx=108 * A_LAT / 8, Ly=62 * H_LAT / 8, Gamma=1.0, beta=0.5, q0=1.0,
                 epsilon=-0.9, g=-2.0, dt=0.1, mean=0.55, noise=0.01, seed=0,
                 steps=500, record_every=100)


def _uniform_noise(shape, mean, amp, seed):
    rng = np.random.default_rng(seed)
    return mean + amp * rng.uniform(-1.0, 1.0, size=shape)


def main(ref_root):
    sys.path.insert(0, os.path.join(HERE, "pyfftw_standin"))
    sys.path.insert(0, os.path.join(ref_root, "src"))
    from pfc_models.models.stdpfc_cpu import simulation as std_cpu
    from pfc_models.models.logpfc_cpu import simulation as log_cpu
    from pfc_models.discretization.spectral import kernels as ref_kernels
    from pfc_models.discretization.spectral import geometry_2d as ref_geom
    from pfc_models.fields import initial_conditions_2d as ref_ic

    manifest = {"generator": "tests/golden/make_golden.py",
                "numpy": np.__version__, "fft": "numpy.fft (pocketfft) via pyfftw stand-in",
                "cases": {}}

    def save(name, cfg, **arrays):
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **arrays)
        manifest["cases"][name] = {"config": {k: (v if not isinstance(v, tuple) else list(v))
                                              for k, v in cfg.items()},
                                   "arrays": sorted(arrays)}
        print(f"wrote {name}.npz ({os.path.getsize(path) / 1024:.1f} KB)")

    # ------------------------------------------------ stdPFC pinned regression
    c = STD_REG
    geom = std_cpu.Build2DGeometry(Nx=c["Nx"], Ny=c["Ny"], Lx=c["Lx"], Ly=c["Ly"])
    prm = std_cpu.BuildStdPFCModelParameters(Gamma=c["Gamma"], beta=c["beta"], q0=c["q0"],
                                             epsilon=c["epsilon"], g=c["g"], dt=c["dt"],
                                             meanDensity=c["mean_solid"])
    sim = std_cpu.BuildNumpyCPU_Simulation(prm, geom, nThreads=1)
    n0 = ref_ic.GeneratePerfectCrystalInitialWithCentralVacancy(
        geom, c["mean_solid"], c["mean_vacancy"], A0=c["A0"], q0=c["q0"])
    sim.State.n[...] = n0
    steps, F, mean = [], [], []
    for s in range(c["steps"] + 1):
        if s % c["record_every"] == 0:
            steps.append(s)
            F.append(float(sim.CalculateFreeEnergy()))
            mean.append(float(sim.State.n.mean()))
        if s < c["steps"]:
            sim.TimeStep()
    save("std_regression", c, n0=n0, steps=np.array(steps), F=np.array(F), mean=np.array(mean),
         n_final=np.array(sim.State.n))

    # ------------------------------------------------ logPFC pinned regression
    c = LOG_REG
    geom = log_cpu.Build2DGeometry(Nx=c["Nx"], Ny=c["Ny"], Lx=c["Lx"], Ly=c["Ly"])
    prm = log_cpu.BuildLogPFCModelParameters(Gamma=c["Gamma"], beta=c["beta"], q0=c["q0"],
                                             epsilon=c["epsilon"], g=c["g"], dt=c["dt"],
                                             meanDensity=c["mean"])
    sim = log_cpu.BuildCupyGPU_Simulation(prm, geom, 1)
    X, Y = geom.X, geom.Y
    phi = c["mean"] * (1 + 0.15 * (2 * np.cos(np.sqrt(3) / 2 * LOG_Q * X) * np.cos(LOG_Q * Y / 2)
                                   + np.cos(LOG_Q * Y)))
    phi += 1e-3 * np.random.default_rng(7).standard_normal(phi.shape)
    phi += c["mean"] - phi.mean()
    phi0 = phi.copy()
    sim.State.phi[...] = phi
    done, F = 0, []
    for s in c["steps"]:
        for _ in range(s - done):
            sim.TimeStep()
        done = s
        F.append(float(sim.CalculateFreeEnergy()))
    save("log_regression", c, phi0=phi0, steps=np.array(c["steps"]), F=np.array(F),
         phi_final=np.array(sim.State.phi), mean_final=np.array(float(sim.State.phi.mean())))

    # ------------------------------------------------ config 1 (256^2, 1000 steps)
    c = CONFIG1
    geom = std_cpu.Build2DGeometry(Nx=c["Nx"], Ny=c["Ny"], Lx=c["Lx"], Ly=c["Ly"])
    prm = std_cpu.BuildStdPFCModelParameters(Gamma=c["Gamma"], beta=c["beta"], q0=c["q0"],
                                             epsilon=c["epsilon"], g=c["g"], dt=c["dt"],
                                             meanDensity=c["mean"])
    sim = std_cpu.BuildNumpyCPU_Simulation(prm, geom, nThreads=1)
    psi0 = _uniform_noise((c["Ny"], c["Nx"]), c["mean"], c["noise"], c["seed"])
    sim.State.n[...] = psi0
    steps, F, mean, l2 = [], [], [], []
    snaps = {}
    t0 = time.time()
    for s in range(c["steps"] + 1):
        if s % c["record_every"] == 0:
            steps.append(s)
            F.append(float(sim.CalculateFreeEnergy()))
            mean.append(float(sim.State.n.mean()))
            l2.append(float(np.sqrt(np.mean(np.square(sim.State.n)))))
            if s in (100, c["steps"]):
                snaps[f"psi_{s}"] = np.array(sim.State.n)
        if s < c["steps"]:
            sim.TimeStep()
    print(f"config1: {time.time() - t0:.1f} s")
    save("config1", c, steps=np.array(steps), F=np.array(F), mean=np.array(mean),
         rms=np.array(l2), **snaps)

    # ------------------------------------------------ smoke marches (264^2, F every step)
    for family, mod, pc in (("std", std_cpu, SMOKE_STD), ("log", log_cpu, SMOKE_LOG)):
        c = dict(SMOKE, **pc)
        geom = mod.Build2DGeometry(Nx=c["Nx"], Ny=c["Ny"], Lx=c["Lx"], Ly=c["Ly"])
        if family == "std":
            prm = mod.BuildStdPFCModelParameters(Gamma=1.0, beta=c["beta"], q0=1.0,
                                                 epsilon=c["epsilon"], g=c["g"], dt=c["dt"],
                                                 meanDensity=c["mean_solid"])
            sim = mod.BuildNumpyCPU_Simulation(prm, geom, nThreads=1)
            field = sim.State.n
        else:
            prm = mod.BuildLogPFCModelParameters(Gamma=1.0, beta=c["beta"], q0=1.0,
                                                 epsilon=c["epsilon"], g=c["g"], dt=c["dt"],
                                                 meanDensity=c["mean_solid"])
            sim = mod.BuildCupyGPU_Simulation(prm, geom, 1)
            field = sim.State.phi
        f0 = ref_ic.GeneratePerfectCrystalInitialWithCentralVacancy(
            geom, c["mean_solid"], c["mean_vacancy"], A0=c["A0"], q0=1.0)
        field[...] = f0
        F, mean = [float(sim.CalculateFreeEnergy())], [float(field.mean())]
        for _ in range(c["steps"]):
            sim.TimeStep()
            F.append(float(sim.CalculateFreeEnergy()))
            mean.append(float(field.mean()))
        save(f"smoke_{family}", c, F=np.array(F), mean=np.array(mean), field_final=np.array(field))

    # ------------------------------------------------ logPFC with noise (128^2, 500 steps)
    c = LOG_NOISE
    geom = log_cpu.Build2DGeometry(Nx=c["Nx"], Ny=c["Ny"], Lx=c["Lx"], Ly=c["Ly"])
    prm = log_cpu.BuildLogPFCModelParameters(Gamma=c["Gamma"], beta=c["beta"], q0=c["q0"],
                                             epsilon=c["epsilon"], g=c["g"], dt=c["dt"],
                                             meanDensity=c["mean"])
    sim = log_cpu.BuildCupyGPU_Simulation(prm, geom, 1)
    phi0 = _uniform_noise((c["Ny"], c["Nx"]), c["mean"], c["noise"], c["seed"])
    sim.State.phi[...] = phi0
    steps, F, mean = [], [], []
    for s in range(c["steps"] + 1):
        if s % c["record_every"] == 0:
            steps.append(s)
            F.append(float(sim.CalculateFreeEnergy()))
            mean.append(float(sim.State.phi.mean()))
        if s < c["steps"]:
            sim.TimeStep()
    save("log_noise", c, steps=np.array(steps), F=np.array(F), mean=np.array(mean),
         phi_final=np.array(sim.State.phi))

    # ------------------------------------------------ substrate: geometry, kernels, ICs
    geom = ref_geom.Build2DGeometry(Nx=28, Ny=24, Lx=2 * A_LAT * 1.1, Ly=H_LAT * 0.9)
    dk = ref_kernels.BuildDerivativeKernels(geom)
    beta, eps, q0, gam, dt = 0.5, -0.9, 1.0, 1.0, 0.1
    Lmu = beta * (q0**2 + dk.d2_dlap) ** 2 + eps
    Ln = gam * dk.d2_dlap * Lmu
    A, B = ref_kernels.kernel_etd(Ln, dt, small_z_tol=2e-5)
    gauss = ref_kernels.kernel_local(geom, w=2 * np.pi)
    ics = dict(
        crystal=ref_ic.GeneratePerfectCrystalInitialConditions(geom, 0.3, A0=0.1, q0=1.0),
        vacancy=ref_ic.GeneratePerfectCrystalInitialWithCentralVacancy(geom, 0.3, 0.1, A0=0.1),
        vacancies=ref_ic.GeneratePerfectCrystalInitialWithVancies(geom, 0.3, 0.1, [(0, 0), (1, 0)], A0=0.1),
        solid_liquid=ref_ic.GeneratePerfectCrystalInitialWithSolidLiquid(
            geom, 0.3, 0.2, [(0, 0, 1, 1)], A0=0.1),
        ring=ref_ic.GenerateDislocationRingInitialConditions(geom, 0.3, A0=0.1, radius=5.0, theta=0.3),
        hot=ref_ic.GenerateHotInitialConditions(geom, 0.4, 0.1, kMax=0.9, seed=3),
        lognormal=ref_ic.GenerateLogNormalHotInitialConditions(geom, 0.4, 0.1, kMax=0.9, seed=3),
    )
    save("substrate", dict(Nx=28, Ny=24, Lx=geom.Lx, Ly=geom.Ly, beta=beta, epsilon=eps, q0=q0,
                           Gamma=gam, dt=dt),
         X=geom.X, Y=geom.Y, KX=geom.KX, KY=geom.KY, K2=geom.K2, d2_dlap=dk.d2_dlap.real,
         A=np.real(A), B=np.real(B), gauss=gauss, **{f"ic_{k}": v for k, v in ics.items()})

    with open(os.path.join(HERE, "manifest.json"), "w") as fh:
        json.dump(manifest, fh, indent=1, sort_keys=True)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <reference checkout>")
    main(sys.argv[1])
