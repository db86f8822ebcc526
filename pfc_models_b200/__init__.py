"""pfc_models_b200 — B200-native (sm_100a) pseudo-spectral ETD1 stepper for
standard and log phase-field-crystal models in 2D.

Submodules mirror the reference catalogue's entry points:
  stdpfc, logpfc   builders and Simulation (models/<slug>/simulation.py)
  spectral         Geometry / Build2DGeometry / kernels (discretization/spectral)
  fields           initial conditions (fields/initial_conditions_2d.py)
  diagnostics      the phase-diagram adapters' diagnose / frozen field / defect screen
  phase_diagram    adapters and batched Get_f_ABC / Find_q0Star / density scans
                   (phase_diagram/q0star.py, frozen_q.py)
The compute path is libpfc_b200.so (C ABI: include/pfc_b200.h), built by
`python -m pfc_models_b200.build`.
"""
__version__ = "0.1.0"
