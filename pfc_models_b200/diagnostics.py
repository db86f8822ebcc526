"""3-mode crystal diagnostics on the device, for the phase-diagram adapters.

`diagnose(sim, structure, cell)` returns what the reference adapters' `diagnose`
returns (src/pfc_models/models/stdpfc_cpu/phase_diagram.py:204-215, the same in
logpfc_cpu/phase_diagram.py): `fitness` = 1 - |mean((n - n3)^2)| with n3 the field
rebuilt from the mean and the 1-, 2- and 3-mode amplitudes, `amplitudes` = (|A|, |B|,
|C|) (mean |n_hat| over each mode set, per site) and `details['maxima_per_cell']` (strict
8-neighbour periodic maxima per rectangular cell). The reference copies the field to
the host, runs an FFT, rebuilds n3 with an inverse FFT and compares in real space; here
`pfc_diagnose_modes` works on the plan's device field and spectrum (one pass over the
field, the deviation by Parseval over the few rebuilt entries) and 48 bytes come back.

`frozen_field(state, params, temp, cell)` returns the logPFC adapter's `FrozenField`
(logpfc_cpu/phase_diagram.py:465-505) with its moments A_n = sum |phi_hat / N|^2 |k_ref|^2n
and local term computed on the device (`pfc_frozen_moments`).

`STRUCTURES` holds the reference's mode tables (phase_diagram.py:57-92): the lattice's
1-, 2- and 3-mode k-vectors as (row, col) indices of one rectangular cell's half
spectrum, the sign of the amplitudes and the ansatz scale; the values are those of the
lattices, kept identical so that the same `structure` names select the same modes.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _lib


@dataclass(frozen=True)
class Structure:
    name: str
    kvectors: tuple
    amplitudeSign: int
    amplitudeScale: float
    maxima_per_cell: int | None


_TRI_MODES = (((1, 1), (2, 0), (-2, 0), (-1, 1)), ((0, 2), (3, 1), (-3, 1)), ((2, 2), (4, 0), (-4, 0), (-2, 2)))
STRUCTURES = {
    "triangle": Structure("triangle", _TRI_MODES, +1, 1.0 / 3, 2),
    "honeycomb": Structure("honeycomb", _TRI_MODES, -1, 1.0 / 3, 4),
    "stripe": Structure("stripe", (((2, 0), (-2, 0)), ((4, 0), (-4, 0)), ((6, 0), (-6, 0))), +1, 1.0 / 2, None),
}
_CELL_KEYS = ("uNx", "uNy", "Mx", "My")


@dataclass
class Diagnostics:
    """Fields of the reference's phase_diagram.q0star.Diagnostics."""
    fitness: float
    amplitudes: tuple
    details: dict = field(default_factory=dict)


def _structure(structure):
    return STRUCTURES[structure] if isinstance(structure, str) else structure


def _cell(cell):
    c = dict(cell)
    if sorted(c) != sorted(_CELL_KEYS):
        raise ValueError(f"cell needs exactly {list(_CELL_KEYS)}, got {sorted(c)}")
    out = {}
    for k in _CELL_KEYS:
        v = c[k]
        if int(v) != v or int(v) < 1:
            raise ValueError(f"cell {k}={v!r} must be a positive integer")
        out[k] = int(v)
    return out


def mode_table(structure, cell):
    """(rows, cols, sets) int32 arrays of the structure's mode indices scaled to the box
    (row * My, col * Mx), in set order."""
    st, c = _structure(structure), _cell(cell)
    rows, cols, sets = [], [], []
    for s, pos in enumerate(st.kvectors):
        for r, q in pos:
            rows.append(r * c["My"])
            cols.append(q * c["Mx"])
            sets.append(s)
    return (np.array(rows, dtype=np.int32), np.array(cols, dtype=np.int32), np.array(sets, dtype=np.int32))


def diagnose(sim, structure, cell):
    """The adapters' `diagnose` on the device (see the module docstring)."""
    import torch
    st, c = _structure(structure), _cell(cell)
    plan = sim.plan
    rows, cols, sets = mode_table(st, c)
    rc = np.ascontiguousarray(np.stack([rows, cols], axis=1).ravel(), dtype=np.int32)
    f = plan.get_state()
    spec = plan.get_spectrum(_lib.SPEC_N_HAT_NOW)
    out = torch.empty(6, dtype=torch.float64, device=f.device)
    stream = ctypes.c_void_p(torch.cuda.current_stream(f.device).cuda_stream)
    rc_err = plan.lib.pfc_diagnose_modes(plan.handle, ctypes.c_void_p(f.data_ptr()),
                                         ctypes.c_void_p(spec.data_ptr()), rc.ctypes.data_as(ctypes.c_void_p),
                                         sets.ctypes.data_as(ctypes.c_void_p), int(len(sets)),
                                         float(st.amplitudeSign), ctypes.c_void_p(out.data_ptr()), stream)
    if rc_err == _lib.PFC_E_ARG and "outside" in _lib.last_error():
        raise IndexError(_lib.last_error())
    _lib.check(rc_err)
    v = out.cpu().tolist()
    return Diagnostics(fitness=v[0], amplitudes=(v[1], v[2], v[3]),
                       details={"maxima_per_cell": v[5] / (c["Mx"] * c["My"]), "mean": v[4]})


class FrozenField:
    """f(q) of one field frozen on the grid while the box scale q00 = q changes
    (models/logpfc_cpu/phase_diagram.py:476-500): f(q) = local + beta/2 (q0^4 A0 -
    2 q0^2 q^2 A1 + q^4 A2), q_opt = q0 sqrt(A1 / A2). A and local come from the device."""

    def __init__(self, A, local, beta, q0):
        self.A = np.asarray(A, dtype=float)
        self.local = float(local)
        self.beta, self.q0 = float(beta), float(q0)

    def f(self, q):
        s, q0 = np.asarray(q, dtype=float) ** 2, self.q0
        A0, A1, A2 = self.A
        return self.local + self.beta / 2 * (q0 ** 4 * A0 - 2 * q0 ** 2 * s * A1 + s ** 2 * A2)

    def q_opt(self):
        return self.q0 * np.sqrt(self.A[1] / self.A[2])


def _log_params(params):
    p = dict(params)
    unknown = sorted(set(p) - {"beta", "g", "v0", "Gamma", "q0"})
    if unknown:
        raise ValueError(f"unknown model parameters {unknown}")
    missing = [k for k in ("beta", "g") if k not in p]
    if missing:
        raise ValueError(f"missing model parameters {missing}")
    if float(p.get("v0", 1.0)) != 1.0:
        raise ValueError("v0 must be 1.0 (the quartic coefficient of the models is 1)")
    return float(p["beta"]), float(p["g"]), 1.0, float(p.get("q0", 1.0))


def _ref_box(c):
    """The q00 = 1 box of a cell (Mx rectangular cells of width 4 pi / sqrt 3, My of 4 pi)."""
    return c["Mx"] * 4 * np.pi / np.sqrt(3.0), c["My"] * 4 * np.pi


def _field_and_spectrum(state, c):
    """(plan, device field, device spectrum, keep-alive) of a Simulation of this package
    (its own field and spectrum) or of an array of the cell's grid (its exact values on
    the device, the spectrum from an FP64 plan of the cell's q00 = 1 box)."""
    import torch
    plan = getattr(state, "plan", None)
    if plan is not None:
        return plan, plan.get_state(), plan.get_spectrum(_lib.SPEC_N_HAT_NOW), None
    from . import stdpfc
    phi = np.ascontiguousarray(np.asarray(state, dtype=float))
    nx, ny = c["uNx"] * c["Mx"], c["uNy"] * c["My"]
    if phi.shape != (ny, nx):
        raise ValueError(f"state has shape {phi.shape}, the cell's grid is {(ny, nx)}")
    lx, ly = _ref_box(c)
    prm = stdpfc.BuildStdPFCModelParameters(Gamma=1.0, beta=1.0, q0=1.0, epsilon=-0.1, g=0.0, dt=0.01)
    holder = stdpfc.BuildB200_Simulation(prm, stdpfc.Build2DGeometry(nx, ny, lx, ly), precision="fp64")
    holder.State.n[...] = phi
    plan = holder.plan
    field = torch.as_tensor(phi, device=plan.device)
    return plan, field, plan.get_spectrum(_lib.SPEC_N_HAT_NOW), holder


def frozen_field(state, params, temp, cell):
    """FrozenField of a logPFC field (the adapter's `frozen_field`, logpfc_cpu/
    phase_diagram.py:503-505). `state` is a Simulation of this package (its field and
    spectrum stay on the device) or an array of the cell's grid."""
    import torch
    beta, g, v0, q0 = _log_params(params)
    c = _cell(cell)
    lx, ly = _ref_box(c)
    plan, f, spec, _keep = _field_and_spectrum(state, c)
    out = torch.empty(4, dtype=torch.float64, device=f.device)
    stream = ctypes.c_void_p(torch.cuda.current_stream(f.device).cuda_stream)
    _lib.check(plan.lib.pfc_frozen_moments(plan.handle, ctypes.c_void_p(f.data_ptr()), ctypes.c_void_p(spec.data_ptr()),
                                           float(lx), float(ly), float(temp), g, v0, ctypes.c_void_p(out.data_ptr()),
                                           stream))
    v = out.cpu().tolist()
    return FrozenField(v[:3], v[3], beta, q0)


PEAK_SPREAD_MAX = 0.20
SUBQ_RATIO_MAX = 1e-3


def defect_diagnostics(state, cell):
    """The logPFC adapter's record-only defect screen for frozen_q (logpfc_cpu/
    phase_diagram.py:509-528) on the device: peak_spread, subq_ratio, n_peaks and
    defect_flag (either above PEAK_SPREAD_MAX / SUBQ_RATIO_MAX). `state` as for
    frozen_field."""
    import torch
    c = _cell(cell)
    lx, ly = _ref_box(c)
    plan, f, spec, _keep = _field_and_spectrum(state, c)
    out = torch.empty(4, dtype=torch.float64, device=f.device)
    stream = ctypes.c_void_p(torch.cuda.current_stream(f.device).cuda_stream)
    _lib.check(plan.lib.pfc_defect_screen(plan.handle, ctypes.c_void_p(f.data_ptr()), ctypes.c_void_p(spec.data_ptr()),
                                          float(lx), float(ly), ctypes.c_void_p(out.data_ptr()), stream))
    spread, ratio, n_peaks, _ = out.cpu().tolist()
    return dict(peak_spread=spread, subq_ratio=ratio, n_peaks=int(n_peaks),
                defect_flag=bool(spread > PEAK_SPREAD_MAX or ratio > SUBQ_RATIO_MAX))
