"""Python host side of the stepper: the reference's `Simulation` object over the C ABI.

`Simulation` keeps the reference's public surface
(models/stdpfc/simulation.py:166-268, models/logpfc/simulation.py:161-263):
`Model`, `Geometry`, `State` (`n`/`phi`, `n_next`/`phi_next`, `n_hat`/`phi_hat`,
`mu`, `local_mu`, `nonlin_mu`, `t`, the host kernel tables), the convenience
views `n`/`phi` and `mu`, the `t` property, `TimeStep`, `CalculateFreeEnergy`
and `Get_local_n`/`Get_local_phi`. The state lives on the GPU in the plan's own
spectral layout; real-space fields are materialised on demand into device
buffers that behave like the reference's CuPy arrays for the idioms its tests
and adapters use (`[...] = array`, `.get()`, `.mean()`, `.copy()`, `.min()`,
`np.asarray(...)`).

PyTorch is used only for device memory and the current CUDA stream; all
arithmetic on the step path runs in the sm_100a kernels of libpfc_b200.so.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _lib
from . import spectral

_PRECISIONS = {"fp64": _lib.FP64_PLAIN, "plain": _lib.FP64_PLAIN, "fp64_plain": _lib.FP64_PLAIN,
               "fp32": _lib.FP32_MIXED, "mixed": _lib.FP32_MIXED, "fp32_mixed": _lib.FP32_MIXED}


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("pfc_models_b200 needs a CUDA device (B200, sm_100a); there is no CPU fallback")
    return torch


def _stream_ptr(torch, device):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


class ModelParameters:
    """Parameter holder; ints and float64 scalars are stored as np.float64, lists and
    tuples as float64 arrays (models/stdpfc/simulation.py:40-58)."""

    def __setattr__(self, name, value):
        if isinstance(value, (int, np.float64)) and not isinstance(value, bool):
            value = np.float64(value)
        elif isinstance(value, (list, tuple)):
            value = np.array(value, dtype=np.float64)
        super().__setattr__(name, value)


class Plan:
    """One C-ABI plan (pfc_plan_create ... pfc_plan_destroy) on one CUDA device."""

    def __init__(self, problem: _lib.PfcProblem, device=None):
        torch = _torch()
        self.torch = torch
        self.lib = _lib.load()
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        self.problem = problem
        self.handle = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _lib.check(self.lib.pfc_plan_create(ctypes.byref(problem), ctypes.byref(self.handle)))
        self.shape = (problem.ny, problem.nx)
        self._out3 = torch.zeros(3, dtype=torch.float64, device=self.device)

    # -- entry points
    def _s(self):
        return _stream_ptr(self.torch, self.device)

    def set_state(self, field):
        t = self.torch
        f = t.as_tensor(field, dtype=t.float64, device=self.device).contiguous()
        if tuple(f.shape) != self.shape:
            f = f.expand(self.shape).contiguous()
        _lib.check(self.lib.pfc_set_state(self.handle, _ptr(f), self._s()))
        return f

    def get_state(self, out=None):
        t = self.torch
        if out is None:
            out = t.empty(self.shape, dtype=t.float64, device=self.device)
        _lib.check(self.lib.pfc_get_state(self.handle, _ptr(out), self._s()))
        return out

    def step(self, nsteps=1):
        _lib.check(self.lib.pfc_step(self.handle, int(nsteps), self._s()))

    def step_timed(self, nsteps=1):
        """Steps and returns (ms in row kernels, ms in column kernels) from CUDA events."""
        a, b = ctypes.c_double(0), ctypes.c_double(0)
        _lib.check(self.lib.pfc_step_timed(self.handle, int(nsteps), ctypes.byref(a), ctypes.byref(b), self._s()))
        return a.value, b.value

    def reduce(self, out=None):
        out = self._out3 if out is None else out
        _lib.check(self.lib.pfc_reduce(self.handle, _ptr(out), self._s()))
        return out

    def get_field(self, which, w=2 * math.pi, out=None):
        t = self.torch
        if out is None:
            out = t.empty(self.shape, dtype=t.float64, device=self.device)
        _lib.check(self.lib.pfc_get_field(self.handle, int(which), float(w), _ptr(out), self._s()))
        return out

    def get_spectrum(self, which=_lib.SPEC_N_HAT, out=None):
        t = self.torch
        if out is None:
            out = t.empty((self.shape[0], self.shape[1] // 2 + 1), dtype=t.complex128, device=self.device)
        _lib.check(self.lib.pfc_get_spectrum(self.handle, int(which), _ptr(out), self._s()))
        return out

    def coefficients(self):
        ny, nx = self.shape
        a = np.empty((ny, nx // 2 + 1))
        b = np.empty((ny, nx // 2 + 1))
        _lib.check(self.lib.pfc_get_coefficients(self.handle, a.ctypes.data_as(ctypes.c_void_p),
                                                 b.ctypes.data_as(ctypes.c_void_p)))
        return a, b

    def status(self):
        v = ctypes.c_int32(0)
        _lib.check(self.lib.pfc_status(self.handle, ctypes.byref(v)))
        return v.value

    def info(self):
        o = (ctypes.c_int64 * 16)()
        _lib.check(self.lib.pfc_plan_info(self.handle, o))
        keys = ("rows_per_cta", "row_threads_per_fft", "row_ctas", "cols_per_cta",
                "col_threads_per_fft", "col_ctas", "row_smem", "col_smem",
                "fast", "fast_rows_per_cta", "fast_row_threads", "fast_row_ctas", "fast_row_smem",
                "fast_col_threads", "fast_col_ctas", "fast_col_smem")
        return dict(zip(keys, list(o)))

    def launches(self):
        return int(self.lib.pfc_launch_count(self.handle))

    def path(self):
        """'mixed_radix', 'pow2', 'fast_mixed' or 'one_cta': the step kernels this plan uses."""
        v = ctypes.c_int32(0)
        _lib.check(self.lib.pfc_plan_path(self.handle, ctypes.byref(v)))
        return {_lib.PATH_MIXED_RADIX: "mixed_radix", _lib.PATH_POW2: "pow2", _lib.PATH_ONE_CTA: "one_cta",
                _lib.PATH_FAST_MIXED: "fast_mixed"}[v.value]

    def variant(self):
        """{"ee_row", "ee_col", "row_tile", "fast"} of the step kernels this plan uses."""
        o = (ctypes.c_int32 * 4)()
        _lib.check(self.lib.pfc_plan_variant(self.handle, o))
        return dict(zip(("ee_row", "ee_col", "row_tile", "fast"), list(o)))

    def close(self):
        if self.handle and self.handle.value:
            self.lib.pfc_plan_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------ device arrays
class DeviceArray:
    """A device-resident array with the CuPy-style idioms the reference's callers
    use: `.get()`, `.mean()`, `.min()`, `.max()`, `.sum()`, `.std()`, `.copy()`,
    `.shape`, `.dtype`, `np.asarray(...)`, arithmetic with NumPy arrays (on the host).
    `.torch()` returns the device tensor itself."""

    __array_priority__ = 100

    def _tensor(self):
        raise NotImplementedError

    def torch(self):
        return self._tensor()

    # host views
    def get(self):
        """Host copy (a new NumPy array), staged through a pinned buffer."""
        t = self._tensor()
        stage = getattr(self, "_stage", None)
        if stage is None or stage.shape != t.shape or stage.dtype != t.dtype:
            import torch
            stage = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
            self._stage = stage
        stage.copy_(t)
        return stage.numpy().copy()

    def __array__(self, dtype=None, copy=None):
        a = self.get()
        return a.astype(dtype) if dtype is not None else a

    def copy(self):
        return self.get().copy()

    # reductions run on the device, results as NumPy scalars
    def mean(self):
        return np.float64(self._tensor().mean().item()) if not self._tensor().is_complex() else \
            np.complex128(self._tensor().mean().item())

    def sum(self):
        return np.float64(self._tensor().sum().item())

    def min(self):
        return np.float64(self._tensor().min().item())

    def max(self):
        return np.float64(self._tensor().max().item())

    def std(self):
        return np.float64(self._tensor().std(unbiased=False).item())

    @property
    def shape(self):
        return tuple(self._tensor().shape)

    @property
    def dtype(self):
        return np.complex128 if self._tensor().is_complex() else np.float64

    @property
    def size(self):
        return int(self._tensor().numel())

    @property
    def ndim(self):
        return self._tensor().dim()

    def __getitem__(self, key):
        return self.get()[key]

    def __len__(self):
        return self.shape[0]

    def __repr__(self):
        return f"{type(self).__name__}(shape={self.shape}, dtype={np.dtype(self.dtype).name}, device=cuda)"

    # arithmetic on host copies (NumPy semantics)
    def _binop(op):
        def f(self, other):
            return op(self.get(), np.asarray(other) if isinstance(other, DeviceArray) else other)
        return f

    def _rbinop(op):
        def f(self, other):
            return op(np.asarray(other) if isinstance(other, DeviceArray) else other, self.get())
        return f

    import operator as _op
    __add__ = _binop(_op.add)
    __radd__ = _rbinop(_op.add)
    __sub__ = _binop(_op.sub)
    __rsub__ = _rbinop(_op.sub)
    __mul__ = _binop(_op.mul)
    __rmul__ = _rbinop(_op.mul)
    __truediv__ = _binop(_op.truediv)
    __rtruediv__ = _rbinop(_op.truediv)
    __pow__ = _binop(_op.pow)
    __lt__ = _binop(_op.lt)
    __gt__ = _binop(_op.gt)
    __le__ = _binop(_op.le)
    __ge__ = _binop(_op.ge)
    __neg__ = lambda self: -self.get()  # noqa: E731
    __abs__ = lambda self: np.abs(self.get())  # noqa: E731
    del _binop, _rbinop, _op


class _Materialised(DeviceArray):
    """Read-only field recomputed on the device when the simulation state changes."""

    def __init__(self, sim, fill):
        self._sim = sim
        self._fill = fill
        self._buf = None
        self._version = -1

    def _tensor(self):
        if self._version != self._sim._version:
            self._buf = self._fill(self._buf)
            self._version = self._sim._version
        return self._buf


class DeviceField(_Materialised):
    """The density field (`State.n` / `State.phi`): readable like `_Materialised`,
    writable with `field[...] = array` (NumPy, torch or scalar; any index)."""

    def __setitem__(self, key, value):
        sim = self._sim
        if key is Ellipsis or (isinstance(key, slice) and key == slice(None)):
            if hasattr(value, "torch") and callable(value.torch):
                value = value.torch()
            sim._set_state(value)
            return
        t = self._tensor().clone()
        torch = sim._plan.torch
        if isinstance(value, DeviceArray):
            value = value.torch()
        t[key] = torch.as_tensor(np.asarray(value) if not torch.is_tensor(value) else value,
                                 dtype=torch.float64, device=t.device)
        sim._set_state(t)


# ------------------------------------------------------------------ state and simulation
class _SimulationState:
    """Mirror of _SimulationState (models/stdpfc/simulation.py:99-164): time, host
    kernel tables, and device views of the fields. `field_name` is 'n' or 'phi'."""

    def __init__(self, sim, field_name):
        self._sim = sim
        self.t = np.float64(0)
        g = sim.Geometry
        self.kSpaceShape = (g.Ny, g.Nx // 2 + 1)
        self.rSpaceShape = (g.Ny, g.Nx)
        self._field_name = field_name
        P = _lib
        field = DeviceField(sim, lambda buf: sim._plan.get_state(buf))
        setattr(self, field_name, field)
        setattr(self, field_name + "_next", field)
        setattr(self, field_name + "_hat", _Materialised(sim, lambda buf: sim._plan.get_spectrum(P.SPEC_N_HAT, buf)))
        self.mu = _Materialised(sim, lambda buf: sim._plan.get_field(sim._mu_flag(P.FIELD_MU), 2 * math.pi, buf))
        self.local_mu = _Materialised(
            sim, lambda buf: sim._plan.get_field(sim._mu_flag(P.FIELD_LOCAL_MU), 2 * math.pi, buf))
        self.nonlin_mu = _Materialised(
            sim, lambda buf: sim._plan.get_field(sim._mu_flag(P.FIELD_NONLIN_MU), 2 * math.pi, buf))
        self._kernels = None

    # host FP64 kernel tables, built on first use (the reference keeps them on the device)
    def _k(self):
        if self._kernels is None:
            sim = self._sim
            m, g = sim.Model, sim.Geometry
            dk = spectral.BuildDerivativeKernels(g)
            lap = dk.d2_dlap.real
            lin_n = spectral.linear_kernel_n(m.Gamma, m.beta, m.q0, m.epsilon, lap)
            A, B = spectral.kernel_etd(lin_n, m.dt, small_z_tol=m.smallZTol)
            self._kernels = dict(
                kernel_laplacian=lap, kernel_d_dx=dk.d_dx, kernel_d_dy=dk.d_dy,
                kernel_gaussian=spectral.kernel_local(g, w=2 * np.pi),
                kernel_lin_mu=spectral.linear_kernel_mu(m.beta, m.q0, m.epsilon, lap),
                kernel_linexp=A, kernel_nonlinexp=B)
        return self._kernels

    def __getattr__(self, name):
        if name.startswith("kernel_"):
            k = self._k()
            for suffix in ("_ndt", "_phidt"):
                if name.endswith(suffix):
                    name = name[: -len(suffix)]
            if name in k:
                return k[name]
        raise AttributeError(name)


def _kernel_flags(kernels, prob):
    """problem.flags bits for the `kernels` choice of a Simulation: "auto" (the variant
    the autotuner cached for this grid, else the defaults), "default", "generic" (the
    mixed-radix kernels everywhere), or a dict with any of "ee_row", "ee_col",
    "row_tile", "col_cta" (columns per CTA of the column kernel), "pdl" (1: both step kernels
    as programmatic dependent launches, 2: the column kernel only) and "packed"
    (1: the two-lane packed FP32 kernels on both passes, 2: row pass only, 3: column pass
    only; ee_* of a packed pass count values per lane), "tma" (the packed row kernel's tile
    staged by the tensor memory accelerator)."""
    if isinstance(kernels, dict):
        return _lib.flag_variant(**{k: kernels.get(k, 0) for k in ("ee_row", "ee_col", "row_tile", "col_cta",
                                                                    "pdl", "packed", "tma", "generic")})
    if kernels == "generic":
        return _lib.FLAG_GENERIC_ONLY
    if kernels == "default":
        return 0
    if kernels == "auto":
        from . import tune
        v = tune.lookup(prob.nx, prob.ny, prob.precision, prob.model)
        return _lib.flag_variant(**v) if v else 0
    raise ValueError(f"kernels must be 'auto', 'default', 'generic' or a variant dict, got {kernels!r}")


class Simulation:
    """The reference's Simulation (models/stdpfc/simulation.py:166-268) backed by a plan."""

    def __init__(self, model: str, modelParameters, geometry, precision="fp64", clamp_log=False, device=None,
                 kernels="auto", graphs=True, pdl=None, one_cta=True, _flags=0, _state_cls=None):
        if model not in ("std", "log"):
            raise ValueError(f"model must be 'std' or 'log', got {model!r}")
        if precision not in _PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(_PRECISIONS)}, got {precision!r}")
        self.Model = modelParameters
        self.Geometry = geometry
        self.model = model
        self.precision = "fp64" if _PRECISIONS[precision] == _lib.FP64_PLAIN else "fp32"
        m = modelParameters
        prob = _lib.PfcProblem()
        prob.nx, prob.ny = int(geometry.Nx), int(geometry.Ny)
        prob.model = _lib.MODEL_LOG if model == "log" else _lib.MODEL_STD
        prob.precision = _PRECISIONS[precision]
        prob.lx, prob.ly = float(geometry.Lx), float(geometry.Ly)
        prob.gamma, prob.beta, prob.q0 = float(m.Gamma), float(m.beta), float(m.q0)
        prob.epsilon, prob.g, prob.dt = float(m.epsilon), float(m.g), float(m.dt)
        prob.small_z_tol = float(getattr(m, "smallZTol", 2e-5))
        prob.min_phi = float(getattr(m, "minPhi", 0.0) or 0.0)
        prob.clamp_log = 1 if clamp_log else 0
        prob.flags = _kernel_flags(kernels, prob) | (0 if graphs else _lib.FLAG_NO_GRAPHS)
        if pdl is not None:   # None: as the variant says
            prob.flags = (prob.flags & ~(_lib.FLAG_PDL | _lib.FLAG_PDL_COL)) | (_lib.FLAG_PDL if pdl else 0)
        if not one_cta:       # small FP64 mixed-radix grids: keep the two-kernel step
            prob.flags |= _lib.FLAG_NO_ONE_CTA
        prob.flags |= int(_flags)
        self._plan = Plan(prob, device)
        self._version = 0
        self._mu_current = False
        name = "phi" if model == "log" else "n"
        self.State = (_state_cls or _SimulationState)(self, name)
        setattr(self, name, getattr(self.State, name))
        self.mu = self.State.mu

    # -- state plumbing
    def _set_state(self, value):
        self._plan.set_state(value)
        self._version += 1
        self._mu_current = False

    def _mu_flag(self, which):
        return which | (_lib.FIELD_OF_CURRENT if self._mu_current else 0)

    @property
    def t(self):
        return self.State.t

    @property
    def plan(self):
        return self._plan

    # -- stepping
    def TimeStep(self):
        """One ETD1 step (models/stdpfc/simulation.py:225-235)."""
        self._plan.step(1)
        self._version += 1
        self._mu_current = False
        self.State.t += self.Model.dt

    def TimeSteps(self, nsteps):
        """`nsteps` ETD1 steps in one call (no host round trip between steps)."""
        nsteps = int(nsteps)
        if nsteps <= 0:
            return
        self._plan.step(nsteps)
        self._version += 1
        self._mu_current = False
        for _ in range(nsteps):
            self.State.t += self.Model.dt

    # mirrors of the reference's batch hooks: after these, State.mu refers to the current field
    def _Batch1_CalcNonlinMu(self):
        self._mu_current = True
        self._version += 1

    def _Batch2_CalcMu_Terms(self):
        self._mu_current = True
        self._version += 1

    # -- observables
    def Reduce(self):
        """(F per site, mu per site, mean density), compensated FP64 on the device; one
        24-byte device-to-host copy."""
        out = self._plan.reduce().cpu().numpy()
        return np.float64(out[0]), np.float64(out[1]), np.float64(out[2])

    def CalculateFreeEnergy(self):
        """Mean free-energy density (models/stdpfc/simulation.py:249-268)."""
        return self.Reduce()[0]

    def CalculateChemicalPotential(self):
        """Mean chemical potential mu = L_mu(0) mean + <N(n)>."""
        return self.Reduce()[1]

    def CalculateMeanDensity(self):
        return self.Reduce()[2]

    def _get_local(self):
        return self._plan.get_field(_lib.FIELD_LOCAL_N, 2 * math.pi).cpu().numpy()

    def Status(self):
        return self._plan.status()


class Batch:
    """Independent simulations stepped in lockstep through pfc_batch_* (one launch per
    class and pass). Accepts `Simulation` objects or `Plan`s of any supported grid (the
    power-of-two and the mixed-radix kernels both batch); they must use one precision and
    one device. The batch borrows the plans: step it only while all of them are open.
    Closing it frees only its own tables, graphs and streams, so it may come before or
    after the plans are closed."""

    def __init__(self, items):
        self.items = list(items)
        if not self.items:
            raise ValueError("Batch needs at least one simulation")
        self.plans = [s.plan if isinstance(s, Simulation) else s for s in self.items]
        self.lib = self.plans[0].lib
        self.torch = self.plans[0].torch
        self.device = self.plans[0].device
        arr = (ctypes.c_void_p * len(self.plans))(*[p.handle.value for p in self.plans])
        self.handle = ctypes.c_void_p()
        with self.torch.cuda.device(self.device):
            _lib.check(self.lib.pfc_batch_create(arr, len(self.plans), ctypes.byref(self.handle)))

    def step(self, nsteps=1):
        """Advances every simulation by `nsteps` (stream-ordered on the current stream)."""
        nsteps = int(nsteps)
        if nsteps <= 0:
            return
        self._step_call(nsteps)
        for s in self.items:
            if isinstance(s, Simulation):
                s._version += 1
                s._mu_current = False
                for _ in range(nsteps):
                    s.State.t += s.Model.dt

    def _step_call(self, nsteps):
        _lib.check(self.lib.pfc_batch_step(self.handle, nsteps, _stream_ptr(self.torch, self.device)))

    def reduce(self):
        """(F per site, mu per site, mean density) of every simulation as an (n, 3) FP64
        array, with one device-to-host copy for the whole batch."""
        t = self.torch
        out = t.empty((len(self.plans), 3), dtype=t.float64, device=self.device)
        for i, p in enumerate(self.plans):
            p.reduce(out[i])
        return out.cpu().numpy()

    @property
    def classes(self):
        return int(self.lib.pfc_batch_classes(self.handle))

    def launches(self):
        return int(self.lib.pfc_batch_launch_count(self.handle))

    def close(self):
        if self.handle and self.handle.value:
            self.lib.pfc_batch_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class QueueBatch(Batch):
    """The same lockstep stepping as `Batch` in one persistent, cooperative launch per
    block of steps over a device list of work items (a row or column tile of one member at
    one step; pfc_queue_*), each item waiting only for the tiles of its own member that it
    needs. Members must be stdPFC plans on the one-lane power-of-two kernels with the
    values per thread the work-queue kernel is built with (`queue_kernels(nx, ny,
    precision)` gives a kernel choice that has them), sides 64 .. 1024. Results are bit
    for bit those of stepping each plan alone."""

    def __init__(self, items):
        self.items = list(items)
        if not self.items:
            raise ValueError("QueueBatch needs at least one simulation")
        self.plans = [s.plan if isinstance(s, Simulation) else s for s in self.items]
        self.lib = self.plans[0].lib
        self.torch = self.plans[0].torch
        self.device = self.plans[0].device
        arr = (ctypes.c_void_p * len(self.plans))(*[p.handle.value for p in self.plans])
        self.handle = ctypes.c_void_p()
        with self.torch.cuda.device(self.device):
            _lib.check(self.lib.pfc_queue_create(arr, len(self.plans), ctypes.byref(self.handle)))

    def _step_call(self, nsteps):
        _lib.check(self.lib.pfc_queue_step(self.handle, nsteps, _stream_ptr(self.torch, self.device)))

    def status(self):
        """Status bits of the launches so far (synchronises): 0, or STATUS_TIMEOUT when a
        bounded wait gave up (the members' states are then undefined)."""
        v = ctypes.c_int32()
        _lib.check(self.lib.pfc_queue_status(self.handle, ctypes.byref(v)))
        return v.value

    def info(self):
        """{"ctas", "ctas_per_sm", "items_per_step", "classes"} of the launch."""
        o = (ctypes.c_int32 * 4)()
        _lib.check(self.lib.pfc_queue_info(self.handle, o))
        return {"ctas": o[0], "ctas_per_sm": o[1], "items_per_step": o[2], "classes": o[3]}

    @property
    def classes(self):
        return self.info()["classes"]

    def launches(self):
        return int(self.lib.pfc_queue_launch_count(self.handle))

    def _test_wait(self, extra, wait_limit):
        _lib.check(self.lib.pfc_test_queue_wait(self.handle, int(extra), int(wait_limit)))

    def close(self):
        if self.handle and self.handle.value:
            self.lib.pfc_queue_destroy(self.handle)
            self.handle = ctypes.c_void_p()


def queue_kernels(nx, ny, precision="fp32"):
    """A `kernels` choice for plans that join a `QueueBatch`: the values per thread the
    work-queue kernel holds (FP32: 8 for rows of up to 256 sites and columns of up to 512,
    else 16; FP64: 8), row tiles of up to 256 threads within 48 KiB of shared memory and
    the widest column CTA."""
    fp64 = precision == "fp64"
    m = nx // 2
    ee_r = 8 if fp64 or m <= 128 else 16
    ee_c = 8 if fp64 or ny <= 512 else 16
    elt = 16 if fp64 else 8
    tpr = max(1, m // ee_r)
    tile = 16
    while tile > 1 and (tile * tpr > 256 or tile * (m + m // 16 + 16) * elt > 48 * 1024):
        tile //= 2
    return {"ee_row": ee_r, "ee_col": ee_c, "row_tile": tile, "col_cta": 0}


def make_parameters(**kw):
    p = ModelParameters()
    for k, v in kw.items():
        setattr(p, k, v)
    return p
