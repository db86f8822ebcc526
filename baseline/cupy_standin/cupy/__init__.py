"""A stand-in for the `cupy` module, backed by torch tensors.

BASELINE INFRASTRUCTURE, not product code. It lets the reference's own CuPy models
(`pfc_models.models.stdpfc`, `logpfc`, `logpfc_extv`) run unmodified where CuPy is not
installed: on a CUDA device it times the reference's GPU path (cuFFT through torch.fft,
one elementwise kernel per array operation, as CuPy issues them); on the host (no CUDA
device, or PFC_CUPY_STANDIN_DEVICE=cpu) it runs the same code in FP64 on the CPU to
generate fixtures. It implements only what those models call: `asarray`, `zeros`,
`where`, `log`, `exp`, `tanh`, `abs`, `fft.rfft2/irfft2`, the numpy dtype aliases, an
array type with views, slice assignment, arithmetic, comparisons, `.get()`, `.min()`,
`.max()`, `.mean()`, `.flat`, and numpy ufunc / `np.where` dispatch (the reference's
`kernel_etd` applies numpy functions to device arrays, as CuPy allows). Host scalars
enter device arithmetic in double precision.
"""
from __future__ import annotations

import os

import numpy as np
import torch

float32 = np.float32
float64 = np.float64
complex64 = np.complex64
complex128 = np.complex128
bool_ = np.bool_

_TORCH = {np.dtype(np.float32): torch.float32, np.dtype(np.float64): torch.float64,
          np.dtype(np.complex64): torch.complex64, np.dtype(np.complex128): torch.complex128,
          np.dtype(np.bool_): torch.bool, np.dtype(np.int64): torch.int64, np.dtype(np.int32): torch.int32}
_NUMPY = {v: k for k, v in _TORCH.items()}


def _device():
    want = os.environ.get("PFC_CUPY_STANDIN_DEVICE")
    if want:
        return torch.device(want)
    return torch.device("cuda") if torch.cuda.is_available() else torch.device("cpu")


DEVICE = _device()


def _tdtype(dtype):
    if dtype is None:
        return None
    if isinstance(dtype, torch.dtype):
        return dtype
    return _TORCH[np.dtype(dtype)]


def _unwrap(x):
    if isinstance(x, ndarray):
        return x._t
    if isinstance(x, np.ndarray):
        return torch.as_tensor(x, device=DEVICE)
    if isinstance(x, np.generic):
        return x.item()
    return x


def _scalar_tensor(x):
    """A host scalar as a 0-d device tensor in double precision (torch's default dtype,
    float32, would round it)."""
    dt = torch.complex128 if isinstance(x, complex) else torch.float64
    return torch.as_tensor(x, dtype=dt, device=DEVICE)


class _Flat:
    def __init__(self, arr):
        self.arr = arr

    def __getitem__(self, i):
        return ndarray(self.arr._t.reshape(-1)[i])

    def __setitem__(self, i, v):
        self.arr._t.view(-1)[i] = _unwrap(v)


class ndarray:
    """A device array: a torch tensor with the numpy/CuPy operator surface the models use."""

    __array_priority__ = 1000

    def __init__(self, t):
        self._t = t

    @property
    def shape(self):
        return tuple(self._t.shape)

    @property
    def dtype(self):
        return _NUMPY[self._t.dtype]

    @property
    def ndim(self):
        return self._t.ndim

    @property
    def size(self):
        return self._t.numel()

    @property
    def real(self):
        return ndarray(self._t.real if self._t.is_complex() else self._t)

    @property
    def imag(self):
        return ndarray(self._t.imag)

    @property
    def flat(self):
        return _Flat(self)

    def get(self):
        return self._t.detach().cpu().numpy().copy()

    def __array__(self, dtype=None, copy=None):
        a = self.get()
        return a.astype(dtype) if dtype is not None else a

    def __float__(self):
        return float(self._t.item())

    def __int__(self):
        return int(self._t.item())

    def __bool__(self):
        return bool(self._t.item())

    def item(self):
        return self._t.item()

    def copy(self):
        return ndarray(self._t.clone())

    def astype(self, dtype):
        return ndarray(self._t.to(_tdtype(dtype)))

    # reductions (0-d device arrays, as CuPy returns)
    def min(self):
        return ndarray(self._t.min())

    def max(self):
        return ndarray(self._t.max())

    def mean(self):
        return ndarray(self._t.mean())

    def sum(self):
        return ndarray(self._t.sum())

    def __getitem__(self, key):
        key = tuple(_unwrap(k) for k in key) if isinstance(key, tuple) else _unwrap(key)
        return ndarray(self._t[key])

    def __setitem__(self, key, value):
        key = tuple(_unwrap(k) for k in key) if isinstance(key, tuple) else _unwrap(key)
        v = _unwrap(value)
        if torch.is_tensor(v):
            v = v.to(self._t.dtype)
        self._t[key] = v

    def __len__(self):
        return self._t.shape[0]

    def _bin(self, other, f):
        return ndarray(f(self._t, _unwrap(other)))

    def __add__(self, o): return self._bin(o, torch.add)
    def __radd__(self, o): return ndarray(_unwrap(o) + self._t)
    def __sub__(self, o): return self._bin(o, torch.sub)
    def __rsub__(self, o): return ndarray(_unwrap(o) - self._t)
    def __mul__(self, o): return self._bin(o, torch.mul)
    def __rmul__(self, o): return ndarray(_unwrap(o) * self._t)
    def __truediv__(self, o): return self._bin(o, torch.div)
    def __rtruediv__(self, o): return ndarray(_unwrap(o) / self._t)
    def __pow__(self, o): return ndarray(self._t ** _unwrap(o))
    def __rpow__(self, o): return ndarray(_unwrap(o) ** self._t)
    def __neg__(self): return ndarray(-self._t)
    def __abs__(self): return ndarray(self._t.abs())
    def __gt__(self, o): return self._bin(o, torch.gt)
    def __ge__(self, o): return self._bin(o, torch.ge)
    def __lt__(self, o): return self._bin(o, torch.lt)
    def __le__(self, o): return self._bin(o, torch.le)

    def __iadd__(self, o):
        self._t += _unwrap(o)
        return self

    def __isub__(self, o):
        self._t -= _unwrap(o)
        return self

    def __imul__(self, o):
        self._t *= _unwrap(o)
        return self

    # numpy dispatch (np.exp(device array) and np.where run on the device, as in CuPy)
    _UFUNCS = {np.exp: torch.exp, np.log: torch.log, np.abs: torch.abs, np.absolute: torch.abs,
               np.tanh: torch.tanh, np.sqrt: torch.sqrt, np.cos: torch.cos, np.sin: torch.sin,
               np.add: torch.add, np.subtract: torch.sub, np.multiply: torch.mul,
               np.true_divide: torch.div, np.negative: torch.neg, np.power: torch.pow,
               np.greater: torch.gt, np.less: torch.lt, np.expm1: torch.expm1}

    def __array_ufunc__(self, ufunc, method, *inputs, **kwargs):
        f = self._UFUNCS.get(ufunc)
        if method != "__call__" or f is None or kwargs:
            return NotImplemented
        args = [_unwrap(x) for x in inputs]
        args = [a if torch.is_tensor(a) else _scalar_tensor(a) for a in args]
        return ndarray(f(*args))

    def __array_function__(self, func, types, args, kwargs):
        if func is np.where:
            return where(*args, **kwargs)
        if func is np.stack:
            return ndarray(torch.stack([_unwrap(a) for a in args[0]], dim=kwargs.get("axis", 0)))
        return NotImplemented

    def __repr__(self):
        return f"cupy_standin.ndarray({self._t!r})"


def asarray(x, dtype=None):
    if isinstance(x, ndarray):
        return x if dtype is None else x.astype(dtype)
    t = torch.as_tensor(np.asarray(x), device=DEVICE)
    if dtype is not None:
        t = t.to(_tdtype(dtype))
    return ndarray(t)


array = asarray


def zeros(shape, dtype=float64):
    return ndarray(torch.zeros(shape, dtype=_tdtype(dtype), device=DEVICE))


def zeros_like(a, dtype=None):
    return ndarray(torch.zeros_like(_unwrap(a), dtype=_tdtype(dtype)))


def where(cond, a, b):
    c = _unwrap(cond)
    ta, tb = _unwrap(a), _unwrap(b)
    if not torch.is_tensor(ta):
        ta = torch.as_tensor(ta, device=c.device, dtype=tb.dtype if torch.is_tensor(tb) else torch.float64)
    if not torch.is_tensor(tb):
        tb = torch.as_tensor(tb, device=c.device, dtype=ta.dtype)
    return ndarray(torch.where(c, ta, tb))


def _u(f):
    def g(x):
        t = _unwrap(x)
        return ndarray(f(t if torch.is_tensor(t) else _scalar_tensor(t)))
    return g


exp = _u(torch.exp)
log = _u(torch.log)
tanh = _u(torch.tanh)
abs = _u(torch.abs)  # noqa: A001
sqrt = _u(torch.sqrt)


class fft:  # noqa: N801  (module-like namespace: cupy.fft)
    @staticmethod
    def rfft2(a, s=None, axes=(-2, -1)):
        return ndarray(torch.fft.rfft2(_unwrap(a), s=s, dim=tuple(axes)))

    @staticmethod
    def irfft2(a, s=None, axes=(-2, -1)):
        return ndarray(torch.fft.irfft2(_unwrap(a), s=None if s is None else tuple(s), dim=tuple(axes)))


class cuda:  # noqa: N801
    class runtime:  # noqa: N801
        @staticmethod
        def getDeviceCount():  # noqa: N802
            return torch.cuda.device_count()
