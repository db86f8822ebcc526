"""Minimal NumPy-backed stand-in for the parts of pyFFTW that pfc_models uses.

Used only by ``tests/golden/make_golden.py`` to run the unmodified reference
CPU models (``stdpfc_cpu``, ``logpfc_cpu``) in a container without libfftw3.
The reference calls exactly two things:

* ``pyfftw.byte_align(array, dtype=None)``: returns an aligned copy/view.
* ``pyfftw.FFTW(in, out, axes, direction, flags, threads)``: a plan whose
  ``__call__(in=None, out=None)`` executes the transform into ``out``.
  FFTW_FORWARD on a real input is an unnormalised r2c; FFTW_BACKWARD from a
  complex half spectrum to a real output is a c2r normalised by 1/N, which is
  pyFFTW's default (``normalise_idft=True``).
"""
import numpy as np


def byte_align(array, n=None, dtype=None):
    a = np.asarray(array)
    if dtype is not None:
        a = a.astype(dtype, copy=False)
    return np.ascontiguousarray(a)


class FFTW:
    def __init__(self, input_array, output_array, axes=(-1,), direction="FFTW_FORWARD",
                 flags=("FFTW_MEASURE",), threads=1, **_):
        self.input_array = input_array
        self.output_array = output_array
        self.axes = tuple(axes)
        self.direction = direction

    def __call__(self, input_array=None, output_array=None, **_):
        src = self.input_array if input_array is None else input_array
        dst = self.output_array if output_array is None else output_array
        if self.direction == "FFTW_FORWARD":
            if np.iscomplexobj(src):
                dst[...] = np.fft.fftn(src, axes=self.axes)
            else:
                dst[...] = np.fft.rfftn(src, axes=self.axes)
        else:
            if np.iscomplexobj(dst):
                dst[...] = np.fft.ifftn(src, axes=self.axes)
            else:
                shape = [dst.shape[a] for a in self.axes]
                dst[...] = np.fft.irfftn(src, s=shape, axes=self.axes)
        return dst
