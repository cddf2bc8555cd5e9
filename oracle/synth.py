"""ctypes wrapper of oracle/libsynth.so: the seeded synthetic particle-image generator
(the package's csrc/synth.cpp, Philox4x32-10 streams) compiled on its own.

TEST AND BASELINE INFRASTRUCTURE ONLY.  The reference arm of bench.py and the parity tests
that drive the reference engine make their input frames with it, so that those processes
load no part of the CUDA engine (lib/libpiv_b200.so).  The frames are the same bytes as
the engine library's piv_synth_pair gives for the same parameters.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libsynth.so"

FIELD_UNIFORM, FIELD_VORTEX, FIELD_FOURIER = 0, 1, 2


class SynthParams(C.Structure):
    """piv_synth_params of include/piv_b200.h."""
    _fields_ = [("Nx", C.c_int), ("Ny", C.c_int), ("ppp", C.c_double), ("sigma", C.c_double),
                ("i_min", C.c_double), ("i_max", C.c_double), ("background", C.c_double),
                ("noise_sigma", C.c_double), ("field", C.c_int), ("a", C.c_double), ("b", C.c_double),
                ("c", C.c_double), ("seed", C.c_uint64)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"generator library missing: {LIB_PATH} (make -C {_HERE})")
        h = C.CDLL(str(LIB_PATH))
        h.piv_synth_pair.argtypes = [C.POINTER(SynthParams), C.POINTER(C.c_uint8), C.POINTER(C.c_uint8)]
        h.piv_synth_pair.restype = C.c_int
        h.piv_synth_field.argtypes = [C.POINTER(SynthParams), C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int,
                                      C.POINTER(C.c_float), C.POINTER(C.c_float)]
        h.piv_synth_field.restype = C.c_int
        _lib = h
    return _lib


def params(Nx, Ny, ppp=0.05, sigma=0.6, i_min=120.0, i_max=255.0, background=10.0, noise_sigma=2.0,
           field=FIELD_UNIFORM, a=0.0, b=0.0, c=0.0, seed=1) -> SynthParams:
    s = SynthParams()
    s.Nx, s.Ny, s.ppp, s.sigma, s.i_min, s.i_max = Nx, Ny, ppp, sigma, i_min, i_max
    s.background, s.noise_sigma, s.field, s.a, s.b, s.c, s.seed = background, noise_sigma, field, a, b, c, seed
    return s


def pair(s: SynthParams):
    """(frame 1, frame 2), uint8 [Ny, Nx] each."""
    f1 = np.empty((s.Ny, s.Nx), np.uint8)
    f2 = np.empty((s.Ny, s.Nx), np.uint8)
    rc = lib().piv_synth_pair(C.byref(s), f1.ctypes.data_as(C.POINTER(C.c_uint8)),
                              f2.ctypes.data_as(C.POINTER(C.c_uint8)))
    if rc != 0:
        raise RuntimeError(f"synthetic pair generation failed ({rc})")
    return f1, f2


def field(s: SynthParams, x, y):
    """The generator's displacement field at the points (x, y)."""
    x = np.ascontiguousarray(x, np.float32)
    y = np.ascontiguousarray(y, np.float32)
    u = np.empty_like(x)
    v = np.empty_like(x)
    fp = C.POINTER(C.c_float)
    rc = lib().piv_synth_field(C.byref(s), x.ctypes.data_as(fp), y.ctypes.data_as(fp), x.size, u.ctypes.data_as(fp),
                               v.ctypes.data_as(fp))
    if rc != 0:
        raise RuntimeError(f"field evaluation failed ({rc})")
    return u, v
