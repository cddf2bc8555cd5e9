"""ctypes wrapper of the reference engine rebuilt for sm_100a (oracle/_ref/libref_xcorr2d.so,
built from the reference sources by `make -C oracle ref`; see ref/ref_capi.cu).

TEST AND BASELINE INFRASTRUCTURE ONLY.  Used by tests/golden/make_golden.py to record
the reference's own outputs as fixtures, and by bench.py's reference arm.  Needs a GPU.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "_ref" / "libref_xcorr2d.so"

_FIELDS = [
    ("device_id", C.c_int), ("ifmhe", C.c_int), ("mhe_ws", C.c_int), ("mhe_thresh", C.c_float),
    ("Nx", C.c_int), ("Ny", C.c_int),
    ("ws_x1", C.c_int), ("ws_y1", C.c_int), ("spacing_x1", C.c_int), ("spacing_y1", C.c_int), ("Npass1", C.c_int),
    ("ws_x2", C.c_int), ("ws_y2", C.c_int), ("spacing_x2", C.c_int), ("spacing_y2", C.c_int), ("Npass2", C.c_int),
    ("Nsec_cc", C.c_int),
    ("wx1_median", C.c_int), ("wy1_median", C.c_int), ("Npass1_median", C.c_int), ("minNneigh_p1", C.c_int),
    ("residual_threshold_p1", C.c_float), ("insert_threshold_p1", C.c_float),
    ("wx1_smooth", C.c_int), ("wy1_smooth", C.c_int), ("Npass1_smooth", C.c_int),
    ("wx2_median", C.c_int), ("wy2_median", C.c_int), ("Npass2_median", C.c_int), ("minNneigh_p2", C.c_int),
    ("residual_threshold_p2", C.c_float), ("insert_threshold_p2", C.c_float),
    ("wx2_smooth", C.c_int), ("wy2_smooth", C.c_int), ("Npass2_smooth", C.c_int),
    ("max_dispx_win_percent1", C.c_float), ("max_dispy_win_percent1", C.c_float),
    ("max_dispx_win_percent2", C.c_float), ("max_dispy_win_percent2", C.c_float),
    ("Npeak_save", C.c_int),
    ("dispx_lim1", C.c_float), ("dispx_lim2", C.c_float), ("dispy_lim1", C.c_float), ("dispy_lim2", C.c_float),
]


class RefParams(C.Structure):
    _fields_ = _FIELDS


def params_from(p) -> RefParams:
    r = RefParams()
    for name, _ in _FIELDS:
        setattr(r, name, getattr(p, "if_mhe" if name == "ifmhe" else name))
    return r


_lib = None
_P = C.c_void_p
_FP = C.POINTER(C.c_float)
_U8P = C.POINTER(C.c_uint8)
_I32P = C.POINTER(C.c_int32)


def available() -> bool:
    return LIB_PATH.exists()


def lib():
    global _lib
    if _lib is None:
        h = C.CDLL(str(LIB_PATH))
        h.ref_create.argtypes = [C.POINTER(RefParams), C.POINTER(_P)]
        h.ref_destroy.argtypes = [_P]
        h.ref_destroy.restype = None
        h.ref_mhe.argtypes = [_P, _U8P, _U8P]
        h.ref_run_pair.argtypes = [_P, _U8P, _U8P]
        h.ref_run_pair_recording.argtypes = [_P, _U8P, _U8P, _FP, _FP, _FP, _FP]
        h.ref_median_only.argtypes = [_P]
        h.ref_get_raw.argtypes = [_P, C.c_int, _FP, _FP, _U8P]
        h.ref_set_raw.argtypes = [_P, C.c_int, _FP, _FP, _U8P]
        h.ref_validate.argtypes = [_P, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_int, C.c_int]
        h.ref_get_filtered.argtypes = [_P, C.c_int, _FP, _FP, _U8P]
        h.ref_get_peaks.argtypes = [_P, C.c_int, _I32P, _I32P, _FP]
        h.ref_get_cc.argtypes = [_P, C.c_int, C.c_int, C.c_int, _FP]
        h.ref_get_deformed.argtypes = [_P, C.c_int, _FP]
        h.ref_write_tecplot.argtypes = [_P, C.c_char_p, C.c_int]
        _lib = h
    return _lib


def _p(a, ct):
    return a.ctypes.data_as(C.POINTER(ct))


class RefEngine:
    def __init__(self, p):
        self.p = p
        self.rp = params_from(p)
        h = _P()
        rc = lib().ref_create(C.byref(self.rp), C.byref(h))
        if rc:
            raise RuntimeError(f"reference init failed ({rc})")
        self.h = h

    def close(self):
        if self.h:
            lib().ref_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def mhe(self, img):
        img = np.ascontiguousarray(img, np.uint8)
        out = np.empty_like(img)
        rc = lib().ref_mhe(self.h, _p(img, C.c_uint8), _p(out, C.c_uint8))
        if rc:
            raise RuntimeError(f"reference MHE failed ({rc})")
        return out

    def run_pair(self, f1, f2):
        f1 = np.ascontiguousarray(f1, np.uint8)
        f2 = np.ascontiguousarray(f2, np.uint8)
        rc = lib().ref_run_pair(self.h, _p(f1, C.c_uint8), _p(f2, C.c_uint8))
        if rc:
            raise RuntimeError(f"reference pair failed ({rc})")

    def run_pair_recording(self, f1, f2, nt1, nt2):
        """run_pair that also returns the filtered field each grid's last pass starts from."""
        f1 = np.ascontiguousarray(f1, np.uint8)
        f2 = np.ascontiguousarray(f2, np.uint8)
        out = {k: np.zeros(n, np.float32) for k, n in (("p1x", nt1), ("p1y", nt1), ("p2x", nt2), ("p2y", nt2))}
        rc = lib().ref_run_pair_recording(self.h, _p(f1, C.c_uint8), _p(f2, C.c_uint8),
                                          _p(out["p1x"], C.c_float), _p(out["p1y"], C.c_float),
                                          _p(out["p2x"], C.c_float), _p(out["p2y"], C.c_float))
        if rc:
            raise RuntimeError(f"reference pair failed ({rc})")
        return out

    def median_only(self):
        rc = lib().ref_median_only(self.h)
        if rc:
            raise RuntimeError(f"reference median-only failed ({rc})")

    def raw(self, grid, nt):
        n = nt * self.p.Npeak_save
        dx = np.empty(n, np.float32)
        dy = np.empty(n, np.float32)
        v = np.empty(n, np.uint8)
        lib().ref_get_raw(self.h, grid, _p(dx, C.c_float), _p(dy, C.c_float), _p(v, C.c_uint8))
        return dx.reshape(nt, -1), dy.reshape(nt, -1), v.reshape(nt, -1)

    def set_raw(self, grid, dx, dy, valid):
        """Raw candidates [Nt][Npeak_save] into the reference's arrays of a grid."""
        dx = np.ascontiguousarray(dx, np.float32)
        dy = np.ascontiguousarray(dy, np.float32)
        valid = np.ascontiguousarray(valid, np.uint8)
        rc = lib().ref_set_raw(self.h, grid, _p(dx, C.c_float), _p(dy, C.c_float), _p(valid, C.c_uint8))
        if rc:
            raise RuntimeError(f"reference set_raw failed ({rc})")

    def validate(self, grid, Npass_median, minN, rthr, ithr, Npass_smooth, iffill=1):
        """The reference's MedianFilter_Smoothing_p1/_p2 on the grid's current raw candidates."""
        rc = lib().ref_validate(self.h, grid, Npass_median, minN, rthr, ithr, Npass_smooth, iffill)
        if rc:
            raise RuntimeError(f"reference validation failed ({rc})")

    def filtered(self, grid, nt):
        dx = np.empty(nt, np.float32)
        dy = np.empty(nt, np.float32)
        v = np.empty(nt, np.uint8)
        lib().ref_get_filtered(self.h, grid, _p(dx, C.c_float), _p(dy, C.c_float), _p(v, C.c_uint8))
        return dx, dy, v

    def peaks(self, grid, nt):
        cnt = np.empty(nt, np.int32)
        idx = np.empty((nt, self.p.Npeak_save), np.int32)
        val = np.empty((nt, self.p.Npeak_save), np.float32)
        lib().ref_get_peaks(self.h, grid, _p(cnt, C.c_int32), _p(idx, C.c_int32), _p(val, C.c_float))
        return cnt, idx, val

    def cc(self, grid, first, n, wsx, wsy):
        out = np.empty((n, wsy, wsx), np.float32)
        lib().ref_get_cc(self.h, grid, first, n, _p(out, C.c_float))
        return out

    def deformed(self, grid, ny_aug, nx_aug):
        out = np.empty((ny_aug, nx_aug), np.float32)
        lib().ref_get_deformed(self.h, grid, _p(out, C.c_float))
        return out

    def write_tecplot(self, path, selection):
        return lib().ref_write_tecplot(self.h, str(path).encode(), selection)
