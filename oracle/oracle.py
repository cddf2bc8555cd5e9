"""ctypes wrapper of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA engine.  Only tests/,
__graft_entry__.smoke() and the cpu_baseline leg of bench.py may use it.  It restates
the reference path (xinzhixue/PIV_xcorr2d_V1.0, xcorr2d_V1.0/xcorr2d_multi_grid.cu and
MHE7_4_gpu.cu); see piv_oracle.h for the function-by-function citations.  Parity is
pinned by tests/golden/ fixtures produced by the reference engine itself rebuilt for
sm_100a (tests/golden/make_golden.py) and by the grid-count and Tecplot-format facts
of the reference's sample outputs.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "liboracle.so"


class OrParams(C.Structure):
    _fields_ = [("Nx", C.c_int), ("Ny", C.c_int), ("Nsec_cc", C.c_int),
                ("ws_x", C.c_int * 2), ("ws_y", C.c_int * 2), ("sp_x", C.c_int * 2), ("sp_y", C.c_int * 2),
                ("Npass", C.c_int * 2), ("wx_med", C.c_int * 2), ("wy_med", C.c_int * 2),
                ("wx_sm", C.c_int * 2), ("wy_sm", C.c_int * 2), ("Npeak_save", C.c_int),
                ("pct_x", C.c_float * 2), ("pct_y", C.c_float * 2),
                ("lim_x1", C.c_float), ("lim_x2", C.c_float), ("lim_y1", C.c_float), ("lim_y2", C.c_float)]


GEOM = ["border_x", "border_y", "hfws_x", "hfws_y", "Npeak", "Nx_vec", "Ny_vec", "Nt_vec", "Neach", "Nlast", "Nsec",
        "Nx_left", "Nx_right", "Ny_left", "Ny_right", "Nx_aug", "Ny_aug", "Nx_aug_ex", "Ny_aug_ex"]


class OrGeom(C.Structure):
    _fields_ = [(n, C.c_int * 2) for n in GEOM]

    def to_dict(self):
        return {n: tuple(getattr(self, n)) for n in GEOM}


class OrValidCfg(C.Structure):
    _fields_ = [("Npass_median", C.c_int), ("minNneigh", C.c_int), ("insert_threshold", C.c_float),
                ("Npass_smooth", C.c_int), ("iffill", C.c_int)]


_FP = C.POINTER(C.c_float)
_U8P = C.POINTER(C.c_uint8)
_I32P = C.POINTER(C.c_int32)


class OrCandidates(C.Structure):
    _fields_ = [("dx", _FP), ("dy", _FP), ("valid", _U8P), ("count", _I32P), ("peak_index", _I32P),
                ("peak_value", _FP), ("flags", _U8P)]


class OrPairOut(C.Structure):
    _fields_ = [("raw", OrCandidates * 2), ("fx", _FP * 2), ("fy", _FP * 2), ("fvalid", _U8P * 2),
                ("fx2_median", _FP), ("fy2_median", _FP), ("fvalid2_median", _U8P), ("deform_oob", C.c_long)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"oracle library missing: {LIB_PATH} (make -C {_HERE})")
        h = C.CDLL(str(LIB_PATH))
        h.or_geometry.argtypes = [C.POINTER(OrParams), C.POINTER(OrGeom)]
        h.or_mhe.argtypes = [_U8P, C.c_int, C.c_int, C.c_int, C.c_float, _U8P]
        h.or_xcorr_plane.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int, C.c_int,
                                     C.POINTER(C.c_double), C.c_int]
        h.or_xcorr_plane.restype = None
        h.or_deform.argtypes = [_U8P, C.POINTER(OrParams), C.POINTER(OrGeom), C.c_int, _FP, _FP, _FP]
        h.or_deform.restype = C.c_long
        h.or_upsample.argtypes = [C.POINTER(OrParams), C.POINTER(OrGeom), _FP, _FP, _FP, _FP]
        h.or_upsample.restype = None
        h.or_correlate_grid.argtypes = [_U8P, _U8P, _FP, C.POINTER(OrParams), C.POINTER(OrGeom), C.c_int, _FP, _FP,
                                        C.c_int, C.POINTER(OrCandidates)]
        h.or_peaks_from_planes.argtypes = [_FP, C.POINTER(OrParams), C.POINTER(OrGeom), C.c_int, _FP, _FP,
                                           C.POINTER(OrCandidates)]
        h.or_validate.argtypes = [_FP, _FP, _U8P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                  C.POINTER(OrValidCfg), _FP, _FP, _U8P, C.POINTER(C.c_int)]
        h.or_run_pair.argtypes = [_U8P, _U8P, C.POINTER(OrParams), C.POINTER(OrValidCfg), C.POINTER(OrValidCfg),
                                  C.c_int, C.POINTER(OrPairOut)]
        h.or_write_tecplot.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _FP, _FP]
        h.or_num_threads.restype = C.c_int
        h.or_set_num_threads.argtypes = [C.c_int]
        h.or_set_num_threads.restype = None
        _lib = h
    return _lib


def _p(a, ct):
    return None if a is None else a.ctypes.data_as(C.POINTER(ct))


def params_from(p) -> OrParams:
    """From an engine PivParams (or anything with the same attribute names)."""
    o = OrParams()
    o.Nx, o.Ny, o.Nsec_cc = p.Nx, p.Ny, p.Nsec_cc
    o.ws_x[:] = [p.ws_x1, p.ws_x2]
    o.ws_y[:] = [p.ws_y1, p.ws_y2]
    o.sp_x[:] = [p.spacing_x1, p.spacing_x2]
    o.sp_y[:] = [p.spacing_y1, p.spacing_y2]
    o.Npass[:] = [p.Npass1, p.Npass2]
    o.wx_med[:] = [p.wx1_median, p.wx2_median]
    o.wy_med[:] = [p.wy1_median, p.wy2_median]
    o.wx_sm[:] = [p.wx1_smooth, p.wx2_smooth]
    o.wy_sm[:] = [p.wy1_smooth, p.wy2_smooth]
    o.Npeak_save = p.Npeak_save
    o.pct_x[:] = [p.max_dispx_win_percent1, p.max_dispx_win_percent2]
    o.pct_y[:] = [p.max_dispy_win_percent1, p.max_dispy_win_percent2]
    o.lim_x1, o.lim_x2, o.lim_y1, o.lim_y2 = p.dispx_lim1, p.dispx_lim2, p.dispy_lim1, p.dispy_lim2
    return o


def valid_cfgs(p):
    v1 = OrValidCfg(p.Npass1_median, p.minNneigh_p1, p.insert_threshold_p1, p.Npass1_smooth, 1)
    v2 = OrValidCfg(p.Npass2_median, p.minNneigh_p2, p.insert_threshold_p2, p.Npass2_smooth, 1)
    return v1, v2


def geometry(op: OrParams):
    g = OrGeom()
    rc = lib().or_geometry(C.byref(op), C.byref(g))
    return rc, g


def mhe(img: np.ndarray, ws: int, thresh: float) -> np.ndarray:
    img = np.ascontiguousarray(img, np.uint8)
    out = np.empty_like(img)
    rc = lib().or_mhe(_p(img, C.c_uint8), img.shape[1], img.shape[0], ws, thresh, _p(out, C.c_uint8))
    if rc:
        raise ValueError(f"or_mhe failed ({rc})")
    return out


def xcorr_plane(w1, w2, direct=False):
    w1 = np.ascontiguousarray(w1, np.float64)
    w2 = np.ascontiguousarray(w2, np.float64)
    wsy, wsx = w1.shape
    out = np.empty((wsy, wsx), np.float64)
    lib().or_xcorr_plane(_p(w1, C.c_double), _p(w2, C.c_double), wsx, wsy, _p(out, C.c_double), int(direct))
    return out


class Candidates:
    def __init__(self, nt, nps):
        self.dx = np.zeros((nt, nps), np.float32)
        self.dy = np.zeros((nt, nps), np.float32)
        self.valid = np.zeros((nt, nps), np.uint8)
        self.count = np.zeros(nt, np.int32)
        self.peak_index = np.zeros((nt, nps), np.int32)
        self.peak_value = np.zeros((nt, nps), np.float32)
        self.flags = np.zeros(nt, np.uint8)

    def struct(self):
        return OrCandidates(_p(self.dx, C.c_float), _p(self.dy, C.c_float), _p(self.valid, C.c_uint8),
                            _p(self.count, C.c_int32), _p(self.peak_index, C.c_int32), _p(self.peak_value, C.c_float),
                            _p(self.flags, C.c_uint8))


def correlate_grid(img1, img2, deformed, op, g, grid, pred_x, pred_y, direct=False) -> Candidates:
    nt = g.Nt_vec[grid]
    c = Candidates(nt, op.Npeak_save)
    s = c.struct()
    img1 = np.ascontiguousarray(img1, np.uint8)
    img2 = None if img2 is None else np.ascontiguousarray(img2, np.uint8)
    deformed = None if deformed is None else np.ascontiguousarray(deformed, np.float32)
    px = np.ascontiguousarray(pred_x, np.float32)
    py = np.ascontiguousarray(pred_y, np.float32)
    rc = lib().or_correlate_grid(_p(img1, C.c_uint8), _p(img2, C.c_uint8), _p(deformed, C.c_float), C.byref(op),
                                 C.byref(g), grid, _p(px, C.c_float), _p(py, C.c_float), int(direct), C.byref(s))
    if rc:
        raise ValueError(f"or_correlate_grid failed ({rc})")
    return c


def peaks_from_planes(cc, op, g, grid, pred_x, pred_y) -> Candidates:
    nt = cc.shape[0]
    c = Candidates(nt, op.Npeak_save)
    s = c.struct()
    cc = np.ascontiguousarray(cc, np.float32)
    px = np.ascontiguousarray(pred_x, np.float32)
    py = np.ascontiguousarray(pred_y, np.float32)
    # the oracle iterates over the grid's windows: pass a sub-geometry for a window subset
    rc = lib().or_peaks_from_planes(_p(cc, C.c_float), C.byref(op), C.byref(g), grid, _p(px, C.c_float),
                                    _p(py, C.c_float), C.byref(s))
    if rc:
        raise ValueError(f"or_peaks_from_planes failed ({rc})")
    return c


def deform(img2, op, g, grid, fx, fy):
    out = np.empty((g.Ny_aug[grid], g.Nx_aug[grid]), np.float32)
    img2 = np.ascontiguousarray(img2, np.uint8)
    fx = np.ascontiguousarray(fx, np.float32)
    fy = np.ascontiguousarray(fy, np.float32)
    oob = lib().or_deform(_p(img2, C.c_uint8), C.byref(op), C.byref(g), grid, _p(fx, C.c_float), _p(fy, C.c_float),
                          _p(out, C.c_float))
    return out, oob


def upsample(op, g, fx1, fy1):
    n2 = g.Nt_vec[1]
    fx2 = np.empty(n2, np.float32)
    fy2 = np.empty(n2, np.float32)
    fx1 = np.ascontiguousarray(fx1, np.float32)
    fy1 = np.ascontiguousarray(fy1, np.float32)
    lib().or_upsample(C.byref(op), C.byref(g), _p(fx1, C.c_float), _p(fy1, C.c_float), _p(fx2, C.c_float),
                      _p(fy2, C.c_float))
    return fx2, fy2


def validate(cdx, cdy, cvalid, nx, ny, nps, wx_med, wy_med, wx_sm, wy_sm, Npass_median, minN, thr, Npass_smooth,
             iffill):
    cdx = np.ascontiguousarray(cdx, np.float32)
    cdy = np.ascontiguousarray(cdy, np.float32)
    cvalid = np.ascontiguousarray(cvalid, np.uint8)
    fx = np.empty(nx * ny, np.float32)
    fy = np.empty(nx * ny, np.float32)
    fv = np.empty(nx * ny, np.uint8)
    it = C.c_int(0)
    cfg = OrValidCfg(Npass_median, minN, thr, Npass_smooth, iffill)
    rc = lib().or_validate(_p(cdx, C.c_float), _p(cdy, C.c_float), _p(cvalid, C.c_uint8), nx, ny, nps, wx_med, wy_med,
                           wx_sm, wy_sm, C.byref(cfg), _p(fx, C.c_float), _p(fy, C.c_float), _p(fv, C.c_uint8),
                           C.byref(it))
    if rc:
        raise ValueError(f"or_validate failed ({rc})")
    return fx, fy, fv, it.value


def run_pair(img1, img2, p, direct=False):
    """Whole pair with engine-style params p (PivParams). Returns a dict of numpy arrays."""
    op = params_from(p)
    rc, g = geometry(op)
    if rc:
        raise ValueError(f"geometry rejected ({rc})")
    v1, v2 = valid_cfgs(p)
    nps = p.Npeak_save
    c = [Candidates(g.Nt_vec[k], nps) for k in range(2)]
    f = [[np.zeros(g.Nt_vec[k], np.float32), np.zeros(g.Nt_vec[k], np.float32), np.zeros(g.Nt_vec[k], np.uint8)]
         for k in range(2)]
    med = [np.zeros(g.Nt_vec[1], np.float32), np.zeros(g.Nt_vec[1], np.float32), np.zeros(g.Nt_vec[1], np.uint8)]
    out = OrPairOut()
    for k in range(2):
        out.raw[k] = c[k].struct()
        out.fx[k] = _p(f[k][0], C.c_float)
        out.fy[k] = _p(f[k][1], C.c_float)
        out.fvalid[k] = _p(f[k][2], C.c_uint8)
    out.fx2_median = _p(med[0], C.c_float)
    out.fy2_median = _p(med[1], C.c_float)
    out.fvalid2_median = _p(med[2], C.c_uint8)
    img1 = np.ascontiguousarray(img1, np.uint8)
    img2 = np.ascontiguousarray(img2, np.uint8)
    rc = lib().or_run_pair(_p(img1, C.c_uint8), _p(img2, C.c_uint8), C.byref(op), C.byref(v1), C.byref(v2),
                           int(direct), C.byref(out))
    if rc:
        raise ValueError(f"or_run_pair failed ({rc})")
    return {"geom": g.to_dict(), "raw": c, "filt": f, "median_only": med, "deform_oob": out.deform_oob}


def write_tecplot(path, nx, ny, spx, spy, raw, nps, dx, dy):
    dx = np.ascontiguousarray(dx, np.float32)
    dy = np.ascontiguousarray(dy, np.float32)
    return lib().or_write_tecplot(str(path).encode(), nx, ny, spx, spy, int(raw), nps, _p(dx, C.c_float),
                                  _p(dy, C.c_float))


def set_threads(n):
    lib().or_set_num_threads(int(n))


def threads():
    return lib().or_num_threads()
