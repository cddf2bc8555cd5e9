"""B200-native multi-grid PIV correlation engine -- Python host side.

A thin ctypes layer over the C-ABI in include/piv_b200.h (lib/libpiv_b200.so).  It
mirrors the reference's engine classes so that code written against them reads the
same (paths relative to xinzhixue/PIV_xcorr2d_V1.0, X/ = xcorr2d_V1.0/):

  xcorr2d_multi   X/xcorr2d_multi_grid.cuh:12-208 (init, prep_img_data, Calc_cc_map_p1,
                  Calc_cc_map_p2, MedianFilter_Smoothing_p1/p2, extend_filtered_vecfield_p1/p2,
                  Upsampling_vector_field, write_vec_data_general, freemem; h_img1_org/h_img2_org)
  mhe_gpu         X/MHE7_4_gpu.h:7-40 (init, processsing, freemem; d_enhanced)

plus `Engine`, the parameter-file level interface (piv_create / piv_run_pair), and the
seeded synthetic pair generator.  There is no CPU fallback: every compute call goes to
the CUDA library, and loading fails loudly when the library is missing.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "lib" / "libpiv_b200.so"

PIV_OK = 0
PIV_ERR_ARG = -1
PIV_ERR_GEOMETRY = -2
PIV_ERR_UNSUPPORTED = -3
PIV_ERR_CUDA = -4
PIV_ERR_ALLOC = -5
PIV_ERR_IO = -6
PIV_ERR_STATE = -7
PIV_ERR_DEVICE = -8

PIV_XCORR_SIMT = 0
PIV_XCORR_TC_SPLIT = 1
PIV_XCORR_TC_BF16 = 2
PIV_XCORR_TC_SPLIT_F16 = 3
PIV_XCORR_TC_F16 = 4

PIV_FIELD_UNIFORM = 0
PIV_FIELD_VORTEX = 1
PIV_FIELD_FOURIER = 2

# (name, ctype) in file order: numeric lines 7..50 of the parameter file.
PARAM_FIELDS = [
    ("device_id", C.c_int), ("if_mhe", C.c_int), ("mhe_ws", C.c_int), ("mhe_thresh", C.c_float),
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


class PivParams(C.Structure):
    _fields_ = PARAM_FIELDS

    def to_dict(self):
        return {k: getattr(self, k) for k, _ in PARAM_FIELDS}


class PivPaths(C.Structure):
    _fields_ = [("prefix_f1", C.c_char * 1024), ("suffix_f1", C.c_char * 256),
                ("prefix_f2", C.c_char * 1024), ("suffix_f2", C.c_char * 256),
                ("dir_index", C.c_char * 1024), ("folder_result", C.c_char * 1024)]


GEOM_FIELDS = ["border_x", "border_y", "hfws_x", "hfws_y", "Npeak", "Nx_vec", "Ny_vec", "Nt_vec", "Neach",
               "Nlast", "Nsec", "Nx_left", "Nx_right", "Ny_left", "Ny_right", "Nx_aug", "Ny_aug", "Nx_aug_ex",
               "Ny_aug_ex"]


class PivGeometry(C.Structure):
    _fields_ = [(n, C.c_int * 2) for n in GEOM_FIELDS]

    def to_dict(self):
        return {n: tuple(getattr(self, n)) for n in GEOM_FIELDS}


class PivSynthParams(C.Structure):
    _fields_ = [("Nx", C.c_int), ("Ny", C.c_int), ("ppp", C.c_double), ("sigma", C.c_double),
                ("i_min", C.c_double), ("i_max", C.c_double), ("background", C.c_double),
                ("noise_sigma", C.c_double), ("field", C.c_int), ("a", C.c_double), ("b", C.c_double),
                ("c", C.c_double), ("seed", C.c_uint64)]


# exported entry points (name, restype, argtypes); the test suite checks this list
# against include/piv_b200.h
_P = C.c_void_p
_F = C.POINTER(C.c_float)
_U8 = C.POINTER(C.c_uint8)
_I32 = C.POINTER(C.c_int32)
EXPORTS = {
    "piv_params_read": (C.c_int, [C.c_char_p, C.POINTER(PivParams), C.POINTER(PivPaths)]),
    "piv_geometry_compute": (C.c_int, [C.POINTER(PivParams), C.POINTER(PivGeometry)]),
    "piv_status_string": (C.c_char_p, [C.c_int]),
    "piv_create": (C.c_int, [C.POINTER(PivParams), C.POINTER(_P)]),
    "piv_destroy": (C.c_int, [_P]),
    "piv_last_error": (C.c_char_p, [_P]),
    "piv_get_geometry": (C.c_int, [_P, C.POINTER(PivGeometry)]),
    "piv_get_params": (C.c_int, [_P, C.POINTER(PivParams)]),
    "piv_host_images": (C.c_int, [_P, C.POINTER(_U8), C.POINTER(_U8)]),
    "piv_set_images": (C.c_int, [_P, _U8, _U8, C.c_size_t]),
    "piv_set_device_images": (C.c_int, [_P, _P, _P]),
    "piv_prep": (C.c_int, [_P]),
    "piv_pass_grid1": (C.c_int, [_P, C.c_int]),
    "piv_validate_grid1": (C.c_int, [_P, C.c_int, C.c_int, C.c_float, C.c_float, C.c_int]),
    "piv_upsample": (C.c_int, [_P]),
    "piv_pass_grid2": (C.c_int, [_P]),
    "piv_validate_grid2": (C.c_int, [_P, C.c_int, C.c_int, C.c_float, C.c_float, C.c_int, C.c_int]),
    "piv_run_pair": (C.c_int, [_P]),
    "piv_synchronize": (C.c_int, [_P]),
    "piv_get_field": (C.c_int, [_P, C.c_int, _F, _F, _F, _F, _U8]),
    "piv_write_tecplot": (C.c_int, [_P, C.c_char_p, C.c_int]),
    "piv_tecplot_write_arrays": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _F, _F]),
    "piv_output_name": (C.c_int, [C.POINTER(PivParams), C.c_char_p, C.c_int, C.c_int, C.c_char_p, C.c_size_t]),
    "piv_npy_write_f32": (C.c_int, [C.c_char_p, _F, C.c_int, C.POINTER(C.c_int)]),
    "piv_tiff_info": (C.c_int, [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "piv_tiff_read8": (C.c_int, [C.c_char_p, _U8, C.c_int, C.c_int]),
    "piv_tiff_write8": (C.c_int, [C.c_char_p, _U8, C.c_int, C.c_int]),
    "piv_get_peaks": (C.c_int, [_P, C.c_int, _I32, _I32, _F]),
    "piv_set_field": (C.c_int, [_P, C.c_int, _F, _F, _U8]),
    "piv_set_candidates": (C.c_int, [_P, C.c_int, _F, _F, _U8]),
    "piv_get_frames": (C.c_int, [_P, _U8, _U8]),
    "piv_get_deformed": (C.c_int, [_P, C.c_int, _F]),
    "piv_debug_cc_planes": (C.c_int, [_P, C.c_int, C.c_int, C.c_int, _F]),
    "piv_stage_times": (C.c_int, [_P, _F]),
    "piv_get_stream": (C.c_int, [_P, C.POINTER(_P)]),
    "piv_xcorr_config": (C.c_int, [_P, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), _F]),
    "piv_kernel_launches_per_pair": (C.c_int, [_P, C.POINTER(C.c_int)]),
    "piv_time_stage": (C.c_int, [_P, C.c_int, C.c_int, _F]),
    "piv_probe_fp32_peak": (C.c_int, [_F]),
    "piv_queue_images": (C.c_int, [_P, _P, _P]),
    "piv_field_async": (C.c_int, [_P, C.c_int, C.POINTER(C.c_int)]),
    "piv_field_wait": (C.c_int, [_P, C.c_int, _F, _F, _F, _F, _U8]),
    "piv_host_alloc": (C.c_int, [C.c_size_t, C.POINTER(_P)]),
    "piv_host_free": (C.c_int, [_P]),
    "piv_set_xcorr_path": (C.c_int, [_P, C.c_int, C.c_int]),
    "piv_get_xcorr_path": (C.c_int, [_P, C.c_int, C.POINTER(C.c_int)]),
    "piv_tc_gemm_check": (C.c_int, [_F, _F, _F, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]),
    "piv_mhe_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_float, C.POINTER(_P)]),
    "piv_mhe_process": (C.c_int, [_P, _P, _P, _P]),
    "piv_mhe_destroy": (C.c_int, [_P]),
    "piv_mhe_process_noalloc": (C.c_int, [_P, _P, C.c_int, C.c_int, C.c_int, C.c_float, _P]),
    "piv_synth_pair": (C.c_int, [C.POINTER(PivSynthParams), _U8, _U8]),
    "piv_synth_field": (C.c_int, [C.POINTER(PivSynthParams), _F, _F, C.c_int, _F, _F]),
    "piv_synth_pair_device": (C.c_int, [C.POINTER(PivSynthParams), _P, _P, _P, _P]),
    "piv_batch_create": (C.c_int, [C.POINTER(PivParams), C.c_int, C.POINTER(_P)]),
    "piv_batch_destroy": (C.c_int, [_P]),
    "piv_batch_last_error": (C.c_char_p, [_P]),
    "piv_batch_engine": (C.c_int, [_P, C.c_int, C.POINTER(_P)]),
    "piv_batch_run": (C.c_int, [_P]),
    "piv_batch_synchronize": (C.c_int, [_P]),
    "piv_batch_stream": (C.c_int, [_P, C.POINTER(_P)]),
    "piv_batch_groups": (C.c_int, [_P, C.c_int] + [C.POINTER(C.c_int)] * 8),
    "piv_net_create": (C.c_int, [C.c_uint64, C.POINTER(_P)]),
    "piv_net_destroy": (C.c_int, [_P]),
    "piv_net_last_error": (C.c_char_p, [_P]),
    "piv_net_num_params": (C.c_int, [_P, C.POINTER(C.c_int64)]),
    "piv_net_layout": (C.c_int, [C.c_int] + [C.POINTER(C.c_int)] * 5),
    "piv_net_get_params": (C.c_int, [_P, _F, C.c_int64]),
    "piv_net_set_params": (C.c_int, [_P, _F, C.c_int64]),
    "piv_net_get_grads": (C.c_int, [_P, _F, C.c_int64]),
    "piv_net_save": (C.c_int, [_P, C.c_char_p]),
    "piv_net_load": (C.c_int, [_P, C.c_char_p]),
    "piv_net_forward": (C.c_int, [_P, _P, C.c_int, C.c_int, C.c_int, _P, _P]),
    "piv_net_loss_grad": (C.c_int, [_P, _P, _P, _P, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_float)]),
    "piv_net_adam_step": (C.c_int, [_P, C.c_float]),
    "piv_net_synchronize": (C.c_int, [_P]),
    "piv_net_features": (C.c_int, [_P, _P, _P]),
    "piv_run_pair_learned": (C.c_int, [_P, _P, C.c_float, C.c_float, C.POINTER(C.c_int), C.POINTER(C.c_float),
                                        C.POINTER(C.c_float)]),
}

_lib_handle = None


def lib():
    """Loads lib/libpiv_b200.so (built by `make -C piv_xcorr2d_v1.0_b200`)."""
    global _lib_handle
    if _lib_handle is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"CUDA engine library missing: {LIB_PATH} (build it with make -C {_HERE})")
        h = C.CDLL(str(LIB_PATH))
        for name, (res, args) in EXPORTS.items():
            fn = getattr(h, name)
            fn.restype = res
            fn.argtypes = args
        _lib_handle = h
    return _lib_handle


class PivError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"[{status}] {msg}")
        self.status = status


def _addr(a, nbytes):
    """Address of a C-contiguous host buffer of at least nbytes (numpy array or a CPU
    torch tensor)."""
    if hasattr(a, "data_ptr"):
        assert a.is_contiguous() and a.numel() * a.element_size() >= nbytes and not a.is_cuda
        return a.data_ptr()
    a = np.asarray(a)
    assert a.flags.c_contiguous and a.nbytes >= nbytes
    return a.ctypes.data


def _ptr(a, ct):
    return a.ctypes.data_as(C.POINTER(ct)) if a is not None else None


def default_params(**kw) -> PivParams:
    """The reference's example parameter file (X/Parameter.dat) as defaults."""
    d = dict(device_id=0, if_mhe=0, mhe_ws=40, mhe_thresh=0.91, Nx=6600, Ny=4400,
             ws_x1=64, ws_y1=64, spacing_x1=32, spacing_y1=32, Npass1=2,
             ws_x2=32, ws_y2=32, spacing_x2=16, spacing_y2=16, Npass2=2, Nsec_cc=1,
             wx1_median=5, wy1_median=5, Npass1_median=2, minNneigh_p1=5, residual_threshold_p1=2.0,
             insert_threshold_p1=3.0, wx1_smooth=3, wy1_smooth=3, Npass1_smooth=1,
             wx2_median=5, wy2_median=5, Npass2_median=2, minNneigh_p2=5, residual_threshold_p2=2.0,
             insert_threshold_p2=3.0, wx2_smooth=3, wy2_smooth=3, Npass2_smooth=1,
             max_dispx_win_percent1=0.4, max_dispy_win_percent1=0.4, max_dispx_win_percent2=0.4,
             max_dispy_win_percent2=0.4, Npeak_save=4, dispx_lim1=-100.0, dispx_lim2=100.0,
             dispy_lim1=-100.0, dispy_lim2=100.0)
    for k in kw:
        if k not in d:
            raise KeyError(k)
    d.update(kw)
    p = PivParams()
    for k, v in d.items():
        setattr(p, k, v)
    return p


def read_params(path):
    """X/main.cpp:93-158: (PivParams, dict of the six path lines)."""
    p, q = PivParams(), PivPaths()
    rc = lib().piv_params_read(str(path).encode(), C.byref(p), C.byref(q))
    if rc != PIV_OK:
        raise PivError(rc, "Can't open parameter file!" if rc == PIV_ERR_IO else "Parameter missing in Parameter.dat!")
    paths = {n: getattr(q, n).decode() for n, _ in PivPaths._fields_}
    return p, paths


def geometry(p: PivParams) -> dict:
    g = PivGeometry()
    rc = lib().piv_geometry_compute(C.byref(p), C.byref(g))
    if rc != PIV_OK:
        raise PivError(rc, lib().piv_status_string(rc).decode())
    return g.to_dict()


def output_name(p: PivParams, folder: str, idx: int, kind: int) -> str:
    buf = C.create_string_buffer(4096)
    rc = lib().piv_output_name(C.byref(p), folder.encode(), idx, kind, buf, 4096)
    if rc != PIV_OK:
        raise PivError(rc, "name too long")
    return buf.value.decode()


def synth_params(Nx, Ny, ppp=0.05, sigma=0.6, i_min=120.0, i_max=255.0, background=10.0, noise_sigma=2.0,
                 field=PIV_FIELD_UNIFORM, a=0.0, b=0.0, c=0.0, seed=1) -> PivSynthParams:
    s = PivSynthParams()
    s.Nx, s.Ny, s.ppp, s.sigma, s.i_min, s.i_max = Nx, Ny, ppp, sigma, i_min, i_max
    s.background, s.noise_sigma, s.field, s.a, s.b, s.c, s.seed = background, noise_sigma, field, a, b, c, seed
    return s


def synth_pair(s: PivSynthParams):
    """Seeded synthetic frame pair (uint8 [Ny, Nx] each), host-side generator."""
    f1 = np.empty((s.Ny, s.Nx), np.uint8)
    f2 = np.empty((s.Ny, s.Nx), np.uint8)
    rc = lib().piv_synth_pair(C.byref(s), _ptr(f1, C.c_uint8), _ptr(f2, C.c_uint8))
    if rc != PIV_OK:
        raise PivError(rc, "synthetic pair generation failed")
    return f1, f2


def synth_field(s: PivSynthParams, x, y):
    x = np.ascontiguousarray(x, np.float32)
    y = np.ascontiguousarray(y, np.float32)
    u = np.empty_like(x)
    v = np.empty_like(x)
    rc = lib().piv_synth_field(C.byref(s), _ptr(x, C.c_float), _ptr(y, C.c_float), x.size, _ptr(u, C.c_float),
                               _ptr(v, C.c_float))
    if rc != PIV_OK:
        raise PivError(rc, "field evaluation failed")
    return u, v


def _dptr(x) -> int:
    """Device address of a torch tensor, or an int address as is."""
    return x if isinstance(x, int) else int(x.data_ptr())


def synth_pair_device(s: PivSynthParams, d_f1, d_f2, d_scratch, stream=None):
    """The same pair as synth_pair rendered on the GPU (asynchronous on `stream`): d_f1, d_f2
    hold Nx*Ny bytes, d_scratch 2*Nx*Ny floats (torch tensors or device addresses)."""
    rc = lib().piv_synth_pair_device(C.byref(s), _dptr(d_f1), _dptr(d_f2), _dptr(d_scratch), stream)
    if rc != PIV_OK:
        raise PivError(rc, "device synthetic pair generation failed")


NET_IN_CHANNELS = 81
NET_LAYERS = 13


def net_layout():
    """[(cin, cout, stride, weight_offset, bias_offset)] of the predictor's 13 layers."""
    out = []
    for i in range(NET_LAYERS):
        v = [C.c_int() for _ in range(5)]
        rc = lib().piv_net_layout(i, *[C.byref(x) for x in v])
        if rc != PIV_OK:
            raise PivError(rc, "layout")
        out.append(tuple(x.value for x in v))
    return out


class Batch:
    """Pairs of uneven size and window shape run together (piv_batch_*): one persistent
    correlation launch per pass and window shape, the pass loop as one CUDA graph.
    `engines[i]` is pair i's engine (set its frames, read its fields)."""

    def __init__(self, params_list):
        n = len(params_list)
        arr = (PivParams * n)(*params_list)
        h = C.c_void_p()
        rc = lib().piv_batch_create(arr, n, C.byref(h))
        if rc != PIV_OK:
            raise PivError(rc, "piv_batch_create failed")
        self.h = h
        self.engines = []
        for i in range(n):
            e = C.c_void_p()
            self._ck(lib().piv_batch_engine(self.h, i, C.byref(e)))
            self.engines.append(Engine._borrowed(e, params_list[i]))

    def _ck(self, rc):
        if rc != PIV_OK:
            raise PivError(rc, lib().piv_batch_last_error(self.h).decode())
        return rc

    def run(self):
        self._ck(lib().piv_batch_run(self.h))

    def synchronize(self):
        self._ck(lib().piv_batch_synchronize(self.h))

    def stream(self) -> int:
        s = C.c_void_p()
        self._ck(lib().piv_batch_stream(self.h, C.byref(s)))
        return s.value or 0

    def groups(self):
        n = C.c_int()
        self._ck(lib().piv_batch_groups(self.h, 0, *([None] * 7), C.byref(n)))
        cols = [(C.c_int * max(n.value, 1))() for _ in range(7)]
        self._ck(lib().piv_batch_groups(self.h, n.value, *cols, C.byref(n)))
        keys = ("wsx", "wsy", "grid", "deformed", "pairs", "variant", "windows_per_cta")
        return [{k: cols[j][i] for j, k in enumerate(keys)} for i in range(n.value)]

    def close(self):
        if getattr(self, "h", None):
            for e in self.engines:
                e.h = None
            lib().piv_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class PredictorNet:
    """The learned grid-1 predictor (piv_net_*): a 4-level U-Net on the cost volume of the
    4x-downsampled frames, BF16 weights, hand-written training and inference kernels."""

    def __init__(self, seed=1, weights=None):
        h = C.c_void_p()
        rc = lib().piv_net_create(seed, C.byref(h))
        if rc != PIV_OK:
            raise PivError(rc, "piv_net_create failed")
        self.h = h
        n = C.c_int64()
        self._ck(lib().piv_net_num_params(self.h, C.byref(n)))
        self.n_params = n.value
        if weights is not None:
            self.load(weights)

    def _ck(self, rc):
        if rc != PIV_OK:
            raise PivError(rc, lib().piv_net_last_error(self.h).decode())
        return rc

    def close(self):
        if getattr(self, "h", None):
            lib().piv_net_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def params(self) -> np.ndarray:
        out = np.empty(self.n_params, np.float32)
        self._ck(lib().piv_net_get_params(self.h, _ptr(out, C.c_float), self.n_params))
        return out

    def set_params(self, v):
        v = np.ascontiguousarray(v, np.float32)
        self._ck(lib().piv_net_set_params(self.h, _ptr(v, C.c_float), v.size))

    def grads(self) -> np.ndarray:
        out = np.empty(self.n_params, np.float32)
        self._ck(lib().piv_net_get_grads(self.h, _ptr(out, C.c_float), self.n_params))
        return out

    def save(self, path):
        self._ck(lib().piv_net_save(self.h, str(path).encode()))

    def load(self, path):
        self._ck(lib().piv_net_load(self.h, str(path).encode()))

    def forward(self, d_in, N, H, W, d_out, stream=None):
        """[N][81][H][W] -> [N][2][H][W] (downsampled px), device buffers."""
        self._ck(lib().piv_net_forward(self.h, _dptr(d_in), N, H, W, _dptr(d_out), stream))

    def loss_grad(self, d_in, d_label, d_mask, N, H, W) -> float:
        loss = C.c_float()
        self._ck(lib().piv_net_loss_grad(self.h, _dptr(d_in), _dptr(d_label), _dptr(d_mask), N, H, W,
                                         C.byref(loss)))
        return loss.value

    def adam_step(self, lr):
        self._ck(lib().piv_net_adam_step(self.h, lr))

    def synchronize(self):
        self._ck(lib().piv_net_synchronize(self.h))


class Engine:
    """One image-pair pipeline on one GPU (piv_create .. piv_destroy)."""

    def __init__(self, params: PivParams):
        self.p = params
        h = C.c_void_p()
        rc = lib().piv_create(C.byref(params), C.byref(h))
        if rc != PIV_OK:
            raise PivError(rc, f"Initialization of xcorr2d_multi class failed! ({lib().piv_status_string(rc).decode()})")
        self.h = h
        g = PivGeometry()
        lib().piv_get_geometry(self.h, C.byref(g))
        self.geom = g.to_dict()

    @classmethod
    def _borrowed(cls, handle, params: PivParams):
        """An engine owned by someone else (a batch): no piv_destroy on close."""
        e = cls.__new__(cls)
        e.p = params
        e.h = handle
        e._owner = False
        g = PivGeometry()
        lib().piv_get_geometry(e.h, C.byref(g))
        e.geom = g.to_dict()
        return e

    # -- lifetime --
    def close(self):
        if getattr(self, "h", None):
            if getattr(self, "_owner", True):
                lib().piv_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _ck(self, rc):
        if rc != PIV_OK:
            raise PivError(rc, lib().piv_last_error(self.h).decode())
        return rc

    # -- frames --
    def host_images(self):
        """numpy views [Ny, Nx] of the engine's pinned frame buffers (h_img1_org, h_img2_org)."""
        a, b = C.POINTER(C.c_uint8)(), C.POINTER(C.c_uint8)()
        self._ck(lib().piv_host_images(self.h, C.byref(a), C.byref(b)))
        n = (self.p.Ny, self.p.Nx)
        return np.ctypeslib.as_array(a, shape=n), np.ctypeslib.as_array(b, shape=n)

    def set_images(self, f1, f2):
        f1 = np.ascontiguousarray(f1, np.uint8)
        f2 = np.ascontiguousarray(f2, np.uint8)
        assert f1.shape == (self.p.Ny, self.p.Nx) and f2.shape == f1.shape
        self._ck(lib().piv_set_images(self.h, _ptr(f1, C.c_uint8), _ptr(f2, C.c_uint8), 0))

    def set_device_images(self, d1: int, d2: int):
        self._ck(lib().piv_set_device_images(self.h, C.c_void_p(d1), C.c_void_p(d2)))

    def queue_images(self, f1, f2):
        """Queues the upload of the next pair (host arrays or host addresses; pinned memory
        overlaps the copy with the pair in flight).  The arrays must stay alive and
        unchanged until that pair has been run and its results read."""
        a1 = f1 if isinstance(f1, int) else _addr(f1, self.p.Nx * self.p.Ny)
        a2 = f2 if isinstance(f2, int) else _addr(f2, self.p.Nx * self.p.Ny)
        self._ck(lib().piv_queue_images(self.h, C.c_void_p(a1), C.c_void_p(a2)))

    # -- stages --
    def prep(self):
        self._ck(lib().piv_prep(self.h))

    def pass_grid1(self, j):
        self._ck(lib().piv_pass_grid1(self.h, j))

    def validate_grid1(self, Npass_median=None, minN=None, rthr=None, ithr=None, Npass_smooth=None):
        p = self.p
        self._ck(lib().piv_validate_grid1(
            self.h, p.Npass1_median if Npass_median is None else Npass_median,
            p.minNneigh_p1 if minN is None else minN, p.residual_threshold_p1 if rthr is None else rthr,
            p.insert_threshold_p1 if ithr is None else ithr, p.Npass1_smooth if Npass_smooth is None else Npass_smooth))

    def upsample(self):
        self._ck(lib().piv_upsample(self.h))

    def pass_grid2(self):
        self._ck(lib().piv_pass_grid2(self.h))

    def validate_grid2(self, Npass_median=None, minN=None, rthr=None, ithr=None, Npass_smooth=None, iffill=1):
        p = self.p
        self._ck(lib().piv_validate_grid2(
            self.h, p.Npass2_median if Npass_median is None else Npass_median,
            p.minNneigh_p2 if minN is None else minN, p.residual_threshold_p2 if rthr is None else rthr,
            p.insert_threshold_p2 if ithr is None else ithr,
            p.Npass2_smooth if Npass_smooth is None else Npass_smooth, iffill))

    def run_pair(self):
        self._ck(lib().piv_run_pair(self.h))

    def synchronize(self):
        self._ck(lib().piv_synchronize(self.h))

    # -- readback --
    def _nt(self, grid):
        return self.geom["Nt_vec"][grid]

    def field(self, selection):
        """(x, y, dx, dy, valid); raw selections (0, 2) give [Nt, Npeak_save] candidate arrays."""
        g = 0 if selection < 2 else 1
        nt = self._nt(g)
        raw = selection in (0, 2)
        n = nt * self.p.Npeak_save if raw else nt
        x = np.empty(nt, np.float32)
        y = np.empty(nt, np.float32)
        dx = np.empty(n, np.float32)
        dy = np.empty(n, np.float32)
        v = np.empty(n, np.uint8)
        self._ck(lib().piv_get_field(self.h, selection, _ptr(x, C.c_float), _ptr(y, C.c_float),
                                     _ptr(dx, C.c_float), _ptr(dy, C.c_float), _ptr(v, C.c_uint8)))
        if raw:
            dx = dx.reshape(nt, -1)
            dy = dy.reshape(nt, -1)
            v = v.reshape(nt, -1)
        return x, y, dx, dy, v

    def field_async(self, selection):
        """Queues the readback of a selection behind the queued work; returns a ticket."""
        t = C.c_int(0)
        self._ck(lib().piv_field_async(self.h, selection, C.byref(t)))
        return (t.value, selection)

    def field_wait(self, ticket):
        """(x, y, dx, dy, valid) of a piv_field_async ticket, as field() returns them."""
        t, selection = ticket
        g = 0 if selection < 2 else 1
        nt = self._nt(g)
        raw = selection in (0, 2)
        n = nt * self.p.Npeak_save if raw else nt
        x = np.empty(nt, np.float32)
        y = np.empty(nt, np.float32)
        dx = np.empty(n, np.float32)
        dy = np.empty(n, np.float32)
        v = np.empty(n, np.uint8)
        self._ck(lib().piv_field_wait(self.h, t, _ptr(x, C.c_float), _ptr(y, C.c_float), _ptr(dx, C.c_float),
                                      _ptr(dy, C.c_float), _ptr(v, C.c_uint8)))
        if raw:
            dx, dy, v = dx.reshape(nt, -1), dy.reshape(nt, -1), v.reshape(nt, -1)
        return x, y, dx, dy, v

    def peaks(self, grid):
        nt, nps = self._nt(grid), self.p.Npeak_save
        cnt = np.empty(nt, np.int32)
        idx = np.empty((nt, nps), np.int32)
        val = np.empty((nt, nps), np.float32)
        self._ck(lib().piv_get_peaks(self.h, grid, _ptr(cnt, C.c_int32), _ptr(idx, C.c_int32),
                                     _ptr(val, C.c_float)))
        return cnt, idx, val

    def set_field(self, grid, dx, dy, valid):
        dx = np.ascontiguousarray(dx, np.float32)
        dy = np.ascontiguousarray(dy, np.float32)
        valid = np.ascontiguousarray(valid, np.uint8)
        self._ck(lib().piv_set_field(self.h, grid, _ptr(dx, C.c_float), _ptr(dy, C.c_float),
                                     _ptr(valid, C.c_uint8)))

    def set_candidates(self, grid, dx, dy, valid):
        dx = np.ascontiguousarray(dx, np.float32)
        dy = np.ascontiguousarray(dy, np.float32)
        valid = np.ascontiguousarray(valid, np.uint8)
        self._ck(lib().piv_set_candidates(self.h, grid, _ptr(dx, C.c_float), _ptr(dy, C.c_float),
                                          _ptr(valid, C.c_uint8)))

    def frames(self):
        f1 = np.empty((self.p.Ny, self.p.Nx), np.uint8)
        f2 = np.empty_like(f1)
        self._ck(lib().piv_get_frames(self.h, _ptr(f1, C.c_uint8), _ptr(f2, C.c_uint8)))
        return f1, f2

    def deformed(self, grid):
        out = np.empty((self.geom["Ny_aug"][grid], self.geom["Nx_aug"][grid]), np.float32)
        self._ck(lib().piv_get_deformed(self.h, grid, _ptr(out, C.c_float)))
        return out

    def cc_planes(self, grid, first, n):
        wsx = self.p.ws_x1 if grid == 0 else self.p.ws_x2
        wsy = self.p.ws_y1 if grid == 0 else self.p.ws_y2
        out = np.empty((n, wsy, wsx), np.float32)
        self._ck(lib().piv_debug_cc_planes(self.h, grid, first, n, _ptr(out, C.c_float)))
        return out

    def write_tecplot(self, path, selection):
        self._ck(lib().piv_write_tecplot(self.h, str(path).encode(), selection))

    def stage_times(self):
        out = np.zeros(5, np.float32)
        self._ck(lib().piv_stage_times(self.h, _ptr(out, C.c_float)))
        return out

    # -- learned form --
    def features(self, net: PredictorNet, d_out):
        """The predictor input of the prepared frames, [81][Ny1_vec][Nx1_vec] into d_out."""
        self._ck(lib().piv_net_features(self.h, net.h, _dptr(d_out)))

    def run_pair_learned(self, net: PredictorNet, max_reject_frac=0.05, max_rms_px=0.5) -> dict:
        """One pair by the learned form, judged; falls back to the plain pair on failure."""
        fb, rej, rms = C.c_int(), C.c_float(), C.c_float()
        self._ck(lib().piv_run_pair_learned(self.h, net.h, max_reject_frac, max_rms_px, C.byref(fb), C.byref(rej),
                                            C.byref(rms)))
        return {"fell_back": bool(fb.value), "reject_frac": rej.value, "rms_px": rms.value}

    def stream(self) -> int:
        s = C.c_void_p()
        self._ck(lib().piv_get_stream(self.h, C.byref(s)))
        return s.value or 0

    def xcorr_config(self, grid):
        """(windows per CTA, threads per CTA, tuned ms per launch) of the grid's fused kernel."""
        b, nt, ms = C.c_int(0), C.c_int(0), C.c_float(0)
        self._ck(lib().piv_xcorr_config(self.h, grid, C.byref(b), C.byref(nt), C.byref(ms)))
        return b.value, nt.value, ms.value

    def launches_per_pair(self):
        n = C.c_int(0)
        self._ck(lib().piv_kernel_launches_per_pair(self.h, C.byref(n)))
        return n.value

    def time_stage(self, which, reps=5):
        ms = C.c_float(0)
        self._ck(lib().piv_time_stage(self.h, which, reps, C.byref(ms)))
        return ms.value

    def set_xcorr_path(self, grid, path):
        self._ck(lib().piv_set_xcorr_path(self.h, grid, path))

    def xcorr_path(self, grid):
        v = C.c_int(0)
        self._ck(lib().piv_get_xcorr_path(self.h, grid, C.byref(v)))
        return v.value


def fp32_peak_tflops():
    t = C.c_float(0)
    rc = lib().piv_probe_fp32_peak(C.byref(t))
    if rc != PIV_OK:
        raise PivError(rc, "FP32 peak probe failed")
    return t.value


def tc_gemm_check(A, B, a_mn=False, b_mn=False, nprod=3):
    """A (128 x K) times B (N x K) transposed on the tcgen05 tensor-core path."""
    A = np.ascontiguousarray(A, np.float32)
    B = np.ascontiguousarray(B, np.float32)
    assert A.shape[0] == 128 and A.shape[1] == B.shape[1]
    D = np.empty((128, B.shape[0]), np.float32)
    rc = lib().piv_tc_gemm_check(_ptr(A, C.c_float), _ptr(B, C.c_float), _ptr(D, C.c_float), B.shape[0],
                                 A.shape[1], int(a_mn), int(b_mn), nprod)
    if rc != PIV_OK:
        raise PivError(rc, "tensor-core check failed")
    return D


class xcorr2d_multi:
    """Method-for-method mirror of the reference class (X/xcorr2d_multi_grid.cuh:12-208)."""

    def __init__(self):
        self._e = None

    def init(self, Nx, Ny, Nsec_cc, ws_x1, ws_y1, spacing_x1, spacing_y1, Npass1, ws_x2, ws_y2, spacing_x2,
             spacing_y2, Npass2, wx1_median, wy1_median, wx2_median, wy2_median, wx1_smooth, wy1_smooth,
             wx2_smooth, wy2_smooth, Npeak_save, max_dispx_percent1, max_dispy_percent1, max_dispx_percent2,
             max_dispy_percent2, dispx_lim1, dispx_lim2, dispy_lim1, dispy_lim2, device_id=0) -> bool:
        p = default_params(
            device_id=device_id, if_mhe=0, Nx=Nx, Ny=Ny, Nsec_cc=Nsec_cc, ws_x1=ws_x1, ws_y1=ws_y1,
            spacing_x1=spacing_x1, spacing_y1=spacing_y1, Npass1=Npass1, ws_x2=ws_x2, ws_y2=ws_y2,
            spacing_x2=spacing_x2, spacing_y2=spacing_y2, Npass2=Npass2, wx1_median=wx1_median,
            wy1_median=wy1_median, wx2_median=wx2_median, wy2_median=wy2_median, wx1_smooth=wx1_smooth,
            wy1_smooth=wy1_smooth, wx2_smooth=wx2_smooth, wy2_smooth=wy2_smooth, Npeak_save=Npeak_save,
            max_dispx_win_percent1=max_dispx_percent1, max_dispy_win_percent1=max_dispy_percent1,
            max_dispx_win_percent2=max_dispx_percent2, max_dispy_win_percent2=max_dispy_percent2,
            dispx_lim1=dispx_lim1, dispx_lim2=dispx_lim2, dispy_lim1=dispy_lim1, dispy_lim2=dispy_lim2)
        try:
            self._e = Engine(p)
        except PivError as err:
            print(err)
            return False
        g = self._e.geom
        self.Nx, self.Ny, self.Nt = Nx, Ny, Nx * Ny
        self.Npass1, self.Npass2, self.Npeak_save = Npass1, Npass2, Npeak_save
        self.Nx1_vec, self.Ny1_vec, self.Nt1_vec = g["Nx_vec"][0], g["Ny_vec"][0], g["Nt_vec"][0]
        self.Nx2_vec, self.Ny2_vec, self.Nt2_vec = g["Nx_vec"][1], g["Ny_vec"][1], g["Nt_vec"][1]
        self.h_img1_org, self.h_img2_org = self._e.host_images()
        return True

    def _call(self, f, *a) -> bool:
        try:
            f(*a)
            return True
        except PivError as err:
            print(err)
            return False

    def prep_img_data(self):
        self._e.prep()

    def Calc_cc_map_p1(self, idx_pass) -> bool:
        return self._call(self._e.pass_grid1, idx_pass)

    def Calc_cc_map_p2(self) -> bool:
        return self._call(self._e.pass_grid2)

    def MedianFilter_Smoothing_p1(self, Npass1_median, minNneigh_p1, residual_threshold_p1, insert_threshold_p1,
                                  Npass1_smooth) -> bool:
        return self._call(self._e.validate_grid1, Npass1_median, minNneigh_p1, residual_threshold_p1,
                          insert_threshold_p1, Npass1_smooth)

    def MedianFilter_Smoothing_p2(self, Npass2_median, minNneigh_p2, residual_threshold_p2, insert_threshold_p2,
                                  Npass2_smooth, iffill_p2) -> bool:
        return self._call(self._e.validate_grid2, Npass2_median, minNneigh_p2, residual_threshold_p2,
                          insert_threshold_p2, Npass2_smooth, iffill_p2)

    def extend_filtered_vecfield_p1(self):
        """No-op: the engine reads the edge-replicated field through clamped indices."""

    def extend_filtered_vecfield_p2(self):
        """No-op: see extend_filtered_vecfield_p1."""

    def Upsampling_vector_field(self) -> bool:
        return self._call(self._e.upsample)

    def write_vec_data_general(self, dir_vec, selection) -> bool:
        return self._call(self._e.write_tecplot, dir_vec, selection)

    def freemem(self):
        if self._e is not None:
            self._e.close()
            self._e = None


class mhe_gpu:
    """Mirror of the reference's MHE class (X/MHE7_4_gpu.h:7-40) on device tensors."""

    def __init__(self):
        self._h = None

    def init(self, Nx_org, Ny_org, m_mhe_ws, m_mhe_thresh) -> bool:
        import torch

        h = C.c_void_p()
        rc = lib().piv_mhe_create(Nx_org, Ny_org, m_mhe_ws, m_mhe_thresh, C.byref(h))
        if rc != PIV_OK:
            print("cudaMalloc ERROR!" if rc == PIV_ERR_ALLOC else "invalid MHE parameters")
            return False
        self._h = h
        self.Nx, self.Ny = Nx_org, Ny_org
        self.d_enhanced = torch.zeros((Ny_org, Nx_org), dtype=torch.uint8, device="cuda")
        return True

    def processsing(self, d_img_org) -> bool:
        """d_img_org: a CUDA uint8 tensor [Ny, Nx]; result in self.d_enhanced."""
        import torch

        assert d_img_org.is_cuda and d_img_org.dtype == torch.uint8 and d_img_org.is_contiguous()
        s = torch.cuda.current_stream().cuda_stream
        rc = lib().piv_mhe_process(self._h, C.c_void_p(d_img_org.data_ptr()),
                                   C.c_void_p(self.d_enhanced.data_ptr()), C.c_void_p(s))
        return rc == PIV_OK

    def freemem(self):
        if self._h is not None:
            lib().piv_mhe_destroy(self._h)
            self._h = None
