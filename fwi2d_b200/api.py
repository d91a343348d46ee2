"""Python binding of libfwi2d.so (include/fwi2d.h) and a mirror of the
reference's classes.

``Context`` is a thin ctypes wrapper over the C ABI.  ``Modeling``,
``Migration`` and ``Inversion`` mirror the public methods of the reference's
classes (src/modeling/modeling.cuh:76-86, src/migration/migration.cuh:32-37,
src/inversion/inversion.cuh:69-82) over that ABI so that a workflow written
against the reference reads the same here.

The CUDA library is the only implementation: importing this module without a
built ``libfwi2d.so`` raises, and every call that needs a GPU fails with the
library's CUDA error instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libfwi2d.so"

FWI_OK = 0
ERRORS = {
    -1: "FWI_ERR_PARAM", -2: "FWI_ERR_IO", -3: "FWI_ERR_CUDA", -4: "FWI_ERR_CFL", -5: "FWI_ERR_NAN",
    -6: "FWI_ERR_TIMEOUT", -7: "FWI_ERR_STATE", -8: "FWI_ERR_ARG", -9: "FWI_ERR_NOMEM",
}
MODE_MODELING, MODE_MIGRATION, MODE_INVERSION = 0, 1, 2

# Every function declared in include/fwi2d.h, with its ctypes signature.
_P = C.c_void_p
_F = C.POINTER(C.c_float)
_I = C.POINTER(C.c_int)
_D = C.POINTER(C.c_double)


class Dims(C.Structure):
    _fields_ = [("nx", C.c_int), ("nz", C.c_int), ("nt", C.c_int), ("nsrc", C.c_int), ("nrec", C.c_int),
                ("nb", C.c_int), ("nxx", C.c_int), ("nzz", C.c_int), ("ldz", C.c_int), ("tlag", C.c_int),
                ("abc_nb", C.c_int), ("rbc_nb", C.c_int), ("dh", C.c_float), ("dt", C.c_float),
                ("fmax", C.c_float), ("vmin", C.c_float), ("vmax", C.c_float)]


SIGNATURES = {
    "fwi_ctx_create": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(_P)]),
    "fwi_ctx_destroy": (None, [_P]),
    "fwi_last_error": (C.c_char_p, [_P]),
    "fwi_get_dims": (C.c_int, [_P, C.POINTER(Dims)]),
    "fwi_get_stream": (C.c_int, [_P, C.POINTER(_P)]),
    "fwi_get_param": (C.c_int, [_P, C.c_char_p, C.c_char_p, C.c_size_t]),
    "fwi_set_seed": (C.c_int, [_P, C.c_uint64]),
    "fwi_set_model": (C.c_int, [_P, _F]),
    "fwi_get_model": (C.c_int, [_P, _F]),
    "fwi_get_wavelet": (C.c_int, [_P, _F]),
    "fwi_get_indices": (C.c_int, [_P, C.c_int, _I, _I, _I]),
    "fwi_get_window": (C.c_int, [_P, C.c_int, _I, _I]),
    "fwi_set_direction": (C.c_int, [_P, _F]),
    "fwi_update_model_bounded": (C.c_int, [_P, C.c_float, C.c_float, C.c_float, _F]),
    "fwi_set_direction_dev": (C.c_int, [_P, C.c_void_p]),
    # fwi2d_nn.h (device pointers as integers)
    "fwi_nn_conv3x3": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int,
                                 C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    "fwi_nn_conv3x3_mma": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int,
                                     C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    "fwi_nn_check": (C.c_int, []),
    "fwi_nn_conv3x3_wgrad_mma": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                           C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "fwi_nn_wgrad_partial_floats": (C.c_size_t, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]),
    "fwi_nn_conv3x3_wgrad": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                       C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "fwi_nn_weight_prep": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    "fwi_nn_pool2": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p]),
    "fwi_nn_pool2_bwd": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p]),
    "fwi_nn_upcat": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
                               C.c_void_p, C.c_void_p]),
    "fwi_nn_upcat_bwd": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                   C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p]),
    "fwi_nn_relu_bwd": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p]),
    "fwi_nn_mse": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_longlong, C.c_float, C.c_void_p,
                             C.c_void_p, C.c_void_p, C.c_void_p]),
    "fwi_nn_adam": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_float, C.c_float,
                              C.c_float, C.c_float, C.c_int, C.c_void_p]),
    "fwi_nn_pack_inputs": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_float,
                                     C.c_void_p, C.c_void_p, C.c_void_p]),
    "fwi_nn_unpack": (C.c_int, [C.c_void_p, C.c_int, C.c_longlong, C.c_void_p, C.c_void_p]),
    "fwi_mute_direct": (C.c_int, [_P, _F, C.c_float, C.c_float, C.c_float]),
    "fwi_mute_direct_dev": (C.c_int, [_P, C.c_void_p, C.c_float, C.c_float, C.c_float]),
    "fwi_smooth_model": (C.c_int, [_P, _F, C.c_float, C.c_float, _F]),
    "fwi_set_shot_range": (C.c_int, [_P, C.c_int, C.c_int]),
    "fwi_gradient_accumulate": (C.c_int, [_P, C.c_int, C.POINTER(C.c_double)]),
    "fwi_gradient_finish": (C.c_int, [_P]),
    "fwi_accumulators": (C.c_int, [_P, C.POINTER(_F), C.POINTER(_F)]),
    "fwi_trial_steps": (C.c_int, [_P, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "fwi_parabola_step": (C.c_int, [_P, C.c_float, C.c_float, C.c_float, C.POINTER(C.c_float)]),
    "fwi_util_window": (C.c_int, [C.c_float, C.c_float, C.c_int, C.c_float, _I, _I]),
    "fwi_model_shot": (C.c_int, [_P, C.c_int, _F]),
    "fwi_model_survey": (C.c_int, [_P, _F]),
    "fwi_model_survey_dev": (C.c_int, [_P, _P]),
    "fwi_rtm_reset": (C.c_int, [_P]),
    "fwi_rtm_shot": (C.c_int, [_P, C.c_int, _F]),
    "fwi_rtm_survey": (C.c_int, [_P, _F]),
    "fwi_rtm_survey_dev": (C.c_int, [_P, _P]),
    "fwi_rtm_image": (C.c_int, [_P, _F]),
    "fwi_rtm_raw": (C.c_int, [_P, _F, _F]),
    "fwi_set_observed": (C.c_int, [_P, _F]),
    "fwi_set_observed_dev": (C.c_int, [_P, _P]),
    "fwi_compute_gradient": (C.c_int, [_P, C.c_int, _D]),
    "fwi_get_gradient": (C.c_int, [_P, _F]),
    "fwi_get_gradient_raw": (C.c_int, [_P, _F, _F]),
    "fwi_linesearch_trial": (C.c_int, [_P, C.c_float, _D]),
    "fwi_optimization": (C.c_int, [_P, C.c_float, _F]),
    "fwi_update_model": (C.c_int, [_P, C.c_float, _F]),
    "fwi_random_boundary": (C.c_int, [_P, C.c_int, _F]),
    "fwi_launch_count": (C.c_int, [_P, C.POINTER(C.c_longlong), C.c_int]),
    "fwi_util_parameter": (C.c_int, [C.c_char_p, C.c_char_p, C.c_char_p, C.c_size_t]),
    "fwi_util_wavelet": (C.c_int, [C.c_int, C.c_float, C.c_float, _F, _I]),
    "fwi_util_b1d": (C.c_int, [C.c_int, C.c_float, _F]),
    "fwi_util_grid_index": (C.c_int, [C.c_int, _F, C.c_float, C.c_int, _I]),
    "fwi_util_bumps": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, C.c_uint64,
                                 C.c_uint32, _F, C.c_int, _I]),
    "fwi_util_normal": (C.c_int, [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint64, _F]),
    "fwi_residual_noalloc": (C.c_int, [_P, _P, _P, C.c_size_t, _P, _P]),
    "fwi_describe": (C.c_int, [_P, C.c_char_p, C.c_size_t]),
    "fwi_fwd_timing": (C.c_int, [_P, C.c_int]),
    "fwi_fwd_timing_read": (C.c_int, [_P, C.POINTER(C.c_double), C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
    "fwi_bwd_timing_read": (C.c_int, [_P, C.POINTER(C.c_double), C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
}


class FwiError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


def load_library(path: Path | str = LIB_PATH) -> C.CDLL:
    path = Path(path)
    if not path.exists():
        raise ImportError(f"{path} is not built; run `python -m fwi2d_b200.build`")
    lib = C.CDLL(str(path))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_lib: C.CDLL | None = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        _lib = load_library()
    return _lib


def _fptr(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(_F)


class Context:
    """One fwi_ctx (one parameters file, one CUDA stream)."""

    def __init__(self, parameters: str | os.PathLike, mode: int):
        self._lib = lib()
        h = _P()
        rc = self._lib.fwi_ctx_create(str(parameters).encode(), mode, C.byref(h))
        if rc != FWI_OK:
            raise FwiError(rc, self._lib.fwi_last_error(None).decode())
        self._h = h
        d = Dims()
        self._lib.fwi_get_dims(self._h, C.byref(d))
        self.dims = d
        self.mode = mode

    # -- plumbing
    def _check(self, rc: int) -> None:
        if rc != FWI_OK:
            raise FwiError(rc, self._lib.fwi_last_error(self._h).decode())

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.fwi_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def stream(self) -> int:
        s = _P()
        self._check(self._lib.fwi_get_stream(self._h, C.byref(s)))
        return s.value or 0

    def param(self, key: str) -> str:
        buf = C.create_string_buffer(4096)
        self._check(self._lib.fwi_get_param(self._h, key.encode(), buf, 4096))
        return buf.value.decode()

    def describe(self) -> str:
        buf = C.create_string_buffer(4096)
        self._check(self._lib.fwi_describe(self._h, buf, 4096))
        return buf.value.decode()

    def fwd_timing(self, enable: bool = True) -> None:
        """Start (reset) or stop CUDA-event timing of the forward kernel."""
        self._check(self._lib.fwi_fwd_timing(self._h, int(enable)))

    def fwd_timing_read(self) -> tuple[float, int, int]:
        """(device ms, forward-kernel launches, grid-point updates) since fwd_timing(True)."""
        ms, n, u = C.c_double(), C.c_longlong(), C.c_longlong()
        self._check(self._lib.fwi_fwd_timing_read(self._h, C.byref(ms), C.byref(n), C.byref(u)))
        return ms.value, n.value, u.value

    def bwd_timing_read(self) -> tuple[float, int, int]:
        """(device ms, backward-kernel launches, grid-point updates) since fwd_timing(True)."""
        ms, n, u = C.c_double(), C.c_longlong(), C.c_longlong()
        self._check(self._lib.fwi_bwd_timing_read(self._h, C.byref(ms), C.byref(n), C.byref(u)))
        return ms.value, n.value, u.value

    def launches(self, reset: bool = False) -> int:
        c = C.c_longlong()
        self._check(self._lib.fwi_launch_count(self._h, C.byref(c), int(reset)))
        return c.value

    # -- model and set-up
    @property
    def shape(self) -> tuple[int, int]:
        return self.dims.nz, self.dims.nx

    def set_seed(self, seed: int) -> None:
        self._check(self._lib.fwi_set_seed(self._h, seed))

    def set_model(self, vp: np.ndarray) -> None:
        """vp: (nz, nx) float32 array (any order); stored z-fastest as the reference files."""
        v = np.asarray(vp, dtype=np.float32)
        flat = np.ascontiguousarray(v.reshape(self.shape).T).ravel()  # column-major, z fastest
        self._check(self._lib.fwi_set_model(self._h, _fptr(flat)))

    def get_model(self) -> np.ndarray:
        out = np.empty(self.dims.nx * self.dims.nz, np.float32)
        self._check(self._lib.fwi_get_model(self._h, _fptr(out)))
        return out.reshape(self.dims.nx, self.dims.nz).T

    def wavelet(self) -> np.ndarray:
        out = np.empty(self.dims.nt, np.float32)
        self._check(self._lib.fwi_get_wavelet(self._h, _fptr(out)))
        return out

    def indices(self, shot: int):
        d = self.dims
        sxz = np.zeros(2, np.int32)
        rx = np.zeros(d.nrec, np.int32)
        rz = np.zeros(d.nrec, np.int32)
        _i = lambda a: a.ctypes.data_as(_I)
        self._check(self._lib.fwi_get_indices(self._h, shot, _i(sxz), _i(rx), _i(rz)))
        return int(sxz[0]), int(sxz[1]), rx, rz

    def window(self, shot: int) -> tuple[int, int]:
        """Aperture window (c0, w) of a shot: model columns c0 .. c0+w-1."""
        c0, w = C.c_int(), C.c_int()
        self._check(self._lib.fwi_get_window(self._h, shot, C.byref(c0), C.byref(w)))
        return c0.value, w.value

    # -- modeling: seismograms returned as (nt, nrec) per shot (trace-major on disk)
    def _seis_view(self, flat: np.ndarray, nshots: int) -> np.ndarray:
        d = self.dims
        return flat.reshape(nshots, d.nrec, d.nt).transpose(0, 2, 1)

    def model_shot(self, shot: int) -> np.ndarray:
        d = self.dims
        out = np.empty(d.nrec * d.nt, np.float32)
        self._check(self._lib.fwi_model_shot(self._h, shot, _fptr(out)))
        return self._seis_view(out, 1)[0]

    def model_survey_raw(self, out: np.ndarray | None = None) -> np.ndarray:
        d = self.dims
        if out is None:
            out = np.empty(d.nsrc * d.nrec * d.nt, np.float32)
        self._check(self._lib.fwi_model_survey(self._h, _fptr(out)))
        return out

    def model_survey(self) -> np.ndarray:
        return self._seis_view(self.model_survey_raw(), self.dims.nsrc)

    def model_survey_dev(self, dev_ptr: int) -> None:
        self._check(self._lib.fwi_model_survey_dev(self._h, C.c_void_p(dev_ptr)))

    # -- migration
    def rtm_reset(self) -> None:
        self._check(self._lib.fwi_rtm_reset(self._h))

    @staticmethod
    def _traces(data: np.ndarray) -> np.ndarray:
        """(.., nt, nrec) -> trace-major float32 flat buffer."""
        a = np.asarray(data, dtype=np.float32)
        return np.ascontiguousarray(np.swapaxes(a, -1, -2)).ravel()

    def rtm_shot(self, shot: int, data: np.ndarray) -> None:
        self._check(self._lib.fwi_rtm_shot(self._h, shot, _fptr(self._traces(data))))

    def rtm_survey(self, data: np.ndarray) -> None:
        self._check(self._lib.fwi_rtm_survey(self._h, _fptr(self._traces(data))))

    def rtm_survey_raw(self, flat: np.ndarray) -> None:
        self._check(self._lib.fwi_rtm_survey(self._h, _fptr(flat)))

    def rtm_survey_dev(self, dev_ptr: int) -> None:
        self._check(self._lib.fwi_rtm_survey_dev(self._h, C.c_void_p(dev_ptr)))

    def _grid_out(self):
        return np.empty(self.dims.nx * self.dims.nz, np.float32)

    def _as2d(self, flat):
        return flat.reshape(self.dims.nx, self.dims.nz).T

    def rtm_image(self) -> np.ndarray:
        out = self._grid_out()
        self._check(self._lib.fwi_rtm_image(self._h, _fptr(out)))
        return self._as2d(out)

    def rtm_raw(self):
        a, b = self._grid_out(), self._grid_out()
        self._check(self._lib.fwi_rtm_raw(self._h, _fptr(a), _fptr(b)))
        return self._as2d(a), self._as2d(b)

    # -- inversion
    def set_observed(self, obs: np.ndarray) -> None:
        """obs: (nsrc, nt, nrec)."""
        self._check(self._lib.fwi_set_observed(self._h, _fptr(self._traces(obs))))

    def set_observed_raw(self, flat: np.ndarray) -> None:
        self._check(self._lib.fwi_set_observed(self._h, _fptr(flat)))

    def set_observed_dev(self, dev_ptr: int) -> None:
        self._check(self._lib.fwi_set_observed_dev(self._h, C.c_void_p(dev_ptr)))

    def compute_gradient(self, with_gradient: bool = True) -> float:
        s = C.c_double()
        self._check(self._lib.fwi_compute_gradient(self._h, int(with_gradient), C.byref(s)))
        return s.value

    def set_direction(self, d: np.ndarray) -> None:
        src = np.ascontiguousarray(np.asarray(d, dtype=np.float32).T).ravel()
        self._check(self._lib.fwi_set_direction(self._h, _fptr(src)))

    def set_direction_dev(self, dev_ptr: int) -> None:
        self._check(self._lib.fwi_set_direction_dev(self._h, C.c_void_p(dev_ptr)))

    def gradient(self) -> np.ndarray:
        out = self._grid_out()
        self._check(self._lib.fwi_get_gradient(self._h, _fptr(out)))
        return self._as2d(out)

    def gradient_raw(self):
        a, b = self._grid_out(), self._grid_out()
        self._check(self._lib.fwi_get_gradient_raw(self._h, _fptr(a), _fptr(b)))
        return self._as2d(a), self._as2d(b)

    def linesearch_trial(self, alpha: float) -> float:
        s = C.c_double()
        self._check(self._lib.fwi_linesearch_trial(self._h, alpha, C.byref(s)))
        return s.value

    def optimization(self, f0: float) -> float:
        s = C.c_float()
        self._check(self._lib.fwi_optimization(self._h, f0, C.byref(s)))
        return s.value

    # -- sharded inversion
    def set_shot_range(self, s0: int, ns: int) -> None:
        self._check(self._lib.fwi_set_shot_range(self._h, s0, ns))

    def gradient_accumulate(self, with_gradient: bool = True) -> float:
        s = C.c_double()
        self._check(self._lib.fwi_gradient_accumulate(self._h, int(with_gradient), C.byref(s)))
        return s.value

    def gradient_finish(self) -> None:
        self._check(self._lib.fwi_gradient_finish(self._h))

    def accumulators(self) -> tuple[int, int, int]:
        """(device address of the raw image / gradient, of the illumination, floats each)."""
        a, b = _F(), _F()
        self._check(self._lib.fwi_accumulators(self._h, C.byref(a), C.byref(b)))
        d = self.dims
        return C.cast(a, C.c_void_p).value, C.cast(b, C.c_void_p).value, d.nz * d.nx

    def trial_steps(self) -> tuple[float, float]:
        a1, a2 = C.c_float(), C.c_float()
        self._check(self._lib.fwi_trial_steps(self._h, C.byref(a1), C.byref(a2)))
        return a1.value, a2.value

    def parabola_step(self, f0: float, f1: float, f2: float) -> float:
        s = C.c_float()
        self._check(self._lib.fwi_parabola_step(self._h, f0, f1, f2, C.byref(s)))
        return s.value

    def update_model(self, step: float) -> np.ndarray:
        out = self._grid_out()
        self._check(self._lib.fwi_update_model(self._h, step, _fptr(out)))
        return self._as2d(out)

    def update_model_bounded(self, step: float, vmin: float, vmax: float) -> np.ndarray:
        out = self._grid_out()
        self._check(self._lib.fwi_update_model_bounded(self._h, step, vmin, vmax, _fptr(out)))
        return self._as2d(out)

    # -- data preparation (run/generate_input_data.py, run/generate_setup.py)
    def mute_direct(self, data: np.ndarray, velocity: float = 3600.0, delay: float = 0.18,
                    gstd: float = 30.0) -> np.ndarray:
        """Muted copy of (nsrc, nt, nrec) seismograms."""
        flat = self._traces(data).copy()
        self._check(self._lib.fwi_mute_direct(self._h, _fptr(flat), velocity, delay, gstd))
        d = self.dims
        return flat.reshape(d.nsrc, d.nrec, d.nt).transpose(0, 2, 1)

    def smooth_model(self, vp: np.ndarray, sigma: float = 3.0, depth_mask: float = 0.0) -> np.ndarray:
        src = np.ascontiguousarray(np.asarray(vp, dtype=np.float32).T).ravel()
        out = self._grid_out()
        self._check(self._lib.fwi_smooth_model(self._h, _fptr(src), sigma, depth_mask, _fptr(out)))
        return self._as2d(out)

    def random_boundary(self, shot: int) -> np.ndarray:
        """Random-boundary velocity of a shot on its RBC grid, (nzz, w + 2 nb)."""
        d = self.dims
        nb = d.rbc_nb
        _, w = self.window(shot)
        nzz, nxx = d.nz + 2 * nb, w + 2 * nb
        out = np.empty(nzz * nxx, np.float32)
        self._check(self._lib.fwi_random_boundary(self._h, shot, _fptr(out)))
        return out.reshape(nxx, nzz).T


# ---------------------------------------------------------------------------
# Host-side utilities (no GPU needed)

def _util_check(rc: int, what: str) -> None:
    if rc != FWI_OK:
        raise FwiError(rc, what)


def util_parameter(path: str | os.PathLike, key: str) -> str:
    buf = C.create_string_buffer(4096)
    _util_check(lib().fwi_util_parameter(str(path).encode(), key.encode(), buf, 4096), f"parameter {key}")
    return buf.value.decode()


def util_wavelet(nt: int, dt: float, fmax: float) -> tuple[np.ndarray, int]:
    out = np.empty(nt, np.float32)
    tl = C.c_int()
    _util_check(lib().fwi_util_wavelet(nt, dt, fmax, _fptr(out), C.byref(tl)), "wavelet")
    return out, tl.value


def util_b1d(nb: int, factor: float) -> np.ndarray:
    out = np.empty(nb, np.float32)
    _util_check(lib().fwi_util_b1d(nb, factor, _fptr(out)), "b1d")
    return out


def util_grid_index(coord: np.ndarray, dh: float, nb: int) -> np.ndarray:
    c = np.ascontiguousarray(coord, dtype=np.float32)
    out = np.empty(c.size, np.int32)
    _util_check(lib().fwi_util_grid_index(c.size, _fptr(c), dh, nb, out.ctypes.data_as(_I)), "grid index")
    return out


def util_window(xs: float, max_offset: float, nx: int, dh: float) -> tuple[int, int]:
    """Aperture window (c0, w) of a source at xs for a maximum offset."""
    c0, w = C.c_int(), C.c_int()
    _util_check(lib().fwi_util_window(xs, max_offset, nx, dh, C.byref(c0), C.byref(w)), "window")
    return c0.value, w.value


def util_bumps(nxx: int, nzz: int, nb: int, dh: float, ratio: float, varVp: float, seed: int, shot: int) -> np.ndarray:
    n = C.c_int()
    _util_check(lib().fwi_util_bumps(nxx, nzz, nb, dh, ratio, varVp, seed, shot, None, 0, C.byref(n)), "bumps")
    out = np.empty(5 * max(n.value, 1), np.float32)
    _util_check(lib().fwi_util_bumps(nxx, nzz, nb, dh, ratio, varVp, seed, shot, _fptr(out), n.value, C.byref(n)),
                "bumps")
    return out[: 5 * n.value].reshape(-1, 5)


def util_normal(seed: int, shot: int, stream: int, ctr: int) -> float:
    out = C.c_float()
    _util_check(lib().fwi_util_normal(seed, shot, stream, ctr, C.byref(out)), "normal")
    return out.value


# ---------------------------------------------------------------------------
# Mirror of the reference classes (method names of the C++ classes).

class Modeling:
    """Modeling (src/modeling/modeling.cuh:18-87) over the C ABI."""

    mode = MODE_MODELING

    def __init__(self, parameters: str | os.PathLike):
        self.parameters = str(parameters)
        self.srcId = 0
        self.ctx: Context | None = None
        self.seismogram: np.ndarray | None = None

    def set_parameters(self) -> None:
        self.ctx = Context(self.parameters, self.mode)

    @property
    def geometry_nsrc(self) -> int:
        return self.ctx.dims.nsrc

    def initialization(self) -> None:
        """Grid indices are computed once per context (modeling.cu:252-277)."""
        if not 0 <= self.srcId < self.ctx.dims.nsrc:
            raise IndexError("srcId out of range")

    def forward_solver(self) -> None:
        self.seismogram = self.ctx.model_shot(self.srcId)

    def get_seismogram(self) -> str:
        """Writes the seismogram of srcId under the reference's file name (modeling.cu:279-284)."""
        d = self.ctx.dims
        folder = self.ctx.param("mod_output_folder")
        name = f"{folder}seismogram_nt{d.nt}_nr{d.nrec}_{int(np.float32(1e6) * np.float32(d.dt))}us_shot_{self.srcId + 1}.bin"
        np.ascontiguousarray(self.seismogram.T).astype(np.float32).tofile(name)
        return name

    def show_information(self) -> None:
        d = self.ctx.dims
        print(f"Model dimensions: (z = {(d.nz - 1) * d.dh}, x = {(d.nx - 1) * d.dh}) m")
        print(f"Running shot {self.srcId + 1} of {d.nsrc} in total")


class Migration(Modeling):
    """Migration (src/migration/migration.cuh:6-38) over the C ABI."""

    mode = MODE_MIGRATION

    def set_parameters(self) -> None:
        super().set_parameters()
        self.ctx.rtm_reset()

    def forward_propagation(self) -> None:
        """The random-boundary forward pass runs with the backward pass in one call."""

    def backward_propagation(self) -> None:
        d = self.ctx.dims
        path = f"{self.ctx.param('mig_input_folder')}{self.ctx.param('mig_input_prefix')}{self.srcId + 1}.bin"
        data = np.fromfile(path, np.float32, d.nt * d.nrec).reshape(d.nrec, d.nt).T
        self.ctx.rtm_shot(self.srcId, data)

    def export_seismic(self) -> str:
        d = self.ctx.dims
        img = self.ctx.rtm_image()
        name = f"{self.ctx.param('mig_output_folder')}RTM_section_{int(d.fmax)}Hz_{d.nz}x{d.nx}_{int(d.dh)}m.bin"
        np.ascontiguousarray(img.T).astype(np.float32).tofile(name)
        return name


class Inversion(Modeling):
    """Inversion (src/inversion/inversion.cuh:6-83) over the C ABI."""

    mode = MODE_INVERSION

    def set_parameters(self) -> None:
        super().set_parameters()
        d = self.ctx.dims
        self.max_iteration = int(self.ctx.param("max_iteration"))
        self.iteration = 0
        self.residuo: list[float] = []
        self.converged = False
        obs = np.empty((d.nsrc, d.nrec, d.nt), np.float32)
        folder, prefix = self.ctx.param("inv_input_folder"), self.ctx.param("inv_input_prefix")
        for s in range(d.nsrc):
            obs[s] = np.fromfile(f"{folder}{prefix}{s + 1}.bin", np.float32, d.nt * d.nrec).reshape(d.nrec, d.nt)
        self.ctx.set_observed_raw(obs.ravel())
        self.step = 0.0
        self.sum_res = 0.0

    def compute_gradient(self) -> None:
        self.sum_res = self.ctx.compute_gradient(self.iteration < self.max_iteration)

    def check_convergence(self) -> None:
        self.iteration += 1
        self.residuo.append(float(np.sqrt(np.float32(self.sum_res))))
        self.converged = self.iteration > self.max_iteration

    def optimization(self) -> None:
        self.step = self.ctx.optimization(self.residuo[-1])

    def update_model(self) -> np.ndarray:
        return self.ctx.update_model(self.step)
