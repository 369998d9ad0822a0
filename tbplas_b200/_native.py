"""ctypes binding of libtbpm_b200.so (C ABI declared in include/tbpm_b200.h).

The library is the only compute path of this package: when it cannot be
loaded, or no CUDA device is visible, every compute entry point raises instead
of falling back to anything else.
"""

import ctypes
import os
import threading
from typing import Dict, Optional

import numpy as np

LIB_NAME = "libtbpm_b200.so"
LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), LIB_NAME)

TBPM_OK = 0
TBPM_ERR_ARG = 1
TBPM_ERR_NORM = 2
TBPM_ERR_NAN = 3
TBPM_ERR_CUDA = 4
TBPM_ERR_TIMEOUT = 5
TBPM_ERR_OOM = 6
TBPM_ERR_STATE = 7

PREC_FP64 = 0
PREC_FP32 = 1
STATE_EXP = 0
STATE_UNIT = 1
LAYOUT_CSR = 0
LAYOUT_DXY = 1

# every symbol include/tbpm_b200.h declares
EXPORTED_SYMBOLS = (
    "tbpm_create", "tbpm_destroy", "tbpm_last_error", "tbpm_set_options",
    "tbpm_get_options", "tbpm_get_stream", "tbpm_last_stats", "tbpm_version",
    "tbpm_ham_upload", "tbpm_ham_release", "tbpm_dos", "tbpm_dos_states",
    "tbpm_accond", "tbpm_accond_states", "tbpm_dccond", "tbpm_dccond_states",
    "tbpm_psi_t", "tbpm_random_states", "tbpm_fermi_cheb_coef",
    "tbpm_cheb_timestep", "tbpm_fermi_apply", "tbpm_session_dos_begin",
    "tbpm_session_advance", "tbpm_session_read", "tbpm_cheb_timestep_noalloc",
    "tbpm_dos_segmented", "tbpm_nn_gemm_tn", "tbpm_nn_transpose_bf16", "tbpm_nn_im2col",
    "tbpm_nn_col2im", "tbpm_nn_bias_act", "tbpm_nn_act_backward", "tbpm_nn_colsum",
    "tbpm_nn_mse", "tbpm_nn_adam", "tbpm_nn_cast_bf16", "tbpm_supercell_ham",
    "tbpm_supercell_csr", "tbpm_dyn_pol", "tbpm_dyn_pol_states", "tbpm_eigenstates",
    "tbpm_eigenstates_states", "tbpm_kbdc", "tbpm_kbdc_states", "tbpm_haydock_coef",
    "tbpm_cond_from_trace", "tbpm_session_export", "tbpm_session_dos_resume",
    "tbpm_nn_gemm_tn_mma", "tbpm_nn_tc_status", "tbpm_trig_sums", "tbpm_trig_cumtrapz",
    "tbpm_selftest_wait_timeout", "tbpm_dccond_accumulate",
)


class TbpmError(RuntimeError):
    """Error status returned by libtbpm_b200."""

    def __init__(self, code: int, message: str) -> None:
        super().__init__(message)
        self.code = code


class NormError(TbpmError):
    """Wave-function norm check failed (the reference Fortran `stop`s here)."""


class DeviceTimeoutError(TbpmError):
    """A bounded device-side wait ran out (TBPM_ERR_TIMEOUT); the results of
    that call are invalid, the context stays usable."""


class NanError(NormError):
    """The norm check found a NaN or infinite norm (TBPM_ERR_NAN); the reference's
    check_norm treats it as a broken norm, so this is a NormError too."""


class Options(ctypes.Structure):
    _fields_ = [
        ("precision", ctypes.c_int),
        ("batch", ctypes.c_int),
        ("state_kind", ctypes.c_int),
        ("verbose", ctypes.c_int),
        ("threads_per_block", ctypes.c_int),
        ("rows_per_tile", ctypes.c_int),
        ("steps_per_graph", ctypes.c_int),
        ("use_graphs", ctypes.c_int),
        ("fp32_chk_thr", ctypes.c_double),
        ("vector_width", ctypes.c_int),
        ("term_kernel", ctypes.c_int),
        ("dc_budget_gb", ctypes.c_double),
    ]


_c_int = ctypes.c_int
_c_i64 = ctypes.c_int64
_c_dbl = ctypes.c_double
_vp = ctypes.c_void_p


class Supercell(ctypes.Structure):
    """struct tbpm_supercell (host pointers into numpy arrays kept alive by the
    caller)."""
    _fields_ = [
        ("lat_vec", _vp),
        ("origin", _vp),
        ("n_orb", _c_int),
        ("orb_pos", _vp),
        ("orb_eng", _vp),
        ("n_hop", _c_int),
        ("hop_ind", _vp),
        ("hop_eng", _vp),
        ("dim", ctypes.c_int32 * 3),
        ("pbc", ctypes.c_int32 * 3),
        ("vac_id_sc", _vp),
        ("n_vac", _c_i64),
        ("sc_orb_eng", _vp),
        ("b_field", _c_dbl),
        ("gauge", _c_int),
        ("rescale", _c_dbl),
    ]

_SIGNATURES = {
    "tbpm_create": (_c_int, [_c_int, ctypes.POINTER(_vp)]),
    "tbpm_destroy": (_c_int, [_vp]),
    "tbpm_last_error": (ctypes.c_char_p, [_vp]),
    "tbpm_set_options": (_c_int, [_vp, ctypes.POINTER(Options)]),
    "tbpm_get_options": (_c_int, [_vp, ctypes.POINTER(Options)]),
    "tbpm_get_stream": (_vp, [_vp]),
    "tbpm_last_stats": (_c_int, [_vp, ctypes.POINTER(_c_i64), ctypes.POINTER(_c_dbl)]),
    "tbpm_version": (_c_int, []),
    "tbpm_ham_upload": (_c_int, [_vp, _vp, _vp, _vp, _c_i64, _c_i64, _vp, _vp, _c_dbl]),
    "tbpm_ham_release": (_c_int, [_vp]),
    "tbpm_dos": (_c_int, [_vp, _vp, _c_int, _vp, _vp, _vp, _c_i64, _c_i64, _c_int, _c_int,
                          _c_int, _c_int, _c_int, _c_dbl, _vp]),
    "tbpm_dos_states": (_c_int, [_vp, _vp, _c_int, _vp, _vp, _vp, _c_i64, _c_i64, _vp, _c_int,
                                 _c_int, _c_int, _c_dbl, _vp, _vp]),
    "tbpm_accond": (_c_int, [_vp, _vp, _c_int, _c_dbl, _c_dbl, _vp, _vp, _vp, _c_i64, _c_i64,
                             _c_dbl, _vp, _vp, _c_int, _c_int, _c_int, _c_int, _c_dbl, _c_int,
                             _c_int, _c_dbl, _vp]),
    "tbpm_accond_states": (_c_int, [_vp, _vp, _c_int, _c_dbl, _c_dbl, _vp, _vp, _vp, _c_i64,
                                    _c_i64, _c_dbl, _vp, _vp, _vp, _c_int, _c_int, _c_int,
                                    _c_dbl, _c_int, _c_dbl, _vp]),
    "tbpm_dccond": (_c_int, [_vp, _vp, _c_int, _c_dbl, _c_dbl, _vp, _vp, _vp, _c_i64, _c_i64,
                             _c_dbl, _vp, _vp, _c_int, _c_int, _c_int, _c_dbl, _vp, _c_int,
                             _vp, _c_int, _c_int, _c_int, _c_dbl, _vp, _vp]),
    "tbpm_dccond_states": (_c_int, [_vp, _vp, _c_int, _vp, _vp, _vp, _c_i64, _c_i64, _c_dbl,
                                    _vp, _vp, _vp, _c_int, _c_int, _c_dbl, _vp, _c_int, _vp,
                                    _c_int, _c_int, _c_dbl, _vp, _vp]),
    "tbpm_psi_t": (_c_int, [_vp, _vp, _c_int, _vp, _vp, _vp, _c_i64, _c_i64, _vp, _vp, _c_int,
                            _c_int, _c_int, _c_dbl, _vp]),
    "tbpm_random_states": (_c_int, [_vp, _c_i64, _c_int, _c_int, _c_int, _c_int, _c_int,
                                    _c_int, _vp]),
    "tbpm_fermi_cheb_coef": (_c_int, [_c_int, _c_dbl, _c_dbl, _c_int, _c_dbl, _vp,
                                      ctypes.POINTER(_c_int)]),
    "tbpm_cheb_timestep": (_c_int, [_vp, _vp, _c_int, _vp, _c_int, _c_int]),
    "tbpm_fermi_apply": (_c_int, [_vp, _vp, _c_int, _vp, _c_int]),
    "tbpm_session_dos_begin": (_c_int, [_vp, _vp, _c_int, _c_int, _c_int, _c_int, _c_int,
                                        _c_int]),
    "tbpm_session_advance": (_c_int, [_vp, _c_int]),
    "tbpm_session_read": (_c_int, [_vp, _vp, _vp, ctypes.POINTER(_c_int)]),
    "tbpm_cheb_timestep_noalloc": (_c_int, [_vp, _vp, _c_int, _vp, _vp, _vp, _c_i64, _c_i64,
                                            _vp, _c_int, _c_int]),
    "tbpm_dos_segmented": (_c_int, [_vp, _vp, _c_int, _vp, _vp, _vp, _c_i64, _c_i64, _vp,
                                    _c_int, _c_int, _c_int, _c_int, _c_int, _c_dbl, _vp, _vp]),
    "tbpm_nn_gemm_tn": (_c_int, [_vp, _c_int, _vp, _c_int, _vp, _c_int, _c_int, _c_int, _c_int,
                                 ctypes.c_float, ctypes.c_float, _vp]),
    "tbpm_nn_gemm_tn_mma": (_c_int, [_vp, _c_int, _vp, _c_int, _vp, _c_int, _c_int, _c_int,
                                    _c_int, ctypes.c_float, ctypes.c_float, _vp]),
    "tbpm_nn_tc_status": (_c_int, [ctypes.POINTER(_c_int)]),
    "tbpm_nn_transpose_bf16": (_c_int, [_vp, _c_int, _c_int, _vp, _vp]),
    "tbpm_nn_im2col": (_c_int, [_vp, _c_int, _c_int, _c_int, _c_int, _c_int, _c_int, _c_int,
                                _vp, _vp]),
    "tbpm_nn_col2im": (_c_int, [_vp, _c_int, _c_int, _c_int, _c_int, _c_int, _c_int, _c_int,
                                _vp, _vp]),
    "tbpm_nn_bias_act": (_c_int, [_vp, _vp, _c_int, _c_int, _c_int, _vp, _vp, _vp, _vp]),
    "tbpm_nn_act_backward": (_c_int, [_vp, _vp, _c_i64, _c_int, _vp, _vp, _vp]),
    "tbpm_nn_colsum": (_c_int, [_vp, _c_int, _c_int, _vp, _vp]),
    "tbpm_nn_mse": (_c_int, [_vp, _vp, _c_i64, _vp, _vp, _vp, _vp]),
    "tbpm_nn_adam": (_c_int, [_vp, _vp, _vp, _vp, _c_i64, ctypes.c_float, ctypes.c_float,
                              ctypes.c_float, ctypes.c_float, ctypes.c_float, _c_int, _vp, _vp]),
    "tbpm_nn_cast_bf16": (_c_int, [_vp, _c_i64, _vp, _vp]),
    "tbpm_supercell_ham": (_c_int, [_vp, ctypes.POINTER(Supercell), _c_int, _c_dbl,
                                    ctypes.POINTER(_c_i64), ctypes.POINTER(_c_i64),
                                    ctypes.POINTER(_c_dbl)]),
    "tbpm_dyn_pol": (_c_int, [_vp, _vp, _c_int, _c_dbl, _c_dbl, _vp, _vp, _vp, _c_i64, _c_i64,
                              _c_dbl, _vp, _vp, _vp, _vp, _vp, _c_int, _c_int, _c_int, _c_int,
                              _c_dbl, _vp, _c_int, _c_int, _c_int, _c_dbl, _vp]),
    "tbpm_dyn_pol_states": (_c_int, [_vp, _vp, _c_int, _c_dbl, _c_dbl, _vp, _vp, _vp, _c_i64,
                                     _c_i64, _vp, _vp, _vp, _vp, _c_int, _vp, _c_int, _c_int,
                                     _c_int, _c_dbl, _c_int, _c_dbl, _vp]),
    "tbpm_eigenstates": (_c_int, [_vp, _vp, _c_int, _vp, _vp, _vp, _c_i64, _c_i64, _c_int,
                                  _c_int, _c_int, _c_dbl, _vp, _c_int, _c_int, _c_int, _c_dbl,
                                  _vp]),
    "tbpm_eigenstates_states": (_c_int, [_vp, _vp, _c_int, _vp, _vp, _vp, _c_i64, _c_i64, _vp,
                                         _c_int, _c_int, _c_dbl, _vp, _c_int, _c_int, _c_dbl,
                                         _vp]),
    "tbpm_kbdc": (_c_int, [_vp, _c_int, _vp, _vp, _vp, _c_i64, _c_i64, _c_dbl, _vp, _vp,
                           _c_int, _c_int, _c_int, _c_int, _vp]),
    "tbpm_kbdc_states": (_c_int, [_vp, _vp, _vp, _vp, _c_i64, _c_i64, _c_dbl, _vp, _vp, _vp,
                                  _c_int, _c_int, _c_int, _vp]),
    "tbpm_haydock_coef": (_c_int, [_vp, _vp, _vp, _vp, _c_i64, _c_i64, _c_dbl, _vp, _c_int,
                                   _vp, _c_int, _c_int, _vp, _vp]),
    "tbpm_session_export": (_c_int, [_vp, _vp, _vp]),
    "tbpm_session_dos_resume": (_c_int, [_vp, _vp, _c_int, _c_int, _vp, _vp, _vp, _vp, _c_int,
                                         _c_int]),
    "tbpm_cond_from_trace": (_c_int, [_vp, _vp, _c_int, _vp, _c_int, _c_dbl, _c_dbl, _c_int,
                                      _c_dbl, _c_int, _vp]),
    "tbpm_supercell_csr": (_c_int, [_vp, ctypes.POINTER(Supercell), _c_int, _c_dbl,
                                    ctypes.POINTER(_c_i64), ctypes.POINTER(_c_i64),
                                    ctypes.POINTER(_c_dbl), _vp, _vp, _vp, _vp, _vp]),
    "tbpm_selftest_wait_timeout": (_c_int, [_vp]),
    "tbpm_dccond_accumulate": (_c_int, [_vp, _vp, _c_int, _vp, _c_int, _c_int, _c_int, _c_int,
                                        _c_int, _c_int, _c_dbl, _vp, _c_int, _vp, _c_int,
                                        _c_int, _c_dbl, _vp, _vp]),
    "tbpm_trig_sums": (_c_int, [_vp, _vp, _c_int, _vp, _vp, _c_int, _vp, _c_int, _c_dbl,
                                _c_int, _c_int, _vp, _vp]),
    "tbpm_trig_cumtrapz": (_c_int, [_vp, _vp, _c_int, _vp, _vp, _c_int, _vp, _c_dbl, _vp,
                                    _vp]),
}

_lib = None
_lib_lock = threading.Lock()


def load_library() -> ctypes.CDLL:
    """Load libtbpm_b200.so (raises if it has not been built)."""
    global _lib
    with _lib_lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(
                    f"{LIB_NAME} not found at {LIB_PATH}; build it with "
                    "`python -m tbplas_b200.build` (nvcc, sm_100a)")
            lib = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in _SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


def ptr(a: Optional[np.ndarray]) -> Optional[int]:
    """Raw data pointer of a contiguous numpy array (None -> NULL)."""
    if a is None:
        return None
    return a.ctypes.data


def as_c(a, dtype) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=dtype))


def raise_for(code: int, message: str) -> None:
    if code == TBPM_OK:
        return
    if code == TBPM_ERR_ARG:
        raise ValueError(message)
    if code == TBPM_ERR_NORM:
        raise NormError(code, message)
    if code == TBPM_ERR_NAN:
        raise NanError(code, message)
    if code == TBPM_ERR_OOM:
        raise MemoryError(message)
    if code == TBPM_ERR_TIMEOUT:
        raise DeviceTimeoutError(code, message)
    raise TbpmError(code, message)


class Context:
    """One libtbpm_b200 context: a CUDA device, its stream and its buffers."""

    def __init__(self, device: int = 0) -> None:
        self._lib = load_library()
        h = _vp()
        rc = self._lib.tbpm_create(int(device), ctypes.byref(h))
        if rc != TBPM_OK:
            raise TbpmError(rc, f"tbpm_create(device={device}) failed: no usable CUDA device")
        self.handle = h
        self.device = int(device)

    def close(self) -> None:
        if getattr(self, "handle", None):
            self._lib.tbpm_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, rc: int) -> None:
        if rc != TBPM_OK:
            msg = self._lib.tbpm_last_error(self.handle)
            raise_for(rc, msg.decode() if msg else f"tbpm error {rc}")

    @property
    def options(self) -> Options:
        o = Options()
        self.check(self._lib.tbpm_get_options(self.handle, ctypes.byref(o)))
        return o

    def set_options(self, **kw) -> None:
        o = self.options
        for k, v in kw.items():
            if not hasattr(o, k):
                raise ValueError(f"unknown option {k}")
            setattr(o, k, v)
        self.check(self._lib.tbpm_set_options(self.handle, ctypes.byref(o)))

    @property
    def stream(self) -> int:
        return self._lib.tbpm_get_stream(self.handle) or 0

    def last_stats(self):
        n = _c_i64()
        b = _c_dbl()
        self.check(self._lib.tbpm_last_stats(self.handle, ctypes.byref(n), ctypes.byref(b)))
        return int(n.value), float(b.value)

    def call(self, name: str, *args) -> None:
        fn = getattr(self._lib, name)
        self.check(fn(self.handle, *args))


_contexts: Dict[int, Context] = {}
_ctx_lock = threading.Lock()


def default_device() -> int:
    """CUDA device of this process: LOCAL_RANK under torchrun, else 0."""
    return int(os.environ.get("TBPM_DEVICE", os.environ.get("LOCAL_RANK", "0")))


def get_context(device: Optional[int] = None) -> Context:
    """Process-wide context per device (created on first use)."""
    dev = default_device() if device is None else int(device)
    with _ctx_lock:
        ctx = _contexts.get(dev)
        if ctx is None:
            ctx = Context(dev)
            _contexts[dev] = ctx
        return ctx


def fermi_cheb_coef(nr_fermi: int, beta: float, mu: float, one_minus_fermi: bool,
                    eps: float) -> np.ndarray:
    """Chebyshev coefficients of the (1 -) Fermi operator (funcs.f90:60-123)."""
    lib = load_library()
    coef = np.zeros(int(nr_fermi), dtype=np.float64)
    n = _c_int(0)
    rc = lib.tbpm_fermi_cheb_coef(int(nr_fermi), float(beta), float(mu),
                                  1 if one_minus_fermi else 0, float(eps), ptr(coef),
                                  ctypes.byref(n))
    raise_for(rc, "tbpm_fermi_cheb_coef: invalid arguments")
    return coef[:n.value].copy()
