"""ctypes binding of libsoliton_b200.so (the C ABI in include/soliton_b200.h).

The library is the only compute path of this package.  If it is missing the
import fails loudly: there is no CPU or pure-PyTorch fallback.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libsoliton_b200.so")

# status codes (include/soliton_b200.h)
SS_OK = 0
SS_ERR_ARG = 1
SS_ERR_CUDA = 2
SS_ERR_NONFINITE = 3
SS_ERR_STATE = 4
SS_ERR_WORKSPACE = 5
SS_ERR_TIMEOUT = 6

# theories
SS_THEORY_CHIRAL_MAGNET = 0
SS_THEORY_BABY_SKYRME = 1
SS_THEORY_GINZBURG_LANDAU = 2
SS_THEORY_ANISOTROPIC = 3

# precision / method
SS_FP64 = 0
SS_FP32 = 1
SS_PLAIN_FP64 = 2
PRECISIONS = {"fp64": SS_FP64, "fp32": SS_FP32, "plain_fp64": SS_PLAIN_FP64}

# charges
SS_CHARGE_SKYRMION = 0
SS_CHARGE_MAGNETIC = 1
SS_CHARGE_VORTEX = 2

# initial conditions (ss_initialize, ss_insert_soliton)
SS_INIT_GROUND = 0
SS_INIT_ANSATZ = 1
SS_ANSATZ_NONE = 0
SS_ANSATZ_BLOCH = 1
SS_ANSATZ_NEEL = 2
SS_ANSATZ_ANTI = 3

# colormaps (ss_render_rgba)
SS_RENDER_JET = 0
SS_RENDER_GRAY = 1
SS_RENDER_MAGNETIZATION = 2

# diagnostic densities (ss_field_density)
SS_DENSITY_HIGGS = 0
SS_DENSITY_HIGGS1 = 1
SS_DENSITY_HIGGS2 = 2
SS_DENSITY_PHASE_DIFFERENCE = 3
SS_DENSITY_SUPERCURRENT = 4
SS_DENSITY_MAGNETIC_FIELD = 5

# couplings
SS_COUPLING_KAPPA = 0
SS_COUPLING_MPI = 1
SS_COUPLING_LAMBDA = 2
SS_COUPLING_COUP_K = 3
SS_COUPLING_COUP_H = 4
SS_COUPLING_COUP_MU = 5


class SolverError(RuntimeError):
    """A native call returned a non-zero status."""

    def __init__(self, status, message):
        super().__init__(f"[{status}] {message}")
        self.status = status


class NonFiniteError(SolverError):
    """A reduction produced NaN or Inf (SS_ERR_NONFINITE)."""


class DeviceTimeoutError(SolverError):
    """A bounded device-side wait expired (SS_ERR_TIMEOUT); re-bind before further use."""


_lib = None

_P = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double
_SIG = {
    "ss_abi_version": ([], _I),
    "ss_status_string": ([_I], ctypes.c_char_p),
    "ss_last_error": ([], ctypes.c_char_p),
    "ss_create": ([_I, _P, _I, _P, _I, _I, ctypes.POINTER(_P)], _I),
    "ss_destroy": ([_P], _I),
    "ss_workspace_bytes": ([_P, ctypes.POINTER(ctypes.c_size_t)], _I),
    "ss_bind": ([_P, _P, _P, _P, ctypes.c_size_t, _P], _I),
    "ss_step": ([_P, _I, _D, _P, _P], _I),
    "ss_step_async": ([_P, _I, _D, _P, _P], _I),
    "ss_check_status": ([_P], _I),
    "ss_tma_enabled": ([_P], _I),
    "ss_autotune": ([_P, _I, _P], _I),
    "ss_get_variant": ([_P, _I], _I),
    "ss_set_variant": ([_P, _I, _I], _I),
    "ss_debug_wait_timeout": ([_P, ctypes.c_longlong, _I], _I),
    "ss_gradient": ([_P, _P, _P, _P], _I),
    "ss_energy_gradient": ([_P, _P, _P], _I),
    "ss_energy_density": ([_P, _P, _P], _I),
    "ss_energy": ([_P, _P, ctypes.POINTER(_D)], _I),
    "ss_energy_projected": ([_P, _P, ctypes.POINTER(_D)], _I),
    "ss_render_rgba": ([_I, _P, _I, _I, _I, _D, _D, _P, _P], _I),
    "ss_initialize": ([_P, _P, _P, _I, _I, _D, _D], _I),
    "ss_text_workspace_bytes": ([ctypes.c_longlong, ctypes.POINTER(ctypes.c_size_t)], _I),
    "ss_format_text": ([_P, _I, ctypes.c_longlong, _I, ctypes.c_longlong, ctypes.c_longlong, _P, ctypes.c_size_t,
                        ctypes.POINTER(ctypes.c_longlong), _P, ctypes.c_size_t, _P], _I),
    "ss_insert_soliton": ([_P, _P, _I, _I, _I, _I, _D], _I),
    "ss_charge_density": ([_P, _P, _I, _P], _I),
    "ss_charge": ([_P, _P, _I, ctypes.POINTER(_D)], _I),
    "ss_coupling_grad": ([_P, _P, _I, ctypes.POINTER(_D)], _I),
    "ss_field_density": ([_P, _P, _I, _P], _I),
    "ss_convert_field": ([_P, _P, _I, _P, _I, _I], _I),
    "ss_energy_gradient_exact": ([_P, _P, _P, _I], _I),
    "ss_set_forcing": ([_P, _P], _I),
    "ss_energy_noalloc": ([_I, _P, _I, _P, _I, _I, _P, ctypes.POINTER(_D), _P], _I),
    "ss_rk4_stage": ([_P, _P, _P, _P, _P, _P, _P, _D], _I),
    "ss_batch_create": ([_I, _I, _P, _I, _P, _I, _I, ctypes.POINTER(_P)], _I),
    "ss_batch_destroy": ([_P], _I),
    "ss_batch_workspace_bytes": ([_P, ctypes.POINTER(ctypes.c_size_t)], _I),
    "ss_batch_bind": ([_P, _P, _P, _P, ctypes.c_size_t, _P], _I),
    "ss_batch_step": ([_P, _I, _P, _P, _P], _I),
    "ss_batch_tma_enabled": ([_P], _I),
    "ss_batch_autotune": ([_P, _I, _P], _I),
    "ss_batch_get_shape": ([_P, _I], _I),
    "ss_batch_set_shape": ([_P, _I, _I], _I),
    "ss_graph_create": ([_P, _I, _P, _P], _I),
    "ss_graph_launch": ([_P], _I),
    "ss_batch_graph_create": ([_P, _I], _I),
    "ss_batch_graph_launch": ([_P], _I),
    "ss_batch_trajectory": ([_P, _I, _P, _P], _I),
    "ss_rk4_finalize": ([_P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P], _I),
}
EXPORTS = tuple(_SIG)


def load(path: str | None = None):
    """Load the native library (once) and declare its signatures."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise ImportError(
            f"libsoliton_b200.so not found at {path}; build it with "
            "`python -m soliton_solver_b200.build` (needs nvcc). There is no fallback path.")
    lib = ctypes.CDLL(path)
    for name, (args, res) in _SIG.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    if lib.ss_abi_version() != 1:
        raise ImportError("libsoliton_b200 ABI version mismatch")
    _lib = lib
    return lib


def check(status: int):
    if status == SS_OK:
        return
    lib = load()
    msg = lib.ss_last_error().decode(errors="replace")
    if status == SS_ERR_ARG:
        raise ValueError(msg)
    if status == SS_ERR_NONFINITE:
        raise NonFiniteError(status, msg)
    if status == SS_ERR_TIMEOUT:
        raise DeviceTimeoutError(status, msg)
    raise SolverError(status, msg)


def call(name: str, *args):
    check(getattr(load(), name)(*args))
