"""ctypes binding of the engine's C ABI (``include/gl_engine.h``).

This is the same binding a maintainer of the reference's Python package would
add: plain ``ctypes`` over ``libgl_b200.so``.  Loading fails loudly when the
library has not been built; there is no CPU fallback.
"""

from __future__ import annotations

import ctypes as C
import os
import threading
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "_native" / "libgl_b200.so"

GL_OK = 0
STATUS_NAMES = {
    0: "GL_OK", 1: "GL_ERR_INVALID_ARGUMENT", 2: "GL_ERR_UNSUPPORTED", 3: "GL_ERR_OPTIONS",
    4: "GL_ERR_UNIFORM_CURRENT", 5: "GL_ERR_COMPONENT_SIZE", 6: "GL_ERR_COMPONENTS",
    7: "GL_ERR_SUPPORT", 8: "GL_ERR_SECTOR", 9: "GL_ERR_ZERO_INPUT", 10: "GL_ERR_ORDER2_DOMAIN",
    11: "GL_ERR_ORDER3_DOMAIN", 12: "GL_ERR_OFF_GRID", 13: "GL_ERR_NYQUIST", 14: "GL_ERR_ALIAS",
    15: "GL_ERR_SCALE", 16: "GL_ERR_RANK", 17: "GL_ERR_EMPTY_SUPPORT", 18: "GL_ERR_OUTSIDE_PLAN",
    19: "GL_ERR_NONFINITE", 20: "GL_ERR_WORKSPACE", 21: "GL_ERR_CUDA", 22: "GL_ERR_TIMEOUT",
    23: "GL_ERR_COEFFICIENTS",
}

COMP_ETA11, COMP_PSI11, COMP_ETA22, COMP_PSI22, COMP_ETA33, COMP_PSI33 = 1, 2, 4, 8, 16, 32
COMP_ETA44, COMP_PSI44 = 64, 128
COMP_NAMES = {COMP_ETA11: "eta11", COMP_PSI11: "psi11", COMP_ETA22: "eta22",
              COMP_PSI22: "psi22", COMP_ETA33: "eta33", COMP_PSI33: "psi33", COMP_ETA44: "eta44",
              COMP_PSI44: "psi44"}
GRID_COMPACT, GRID_REFERENCE = 0, 1
OUT_COMPLEX, OUT_REAL = 0, 1
SPECTRA_FULL, SPECTRA_BOX = 0, 1
MAX_LANES = 8  # GL_MAX_LANES


class PlanDesc(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int),
        ("lx", C.c_double), ("ly", C.c_double),
        ("depth", C.c_double), ("gravity", C.c_double),
        ("order", C.c_int), ("components", C.c_int),
        ("eta22_rank", C.c_int), ("inner_rank", C.c_int), ("outer_rank", C.c_int),
        ("allow_below_model_parent_domain", C.c_int),
        ("box_x0", C.c_int), ("box_y0", C.c_int), ("box_w", C.c_int), ("box_h", C.c_int),
        ("grid", C.c_int), ("max_units", C.c_int), ("output", C.c_int),
    ]


class Eta44Desc(C.Structure):
    _fields_ = [("n", C.c_int), ("dk", C.c_double), ("depth", C.c_double),
                ("peak_depth", C.c_double), ("rank", C.c_int),
                ("nodes", C.POINTER(C.c_double)), ("weights", C.POINTER(C.c_double)),
                ("box_x0", C.c_int), ("box_y0", C.c_int), ("box_w", C.c_int), ("box_h", C.c_int),
                ("max_units", C.c_int), ("output", C.c_int), ("components", C.c_int),
                ("gravity", C.c_double)]


class ModalDesc(C.Structure):
    _fields_ = [("points", C.c_int), ("width", C.c_int), ("order", C.c_int),
                ("base_bin", C.c_int), ("count", C.c_int), ("q_step", C.c_double),
                ("freq_step", C.c_double), ("depth", C.c_double), ("scale22", C.c_double),
                ("lambda2", C.c_double), ("lambda3", C.c_double), ("rank", C.c_int),
                ("nodes", C.POINTER(C.c_double)), ("weights", C.POINTER(C.c_double))]


class Eta20Desc(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("span", C.c_int), ("base_bin", C.c_int),
                ("count", C.c_int), ("qx_step", C.c_double), ("qy_step", C.c_double),
                ("freq_step", C.c_double), ("depth", C.c_double), ("dq", C.c_double),
                ("rank", C.c_int), ("nodes", C.POINTER(C.c_double)),
                ("weights", C.POINTER(C.c_double))]


class Tuning(C.Structure):
    _fields_ = [("pair_row_groups", C.c_int), ("triple_row_groups", C.c_int),
                ("col_block_columns", C.c_int)]


class PlanInfo(C.Structure):
    _fields_ = [
        ("ncx", C.c_int), ("ncy", C.c_int),
        ("box1", C.c_int * 4), ("box2", C.c_int * 4), ("box3", C.c_int * 4),
        ("n_components", C.c_int), ("component_ids", C.c_int * 6),
        ("transforms_per_unit", C.c_double),
        ("ncy_pair", C.c_int), ("ncy_triple", C.c_int), ("ncx_pair", C.c_int),
    ]


class KernelStat(C.Structure):
    _fields_ = [("name", C.c_char * 40), ("launches", C.c_int), ("ms_total", C.c_double),
                ("bytes_total", C.c_double)]


class WitStats(C.Structure):
    _fields_ = [("candidates", C.c_ulonglong), ("kept", C.c_ulonglong), ("near", C.c_ulonglong),
                ("strict_zero_output", C.c_ulonglong), ("strict_zero_intermediate", C.c_ulonglong),
                ("max_residual", C.c_double), ("min_detuning", C.c_double),
                ("max_strict_zero_source", C.c_double)]


# name -> (restype, argtypes); every symbol declared in include/gl_engine.h
SIGNATURES = {
    "gl_plan_create": (C.c_int, [C.POINTER(C.c_void_p), C.POINTER(PlanDesc)]),
    "gl_plan_destroy": (None, [C.c_void_p]),
    "gl_eta44_plan_create": (C.c_int, [C.POINTER(C.c_void_p), C.POINTER(Eta44Desc)]),
    "gl_eta44_execute_partial": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int,
                                           C.c_int, C.c_void_p, C.c_void_p, C.c_size_t,
                                           C.c_void_p, C.c_void_p]),
    "gl_eta44_execute_part": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int,
                                        C.c_int, C.c_void_p, C.c_void_p, C.c_size_t,
                                        C.c_void_p, C.c_void_p]),
    "gl_eta44_finalize": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_size_t, C.c_void_p]),
    "gl_plan_get_info": (C.c_int, [C.c_void_p, C.POINTER(PlanInfo)]),
    "gl_workspace_size": (C.c_int, [C.c_void_p, C.POINTER(C.c_size_t)]),
    "gl_plan_set_wait_test": (C.c_int, [C.c_void_p, C.c_uint, C.c_longlong]),
    "gl_plan_set_tuning": (C.c_int, [C.c_void_p, C.POINTER(Tuning)]),
    "gl_plan_set_lanes": (C.c_int, [C.c_void_p, C.c_int]),
    "gl_deposit_modes": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int,
                                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "gl_execute": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                             C.c_size_t, C.c_void_p, C.c_void_p]),
    "gl_adjoint_workspace_size": (C.c_int, [C.c_void_p, C.POINTER(C.c_size_t)]),
    "gl_adjoint_execute": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                                     C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p]),
    "gl_deposit_modes_adjoint": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                           C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.c_void_p]),
    "gl_modal_workspace_size": (C.c_int, [C.POINTER(ModalDesc), C.POINTER(C.c_size_t)]),
    "gl_modal_level": (C.c_int, [C.POINTER(ModalDesc), C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                 C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p]),
    "gl_eta20_workspace_size": (C.c_int, [C.POINTER(Eta20Desc), C.POINTER(C.c_size_t)]),
    "gl_eta20_level": (C.c_int, [C.POINTER(Eta20Desc), C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                 C.c_void_p, C.c_size_t, C.c_void_p]),
    "gl_series_synthesize": (C.c_int, [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                       C.c_void_p]),
    "gl_fft2": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "gl_box_synthesize_noalloc": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                            C.c_int, C.c_void_p, C.c_double, C.c_void_p, C.c_int,
                                            C.c_void_p]),
    "gl_wit_workspace_size": (C.c_size_t, [C.c_int]),
    "gl_wit_eta44": (C.c_int, [C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int,
                               C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                               C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p]),
    "gl_wit_read_stats": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(WitStats)]),
    "gl_wit_sector": (C.c_int, [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int,
                                C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p]),
    "gl_wit_read_sector_stats": (C.c_int, [C.c_int, C.c_void_p, C.c_int, C.POINTER(WitStats)]),
    "gl_wit_candidates": (C.c_ulonglong, [C.c_int, C.c_int]),
    "gl_wit_sector_range": (C.c_int, [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                                      C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                      C.c_double, C.c_ulonglong, C.c_ulonglong, C.c_void_p,
                                      C.c_void_p, C.c_size_t, C.c_void_p]),
    "gl_gauss_laguerre": (C.c_int, [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "gl_dispersion_solve": (C.c_int, [C.c_int, C.POINTER(C.c_double), C.c_double, C.c_double,
                                      C.POINTER(C.c_double)]),
    "gl_get_last_error": (C.c_size_t, [C.c_char_p, C.c_size_t]),
    "gl_launch_count": (C.c_ulonglong, []),
    "gl_profile_begin": (C.c_int, []),
    "gl_profile_end": (C.c_int, [C.POINTER(KernelStat), C.c_int, C.POINTER(C.c_int)]),
    "gl_version": (C.c_char_p, []),
}

_lib = None
_lock = threading.Lock()


def load(path: Path | None = None) -> C.CDLL:
    """Load (once) and type the engine library.  Raises if it is missing."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        env = os.environ.get("GL_ENGINE_LIB")
        p = Path(path) if path else (Path(env) if env else LIB_PATH)
        if not p.exists():
            raise RuntimeError(
                f"GL engine library not built: {p} is missing "
                "(run `python __graft_entry__.py build` or gl_engine.build.build())")
        lib = C.CDLL(str(p))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def last_error() -> str:
    lib = load()
    buf = C.create_string_buffer(1024)
    lib.gl_get_last_error(buf, len(buf))
    return buf.value.decode("utf-8", "replace")


class EngineError(RuntimeError):
    """A C-ABI call returned a non-zero gl_status."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status
        self.message = message


def check(status: int) -> None:
    if status != GL_OK:
        raise EngineError(status, last_error())


def launch_count() -> int:
    return int(load().gl_launch_count())


def profile_begin() -> None:
    check(load().gl_profile_begin())


def profile_end() -> list[dict]:
    """Per-kernel {name, launches, ms_total, bytes_total} since profile_begin()."""
    lib = load()
    stats = (KernelStat * 64)()
    n = C.c_int()
    check(lib.gl_profile_end(stats, 64, C.byref(n)))
    return [{"name": stats[i].name.decode(), "launches": stats[i].launches,
             "ms_total": stats[i].ms_total, "bytes_total": stats[i].bytes_total}
            for i in range(min(n.value, 64))]
