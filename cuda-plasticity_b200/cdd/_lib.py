"""ctypes binding of libcdd.so (the C ABI declared in include/cdd.h).

The shared library is built in-tree by ``cuda-plasticity_b200/build.py`` next to this file. There
is no fallback: if it is missing or fails to load, ``load()`` raises.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcdd.so")

CDD_OK = 0
CDD_ERR_ARG = 1
CDD_ERR_SHAPE = 2
CDD_ERR_CUDA = 3
CDD_ERR_NONFINITE = 4
CDD_ERR_TIMEOUT = 5
CDD_ERR_UNSUPPORTED = 6
CDD_ERR_ALLOC = 7
CDD_ERR_IO = 8
CDD_OBS_BETA_ELASTIC = 0
CDD_OBS_ROTATION = 1
CDD_OBS_RODRIGUES = 2
CDD_OBS_RHO = 3
CDD_OBS_RODRIGUES_RHO = 4
CDD_OBS_SINK = 0x100
STATUS_NAMES = {0: "OK", 1: "ERR_ARG", 2: "ERR_SHAPE", 3: "ERR_CUDA", 4: "ERR_NONFINITE",
                5: "ERR_TIMEOUT", 6: "ERR_UNSUPPORTED", 7: "ERR_ALLOC"}

CDD_F64 = 0
CDD_F32 = 1


class cdd_instance(ctypes.Structure):
    _fields_ = [
        ("ndim", ctypes.c_int),
        ("shape", ctypes.c_int * 3),
        ("mu", ctypes.c_double),
        ("nu", ctypes.c_double),
        ("Lambda", ctypes.c_double),
        ("cfl", ctypes.c_double),
        ("has_load", ctypes.c_int),
        ("load_rate", ctypes.c_double * 3),
        ("load_initial", ctypes.c_double * 3),
        ("load_t0", ctypes.c_double),
        ("load_mu", ctypes.c_double),
        ("load_nu", ctypes.c_double),
        ("dynamics", ctypes.c_int),
        ("vacancy", ctypes.c_int),
        ("vac_alpha", ctypes.c_double),
        ("vac_beta", ctypes.c_double),
        ("vac_gamma", ctypes.c_double),
        ("dt_max", ctypes.c_double),
    ]


CDD_DYN_GLIDE_CLIMB, CDD_DYN_GLIDE_ONLY = 0, 1


class cdd_tuning(ctypes.Structure):
    """Per-instance launch-shape choices (include/cdd.h); 0 keeps the built-in rule."""
    _fields_ = [
        ("fft_radix", ctypes.c_int),
        ("rows_lines", ctypes.c_int),
        ("mid_cols", ctypes.c_int),
        ("green_cols", ctypes.c_int),
        ("stencil_planes", ctypes.c_int),
        ("plane_fft", ctypes.c_int),
    ]

    KEYS = ("fft_radix", "rows_lines", "mid_cols", "green_cols", "stencil_planes", "plane_fft")

    @classmethod
    def from_dict(cls, d):
        d = d or {}
        return cls(*[int(d.get(k, 0) or 0) for k in cls.KEYS])

    def to_dict(self):
        return {k: int(getattr(self, k)) for k in self.KEYS}


class CDDError(RuntimeError):
    def __init__(self, code, msg):
        self.code = code
        super().__init__("%s: %s" % (STATUS_NAMES.get(code, str(code)), msg))


_lib = None

CDD_PBAR = 9   # doubles per instance in the parameter cotangent of cdd_step_adjoint

_PROTOS = {
    "cdd_plan_create_tuned": (ctypes.c_int, [ctypes.POINTER(cdd_instance), ctypes.c_int, ctypes.c_int,
                                             ctypes.POINTER(cdd_tuning), ctypes.POINTER(ctypes.c_void_p)]),
    "cdd_plan_tuning": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(cdd_tuning)]),
    "cdd_plan_create": (ctypes.c_int, [ctypes.POINTER(cdd_instance), ctypes.c_int, ctypes.c_int,
                                       ctypes.POINTER(ctypes.c_void_p)]),
    "cdd_plan_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "cdd_plan_num_instances": (ctypes.c_int, [ctypes.c_void_p]),
    "cdd_plan_precision": (ctypes.c_int, [ctypes.c_void_p]),
    "cdd_plan_field_elems": (ctypes.c_longlong, [ctypes.c_void_p]),
    "cdd_plan_field_offset": (ctypes.c_longlong, [ctypes.c_void_p, ctypes.c_int]),
    "cdd_plan_stress_elems": (ctypes.c_longlong, [ctypes.c_void_p]),
    "cdd_plan_stress_offset": (ctypes.c_longlong, [ctypes.c_void_p, ctypes.c_int]),
    "cdd_plan_cells": (ctypes.c_longlong, [ctypes.c_void_p, ctypes.c_int]),
    "cdd_plan_scratch_bytes": (ctypes.c_longlong, [ctypes.c_void_p]),
    "cdd_stress": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "cdd_flux": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p,
                                ctypes.c_void_p, ctypes.c_void_p]),
    "cdd_set_time": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                    ctypes.POINTER(ctypes.c_double)]),
    "cdd_get_time": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                    ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)]),
    "cdd_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "cdd_step_fixed": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p]),
    "cdd_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]),
    "cdd_observables": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                       ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]),
    "cdd_check_status": (ctypes.c_int, [ctypes.c_void_p]),
    "cdd_flux_vjp": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p,
                                    ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "cdd_flux_branches": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p,
                                         ctypes.c_void_p]),
    "cdd_plan_record_elems": (ctypes.c_longlong, [ctypes.c_void_p]),
    "cdd_step_record": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_void_p, ctypes.c_void_p]),
    "cdd_step_adjoint": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "cdd_flux_with_stress": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double,
                                            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "cdd_stress_adjoint": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "cdd_stress_dnu": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "cdd_stress_noalloc": (ctypes.c_int, [ctypes.POINTER(cdd_instance), ctypes.c_int, ctypes.c_void_p,
                                          ctypes.c_void_p, ctypes.c_void_p]),
    "cdd_set_vacancy": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "cdd_observe_field": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p]),
    "cdd_field_import": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                        ctypes.c_void_p, ctypes.c_void_p]),
    "cdd_field_export": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_int, ctypes.c_void_p]),
    "cdd_ics_read": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_void_p,
                                    ctypes.c_void_p]),
    "cdd_ics_write": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_void_p,
                                     ctypes.c_void_p]),
    "cdd_plas_append": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_double,
                                       ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "cdd_plas_frames": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_int,
                                       ctypes.POINTER(ctypes.c_longlong)]),
    "cdd_plas_read": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_int,
                                     ctypes.c_longlong, ctypes.POINTER(ctypes.c_double), ctypes.c_void_p,
                                     ctypes.c_void_p]),
    "cdd_last_error": (ctypes.c_char_p, []),
    "cdd_version": (ctypes.c_char_p, []),
}


def load():
    """Load libcdd.so once and return the ctypes handle (raises if it is absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("libcdd.so not built: run `python cuda-plasticity_b200/build.py` "
                           "(expected at %s)" % LIB_PATH)
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in _PROTOS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def exported_names():
    return sorted(_PROTOS)


def check(rc):
    """Raise CDDError for a nonzero status, with the library's message."""
    if rc != CDD_OK:
        msg = load().cdd_last_error().decode(errors="replace")
        raise CDDError(rc, msg)
    return rc
