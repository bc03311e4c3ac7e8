"""Torch-facing wrapper of the libcdd C ABI: a plan over a batch of CDD instances.

Device memory and streams come from PyTorch; every computation runs in libcdd.so. A packed field
is a 1-D tensor of ``plan.field_elems`` elements (FP64 or FP32 by plan precision); instance ``i``
occupies ``field_view(t, i)``, shaped ``(9,) + shape`` with the last grid axis contiguous.
"""
import ctypes
import os
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np
import torch

from . import _lib
from ._lib import CDDError, check


@dataclass
class Instance:
    """One simulation: grid, material, dynamics and loading (see cdd_instance in include/cdd.h)."""
    shape: Sequence[int]
    mu: float = 1.0
    nu: float = 0.3
    Lambda: float = 0.0
    cfl: float = 0.25
    load_rate: Optional[Sequence[float]] = None
    load_initial: Sequence[float] = (0.0, 0.0, 0.0)
    load_t0: float = 0.0
    load_mu: Optional[float] = None
    load_nu: Optional[float] = None
    glide_only: bool = False   # the glide-only dynamics (CentralUpwindHJBetaPGlideOnlyDynamics.py)
    # vacancy coupling (VacancyDynamics.py): (alpha, beta, gamma) of sigma_ii -= alpha c,
    # c += beta d tr(beta^P), diffusion constant gamma; None: no vacancies
    vacancy: Optional[Sequence[float]] = None
    dt_max: float = 0.0        # > 0: upper bound of the adaptive step (the splitting mover's dtBound)

    def to_c(self):
        c = _lib.cdd_instance()
        shp = tuple(int(v) for v in self.shape)
        c.ndim = len(shp)
        for a in range(3):
            c.shape[a] = shp[a] if a < len(shp) else 1
        c.mu, c.nu, c.Lambda, c.cfl = float(self.mu), float(self.nu), float(self.Lambda), float(self.cfl)
        c.has_load = 0 if self.load_rate is None else 1
        rate = (0., 0., 0.) if self.load_rate is None else self.load_rate
        for a in range(3):
            c.load_rate[a] = float(rate[a])
            c.load_initial[a] = float(self.load_initial[a])
        c.load_t0 = float(self.load_t0)
        c.load_mu = float(self.mu if self.load_mu is None else self.load_mu)
        c.load_nu = float(self.nu if self.load_nu is None else self.load_nu)
        c.dynamics = _lib.CDD_DYN_GLIDE_ONLY if self.glide_only else _lib.CDD_DYN_GLIDE_CLIMB
        c.vacancy = 0 if self.vacancy is None else 1
        if self.vacancy is not None:
            c.vac_alpha, c.vac_beta, c.vac_gamma = (float(v) for v in self.vacancy)
        c.dt_max = float(self.dt_max)
        return c

    @property
    def cells(self):
        return int(np.prod(self.shape))


def _stream(stream=None):
    if stream is None:
        stream = torch.cuda.current_stream()
    return ctypes.c_void_p(stream.cuda_stream)


class Plan:
    """A batch of instances at one precision ("f64" or "f32") on the current CUDA device.

    tuning: None (built-in launch shapes), a list with one dict per instance (keys of
    ``_lib.cdd_tuning``: fft_radix, rows_lines, mid_cols, green_cols, stencil_planes; missing or 0
    keeps the built-in rule), or "auto" (``cdd.autotune`` picks them by timing, cached per GPU,
    precision and shape).
    """

    def __init__(self, instances, precision="f64", device=None, tuning=None):
        if isinstance(instances, Instance):
            instances = [instances]
        self.instances = list(instances)
        if precision not in ("f64", "f32"):
            raise ValueError("precision must be 'f64' or 'f32'")
        self.precision = precision
        self.dtype = torch.float64 if precision == "f64" else torch.float32
        if not torch.cuda.is_available():
            raise RuntimeError("cdd.Plan needs a CUDA device (sm_100a)")
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        self.lib = _lib.load()
        arr = (_lib.cdd_instance * len(self.instances))(*[i.to_c() for i in self.instances])
        n = len(self.instances)
        if isinstance(tuning, str):
            if tuning != "auto":
                raise ValueError("tuning must be None, a list of dicts or 'auto'")
            from . import autotune
            with torch.cuda.device(self.device):
                tuning = [autotune.best(inst, precision) for inst in self.instances]
        tune = None
        if tuning is not None:
            if len(tuning) != n:
                raise ValueError("tuning needs one entry per instance")
            tune = (_lib.cdd_tuning * n)(*[_lib.cdd_tuning.from_dict(t) for t in tuning])
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            check(self.lib.cdd_plan_create_tuned(arr, n, _lib.CDD_F64 if precision == "f64" else _lib.CDD_F32,
                                                 tune, ctypes.byref(h)))
        self.handle = h
        self.field_elems = int(self.lib.cdd_plan_field_elems(h))
        self.stress_elems = int(self.lib.cdd_plan_stress_elems(h))
        self.field_offsets = [int(self.lib.cdd_plan_field_offset(h, i)) for i in range(n)]
        self.stress_offsets = [int(self.lib.cdd_plan_stress_offset(h, i)) for i in range(n)]
        self.cells = [int(self.lib.cdd_plan_cells(h, i)) for i in range(n)]
        self.total_cells = int(self.lib.cdd_plan_cells(h, -1))
        self.scratch_bytes = int(self.lib.cdd_plan_scratch_bytes(h))

    def tuning(self, i=0):
        """The launch shapes instance i runs with (dict)."""
        t = _lib.cdd_tuning()
        check(self.lib.cdd_plan_tuning(self.handle, int(i), ctypes.byref(t)))
        return t.to_dict()

    # ------------------------------------------------------------------ lifetime
    def close(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            self.lib.cdd_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------------ buffers
    def empty_field(self):
        return torch.empty(self.field_elems, dtype=self.dtype, device=self.device)

    def empty_stress(self):
        return torch.empty(self.stress_elems, dtype=self.dtype, device=self.device)

    def field_view(self, buf, i):
        inst = self.instances[i]
        o = self.field_offsets[i]
        return buf[o:o + 9 * self.cells[i]].view((9,) + tuple(inst.shape))

    def stress_view(self, buf, i):
        inst = self.instances[i]
        o = self.stress_offsets[i]
        return buf[o:o + 6 * self.cells[i]].view((6,) + tuple(inst.shape))

    def pack(self, arrays):
        """Copy a list of (9,)+shape arrays (numpy or torch) into a new packed device field."""
        buf = self.empty_field()
        for i, a in enumerate(arrays):
            t = torch.as_tensor(np.ascontiguousarray(a) if isinstance(a, np.ndarray) else a)
            self.field_view(buf, i).copy_(t.to(self.dtype))
        return buf

    def unpack(self, buf):
        return [self.field_view(buf, i).detach().cpu().numpy() for i in range(len(self.instances))]

    def _check_field(self, buf, name="beta"):
        if not isinstance(buf, torch.Tensor) or buf.dtype != self.dtype or not buf.is_cuda \
                or not buf.is_contiguous() or buf.numel() != self.field_elems:
            raise ValueError("%s must be a contiguous %s CUDA tensor of %d elements"
                             % (name, self.dtype, self.field_elems))

    # ------------------------------------------------------------------ operators
    def stress(self, beta, out=None, stream=None):
        """Internal stress (6 symmetric components per instance) of a packed field."""
        self._check_field(beta)
        out = self.empty_stress() if out is None else out
        check(self.lib.cdd_stress(self.handle, ctypes.c_void_p(beta.data_ptr()),
                                  ctypes.c_void_p(out.data_ptr()), _stream(stream)))
        return out

    def flux(self, beta, t=0.0, want_speed=True, stream=None, sigma=None, out=None):
        """(rhs, speed) of the central-upwind flux at time t; speed is one value per cell.
        sigma: a packed 6-component internal stress to use instead of computing it (the applied
        load of time t is still added); out: a packed field to write rhs into."""
        self._check_field(beta)
        rhs = self.empty_field() if out is None else out
        speed = torch.empty(self.total_cells, dtype=self.dtype, device=self.device) if want_speed else None
        sp = ctypes.c_void_p(speed.data_ptr() if speed is not None else 0)
        if sigma is None:
            check(self.lib.cdd_flux(self.handle, ctypes.c_void_p(beta.data_ptr()), float(t),
                                    ctypes.c_void_p(rhs.data_ptr()), sp, _stream(stream)))
        else:
            if sigma.numel() != self.stress_elems or sigma.dtype != self.dtype:
                raise ValueError("sigma must be a packed stress of this plan")
            check(self.lib.cdd_flux_with_stress(self.handle, ctypes.c_void_p(beta.data_ptr()),
                                                ctypes.c_void_p(sigma.data_ptr()), float(t),
                                                ctypes.c_void_p(rhs.data_ptr()), sp, _stream(stream)))
        return rhs, speed

    def set_time(self, t=None, t_end=None):
        n = len(self.instances)
        def arr(v):
            if v is None:
                return None
            v = np.broadcast_to(np.asarray(v, dtype=np.float64), (n,)).copy()
            return (ctypes.c_double * n)(*v)
        torch.cuda.current_stream().synchronize()
        check(self.lib.cdd_set_time(self.handle, arr(t), arr(t_end)))

    def get_time(self):
        """(t, dt_last, active) arrays; synchronises."""
        n = len(self.instances)
        t = (ctypes.c_double * n)()
        dt = (ctypes.c_double * n)()
        act = (ctypes.c_int * n)()
        torch.cuda.current_stream().synchronize()
        check(self.lib.cdd_get_time(self.handle, t, dt, act))
        return np.array(t[:]), np.array(dt[:]), np.array(act[:], dtype=bool)

    def step(self, beta, stream=None):
        self._check_field(beta)
        check(self.lib.cdd_step(self.handle, ctypes.c_void_p(beta.data_ptr()), _stream(stream)))

    def step_fixed(self, beta, dt, stream=None):
        self._check_field(beta)
        check(self.lib.cdd_step_fixed(self.handle, ctypes.c_void_p(beta.data_ptr()), float(dt),
                                      _stream(stream)))

    def run(self, beta, n_steps, graph=True, stream=None):
        self._check_field(beta)
        check(self.lib.cdd_run(self.handle, ctypes.c_void_p(beta.data_ptr()), int(n_steps),
                               1 if graph else 0, _stream(stream)))

    def observables(self, beta, stream=None):
        """(energy, mean_zz) arrays over instances, FP64; synchronises."""
        self._check_field(beta)
        n = len(self.instances)
        e = (ctypes.c_double * n)()
        m = (ctypes.c_double * n)()
        check(self.lib.cdd_observables(self.handle, ctypes.c_void_p(beta.data_ptr()), e, m,
                                       _stream(stream)))
        return np.array(e[:]), np.array(m[:])

    def check_status(self):
        torch.cuda.current_stream().synchronize()
        check(self.lib.cdd_check_status(self.handle))

    # ------------------------------------------------------------------ vacancy coupling
    def empty_vacancy(self):
        """A zeroed buffer of vacancy concentrations (one value per cell of every instance)."""
        return torch.zeros(self.field_elems // 9, dtype=self.dtype, device=self.device)

    def vacancy_view(self, buf, i):
        o = self.field_offsets[i] // 9
        return buf[o:o + self.cells[i]].view(tuple(self.instances[i].shape))

    def set_vacancy(self, c):
        """Register the vacancy-concentration buffer that later steps and fluxes read and update
        (None clears it)."""
        if c is not None and (not c.is_cuda or c.dtype != self.dtype or not c.is_contiguous()
                              or c.numel() != self.field_elems // 9):
            raise ValueError("c must be a contiguous %s CUDA tensor of %d elements" % (self.dtype, self.field_elems // 9))
        self._vacancy = c
        check(self.lib.cdd_set_vacancy(self.handle, ctypes.c_void_p(0 if c is None else c.data_ptr())))

    # ------------------------------------------------------------------ field observables
    # name -> (cdd_observable, components); see cdd_observe_field in include/cdd.h
    OBSERVABLES = {"beta_elastic": (_lib.CDD_OBS_BETA_ELASTIC, 9), "rotation": (_lib.CDD_OBS_ROTATION, 3),
                   "rodrigues": (_lib.CDD_OBS_RODRIGUES, 3), "rho": (_lib.CDD_OBS_RHO, 9),
                   "rodrigues_rho": (_lib.CDD_OBS_RODRIGUES_RHO, 3)}

    def observe(self, kind, beta, out=None, stream=None, sin_k=False):
        """A k-space field observable of every instance of beta: "beta_elastic" (9 components),
        "rotation" (3: xy, xz, yz of the antisymmetric part of beta^E), "rodrigues" (3: x, y, z,
        from beta^P), "rho" (9: the Nye density) or "rodrigues_rho" (3: the Rodrigues vector of
        the Nye density field passed as beta, i.e. what "rho" returns). sin_k: the reference's
        type 'sinK' k tables. Returns a packed buffer; ``observable_view`` gives instance i."""
        self._check_field(beta)
        code, nc = self.OBSERVABLES[kind]
        if sin_k:
            code |= _lib.CDD_OBS_SINK
        n = self.field_elems if nc == 9 else self.field_elems // 3
        if out is None:
            out = torch.empty(n, dtype=self.dtype, device=self.device)
        elif out.numel() != n or out.dtype != self.dtype or not out.is_contiguous():
            raise ValueError("out must be a contiguous %s tensor of %d elements" % (self.dtype, n))
        check(self.lib.cdd_observe_field(self.handle, code, ctypes.c_void_p(beta.data_ptr()),
                                         ctypes.c_void_p(out.data_ptr()), _stream(stream)))
        return out

    def observable_view(self, buf, i, kind):
        nc = self.OBSERVABLES[kind][1]
        o = self.field_offsets[i] * nc // 9
        return buf[o:o + nc * self.cells[i]].view((nc,) + tuple(self.instances[i].shape))

    # ------------------------------------------------------------------ reference file formats
    # The CUDA solver's files keep each of the 9 components with grid axis 0 fastest; see
    # include/cdd.h (cdd_field_export ... cdd_plas_read) for the .ics and .plas layouts.
    def _file_prec(self, precision):
        if precision is None:
            return _lib.CDD_F64 if self.dtype == torch.float64 else _lib.CDD_F32
        return {"f64": _lib.CDD_F64, "f32": _lib.CDD_F32}[precision]

    def export_field(self, beta, i=0, precision="f64", stream=None):
        """Instance i of beta in the files' layout: a device tensor of shape (9,) + the grid
        reversed (element [c, i2, i1, i0] = component c at (i0, i1, i2))."""
        self._check_field(beta)
        code = self._file_prec(precision)
        out = torch.empty((9,) + tuple(reversed(self.instances[i].shape)),
                          dtype=torch.float64 if code == _lib.CDD_F64 else torch.float32, device=self.device)
        check(self.lib.cdd_field_export(self.handle, int(i), ctypes.c_void_p(beta.data_ptr()),
                                        ctypes.c_void_p(out.data_ptr()), code, _stream(stream)))
        return out

    def import_field(self, src, beta, i=0, stream=None):
        """Write a contiguous CUDA tensor in the files' layout (9 * cells FP64 or FP32 values) into
        instance i of beta."""
        self._check_field(beta)
        if not src.is_cuda or not src.is_contiguous() or src.numel() != 9 * self.cells[i] \
                or src.dtype not in (torch.float64, torch.float32):
            raise ValueError("src must be a contiguous FP64/FP32 CUDA tensor of 9 * cells values")
        code = _lib.CDD_F64 if src.dtype == torch.float64 else _lib.CDD_F32
        check(self.lib.cdd_field_import(self.handle, int(i), ctypes.c_void_p(src.data_ptr()), code,
                                        ctypes.c_void_p(beta.data_ptr()), _stream(stream)))
        return beta

    def read_ics(self, path, beta=None, i=0, stream=None):
        """Load an .ics initial condition (float64) into instance i of beta (a new zero field when
        None); returns beta."""
        if beta is None:
            beta = torch.zeros(self.field_elems, dtype=self.dtype, device=self.device)
        self._check_field(beta)
        check(self.lib.cdd_ics_read(self.handle, int(i), os.fsencode(path), ctypes.c_void_p(beta.data_ptr()),
                                    _stream(stream)))
        return beta

    def write_ics(self, path, beta, i=0, stream=None):
        self._check_field(beta)
        check(self.lib.cdd_ics_write(self.handle, int(i), os.fsencode(path), ctypes.c_void_p(beta.data_ptr()),
                                     _stream(stream)))

    def append_plas(self, path, t, beta, i=0, precision=None, stream=None):
        """Append the frame (t, instance i of beta) to a .plas file in `precision` ("f64" or "f32";
        default: the plan's)."""
        self._check_field(beta)
        check(self.lib.cdd_plas_append(self.handle, int(i), os.fsencode(path), float(t),
                                       ctypes.c_void_p(beta.data_ptr()), self._file_prec(precision),
                                       _stream(stream)))

    def plas_frames(self, path, i=0, precision=None):
        n = ctypes.c_longlong(0)
        check(self.lib.cdd_plas_frames(self.handle, int(i), os.fsencode(path), self._file_prec(precision),
                                       ctypes.byref(n)))
        return int(n.value)

    def read_plas(self, path, beta=None, i=0, frame=-1, precision=None, stream=None):
        """Frame `frame` (negative: from the end) of a .plas file into instance i of beta (a new
        zero field when None); returns (t, beta)."""
        if beta is None:
            beta = torch.zeros(self.field_elems, dtype=self.dtype, device=self.device)
        self._check_field(beta)
        t = ctypes.c_double(0.0)
        check(self.lib.cdd_plas_read(self.handle, int(i), os.fsencode(path), self._file_prec(precision),
                                     int(frame), ctypes.byref(t), ctypes.c_void_p(beta.data_ptr()),
                                     _stream(stream)))
        return float(t.value), beta

    def restart_from_plas(self, path, beta=None, i=0, precision=None, stream=None):
        """Continue from the last frame of a .plas file, as the CUDA solver's restart does
        (plasticity.cu L107-123): instance i's field and clock are set from the frame. Returns
        (t, beta)."""
        t, beta = self.read_plas(path, beta, i, -1, precision, stream)
        tt, _, _ = self.get_time()
        tt[i] = t
        self.set_time(tt)
        return t, beta


def stress_to_tensor9(s6):
    """Expand (6,)+grid symmetric storage xx, xy, xz, yy, yz, zz to (9,)+grid."""
    idx = [0, 1, 2, 1, 3, 4, 2, 4, 5]
    return s6[idx]
