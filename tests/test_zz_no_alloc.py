"""cdd_stress_noalloc: the stress solve for callers that cannot allocate device memory.

Such callers (a host that owns every device allocation, code inside a CUDA-graph capture region,
a service that must not allocate after start-up) cannot create a cdd_plan, so this entry point
keeps its scratch in a fixed array inside libcdd. The test calls it through the C ABI, twice in a
row on different inputs, and checks each result against cdd_stress (the plan path) within the
tolerances of the other stress tests: rel-L2 1e-13 in FP64, 1e-6 in FP32. This file sorts last
so that a run stopping at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import cdd
from cdd import _lib


def _rel(a, b):
    a = a.double()
    b = b.double()
    return float((a - b).norm() / b.norm())


@pytest.mark.parametrize("shape,precision,tol", [((32, 32, 32), "f64", 1e-13),
                                                 ((24, 40, 16), "f32", 1e-6),
                                                 ((64, 48), "f64", 1e-13)])
def test_noalloc_stress_matches_plan_stress_twice(shape, precision, tol):
    lib = _lib.load()
    inst = cdd.Instance(shape, mu=1.0, nu=0.3)
    plan = cdd.Plan([inst], precision)
    cinst = inst.to_c()
    prec = _lib.CDD_F64 if precision == "f64" else _lib.CDD_F32
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for seed in (11, 12):
        beta = plan.pack([cdd.gaussian_random_field(shape, 0.06, 0.05, seed)])
        ref = plan.stress(beta)
        out = torch.full_like(ref, float("nan"))
        rc = lib.cdd_stress_noalloc(ctypes.byref(cinst), prec, ctypes.c_void_p(beta.data_ptr()),
                                    ctypes.c_void_p(out.data_ptr()), stream)
        _lib.check(rc)
        torch.cuda.synchronize()
        assert torch.isfinite(out).all()
        assert _rel(out, ref) < tol


def test_noalloc_rejects_grid_larger_than_scratch():
    lib = _lib.load()
    inst = cdd.Instance((128, 128, 128)).to_c()
    rc = lib.cdd_stress_noalloc(ctypes.byref(inst), _lib.CDD_F64, ctypes.c_void_p(16), ctypes.c_void_p(16),
                                ctypes.c_void_p(0))
    assert rc == _lib.CDD_ERR_SHAPE
    msg = lib.cdd_last_error().decode()
    assert "scratch" in msg and str(32 << 20) in msg
