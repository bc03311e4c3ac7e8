"""cdd_stress_noalloc: the stress solve for callers that cannot allocate device memory.

Such callers (a host that owns every device allocation through its own allocator, a service that
must not allocate after start-up) cannot create a cdd_plan, so this entry point keeps its scratch
in a fixed array inside libcdd. The test calls it through the C ABI, twice in a row on different
inputs, and checks each result against cdd_stress (the plan path) within the tolerances of the
other stress tests (rel-L2 1e-13 in FP64, 1e-6 in FP32) and against the CPU oracle's stress
(rel-L2 1e-12 in FP64, 1e-5 in FP32). This file sorts last so that a run stopping at the first
failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import cdd
import cdd_oracle as O
from cdd import _lib


def _rel(a, b):
    a = a.double()
    b = b.double()
    return float((a - b).norm() / b.norm())


@pytest.mark.parametrize("shape,precision,tol,tol_oracle", [((32, 32, 32), "f64", 1e-13, 1e-12),
                                                            ((24, 40, 16), "f32", 1e-6, 1e-5),
                                                            ((64, 48), "f64", 1e-13, 1e-12)])
def test_noalloc_stress_matches_plan_stress_twice(shape, precision, tol, tol_oracle):
    lib = _lib.load()
    inst = cdd.Instance(shape, mu=1.0, nu=0.3)
    plan = cdd.Plan([inst], precision)
    cinst = inst.to_c()
    prec = _lib.CDD_F64 if precision == "f64" else _lib.CDD_F32
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    sym = [0, 1, 2, 4, 5, 8]   # xx, xy, xz, yy, yz, zz of the oracle's 9-component stress
    for seed in (11, 12):
        b0 = cdd.gaussian_random_field(shape, 0.06, 0.05, seed)
        beta = plan.pack([b0])
        ref = plan.stress(beta)
        out = torch.full_like(ref, float("nan"))
        rc = lib.cdd_stress_noalloc(ctypes.byref(cinst), prec, ctypes.c_void_p(beta.data_ptr()),
                                    ctypes.c_void_p(out.data_ptr()), stream)
        _lib.check(rc)
        torch.cuda.synchronize()
        assert torch.isfinite(out).all()
        assert _rel(out, ref) < tol
        want = torch.from_numpy(O.stress(b0, 1.0, 0.3)[sym])
        assert _rel(plan.stress_view(out, 0).cpu(), want) < tol_oracle


def test_noalloc_rejects_grid_larger_than_scratch():
    lib = _lib.load()
    inst = cdd.Instance((128, 128, 128)).to_c()
    rc = lib.cdd_stress_noalloc(ctypes.byref(inst), _lib.CDD_F64, ctypes.c_void_p(16), ctypes.c_void_p(16),
                                ctypes.c_void_p(0))
    assert rc == _lib.CDD_ERR_SHAPE
    msg = lib.cdd_last_error().decode()
    assert "scratch" in msg and str(32 << 20) in msg
