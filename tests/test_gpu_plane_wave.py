"""Known answers on the GPU: the stress of single Fourier modes against its closed form
(tests/plane_wave.py), at the benchmark's 256^3 and on mixed-radix and 2-D-like shapes, FP64 and
FP32 (the FP32 form's separate k = 0 path sees a zero mean here)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import cdd
import plane_wave as PW

SYM = [0, 1, 2, 4, 5, 8]


@pytest.mark.parametrize("shape,m", [((256, 256, 256), (3, -7, 11)), ((96, 40, 48), (5, 2, -9)),
                                     ((8, 128, 256), (1, 30, 64))])
@pytest.mark.parametrize("prec,tol", [("f64", 1e-12), ("f32", 2e-6)])
def test_stress_of_a_single_mode(shape, m, prec, tol):
    rng = np.random.default_rng(7)
    B = rng.standard_normal((3, 3))
    plan = cdd.Plan([cdd.Instance(shape, mu=1.1, nu=0.31)], prec)
    got = plan.stress_view(plan.stress(plan.pack([PW.field(shape, m, B)])), 0).double().cpu().numpy()
    want = PW.stress(shape, m, B, 1.1, 0.31)[SYM]
    assert np.abs(got - want).max() < tol * np.abs(want).max()
