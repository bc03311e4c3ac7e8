"""The benchmark's full size, 256^3: the FP64 stress against the oracle, and size-independent
properties the oracle cannot afford at this size (linearity of the stress operator, periodic
translation invariance of the flux, the uniform-field known answer, the FP32 form against FP64)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import cdd
import cdd_oracle as O

pytestmark = pytest.mark.gpu

N = 256
SHAPE = (N, N, N)


def rel(a, b):
    a, b = torch.as_tensor(a).double(), torch.as_tensor(b).double()
    return float(torch.linalg.norm(a - b) / torch.linalg.norm(b))


@pytest.fixture(scope="module")
def field():
    from cdd.initial import gaussian_random_field_torch
    return gaussian_random_field_torch(SHAPE, 0.03, 0.05, 100, device="cuda", dtype=torch.float64)


def test_stress_matches_oracle_at_full_size(field):
    plan = cdd.Plan([cdd.Instance(SHAPE, mu=1.0, nu=0.3)], "f64")
    s6 = plan.stress_view(plan.stress(plan.pack([field])), 0).cpu().numpy()
    want = O.stress(field.cpu().numpy(), 1.0, 0.3)
    idx = [0, 1, 2, 4, 5, 8]                 # xx xy xz yy yz zz of the 9-component oracle stress
    assert rel(s6, want[idx]) < 1e-12


def test_stress_is_linear(field):
    plan = cdd.Plan([cdd.Instance(SHAPE, mu=1.0, nu=0.3)], "f64")
    b1 = plan.pack([field])
    b2 = plan.pack([torch.roll(field, shifts=(3, -5, 7), dims=(1, 2, 3)).flip(0)])
    s1, s2 = plan.stress(b1).clone(), plan.stress(b2).clone()
    s12 = plan.stress(0.75 * b1 - 1.25 * b2)
    assert rel(s12, 0.75 * s1 - 1.25 * s2) < 1e-13


def test_flux_is_translation_invariant(field):
    inst = cdd.Instance(SHAPE, mu=1.0, nu=0.3, load_rate=(-0.025, -0.025, 0.05))
    plan = cdd.Plan([inst], "f64")
    rhs, speed = plan.flux(plan.pack([field]), 0.3)
    rhs = plan.field_view(rhs, 0).clone()
    speed = speed.view(SHAPE).clone()
    sh = (17, -33, 64)
    rhs2, speed2 = plan.flux(plan.pack([torch.roll(field, shifts=sh, dims=(1, 2, 3))]), 0.3)
    assert rel(plan.field_view(rhs2, 0), torch.roll(rhs, shifts=sh, dims=(1, 2, 3))) < 1e-11
    assert rel(speed2.view(SHAPE), torch.roll(speed, shifts=sh, dims=(0, 1, 2))) < 1e-11


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_uniform_field_known_answer(prec):
    """A uniform beta^P has no gradients: rhs = 0 and speed = 3 ME (CentralUpwindHJ3D.py L239-241)."""
    plan = cdd.Plan([cdd.Instance(SHAPE, mu=1.0, nu=0.3)], prec)
    b = torch.tensor([0.01, -0.02, 0.005, 0.003, 0.0, 0.007, -0.004, 0.002, -0.01], dtype=torch.float64)
    beta = plan.pack([b.view(9, 1, 1, 1).expand((9,) + SHAPE)])
    rhs, speed = plan.flux(beta, 0.0)
    assert not rhs.any()
    assert torch.all(speed == speed.new_tensor(3 * O.ME))


def test_fp32_form_within_tolerance_of_fp64(field):
    inst = cdd.Instance(SHAPE, mu=1.0, nu=0.3, load_rate=(-0.025, -0.025, 0.05))
    p64, p32 = cdd.Plan([inst], "f64"), cdd.Plan([inst], "f32")
    b64, b32 = p64.pack([field]), p32.pack([field])
    for p, b in ((p64, b64), (p32, b32)):
        p.set_time(0.0, 1e30)
        p.run(b, 2, graph=True)
    for c in range(9):
        assert rel(p32.field_view(b32, 0)[c], p64.field_view(b64, 0)[c]) < 1e-5
