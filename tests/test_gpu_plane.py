"""The fused plane passes of the FP32 stress solve (tuning plane_fft = 1; k_plane_fwd / k_plane_inv:
the contiguous-axis and axis-1 transforms of each z-plane in one cluster kernel each way, spectra
exchanged through distributed shared memory) against the separate row / axis-1 passes (the
built-in choice) and the CPU oracle, and the stage-2 forward pass that forms F0 = u + dt rhs in both."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import cdd
import cdd_oracle as O
from cdd import _lib

SYM = [0, 1, 2, 4, 5, 8]   # xx, xy, xz, yy, yz, zz of the oracle's 9-component stress
# (n0, n1, n2): n1 and the contiguous n2 powers of two the plane passes accept
SHAPES = [(16, 64, 128), (8, 128, 64), (32, 32, 256), (12, 64, 128)]


def _rel(a, b):
    a = torch.as_tensor(a).double().cpu()
    b = torch.as_tensor(b).double().cpu()
    return float((a - b).norm() / b.norm())


def _plan(shape, plane, load=True, prec="f32"):
    inst = cdd.Instance(shape, mu=1.0, nu=0.3, cfl=0.25, load_rate=(-0.025, -0.025, 0.05) if load else None)
    return cdd.Plan([inst], prec, tuning=[{"plane_fft": plane}])


@pytest.mark.parametrize("shape", SHAPES)
def test_plane_stress_matches_separate_passes_and_oracle(shape):
    b0 = cdd.gaussian_random_field(shape, 0.06, 0.05, 31)
    on, off = _plan(shape, 1), _plan(shape, -1)
    assert on.tuning(0)["plane_fft"] == 1 and off.tuning(0)["plane_fft"] == -1
    s_on = on.stress_view(on.stress(on.pack([b0])), 0)
    s_off = off.stress_view(off.stress(off.pack([b0])), 0)
    assert torch.isfinite(s_on).all()
    assert _rel(s_on, s_off) < 1e-6
    assert _rel(s_on, O.stress(b0, 1.0, 0.3)[SYM]) < 1e-5


@pytest.mark.parametrize("shape", SHAPES[:2])
def test_plane_steps_match_separate_passes_and_fp64(shape):
    b0 = cdd.gaussian_random_field(shape, 0.05, 0.05, 32)
    out = {}
    for key, plane, prec in (("on", 1, "f32"), ("off", -1, "f32"), ("f64", 0, "f64")):
        p = _plan(shape, plane, prec=prec)
        b = p.pack([b0])
        p.set_time(0.0, 1e30)
        p.run(b, 3, graph=True)
        p.check_status()
        out[key] = p.field_view(b, 0).double().cpu()
    assert _rel(out["on"], out["off"]) < 1e-5
    assert _rel(out["on"], out["f64"]) < 1e-5


def test_mixed_plan_runs_each_instance_like_its_single_plan():
    """A batch of plane-pass and separate-pass instances (3-D eligible, 3-D not eligible, 2-D): the
    separate passes skip the plane instances and the plane passes the others; every instance equals
    its single plan bitwise."""
    shapes = [(16, 64, 128), (24, 24, 24), (64, 64), (8, 128, 64)]
    insts = [cdd.Instance(sh, mu=1.0, nu=0.3, cfl=0.25) for sh in shapes]
    fields = [cdd.gaussian_random_field(sh, 0.06, 0.05, 40 + i) for i, sh in enumerate(shapes)]
    tun = [{"plane_fft": 1}, {}, {}, {"plane_fft": 1}]
    batch = cdd.Plan(insts, "f32", tuning=tun)
    assert [batch.tuning(i)["plane_fft"] for i in range(4)] == [1, -1, 0, 1]
    bb = batch.pack(fields)
    batch.set_time(0.0, 1e30)
    batch.run(bb, 2, graph=True)
    for i, inst in enumerate(insts):
        single = cdd.Plan([inst], "f32", tuning=[tun[i]])
        bs = single.pack([fields[i]])
        single.set_time(0.0, 1e30)
        single.run(bs, 2, graph=True)
        assert torch.equal(batch.field_view(bb, i), single.field_view(bs, 0)), shapes[i]


def test_plane_required_on_an_ineligible_shape_is_rejected():
    with pytest.raises(_lib.CDDError) as e:
        _plan((24, 24, 24), 1)
    assert e.value.code == _lib.CDD_ERR_ARG
    with pytest.raises(_lib.CDDError):
        _plan((16, 64, 128), 1, prec="f64")
