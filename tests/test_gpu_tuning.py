"""Launch-shape tuning (cdd_plan_create_tuned, cdd/autotune.py): every knob gives the built-in
plan's results to rounding, the plan reports the shapes it uses, and the autotuner returns and
caches a valid choice."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import cdd
from cdd import autotune


def rel(a, b):
    a = torch.as_tensor(a).double()
    b = torch.as_tensor(b).double()
    return float((a - b).norm() / b.norm())


TUNINGS = [dict(fft_radix=8), dict(fft_radix=4), dict(rows_lines=4), dict(mid_cols=4), dict(green_cols=1),
           dict(green_cols=8), dict(stencil_planes=2), dict(stencil_planes=8),
           dict(fft_radix=8, mid_cols=8, green_cols=2, stencil_planes=4)]


@pytest.mark.parametrize("shape", [(32, 48, 64), (48, 40, 80), (64, 96)])
@pytest.mark.parametrize("tune", TUNINGS)
def test_tuned_plan_matches_builtin(shape, tune):
    b0 = cdd.gaussian_random_field(shape, 0.05, 0.05, 21)
    inst = cdd.Instance(shape, load_rate=(-0.025, -0.025, 0.05))
    ref = cdd.Plan([inst], "f64")
    got = cdd.Plan([inst], "f64", tuning=[tune])
    eff = got.tuning(0)
    for k, v in tune.items():
        if k in ("mid_cols", "stencil_planes") and len(shape) == 2:
            continue
        assert eff[k] == v, (k, eff)
    br, bg = ref.pack([b0]), got.pack([b0])
    assert rel(got.stress(bg), ref.stress(br)) < 1e-12
    for p, b in ((ref, br), (got, bg)):
        p.set_time(0.0, 1e30)
        p.step(b)
        p.step(b)
    assert rel(bg, br) < 1e-11


def test_tuning_too_large_for_shared_memory_is_rejected():
    inst = cdd.Instance((256, 64, 64))
    with pytest.raises(cdd.CDDError) as ei:
        cdd.Plan([inst], "f64", tuning=[dict(green_cols=64)])
    assert ei.value.code == 1


def test_autotuner_returns_valid_cached_choice(tmp_path, monkeypatch):
    monkeypatch.setenv("CDD_TUNE_CACHE", str(tmp_path / "tune.json"))
    inst = cdd.Instance((32, 32, 32))
    t, ms, base_ms, tried = autotune.tune(inst, "f32", reps=3, sweeps=1)
    assert ms <= base_ms and len(tried) >= 5
    plan = cdd.Plan([inst], "f32", tuning="auto")
    cached = autotune.load_cache()
    assert len(cached) == 1
    (entry,) = cached.values()
    assert set(entry["tuning"]) == set(autotune.KNOBS)
    assert plan.tuning(0)["fft_radix"] == entry["tuning"]["fft_radix"]


def test_plans_with_different_shared_memory_needs_coexist():
    """The dynamic shared-memory limit is a property of each kernel function shared by all plans: a
    plan created later (smaller grid, 2-D) must not break an earlier one's launches."""
    specs = [((64, 64, 256), "f32"), ((16, 16, 16), "f32"), ((64, 128), "f32")]
    plans = [(cdd.Plan([cdd.Instance(s)], prec), s) for s, prec in specs]
    for plan, shape in plans:
        b = plan.pack([cdd.gaussian_random_field(shape, 0.05, 0.05, 3)])
        s6 = plan.stress(b)
        plan.set_time(0.0, 1e30)
        plan.step(b)
        torch.cuda.synchronize()
        assert torch.isfinite(s6).all() and torch.isfinite(b).all()
        plan.check_status()


@pytest.mark.parametrize("shape", [(16, 16, 16), (32, 24, 32), (24, 16, 64)])
@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_stencil_plane_chunks_do_not_change_results(shape, prec):
    """The planes each stencil block marches (thread-staged and TMA-staged) change only the work
    split: every cell runs the same code, so the fields agree bitwise."""
    b0 = cdd.gaussian_random_field(shape, 0.05, 0.05, 5)
    inst = cdd.Instance(shape, load_rate=(-0.025, -0.025, 0.05))
    outs = []
    for planes in (1, 3, 8):
        plan = cdd.Plan([inst], prec, tuning=[dict(stencil_planes=planes)])
        b = plan.pack([b0])
        plan.set_time(0.0, 1e30)
        plan.run(b, 2, graph=False)
        outs.append(b)
    assert torch.equal(outs[0], outs[1]) and torch.equal(outs[0], outs[2])
    assert torch.isfinite(outs[0]).all()
