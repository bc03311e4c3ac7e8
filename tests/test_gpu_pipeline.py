"""cdd.HostPipeline: steps of host-resident fields with the copies overlapped, against the same steps
done serially (copy in, step, copy out on one stream)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import cdd

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec,depth", [("f32", 2), ("f64", 2), ("f32", 3)])
def test_pipeline_matches_serial_steps(prec, depth):
    from cdd.initial import gaussian_random_field
    shape = (32, 32, 32)
    inst = cdd.Instance(shape, load_rate=(-0.025, -0.025, 0.05))
    dt = torch.float32 if prec == "f32" else torch.float64
    inputs = [torch.as_tensor(gaussian_random_field(shape, 0.05, 0.05, 10 + k)).to(dt).reshape(-1).pin_memory()
              for k in range(5)]
    # serial reference: one buffer, one stream
    ref_plan = cdd.Plan([inst], prec)
    ref_plan.set_time(0.0, 1e30)
    buf = ref_plan.empty_field()
    want = []
    for h in inputs:
        buf.copy_(h)
        ref_plan.step(buf)
        want.append(buf.cpu().clone())
    plan = cdd.Plan([inst], prec)
    plan.set_time(0.0, 1e30)
    pipe = cdd.HostPipeline(plan, depth=depth)
    outs = [torch.empty_like(h).pin_memory() for h in inputs]
    for h, o in zip(inputs, outs):
        pipe.step(h, o)
    pipe.synchronize()
    for o, w in zip(outs, want):
        assert torch.equal(o, w)
    assert np.array_equal(plan.get_time()[0], ref_plan.get_time()[0])
    with pytest.raises(ValueError):
        pipe.step(inputs[0].cuda(), outs[0])
