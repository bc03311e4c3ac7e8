"""Adjoint of the CDD step: transposed stress operator, nu-derivative, flux VJP and the checkpointed
rollout gradient, against the dot-product identity, finite differences and torch autograd through a
plain-torch FP64 restatement of the step (tests/torch_ref.py)."""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import cdd
from cdd import _lib
from cdd.adjoint import Rollout, RolloutLoss, CZZ
from cdd.engine import _stream
import torch_ref as R


def P(t):
    return ctypes.c_void_p(t.data_ptr())


def rel(a, b):
    a = torch.as_tensor(a).double().cpu()
    b = torch.as_tensor(b).double().cpu()
    return float((a - b).norm() / b.norm())


@pytest.mark.parametrize("shape", [(12, 16, 20), (16, 24), (24, 12, 8)])
def test_stress_adjoint_dot_product(shape):
    plan = cdd.Plan([cdd.Instance(shape)], "f64")
    x = plan.pack([cdd.gaussian_random_field(shape, 0.08, 0.05, 1)])
    y = torch.randn(plan.stress_elems, dtype=torch.float64, device=plan.device)
    Sx = plan.stress(x)
    STy = plan.empty_field()
    _lib.check(plan.lib.cdd_stress_adjoint(plan.handle, P(y), P(STy), _stream()))
    lhs = float((Sx * y).sum())
    rhs = float((x * STy).sum())
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_stress_dnu_matches_finite_difference():
    shape = (12, 12, 16)
    b = cdd.gaussian_random_field(shape, 0.06, 0.05, 2)
    h = 1e-6
    out = {}
    for nu in (0.3 - h, 0.3 + h, 0.3):
        plan = cdd.Plan([cdd.Instance(shape, mu=1.3, nu=nu)], "f64")
        beta = plan.pack([b])
        out[nu] = (plan, beta, plan.stress(beta))
    fd = (out[0.3 + h][2] - out[0.3 - h][2]) / (2 * h)
    plan, beta, _ = out[0.3]
    d = plan.empty_stress()
    _lib.check(plan.lib.cdd_stress_dnu(plan.handle, P(beta), P(d), _stream()))
    assert rel(d, fd) < 1e-8


@pytest.mark.parametrize("shape,Lambda,rate", [((12, 12, 12), 0.0, 0.05), ((16, 16), 0.0, None),
                                               ((10, 12, 8), 1.0, 0.03)])
def test_flux_vjp_matches_torch_autograd(shape, Lambda, rate):
    b0 = cdd.gaussian_random_field(shape, 0.07, 0.05, 3)
    t = 0.7
    load = None if rate is None else tuple(rate * CZZ)
    plan = cdd.Plan([cdd.Instance(shape, mu=1.0, nu=0.3, Lambda=Lambda, load_rate=load)], "f64")
    beta = plan.pack([b0])
    g = torch.randn(plan.field_elems, dtype=torch.float64, device=plan.device)
    vb = plan.empty_field()
    sb = plan.empty_stress()
    lb = torch.zeros(3, dtype=torch.float64, device=plan.device)
    _lib.check(plan.lib.cdd_flux_vjp(plan.handle, P(beta), ctypes.c_double(t), P(g), P(vb), P(sb), P(lb),
                                     _stream()))
    bt = torch.tensor(b0, dtype=torch.float64, device=plan.device, requires_grad=True)
    rz = None if rate is None else torch.tensor(rate, dtype=torch.float64, device=plan.device)
    rhs = R.flux(bt, R.total_stress(bt, t, 1.0, 0.3, rz), Lambda)
    (gt,) = torch.autograd.grad(rhs, bt, grad_outputs=plan.field_view(g, 0))
    assert rel(plan.field_view(vb, 0), gt) < 1e-10
    plan.check_status()


def _rollout_torch(b0, mu, nu, rz, dt, n):
    u = b0
    for k in range(n):
        u = R.step_fixed(u, k * dt, dt, mu, nu, rz)
    return R.loss(u, mu, nu)


def test_rollout_gradient_matches_torch_autograd():
    shape = (10, 12, 12)
    b0 = cdd.gaussian_random_field(shape, 0.06, 0.05, 4)
    mu, nu, r, dt, n = 1.1, 0.28, 0.05, 2e-3, 4
    ro = Rollout(shape, mu, nu, r, dt, n, precision="f64", checkpoint_every=3)
    beta = ro.plan.pack([b0])
    _, loss = ro.forward(beta)
    gb, grads = ro.backward()
    dev = ro.plan.device
    bt = torch.tensor(b0, dtype=torch.float64, device=dev, requires_grad=True)
    mt = torch.tensor(mu, dtype=torch.float64, device=dev, requires_grad=True)
    nt = torch.tensor(nu, dtype=torch.float64, device=dev, requires_grad=True)
    rt = torch.tensor(r, dtype=torch.float64, device=dev, requires_grad=True)
    L = _rollout_torch(bt, mt, nt, rt, dt, n)
    L.backward()
    assert abs(loss - float(L.detach())) <= 1e-10 * abs(float(L.detach()))
    assert rel(ro.plan.field_view(gb, 0), bt.grad) < 1e-9
    for name, t in (("mu", mt), ("nu", nt), ("rate_zz", rt)):
        assert abs(grads[name] - float(t.grad)) <= 1e-8 * max(abs(float(t.grad)), 1e-12), name


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_rollout_overlapped_sweep_equals_serial(precision):
    """The overlapped reverse sweep (segment re-runs on a second stream with a second plan and a
    double buffer of records) gives bitwise the gradients of the serial sweep: 4 segments, so both
    record buffers are reused."""
    shape = (16, 16, 16)
    b0 = cdd.gaussian_random_field(shape, 0.06, 0.05, 8)
    out = []
    for overlap in (True, False):
        ro = Rollout(shape, 1.0, 0.3, 0.05, 2e-3, 7, precision=precision, checkpoint_every=2, overlap=overlap)
        _, loss = ro.forward(ro.plan.pack([b0]))
        gb, grads = ro.backward()
        out.append((loss, gb.clone(), grads))
    (la, ga, da), (lb, gbb, db) = out
    assert la == lb
    assert torch.equal(ga, gbb)
    assert da == db


def test_rollout_gradient_matches_finite_differences():
    """FP64 central differences at 32^3 with h = 1e-6 along 8 seeded random directions (unit-L2
    smooth random fields) and in mu, nu and the strain rate, over 5 RK3 steps at the fixed dt of the
    step-0 CFL. A direction is redrawn when the branch records (limiter selections and the corners
    attaining the speed maxima, cdd_flux_branches) of any of the 15 flux evaluations differ between
    the +h or -h trajectory and the unperturbed one -- the loss is only piecewise smooth -- or when
    it is nearly orthogonal to the gradient (|dJ| < 2e-3 |grad J|), where FP64 roundoff in J / h
    (about 3e-8) exceeds 1e-6 of the derivative."""
    shape = (32, 32, 32)
    b0 = cdd.gaussian_random_field(shape, 0.05, 0.05, 5)
    mu, nu, r, n = 1.0, 0.3, 0.05, 5
    probe = cdd.Plan([cdd.Instance(shape, mu=mu, nu=nu, load_rate=tuple(r * CZZ))], "f64")
    _, speed = probe.flux(probe.pack([b0]), 0.0)
    dt = 0.25 / (32 * float(speed.max()))            # fixed dt from the step-0 CFL
    ro = Rollout(shape, mu, nu, r, dt, n, precision="f64", checkpoint_every=2)
    T0 = ro.branch_trace(ro.plan.pack([b0]))
    ro.forward(ro.plan.pack([b0]))
    gb, grads = ro.backward()
    g = ro.plan.field_view(gb, 0).cpu().numpy()
    gnorm = float(np.linalg.norm(g))

    def J(b=b0, m=mu, v=nu, rr=r):
        ro2 = Rollout(shape, m, v, rr, dt, n, precision="f64", checkpoint_every=n)
        beta = ro2.plan.pack([b])
        flips = int((ro2.branch_trace(beta) != T0).sum())
        return ro2.forward(beta)[1], flips

    h = 1e-6
    rng = np.random.default_rng(11)
    checked = tries = 0
    while checked < 8 and tries < 40:
        tries += 1
        d = cdd.gaussian_random_field(shape, 0.05, 0.05, int(rng.integers(1 << 30)))
        d /= np.linalg.norm(d)
        ad = float((g * d).sum())
        if abs(ad) < 2e-3 * gnorm:
            continue
        (jp, fp), (jm, fm) = J(b0 + h * d), J(b0 - h * d)
        if fp or fm:
            continue                                  # a branch flipped inside [-h, h]: redraw
        fd = (jp - jm) / (2 * h)
        assert abs(ad - fd) <= 1e-6 * abs(fd), (ad, fd)
        checked += 1
    assert checked == 8, (checked, tries)
    for name, kw, val in (("mu", "m", mu), ("nu", "v", nu), ("rate_zz", "rr", r)):
        fd = (J(**{kw: val + h})[0] - J(**{kw: val - h})[0]) / (2 * h)
        assert abs(grads[name] - fd) <= 1e-6 * abs(fd), (name, grads[name], fd)


def test_branch_record_detects_limiter_flip():
    """cdd_flux_branches follows the minmod selections: a sine profile along the last axis with a
    -1e-3 or +1e-3 bump at one point selects differently next to the bump (numpy: the forward
    selections at x = 3..6 go 2,0,0,1 -> 1,2,1,2); a zero field records all zeros."""
    shape = (8, 8, 16)
    base = np.zeros((9,) + shape)
    x = np.arange(16.0)
    plan = cdd.Plan([cdd.Instance(shape)], "f64")
    recs = []
    for eps in (-1e-3, 0.0, 1e-3):
        b = base.copy()
        prof = 0.01 * np.sin(2 * np.pi * x / 16) + eps * (x == 5)
        b[0] = prof[None, None, :]
        b[4] = 0.5 * prof[None, None, :]
        beta = plan.pack([b])
        flags = torch.empty(4 * plan.total_cells, dtype=torch.int32, device=plan.device)
        _lib.check(plan.lib.cdd_flux_branches(plan.handle, P(beta), ctypes.c_double(0.0), P(flags), _stream()))
        recs.append(flags.cpu().numpy())
    assert (recs[0] != recs[2]).any()
    same = cdd.Plan([cdd.Instance(shape)], "f64")
    beta = same.pack([base])
    flags = torch.empty(4 * same.total_cells, dtype=torch.int32, device=same.device)
    _lib.check(same.lib.cdd_flux_branches(same.handle, P(beta), ctypes.c_double(0.0), P(flags), _stream()))
    # a zero field: every minmod returns 0 (selection 0), every corner speed is 0 (zero entry)
    assert int(flags.abs().sum()) == 0


def test_autograd_function_fp32_rollout():
    shape = (16, 16, 16)
    b0 = torch.tensor(cdd.gaussian_random_field(shape, 0.05, 0.05, 6).reshape(-1), device="cuda")
    b0.requires_grad_(True)
    mu = torch.tensor(1.0, dtype=torch.float64, device="cuda", requires_grad=True)
    nu = torch.tensor(0.3, dtype=torch.float64, device="cuda", requires_grad=True)
    rz = torch.tensor(0.05, dtype=torch.float64, device="cuda", requires_grad=True)
    loss = RolloutLoss.apply(b0, mu, nu, rz, shape, 1e-3, 6, "f32", 3)
    loss.backward()
    assert torch.isfinite(b0.grad).all() and float(b0.grad.abs().sum()) > 0
    # FP32 gradient against the FP64 one
    ro = Rollout(shape, 1.0, 0.3, 0.05, 1e-3, 6, precision="f64", checkpoint_every=3)
    ro.forward(b0.detach().double())
    g64, grads = ro.backward()
    assert rel(b0.grad, g64) < 1e-4
    assert abs(float(mu.grad) - grads["mu"]) <= 1e-4 * abs(grads["mu"])


def test_step_record_matches_fixed_step_bitwise():
    shape = (10, 24, 64)                      # TMA-staged planes in FP32 and FP64
    b0 = cdd.gaussian_random_field(shape, 0.06, 0.05, 7)
    for prec in ("f64", "f32"):
        plan = cdd.Plan([cdd.Instance(shape, mu=1.2, nu=0.27, load_rate=tuple(0.04 * CZZ))], prec)
        a = plan.pack([b0])
        b = a.clone()
        c = a.clone()
        plan.set_time(0.3, 1e300)
        plan.step_fixed(a, 1e-3)
        _lib.check(plan.lib.cdd_step_record(plan.handle, P(b), 0.3, 1e-3, None, _stream()))
        n = int(plan.lib.cdd_plan_record_elems(plan.handle))
        raw = torch.empty(n + 64, dtype=plan.dtype, device=plan.device)
        off = (-raw.data_ptr() % 256) // raw.element_size()
        rec = raw[off:off + n]
        _lib.check(plan.lib.cdd_step_record(plan.handle, P(c), 0.3, 1e-3, P(rec), _stream()))
        assert torch.equal(a, b) and torch.equal(a, c), prec
        assert torch.equal(rec[:plan.field_elems], plan.pack([b0]))   # the record starts with u


def test_batched_step_adjoint_matches_single_instances():
    """cdd_step_adjoint on a plan of two instances (different grids, materials and loads) equals
    the single-instance results, parameter cotangents per instance included."""
    specs = [((12, 16, 20), 1.0, 0.3, 0.05), ((16, 24), 1.3, 0.25, None)]
    fields = [cdd.gaussian_random_field(s, 0.06, 0.05, 10 + i) for i, (s, *_r) in enumerate(specs)]
    insts = [cdd.Instance(s, mu=m, nu=v, load_rate=None if r is None else tuple(r * CZZ)) for s, m, v, r in specs]

    def run(plan, arrays, seeds):
        u = plan.pack(arrays)
        n = int(plan.lib.cdd_plan_record_elems(plan.handle))
        raw = torch.empty(n + 64, dtype=plan.dtype, device=plan.device)
        off = (-raw.data_ptr() % 256) // raw.element_size()
        rec = raw[off:off + n]
        _lib.check(plan.lib.cdd_step_record(plan.handle, P(u), 0.2, 2e-3, P(rec), _stream()))
        ub = plan.pack(seeds)
        pbar = torch.zeros(_lib.CDD_PBAR * len(arrays), dtype=torch.float64, device=plan.device)
        _lib.check(plan.lib.cdd_step_adjoint(plan.handle, P(rec), 0.2, 2e-3, P(ub), P(pbar), _stream()))
        return [plan.field_view(ub, i).clone() for i in range(len(arrays))], pbar.view(len(arrays), -1)

    rng = np.random.default_rng(3)
    seeds = [rng.standard_normal((9,) + s) for s, *_r in specs]
    both, pb = run(cdd.Plan(insts, "f64"), fields, seeds)
    for i in range(2):
        one, pb1 = run(cdd.Plan([insts[i]], "f64"), [fields[i]], [seeds[i]])
        assert rel(both[i], one[0]) < 1e-13
        assert torch.allclose(pb[i], pb1[0], rtol=1e-12, atol=1e-14)
