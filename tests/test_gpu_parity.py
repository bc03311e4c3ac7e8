"""GPU parity of the CUDA path (libcdd.so through its C ABI) against the reference's golden vectors
and the CPU oracle.

Tolerances (FP64 form): stress and flux fields rel-L2 <= 1e-12, one step <= 1e-11, ten steps
<= 1e-10 (the drop-in bar), energy / mean-strain curves relative 1e-8 over full runs.
FP32 form: per-field rel-L2 <= 1e-5 after 10 steps against the FP64 form.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import cdd
import cdd_oracle as O
from conftest import golden_path

FIELD_CASES = ["g3d_16", "g2d_32", "g3d_aniso", "g3d_lambda", "g3d_load", "g2d_48_tend", "g3d_glide",
               "g2d_glide"]
T_END = {"g2d_48_tend": 0.004}


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def inst_of(g):
    lr = g["load_rate"]
    return cdd.Instance(shape=tuple(int(v) for v in g["shape"]), mu=float(g["mu"]), nu=float(g["nu"]),
                        Lambda=float(g["Lambda"]), cfl=float(g["cfl"]),
                        load_rate=tuple(lr) if np.any(lr) else None, glide_only=glide_of(g))


def glide_of(g):
    return bool(int(g["glide"])) if "glide" in g.files else False


def params_of(g):
    lr = g["load_rate"]
    return O.Params(mu=float(g["mu"]), nu=float(g["nu"]), Lambda=float(g["Lambda"]),
                    cfl=float(g["cfl"]), load_rate=lr if np.any(lr) else None, glide=glide_of(g))


SYM = [0, 1, 2, 4, 5, 8]   # xx xy xz yy yz zz in the 9-component order


@pytest.mark.parametrize("name", FIELD_CASES)
def test_stress_matches_reference(name):
    g = np.load(golden_path(name))
    plan = cdd.Plan([inst_of(g)], "f64")
    beta = plan.pack([g["beta0"]])
    s6 = plan.stress(beta)
    torch.cuda.synchronize()
    got = plan.stress_view(s6, 0).cpu().numpy()
    assert rel(got, g["sigma"][SYM]) < 1e-12


@pytest.mark.parametrize("name", FIELD_CASES)
def test_flux_matches_reference(name):
    g = np.load(golden_path(name))
    plan = cdd.Plan([inst_of(g)], "f64")
    beta = plan.pack([g["beta0"]])
    rhs, speed = plan.flux(beta, 0.0)
    torch.cuda.synchronize()
    assert rel(plan.field_view(rhs, 0).cpu().numpy(), g["rhs"]) < 1e-12
    assert rel(speed.cpu().numpy().reshape(g["speed"].shape), g["speed"]) < 1e-12


@pytest.mark.parametrize("name", FIELD_CASES)
def test_steps_match_reference(name):
    g = np.load(golden_path(name))
    plan = cdd.Plan([inst_of(g)], "f64")
    beta = plan.pack([g["beta0"]])
    plan.set_time(0.0, T_END.get(name, 1e30))
    plan.step(beta)
    t, dt, act = plan.get_time()
    assert abs(dt[0] - g["dts"][0]) <= 1e-12 * g["dts"][0]
    assert rel(plan.field_view(beta, 0).cpu().numpy(), g["beta1"]) < 1e-11
    for _ in range(int(g["steps"]) - 1):
        plan.step(beta)
    t, dt, act = plan.get_time()
    assert rel(plan.field_view(beta, 0).cpu().numpy(), g["beta_final"]) < 1e-10
    assert abs(t[0] - float(g["t_final"])) <= 1e-12 * float(g["t_final"])
    plan.check_status()


@pytest.mark.parametrize("name", ["c1_2d_128", "c2_3d_32"])
def test_observable_curves_full_run(name):
    """Energy and mean-strain curves over the whole run agree with the reference to 1e-8."""
    g = np.load(golden_path(name))
    shape = tuple(int(v) for v in g["shape"])
    b0 = cdd.gaussian_random_field(shape, float(g["sigma_f"]), 0.05, int(g["seed"]))
    plan = cdd.Plan([inst_of(g)], "f64")
    beta = plan.pack([b0])
    plan.set_time(0.0, 1e30)
    e, m = plan.observables(beta)
    energies, means = [e[0]], [m[0]]
    for _ in range(int(g["steps"])):
        plan.step(beta)
        e, m = plan.observables(beta)
        energies.append(e[0])
        means.append(m[0])
    t, _, _ = plan.get_time()
    np.testing.assert_allclose(energies, g["energy"], rtol=1e-8)
    np.testing.assert_allclose(means, g["mean_zz"], rtol=1e-8, atol=1e-14)
    assert abs(t[0] - float(g["t_final"])) <= 1e-10 * float(g["t_final"])
    fin = plan.field_view(beta, 0).cpu().numpy().reshape(9, -1)
    np.testing.assert_allclose((fin ** 2).sum(axis=1), g["final_sumsq"], rtol=1e-8)


def test_batched_plan_matches_single_plans_bitwise():
    names = ["g3d_16", "g2d_32", "g3d_aniso", "g3d_load"]
    gs = [np.load(golden_path(n)) for n in names]
    batch = cdd.Plan([inst_of(g) for g in gs], "f64")
    bb = batch.pack([g["beta0"] for g in gs])
    batch.set_time(0.0, 1e30)
    for _ in range(2):
        batch.step(bb)
    for i, g in enumerate(gs):
        single = cdd.Plan([inst_of(g)], "f64")
        bs = single.pack([g["beta0"]])
        single.set_time(0.0, 1e30)
        for _ in range(2):
            single.step(bs)
        assert torch.equal(batch.field_view(bb, i), single.field_view(bs, 0))


def test_graph_run_equals_eager_steps():
    g = np.load(golden_path("g3d_16"))
    p1 = cdd.Plan([inst_of(g)], "f64")
    p2 = cdd.Plan([inst_of(g)], "f64")
    b1 = p1.pack([g["beta0"]])
    b2 = p2.pack([g["beta0"]])
    p1.set_time(0.0, 1e30)
    p2.set_time(0.0, 1e30)
    p1.run(b1, 4, graph=True)
    for _ in range(4):
        p2.step(b2)
    torch.cuda.synchronize()
    assert torch.equal(b1, b2)
    assert np.array_equal(p1.get_time()[0], p2.get_time()[0])


@pytest.mark.parametrize("shape", [(24, 48, 20), (40, 12), (12, 10, 16), (96, 8)])
def test_mixed_radix_shapes_against_oracle(shape):
    b0 = cdd.gaussian_random_field(shape, 0.06, 0.05, 21)
    p = O.Params(mu=1.0, nu=0.3)
    plan = cdd.Plan([cdd.Instance(shape)], "f64")
    beta = plan.pack([b0])
    s6 = plan.stress(beta)
    torch.cuda.synchronize()
    assert rel(plan.stress_view(s6, 0).cpu().numpy(), O.stress(b0, 1.0, 0.3)[SYM]) < 1e-12
    plan.set_time(0.0, 1e30)
    plan.step(beta)
    ref, dt = O.rk3_step(b0, 0.0, 1e30, p)
    assert rel(plan.field_view(beta, 0).cpu().numpy(), ref) < 1e-11


def test_fixed_dt_step_against_oracle():
    g = np.load(golden_path("g3d_load"))
    p = params_of(g)
    plan = cdd.Plan([inst_of(g)], "f64")
    beta = plan.pack([g["beta0"]])
    plan.set_time(0.1, 1e30)
    plan.step_fixed(beta, 1.5e-3)
    ref, _ = O.rk3_step(g["beta0"], 0.1, 1e30, p, fixed_dt=1.5e-3)
    assert rel(plan.field_view(beta, 0).cpu().numpy(), ref) < 1e-11


def test_uniform_state_known_answer():
    shape = (8, 8, 8)
    m = np.arange(1, 10, dtype=float) * 0.01
    b0 = m.reshape(9, 1, 1, 1) * np.ones((9,) + shape)
    plan = cdd.Plan([cdd.Instance(shape)], "f64")
    beta = plan.pack([b0])
    rhs, speed = plan.flux(beta)
    s6 = plan.stress(beta)
    torch.cuda.synchronize()
    lamb = 2 * 0.3 / (1 - 0.6)
    M = m.reshape(3, 3)
    expect = (-lamb * np.trace(M) * np.eye(3) - (M + M.T)).reshape(9)[SYM]
    got = plan.stress_view(s6, 0).cpu().numpy().reshape(6, -1)
    np.testing.assert_allclose(got, np.repeat(expect[:, None], got.shape[1], axis=1), atol=1e-14)
    assert float(rhs.abs().max()) == 0.0
    np.testing.assert_allclose(speed.cpu().numpy(), 3 * O.ME)


def test_end_time_reached_then_inactive():
    g = np.load(golden_path("g2d_48_tend"))
    plan = cdd.Plan([inst_of(g)], "f64")
    beta = plan.pack([g["beta0"]])
    plan.set_time(0.0, 0.004)
    for _ in range(int(g["steps"])):
        plan.step(beta)
    t, dt, act = plan.get_time()
    assert t[0] == 0.004
    before = beta.clone()
    plan.step(beta)
    t2, dt2, act2 = plan.get_time()
    assert not act2[0] and dt2[0] == 0.0 and t2[0] == 0.004
    assert torch.equal(before, beta)


@pytest.mark.parametrize("prec,shape", [("f64", (12, 12, 12)), ("f32", (12, 12, 12)), ("f32", (8, 16, 48)),
                                        ("f64", (8, 16, 48)), ("f32", (16, 48))])
def test_nonfinite_state_is_reported_and_not_applied(prec, shape):
    """A NaN in the field reaches the CFL maximum (FP32: through the NaN-propagating corner-speed
    extremes) on thread-staged and TMA-staged planes: the step is not applied."""
    b0 = cdd.gaussian_random_field(shape, 0.06, 0.05, 3)
    b0[(4,) + tuple(3 for _ in shape)] = np.nan
    plan = cdd.Plan([cdd.Instance(shape)], prec)
    beta = plan.pack([b0])
    before = beta.clone()
    plan.set_time(0.0, 1e30)
    plan.step(beta)
    with pytest.raises(cdd.CDDError) as ei:
        plan.check_status()
    assert ei.value.code == 4
    assert torch.equal(torch.nan_to_num(before, nan=7.0), torch.nan_to_num(beta, nan=7.0))
    plan.check_status()   # cleared


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_nonfinite_stress_gives_nonfinite_speed(prec):
    """A NaN in the stress handed to the flux makes the corner velocities of that cell NaN; its CFL
    speed comes back non-finite and the other cells' speeds stay finite."""
    shape = (8, 16, 48)
    b0 = cdd.gaussian_random_field(shape, 0.06, 0.05, 5)
    plan = cdd.Plan([cdd.Instance(shape)], prec)
    beta = plan.pack([b0])
    s6 = plan.stress(beta)
    plan.stress_view(s6, 0)[1, 2, 5, 7] = float("nan")
    _, speed = plan.flux(beta, 0.0, sigma=s6)
    sp = speed.reshape(shape).cpu().numpy()
    assert not np.isfinite(sp[2, 5, 7])
    mask = np.ones(shape, dtype=bool)
    mask[2, 5, 7] = False
    assert np.isfinite(sp[mask]).all()


def test_fp32_form_error_against_fp64():
    shape = (32, 32, 32)
    b0 = cdd.gaussian_random_field(shape, 0.04, 0.05, 5)
    inst = cdd.Instance(shape, load_rate=(-0.025, -0.025, 0.05))
    p64 = cdd.Plan([inst], "f64")
    p32 = cdd.Plan([inst], "f32")
    b64 = p64.pack([b0])
    b32 = p32.pack([b0])
    for p in (p64, p32):
        p.set_time(0.0, 1e30)
    for _ in range(10):
        p64.step(b64)
        p32.step(b32)
    x64 = p64.field_view(b64, 0).cpu().numpy()
    x32 = p32.field_view(b32, 0).cpu().numpy().astype(np.float64)
    for c in range(9):
        assert rel(x32[c], x64[c]) < 1e-5, c
    e64, m64 = p64.observables(b64)
    e32, m32 = p32.observables(b32)
    assert abs(e32[0] - e64[0]) <= 1e-5 * abs(e64[0])
    assert abs(m32[0] - m64[0]) <= 1e-6 * max(abs(m64[0]), 1e-3)


@pytest.mark.parametrize("shape,load", [((12, 40, 72), None), ((10, 24, 64), (-0.025, -0.025, 0.05)),
                                        ((8, 18, 48), (-0.025, -0.025, 0.05)), ((18, 48), None),
                                        ((40, 64), (-0.025, -0.025, 0.05))])
def test_tma_staged_planes_against_oracle(shape, load):
    """Grids wide enough for the TMA plane path (x >= 40), 3-D and 2-D: edge tiles in x and y,
    partial last tiles (x 72 and 48, y 18: shifted back inside the grid), FP64."""
    b0 = cdd.gaussian_random_field(shape, 0.06, 0.05, 31)
    p = O.Params(mu=1.0, nu=0.3, load_rate=load)
    plan = cdd.Plan([cdd.Instance(shape, load_rate=load)], "f64")
    beta = plan.pack([b0])
    rhs, speed = plan.flux(beta, 0.0)
    ref_rhs, ref_speed = O.full_flux(b0, 0.0, p)
    torch.cuda.synchronize()
    assert rel(plan.field_view(rhs, 0).cpu().numpy(), ref_rhs) < 1e-12
    assert rel(speed.cpu().numpy().reshape(shape), ref_speed) < 1e-12
    plan.set_time(0.0, 1e30)
    plan.step(beta)
    ref, _ = O.rk3_step(b0, 0.0, 1e30, p)
    assert rel(plan.field_view(beta, 0).cpu().numpy(), ref) < 1e-11
    plan.check_status()


@pytest.mark.parametrize("shape,load", [((12, 40, 72), None), ((10, 20, 64), (-0.025, -0.025, 0.05)),
                                        ((8, 18, 48), (-0.025, -0.025, 0.05)), ((6, 12, 40), None),
                                        ((18, 48), None), ((36, 64), (-0.025, -0.025, 0.05))])
def test_tma_staged_planes_fp32_against_oracle(shape, load):
    """The FP32 stencil's TMA plane path (32 x 8 tiles of 256 threads): edge tiles, partial last
    tiles in x and y (y 20, 18, 12 and 36 are not multiples of 8: the last tile is shifted back
    inside the grid), 2-D grids, and the stage updates whose beta_n rows are prefetched into L2,
    against the FP64 oracle (FP32 rounding: 5e-6 rel-L2); a batch of the shapes equals the single
    plans bitwise."""
    b0 = cdd.gaussian_random_field(shape, 0.06, 0.05, 33)
    p = O.Params(mu=1.0, nu=0.3, load_rate=load)
    plan = cdd.Plan([cdd.Instance(shape, load_rate=load)], "f32")
    beta = plan.pack([b0])
    rhs, speed = plan.flux(beta, 0.0)
    ref_rhs, ref_speed = O.full_flux(b0, 0.0, p)
    torch.cuda.synchronize()
    assert rel(plan.field_view(rhs, 0).cpu().numpy().astype(np.float64), ref_rhs) < 5e-6
    assert rel(speed.cpu().numpy().reshape(shape).astype(np.float64), ref_speed) < 5e-6
    plan.set_time(0.0, 1e30)
    plan.step(beta)
    ref, _ = O.rk3_step(b0, 0.0, 1e30, p)
    assert rel(plan.field_view(beta, 0).cpu().numpy().astype(np.float64), ref) < 5e-6
    plan.check_status()


def test_fp32_tma_batch_of_partial_tiles_equals_single_plans():
    shapes = [(10, 20, 64), (8, 18, 48), (18, 48), (6, 12, 40)]
    fields = [cdd.gaussian_random_field(s, 0.06, 0.05, 50 + i) for i, s in enumerate(shapes)]
    insts = [cdd.Instance(s, load_rate=(-0.025, -0.025, 0.05)) for s in shapes]
    batch = cdd.Plan(insts, "f32")
    bb = batch.pack(fields)
    batch.set_time(0.0, 1e30)
    batch.run(bb, 3, graph=False)
    batch.check_status()
    for i in range(len(shapes)):
        single = cdd.Plan([insts[i]], "f32")
        bs = single.pack([fields[i]])
        single.set_time(0.0, 1e30)
        single.run(bs, 3, graph=False)
        assert torch.equal(batch.field_view(bb, i), single.field_view(bs, 0)), i


def test_tma_fp32_matches_fp64_and_batch_mixes_paths():
    """FP32 TMA path against FP64, and a batch mixing TMA-staged and thread-staged instances."""
    shapes = [(16, 24, 80), (12, 12, 12), (32, 32)]
    fields = [cdd.gaussian_random_field(s, 0.06, 0.05, 40 + i) for i, s in enumerate(shapes)]
    insts = [cdd.Instance(s) for s in shapes]
    p64 = cdd.Plan(insts, "f64")
    p32 = cdd.Plan(insts, "f32")
    b64 = p64.pack(fields)
    b32 = p32.pack(fields)
    for p in (p64, p32):
        p.set_time(0.0, 1e30)
    for _ in range(3):
        p64.step(b64)
        p32.step(b32)
    for i in range(len(shapes)):
        x64 = p64.field_view(b64, i).cpu().numpy()
        x32 = p32.field_view(b32, i).cpu().numpy().astype(np.float64)
        assert rel(x32, x64) < 2e-6, i
        single = cdd.Plan([insts[i]], "f64")
        bs = single.pack([fields[i]])
        single.set_time(0.0, 1e30)
        for _ in range(3):
            single.step(bs)
        assert torch.equal(single.field_view(bs, 0), p64.field_view(b64, i))
    p64.check_status()
    p32.check_status()


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_same_shape_runs_share_tensor_maps_and_overflow_to_thread_staging(prec):
    """Runs of consecutive same-shape instances share one 5-D tensor map (instance = 5th
    coordinate); past the plan's map budget (32 runs) instances fall back to thread-staged planes.
    Every instance equals its single-instance plan bitwise."""
    a, b = (4, 8, 40), (6, 8, 48)
    shapes = [a, a, a, b, a, a] + [a if k % 2 == 0 else b for k in range(34)]
    fields = [cdd.gaussian_random_field(s, 0.08, 0.05, 300 + i) for i, s in enumerate(shapes)]
    insts = [cdd.Instance(s, load_rate=(-0.025, -0.025, 0.05)) for s in shapes]
    batch = cdd.Plan(insts, prec)
    bb = batch.pack(fields)
    batch.set_time(0.0, 1e30)
    batch.run(bb, 2, graph=False)
    batch.check_status()
    for i in [0, 1, 2, 3, 4, 5, 6, 7, 36, 37, 38, 39]:
        single = cdd.Plan([insts[i]], prec)
        bs = single.pack([fields[i]])
        single.set_time(0.0, 1e30)
        single.run(bs, 2, graph=False)
        assert torch.equal(batch.field_view(bb, i), single.field_view(bs, 0)), i


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_flux_with_given_stress_equals_flux(prec):
    """cdd_flux_with_stress on the plan's own stress reproduces cdd_flux bitwise (load included);
    a scaled stress gives a different flux."""
    shape = (16, 24, 48)
    b0 = cdd.gaussian_random_field(shape, 0.05, 0.05, 9)
    plan = cdd.Plan([cdd.Instance(shape, load_rate=(-0.025, -0.025, 0.05))], prec)
    beta = plan.pack([b0])
    rhs, speed = plan.flux(beta, 0.3)
    s6 = plan.stress(beta)
    rhs2, speed2 = plan.flux(beta, 0.3, sigma=s6)
    assert torch.equal(rhs, rhs2) and torch.equal(speed, speed2)
    rhs3, _ = plan.flux(beta, 0.3, sigma=2 * s6)
    assert not torch.equal(rhs, rhs3)



@pytest.mark.parametrize("shape", [(32, 32, 32), (24, 16, 64), (64, 64)])
def test_glide_only_fp32_form_and_batched_with_glide_climb(shape):
    """Glide-only dynamics: FP32 form within 1e-5 of FP64 after 10 steps; a plan mixing a
    glide-only and a glide-and-climb instance gives each its single-plan result: bitwise for the
    glide-only one (same kernel variant), to rounding for the other (the mixed plan runs it in the
    variant compiled with the projection, whose instruction scheduling may contract differently)."""
    b0 = cdd.gaussian_random_field(shape, 0.05, 0.05, 13)
    glide = cdd.Instance(shape, load_rate=(-0.025, -0.025, 0.05), glide_only=True)
    out = {}
    for prec in ("f64", "f32"):
        plan = cdd.Plan([glide], prec)
        b = plan.pack([b0])
        plan.set_time(0.0, 1e30)
        plan.run(b, 10, graph=True)
        plan.check_status()
        out[prec] = plan.field_view(b, 0).double().cpu().numpy()
    for c in range(9):
        assert rel(out["f32"][c], out["f64"][c]) < 1e-5, c
    climb = cdd.Instance(shape, load_rate=(-0.025, -0.025, 0.05))
    mixed = cdd.Plan([glide, climb], "f64")
    bm = mixed.pack([b0, b0])
    mixed.set_time(0.0, 1e30)
    mixed.run(bm, 2, graph=False)
    for i, inst in enumerate((glide, climb)):
        single = cdd.Plan([inst], "f64")
        bs = single.pack([b0])
        single.set_time(0.0, 1e30)
        single.run(bs, 2, graph=False)
        if i == 0:
            assert torch.equal(mixed.field_view(bm, i), single.field_view(bs, 0))
        else:
            assert rel(mixed.field_view(bm, i).cpu().numpy(), single.field_view(bs, 0).cpu().numpy()) < 1e-13
    assert not torch.equal(mixed.field_view(bm, 0), mixed.field_view(bm, 1))


def test_adjoint_rejects_glide_only():
    import ctypes
    from cdd import _lib
    shape = (16, 16, 16)
    plan = cdd.Plan([cdd.Instance(shape, glide_only=True)], "f64")
    b = plan.pack([cdd.gaussian_random_field(shape, 0.05, 0.05, 1)])
    g = torch.zeros_like(b)
    vb, sb = plan.empty_field(), plan.empty_stress()
    P = lambda t: ctypes.c_void_p(t.data_ptr())
    rc = plan.lib.cdd_flux_vjp(plan.handle, P(b), ctypes.c_double(0.0), P(g), P(vb), P(sb), None, None)
    assert rc == _lib.CDD_ERR_UNSUPPORTED
    with pytest.raises(cdd.CDDError):
        cdd.Plan([cdd.Instance(shape, Lambda=1.0, glide_only=True)], "f64")


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_steps_are_deterministic(prec):
    """Two runs of the same plan from the same state are bitwise equal: every reduction (speed
    maxima, observable sums, the FP32 form's FP64 means, which one cluster of blocks per component
    adds in rank order) has a fixed order."""
    shapes = [(64, 64, 64), (48, 48), (16, 24, 80)]
    fields = [cdd.gaussian_random_field(s, 0.05, 0.05, 500 + i) for i, s in enumerate(shapes)]
    insts = [cdd.Instance(s, load_rate=(-0.025, -0.025, 0.05)) for s in shapes]
    outs = []
    for _ in range(2):
        plan = cdd.Plan(insts, prec)
        b = plan.pack(fields)
        plan.set_time(0.0, 1e30)
        plan.run(b, 3, graph=True)
        e, m = plan.observables(b)
        outs.append((b.clone(), np.asarray(e).copy(), np.asarray(m).copy(), plan.get_time()[0].copy()))
        plan.check_status()
    assert torch.equal(outs[0][0], outs[1][0])
    for k in (1, 2, 3):
        assert np.array_equal(outs[0][k], outs[1][k])
