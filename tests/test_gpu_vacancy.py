"""Vacancy-coupled dynamics on the GPU (cdd_instance.vacancy, cdd_set_vacancy): operator-splitting
steps against the reference's own BetaP_VacancyDynamics + OperatorSplittingTVDRK_FieldMover
(tests/golden/vacancy.npz) in FP64 and FP32, the flux against the oracle, CUDA graphs, mixed plans,
the step bound and the error paths."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import cdd
import cdd_oracle as O
from conftest import golden_path

pytestmark = pytest.mark.gpu

G = np.load(golden_path("vacancy"))
VAC = (float(G["alpha"]), float(G["beta"]), float(G["gamma"]))


def rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def inst_for(key):
    shape = G["beta0_" + key].shape[1:]
    return cdd.Instance(shape, mu=float(G["mu"]), nu=float(G["nu"]), cfl=float(G["cfl"]), vacancy=VAC,
                        dt_max=float(G["dt_bound_" + key]))


@pytest.mark.parametrize("key", ["3d", "2d"])
@pytest.mark.parametrize("prec,tol", [("f64", 1e-10), ("f32", 1e-5)])
def test_vacancy_steps_match_reference(key, prec, tol):
    plan = cdd.Plan([inst_for(key)], prec)
    beta = plan.pack([G["beta0_" + key]])
    c = plan.empty_vacancy()
    plan.vacancy_view(c, 0).copy_(torch.as_tensor(G["c0_" + key]))
    plan.set_vacancy(c)
    plan.set_time(0.0, 1e30)
    for k in range(3):
        plan.step(beta)
        dt = plan.get_time()[1][0]
        # dt = CFL / max speed: FP32 forms the speed in FP32 (the maximum and dt are FP64)
        assert abs(dt - G["dts_" + key][k]) <= (1e-12 if prec == "f64" else tol) * G["dts_" + key][k]
        assert rel(plan.field_view(beta, 0).cpu(), G["betas_" + key][k]) < tol
        assert rel(plan.vacancy_view(c, 0).cpu(), G["cs_" + key][k]) < tol
    plan.check_status()


def test_vacancy_flux_matches_oracle():
    key = "3d"
    p = O.Params(mu=float(G["mu"]), nu=float(G["nu"]), vacancy=VAC)
    plan = cdd.Plan([inst_for(key)], "f64")
    beta = plan.pack([G["beta0_" + key]])
    c = plan.empty_vacancy()
    plan.vacancy_view(c, 0).copy_(torch.as_tensor(G["c0_" + key]))
    plan.set_vacancy(c)
    rhs, speed = plan.flux(beta, 0.0)
    want, wspeed = O.vacancy_flux(G["beta0_" + key], G["c0_" + key], p)
    assert rel(plan.field_view(rhs, 0).cpu(), want) < 1e-12
    assert rel(speed.cpu().reshape(wspeed.shape), wspeed) < 1e-12


def test_graph_run_equals_steps_and_recaptures_on_new_buffer():
    key = "3d"
    inst = inst_for(key)
    outs = []
    for graph in (False, True):
        plan = cdd.Plan([inst], "f64")
        beta = plan.pack([G["beta0_" + key]])
        c = plan.empty_vacancy()
        plan.vacancy_view(c, 0).copy_(torch.as_tensor(G["c0_" + key]))
        plan.set_vacancy(c)
        plan.set_time(0.0, 1e30)
        plan.run(beta, 2, graph=graph)
        c_before = c.clone()
        c2 = c.clone()                       # a new buffer: the graph must read and update it from now on
        plan.set_vacancy(c2)
        plan.run(beta, 1, graph=graph)
        assert torch.equal(c, c_before)      # the old buffer is left alone
        assert not torch.equal(c2, c_before)
        outs.append((beta.clone(), c2.clone()))
    assert torch.equal(outs[0][0], outs[1][0]) and torch.equal(outs[0][1], outs[1][1])


def test_mixed_plan_gives_each_instance_its_single_result():
    key = "3d"
    plain = cdd.Instance((16, 16, 16), mu=1.0, nu=0.3, load_rate=(-0.025, -0.025, 0.05))
    from cdd.initial import gaussian_random_field
    b_plain = gaussian_random_field((16, 16, 16), 0.05, 0.05, 77)
    mixed = cdd.Plan([plain, inst_for(key)], "f64")
    bm = mixed.pack([b_plain, G["beta0_" + key]])
    cm = mixed.empty_vacancy()
    mixed.vacancy_view(cm, 1).copy_(torch.as_tensor(G["c0_" + key]))
    mixed.set_vacancy(cm)
    mixed.set_time(0.0, 1e30)
    mixed.run(bm, 2, graph=False)
    sp = cdd.Plan([plain], "f64")
    bp = sp.pack([b_plain])
    sp.set_time(0.0, 1e30)
    sp.run(bp, 2, graph=False)
    assert torch.equal(mixed.field_view(bm, 0), sp.field_view(bp, 0))
    sv = cdd.Plan([inst_for(key)], "f64")
    bv = sv.pack([G["beta0_" + key]])
    cv = sv.empty_vacancy()
    sv.vacancy_view(cv, 0).copy_(torch.as_tensor(G["c0_" + key]))
    sv.set_vacancy(cv)
    sv.set_time(0.0, 1e30)
    sv.run(bv, 2, graph=False)
    assert torch.equal(mixed.field_view(bm, 1), sv.field_view(bv, 0))
    assert torch.equal(mixed.vacancy_view(cm, 1), sv.vacancy_view(cv, 0))


def test_dt_max_bounds_the_adaptive_step():
    from cdd.initial import gaussian_random_field
    b0 = gaussian_random_field((16, 16, 16), 0.05, 0.05, 5)
    free = cdd.Plan([cdd.Instance((16, 16, 16))], "f64")
    bf = free.pack([b0])
    free.set_time(0.0, 1e30)
    free.step(bf)
    dt_free = free.get_time()[1][0]
    bounded = cdd.Plan([cdd.Instance((16, 16, 16), dt_max=0.5 * dt_free)], "f64")
    bb = bounded.pack([b0])
    bounded.set_time(0.0, 1e30)
    bounded.step(bb)
    assert bounded.get_time()[1][0] == 0.5 * dt_free


def test_vacancy_errors():
    plan = cdd.Plan([inst_for("3d")], "f64")
    beta = plan.pack([G["beta0_3d"]])
    with pytest.raises(cdd.CDDError):
        plan.step(beta)                      # no vacancy buffer registered
    with pytest.raises(cdd.CDDError):
        plan.flux(beta, 0.0)
    # the adjoint's record path rejects vacancy instances
    bad = cdd.Plan([cdd.Instance((8, 8, 8), mu=0.5, nu=0.3, vacancy=VAC)], "f64")
    rec = torch.zeros(int(bad.lib.cdd_plan_record_elems(bad.handle)) + 64, dtype=torch.float64, device="cuda")
    off = (-rec.data_ptr() % 256) // 8
    import ctypes
    rc = bad.lib.cdd_step_record(bad.handle, ctypes.c_void_p(bad.pack([G["beta0_3d"]]).data_ptr()), 0.0, 1e-3,
                                 ctypes.c_void_p(rec[off:].data_ptr()), ctypes.c_void_p(0))
    assert rc == 6   # CDD_ERR_UNSUPPORTED


@pytest.mark.parametrize("key", ["3d", "2d"])
def test_facade_operator_splitting_mover_matches_reference(key):
    """The reference's own API: VacancyState, BetaP_VacancyDynamics, OperatorSplittingTVDRK_FieldMover."""
    from Plasticity.PlasticityStates import VacancyState
    from Plasticity.FieldDynamics import VacancyDynamics
    from Plasticity.FieldMovers import FieldMover
    beta0 = G["beta0_" + key]
    shape = beta0.shape[1:]
    st = VacancyState.VacancyState(shape, mu=0.5, nu=0.3)
    for c, comp in enumerate(O.COMPONENTS):
        st.betaP_V[comp] = beta0[c].copy()
    st.betaP_V["s", "s"] = G["c0_" + key].copy()
    dyn = VacancyDynamics.BetaP_VacancyDynamics(alpha=VAC[0], beta=VAC[1], gamma=VAC[2])
    mover = FieldMover.OperatorSplittingTVDRK_FieldMover(CFLsafeFactor=float(G["cfl"]),
                                                        dtBound=float(G["dt_bound_" + key]))
    t = 0.0
    for k in range(3):
        st, dt = mover.CalculateOneAdaptiveTimeStep(t, st, dyn, 1e30)
        t += dt
        assert abs(dt - G["dts_" + key][k]) <= 1e-12 * G["dts_" + key][k]
        got = np.stack([np.asarray(st.betaP_V[comp]) for comp in O.COMPONENTS])
        assert rel(got, G["betas_" + key][k]) < 1e-10
        assert rel(np.asarray(st.betaP_V["s", "s"]), G["cs_" + key][k]) < 1e-10
