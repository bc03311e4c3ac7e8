"""Field observables on the GPU (cdd_observe_field): beta^E, rotation, Rodrigues vector and Nye
density against the reference's own PlasticityState methods (tests/golden/observables.npz) and the
oracle, FP64 and FP32, batched plans, and the facade methods."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import cdd
import cdd_oracle as O
from conftest import golden_path

pytestmark = pytest.mark.gpu

G = np.load(golden_path("observables"))
KEYS = ["c", "a", "2d"]


def rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def rot3(rot9):
    return np.stack([rot9[1], rot9[2], rot9[5]])


def observe_all(plan, beta, i):
    return {k: plan.observable_view(plan.observe(k, beta), i, k).cpu().numpy()
            for k in ("beta_elastic", "rotation", "rodrigues", "rho")}


@pytest.mark.parametrize("key", KEYS)
@pytest.mark.parametrize("prec,tol", [("f64", 1e-12), ("f32", 1e-5)])
def test_observables_match_reference(key, prec, tol):
    beta0 = G["beta_" + key]
    plan = cdd.Plan([cdd.Instance(beta0.shape[1:], mu=1.0, nu=0.3)], prec)
    got = observe_all(plan, plan.pack([beta0]), 0)
    assert rel(got["beta_elastic"], G["betaE_" + key]) < tol
    assert rel(got["rotation"], rot3(G["rot_" + key])) < tol
    assert rel(got["rodrigues"], G["rod_" + key]) < tol
    assert rel(got["rho"], G["rho_" + key]) < tol


def test_observables_large_noncubic_vs_oracle():
    from cdd.initial import gaussian_random_field
    shape = (64, 48, 32)
    beta0 = gaussian_random_field(shape, 0.05, 0.05, 9)
    plan = cdd.Plan([cdd.Instance(shape, mu=1.0, nu=0.3)], "f64")
    got = observe_all(plan, plan.pack([beta0]), 0)
    assert rel(got["beta_elastic"], O.beta_elastic(beta0, 1.0, 0.3)) < 1e-12
    assert rel(got["rotation"], rot3(O.rotation_field(beta0, 1.0, 0.3))) < 1e-12
    assert rel(got["rodrigues"], O.rodrigues(beta0)) < 1e-12
    assert rel(got["rho"], O.rho_fourier(beta0)) < 1e-12


def test_batched_plan_gives_each_instance_its_single_result():
    betas = [G["beta_" + k] for k in KEYS]
    insts = [cdd.Instance(b.shape[1:], mu=1.0, nu=0.3) for b in betas]
    batch = cdd.Plan(insts, "f64")
    bb = batch.pack(betas)
    for i, (inst, b) in enumerate(zip(insts, betas)):
        single = cdd.Plan([inst], "f64")
        want = observe_all(single, single.pack([b]), 0)
        got = observe_all(batch, bb, i)
        for k in want:
            assert np.array_equal(got[k], want[k]), (i, k)


def test_facade_observables():
    from Plasticity.Fields import Fields
    from Plasticity.PlasticityStates import PlasticityState
    beta0 = G["beta_c"]
    shape = beta0.shape[1:]
    st = PlasticityState.PlasticityState(shape, mu=1.0, nu=0.3)
    st.betaP = Fields.from_stack(shape, beta0)
    assert rel(st.CalculateBetaElastic().stack(), G["betaE_c"]) < 1e-12
    rot = st.CalculateRotationField().stack()
    assert rel(rot, G["rot_c"]) < 1e-12
    assert np.all(rot[[0, 4, 8]] == 0)
    rod = st.CalculateRotationRodrigues()
    assert rel(np.stack([np.asarray(rod[a]) for a in "xyz"]), G["rod_c"]) < 1e-12
    rodE = st.CalculateRotationRodrigues(source='betaE')
    r9 = G["rot_c"]
    assert rel(np.stack([np.asarray(rodE[a]) for a in "xyz"]), np.stack([r9[5], r9[6], r9[1]])) < 1e-12
    assert rel(st.CalculateRhoFourier().stack(), G["rho_c"]) < 1e-12


@pytest.mark.parametrize("key", KEYS)
@pytest.mark.parametrize("prec,tol", [("f64", 1e-12), ("f32", 1e-5)])
def test_sink_tables_and_rodrigues_from_rho_match_reference(key, prec, tol):
    """type 'sinK' (the sine k tables, CDD_OBS_SINK) for every observable, and the Rodrigues vector
    from the Nye density field (CDD_OBS_RODRIGUES_RHO, source 'rho') with both tables."""
    beta0 = G["beta_" + key]
    plan = cdd.Plan([cdd.Instance(beta0.shape[1:], mu=1.0, nu=0.3)], prec)
    beta = plan.pack([beta0])
    view = lambda kind, buf: plan.observable_view(buf, 0, kind).cpu().numpy()
    assert rel(view("beta_elastic", plan.observe("beta_elastic", beta, sin_k=True)), G["betaE_sink_" + key]) < tol
    assert rel(view("rotation", plan.observe("rotation", beta, sin_k=True)), rot3(G["rot_sink_" + key])) < tol
    assert rel(view("rodrigues", plan.observe("rodrigues", beta, sin_k=True)), G["rod_sink_" + key]) < tol
    assert rel(view("rho", plan.observe("rho", beta, sin_k=True)), G["rho_sink_" + key]) < tol
    for sink, tag in ((False, "rodrho_"), (True, "rodrho_sink_")):
        rho = plan.observe("rho", beta, sin_k=sink)
        got = view("rodrigues_rho", plan.observe("rodrigues_rho", rho, sin_k=sink))
        assert rel(got, G[tag + key]) < tol, (sink, rel(got, G[tag + key]))


def test_facade_sink_and_rho_source():
    from Plasticity.PlasticityStates import PlasticityState
    from Plasticity.Fields import Fields
    beta0 = G["beta_c"]
    st = PlasticityState.PlasticityState(beta0.shape[1:], mu=1.0, nu=0.3)
    st.betaP = Fields.from_stack(beta0.shape[1:], beta0)
    rod = st.CalculateRotationRodrigues(type='sinK', source='rho')
    assert rel(np.stack([np.asarray(rod[a]) for a in "xyz"]), G["rodrho_sink_c"]) < 1e-12
    rho = st.CalculateRhoFourier(type='sinK')
    assert rel(rho.stack(), G["rho_sink_c"]) < 1e-12
