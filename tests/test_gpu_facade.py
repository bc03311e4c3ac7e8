"""The Plasticity facades drive the GPU path like the reference's own drivers do
(RunPython.py L131-256): PlasticitySystem + TVDRungeKutta_FieldMover + BetaPDynamics, compared
with the reference's golden vectors and the oracle."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import cdd_oracle as O
from conftest import golden_path

from Plasticity import PlasticitySystem
from Plasticity.Fields import Fields
from Plasticity.FieldMovers import FieldMover
from Plasticity.FieldDynamics import CentralUpwindHJBetaPDynamics3D, CentralUpwindHJBetaPDynamics
from Plasticity.FieldDynamics import CentralUpwindHJBetaPGlideOnlyDynamics
from Plasticity.FieldDynamics import engine
from Plasticity.PlasticityStates import PlasticityState
from Plasticity.Observers import Observer
from Plasticity import RunPython


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(b))


def state_of(g):
    shape = tuple(int(v) for v in g["shape"])
    st = PlasticityState.PlasticityState(shape, mu=float(g["mu"]), nu=float(g["nu"]))
    st.betaP = Fields.from_stack(shape, g["beta0"])
    return st


@pytest.mark.parametrize("name,module", [("g3d_16", CentralUpwindHJBetaPDynamics3D),
                                         ("g2d_32", CentralUpwindHJBetaPDynamics)])
def test_system_run_matches_reference(name, module):
    g = np.load(golden_path(name))
    st = state_of(g)
    recall = Observer.RecallStateObserver()
    times = []

    class Times(Observer.Observer):
        def Update(self, t, s):
            times.append(t)

    system = PlasticitySystem.PlasticitySystem(st.gridShape, st, FieldMover.TVDRungeKutta_FieldMover(CFLsafeFactor=0.25),
                                               module.BetaPDynamics(Lambda=0), [recall, Times()])
    # end a hair before the reference's final time: the summed dts differ in the last bits, and
    # the clamp to endTime then ends the run after exactly the reference's number of steps
    system.Run(startTime=0.0, endTime=float(g["t_final"]) * (1.0 - 1e-12))
    assert len(times) == int(g["steps"])
    np.testing.assert_allclose(np.diff([0.0] + times)[:-1], g["dts"][:-1], rtol=1e-11)
    assert rel(recall.state.betaP.stack(), g["beta_final"]) < 1e-10


def test_flux_sigma_energy_through_facades():
    g = np.load(golden_path("g2d_32"))
    st = state_of(g)
    dyn = CentralUpwindHJBetaPDynamics.BetaPDynamics()
    rhs, speed = dyn.CalculateFlux(0.0, st, CFLCondition=True)
    assert rel(rhs.stack(), g["rhs"]) < 1e-12
    assert rel(speed, g["speed"]) < 1e-12
    sig = st.CalculateSigma()
    assert rel(sig.stack(), g["sigma"]) < 1e-12
    e = float(np.sum(st.CalculateElasticEnergy()))
    assert abs(e - g["energy"][0]) <= 1e-12 * abs(g["energy"][0])


def test_loading_dynamics_uses_module_constants():
    """UpwindLoadingBetaPDynamics converts the applied strain with RunPython's mu=0.5, nu=0.3."""
    shape = (12, 12, 12)
    from cdd.initial import gaussian_random_field
    b0 = gaussian_random_field(shape, 0.06, 0.05, 9)
    st = PlasticityState.PlasticityState(shape, mu=1.0, nu=0.3)
    st.betaP = Fields.from_stack(shape, b0)
    rate = np.array([-0.025, -0.025, 0.05])
    dyn = RunPython.UpwindLoadingBetaPDynamics(rate=rate, initial=np.array([0.01, 0.0, 0.0]), initT=0.1)
    mover = FieldMover.TVDRungeKutta_FieldMover(CFLsafeFactor=0.25)
    s1, dt = mover.CalculateOneAdaptiveTimeStep(0.3, st, dyn, 10.0)
    p = O.Params(mu=1.0, nu=0.3, cfl=0.25, load_rate=rate, load_initial=(0.01, 0., 0.), load_t0=0.1,
                 load_mu=0.5, load_nu=0.3)
    ref, dt_ref = O.rk3_step(b0, 0.3, 10.0, p)
    assert abs(dt - dt_ref) <= 1e-12 * dt_ref
    assert rel(s1.betaP.stack(), ref) < 1e-11


def test_precision_switch_and_energy_observer():
    g = np.load(golden_path("g3d_16"))
    engine.set_precision("f32")
    try:
        st = state_of(g)
        mover = FieldMover.TVDRungeKutta_FieldMover(CFLsafeFactor=0.25)
        dyn = CentralUpwindHJBetaPDynamics3D.BetaPDynamics()
        watch = Observer.EnergyDownhillObserver()
        for _ in range(3):
            st, dt = mover.CalculateOneAdaptiveTimeStep(0.0, st, dyn, 1e30)
            watch.Update(0.0, st)
        assert watch.countTotal == 3
        ref = g["beta0"]
        p = O.Params(mu=1.0, nu=0.3, cfl=0.25)
        for _ in range(3):
            ref, _ = O.rk3_step(ref, 0.0, 1e30, p)
        assert rel(st.betaP.stack(), ref) < 1e-5
    finally:
        engine.set_precision("f64")



def test_glide_only_system_run_matches_reference():
    """The glide-only facade (CentralUpwindHJBetaPGlideOnlyDynamics.BetaPDynamics) over a 2-D run,
    against the reference's own glide-only golden vectors."""
    g = np.load(golden_path("g2d_glide"))
    st = state_of(g)
    dyn = CentralUpwindHJBetaPGlideOnlyDynamics.BetaPDynamics()
    rhs, speed = dyn.CalculateFlux(0.0, st, CFLCondition=True)
    assert rel(rhs.stack(), g["rhs"]) < 1e-12
    assert rel(np.asarray(speed), g["speed"]) < 1e-12
    recall = Observer.RecallStateObserver()
    system = PlasticitySystem.PlasticitySystem(st.gridShape, st, FieldMover.TVDRungeKutta_FieldMover(CFLsafeFactor=0.25),
                                               dyn, [recall])
    system.Run(startTime=0.0, endTime=float(g["t_final"]) * (1.0 - 1e-12))
    assert rel(recall.state.betaP.stack(), g["beta_final"]) < 1e-10


def test_runpython_style_start_from_gaussian_random_initializer():
    """A RunPython.py-style run (L141-161, L181-186, L216-255): the state comes from
    FieldInitializer.GaussianRandomInitializer(gridShape, lengthscale 0.2, seed) with the state
    class's default mu = 0.5, nu = 0.3, the 'gcd' method's 2-D module dynamics (Lambda = 0) and mover
    (CFL 0.1), and PlasticitySystem.Run over RunPython's first output interval [0, 0.01]; the result
    equals the oracle's steps of the same initial field."""
    from Plasticity.FieldInitializers import FieldInitializer
    gridShape = (32, 32)
    state = FieldInitializer.GaussianRandomInitializer(gridShape, 0.2, 3)
    b0 = state.betaP.stack()
    obs = Observer.RecallStateObserver()
    system = PlasticitySystem.PlasticitySystem(gridShape, state, FieldMover.TVDRungeKutta_FieldMover(CFLsafeFactor=0.1),
                                               CentralUpwindHJBetaPDynamics.BetaPDynamics(Lambda=0), [obs])
    system.Run(startTime=0.0, endTime=0.01)
    ref, t = O.run(b0, 0.0, 0.01, O.Params(mu=0.5, nu=0.3, cfl=0.1))
    assert abs(t - 0.01) < 1e-15
    assert rel(obs.state.betaP.stack(), ref) < 1e-10
