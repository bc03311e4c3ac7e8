"""beta^P dynamics of the central-upwind scheme (reference:
Plasticity/FieldDynamics/CentralUpwindHJBetaPDynamics3D.py L10-221), computed by libcdd.so.

``BetaPDynamics(Lambda=0)`` is glide and climb; Lambda != 0 adds the glide projection
(L126-133, L195-200). ``CalculateFlux(time, state, CFLCondition)`` returns the rhs TensorField
and, with CFLCondition, the per-cell wave speed a_tot + b_tot (+ c_tot).
"""
import numpy

from Plasticity.FieldDynamics.CentralUpwindHJ3D import CentralUpwindHJDynamics
from Plasticity.FieldDynamics import engine
from Plasticity.Fields import Fields
from Plasticity.GridArray import GridArray


class BetaPDynamics(CentralUpwindHJDynamics):
    def __init__(self, Dx=None, Lambda=0, coreEnergy=0, coreEnergyLog=0):
        self.Dx = Dx
        self.Lambda = Lambda
        self.coreEnergy = coreEnergy
        self.coreEnergyLog = coreEnergyLog
        self.counter = 0
        self.prevTimeStep = False
        self.time = None
        self.vtime = None
        self.velocity = {}

    # loading: subclasses return (rate[3], initial[3], t0, load_mu, load_nu)
    def load_spec(self, state):
        return None

    def plan(self, state, cfl=0.25):
        if self.Dx is not None and abs(self.Dx - 1.0 / state.gridShape[-1]) > 1e-15 * self.Dx:
            raise NotImplementedError("the GPU path uses Dx = 1/gridShape[-1]")
        return engine.plan_for(state.gridShape, state.mu, state.nu, self.Lambda, cfl, self.load_spec(state))

    def GetSigma(self, state, time):
        return state.CalculateSigma()

    def CalculateFlux(self, time, state, CFLCondition=False):
        self.state = state
        self.time = time
        p = self.plan(state)
        beta = p.pack_state(state)
        rhs, speed = p.flux(beta, time, want_speed=CFLCondition)
        rhs_f = Fields.from_stack(state.gridShape, p.field_view(rhs, 0).double().cpu().numpy())
        if CFLCondition:
            sp = GridArray.GridArray(speed.double().cpu().numpy().reshape(state.gridShape))
            return rhs_f, sp
        return rhs_f
