"""beta^P dynamics coupled to a vacancy concentration (reference:
Plasticity/FieldDynamics/VacancyDynamics.py L16-61), computed by libcdd.so.

The flux uses sigma_ii - alpha c (GetSigma L23-29); OperatorSplittingTVDRK_FieldMover advances
beta^P by TVD-RK3 and then c by c += beta d tr(beta^P) and exact diffusion with constant gamma,
all on the GPU in one step (cdd_instance.vacancy). The stress is that of the beta^P state the
reference's DecoupleState builds, with PlasticityState's default mu 0.5, nu 0.3.
"""
from Plasticity.FieldDynamics.CentralUpwindHJBetaPDynamics3D import BetaPDynamics
from Plasticity.FieldDynamics import engine
from Plasticity.Fields import Fields
from Plasticity.GridArray import GridArray

DECOUPLED_MU, DECOUPLED_NU = 0.5, 0.3   # PlasticityState defaults (VacancyState.DecoupleState)


class BetaP_VacancyDynamics(BetaPDynamics):
    def __init__(self, Dx=None, Lambda=0, coreEnergy=0, coreEnergyLog=0, gamma=1., alpha=1., beta=1.):
        BetaPDynamics.__init__(self, Dx, Lambda=Lambda, coreEnergy=coreEnergy, coreEnergyLog=coreEnergyLog)
        self.gamma = gamma
        self.alpha = alpha
        self.beta = beta

    def plan(self, state, cfl=0.25, dt_max=0.0):
        if self.Dx is not None and abs(self.Dx - 1.0 / state.gridShape[-1]) > 1e-15 * self.Dx:
            raise NotImplementedError("the GPU path uses Dx = 1/gridShape[-1]")
        return engine.plan_for(state.gridShape, DECOUPLED_MU, DECOUPLED_NU, self.Lambda, cfl, None,
                               vacancy=(self.alpha, self.beta, self.gamma), dt_max=dt_max or 0.0)

    def CalculateFlux(self, time, betaPstate, cfield, CFLCondition=False):
        """(rhs[, per-cell speed]) of beta^P with the concentration cfield (a grid array)."""
        import torch
        p = self.plan(betaPstate)
        beta = p.pack_state(betaPstate)
        c = torch.as_tensor(__import__('numpy').asarray(cfield, dtype='float64')).to(p.device, p.dtype).reshape(-1)
        full = p.empty_vacancy()
        full.copy_(c)
        p.set_vacancy(full)
        rhs, speed = p.flux(beta, time, want_speed=CFLCondition)
        p.set_vacancy(None)
        rhs_f = Fields.from_stack(betaPstate.gridShape, p.field_view(rhs, 0).double().cpu().numpy())
        if CFLCondition:
            return rhs_f, GridArray.GridArray(speed.double().cpu().numpy().reshape(betaPstate.gridShape))
        return rhs_f

    def CalculateVFlux(self, cfield, delta_c, dt, ktools):
        raise NotImplementedError("the concentration update runs inside the GPU step "
                                  "(OperatorSplittingTVDRK_FieldMover)")

    def DiffusionEvolution(self, cfield, timeStep, ktools):
        raise NotImplementedError("the diffusion runs inside the GPU step (OperatorSplittingTVDRK_FieldMover)")
