"""Glide-only beta^P dynamics of the central-upwind scheme (reference:
Plasticity/FieldDynamics/CentralUpwindHJBetaPGlideOnlyDynamics.py L10-262), computed by libcdd.so.

The dislocation velocity is the climb velocity projected so that it carries no climb
(BetaP3D_Velocity L152-201; 2-D BetaP2D_Velocity L96-129), then divided by |rho|; the Hamiltonian
has no Lambda term. ``BetaPDynamics(Dx=None, coreEnergy=0, coreEnergyLog=0)`` has the reference's
signature; ``CalculateFlux(time, state, CFLCondition)`` and the loading hook (``load_spec``, used
by RunPython-style subclasses) are those of the glide-and-climb module. Grids may be 2-D or 3-D.
"""
from Plasticity.FieldDynamics import engine
from Plasticity.FieldDynamics.CentralUpwindHJBetaPDynamics3D import BetaPDynamics as _BetaPDynamics


class BetaPDynamics(_BetaPDynamics):
    def __init__(self, Dx=None, coreEnergy=0, coreEnergyLog=0):
        _BetaPDynamics.__init__(self, Dx=Dx, Lambda=0, coreEnergy=coreEnergy, coreEnergyLog=coreEnergyLog)

    def plan(self, state, cfl=0.25):
        if self.Dx is not None and abs(self.Dx - 1.0 / state.gridShape[-1]) > 1e-15 * self.Dx:
            raise NotImplementedError("the GPU path uses Dx = 1/gridShape[-1]")
        return engine.plan_for(state.gridShape, state.mu, state.nu, 0.0, cfl, self.load_spec(state), glide=True)
