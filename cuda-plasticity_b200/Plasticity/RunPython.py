"""Loading dynamics of the reference driver (Plasticity/RunPython.py L19-50).

``ExternalStrain`` adds sigma_ii += lamb tr(eps) + 2 mu eps_i with the module-level mu = 0.5,
nu = 0.3 (not the state's), exactly as the reference does; ``UpwindLoadingBetaPDynamics`` applies
eps = initial + rate (t - initT) at the step-start time of every stage. Its constructor forwards
(Dx, coreEnergy, coreEnergyLog) positionally to BetaPDynamics as the reference does, so the
glide projection Lambda it runs with is the ``coreEnergy`` argument (0 by default).
"""
import numpy

from Plasticity.Constants import x, y, z
from Plasticity.FieldDynamics import CentralUpwindHJBetaPDynamics

mu, nu = 0.5, 0.3
lamb = 2. * mu * nu / (1. - 2. * nu)


def ExternalStrain(sigma, primaryStrain):
    strains = {x: primaryStrain[0], y: primaryStrain[1], z: primaryStrain[2]}
    strain_trace = strains[x] + strains[y] + strains[z]
    for i in (x, y, z):
        sigma[i, i] += lamb * strain_trace + 2. * mu * strains[i]
    return sigma


def ExternalStress(sigma, primaryStress):
    for k, i in enumerate((x, y, z)):
        sigma[i, i] += primaryStress[k]
    return sigma


class UpwindLoadingBetaPDynamics(CentralUpwindHJBetaPDynamics.BetaPDynamics):
    def __init__(self, Dx=None, Lambda=0, coreEnergy=0, coreEnergyLog=0, rate=None, type='strain',
                 initial=numpy.array([0., 0., 0.]), initT=0.):
        CentralUpwindHJBetaPDynamics.BetaPDynamics.__init__(self, Dx, coreEnergy, coreEnergyLog)
        self.rate = rate
        self.type = type
        self.initial = initial
        self.initT = initT

    def load_spec(self, state):
        rate = numpy.zeros(3) if self.rate is None else numpy.asarray(self.rate, float)
        if self.type == 'strain':
            return (tuple(rate), tuple(numpy.asarray(self.initial, float)), float(self.initT), mu, nu)
        # stress loading: sigma_ii += s_i, i.e. unit 2 mu_L with lamb_L = 0
        return (tuple(rate), tuple(numpy.asarray(self.initial, float)), float(self.initT), 0.5, 0.0)

    def GetSigma(self, state, time):
        sigma = state.CalculateSigma()
        eps = self.initial + (numpy.zeros(3) if self.rate is None else self.rate) * (time - self.initT)
        if self.type == 'strain':
            return ExternalStrain(sigma, eps)
        return ExternalStress(sigma, eps)
