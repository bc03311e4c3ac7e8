"""Base class of field dynamics (reference: Plasticity/FieldDynamics/FieldDynamics.py L6-14)."""


class FieldDynamics:
    def __init__(self, Lambda=0):
        self.Lambda = Lambda

    def GetSigma(self, state, time=None):
        return state.CalculateSigma()
