"""beta^P plus a vacancy concentration (reference: Plasticity/PlasticityStates/VacancyState.py L9-45).

The order-parameter field betaP_V has the components ('s', 's') (the concentration c) and the nine
of beta^P, in sorted order as the reference's TensorScalarMixedField. It is a view: reading or
assigning a component reads or assigns the state's beta^P or c. The concentration lives on the GPU
between steps of OperatorSplittingTVDRK_FieldMover, like beta^P.
"""
import numpy

from Plasticity.Fields import Fields
from Plasticity.GridArray import GridArray
from Plasticity.PlasticityStates import PlasticityState

S = ('s', 's')


class _MixedField:
    """betaP_V: ('s', 's') -> c, the other components -> beta^P."""

    def __init__(self, state):
        self.state = state
        self.components = [S] + list(Fields.TensorField(state.gridShape).components)

    def __getitem__(self, comp):
        return self.state.cfield if tuple(comp) == S else self.state.betaP[comp]

    def __setitem__(self, comp, value):
        if tuple(comp) == S:
            self.state.cfield = value
        else:
            self.state.betaP[comp] = value

    def stack(self, dtype=numpy.float64):
        return numpy.stack([numpy.asarray(self[c], dtype=dtype) for c in self.components])


class VacancyState(PlasticityState.PlasticityState):
    def __init__(self, gridShape, field=None, nu=0.3, mu=0.5, inherit=None, alpha=1.):
        self._c = numpy.zeros(tuple(gridShape))
        self._cdev = None
        self.alpha = getattr(inherit, "alpha", alpha) if inherit is not None else alpha
        PlasticityState.PlasticityState.__init__(self, gridShape, field=field, nu=nu, mu=mu, inherit=inherit)

    # ---------------------------------------------------------------- the concentration
    @property
    def cfield(self):
        if self._cdev is not None:
            self._c = self._cdev.detach().to('cpu', dtype=__import__('torch').float64).numpy().copy()
            self._cdev = None
        return GridArray.GridArray(self._c) if not isinstance(self._c, GridArray.GridArray) else self._c

    @cfield.setter
    def cfield(self, value):
        self._c = numpy.array(value, dtype=numpy.float64)
        self._cdev = None

    def cfield_device(self, dtype, device):
        """c as a tensor on the GPU (uploaded from the host when needed)."""
        import torch
        if self._cdev is None or self._cdev.dtype != dtype or self._cdev.device != device:
            src = self._cdev if self._cdev is not None else torch.as_tensor(numpy.asarray(self._c))
            self._cdev = src.to(device=device, dtype=dtype).contiguous()
        return self._cdev

    def _set_cdevice(self, tensor):
        self._cdev = tensor

    # ---------------------------------------------------------------- the reference's interface
    @property
    def betaP_V(self):
        return _MixedField(self)

    @betaP_V.setter
    def betaP_V(self, value):
        for comp in value.components:
            _MixedField(self)[comp] = value[comp]

    def GetOrderParameterField(self):
        return self.betaP_V

    def ExtractBetaPField(self):
        return self.betaP

    def DecoupleState(self):
        """(beta^P state with PlasticityState's default mu, nu, as the reference builds it; c)."""
        st = PlasticityState.PlasticityState(self.gridShape, field=self.ExtractBetaPField())
        return st, self.cfield

    def RecoupleState(self, betaPstate, cfield):
        self.betaP = betaPstate.betaP
        self.cfield = cfield

    def copy(self):
        s = VacancyState(self.gridShape, inherit=self)
        s.betaP = Fields.from_stack(self.gridShape, self.betaP.stack())
        s.cfield = numpy.array(self.cfield)
        return s
