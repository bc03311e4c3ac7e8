"""PlasticityState facade (reference: Plasticity/PlasticityStates/PlasticityState.py L19-551).

The plastic distortion lives on the GPU while a simulation runs and is copied to host
GridArrays when ``betaP`` is read. Reading ``betaP`` hands out the host arrays, which the caller
may modify in place, so the next GPU use re-uploads them. Stress and energy come from libcdd.
"""
import numpy

from Plasticity.Constants import x, y, z
from Plasticity.Fields import Fields
from Plasticity.GridArray import GridArray
from Plasticity.GridArray import FourierSpaceTools
from Plasticity import NumericalMethods

ME = NumericalMethods.ME
SYM6 = [('x', 'x'), ('x', 'y'), ('x', 'z'), ('y', 'y'), ('y', 'z'), ('z', 'z')]


class PlasticityState:
    """beta^P on a periodic grid with shear modulus mu and Poisson ratio nu."""

    def __init__(self, gridShape, field=None, nu=0.3, mu=0.5, inherit=None):
        self.gridShape = tuple(gridShape)
        self.dimension = len(self.gridShape)
        if inherit is not None:
            self.nu, self.mu = inherit.nu, inherit.mu
        else:
            self.nu, self.mu = nu, mu
        self._field = None
        self._dev = None          # torch tensor (9,) + grid on the GPU, or None
        self._host_ok = False
        self.UpdateOrderParameterField(field)

    # ---------------------------------------------------------------- field access
    @property
    def ktools(self):
        return FourierSpaceTools.FourierSpaceTools(self.gridShape)

    @property
    def betaP(self):
        self._sync_host()
        self._dev = None          # the caller may modify the host arrays in place
        return self._field

    @betaP.setter
    def betaP(self, value):
        self._field = value
        self._host_ok = True
        self._dev = None

    def GetOrderParameterField(self):
        return self.betaP

    def UpdateOrderParameterField(self, orderParameterFieldState):
        if orderParameterFieldState is None:
            self.betaP = Fields.TensorField(self.gridShape)
        else:
            self.betaP = orderParameterFieldState

    def evaluate(self):
        return self

    def _sync_host(self):
        if not self._host_ok:
            arr = self._dev.detach().to('cpu', dtype=__import__('torch').float64).numpy()
            self._field = Fields.from_stack(self.gridShape, arr)
            self._host_ok = True

    def device_tensor(self, dtype, device):
        """(9,) + grid tensor on the GPU, uploading the host field if needed."""
        import torch
        if self._dev is None or self._dev.dtype != dtype or self._dev.device != device:
            if self._dev is not None and not self._host_ok:
                self._dev = self._dev.to(device=device, dtype=dtype)
            else:
                arr = self._field.stack(numpy.float64)
                self._dev = torch.as_tensor(arr).to(device=device, dtype=dtype).contiguous()
        return self._dev

    def _set_device(self, tensor):
        self._dev = tensor
        self._host_ok = False

    def copy(self):
        s = self.__class__(self.gridShape, inherit=self)
        if self._dev is not None and not self._host_ok:
            s._set_device(self._dev.clone())
        else:
            s.betaP = self._field.numpy_arrays() * 1.0
        return s

    # ---------------------------------------------------------------- physics
    def _engine(self):
        from Plasticity.FieldDynamics.engine import plan_for
        return plan_for(self.gridShape, self.mu, self.nu)

    def CalculateSigma(self, type='k', source='betaE'):
        """Internal stress (PlasticityState.py L85-127, source 'betaE'), 9-component TensorField."""
        if type != 'k' or source not in ('betaE', 'betaP'):
            raise NotImplementedError("CalculateSigma supports type='k', source='betaE'/'betaP' on the GPU")
        s6 = self._sigma6()
        arr = s6[[0, 1, 2, 1, 3, 4, 2, 4, 5]].detach().to('cpu').double().numpy()
        return Fields.from_stack(self.gridShape, arr)

    def _sigma6(self):
        plan = self._engine()
        beta = plan.pack_state(self)
        s = plan.stress(beta)
        return plan.stress_view(s, 0)

    def CalculateElasticEnergy(self, type='k', source='betaE'):
        """Elastic energy density 1/2 S:sigma sigma per cell (PlasticityState.py L317-330)."""
        s = self._sigma6().double()
        sq = s[0] ** 2 + s[3] ** 2 + s[5] ** 2 + 2.0 * (s[1] ** 2 + s[2] ** 2 + s[4] ** 2)
        tr = s[0] + s[3] + s[5]
        e = (sq - self.nu / (1.0 + self.nu) * tr * tr) / (4.0 * self.mu)
        return GridArray.GridArray(e.cpu().numpy())

    @staticmethod
    def _sin_k(type):
        if type not in ('k', 'sinK'):
            raise ValueError("type must be 'k' or 'sinK'")
        return type == 'sinK'

    def _observe(self, kind, type='k'):
        """A k-space observable of this state's beta^P on the GPU (cdd.Plan.observe), as host FP64;
        type 'sinK' uses the sine k tables (FourierSpaceTools(gridShape, func=sin))."""
        plan = self._engine()
        out = plan.observe(kind, plan.pack_state(self), sin_k=self._sin_k(type))
        return plan.observable_view(out, 0, kind).detach().to('cpu').double().numpy()

    def CalculateBetaElastic(self, type='k'):
        """beta^E = IFFT(kmask T beta^P^) - beta^P (PlasticityState.py L357-390), on the GPU."""
        return Fields.from_stack(self.gridShape, self._observe("beta_elastic", type))

    def CalculateRotationField(self, type='k'):
        """rotE_ij = (beta^E_ij - beta^E_ji) / 2 (PlasticityState.py L435-446), on the GPU."""
        w = self._observe("rotation", type)   # xy, xz, yz
        full = numpy.zeros((9,) + tuple(self.gridShape))
        for c, (i, j) in enumerate(((0, 1), (0, 2), (1, 2))):
            full[3 * i + j] = w[c]
            full[3 * j + i] = -w[c]
        return Fields.from_stack(self.gridShape, full)

    def CalculateRotationRodrigues(self, type='k', source='betaP'):
        """Rodrigues rotation vector (PlasticityState.py L447-494), on the GPU: source 'betaP' (the
        reference's default) from beta^P's transform, 'betaE' from the rotation field, 'rho' from
        the Nye density field (which loses the means, as in the reference)."""
        sin_k = self._sin_k(type)
        if source == 'betaP':
            rod = self._observe("rodrigues", type)
        elif source == 'betaE':
            w = self._observe("rotation", type)
            rod = numpy.stack([w[2], -w[1], w[0]])
        elif source == 'rho':
            plan = self._engine()
            rho = plan.observe("rho", plan.pack_state(self), sin_k=sin_k)
            out = plan.observe("rodrigues_rho", rho, sin_k=sin_k)
            rod = plan.observable_view(out, 0, "rodrigues_rho").detach().to('cpu').double().numpy()
        else:
            raise ValueError("source must be 'betaP', 'betaE' or 'rho'")
        return Fields.from_stack(self.gridShape, rod, components=[x, y, z])

    def CalculateRhoFourier(self, type='k'):
        """Nye dislocation density rho_ij = -eps_ikl d_k betaP_lj by Fourier derivatives
        (PlasticityState.py L264-304), on the GPU."""
        return Fields.from_stack(self.gridShape, self._observe("rho", type))

    # ---------------------------------------------------------------- state algebra
    def _combine(self, other, op):
        f = self.GetOrderParameterField()
        g = other.GetOrderParameterField() if isinstance(other, PlasticityState) else other
        return self.__class__(self.gridShape, field=op(f, g), inherit=self)

    def __mul__(self, o):
        return self._combine(o, lambda a, b: a * b)

    def __rmul__(self, o):
        return self.__mul__(o)

    def __add__(self, o):
        return self._combine(o, lambda a, b: a + b)

    def __radd__(self, o):
        return self.__add__(o)

    def __sub__(self, o):
        return self._combine(o, lambda a, b: a - b)

    def __truediv__(self, o):
        return self._combine(o, lambda a, b: a / b)
