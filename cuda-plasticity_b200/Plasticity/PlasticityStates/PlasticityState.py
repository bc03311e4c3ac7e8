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

    def CalculateBetaElastic(self, type='k'):
        """beta^E = IFFT(kmask T beta^P) - beta^P on the host (PlasticityState.py L357-390).

        T contracted with beta^P^ is k_i g_j with g_j = k_j (A s / kSq - B r / kSqSq)
        + (p_j + q_j) / kSq (s = trace, p_j = k_m b_mj, q_j = b_jn k_n, r = k_m q_m).
        """
        K = FourierSpaceTools.FourierSpaceTools(self.gridShape)
        k = [numpy.asarray(K.kx), numpy.asarray(K.ky), numpy.asarray(K.kz)]
        kSq = numpy.asarray(K.kSq) + ME
        kSqSq = numpy.asarray(K.kSqSq) + ME
        lamb = 2. * self.mu * self.nu / (1. - 2. * self.nu)
        A = lamb / (lamb + 2. * self.mu)
        B = 2. * (lamb + self.mu) / (lamb + 2. * self.mu)
        bh = numpy.fft.rfftn(self.betaP.stack(), axes=tuple(range(1, self.dimension + 1)))
        b = lambda i, j: bh[3 * i + j]
        s = b(0, 0) + b(1, 1) + b(2, 2)
        p = [k[0] * b(0, j) + k[1] * b(1, j) + k[2] * b(2, j) for j in range(3)]
        q = [b(j, 0) * k[0] + b(j, 1) * k[1] + b(j, 2) * k[2] for j in range(3)]
        r = k[0] * q[0] + k[1] * q[1] + k[2] * q[2]
        c = A * s / kSq - B * r / kSqSq
        g = [k[j] * c + (p[j] + q[j]) / kSq for j in range(3)]
        mask = numpy.asarray(K.kmask)
        out = numpy.stack([mask * k[i] * g[j] for i in range(3) for j in range(3)])
        be = numpy.fft.irfftn(out, s=self.gridShape, axes=tuple(range(1, self.dimension + 1)))
        return Fields.from_stack(self.gridShape, be - self.betaP.stack())

    def CalculateRhoFourier(self, type='k'):
        """Nye dislocation density rho_ij = -eps_ikl d_k betaP_lj by Fourier derivatives
        (PlasticityState.py L264-304), on the host."""
        K = FourierSpaceTools.FourierSpaceTools(self.gridShape)
        Kb = self.betaP.FFT()
        ks = [K.kx, K.ky, K.kz]
        D = [Kb * (1.0j * ks[d]) for d in range(self.dimension if self.dimension > 1 else 1)]
        Kr = Fields.TensorField(self.gridShape, kspace=True)
        for i in (x, y, z):
            if self.dimension == 3:
                Kr[x, i] = D[2][y, i] - D[1][z, i]
                Kr[y, i] = D[0][z, i] - D[2][x, i]
                Kr[z, i] = D[1][x, i] - D[0][y, i]
            elif self.dimension == 2:
                Kr[x, i] = -D[1][z, i]
                Kr[y, i] = D[0][z, i]
                Kr[z, i] = D[1][x, i] - D[0][y, i]
        return Kr.IFFT()

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
