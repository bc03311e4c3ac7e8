"""Hand-written adjoint of the fixed-dt TVD-RK3 trajectory, behind a torch.autograd.Function.

Forward: u_{n+1} = Step(u_n) with the three stages of FieldMover.CalculateOneFixedTimeStep
(Plasticity/FieldMovers/FieldMover.py L38-58), L(v) = flux(v, S(v) + load(t_n)) at the step-start
time t_n, for n_steps steps from u_0; loss J = E(u_N) + w_zz * mean(u_N,zz) with E the elastic
energy (PlasticityState.CalculateElasticEnergy L317-330 summed over cells).

Reverse, per step (cotangent F2b of u_{n+1}; F0, F1 recomputed from u_n):
    ub  = F2b / 3 ;  F1b = 2/3 F2b + L_{F1}^T (2/3 dt F2b)
    ub += 3/4 F1b ;  F0b = 1/4 F1b + L_{F0}^T (1/4 dt F1b)
    ub += F0b + L_u^T (dt F0b)
where L_v^T g = cdd_flux_vjp (stencil VJP with recorded limiter branches + transposed Green's
function). Checkpoints every ``checkpoint_every`` steps; the states inside a segment are recomputed
from its checkpoint. Parameter gradients: mu and nu through the stress operator
((dS/dmu) v = S v / mu, (dS/dnu) v by cdd_stress_dnu), through the load conversion
(load_i = lamb tr(eps) + 2 mu eps_i with the instance's mu, nu) and through E; the applied strain
rate as rate = r (-1/2, -1/2, 1) (traceless), eps = rate (t - t0).
"""
import numpy as np
import torch

from . import _lib
from .engine import Instance, Plan, _stream
from ._lib import check

CZZ = np.array([-0.5, -0.5, 1.0])   # traceless zz loading direction


def _ptr(t):
    import ctypes
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


def energy_of_stress(s6, mu, nu):
    """Total elastic energy from 6-component internal stress (symmetric storage), FP64."""
    s = s6.double()
    sq = s[0] ** 2 + s[3] ** 2 + s[5] ** 2 + 2.0 * (s[1] ** 2 + s[2] ** 2 + s[4] ** 2)
    tr = s[0] + s[3] + s[5]
    return ((sq - nu / (1.0 + nu) * tr * tr) / (4.0 * mu)).sum()


def energy_grad_of_stress(s6, mu, nu):
    """d E / d(stored stress components), same dtype as s6."""
    tr = s6[0] + s6[3] + s6[5]
    g = torch.empty_like(s6)
    c = nu / (1.0 + nu)
    g[0] = (2.0 * s6[0] - 2.0 * c * tr) / (4.0 * mu)
    g[3] = (2.0 * s6[3] - 2.0 * c * tr) / (4.0 * mu)
    g[5] = (2.0 * s6[5] - 2.0 * c * tr) / (4.0 * mu)
    g[1] = s6[1] / mu
    g[2] = s6[2] / mu
    g[4] = s6[4] / mu
    return g


class Rollout:
    """Fixed-dt trajectory of one instance with its adjoint.

    shape, mu, nu: grid and material; rate_zz: r of the traceless applied strain rate
    r (-1/2, -1/2, 1) (None: no load); dt: fixed step; precision "f64" or "f32".
    """

    def __init__(self, shape, mu, nu, rate_zz, dt, n_steps, precision="f32", checkpoint_every=20,
                 t0=0.0, w_zz=10.0, Lambda=0.0):
        self.shape = tuple(shape)
        self.mu, self.nu = float(mu), float(nu)
        self.rate_zz = None if rate_zz is None else float(rate_zz)
        self.dt, self.n_steps, self.t0 = float(dt), int(n_steps), float(t0)
        self.K = max(1, int(checkpoint_every))
        self.w_zz = float(w_zz)
        load = None if rate_zz is None else tuple(self.rate_zz * CZZ)
        self.inst = Instance(self.shape, mu=self.mu, nu=self.nu, Lambda=Lambda, cfl=0.25, load_rate=load,
                             load_t0=self.t0)
        self.plan = Plan([self.inst], precision)
        self.lib = self.plan.lib
        self.cells = int(np.prod(self.shape))
        self.checkpoints = {}

    # ------------------------------------------------------------------ forward
    def _step(self, u, n):
        self.plan.set_time(self.t0 + n * self.dt, 1e300)
        self.plan.step_fixed(u, self.dt)

    def forward(self, beta0):
        """Run n_steps from beta0 (packed field, plan dtype); returns (u_N, loss as float)."""
        p = self.plan
        u = beta0.detach().clone()
        self.checkpoints = {}
        for n in range(self.n_steps):
            if n % self.K == 0:
                self.checkpoints[n] = u.clone()
            self._step(u, n)
        self.uN = u
        s6 = p.stress_view(p.stress(u), 0)
        loss = energy_of_stress(s6, self.mu, self.nu) + self.w_zz * p.field_view(u, 0)[8].double().mean()
        return u, float(loss)

    def branch_trace(self, beta0):
        """Branch records (cdd_flux_branches) of the 3 * n_steps flux evaluations of the trajectory
        from beta0, at the states the reverse sweep differentiates at: an int32 tensor of shape
        (3 * n_steps, 4 * cells). Two initial states with equal traces lie on the same smooth
        piece of the loss."""
        p = self.plan
        out = torch.empty((3 * self.n_steps, 4 * self.cells), dtype=torch.int32, device=p.device)
        u = beta0.detach().clone()
        dt = self.dt
        for n in range(self.n_steps):
            t = self.t0 + n * dt
            F0 = u + dt * self._flux(u, t)
            F1 = 0.75 * u + 0.25 * F0 + 0.25 * dt * self._flux(F0, t)
            for k, v in enumerate((u, F0, F1)):
                check(self.lib.cdd_flux_branches(p.handle, _ptr(v), float(t), _ptr(out[3 * n + k]), _stream()))
            self._step(u, n)
        return out

    # ------------------------------------------------------------------ reverse
    def _flux(self, v, t):
        rhs, _ = self.plan.flux(v, t, want_speed=False)
        return rhs

    def _vjp(self, v, t, g, grads):
        """Returns L_v^T g and accumulates parameter gradients."""
        p = self.plan
        vb = torch.zeros(p.field_elems, dtype=p.dtype, device=p.device)
        sb = torch.zeros(p.stress_elems, dtype=p.dtype, device=p.device)
        lb = torch.zeros(3, dtype=torch.float64, device=p.device)
        check(self.lib.cdd_flux_vjp(p.handle, _ptr(v), float(t), _ptr(g), _ptr(vb), _ptr(sb), _ptr(lb),
                                    _stream()))
        self._param_terms(v, sb, lb, t, grads)
        return vb

    def _param_terms(self, v, sb, lb, t, grads):
        p = self.plan
        mu, nu = self.mu, self.nu
        s_int = p.stress_view(p.stress(v), 0)
        s_nu = p.empty_stress()
        check(self.lib.cdd_stress_dnu(p.handle, _ptr(v), _ptr(s_nu), _stream()))
        sbd = p.stress_view(sb, 0).double()
        grads["mu"] += float((sbd * s_int.double()).sum()) / mu
        grads["nu"] += float((sbd * p.stress_view(s_nu, 0).double()).sum())
        if self.rate_zz is not None:
            L = lb.cpu().numpy()
            eps = self.rate_zz * CZZ * (t - self.t0)
            lamb = 2.0 * mu * nu / (1.0 - 2.0 * nu)
            tr = eps.sum()
            dload_dmu = lamb / mu * tr + 2.0 * eps
            dload_dnu = 2.0 * mu / (1.0 - 2.0 * nu) ** 2 * tr * np.ones(3)
            dload_dr = (lamb * CZZ.sum() + 2.0 * mu * CZZ) * (t - self.t0)
            grads["mu"] += float(L @ dload_dmu)
            grads["nu"] += float(L @ dload_dnu)
            grads["rate_zz"] += float(L @ dload_dr)

    def backward(self):
        """Gradients of the loss: (d/d beta0 as a packed field, dict of mu, nu, rate_zz)."""
        p = self.plan
        grads = {"mu": 0.0, "nu": 0.0, "rate_zz": 0.0}
        mu, nu = self.mu, self.nu
        u = self.uN
        # loss terms at the final state
        s6 = p.stress_view(p.stress(u), 0)
        sEbuf = torch.zeros(p.stress_elems, dtype=p.dtype, device=p.device)
        sE = p.stress_view(sEbuf, 0)
        sE.copy_(energy_grad_of_stress(s6, mu, nu))
        ub = torch.zeros(p.field_elems, dtype=p.dtype, device=p.device)
        check(self.lib.cdd_stress_adjoint(p.handle, _ptr(sEbuf), _ptr(ub), _stream()))
        p.field_view(ub, 0)[8] += self.w_zz / self.cells
        E = energy_of_stress(s6, mu, nu)
        tr = (s6[0] + s6[3] + s6[5]).double()
        s_nu = p.empty_stress()
        check(self.lib.cdd_stress_dnu(p.handle, _ptr(u), _ptr(s_nu), _stream()))
        grads["mu"] += float(-E / mu + (sE.double() * s6.double()).sum() / mu)
        grads["nu"] += float((-(tr * tr) / (4.0 * mu * (1.0 + nu) ** 2)).sum()
                             + (sE.double() * p.stress_view(s_nu, 0).double()).sum())
        # reverse sweep over checkpoint segments
        dt = self.dt
        starts = sorted(self.checkpoints)
        for s0 in reversed(starts):
            s1 = min(s0 + self.K, self.n_steps)
            states = [self.checkpoints[s0].clone()]
            for n in range(s0, s1 - 1):
                v = states[-1].clone()
                self._step(v, n)
                states.append(v)
            for n in range(s1 - 1, s0 - 1, -1):
                un = states[n - s0]
                t = self.t0 + n * dt
                F0 = un + dt * self._flux(un, t)
                F1 = 0.75 * un + 0.25 * F0 + 0.25 * dt * self._flux(F0, t)
                F2b = ub
                ub_new = F2b / 3.0
                F1b = (2.0 / 3.0) * F2b + self._vjp(F1, t, (2.0 / 3.0) * dt * F2b, grads)
                ub_new += 0.75 * F1b
                F0b = 0.25 * F1b + self._vjp(F0, t, 0.25 * dt * F1b, grads)
                ub_new += F0b + self._vjp(un, t, dt * F0b, grads)
                ub = ub_new
        p.check_status()
        return ub, grads


class RolloutLoss(torch.autograd.Function):
    """loss = E(u_N) + w_zz mean(u_N,zz) of a fixed-dt rollout; differentiable in beta0 (packed
    field tensor), mu, nu and rate_zz (0-d tensors)."""

    @staticmethod
    def forward(ctx, beta0, mu, nu, rate_zz, shape, dt, n_steps, precision, checkpoint_every):
        ro = Rollout(shape, float(mu), float(nu), float(rate_zz), dt, n_steps, precision=precision,
                     checkpoint_every=checkpoint_every)
        b = ro.plan.pack([beta0.detach().reshape((9,) + ro.shape)])
        _, loss = ro.forward(b)
        ctx.ro = ro
        ctx.in_dtype = beta0.dtype
        ctx.in_shape = beta0.shape
        return torch.tensor(loss, dtype=torch.float64, device=beta0.device)

    @staticmethod
    def backward(ctx, g):
        gb, grads = ctx.ro.backward()
        gv = float(g)
        dev = gb.device
        tens = lambda v: torch.tensor(v * gv, dtype=torch.float64, device=dev)
        gbeta = ctx.ro.plan.field_view(gb, 0).reshape(ctx.in_shape).to(ctx.in_dtype) * gv
        return (gbeta, tens(grads["mu"]), tens(grads["nu"]), tens(grads["rate_zz"]),
                None, None, None, None, None)
