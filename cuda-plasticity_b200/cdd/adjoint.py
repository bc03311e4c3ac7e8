"""Hand-written adjoint of the fixed-dt TVD-RK3 trajectory, behind a torch.autograd.Function.

Forward: u_{n+1} = Step(u_n) with the three stages of FieldMover.CalculateOneFixedTimeStep
(Plasticity/FieldMovers/FieldMover.py L38-58), L(v) = flux(v, S(v) + load(t_n)) at the step-start
time t_n, for n_steps steps from u_0; loss J = E(u_N) + w_zz * mean(u_N,zz) with E the elastic
energy (PlasticityState.CalculateElasticEnergy L317-330 summed over cells).

Reverse, per step (cotangent F2b of u_{n+1}; stage states, stresses and k-space data recorded
by cdd_step_record while re-running the step's checkpoint segment), in cdd_step_adjoint:
    F1b = 2/3 F2b + 2/3 dt L_{F1}^T F2b ;  F0b = 1/4 F1b + 1/4 dt L_{F0}^T F1b
    ub  = 1/3 F2b + 3/4 F1b + F0b + dt L_u^T F0b
with L_v^T the flux VJP (stencil VJP with recorded limiter branches + transposed Green's function).
Parameter gradients: mu through the stress (S ~ mu), nu through lambda (pointwise) and through the
Green's function coefficients (a Parseval sum in k-space), both also through the load conversion
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
    r (-1/2, -1/2, 1) (None: no load); dt: fixed step; precision "f64" or "f32"; tuning: launch
    shapes as for ``cdd.Plan`` (None, [dict] or "auto").
    The forward keeps a copy of the state every ``checkpoint_every`` steps and runs the last
    segment with cdd_step_record (saving stage states, stresses and k-space data); the reverse
    sweep walks that segment backwards with cdd_step_adjoint straight away and re-runs each earlier
    segment from its checkpoint with records before walking it back. Nothing synchronises the host
    until the parameter cotangents are read at the end.

    overlap (default): the re-run of the next segment back goes to a second CUDA stream with a
    second plan of the same instance (its own scratch) and the other half of a double buffer of
    records, so that it runs while the current segment is walked back on the caller's stream;
    events order a segment's walk after its re-run and a buffer's reuse after the walk that read
    it. The kernels and their inputs are those of the serial sweep (overlap=False), so the results
    are bitwise the same. It holds twice the records (2 x checkpoint_every, about 50 MB each at 64^3
    FP32, 3.2 GB at 256^3) and a second plan's scratch; overlap=False keeps one segment's.
    """

    def __init__(self, shape, mu, nu, rate_zz, dt, n_steps, precision="f32", checkpoint_every=20,
                 t0=0.0, w_zz=10.0, Lambda=0.0, tuning=None, overlap=True):
        self.shape = tuple(shape)
        self.mu, self.nu = float(mu), float(nu)
        self.rate_zz = None if rate_zz is None else float(rate_zz)
        self.dt, self.n_steps, self.t0 = float(dt), int(n_steps), float(t0)
        self.K = max(1, int(checkpoint_every))
        self.w_zz = float(w_zz)
        load = None if rate_zz is None else tuple(self.rate_zz * CZZ)
        self.inst = Instance(self.shape, mu=self.mu, nu=self.nu, Lambda=Lambda, cfl=0.25, load_rate=load,
                             load_t0=self.t0)
        self.plan = Plan([self.inst], precision, tuning=tuning)
        self.overlap = bool(overlap)
        self.plan_rerun = None   # the overlapped sweep's second plan, made on its first use
        self._side = None
        self.lib = self.plan.lib
        self.cells = int(np.prod(self.shape))
        self.checkpoints = {}
        self.rec_elems = int(self.lib.cdd_plan_record_elems(self.plan.handle))
        self._records = None
        self._tail = None   # start of the segment whose records the last forward left in the buffer

    def time(self, n):
        return self.t0 + n * self.dt

    # ------------------------------------------------------------------ forward
    def _step(self, u, n, rec=None, plan=None, stream=None):
        plan = self.plan if plan is None else plan
        check(self.lib.cdd_step_record(plan.handle, _ptr(u), self.time(n), self.dt, _ptr(rec), _stream(stream)))

    def forward(self, beta0):
        """Run n_steps from beta0 (packed field, plan dtype); returns (u_N, loss as float)."""
        p = self.plan
        u = beta0.detach().clone()
        self.checkpoints = {}
        tail = ((self.n_steps - 1) // self.K) * self.K
        recs = self._record_buffer(self.K)
        self._tail = None
        for n in range(self.n_steps):
            if n % self.K == 0:
                self.checkpoints[n] = u.clone()
            self._step(u, n, recs[n - tail] if n >= tail else None)
        self._tail = tail
        self.uN = u
        s6 = p.stress_view(p.stress(u), 0)
        loss = energy_of_stress(s6, self.mu, self.nu) + self.w_zz * p.field_view(u, 0)[8].double().mean()
        return u, float(loss)

    def branch_trace(self, beta0):
        """Branch records (cdd_flux_branches) of the 3 * n_steps flux evaluations of the trajectory
        from beta0, at the stage states the reverse sweep differentiates at: an int32 tensor of
        shape (3 * n_steps, 4 * cells). Two initial states with equal traces lie on the same smooth
        piece of the loss."""
        p = self.plan
        out = torch.empty((3 * self.n_steps, 4 * self.cells), dtype=torch.int32, device=p.device)
        rec = self._record_buffer(1)[0]
        self._tail = None   # the forward's records of its last segment are overwritten
        u = beta0.detach().clone()
        for n in range(self.n_steps):
            self._step(u, n, rec)
            for k, part in enumerate(self._record_parts(rec)):
                check(self.lib.cdd_flux_branches(p.handle, _ptr(part), self.time(n), _ptr(out[3 * n + k]),
                                                 _stream()))
        return out

    # ------------------------------------------------------------------ reverse
    def _record_buffer(self, k, half=0):
        """k step records (256-byte aligned); half 1 is the second buffer of the overlapped sweep."""
        nb = 2 if self.overlap else 1
        if self._records is None or self._records.shape[0] < nb * k:
            el = torch.tensor([], dtype=self.plan.dtype).element_size()
            pad = 256 // el
            raw = torch.empty(nb * k * self.rec_elems + pad, dtype=self.plan.dtype, device=self.plan.device)
            off = (-raw.data_ptr() % 256) // el
            self._raw = raw
            self._records = raw[off:off + nb * k * self.rec_elems].view(nb * k, self.rec_elems)
        return self._records[half * k:(half + 1) * k]

    def _record_parts(self, rec):
        """Views of the states u, F0, F1 inside a record (the first three 256-byte aligned parts)."""
        el = rec.element_size()
        step = -(-self.plan.field_elems * el // 256) * 256 // el
        return [rec[i * step:i * step + self.plan.field_elems] for i in range(3)]

    def backward(self):
        """Gradients of the loss: (d/d beta0 as a packed field, dict of mu, nu, rate_zz)."""
        p = self.plan
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
        g_mu_loss = -E / mu + (sE.double() * s6.double()).sum() / mu
        g_nu_loss = (-(tr * tr) / (4.0 * mu * (1.0 + nu) ** 2)).sum() + \
            (sE.double() * p.stress_view(s_nu, 0).double()).sum()
        # reverse sweep over checkpoint segments
        pbar = torch.zeros(_lib.CDD_PBAR, dtype=torch.float64, device=p.device)
        if self.overlap:
            self._sweep_overlapped(ub, pbar)
        else:
            recs = self._record_buffer(self.K)
            for s0 in sorted(self.checkpoints, reverse=True):
                s1 = min(s0 + self.K, self.n_steps)
                if s0 != self._tail:
                    v = self.checkpoints[s0].clone()
                    for n in range(s0, s1):
                        self._step(v, n, recs[n - s0])
                self._tail = None
                for n in range(s1 - 1, s0 - 1, -1):
                    check(self.lib.cdd_step_adjoint(p.handle, _ptr(recs[n - s0]), self.time(n), self.dt, _ptr(ub),
                                                    _ptr(pbar), _stream()))
        pb = pbar.cpu().numpy()
        lamb = 2.0 * mu * nu / (1.0 - 2.0 * nu)
        dlam = 2.0 * mu / (1.0 - 2.0 * nu) ** 2
        dA = 1.0 / (1.0 - nu) ** 2
        grads = {"mu": float(g_mu_loss) + pb[0] / mu,
                 "nu": float(g_nu_loss) + pb[1] * dlam / (2.0 * mu + 3.0 * lamb) + pb[2] * dA,
                 "rate_zz": 0.0}
        if self.rate_zz is not None:
            # load_i(t) = lamb tr(eps) + 2 mu eps_i, eps = rate (t - t0), rate = r CZZ (traceless)
            L, Lt = pb[3:6], pb[6:9]
            rate = self.rate_zz * CZZ
            grads["mu"] += float(Lt @ (lamb / mu * rate.sum() + 2.0 * rate))
            grads["nu"] += float(Lt @ (dlam * rate.sum() * np.ones(3)))
            grads["rate_zz"] += float(Lt @ (lamb * CZZ.sum() + 2.0 * mu * CZZ))
        p.check_status()
        if self.plan_rerun is not None:
            self.plan_rerun.check_status()
        return ub, grads

    def _sweep_overlapped(self, ub, pbar):
        """Reverse sweep with the re-run of segment i + 1 (next one back) on a side stream while
        segment i is walked back on the current stream. Segment i uses record buffer i % 2."""
        p = self.plan
        main = torch.cuda.current_stream(p.device)
        if self.plan_rerun is None:
            # the re-runs: same instance and launch shapes, separate scratch
            self.plan_rerun = Plan([self.inst], p.precision, tuning=[p.tuning(0)])
        if self._side is None:
            self._side = torch.cuda.Stream(device=p.device)
        side = self._side
        segs = sorted(self.checkpoints, reverse=True)
        start = torch.cuda.Event()
        start.record(main)          # the forward, checkpoints and loss terms are in main's order
        side.wait_event(start)
        ready, walked = {}, {}
        held = []                   # re-run states, kept until the sweep ends (side-stream work)

        def rerun(i):
            s0 = segs[i]
            s1 = min(s0 + self.K, self.n_steps)
            recs = self._record_buffer(self.K, i % 2)
            with torch.cuda.stream(side):
                if i - 2 in walked:
                    side.wait_event(walked[i - 2])   # buffer i % 2 was read by segment i - 2
                v = self.checkpoints[s0].clone()
                held.append(v)
                for n in range(s0, s1):
                    self._step(v, n, recs[n - s0], plan=self.plan_rerun, stream=side)
                ev = torch.cuda.Event()
                ev.record(side)
            ready[i] = ev

        if segs and segs[0] != self._tail:
            rerun(0)
        self._tail = None
        for i, s0 in enumerate(segs):
            if i + 1 < len(segs):
                rerun(i + 1)
            if i in ready:
                main.wait_event(ready[i])
            s1 = min(s0 + self.K, self.n_steps)
            recs = self._record_buffer(self.K, i % 2)
            for n in range(s1 - 1, s0 - 1, -1):
                check(self.lib.cdd_step_adjoint(p.handle, _ptr(recs[n - s0]), self.time(n), self.dt, _ptr(ub),
                                                _ptr(pbar), _stream(main)))
            ev = torch.cuda.Event()
            ev.record(main)
            walked[i] = ev
        # every side-stream re-run precedes a walk on main, so main's order now covers all of them;
        # the re-run states (side-stream allocations) return to the side stream's pool
        del held


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
