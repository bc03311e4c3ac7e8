"""TVD Runge-Kutta 3 field mover (reference: Plasticity/FieldMovers/FieldMover.py L8-141).

Each step runs on the GPU through libcdd (cdd_step / cdd_step_fixed); the returned state is a
new object holding its own device copy, as the reference returns a new state per step.
"""


class FieldMover:
    def Run(self, state, observers, dynamics, startTime, endTime, dT):
        raise NotImplementedError


class TVDRungeKutta_FieldMover(FieldMover):
    def __init__(self, CFLsafeFactor=0.1, dtBound=0.01):
        self.CFLsafeFactor = CFLsafeFactor
        self.dtBound = dtBound

    def Run(self, state, observers, dynamics=None, startTime=0., endTime=10., fixedTimeStep=None):
        t = startTime
        numberOfSteps = 0
        while True:
            if fixedTimeStep is not None:
                state, dt = self.CalculateOneFixedTimeStep(t, state, dynamics, endTime, fixedTimeStep)
            else:
                state, dt = self.CalculateOneAdaptiveTimeStep(t, state, dynamics, endTime)
            t += dt
            numberOfSteps += 1
            for observer in observers:
                observer.Update(t, state)
            if t >= endTime:
                break

    def _step(self, time, state, dynamics, endTime, fixed_dt):
        plan = dynamics.plan(state, cfl=self.CFLsafeFactor)
        beta = plan.pack_state(state).clone()
        plan.set_time(time, endTime)
        if fixed_dt is None:
            plan.step(beta)
        else:
            plan.step_fixed(beta, fixed_dt)
        _, dt, _ = plan.get_time()
        plan.check_status()
        new = state.__class__(state.gridShape, inherit=state)
        new._set_device(beta.view((9,) + tuple(state.gridShape)))
        return new, float(dt[0])

    def CalculateOneAdaptiveTimeStep(self, time, state, dynamics, endTime):
        return self._step(time, state, dynamics, endTime, None)

    def CalculateOneFixedTimeStep(self, time, state, dynamics, endTime, timeStep):
        return self._step(time, state, dynamics, endTime, timeStep)


class OperatorSplittingTVDRK_FieldMover(TVDRungeKutta_FieldMover):
    """TVD-RK3 of beta^P with the vacancy concentration split off (reference: FieldMover.py
    L318-380): one GPU step advances beta^P with c fixed, then c += beta d tr(beta^P) and the exact
    diffusion (cdd_instance.vacancy). The adaptive step is bounded by dtBound (None: no bound). A
    fixed step also applies the new beta^P (the reference's fixed-step variant recouples the
    step-start beta^P, L337, and so leaves beta^P unchanged)."""

    def _step(self, time, state, dynamics, endTime, fixed_dt):
        plan = dynamics.plan(state, cfl=self.CFLsafeFactor, dt_max=self.dtBound or 0.0)
        beta = plan.pack_state(state).clone()
        c = plan.empty_vacancy()
        c.copy_(state.cfield_device(plan.dtype, plan.device).reshape(-1))
        plan.set_vacancy(c)
        plan.set_time(time, endTime)
        if fixed_dt is None:
            plan.step(beta)
        else:
            plan.step_fixed(beta, fixed_dt)
        _, dt, _ = plan.get_time()
        plan.check_status()
        plan.set_vacancy(None)
        new = state.__class__(state.gridShape, inherit=state)
        new._set_device(beta.view((9,) + tuple(state.gridShape)))
        new._set_cdevice(c.view(tuple(state.gridShape)))
        return new, float(dt[0])
