"""Bridge from the facades to libcdd: one cached cdd.Plan per (grid, material, dynamics, loading,
precision) and the helpers the movers and dynamics share."""
import torch

import cdd

_PLANS = {}
_PRECISION = "f64"


def set_precision(precision):
    """Precision of the GPU path used by the facades: "f64" (default, the drop-in) or "f32"."""
    global _PRECISION
    if precision not in ("f64", "f32"):
        raise ValueError("precision must be 'f64' or 'f32'")
    _PRECISION = precision


def get_precision():
    return _PRECISION


class FacadePlan(cdd.Plan):
    def pack_state(self, state):
        """Packed 1-instance field holding the state's beta^P (a view of its device tensor)."""
        t = state.device_tensor(self.dtype, self.device)
        return t.reshape(-1)


def plan_for(gridShape, mu, nu, Lambda=0.0, cfl=0.25, load=None, precision=None, glide=False, vacancy=None,
             dt_max=0.0):
    """load: None or (rate[3], initial[3], t0, load_mu, load_nu); glide: glide-only dynamics;
    vacancy: None or (alpha, beta, gamma) of the vacancy coupling; dt_max: bound of the step."""
    precision = precision or _PRECISION
    key = (tuple(gridShape), float(mu), float(nu), float(Lambda), float(cfl),
           None if load is None else (tuple(load[0]), tuple(load[1]), float(load[2]), float(load[3]),
                                      float(load[4])), precision, bool(glide),
           None if vacancy is None else tuple(float(v) for v in vacancy), float(dt_max))
    p = _PLANS.get(key)
    if p is None:
        kw = dict(mu=mu, nu=nu, Lambda=Lambda, cfl=cfl, glide_only=glide, vacancy=vacancy, dt_max=dt_max)
        if load is None:
            inst = cdd.Instance(tuple(gridShape), **kw)
        else:
            inst = cdd.Instance(tuple(gridShape), load_rate=tuple(load[0]), load_initial=tuple(load[1]),
                                load_t0=load[2], load_mu=load[3], load_nu=load[4], **kw)
        p = FacadePlan([inst], precision)
        _PLANS[key] = p
    return p


def clear_plans():
    _PLANS.clear()
    torch.cuda.empty_cache()
