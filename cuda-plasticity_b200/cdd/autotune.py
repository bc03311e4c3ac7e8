"""Autotuner of the launch shapes: FFT radix plans, FFT tile widths and stencil plane chunks.

For one grid shape and precision it builds plans with candidate ``cdd_tuning`` values
(``include/cdd.h``), times whole fixed-dt TVD-RK3 steps on the current GPU with CUDA events, and
keeps the fastest. The search is a coordinate descent from the built-in rule: one knob at a time,
the others held at their current best, over a few sweeps until nothing improves. Results are cached
in a JSON file (``CDD_TUNE_CACHE``, default ``~/.cache/cdd_tune.json``) keyed by GPU name,
precision and shape, so a shape is tuned once per GPU model. No knob changes the mathematics:
results agree with the built-in shapes to rounding (different radix orders round differently).
"""
import json
import os

import numpy as np

from . import _lib

KNOBS = ("stencil_planes", "fft_radix", "green_cols", "mid_cols", "rows_lines", "plane_fft")


def cache_path():
    return os.environ.get("CDD_TUNE_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "cdd_tune.json"))


def cache_key(gpu, precision, shape):
    return "%s|%s|%s" % (gpu, precision, "x".join(str(int(n)) for n in shape))


def load_cache(path=None):
    path = path or cache_path()
    try:
        with open(path) as f:
            d = json.load(f)
        return d if isinstance(d, dict) else {}
    except (OSError, ValueError):
        return {}


def save_cache(d, path=None):
    path = path or cache_path()
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    tmp = "%s.%d.tmp" % (path, os.getpid())   # ranks of one job may save at the same time
    with open(tmp, "w") as f:
        json.dump(d, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def candidates(knob, shape, current):
    """Values of one knob to try, given the plan's current effective value of it."""
    nd = len(shape)
    v = int(current.get(knob, 0) or 0)
    if knob == "fft_radix":
        return [16, 8, 4]
    if knob == "stencil_planes":
        if nd != 3:
            return []
        return sorted({p for p in (2, 4, 8, 16, 32, 64) if p <= shape[0]} | ({v} if v else set()))
    if knob == "mid_cols" and nd != 3:
        return []
    if knob == "plane_fft":
        # fused plane passes (1) or separate row and axis-1 passes (-1); 0: not applicable
        return [1, -1] if v else []
    if v <= 0:
        return []
    return sorted({max(1, v // 2), v, v * 2})


def _time_steps(plan, beta, reps):
    import torch
    st = torch.cuda.current_stream()
    for _ in range(2):
        plan.step_fixed(beta, 1e-9)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    times = []
    for _ in range(reps):
        torch.cuda.synchronize()
        e0.record(st)
        plan.step_fixed(beta, 1e-9)
        e1.record(st)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    return float(np.median(times))


def tune(inst, precision, reps=5, sweeps=2, verbose=False):
    """Tune one instance's launch shapes. Returns (best tuning dict, best ms per step, built-in ms,
    list of (tuning, ms) tried)."""
    import torch
    from .engine import Instance, Plan
    from .initial import gaussian_random_field_torch
    one = Instance(tuple(inst.shape), mu=inst.mu, nu=inst.nu, Lambda=inst.Lambda, cfl=inst.cfl,
                   load_rate=inst.load_rate, glide_only=inst.glide_only)
    field = gaussian_random_field_torch(tuple(inst.shape), 0.04, 0.05, 7, device="cuda")
    tried = {}

    def run(t):
        key = tuple(sorted(t.items()))
        if key in tried:
            return tried[key]
        try:
            plan = Plan([one], precision, tuning=[t])
        except _lib.CDDError:
            tried[key] = (None, None)
            return tried[key]
        beta = plan.pack([field])
        ms = _time_steps(plan, beta, reps)
        eff = plan.tuning(0)
        plan.close()
        del beta
        torch.cuda.empty_cache()
        tried[key] = (ms, eff)
        if verbose:
            print("  %s -> %.3f ms" % (t, ms))
        return tried[key]

    base_ms, best = run({})
    best_ms = base_ms
    cur = dict(best)
    for _ in range(sweeps):
        improved = False
        for knob in KNOBS:
            for v in candidates(knob, inst.shape, cur):
                t = dict(cur)
                t[knob] = v
                ms, eff = run(t)
                if ms is not None and ms < best_ms * 0.99:
                    best_ms, cur, improved = ms, dict(eff), True
        if not improved:
            break
    history = [(dict(k), v[0]) for k, v in tried.items()]
    return cur, best_ms, base_ms, history


def best(inst, precision, use_cache=True, verbose=False):
    """The tuned launch shapes of inst (a cdd.Instance) at precision, from the cache or by tuning."""
    import torch
    gpu = torch.cuda.get_device_name()
    key = cache_key(gpu, precision + ("-glide" if inst.glide_only else ""), inst.shape)
    cache = load_cache() if use_cache else {}
    if key in cache:
        return dict(cache[key]["tuning"])
    t, ms, base_ms, _ = tune(inst, precision, verbose=verbose)
    if use_cache:
        cache = load_cache()
        cache[key] = {"tuning": t, "ms_per_step": ms, "builtin_ms_per_step": base_ms}
        try:
            save_cache(cache)
        except OSError:
            pass
    return t
