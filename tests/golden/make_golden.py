"""Generate the golden vectors in this folder by running the reference's own Python FP64 path.

The reference (mattbierbaum/cuda-plasticity, ``Plasticity/``) is Python 2 code. This script copies
the modules of the time-step path into ``oracle/_refpy/Plasticity`` (git-ignored and not shipped to
GPU machines) and applies mechanical Python-3 / numpy-2 patches, none of which touches arithmetic:

  (i)   ``raise E, "msg"`` -> ``raise E("msg")`` and ``print "..."`` -> ``print(...)``;
  (ii)  ``/2+1`` -> ``//2+1`` (integer half-spectrum sizes, GridArray/FourierSpaceTools.py L17-45);
  (iii) ``__div__``/``__rdiv__`` -> ``__truediv__``/``__rtruediv__`` (Fields.py, PlasticityState.py);
  (iv)  ``from scipy import fromfunction, sin, pi`` -> ``from numpy import ...`` (PlasticityState.py L4);
  (v)   ``copy=False`` -> ``copy=None`` (numpy-2 semantics, GridArray.py L8-9);
  (vi)  tabs expanded;
  (ix)  the operator-splitting mover's CFL step ``dt = self.CFLsafeFactor / sum`` (a 0-d array)
        becomes a Python float, as the main mover's ``dt = dt.tolist()`` does (FieldMover.py L96-99):
        under numpy 2 a 0-d array times the reference's Field objects builds an object array.

It then drives the reference through its public API -- ``PlasticityState``, the
``BetaPDynamics.CalculateFlux`` of CentralUpwindHJBetaPDynamics3D.py (3-D) or of
CentralUpwindHJBetaPDynamics.py (2-D, the module RunPython.py imports), and
``TVDRungeKutta_FieldMover.CalculateOneAdaptiveTimeStep`` -- on seeded inputs from
``cdd.initial.gaussian_random_field`` and writes ``*.npz`` fixtures next to this file.

``initializer.npz`` holds states of the reference's GaussianRandomInitializer (``run_initializer_case``).
``observables.npz`` holds the field observables of PlasticityState (beta^E, rotation, Rodrigues
vector from beta^P and from rho, Nye density; with the 'k' and the 'sinK' tables) of seeded fields. ``io_formats.npz`` pins the CUDA solver's file formats: the reference's convertStateToCUDA and
LoadStateRaw run from their source text (``run_io_case``).

``c2_3d_64`` and ``c2_3d_128`` are compact fixtures of 10 steps at the config-2 sizes (sigma 0.04, the
applied strain rate diag(-0.025, -0.025, 0.05)): instead of whole fields they hold the dt sequence,
the energy and mean-strain curves, per-component sums and sums of squares after steps 1 and 10, and
the 9 components of 4096 seeded sample cells after steps 1 and 10 (``run_case`` with ``samples``).

Usage: ``python tests/golden/make_golden.py --reference PATH [--only NAME]`` (PATH is the reference
checkout; the environment variable CDD_REFERENCE may give it instead; CDD_REFPY_DIR may move the
patched copy elsewhere, e.g. to run two cases at once). Only this script reads the reference tree;
tests read the committed ``.npz`` files.
"""
import argparse
import os
import re
import shutil
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
PATCHED = os.environ.get("CDD_REFPY_DIR") or os.path.join(REPO, "oracle", "_refpy")

MODULES = [
    "__init__.py", "Constants.py", "NumericalMethods.py", "PlasticitySystem.py",
    "GridArray/__init__.py", "GridArray/GridArray.py", "GridArray/FourierSpaceTools.py",
    "Fields/__init__.py", "Fields/Fields.py",
    "PlasticityStates/__init__.py", "PlasticityStates/PlasticityState.py",
    "PlasticityStates/BurgersState.py",
    "FieldDynamics/__init__.py", "FieldDynamics/FieldDynamics.py",
    "FieldDynamics/CentralUpwindHJ.py", "FieldDynamics/CentralUpwindHJ3D.py",
    "FieldDynamics/CentralUpwindHJBetaPDynamics.py",
    "FieldDynamics/CentralUpwindHJBetaPDynamics3D.py",
    "FieldDynamics/CentralUpwindHJBetaPGlideOnlyDynamics.py",
    "FieldMovers/__init__.py", "FieldMovers/FieldMover.py",
    "PlasticityStates/VacancyState.py", "FieldDynamics/VacancyDynamics.py",
]


def _patch(text):
    text = text.expandtabs(8)                                               # (vi)
    text = re.sub(r'raise (\w+), (".*?")', r"raise \1(\2)", text)           # (i)
    text = re.sub(r'^(\s*)print (".*)$', r"\1print(\2)", text, flags=re.M)  # (i)
    text = text.replace("/2+1", "//2+1")                                    # (ii)
    text = text.replace("__rdiv__", "__rtruediv__").replace("__div__", "__truediv__")  # (iii)
    text = text.replace("from scipy import fromfunction, sin, pi",
                        "from numpy import fromfunction, sin, pi")         # (iv)
    text = text.replace("copy=False", "copy=None")                          # (v)
    text = text.replace("dt = self.CFLsafeFactor / sum\n        if (dt > self.dtBound)",
                        "dt = float(self.CFLsafeFactor / sum)\n        if (dt > self.dtBound)")  # (ix)
    return text


def build_patched_copy(reference):
    src_root = os.path.join(reference, "Plasticity")
    dst_root = os.path.join(PATCHED, "Plasticity")
    if os.path.isdir(PATCHED):
        shutil.rmtree(PATCHED)
    for rel in MODULES:
        dst = os.path.join(dst_root, rel)
        os.makedirs(os.path.dirname(dst), exist_ok=True)
        with open(os.path.join(src_root, rel)) as f:
            text = f.read()
        with open(dst, "w") as f:
            f.write(_patch(text))
    return PATCHED


COMPONENTS = [(a, b) for a in "xyz" for b in "xyz"]


def _import_reference():
    sys.path.insert(0, PATCHED)
    from Plasticity.PlasticityStates import PlasticityState
    from Plasticity.GridArray import GridArray
    from Plasticity.FieldMovers import FieldMover
    from Plasticity.FieldDynamics import CentralUpwindHJBetaPDynamics3D as Dyn3
    from Plasticity.FieldDynamics import CentralUpwindHJBetaPDynamics as Dyn2
    from Plasticity.FieldDynamics import CentralUpwindHJBetaPGlideOnlyDynamics as Glide
    return PlasticityState, GridArray, FieldMover, Dyn3, Dyn2, Glide


def run_case(name, shape, sigma_f, seed, steps, mu=1.0, nu=0.3, Lambda=0, cfl=0.25,
             load_rate=None, store_fields=True, t_end=1e30, glide=False, samples=0):
    """One reference run. ``samples`` > 0 makes a compact fixture: no whole
    fields, but the 9 components of that many seeded sample cells and per-component sums and sums
    of squares after the first and the last step, plus the initial field's sums as a check that
    the generator reproduces it."""
    PlasticityState, GridArray, FieldMover, Dyn3, Dyn2, Glide = _import_reference()
    sys.path.insert(0, os.path.join(REPO, "cuda-plasticity_b200"))
    from cdd.initial import gaussian_random_field

    beta0 = gaussian_random_field(shape, sigma_f, 0.05, seed)
    shape = tuple(shape)
    mod = Glide if glide else (Dyn3 if len(shape) == 3 else Dyn2)
    kw = {} if glide else {"Lambda": Lambda}

    if load_rate is None:
        dynamics = mod.BetaPDynamics(**kw)
    else:
        rate = np.asarray(load_rate, dtype=np.float64)

        class LoadedDynamics(mod.BetaPDynamics):
            """RunPython.py L21-26/L35-50 loading, with the state's own mu and nu."""
            def GetSigma(self, state, time):
                sigma = state.CalculateSigma()
                lamb = 2. * state.mu * state.nu / (1. - 2. * state.nu)
                eps = rate * time
                tr = eps[0] + eps[1] + eps[2]
                for i, a in enumerate("xyz"):
                    sigma[a, a] += lamb * tr + 2. * state.mu * eps[i]
                return sigma
        dynamics = LoadedDynamics(**kw)

    def make_state(arr):
        st = PlasticityState.PlasticityState(shape, mu=mu, nu=nu)
        for c, comp in enumerate(COMPONENTS):
            st.betaP[comp] = GridArray.GridArray(arr[c].copy())
        return st

    def to_array(st):
        return np.stack([np.asarray(st.betaP[comp]) for comp in COMPONENTS])

    def observables(st):
        e = float(np.sum(st.CalculateElasticEnergy()))
        m = float(np.asarray(st.betaP["z", "z"]).mean())
        return e, m

    out = {"shape": np.array(shape), "sigma_f": sigma_f, "seed": seed, "mu": mu, "nu": nu,
           "Lambda": Lambda, "cfl": cfl, "glide": int(glide),
           "load_rate": np.zeros(3) if load_rate is None else np.asarray(load_rate, float)}
    if samples:
        rs = np.random.default_rng(10_000 + seed)
        n_cells = int(np.prod(shape))
        idx = np.sort(rs.choice(n_cells, size=samples, replace=False))
        out["sample_idx"] = idx
        out["beta0_sum"] = beta0.reshape(9, -1).sum(axis=1)
        out["beta0_sumsq"] = (beta0.reshape(9, -1) ** 2).sum(axis=1)

        def record(tag, arr):
            flat = arr.reshape(9, -1)
            out["sample_" + tag] = flat[:, idx].copy()
            out["sum_" + tag] = flat.sum(axis=1)
            out["sumsq_" + tag] = (flat ** 2).sum(axis=1)
    state = make_state(beta0)
    t0 = time.time()
    sig = state.CalculateSigma()
    rhs, speed = dynamics.CalculateFlux(0.0, state, CFLCondition=True)
    if store_fields:
        out["beta0"] = beta0
        out["sigma"] = np.stack([np.asarray(sig[comp]) for comp in COMPONENTS])
        out["rhs"] = np.stack([np.asarray(rhs[comp]) for comp in COMPONENTS])
        out["speed"] = np.asarray(speed)
    mover = FieldMover.TVDRungeKutta_FieldMover(CFLsafeFactor=cfl)
    t = 0.0
    energies, means, dts = [], [], []
    e, m = observables(state)
    energies.append(e)
    means.append(m)
    for n in range(steps):
        state, dt = mover.CalculateOneAdaptiveTimeStep(t, state, dynamics, t_end)
        t += dt
        dts.append(dt)
        e, m = observables(state)
        energies.append(e)
        means.append(m)
        if store_fields and n == 0:
            out["beta1"] = to_array(state)
        if samples and n == 0:
            record("step1", to_array(state))
        print("  %s step %d dt=%.6e %.0fs" % (name, n + 1, dt, time.time() - t0), flush=True)
    final = to_array(state)
    if samples:
        record("final", final)
    if store_fields:
        out["beta_final"] = final
    out["steps"] = steps
    out["dts"] = np.array(dts)
    out["t_final"] = t
    out["energy"] = np.array(energies)
    out["mean_zz"] = np.array(means)
    out["final_sum"] = final.reshape(9, -1).sum(axis=1)
    out["final_sumsq"] = (final.reshape(9, -1) ** 2).sum(axis=1)
    out["wall_s"] = time.time() - t0
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **out)
    print("%-16s shape=%-14s steps=%-4d wall=%.1fs -> %s"
          % (name, shape, steps, out["wall_s"], os.path.relpath(path, REPO)))


# ---- the CUDA solver's file formats: the reference's own writer and reader, run from their source
# text (their modules do not import under Python 3: RunCUDA.py needs simplejson and Configure,
# FieldInitializer.py state classes and scipy names that are gone), with two more mechanical
# patches: (vii) ``numpy.fromstring(`` -> ``numpy.frombuffer(`` (binary fromstring is removed in
# numpy 2) and (viii) ``tp = range(dim)`` -> ``tp = list(range(dim))`` (a Python-3 range has no
# reverse()).
IO_PATCHES = [("numpy.fromstring(", "numpy.frombuffer("), ("tp = range(dim)", "tp = list(range(dim))")]


def _reference_function(reference, rel, name, patches=()):
    with open(os.path.join(reference, "Plasticity", rel)) as f:
        src = f.read().expandtabs(8)
    m = re.search(r"^def %s\(.*?(?=^\S)" % name, src, flags=re.M | re.S)
    text = _patch(m.group(0))
    for a, b in patches:
        text = text.replace(a, b)
    return text


def run_io_case(reference, name="io_formats"):
    """convertStateToCUDA (RunCUDA.py L9-22) writes .ics bytes of seeded states; .plas files of
    three frames [t][field] are framed as ContinueWriteMatrix does (assist.h L164-192: the time in
    the data type, then the field in the .ics layout); LoadStateRaw (FieldInitializer.py L61-103)
    reads them back (last frame, and the first frame with t >= 0.15), in float64 and float32."""
    import tempfile
    PlasticityState, GridArray = _import_reference()[:2]
    ns = {"numpy": np, "PlasticityState": PlasticityState, "GridArray": GridArray}
    exec(_reference_function(reference, "RunCUDA.py", "convertStateToCUDA"), ns)
    exec(_reference_function(reference, "FieldInitializers/FieldInitializer.py", "ReformatState"), ns)
    exec(_reference_function(reference, "FieldInitializers/FieldInitializer.py", "LoadStateRaw", IO_PATCHES), ns)
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        for dim, N, seed in ((3, 8, 21), (2, 12, 22)):
            shape = (N,) * dim
            rng = np.random.default_rng(seed)
            fields = [rng.standard_normal((9,) + shape) for _ in range(3)]
            times = [0.1, 0.2, 0.3]
            ics = []
            for k, f in enumerate(fields):
                st = PlasticityState.PlasticityState(shape)
                for c, comp in enumerate(COMPONENTS):
                    st.betaP[comp] = GridArray.GridArray(f[c].copy())
                path = os.path.join(tmp, "s%d.ics" % k)
                ns["convertStateToCUDA"](st, path)
                with open(path, "rb") as fh:
                    ics.append(fh.read())
            key = "%dd" % dim
            out["fields_" + key] = np.stack(fields)
            out["times_" + key] = np.array(times)
            out["ics_" + key] = np.frombuffer(ics[0], np.uint8)
            for dt in ("float64", "float32"):
                raw = b"".join(np.array([t], dt).tobytes() + np.frombuffer(b, np.float64).astype(dt).tobytes()
                               for t, b in zip(times, ics))
                path = os.path.join(tmp, "run_%s.plas" % dt)
                with open(path, "wb") as fh:
                    fh.write(raw)
                out["plas_%s_%s" % (key, dt)] = np.frombuffer(raw, np.uint8)
                for tag, tsel in (("last", None), ("t015", 0.15)):
                    t, st = ns["LoadStateRaw"](path, N, dim, time=tsel, dtype=dt)
                    out["load_%s_%s_%s_t" % (key, dt, tag)] = np.asarray(t, dtype=np.float64).reshape(-1)
                    out["load_%s_%s_%s" % (key, dt, tag)] = np.stack(
                        [np.asarray(st.betaP[comp]) for comp in COMPONENTS])
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **out)
    print("%-16s -> %s" % (name, os.path.relpath(path, REPO)))


def run_observables_case(name="observables"):
    """The field observables of PlasticityState (CalculateBetaElastic L357-390, CalculateRotationField
    L435-446, CalculateRotationRodrigues L447-475 with source 'betaP', CalculateRhoFourier L264-304)
    of seeded fields: a cubic and a non-cubic 3-D grid and a 2-D grid."""
    PlasticityState, GridArray = _import_reference()[:2]
    sys.path.insert(0, os.path.join(REPO, "cuda-plasticity_b200"))
    from cdd.initial import gaussian_random_field
    out = {}
    for key, shape, seed in (("c", (8, 8, 8), 41), ("a", (6, 8, 12), 42), ("2d", (16, 16), 43)):
        beta = gaussian_random_field(shape, 0.06, 0.05, seed)
        st = PlasticityState.PlasticityState(shape, mu=1.0, nu=0.3)
        for c, comp in enumerate(COMPONENTS):
            st.betaP[comp] = GridArray.GridArray(beta[c].copy())
        stack9 = lambda f: np.stack([np.asarray(f[comp]) for comp in COMPONENTS])
        out["beta_" + key] = beta
        out["betaE_" + key] = stack9(st.CalculateBetaElastic())
        out["rot_" + key] = stack9(st.CalculateRotationField())
        rod = st.CalculateRotationRodrigues()
        out["rod_" + key] = np.stack([np.asarray(rod[a]) for a in "xyz"])
        out["rho_" + key] = stack9(st.CalculateRhoFourier())
        # the 'sinK' tools (FourierSpaceTools with func=sin) and the Rodrigues vector from rho
        out["betaE_sink_" + key] = stack9(st.CalculateBetaElastic(type='sinK'))
        out["rot_sink_" + key] = stack9(st.CalculateRotationField(type='sinK'))
        rod = st.CalculateRotationRodrigues(type='sinK')
        out["rod_sink_" + key] = np.stack([np.asarray(rod[a]) for a in "xyz"])
        out["rho_sink_" + key] = stack9(st.CalculateRhoFourier(type='sinK'))
        for tag, typ in (("rodrho_", 'k'), ("rodrho_sink_", 'sinK')):
            rod = st.CalculateRotationRodrigues(type=typ, source='rho')
            out[tag + key] = np.stack([np.asarray(rod[a]) for a in "xyz"])
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **out)
    print("%-16s -> %s" % (name, os.path.relpath(path, REPO)))


def run_vacancy_case(name="vacancy"):
    """The vacancy-coupled dynamics (BetaP_VacancyDynamics, VacancyDynamics.py) stepped by
    OperatorSplittingTVDRK_FieldMover.CalculateOneAdaptiveTimeStep (FieldMover.py L344-380): 3-D
    8^3 with the default dtBound 0.01, and 2-D 16^2 with dtBound 1 (the CFL step); 3 steps each.
    DecoupleState builds the beta^P state with PlasticityState's defaults mu 0.5, nu 0.3."""
    sys.path.insert(0, PATCHED)
    from Plasticity.PlasticityStates import VacancyState
    from Plasticity.FieldDynamics import VacancyDynamics
    from Plasticity.FieldMovers import FieldMover
    from Plasticity.GridArray import GridArray
    sys.path.insert(0, os.path.join(REPO, "cuda-plasticity_b200"))
    from cdd.initial import gaussian_random_field
    out = {"alpha": 0.5, "beta": 0.7, "gamma": 0.02, "mu": 0.5, "nu": 0.3, "cfl": 0.25}
    for key, shape, seed, bound in (("3d", (8, 8, 8), 51, 0.01), ("2d", (16, 16), 52, 1.0)):
        beta0 = gaussian_random_field(shape, 0.06, 0.05, seed)
        c0 = 0.01 * np.random.default_rng(seed).standard_normal(shape)
        st = VacancyState.VacancyState(shape, mu=0.5, nu=0.3)
        for c, comp in enumerate(COMPONENTS):
            st.betaP_V[comp] = GridArray.GridArray(beta0[c].copy())
        st.betaP_V["s", "s"] = GridArray.GridArray(c0.copy())
        dyn = VacancyDynamics.BetaP_VacancyDynamics(alpha=out["alpha"], beta=out["beta"], gamma=out["gamma"])
        mover = FieldMover.OperatorSplittingTVDRK_FieldMover(CFLsafeFactor=out["cfl"], dtBound=bound)
        t, betas, cs, dts = 0.0, [], [], []
        for _ in range(3):
            st, dt = mover.CalculateOneAdaptiveTimeStep(t, st, dyn, 1e30)
            t += dt
            betas.append(np.stack([np.asarray(st.betaP_V[comp]) for comp in COMPONENTS]))
            cs.append(np.asarray(st.betaP_V["s", "s"]).copy())
            dts.append(dt)
        out["beta0_" + key], out["c0_" + key], out["dt_bound_" + key] = beta0, c0, bound
        out["betas_" + key], out["cs_" + key], out["dts_" + key] = np.stack(betas), np.stack(cs), np.array(dts)
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **out)
    print("%-16s -> %s" % (name, os.path.relpath(path, REPO)))


def run_initializer_case(reference, name="initializer"):
    """The reference's random initial condition, GaussianRandomInitializer (FieldInitializer.py
    L153-209) with its ResizeState / ResampleArray (L421-442), run from their source text (the
    module imports state classes that are not part of the time-step path). Names the module takes
    from old scipy (random, sqrt, pi, exp) are numpy's, which is what those scipy names were."""
    PlasticityState, GridArray = _import_reference()[:2]
    sys.path.insert(0, PATCHED)
    from Plasticity.PlasticityStates import VacancyState
    from Plasticity.GridArray import FourierSpaceTools
    import copy as copy_module
    ns = {"numpy": np, "random": np.random, "fft": np.fft, "sqrt": np.sqrt, "pi": np.pi, "exp": np.exp,
          "copy": copy_module, "PlasticityState": PlasticityState, "VacancyState": VacancyState,
          "FourierSpaceTools": FourierSpaceTools, "GridArray": GridArray}
    exec(_reference_function(reference, "FieldInitializers/FieldInitializer.py", "ReformatState"), ns)
    exec(_reference_function(reference, "FieldInitializers/FieldInitializer.py", "ResampleArray"), ns)
    exec(_reference_function(reference, "FieldInitializers/FieldInitializer.py", "ResizeState"), ns)
    exec(_reference_function(reference, "FieldInitializers/FieldInitializer.py", "GaussianRandomInitializer"), ns)
    out = {}
    for key, shape, sigma, seed, vac in (("r3", (16, 16, 16), 0.2, 3, None), ("n2", (128, 128), 0.2, 5, None),
                                         ("r2", (64, 64), 0.1, 7, None), ("v2", (16, 16), 0.2, 9, 0.5)):
        st = ns["GaussianRandomInitializer"](shape, sigma, seed, vacancy=vac)
        field = st.GetOrderParameterField()
        out["shape_" + key] = np.array(shape)
        out["sigma_" + key] = sigma
        out["seed_" + key] = seed
        out["vacancy_" + key] = -1.0 if vac is None else vac
        out["components_" + key] = np.array(["".join(c) for c in field.components])
        out["field_" + key] = np.stack([np.asarray(field[c]) for c in field.components])
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **out)
    print("%-16s -> %s" % (name, os.path.relpath(path, REPO)))


CASES = {
    # one flux, one step and 10 steps of 3-D glide+climb dynamics
    "g3d_16": dict(shape=(16, 16, 16), sigma_f=0.05, seed=1, steps=10),
    # 2-D twin modules, 20 steps
    "g2d_32": dict(shape=(32, 32), sigma_f=0.05, seed=2, steps=20),
    # non-cubic 3-D grid: the k tables use each axis' own size, Dx uses the last axis
    "g3d_aniso": dict(shape=(8, 12, 16), sigma_f=0.06, seed=3, steps=3),
    # glide-projected dynamics (Lambda = 1)
    "g3d_lambda": dict(shape=(12, 12, 12), sigma_f=0.06, seed=4, steps=3, Lambda=1),
    # applied strain rate diag(-0.025, -0.025, 0.05), mu = 1
    "g3d_load": dict(shape=(12, 12, 12), sigma_f=0.06, seed=5, steps=3,
                     load_rate=(-0.025, -0.025, 0.05)),
    # 2-D run at mixed-radix size (48 = 16 * 3) and a clamped end time
    "g2d_48_tend": dict(shape=(48, 48), sigma_f=0.05, seed=6, steps=6, t_end=0.004),
    # glide-only dynamics (CentralUpwindHJBetaPGlideOnlyDynamics.py), 3-D with load and 2-D
    "g3d_glide": dict(shape=(12, 12, 12), sigma_f=0.06, seed=7, steps=3, glide=True,
                      load_rate=(-0.025, -0.025, 0.05)),
    "g2d_glide": dict(shape=(32, 32), sigma_f=0.05, seed=8, steps=5, glide=True),
    # config-1 style curves: 2-D 128^2, sigma 0.05, no load, 100 steps (observables only)
    "c1_2d_128": dict(shape=(128, 128), sigma_f=0.05, seed=11, steps=100, store_fields=False),
    # config-2 style curves at reduced size: 3-D 32^3, sigma 0.04, applied strain rate, 40 steps
    "c2_3d_32": dict(shape=(32, 32, 32), sigma_f=0.04, seed=12, steps=40, store_fields=False,
                     load_rate=(-0.025, -0.025, 0.05)),
    # config-2 fields at 64^3 and 128^3 (sigma 0.04, applied strain rate), 10 steps, compact
    "c2_3d_64": dict(shape=(64, 64, 64), sigma_f=0.04, seed=13, steps=10, store_fields=False,
                     load_rate=(-0.025, -0.025, 0.05), samples=4096),
    "c2_3d_128": dict(shape=(128, 128, 128), sigma_f=0.04, seed=14, steps=10, store_fields=False,
                      load_rate=(-0.025, -0.025, 0.05), samples=4096),
}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("CDD_REFERENCE"),
                    help="path of the reference checkout (or set CDD_REFERENCE)")
    ap.add_argument("--only", default=None)
    args = ap.parse_args()
    if not args.reference:
        ap.error("give --reference PATH (the reference checkout) or set CDD_REFERENCE")
    build_patched_copy(args.reference)
    if args.only in (None, "io_formats"):
        run_io_case(args.reference)
    if args.only in (None, "observables"):
        run_observables_case()
    if args.only in (None, "vacancy"):
        run_vacancy_case()
    if args.only in (None, "initializer"):
        run_initializer_case(args.reference)
    for name, kw in CASES.items():
        if args.only and name != args.only:
            continue
        run_case(name, **kw)


if __name__ == "__main__":
    main()
