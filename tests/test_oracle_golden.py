"""Pin the CPU oracle against golden vectors produced by the reference's own Python path.

The fixtures come from tests/golden/make_golden.py (reference modules, mechanically patched to
Python 3, run on seeded inputs). The oracle follows the reference's operation order, so the
expected agreement is exact; the tolerance below only absorbs libm/FFT build differences.
"""
import numpy as np
import pytest

import cdd_oracle as O
from conftest import golden_path

TOL = 1e-13
FIELD_CASES = ["g3d_16", "g2d_32", "g3d_aniso", "g3d_lambda", "g3d_load", "g2d_48_tend", "g3d_glide",
               "g2d_glide"]
T_END = {"g2d_48_tend": 0.004}


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def params_of(g):
    lr = g["load_rate"]
    return O.Params(mu=float(g["mu"]), nu=float(g["nu"]), Lambda=int(g["Lambda"]),
                    cfl=float(g["cfl"]), load_rate=lr if np.any(lr) else None,
                    glide=bool(int(g["glide"])) if "glide" in g.files else False)


@pytest.mark.parametrize("name", FIELD_CASES)
def test_stress_flux_step(name):
    g = np.load(golden_path(name))
    p = params_of(g)
    b = g["beta0"]
    assert rel(O.stress(b, p.mu, p.nu), g["sigma"]) < TOL
    rhs, speed = O.full_flux(b, 0.0, p)
    assert rel(rhs, g["rhs"]) < TOL
    assert rel(speed, g["speed"]) < TOL
    b1, dt = O.rk3_step(b, 0.0, T_END.get(name, 1e30), p)
    assert abs(dt - g["dts"][0]) <= 1e-15 * abs(g["dts"][0])
    assert rel(b1, g["beta1"]) < TOL


@pytest.mark.parametrize("name", FIELD_CASES)
def test_multistep_and_observables(name):
    g = np.load(golden_path(name))
    p = params_of(g)
    b, t = g["beta0"], 0.0
    t_end = T_END.get(name, 1e30)
    energies = [O.elastic_energy(b, p.mu, p.nu)]
    for _ in range(int(g["steps"])):
        b, dt = O.rk3_step(b, t, t_end, p)
        t += dt
        energies.append(O.elastic_energy(b, p.mu, p.nu))
    assert rel(b, g["beta_final"]) < 1e-12
    assert abs(t - float(g["t_final"])) <= 1e-14 * max(abs(t), 1e-300)
    np.testing.assert_allclose(energies, g["energy"], rtol=1e-12)
    assert abs(O.mean_strain_zz(b) - g["mean_zz"][-1]) < 1e-15


def test_clamped_end_time_reached():
    g = np.load(golden_path("g2d_48_tend"))
    assert abs(float(g["t_final"]) - 0.004) < 1e-18
    assert g["dts"][-1] == 0.0


def test_uniform_beta_known_answer():
    """Uniform beta: sigma is the mean-field stress, rhs = 0, speed = 3 ME (3-D)."""
    b0 = np.arange(1, 10, dtype=float).reshape(9, 1, 1, 1) * 0.01 * np.ones((9, 8, 8, 8))
    mu, nu = 1.0, 0.3
    lamb = 2 * mu * nu / (1 - 2 * nu)
    sig = O.stress(b0, mu, nu)
    m = b0[:, 0, 0, 0].reshape(3, 3)
    expect = -lamb * np.trace(m) * np.eye(3) - mu * (m + m.T)
    np.testing.assert_allclose(sig[:, 0, 0, 0].reshape(3, 3), expect, atol=1e-15)
    rhs, speed = O.flux(b0, sig)
    assert np.all(rhs == 0)
    np.testing.assert_allclose(speed, 3 * O.ME)


@pytest.mark.parametrize("name,steps", [("c1_2d_128", 100), ("c2_3d_32", 40)])
def test_curves_short_prefix(name, steps):
    """First steps of the long-run observable curves (the full curves run in the GPU tests)."""
    import os
    path = golden_path(name)
    if not os.path.exists(path):
        pytest.skip("fixture not generated")
    g = np.load(path)
    from cdd.initial import gaussian_random_field
    shape = tuple(int(v) for v in g["shape"])
    b = gaussian_random_field(shape, float(g["sigma_f"]), 0.05, int(g["seed"]))
    p = params_of(g)
    n = 3 if len(shape) == 2 else 1
    t = 0.0
    for k in range(n):
        b, dt = O.rk3_step(b, t, 1e30, p)
        t += dt
        assert abs(dt - g["dts"][k]) <= 1e-14 * dt
    assert abs(O.elastic_energy(b, p.mu, p.nu) - g["energy"][n]) <= 1e-12 * abs(g["energy"][n])
