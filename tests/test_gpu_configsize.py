"""Ten adaptive TVD-RK3 steps at the config-2 grid sizes (64^3 and 128^3, sigma 0.04, applied
strain rate diag(-0.025, -0.025, 0.05), mu 1, nu 0.3, CFL 0.25) in FP64 through the C ABI, against
compact fixtures the reference itself produced on the same seeded fields
(tests/golden/make_golden.py: TVDRungeKutta_FieldMover.CalculateOneAdaptiveTimeStep,
FieldMover.py L61-141, with CentralUpwindHJBetaPDynamics3D.BetaPDynamics(Lambda=0) and the
RunPython.py loading). The fixtures hold the dt sequence, the energy and mean-strain curves,
per-component sums and sums of squares and 4096 sampled cells after steps 1 and 10.

Each case runs twice: with 16-plane stencil chunks (the TMA march of the benchmark's 256^3 plans)
and with the built-in chunking, so the production march at these sizes is pinned to the reference.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import cdd
from conftest import golden_path


def _check_state(plan, beta, g, tag):
    fin = plan.field_view(beta, 0).cpu().numpy().reshape(9, -1)
    idx = g["sample_idx"]
    got = fin[:, idx]
    want = g["sample_" + tag]
    # 1e-10 relative to each component's sample norm (the north-star FP64 bar)
    for c in range(9):
        err = np.linalg.norm(got[c] - want[c]) / np.linalg.norm(want[c])
        assert err < 1e-10, (tag, c, err)
    np.testing.assert_allclose(fin.sum(axis=1), g["sum_" + tag], rtol=1e-10,
                               atol=1e-10 * np.abs(g["sum_" + tag]).max())
    np.testing.assert_allclose((fin ** 2).sum(axis=1), g["sumsq_" + tag], rtol=1e-10)


@pytest.mark.parametrize("planes", [16, 0])
@pytest.mark.parametrize("name", ["c2_3d_64", "c2_3d_128"])
def test_config2_ten_steps_match_reference(name, planes):
    g = np.load(golden_path(name))
    shape = tuple(int(v) for v in g["shape"])
    b0 = cdd.gaussian_random_field(shape, float(g["sigma_f"]), 0.05, int(g["seed"]))
    np.testing.assert_allclose(b0.reshape(9, -1).sum(axis=1), g["beta0_sum"], rtol=0, atol=1e-12)
    np.testing.assert_allclose((b0.reshape(9, -1) ** 2).sum(axis=1), g["beta0_sumsq"], rtol=1e-14)
    inst = cdd.Instance(shape, mu=float(g["mu"]), nu=float(g["nu"]), Lambda=float(g["Lambda"]),
                        cfl=float(g["cfl"]), load_rate=tuple(float(v) for v in g["load_rate"]))
    plan = cdd.Plan([inst], "f64", tuning=[{"stencil_planes": planes}])
    if planes:
        assert plan.tuning(0)["stencil_planes"] == planes
    beta = plan.pack([b0])
    plan.set_time(0.0, 1e30)
    e, m = plan.observables(beta)
    energies, means, dts = [e[0]], [m[0]], []
    for n in range(int(g["steps"])):
        plan.step(beta)
        plan.check_status()
        _, dt, _ = plan.get_time()
        dts.append(dt[0])
        e, m = plan.observables(beta)
        energies.append(e[0])
        means.append(m[0])
        if n == 0:
            _check_state(plan, beta, g, "step1")
    np.testing.assert_allclose(dts, g["dts"], rtol=1e-12)
    np.testing.assert_allclose(energies, g["energy"], rtol=1e-10)
    np.testing.assert_allclose(means, g["mean_zz"], rtol=1e-10, atol=1e-15)
    _check_state(plan, beta, g, "final")
