"""The oracle's vacancy-coupled operator-splitting step against the reference's own
BetaP_VacancyDynamics + OperatorSplittingTVDRK_FieldMover (tests/golden/vacancy.npz)."""
import numpy as np
import pytest

import cdd_oracle as O
from conftest import golden_path

G = np.load(golden_path("vacancy"))


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


@pytest.mark.parametrize("key", ["3d", "2d"])
def test_oracle_vacancy_steps_match_reference(key):
    p = O.Params(mu=float(G["mu"]), nu=float(G["nu"]), cfl=float(G["cfl"]),
                 vacancy=(float(G["alpha"]), float(G["beta"]), float(G["gamma"])),
                 dt_bound=float(G["dt_bound_" + key]))
    beta, c, t = G["beta0_" + key], G["c0_" + key], 0.0
    for k in range(3):
        beta, c, dt = O.vacancy_step(beta, c, t, 1e30, p)
        t += dt
        assert dt == G["dts_" + key][k]
        assert rel(beta, G["betas_" + key][k]) < 1e-13
        assert rel(c, G["cs_" + key][k]) < 1e-13
