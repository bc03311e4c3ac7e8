"""The oracle's stress against the analytic stress of single Fourier modes (tests/plane_wave.py)."""
import numpy as np
import pytest

import cdd_oracle as O
import plane_wave as PW


@pytest.mark.parametrize("shape,m", [((16, 16, 16), (1, 2, 3)), ((8, 12, 16), (2, -1, 5)), ((16, 16, 16), (0, 0, 4))])
def test_oracle_stress_of_a_single_mode(shape, m):
    rng = np.random.default_rng(5)
    B = rng.standard_normal((3, 3))
    got = O.stress(PW.field(shape, m, B), 1.3, 0.27)
    want = PW.stress(shape, m, B, 1.3, 0.27)
    assert np.abs(got - want).max() < 1e-12 * np.abs(want).max()
