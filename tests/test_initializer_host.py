"""The reference's random initial condition (GaussianRandomInitializer, FieldInitializer.py L153-209,
with ResizeState L430-442) through the facade, against states the reference itself produced from
the same seeds (tests/golden/initializer.npz, made by tests/golden/make_golden.py)."""
import numpy as np
import pytest

from conftest import golden_path

from Plasticity.FieldInitializers import FieldInitializer

FIX = golden_path("initializer")


@pytest.mark.parametrize("key", ["r3", "n2", "r2", "v2"])
def test_gaussian_random_initializer_matches_reference(key):
    g = np.load(FIX)
    shape = tuple(int(v) for v in g["shape_" + key])
    vac = float(g["vacancy_" + key])
    st = FieldInitializer.GaussianRandomInitializer(shape, float(g["sigma_" + key]), int(g["seed_" + key]),
                                                    vacancy=None if vac < 0 else vac)
    field = st.GetOrderParameterField()
    assert ["".join(c) for c in field.components] == [str(c) for c in g["components_" + key]]
    got = np.stack([np.asarray(field[c]) for c in field.components])
    want = g["field_" + key]
    assert got.shape == want.shape
    # same numpy generator, FFTs and scipy resampling as the reference: equal to the last bit
    np.testing.assert_array_equal(got, want)
    assert st.gridShape == shape


def test_resize_state_keeps_band_limited_content():
    """A single Fourier mode resampled from 16^2 to 32^2 keeps its values at the shared points."""
    from Plasticity.PlasticityStates import PlasticityState
    st = PlasticityState.PlasticityState((16, 16))
    x = np.arange(16) / 16.0
    wave = np.sin(2 * np.pi * 3 * x)[:, None] * np.cos(2 * np.pi * 2 * x)[None, :]
    for c in st.betaP.components:
        st.betaP[c] = wave
    big = FieldInitializer.ResizeState(st, 32, Dim=2)
    assert big.gridShape == (32, 32)
    np.testing.assert_allclose(np.asarray(big.betaP["x", "y"])[::2, ::2], wave, atol=1e-12)
