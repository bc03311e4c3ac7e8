"""Host-side parts of the Plasticity facades (no GPU): k tables, limited derivatives, field
algebra and the raw-file formats, against the oracle and the reference's conventions."""
import numpy as np
import pytest

import cdd_oracle as O
from conftest import golden_path

from Plasticity.Fields import Fields
from Plasticity.GridArray import FourierSpaceTools
from Plasticity.PlasticityStates import PlasticityState
from Plasticity.FieldDynamics.CentralUpwindHJ3D import FindDerivatives
from Plasticity.Observers import Observer
from Plasticity.FieldInitializers import FieldInitializer


@pytest.mark.parametrize("shape", [(8, 12, 16), (16, 16, 16), (32, 32), (48, 20)])
def test_fourier_tools_match_reference_tables(shape):
    K = FourierSpaceTools.FourierSpaceTools(shape)
    k, kSq, kSqSq, kmask = O.k_tables(shape)
    np.testing.assert_array_equal(np.asarray(K.kx), k[0])
    np.testing.assert_array_equal(np.asarray(K.ky), k[1])
    np.testing.assert_array_equal(np.asarray(K.kSq), kSq)
    np.testing.assert_array_equal(np.asarray(K.kmask), kmask)


@pytest.mark.parametrize("name", ["g3d_16", "g2d_32", "g3d_aniso"])
def test_limited_derivatives_match_oracle(name):
    """(The facade's k-space observables run on the GPU: tests/test_gpu_observables.py.)"""
    g = np.load(golden_path(name))
    shape = tuple(int(v) for v in g["shape"])
    st = PlasticityState.PlasticityState(shape, mu=float(g["mu"]), nu=float(g["nu"]))
    st.betaP = Fields.from_stack(shape, g["beta0"])
    for axis in range(len(shape)):
        dp, dm = FindDerivatives(st.betaP, axis)
        rp, rm = O.find_derivatives(g["beta0"], axis, 1.0 / shape[-1])
        np.testing.assert_allclose(dp.stack(), rp, rtol=0, atol=1e-12 * np.abs(rp).max())
        np.testing.assert_allclose(dm.stack(), rm, rtol=0, atol=1e-12 * np.abs(rm).max())


def test_field_algebra_and_component_order():
    f = Fields.TensorField((4, 4))
    assert f.components == [(a, b) for a in "xyz" for b in "xyz"]
    arr = np.arange(9 * 16, dtype=float).reshape(9, 4, 4)
    f = Fields.from_stack((4, 4), arr)
    g = 2.0 * f - f / 2.0 + 1.0
    np.testing.assert_allclose(g.stack(), 1.5 * arr + 1.0)
    s = Fields.SymmetricTensorField((4, 4))
    s['y', 'x'] = np.ones((4, 4))
    assert np.all(s['x', 'y'] == 1.0)


def test_raw_record_and_load_roundtrip(tmp_path):
    """RecordStateObserverRaw writes [t][components C-order]; LoadStateRaw reads the last frame
    and, like the reference, treats each component as first-axis-fastest (transposes it)."""
    shape = (6, 6, 6)
    rng = np.random.default_rng(0)
    arr = rng.standard_normal((9,) + shape)
    st = PlasticityState.PlasticityState(shape)
    st.betaP = Fields.from_stack(shape, arr)
    path = str(tmp_path / "run.plas")
    obs = Observer.RecordStateObserverRaw(filename=path)
    obs.Update(0.5, st)
    obs.Update(1.25, st)
    obs.file.close()
    raw = np.fromfile(path, dtype=np.float64)
    assert raw.size == 2 * (1 + 9 * 216)
    assert raw[0] == 0.5 and raw[1 + 9 * 216] == 1.25
    t, loaded = FieldInitializer.LoadStateRaw(path, 6, 3)
    assert float(t[0]) == 1.25
    got = loaded.betaP.stack()
    for c in range(9):
        np.testing.assert_array_equal(got[c], arr[c].transpose(2, 1, 0))
