"""The reference CUDA solver's file formats on the host: the oracle's restatement and the facade's
LoadStateRaw against the reference's own convertStateToCUDA / LoadStateRaw outputs
(tests/golden/io_formats.npz, made by tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

import cdd_oracle as O
from conftest import golden_path

G = np.load(golden_path("io_formats"))


@pytest.mark.parametrize("key", ["3d", "2d"])
def test_ics_bytes_match_convertStateToCUDA(key):
    field = G["fields_" + key][0]
    assert O.ics_bytes(field) == G["ics_" + key].tobytes()
    shape = field.shape[1:]
    back = O.from_file_layout(np.frombuffer(G["ics_" + key].tobytes(), np.float64), shape)
    assert np.array_equal(back, field)


@pytest.mark.parametrize("key", ["3d", "2d"])
@pytest.mark.parametrize("dt", ["float64", "float32"])
def test_plas_frames_match_LoadStateRaw(key, dt):
    fields, times = G["fields_" + key], G["times_" + key]
    raw = b"".join(O.plas_frame_bytes(t, f, dt) for t, f in zip(times, fields))
    assert raw == G["plas_%s_%s" % (key, dt)].tobytes()
    shape = fields.shape[2:]
    for tag, tsel in (("last", None), ("t015", 0.15)):
        t, f = O.read_plas(raw, shape, dt, time=tsel)
        assert t == G["load_%s_%s_%s_t" % (key, dt, tag)][0]
        assert np.array_equal(f, G["load_%s_%s_%s" % (key, dt, tag)])


@pytest.mark.parametrize("key", ["3d", "2d"])
def test_facade_LoadStateRaw_matches_reference(key, tmp_path):
    from Plasticity.FieldInitializers import FieldInitializer
    fields = G["fields_" + key]
    N, dim = fields.shape[2], fields.ndim - 2
    for dt in ("float64", "float32"):
        path = os.path.join(tmp_path, "run.plas")
        with open(path, "wb") as f:
            f.write(G["plas_%s_%s" % (key, dt)].tobytes())
        for tag, tsel in (("last", None), ("t015", 0.15)):
            t, st = FieldInitializer.LoadStateRaw(path, N, dim, time=tsel, dtype=dt)
            got = np.stack([np.asarray(st.betaP[c]) for c in O.COMPONENTS])
            assert float(np.asarray(t).reshape(-1)[0]) == G["load_%s_%s_%s_t" % (key, dt, tag)][0]
            assert np.array_equal(got, G["load_%s_%s_%s" % (key, dt, tag)])
