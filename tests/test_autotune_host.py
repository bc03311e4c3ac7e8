"""Host logic of the launch-shape autotuner (cdd/autotune.py): candidate values per knob and the
JSON cache."""
import json

from cdd import autotune


def test_candidates_per_knob():
    cur = {"fft_radix": 16, "rows_lines": 16, "mid_cols": 16, "green_cols": 4, "stencil_planes": 2}
    assert autotune.candidates("fft_radix", (64, 64, 64), cur) == [16, 8, 4]
    assert autotune.candidates("stencil_planes", (64, 64, 64), cur) == [2, 4, 8, 16, 32, 64]
    assert autotune.candidates("stencil_planes", (12, 64, 64), cur) == [2, 4, 8]
    assert autotune.candidates("stencil_planes", (64, 64), cur) == []
    assert autotune.candidates("mid_cols", (64, 64), cur) == []
    assert autotune.candidates("mid_cols", (64, 64, 64), cur) == [8, 16, 32]
    assert autotune.candidates("green_cols", (64, 64, 64), {"green_cols": 1}) == [1, 2]
    assert autotune.candidates("rows_lines", (64, 64, 64), {"rows_lines": 0}) == []


def test_cache_round_trip(tmp_path, monkeypatch):
    path = tmp_path / "sub" / "tune.json"
    monkeypatch.setenv("CDD_TUNE_CACHE", str(path))
    assert autotune.load_cache() == {}
    key = autotune.cache_key("NVIDIA B200", "f32", (256, 256, 256))
    assert key == "NVIDIA B200|f32|256x256x256"
    autotune.save_cache({key: {"tuning": {"fft_radix": 8}, "ms_per_step": 1.0}})
    assert json.loads(path.read_text())[key]["tuning"] == {"fft_radix": 8}
    assert autotune.load_cache()[key]["ms_per_step"] == 1.0
    path.write_text("not json")
    assert autotune.load_cache() == {}
