"""The ensemble's launch-shape autotuner (autotune.py) on the host, with the
GPU timing replaced by a synthetic cost: coordinate descent keeps a
candidate only when it gains more than 1 %, holds the other fields, and
the choices are cached per device name and box side."""
import json

import pytest

torch = pytest.importorskip("torch")

from distributednavierstokes_b200 import autotune  # noqa: E402


def fake_timer(calls):
    def _time_step(n, visc, tuning, steps, repeats, device):
        calls.append(dict(tuning))
        ms = 1.0
        if tuning.get("lines_z4") == 8:
            ms -= 0.10          # kept
        if tuning.get("lines_y") == 16:
            ms -= 0.005         # 0.5 %: below the threshold, not kept
        if (tuning.get("cell_bx"), tuning.get("cell_by")) == (32, 4):
            ms -= 0.20          # kept
        if tuning.get("lines_x") == 2:
            ms += 0.3           # slower: not kept
        return ms, dict(tuning)
    return _time_step


def test_coordinate_descent(monkeypatch):
    calls = []
    monkeypatch.setattr(autotune, "_time_step", fake_timer(calls))
    eff, ms, tried = autotune.tune(64, device="cpu")
    assert eff == {"lines_z4": 8, "cell_bx": 32, "cell_by": 4}
    assert abs(ms - 0.70) < 1e-12
    # the default plus one timing per candidate of every field
    assert len(calls) == 1 + sum(len(v) for v in autotune.CANDIDATES.values())
    assert tried["default"] == 1.0 and abs(tried["lines_y=16"] - 0.895) < 1e-12
    # later fields are tried on top of the earlier choices
    assert all(c.get("lines_z4") == 8 for c in calls[1 + len(autotune.CANDIDATES["lines_z4"]):])


def test_cache_per_device_and_side(monkeypatch, tmp_path):
    calls = []

    def fake_tune(n, visc, device=None, log=None, **kw):
        calls.append(n)
        return {"lines_z4": n // 8}, 0.1 * n, {"default": 0.1 * n}

    monkeypatch.setattr(autotune, "tune", fake_tune)
    monkeypatch.setattr(torch.cuda, "get_device_name", lambda device=None: "TestGPU")
    cache = str(tmp_path / "tuning.json")
    out, rep = autotune.tune_sizes([64, 32, 64], cache=cache, device="cpu")
    assert calls == [32, 64] and out == {32: {"lines_z4": 4}, 64: {"lines_z4": 8}}
    assert not rep[32]["cached"]
    with open(cache) as f:
        assert set(json.load(f)) == {"TestGPU|periodic|32", "TestGPU|periodic|64"}
    out2, rep2 = autotune.tune_sizes([32, 64], cache=cache, device="cpu")
    assert calls == [32, 64] and out2 == out and rep2[64]["cached"]
    autotune.tune_sizes([32], cache=cache, device="cpu", refresh=True)
    assert calls == [32, 64, 32]
    monkeypatch.setattr(torch.cuda, "get_device_name", lambda device=None: "OtherGPU")
    autotune.tune_sizes([32], cache=cache, device="cpu")
    assert calls == [32, 64, 32, 32]
