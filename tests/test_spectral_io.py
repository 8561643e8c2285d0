"""Spectral snapshot / checkpoint IO in the reference's file format
(src/spectral/io.jl), on CPU with host arrays: byte-exact round trip, the
TOML sidecar's keys, the .bin byte layout (column-major compact state,
components one after another), checkpoint listing and retention, the
snapshot saver's numbering and restart skip, and spectral_from_rfft against
the oracle's truncation."""
import math
import os
import tomllib
from collections import namedtuple

import numpy as np
import pytest

import spectral_oracle as SO

sio = pytest.importorskip("distributednavierstokes_b200.spectral_io")

State = namedtuple("State", "uh t n")


class Setup:
    def __init__(self, n, kcut=None, l=2 * math.pi, visc=1e-3):
        self.n, self.l, self.visc = n, l, visc
        self.kcut = n // 3 if kcut is None else kcut
        self.m = 2 * self.kcut + 1


def test_round_trip_and_sidecar(tmp_path):
    s = Setup(12)
    O = SO.Spectral(12)
    uh = O.random(3)
    prefix = os.path.join(tmp_path, "field")
    sio.spectral_save(prefix, uh, s, time=1.5, step=7, meta=dict(eref=[0.1, 0.2], tag="x"))
    assert sorted(os.listdir(tmp_path)) == ["field.bin", "field.toml"]
    with open(prefix + ".toml", "rb") as fh:
        d = tomllib.load(fh)
    assert d["format"] == "DistributedNavierStokes spectral state" and d["version"] == 1
    assert (d["n"], d["kcut"], d["m"], d["eltype"], d["data"]) == (12, 4, 9, "Float64", "field.bin")
    assert d["time"] == 1.5 and d["step"] == 7 and d["meta"] == dict(eref=[0.1, 0.2], tag="x")
    # byte layout: component c, then kz, ky, kx (kx fastest), re/im interleaved
    raw = np.fromfile(prefix + ".bin", dtype=np.float64)
    c, k, j, i = 1, 5, 2, 3
    off = 2 * (i + (s.kcut + 1) * (j + s.m * (k + s.m * c)))
    assert raw[off] == uh[c, k, j, i].real and raw[off + 1] == uh[c, k, j, i].imag
    u2 = np.zeros_like(uh)
    md = sio.spectral_load(u2, prefix, s)
    assert np.array_equal(u2, uh) and md == dict(time=1.5, step=7, meta=d["meta"])
    # another transform grid with the same retained modes loads; another kcut does not
    sio.spectral_load(np.zeros_like(uh), prefix, Setup(14, kcut=4))
    with pytest.raises(ValueError):
        sio.spectral_load(np.zeros_like(uh), prefix, Setup(18))


def test_checkpoints_and_snapshots(tmp_path):
    s = Setup(12)
    uh = SO.Spectral(12).random(1)
    prefix = os.path.join(tmp_path, "ck")
    stop = os.path.join(tmp_path, "STOP")
    proc = sio.checkpointer(prefix, interval=0.0, stopfile=stop, keep=2)
    for n in (3, 10, 25):
        assert proc(State(uh, 0.1 * n, n), s) is None
    lst = sio.checkpointlist(prefix)
    assert [os.path.basename(p) for p in lst] == ["ck_000000010", "ck_000000025"]
    assert sio.spectral_latest(prefix) == lst[-1]
    open(stop, "w").close()
    assert proc(State(uh, 3.0, 30), s) == "stop"
    snap = sio.snapshotsaver(os.path.join(tmp_path, "snap"), times=[0.5, 0.2, 1.0], stats=False,
                             tstart=0.3)
    for n, t in ((1, 0.25), (2, 0.5), (3, 0.75), (4, 1.0)):
        snap(State(uh, t, n), s)
    names = sorted(f for f in os.listdir(tmp_path) if f.startswith("snap"))
    assert names == ["snap_0002.bin", "snap_0002.toml", "snap_0003.bin", "snap_0003.toml"]


def test_from_rfft_matches_truncation():
    s = Setup(12)
    O = SO.Spectral(12)
    rng = np.random.default_rng(2)
    v = rng.standard_normal((3, 16, 16, 16))
    F = [np.fft.rfftn(v[c], axes=(0, 1, 2)) / 16 ** 3 for c in range(3)]
    uh = sio.spectral_from_rfft(O.zeros(), F, s)
    cf = np.array([j if j <= s.kcut else j - s.m for j in range(s.m)])
    assert np.array_equal(uh[2], F[2][np.ix_(cf % 16, cf % 16, np.arange(s.kcut + 1))])
    with pytest.raises(ValueError):
        sio.spectral_from_rfft(O.zeros(), [f[:8, :8, :5] for f in F], Setup(12))


def test_etacells_and_celldir():
    cells = sio.etacells(deta=[2.0, 4.0], eta=0.05, l=2 * math.pi, Ms=[64, 256, 128])
    # delta/h = deta * eta * M / l inside [2, 5]
    assert [(c["M"], c["deta"]) for c in cells] == [(128, 2.0), (256, 2.0), (64, 4.0), (128, 4.0)]
    assert cells[0]["dfac"] == float(f"{2.0 * 0.05 * 128 / (2 * math.pi):.4g}")
    c = dict(M=64, kernel="gaussian", dfac=2.0)
    assert sio.celldir("out", c, True) == os.path.join("out", "delta=2.0")
    assert sio.celldir("out", c, False) == os.path.join("out", "filter=gaussian", "M=64", "delta=2.0")
