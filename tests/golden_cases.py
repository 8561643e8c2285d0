"""Golden-fixture cases: small runs whose oracle outputs are committed under
tests/golden/ (written by tests/golden/make_golden.py) and compared, in
tests/test_gpu_parity.py, with the CUDA library on the same inputs.

The first three are the reference's decomposition-invariance `runcase`
(test/mpitests.jl:158-198, single rank): periodic explicit, wall explicit,
wall implicit, 5 steps of 0.01, statistics sampled every 2 steps.  The last
one is a scaled-down version of the 64^3 channel benchmark case
(tanh-stretched walls, noise initial condition, CFL-adaptive).
"""
import math

import numpy as np

import refcases as R

CHANNEL_C1 = dict(lims=((0.0, 4 * math.pi), (-1.0, 1.0), (0.0, 4 * math.pi / 3)),
                  bc=("periodic", "wall", "periodic"), stretch=R.tanhstretch(1.5),
                  visc=1 / 180, bodyforce=(1.0, 0.0, 0.0))


def runcase_spec(bcy, yd):
    return dict(setup=R.case_kwargs(bcy, visc=0.02, bodyforce=(0.5, 0.0, 0.0), ydiffusion=yd),
                ic="runcase", tlims=(0.0, 0.05), dt=0.01, cfl=None,
                stats="channel" if bcy == "wall" else "spectrum", nupdate=2)


SPECS = {
    "runcase_periodic_explicit": runcase_spec("periodic", "explicit"),
    "runcase_wall_explicit": runcase_spec("wall", "explicit"),
    "runcase_wall_implicit": runcase_spec("wall", "implicit"),
    "channel_noise_cfl": dict(setup=dict(n=(32, 24, 16), ydiffusion="explicit", **CHANNEL_C1),
                              ic="channel_noise", tlims=(0.0, 1.0), dt=None, cfl=0.5,
                              max_steps=10, stats=None),
}


def _oracle_run(O, spec):
    s = O.Setup(**spec["setup"])
    u = s.vectorfield()
    if spec["ic"] == "runcase":
        s.velocityfield(u, **R.RUNCASE_IC)
    else:
        s.velocityfield(u, x=lambda x, y, z: 1.5 * (1 - y ** 2))
        for c in "xyz":
            s.noise(u[c], c, 0, 0.1)
        s.exchange_halo(u)
    procs = []
    acc = None
    if spec.get("stats") == "channel":
        acc = s.channelstats(nupdate=spec["nupdate"])
        procs.append(acc["sample"])
    elif spec.get("stats") == "spectrum":
        acc = s.spectrumstats(nupdate=spec["nupdate"])
        procs.append(acc["sample"])
    p, t, n = s.solve(u, spec["tlims"], dt=spec["dt"], cfl=spec["cfl"] or 0.5,
                      processors=procs, max_steps=spec.get("max_steps"))
    out = {"ux": u["x"], "uy": u["y"], "uz": u["z"], "p": p, "t": np.array(t), "n": np.array(n)}
    if spec.get("stats") == "channel":
        prof = s.channelprofiles(acc)
        for k in ("U", "V", "W", "uu", "vv", "ww", "uv"):
            out["prof_" + k] = prof[k]
    elif spec.get("stats") == "spectrum":
        out["E"] = s.energyspectrum(acc)[1]
    return out


CASES = {name: (lambda O, spec=spec: _oracle_run(O, spec)) for name, spec in SPECS.items()}
