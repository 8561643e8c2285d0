"""dnsb_poisson_noalloc, the allocation-free Poisson solve, against
dnsb_poisson and the oracle on two calls in a row, through the C ABI.

Callers whose device memory belongs to a capped pooling allocator, or whose
timed loops cannot take the implicit synchronisation of cudaMalloc, cannot
create a context; this entry point serves them with a fixed scratch array
inside the library.  It runs the transforms of dnsb_poisson's Stockham path
(with walls, the one-thread-per-line Thomas y-solve instead of the chunked
one), so its result must equal the context-based solve and the oracle
within the Poisson tolerance of the other tests.  The cases include a grid
exactly at the spectrum limit ((nx/2+1)*ny*nz = 2^20), the longest z-lines
(nz = 4096, the largest shared-memory request) and a non-default stream.
This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

import refcases as R

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 1e-12

CASES = {
    "channel": R.channel_kwargs(n=(32, 24, 16)),
    "periodic": dict(n=(16, 12, 8)),
    "wall": R.case_kwargs("wall"),
    # (30/2 + 1) * 256 * 256 = 2^20 spectrum values: exactly at the limit
    "at_spectrum_limit": dict(n=(30, 256, 256)),
    # nz = 4096: one z-line per CTA and the largest shared-memory request
    # (196 KB); a context cannot be created at this length (its opt-in TMA
    # z-transform would need more shared memory), so only the oracle checks it
    "nz4096": dict(n=(8, 16, 4096)),
}
NO_CONTEXT = {"nz4096"}


def _grid(_lib, s):
    g = _lib.dnsb_grid()
    g.nx, g.ny, g.nz = s.n
    g.bc_y = 1 if s.wall else 0
    g.ydiffusion = 0
    g.dx, g.dz = s.dx, s.dz
    dy = np.ascontiguousarray(s.dy)
    dyu = np.ascontiguousarray(s.dyu)
    g.dy = dy.ctypes.data_as(ctypes.c_void_p)
    g.dyu = dyu.ctypes.data_as(ctypes.c_void_p)
    g.visc = s.visc
    return g, (dy, dyu)   # the arrays must outlive the calls


@pytest.mark.parametrize("side_stream", [False, True])
@pytest.mark.parametrize("case", list(CASES))
def test_poisson_noalloc_matches_poisson(oracle_mod, case, side_stream):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    if side_stream and case not in ("channel", "periodic"):
        pytest.skip("the stream variant runs on the small cases")
    import distributednavierstokes_b200 as dns
    from distributednavierstokes_b200 import _lib

    kw = CASES[case]
    lib = _lib.load()
    so = oracle_mod.Setup(**kw)
    s = None if case in NO_CONTEXT else dns.setup(**kw)
    g, keep = _grid(_lib, s or so)
    nx, ny, nz = so.n
    rng = np.random.default_rng(11)
    ts = torch.cuda.Stream() if side_stream else torch.cuda.current_stream()
    stream = ctypes.c_void_p(ts.cuda_stream)
    for call in range(2):  # two calls in a row share the scratch
        rh = rng.standard_normal((nz, ny, nx))
        r = torch.from_numpy(rh).cuda()
        p_new = torch.zeros((nz + 2, ny + 2, nx + 2), dtype=torch.float64, device="cuda")
        if s is not None:
            s.poisson["r"].copy_(r)
            p_ref = dns.scalarfield(s)
            dns.poisson(p_ref, s)
        torch.cuda.synchronize()
        rc = lib.dnsb_poisson_noalloc(ctypes.byref(g), ctypes.c_void_p(r.data_ptr()),
                                      ctypes.c_void_p(p_new.data_ptr()), stream)
        assert rc == 0, lib.dnsb_last_error(None)
        ts.synchronize()
        a = p_new[1:-1, 1:-1, 1:-1].cpu().numpy()
        if s is not None:
            b = dns.interior(p_ref).cpu().numpy()
            assert np.max(np.abs(a - b)) <= TOL * np.max(np.abs(b)), call
        po = so.scalarfield()
        so.poisson(rh, po)
        c = po[1:-1, 1:-1, 1:-1]
        assert np.max(np.abs(a - c)) <= TOL * np.max(np.abs(c)), call
    del keep


def test_poisson_noalloc_rejects_oversize():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from distributednavierstokes_b200 import _lib

    lib = _lib.load()
    g = _lib.dnsb_grid()
    g.nx, g.ny, g.nz = 256, 256, 256   # (129*256*256) > 2^20 spectrum values
    g.bc_y, g.ydiffusion = 0, 0
    g.dx = g.dz = 0.1
    dy = np.full(258, 0.1)
    g.dy = dy.ctypes.data_as(ctypes.c_void_p)
    g.dyu = dy.ctypes.data_as(ctypes.c_void_p)
    x = torch.zeros(8, dtype=torch.float64, device="cuda")
    rc = lib.dnsb_poisson_noalloc(ctypes.byref(g), ctypes.c_void_p(x.data_ptr()),
                                  ctypes.c_void_p(x.data_ptr()), None)
    assert rc == 3
    assert b"exceeds its fixed scratch" in lib.dnsb_last_error(None)
    g.nx, g.ny, g.nz = 32, 16, 8200     # one length beyond 4096
    rc = lib.dnsb_poisson_noalloc(ctypes.byref(g), ctypes.c_void_p(x.data_ptr()),
                                  ctypes.c_void_p(x.data_ptr()), None)
    assert rc == 3
