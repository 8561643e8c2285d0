"""dnsb_poisson_noalloc, the allocation-free Poisson solve, against
dnsb_poisson on two calls in a row, through the C ABI.

Callers whose device memory belongs to a capped pooling allocator, or whose
timed loops cannot take the implicit synchronisation of cudaMalloc, cannot
create a context; this entry point serves them with a fixed scratch array
inside the library.  Its result must equal the context-based solve (same
kernels, same launch shapes) within the Poisson tolerance of the other
tests.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

import refcases as R

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.mark.parametrize("kw", [R.channel_kwargs(n=(32, 24, 16)), dict(n=(16, 12, 8)),
                                R.case_kwargs("wall")])
def test_poisson_noalloc_matches_poisson(kw):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import distributednavierstokes_b200 as dns
    from distributednavierstokes_b200 import _lib

    lib = _lib.load()
    s = dns.setup(**kw)
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
    nx, ny, nz = s.n
    rng = np.random.default_rng(11)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call in range(2):  # two calls in a row share the scratch
        r = torch.from_numpy(rng.standard_normal((nz, ny, nx))).cuda()
        s.poisson["r"].copy_(r)
        p_ref = dns.scalarfield(s)
        dns.poisson(p_ref, s)
        p_new = dns.scalarfield(s)
        rc = lib.dnsb_poisson_noalloc(ctypes.byref(g), ctypes.c_void_p(r.data_ptr()),
                                      ctypes.c_void_p(p_new.data_ptr()), stream)
        assert rc == 0, lib.dnsb_last_error(None)
        torch.cuda.synchronize()
        a = dns.interior(p_new).cpu().numpy()
        b = dns.interior(p_ref).cpu().numpy()
        assert np.max(np.abs(a - b)) <= TOL * np.max(np.abs(b)), call


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
