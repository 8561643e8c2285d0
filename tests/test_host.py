"""CPU tests of the host side: the C ABI's symbol table, the host mirror's
setup/griddata logic against the oracle, argument validation, and the
multi-rank (replica) benchmark plumbing on gloo ranks."""
import ctypes
import math
import os
import re

import numpy as np
import pytest

import refcases as R

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    names = set()
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if h.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", h)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names |= set(re.findall(r"\b(dnsb_[a-z_0-9]+)\s*\(", txt))
    return sorted(names)


def header_arities():
    """{name: number of parameters} of every prototype in include/*.h."""
    out = {}
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not h.endswith(".h"):
            continue
        txt = open(os.path.join(ROOT, "include", h)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        txt = re.sub(r"//[^\n]*", "", txt)
        for m in re.finditer(r"\b(dnsb_[a-z_0-9]+)\s*\(([^;{]*?)\)\s*;", txt):
            params = " ".join(m.group(2).split())
            out[m.group(1)] = 0 if params in ("", "void") else params.count(",") + 1
    return out


def test_binding_arities_match_headers():
    """Every ctypes binding takes as many arguments as its C prototype (a
    wrong count would shift the arguments of a call silently)."""
    from distributednavierstokes_b200 import _lib

    ar = header_arities()
    assert sorted(ar) == sorted(_lib.SIGNATURES)
    bad = {n: (ar[n], len(_lib.SIGNATURES[n][1])) for n in ar if ar[n] != len(_lib.SIGNATURES[n][1])}
    assert not bad, bad


def test_library_exports_every_header_symbol():
    from distributednavierstokes_b200 import _lib, build

    build.build()
    lib = ctypes.CDLL(_lib.LIBPATH)
    names = header_functions()
    assert len(names) >= 25
    for name in names:
        assert hasattr(lib, name), name
    # the Python binding declares exactly the header's entry points
    assert sorted(_lib.SIGNATURES) == names
    _lib.load()  # binds argtypes for all of them


def test_version_and_error_without_gpu():
    from distributednavierstokes_b200 import _lib

    lib = _lib.load()
    assert lib.dnsb_version() == 1
    # create with a bad grid fails cleanly (validation precedes any CUDA call)
    g = _lib.dnsb_grid()
    g.nx, g.ny, g.nz = 7, 8, 8
    ctx = ctypes.c_void_p()
    assert lib.dnsb_create(ctypes.byref(g), 0, None, ctypes.byref(ctx)) == 1
    assert b"even" in lib.dnsb_last_error(None)
    assert not ctx.value
    g.nx = 8
    g.bc_y, g.ydiffusion = 0, 1
    assert lib.dnsb_create(ctypes.byref(g), 0, None, ctypes.byref(ctx)) == 1
    assert b"requires bc[2] == :wall" in lib.dnsb_last_error(None)
    assert lib.dnsb_kind_name(0) == b"momentum"
    assert lib.dnsb_launch_count(None) == -1


@pytest.mark.parametrize("kw", [R.channel_kwargs(), R.case_kwargs("periodic"), R.case_kwargs("wall"),
                                R.channel_kwargs(n=(8, 48, 8), stretch=R.tanhstretch(2.5))])
def test_griddata_matches_oracle(oracle_mod, kw):
    from distributednavierstokes_b200.api import griddata

    so = oracle_mod.Setup(**kw)
    gd = griddata(kw["n"], kw["lims"], kw["bc"], kw.get("stretch"))
    assert gd["dx"] == so.dx and gd["dz"] == so.dz and gd["dymin"] == so.dymin
    assert np.array_equal(gd["dy"], so.dy)
    assert np.array_equal(gd["dyu"], so.dyu)
    for k in ("xf", "xc", "zf", "zc", "yf", "yc"):
        assert np.array_equal(gd[k], getattr(so, k)), k


def test_setup_validation():
    import distributednavierstokes_b200 as dns

    with pytest.raises(ValueError, match="x and z must be periodic"):
        dns.setup(n=(8, 8, 8), bc=("wall", "periodic", "periodic"))
    with pytest.raises(ValueError, match="bc\\[2\\]"):
        dns.setup(n=(8, 8, 8), bc=("periodic", "inflow", "periodic"))
    with pytest.raises(ValueError, match="ydiffusion"):
        dns.setup(n=(8, 8, 8), ydiffusion="crank")
    with pytest.raises(ValueError, match="order"):
        dns.setup(n=(8, 8, 8), order=4)
    with pytest.raises(ValueError, match="implicit"):
        dns.setup(n=(8, 8, 8), ydiffusion="implicit")
    with pytest.raises(ValueError, match="procgrid"):
        dns.setup(n=(8, 8, 8), procgrid=(2, 1))


def test_bench_helpers():
    import bench

    y = np.linspace(-1, 1, 9)
    U = bench.reichardt(y, 395.0)
    assert U[0] == 0 and U[-1] == 0 and abs(U[4] - U.max()) < 1e-12
    assert 18 < U.max() < 23
    wl = bench.WORKLOADS["channel384_implicit"]
    spec = 193 / 192
    total = sum(bench.passes(k, True, spec) for k in
                ("momentum", "cn_solve", "div_rfft_x", "fft_z", "y_solve", "ifft_z", "irfft_x",
                 "grad_update"))
    assert 39 < total < 45  # the default path moves fewer bytes than 45 passes
    assert wl["bytes_per_cell_step"] == 45 * 3 * 8


def _gloo_worker(rank, world, port, out):
    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    # each replica times its own steps; the job time is the max over ranks
    t = torch.tensor([10.0 + rank], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    cells = 1000
    value = world * cells * 5 / (float(t.item()) / 1e3)
    out.put((rank, float(t.item()), value))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_timing_max_over_ranks_gloo():
    import multiprocessing as mp
    import socket

    ctx = mp.get_context("spawn")
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    q = ctx.Queue()
    ps = [ctx.Process(target=_gloo_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=60) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [11.0, 11.0]
    assert res[0][2] == res[1][2] == 2 * 1000 * 5 / 0.011


def test_ensemble_partition_balanced_and_deterministic():
    """Ensemble members are partitioned across ranks with no collective:
    every rank derives the same owner list, each member has one owner, and
    the largest-first assignment keeps the loads within one member."""
    import numpy as np

    import bench

    rng = np.random.default_rng(12345)
    cells = [int(n) ** 3 for n in rng.choice((32, 48, 64, 96, 128), size=64)]
    for world in (1, 2, 4, 8):
        owner = bench.partition_members(cells, world)
        assert owner == bench.partition_members(cells, world)
        assert sorted(set(owner)) == list(range(world))
        loads = [sum(c for c, o in zip(cells, owner) if o == r) for r in range(world)]
        assert max(loads) - min(loads) <= max(cells)


def _slab_data_movement_rank(rank, world, port, errq):
    """One gloo rank of test_slab_exchanges_gloo."""
    import os
    import types

    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    try:
        import datetime

        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
        from distributednavierstokes_b200 import slab

        comm = slab.TorchComm()
        nx, ny, nz = 6, 3, 8
        nkx_all, nzl = nx // 2 + 1, nz // world
        kx0, nkx = slab.split(nkx_all, world)[rank]
        part = types.SimpleNamespace(rank=rank, nzl=nzl, k0=rank * nzl, nkx_all=nkx_all, kx0=kx0, nkx=nkx,
                                     ny=ny, nz=nz)
        # the spectrum of global plane z at (kx, j): (1000 kx + 10 j + z, -z)
        kx = torch.arange(nkx_all, dtype=torch.float64)[:, None, None]
        j = torch.arange(ny, dtype=torch.float64)[None, :, None]
        z = torch.arange(part.k0, part.k0 + nzl, dtype=torch.float64)[None, None, :]
        S = torch.stack([(1000 * kx + 10 * j + z).expand(nkx_all, ny, nzl), (-z).expand(nkx_all, ny, nzl)],
                        dim=-1).contiguous()
        part.S = S.view(-1)
        part.St = torch.zeros(nkx * ny * nz * 2, dtype=torch.float64)
        part.rbuf = torch.zeros(nkx * ny * nzl * 2, dtype=torch.float64)
        parts = {rank: part}
        slab.to_kx(parts, comm)
        St = part.St.view(nkx, ny, nz, 2)
        kxs = torch.arange(kx0, kx0 + nkx, dtype=torch.float64)[:, None, None]
        zs = torch.arange(nz, dtype=torch.float64)[None, None, :]
        assert torch.equal(St[..., 0], (1000 * kxs + 10 * j + zs).expand(nkx, ny, nz))
        assert torch.equal(St[..., 1], (-zs).expand(nkx, ny, nz))
        ref = part.S.clone()
        part.S.zero_()
        slab.from_kx(parts, comm)
        assert torch.equal(part.S, ref)
        # halos: field value = global plane index of each interior plane
        f = torch.zeros((nzl + 2, 2, 2), dtype=torch.float64)
        for k in range(nzl):
            f[k + 1] = part.k0 + k
        slab.halo_z(parts, comm, lambda p: [f])
        assert float(f[0].max()) == (part.k0 - 1) % nz and float(f[-1].max()) == (part.k0 + nzl) % nz
        dist.destroy_process_group()
    except BaseException as e:  # noqa: BLE001
        errq.put(f"rank {rank}: {type(e).__name__}: {e}")
        raise


def test_slab_exchanges_gloo():
    """The z-slab decomposition's data movement on two gloo ranks (CPU): the
    spectrum transposes z-slabs -> kx-slabs -> z-slabs and the periodic
    z-halo exchange place every value where the (P,1) layout wants it."""
    import multiprocessing as mp
    import socket

    ctx = mp.get_context("spawn")
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    errq = ctx.Queue()
    procs = [ctx.Process(target=_slab_data_movement_rank, args=(r, 2, port, errq)) for r in range(2)]
    for pr in procs:
        pr.start()
    for pr in procs:
        pr.join(120)
    errs = []
    while not errq.empty():
        errs.append(errq.get())
    assert not errs, errs
    assert all(pr.exitcode == 0 for pr in procs), [pr.exitcode for pr in procs]
