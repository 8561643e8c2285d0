"""z-slab decomposition of the FV step over ranks: the reference's (P,1)
process grid (z split over P ranks, y and x whole; layout.jl:15 puts z on
processor axis 1), with its two kinds of exchange:

* halos (halo.jl:81-126): the ghost planes K = 0 and K = nz_local + 1 of a
  rank's fields are the boundary planes of its z-neighbours (periodic in z),
  contiguous in the column-major ghosted layout, sent whole;
* transposes (transpose.jl:47-122): poisson! x-transforms a rank's planes
  locally (dnsb_poisson_x), then redistributes the spectrum from z-slabs to
  kx-slabs (every z of a range of kx planes) so that the z-transform and the
  y-solve see whole lines (dnsb_poisson_zy), and back before the inverse
  x-transform (dnsb_poisson_xinv).  x and y never leave a rank, so walls,
  the Crank-Nicolson y-solve and the x-transforms need no communication.

The orchestration is written once over a communicator: `LocalComm` runs P
ranks in one process on one GPU (every exchange a device copy; used by the
decomposition-invariance tests) and `TorchComm` one rank per process
(torch.distributed: NCCL between GPUs, gloo for the CPU test of the data
movement).  Every function takes `parts`, the ranks this process holds
(all P for LocalComm, its own for TorchComm), and performs each exchange
as one batch of point-to-point messages.
"""
import ctypes
import math

import numpy as np
import torch

from . import _lib
from . import api
from ._lib import check


# ------------------------------------------------------------ communicators

class LocalComm:
    """P ranks emulated in one process: messages are copies."""

    def __init__(self, size):
        self.size = int(size)
        self.local_ranks = list(range(self.size))

    def exchange(self, msgs):
        """msgs: (src, dst, send tensor or None, recv tensor or None)."""
        for src, dst, snd, rcv in msgs:
            rcv.copy_(snd)

    def allreduce(self, values, op):
        vals = list(values.values())
        return max(vals) if op == "max" else min(vals) if op == "min" else sum(vals)


class TorchComm:
    """One rank per process over torch.distributed (NCCL / gloo)."""

    def __init__(self, group=None):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.size = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self.local_ranks = [self.rank]

    def exchange(self, msgs):
        ops = []
        for src, dst, snd, rcv in msgs:
            if src == self.rank and dst == self.rank:
                rcv.copy_(snd)
            elif src == self.rank:
                ops.append(self.dist.P2POp(self.dist.isend, snd.contiguous(), dst, self.group))
            elif dst == self.rank:
                ops.append(self.dist.P2POp(self.dist.irecv, rcv, src, self.group))
        if ops:
            for w in self.dist.batch_isend_irecv(ops):
                w.wait()

    def allreduce(self, values, op):
        v = float(values[self.rank])
        dev = torch.device("cuda", torch.cuda.current_device()) if self.dist.get_backend(self.group) == "nccl" \
            else torch.device("cpu")
        t = torch.tensor([v], dtype=torch.float64, device=dev)
        rop = {"max": self.dist.ReduceOp.MAX, "min": self.dist.ReduceOp.MIN,
               "sum": self.dist.ReduceOp.SUM}[op]
        self.dist.all_reduce(t, op=rop, group=self.group)
        return float(t.item())


# -------------------------------------------------------------------- parts

def split(n, parts):
    """Contiguous ranges of 0..n-1 over `parts` (the first n % parts one longer)."""
    base, extra = divmod(n, parts)
    out, o = [], 0
    for r in range(parts):
        m = base + (r < extra)
        out.append((o, m))
        o += m
    return out


class Part:
    """One rank's share: its planes k0..k0+nzl-1 (a local setup of the same
    x and y grid), its kx-slab kx0..kx0+nkx-1 of the spectrum, and the
    global setup whose plans and tables the kx-slab phase uses."""

    def __init__(self, rank, P, global_kwargs, global_setup, device):
        kw = dict(global_kwargs)
        nx, ny, nz = kw["n"]
        if nz % P:
            raise ValueError(f"nz = {nz} must split evenly over {P} ranks")
        self.rank, self.P = rank, P
        self.nzl = nz // P
        self.k0 = rank * self.nzl
        lims = kw.get("lims", ((0.0, 2 * math.pi),) * 3)
        z0, z1 = lims[2]
        dz = (z1 - z0) / nz
        kw["lims"] = (lims[0], lims[1], (z0 + self.k0 * dz, z0 + (self.k0 + self.nzl) * dz))
        kw["n"] = (nx, ny, self.nzl)
        kw["device"] = device
        self.s = api.setup(**kw)
        self.sg = global_setup
        self.nkx_all = nx // 2 + 1
        self.kx0, self.nkx = split(self.nkx_all, P)[rank]
        self.ny, self.nz = ny, nz
        lib = _lib.load()
        S, a, b, c = ctypes.c_void_p(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(lib.dnsb_spectrum(self.s.ctx, ctypes.byref(S), ctypes.byref(a), ctypes.byref(b),
                                ctypes.byref(c)), self.s._ctx)
        assert (a.value, b.value, c.value) == (self.nkx_all, ny, self.nzl)
        self._S = S.value
        # a view of the local spectrum (complex as float64 pairs) and the kx-slab
        n = self.nkx_all * ny * self.nzl * 2
        self.S = _device_view(self._S, n, device)
        self.St = torch.zeros(self.nkx * ny * nz * 2, dtype=torch.float64, device=device)
        self.rbuf = torch.zeros(self.nkx * ny * self.nzl * 2, dtype=torch.float64, device=device)
        self.r = torch.zeros((self.nzl, ny, nx), dtype=torch.float64, device=device)

    def close(self):
        self.s.close()


def _device_view(ptr, n, device):
    """A float64 tensor over n doubles of library-owned device memory."""
    class _Holder:
        pass

    h = _Holder()
    h.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False), "version": 3}
    return torch.as_tensor(h, device=device)


def make_parts(comm, global_kwargs, device=None):
    """The parts this process holds, and the global setup they share."""
    device = device or torch.device("cuda", torch.cuda.current_device())
    kw = dict(global_kwargs, device=device)
    sg = api.setup(**kw)
    return {r: Part(r, comm.size, global_kwargs, sg, device) for r in comm.local_ranks}, sg


# ---------------------------------------------------------------- exchanges

def halo_z(parts, comm, fields):
    """exchange_halo! in z: ghost plane 0 of rank r <- plane nzl of rank r-1,
    ghost plane nzl+1 <- plane 1 of rank r+1 (periodic); fields(part) ->
    list of ghosted tensors (nzl+2, ny+2, nx+2)."""
    P = comm.size
    msgs = []
    nfield = None
    for r in range(P):
        lo, hi = (r - 1) % P, (r + 1) % P
        fr = fields(parts[r]) if r in parts else None
        flo = fields(parts[lo]) if lo in parts else None
        fhi = fields(parts[hi]) if hi in parts else None
        nfield = nfield or len(fr or flo or fhi)
        for i in range(nfield):
            # r sends its top interior plane up and its bottom one down
            if fr is not None or fhi is not None:
                snd = fr[i][-2] if fr is not None else None
                rcv = fhi[i][0] if fhi is not None else None
                msgs.append((r, hi, snd, rcv))
            if fr is not None or flo is not None:
                snd = fr[i][1] if fr is not None else None
                rcv = flo[i][-1] if flo is not None else None
                msgs.append((r, lo, snd, rcv))
    comm.exchange([m for m in msgs if m[2] is not None or m[3] is not None])


def _zblock_copy(part, dst, src, nkx, nz_dst, z_dst, nz_src, z_src, n):
    """dst[kx][j][z_dst + z] = src[kx][j][z_src + z] (complex pairs)."""
    if dst.is_cuda:
        check(_lib.load().dnsb_zblock_copy(part.s.ctx, ctypes.c_void_p(dst.data_ptr()),
                                           ctypes.c_void_p(src.data_ptr()), nkx, part.ny, nz_dst,
                                           z_dst, nz_src, z_src, n), part.s._ctx)
    else:   # host arrays: the data movement of the CPU test
        d = dst.view(nkx, part.ny, nz_dst, 2)
        s = src.view(nkx, part.ny, nz_src, 2)
        d[:, :, z_dst:z_dst + n] = s[:, :, z_src:z_src + n]


def to_kx(parts, comm):
    """z-slabs -> kx-slabs: rank r's planes of kx-range(d) go to rank d,
    which places them at z offset k0(r) of its slab."""
    P = comm.size
    one = next(iter(parts.values()))
    ranges = split(one.nkx_all, P)
    nzl, ny = one.nzl, one.ny
    for step in range(P):
        msgs = []
        for r in range(P):
            d = (r + step) % P
            kx0, nkx = ranges[d]
            snd = parts[r].S[kx0 * ny * nzl * 2:(kx0 + nkx) * ny * nzl * 2] if r in parts else None
            rcv = parts[d].rbuf[:nkx * ny * nzl * 2] if d in parts else None
            msgs.append((r, d, snd, rcv))
        # messages of one shift are independent: each receiver unpacks its own
        comm.exchange([m for m in msgs if m[2] is not None or m[3] is not None])
        for r in range(P):
            d = (r + step) % P
            if d in parts:
                p = parts[d]
                _zblock_copy(p, p.St, p.rbuf, p.nkx, p.nz, r * nzl, nzl, 0, nzl)


def from_kx(parts, comm):
    """kx-slabs -> z-slabs (the inverse of to_kx)."""
    P = comm.size
    one = next(iter(parts.values()))
    ranges = split(one.nkx_all, P)
    nzl, ny = one.nzl, one.ny
    for step in range(P):
        msgs = []
        for d in range(P):
            r = (d + step) % P   # rank d sends rank r's planes back to r
            kx0, nkx = ranges[d]
            if d in parts:
                p = parts[d]
                _zblock_copy(p, p.rbuf, p.St, p.nkx, nzl, 0, p.nz, r * nzl, nzl)
                snd = p.rbuf[:nkx * ny * nzl * 2]
            else:
                snd = None
            rcv = parts[r].S[kx0 * ny * nzl * 2:(kx0 + nkx) * ny * nzl * 2] if r in parts else None
            msgs.append((d, r, snd, rcv))
        comm.exchange([m for m in msgs if m[2] is not None or m[3] is not None])


# --------------------------------------------------------------- operators

def poisson(parts, comm, r_of, p_of):
    """poisson! (src/poisson.jl:147-161) over the slabs: r_of(part) the
    ghost-free right-hand side, p_of(part) the ghosted output (halos valid)."""
    lib = _lib.load()
    for p in parts.values():
        check(lib.dnsb_poisson_x(p.s.ctx, api._ptr(r_of(p))), p.s._ctx)
    to_kx(parts, comm)
    for p in parts.values():
        check(lib.dnsb_poisson_zy(p.sg.ctx, ctypes.c_void_p(p.St.data_ptr()), p.kx0, p.nkx),
              p.sg._ctx)
    from_kx(parts, comm)
    for p in parts.values():
        check(lib.dnsb_poisson_xinv(p.s.ctx, api._ptr(p_of(p))), p.s._ctx)
    halo_z(parts, comm, lambda p: [p_of(p)])


def project(parts, comm, u_of, psi_of):
    """project!(u, psi, setup) (src/timestep.jl:25-31) over the slabs."""
    for p in parts.values():
        api.divergence(p.r, u_of(p), p.s)
    poisson(parts, comm, lambda p: p.r, psi_of)
    for p in parts.values():
        u = u_of(p)
        api.pressuregrad_update(u, psi_of(p), p.s)
        api.exchange_halo(u, p.s)
    halo_z(parts, comm, lambda p: [u_of(p)[c] for c in "xyz"])


def step(parts, comm, state_of, dt):
    """step!(u, p, q, delta, setup, dt) (src/timestep.jl:41-63) over the
    slabs; state_of(part) -> (u, p, q) or (u, p, q, delta).  Explicit
    y-diffusion: u += B q, halo, projection into p.  Semi-implicit: the
    Crank-Nicolson update (imex_update!, y-lines whole on every rank), halo,
    projection into delta, p += delta / (alpha dt), halo of p."""
    from .les_closure import sfs_stage

    lib = _lib.load()
    one = next(iter(parts.values()))
    for A, B, al in zip(api.RK3["A"], api.RK3["B"], api.RK3["alpha"]):
        for p in parts.values():
            st = state_of(p)
            u, pr, q = st[0], st[1], st[2]
            api.momentum(q, u, A, dt, p.s)
            if p.s.imexy:
                api.imex_update(u, q, pr, B, al, dt, p.s)
            else:
                sfs_stage(None, q, u, dt, B, p.s)
        halo_z(parts, comm, lambda p: [state_of(p)[0][c] for c in "xyz"])
        if one.s.imexy:
            project(parts, comm, lambda p: state_of(p)[0], lambda p: state_of(p)[3])
            for p in parts.values():
                st = state_of(p)
                check(lib.dnsb_axpy(p.s.ctx, api._ptr(st[1]), api._ptr(st[3]), 1.0 / (al * dt)), p.s._ctx)
                api.exchange_halo(st[1], "p", p.s)
            halo_z(parts, comm, lambda p: [state_of(p)[1]])
        else:
            project(parts, comm, lambda p: state_of(p)[0], lambda p: state_of(p)[1])


def cfl_timestep(parts, comm, u_of, cfl):
    """cfl_timestep (src/timestep.jl:69-80): the minimum over the ranks."""
    return comm.allreduce({r: api.cfl_timestep(u_of(p), p.s, cfl) for r, p in parts.items()}, "min")


def maxdiv(parts, comm, u_of):
    return comm.allreduce({r: api.maxdiv(u_of(p), p.s) for r, p in parts.items()}, "max")


# ------------------------------------------------------ scatter and gather

def scatter(parts, field):
    """A rank's ghosted slab (planes k0-1 .. k0+nzl) of a global ghosted
    field (nz+2, ny+2, nx+2) whose halos are valid."""
    return {r: field[p.k0:p.k0 + p.nzl + 2].clone() for r, p in parts.items()}


def gather_interior(parts, fields, nz):
    """The global interior planes from the ranks' slabs (all ranks local)."""
    one = next(iter(parts.values()))
    out = torch.empty((nz,) + tuple(fields[one.rank].shape[1:]), dtype=torch.float64,
                      device=fields[one.rank].device)
    for r, p in parts.items():
        out[p.k0:p.k0 + p.nzl] = fields[r][1:-1]
    return out
