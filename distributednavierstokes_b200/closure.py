"""The sub-filter-stress CNN closure (libdnsb's tensor-core network).

No counterpart in the reference: DistributedNavierStokes has no learned
closure.  The training pairs follow its SFS sampler (filtered velocity
u_bar and trace-free tau = filter(u u) - u_bar u_bar,
src/spectral/les.jl:302-370) on the library's own FV DNS, so this module
adds: the dataset (normalised u_bar, tau on the cell centres of the coarse
periodic grid), the network (C ABI include/dnsb_cnn.h: BF16 implicit-GEMM
convolutions on tcgen05 tensor cores, FP32 accumulation, Adam), and its
evaluation on a periodic FV state.

Array conventions: numpy / torch arrays [c, z, y, x] (x fastest), as the
library's fields.
"""
import ctypes
import math

import numpy as np

from . import _lib
from ._lib import check_cnn

CHANNELS = (3, 32, 32, 32, 6)
HALO = 4
TAU = ("xx", "yy", "zz", "xy", "yz", "zx")


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


class Closure:
    """The network and its optimiser state on one GPU.

    batch, crop: training geometry (batch crops of side crop, each taken with
    a halo of 4 cells from its periodic parent field); nfield: side of the
    periodic field it is evaluated on (0: no inference geometry)."""

    def __init__(self, batch=8, crop=32, nfield=0, device=None, seed=0):
        import torch

        self.device = device if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.batch, self.crop, self.nfield = int(batch), int(crop), int(nfield)
        lib = _lib.load()
        h = ctypes.c_void_p()
        stream = torch.cuda.current_stream(self.device).cuda_stream
        check_cnn(lib.dnsb_cnn_create(self.device.index or 0, ctypes.c_void_p(stream), self.batch,
                                      self.crop, self.nfield, ctypes.byref(h)))
        self._h = h
        self.nparams = lib.dnsb_cnn_param_count(h)
        self._data = None
        check_cnn(lib.dnsb_cnn_init(h, int(seed)), h)

    @property
    def handle(self):
        if self._h is None:
            raise RuntimeError("closure is closed")
        return self._h

    def _stream(self):
        import torch

        _lib.load().dnsb_cnn_set_stream(self.handle, ctypes.c_void_p(
            torch.cuda.current_stream(self.device).cuda_stream))

    def close(self):
        if self._h is not None:
            _lib.load().dnsb_cnn_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---------------------------------------------------------- parameters
    def get_params(self):
        out = np.zeros(self.nparams, dtype=np.float32)
        check_cnn(_lib.load().dnsb_cnn_get_params(self.handle, out.ctypes.data_as(ctypes.c_void_p)),
                  self.handle)
        return out

    def set_params(self, params):
        a = np.ascontiguousarray(params, dtype=np.float32)
        if a.size != self.nparams:
            raise ValueError(f"need {self.nparams} parameters, got {a.size}")
        self._stream()
        check_cnn(_lib.load().dnsb_cnn_set_params(self.handle, a.ctypes.data_as(ctypes.c_void_p)),
                  self.handle)

    def set_scales(self, in_scale, out_scale):
        a = np.ascontiguousarray(in_scale, dtype=np.float32)
        b = np.ascontiguousarray(out_scale, dtype=np.float32)
        if a.size != 3 or b.size != 6:
            raise ValueError("in_scale has 3 values, out_scale 6")
        self.in_scale, self.out_scale = a.copy(), b.copy()
        self._stream()
        check_cnn(_lib.load().dnsb_cnn_set_scales(self.handle, a.ctypes.data_as(ctypes.c_void_p),
                                                  b.ctypes.data_as(ctypes.c_void_p)), self.handle)

    # ------------------------------------------------------------ training
    def set_dataset(self, data):
        """data: DEVICE float32 tensor [S, 9, n, n, n] (normalised u_bar, tau)."""
        import torch

        if data.dtype != torch.float32 or data.dim() != 5 or data.shape[1] != 9 or not data.is_cuda:
            raise ValueError("dataset must be a CUDA float32 tensor [S, 9, n, n, n]")
        data = data.contiguous()
        self._data = data   # borrowed by the library
        check_cnn(_lib.load().dnsb_cnn_set_dataset(self.handle, _p(data), data.shape[0], data.shape[2]),
                  self.handle)

    def train(self, nsteps, lr=1e-3, seed=0):
        """nsteps Adam steps on random crops (asynchronous)."""
        self._stream()
        check_cnn(_lib.load().dnsb_cnn_train(self.handle, int(nsteps), float(lr), int(seed)),
                  self.handle)

    def steps(self):
        n = ctypes.c_long()
        check_cnn(_lib.load().dnsb_cnn_steps(self.handle, ctypes.byref(n)), self.handle)
        return n.value

    def losses(self, first=0, count=None):
        n = self.steps()
        count = n - first if count is None else count
        out = np.zeros(max(count, 0), dtype=np.float32)
        check_cnn(_lib.load().dnsb_cnn_losses(self.handle, out.ctypes.data_as(ctypes.c_void_p),
                                              int(first), int(count)), self.handle)
        return out

    def batch_grads(self, x, t, nadam=0, lr=1e-3):
        """One forward + backward pass on a caller batch (x [B, 3, P, P, P],
        t [B, 6, crop, crop, crop], CUDA float32): (loss, gradients); with
        nadam > 0 also nadam Adam steps on it."""
        g = np.zeros(self.nparams, dtype=np.float32)
        loss = ctypes.c_float()
        self._stream()
        check_cnn(_lib.load().dnsb_cnn_batch(self.handle, _p(x.contiguous()), _p(t.contiguous()),
                                             int(nadam), float(lr), ctypes.byref(loss),
                                             g.ctypes.data_as(ctypes.c_void_p)), self.handle)
        return float(loss.value), g

    # ----------------------------------------------------------- inference
    def infer_cells(self, v, tau=None):
        """v: CUDA float64 [3, n, n, n] cell-centred velocity -> tau [6, n, n, n]."""
        import torch

        n = self.nfield
        tau = tau if tau is not None else torch.empty((6, n, n, n), dtype=torch.float64, device=v.device)
        self._stream()
        check_cnn(_lib.load().dnsb_cnn_infer_cells(self.handle, _p(v.contiguous()), _p(tau)), self.handle)
        return tau

    def infer(self, u, tau=None):
        """u: staggered ghosted FV velocity of the periodic n^3 box -> tau [6, n, n, n]."""
        import torch

        n = self.nfield
        tau = tau if tau is not None else torch.empty((6, n, n, n), dtype=torch.float64,
                                                      device=u["x"].device)
        self._stream()
        check_cnn(_lib.load().dnsb_cnn_infer(self.handle, _p(u["x"]), _p(u["y"]), _p(u["z"]), _p(tau)),
                  self.handle)
        return tau

    # ------------------------------------------------------- instrumentation
    def profile(self, enable=True):
        check_cnn(_lib.load().dnsb_cnn_profile(self.handle, 1 if enable else 0), self.handle)

    def profile_read(self):
        """{kind: (ms, launches, algorithmic flops)} since profile(True)."""
        out = {}
        for k, name in enumerate(("conv_forward", "conv_transposed", "weight_grad", "other")):
            ms, n, fl = ctypes.c_double(), ctypes.c_long(), ctypes.c_double()
            check_cnn(_lib.load().dnsb_cnn_profile_read(self.handle, k, ctypes.byref(ms), ctypes.byref(n),
                                                        ctypes.byref(fl)), self.handle)
            out[name] = (ms.value, n.value, fl.value)
        return out

    def launch_count(self):
        return _lib.load().dnsb_cnn_launch_count(self.handle)


def unflatten(params):
    """The flat parameter vector -> [(W[27, cout, cin], b[cout])] per layer."""
    out, o = [], 0
    for L in range(4):
        cin, cout = CHANNELS[L], CHANNELS[L + 1]
        nw = 27 * cout * cin
        W = np.asarray(params[o:o + nw], dtype=np.float64).reshape(27, cout, cin)
        o += nw
        b = np.asarray(params[o:o + cout], dtype=np.float64)
        o += cout
        out.append((W, b))
    return out


def flatten(layers):
    return np.concatenate([np.concatenate([W.ravel(), b.ravel()]) for W, b in layers]).astype(np.float32)
