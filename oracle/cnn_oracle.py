"""CPU oracle of the sub-filter-stress CNN closure (test infrastructure).

Only the tests, the smoke check and the benchmark's CPU baseline use this
module, as the checker of the device kernels; the product never imports it.

The reference (DistributedNavierStokes) has no neural closure: the network
has no counterpart there.  Its definition here is the one the device
kernels implement, restated in float64 numpy with the same storage
roundings, so that the two can be compared:

* 4 convolution layers, 3x3x3 kernels, channels 3 -> 32 -> 32 -> 32 -> 6,
  bias on every layer, GELU in its tanh form
  (0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3))), evaluated as z sigma(2u))
  after the first three;
* periodic padding on the full periodic field.  Training crops carry a halo
  of 4 cells taken from their periodic parent field and the layers are
  "valid" convolutions (each shrinks the box by 2), so a crop's outputs are
  exactly the full field's outputs on that crop;
* BF16 storage of weights, activations, pre-activations and back-propagated
  gradients (round to nearest even from the FP32 value), accumulation in
  FP32 on the device (float64 here), FP32 master weights and Adam state;
* loss = mean over the valid outputs and the 6 components of (y - t)^2 on
  the per-component normalised stress; dL/dy is stored in BF16.

Layouts: activations are numpy arrays (B, C, P, P, P) indexed [b, c, z, y, x];
weights W[t, co, ci] with tap t = (dz * 3 + dy) * 3 + dx, the input voxel of
output (x, y, z) for tap (dx, dy, dz) being (x + dx, y + dy, z + dz).
"""
import math

import numpy as np

CHANNELS = (3, 32, 32, 32, 6)
NLAYERS = 4
HALO = 4            # cells of halo a crop needs (one per layer)
TAPS = [(dz, dy, dx) for dz in range(3) for dy in range(3) for dx in range(3)]


def bf16(x):
    """Round to BF16 (nearest even) from the FP32 value, returned as float64."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return (r.astype(np.uint32)).view(np.float32).astype(np.float64)


def f32(x):
    return np.asarray(x, dtype=np.float32).astype(np.float64)


GELU_C = math.sqrt(2.0 / math.pi)
GELU_A = 0.044715


def _sigmoid2u(z):
    u2 = 2.0 * GELU_C * (z + GELU_A * z ** 3)
    return 1.0 / (1.0 + np.exp(-u2))


def gelu(z):
    """GELU in its tanh form: 0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3)))
    = z sigma(2u)."""
    with np.errstate(over="ignore"):
        return z * _sigmoid2u(z)


def gelu_grad(z):
    with np.errstate(over="ignore"):
        sg = _sigmoid2u(z)
    du2 = 2.0 * GELU_C * (1.0 + 3.0 * GELU_A * z * z)
    return sg + z * sg * (1.0 - sg) * du2


def init_params(seed=0, channels=CHANNELS):
    """Uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) weights and biases from a
    splitmix64 stream, element order (layer, W[t, co, ci] row-major, b[co]);
    the library's dnsb_cnn_init draws the same numbers."""
    params = []
    ctr = 0
    for L in range(NLAYERS):
        cin, cout = channels[L], channels[L + 1]
        bound = 1.0 / math.sqrt(27 * cin)
        nW, nb = 27 * cout * cin, cout
        u = _uniforms(seed, ctr, nW + nb)
        ctr += nW + nb
        W = f32((2 * u[:nW] - 1) * bound).reshape(27, cout, cin)
        b = f32((2 * u[nW:] - 1) * bound)
        params.append((W, b))
    return params


def _uniforms(seed, start, n):
    """U in (0, 1): ((splitmix64(seed + i) >> 11) + 0.5) * 2^-53 for i in
    start..start+n-1 (the key/uniform mapping of src/spectral/ic.jl:31-45)."""
    seed = np.uint64(seed & 0xFFFFFFFFFFFFFFFF)
    i = np.arange(start, start + n, dtype=np.uint64)
    with np.errstate(over="ignore"):
        x = seed + i + np.uint64(0x9E3779B97F4A7C15)
        z = x
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return ((z >> np.uint64(11)).astype(np.float64) + 0.5) * 2.0 ** -53


def conv_valid(x, W, shift=0):
    """out[b, co, z, y, x] = sum_{t, ci} W[t, co, ci] x[b, ci, z+s+dz, y+s+dy, x+s+dx]
    on the output box of side P - 2 - 2*shift... for shift 0 the valid
    convolution (side P - 2); reads outside x are zero."""
    B, C, P = x.shape[0], x.shape[1], x.shape[2]
    D = P - 2
    out = np.zeros((B, W.shape[1], D, D, D))
    for t, (dz, dy, dx) in enumerate(TAPS):
        xs = x[:, :, dz:dz + D, dy:dy + D, dx:dx + D]
        out += np.einsum("oc,bczyx->bozyx", W[t], xs, optimize=True)
    return out


def conv_full(g, W):
    """The transpose of conv_valid: g (B, Cout, D, D, D) -> (B, Cin, D+2, D+2, D+2),
    dx[i] = sum_d g[i - d] W[d] (zero outside g)."""
    B, Co, D = g.shape[0], g.shape[1], g.shape[2]
    Ci = W.shape[2]
    out = np.zeros((B, Ci, D + 2, D + 2, D + 2))
    for t, (dz, dy, dx) in enumerate(TAPS):
        out[:, :, dz:dz + D, dy:dy + D, dx:dx + D] += np.einsum("oc,bozyx->bczyx", W[t], g,
                                                                 optimize=True)
    return out


def wgrad(h, g):
    """dW[t, co, ci] = sum_o g[o, co] h[o + t, ci], db[co] = sum_o g[o, co]."""
    D = g.shape[2]
    dW = np.zeros((27, g.shape[1], h.shape[1]))
    for t, (dz, dy, dx) in enumerate(TAPS):
        hs = h[:, :, dz:dz + D, dy:dy + D, dx:dx + D]
        dW[t] = np.einsum("bozyx,bczyx->oc", g, hs, optimize=True)
    return dW, g.sum(axis=(0, 2, 3, 4))


def forward(params, x0, store=True):
    """x0: (B, 3, P, P, P) input crop (already BF16-representable).  Returns
    the list of (z_L, h_L) for the hidden layers and the FP32 output y
    (B, 6, P-8, P-8, P-8)."""
    h = bf16(x0)
    acts = [(None, h)]
    for L in range(NLAYERS):
        W, b = params[L]
        Wb = bf16(W)
        acc = conv_valid(h, Wb) + b[None, :, None, None, None]
        if L < NLAYERS - 1:
            z32 = f32(acc)
            z = bf16(z32)
            h = bf16(gelu(z32))
            acts.append((z, h))
        else:
            y = f32(acc)
    return acts, y


def loss_and_grads(params, x0, t):
    """Loss (mean of (y - t)^2) and the gradients of every W, b, with the
    device's storage roundings; t: (B, 6, P-8, P-8, P-8)."""
    acts, y = forward(params, x0)
    count = y.size
    diff = y - t
    loss = float(np.sum(diff * diff) / count)
    g = bf16(2.0 * diff / count)
    grads = [None] * NLAYERS
    for L in range(NLAYERS - 1, -1, -1):
        W, b = params[L]
        h_in = acts[L][1]
        dW, db = wgrad(h_in, g)
        grads[L] = (dW, db)
        if L > 0:
            dh = conv_full(g, bf16(W))
            z = acts[L][0]
            g = bf16(f32(dh) * gelu_grad(z))
    return loss, grads, y


class Adam:
    """Adam (Kingma & Ba) with bias correction, FP32 state; the update of
    each parameter p with gradient g at step t:
    m = b1 m + (1-b1) g, v = b2 v + (1-b2) g^2,
    p -= lr (m / (1 - b1^t)) / (sqrt(v / (1 - b2^t)) + eps)."""

    def __init__(self, params, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
        self.lr, self.b1, self.b2, self.eps = lr, beta1, beta2, eps
        self.m = [[np.zeros_like(W), np.zeros_like(b)] for W, b in params]
        self.v = [[np.zeros_like(W), np.zeros_like(b)] for W, b in params]
        self.t = 0

    def step(self, params, grads):
        self.t += 1
        c1 = 1 - self.b1 ** self.t
        c2 = 1 - self.b2 ** self.t
        out = []
        for L, (pw, gw) in enumerate(zip(params, grads)):
            new = []
            for k in range(2):
                g = gw[k]
                self.m[L][k] = f32(self.b1 * self.m[L][k] + (1 - self.b1) * g)
                self.v[L][k] = f32(self.b2 * self.v[L][k] + (1 - self.b2) * g * g)
                upd = (self.m[L][k] / c1) / (np.sqrt(self.v[L][k] / c2) + self.eps)
                new.append(f32(pw[k] - self.lr * upd))
            out.append(tuple(new))
        return out


def periodic_infer(params, u3):
    """The network on a full periodic field u3 (3, n, n, n) [c, z, y, x]:
    the field extended by a periodic halo of 4, then the valid layers;
    returns (6, n, n, n)."""
    x = np.pad(u3, ((0, 0), (HALO, HALO), (HALO, HALO), (HALO, HALO)), mode="wrap")
    _, y = forward(params, bf16(x)[None])
    return y[0]
