"""The CNN closure's tensor-core kernels against the CPU oracle
(oracle/cnn_oracle.py, float64 with the device's BF16 storage roundings),
through the C ABI (include/dnsb_cnn.h).

Tolerances.  Both sides round the same values to BF16 at the same points;
they differ by the FP32 accumulation order (and FP32 erf/exp) of the device,
which moves a value across a BF16 rounding boundary now and then (one BF16
ulp = 2^-8 relative).  So: outputs and gradients are compared as relative
L2 norms of the difference (<= 5e-3) and relative max-norms (<= 1e-2), the
loss to 1e-4 relative; the initial parameters are bit-identical.  (Measured
on B200: inference 4.6e-4 / 1.5e-3, gradients <= 2.1e-3 / 1.7e-3, the loss
1e-5.)
"""
import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def C():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import cnn_oracle
    from distributednavierstokes_b200 import closure

    return closure, cnn_oracle


def l2rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def maxrel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def test_init_params_bit_identical(C):
    closure, O = C
    cl = closure.Closure(batch=1, crop=8, seed=7)
    p = cl.get_params()
    ref = O.init_params(7)
    assert p.size == sum(W.size + b.size for W, b in ref) == 63174
    assert np.array_equal(p, closure.flatten(ref))
    cl.close()


@pytest.mark.parametrize("n", [16, 24])
def test_inference_matches_oracle(C, n):
    """The four layers on a periodic field (halo 4, valid convolutions):
    forward GELU epilogues and the output epilogue with its scales."""
    closure, O = C
    cl = closure.Closure(batch=0, crop=0, nfield=n, seed=3)
    rng = np.random.default_rng(5)
    # weights 3x their initial scale so that the activations are O(1)
    params = closure.unflatten(cl.get_params())
    params = [(W * 3, b * 3) for W, b in params]
    cl.set_params(closure.flatten(params))
    params = closure.unflatten(cl.get_params())
    insc = np.array([1.5, 0.5, 2.0], dtype=np.float32)
    outsc = np.array([1, 2, 3, 0.5, 0.25, 4], dtype=np.float32)
    cl.set_scales(insc, outsc)
    v = rng.standard_normal((3, n, n, n))
    tau = cl.infer_cells(torch.from_numpy(v).cuda())
    torch.cuda.synchronize()
    got = tau.cpu().numpy()
    x = O.f32(v * insc.astype(np.float64)[:, None, None, None])
    ref = O.periodic_infer(params, x) * outsc.astype(np.float64)[:, None, None, None]
    e2, em = l2rel(got, ref), maxrel(got, ref)
    print(f"inference n={n}: l2 {e2:.2e} max {em:.2e}")
    assert e2 <= 5e-3 and em <= 1e-2
    cl.close()


@pytest.mark.parametrize("batch,crop", [(2, 8), (1, 16)])
def test_loss_and_gradients_match_oracle(C, batch, crop):
    """Forward with the loss epilogue, the transposed convolutions with the
    GELU-derivative epilogue and the MN-major weight-gradient GEMMs (split-K
    reduced, bias gradients from the ones row) against the oracle."""
    closure, O = C
    cl = closure.Closure(batch=batch, crop=crop, seed=11)
    params = closure.unflatten(cl.get_params())
    params = [(W * 3, b * 3) for W, b in params]
    cl.set_params(closure.flatten(params))
    params = closure.unflatten(cl.get_params())
    P = crop + 8
    rng = np.random.default_rng(2)
    x = O.f32(rng.standard_normal((batch, 3, P, P, P)))
    t = O.f32(rng.standard_normal((batch, 6, crop, crop, crop)))
    loss, g = cl.batch_grads(torch.from_numpy(x.astype(np.float32)).cuda(),
                             torch.from_numpy(t.astype(np.float32)).cuda())
    lref, gref, _ = O.loss_and_grads(params, x, t)
    print(f"loss {loss:.6e} oracle {lref:.6e}")
    assert math.isclose(loss, lref, rel_tol=1e-4)
    gd = closure.unflatten(g)
    for L in range(4):
        for k, name in enumerate(("W", "b")):
            e2, em = l2rel(gd[L][k], gref[L][k]), maxrel(gd[L][k], gref[L][k])
            print(f"layer {L + 1} d{name}: l2 {e2:.2e} max {em:.2e}")
            assert e2 <= 5e-3 and em <= 1e-2, (L, name, e2, em)
    cl.close()


def test_adam_steps_match_oracle(C):
    """Three Adam steps on one batch: the parameter updates agree with the
    oracle's (FP32 Adam on the oracle's gradients)."""
    closure, O = C
    cl = closure.Closure(batch=1, crop=8, seed=13)
    p0 = cl.get_params()
    params = closure.unflatten(p0)
    P = 16
    rng = np.random.default_rng(4)
    x = O.f32(rng.standard_normal((1, 3, P, P, P)))
    t = O.f32(rng.standard_normal((1, 6, 8, 8, 8)))
    lr = 1e-3
    cl.batch_grads(torch.from_numpy(x.astype(np.float32)).cuda(),
                   torch.from_numpy(t.astype(np.float32)).cuda(), nadam=3, lr=lr)
    p1 = cl.get_params()
    assert cl.steps() == 3
    opt = O.Adam(params, lr=lr)
    pr = params
    for _ in range(3):
        _, gr, _ = O.loss_and_grads(pr, x, t)
        pr = opt.step(pr, gr)
    ref = closure.flatten(pr).astype(np.float64)
    du, dr = p1.astype(np.float64) - p0, ref - p0
    # Adam's first steps move every weight by about lr * sign(g); weights
    # whose gradient is near zero may take the other sign
    close = np.abs(du - dr) <= 0.05 * lr * 3
    print(f"adam: {close.mean():.4f} of the updates within 5%; l2 {l2rel(du, dr):.2e}")
    assert close.mean() >= 0.98 and l2rel(du, dr) <= 0.1
    cl.close()


def test_training_reduces_loss(C):
    """Teacher-student: a random network of the same architecture makes the
    targets of a small periodic dataset; 300 Adam steps on random crops bring
    the loss well below its start."""
    closure, O = C
    n, S = 16, 3
    rng = np.random.default_rng(8)
    teacher = [(W * 2, b) for W, b in O.init_params(99)]
    data = np.zeros((S, 9, n, n, n), dtype=np.float32)
    k = np.fft.fftfreq(n) * n
    kk = k[:, None, None] ** 2 + k[None, :, None] ** 2 + k[None, None, :] ** 2
    for s in range(S):
        u = np.stack([np.real(np.fft.ifftn(np.fft.fftn(rng.standard_normal((n, n, n))) *
                                           np.exp(-kk / 8))) for _ in range(3)])
        u /= u.std()
        data[s, :3] = u
        data[s, 3:] = O.periodic_infer(teacher, O.bf16(u))
    data[:, 3:] /= data[:, 3:].std(axis=(0, 2, 3, 4), keepdims=True)
    cl = closure.Closure(batch=4, crop=8, seed=1)
    d = torch.from_numpy(data).cuda()
    cl.set_dataset(d)
    cl.train(300, lr=2e-3, seed=5)
    losses = cl.losses()
    assert losses.size == 300 and np.all(np.isfinite(losses))
    first, last = losses[:20].mean(), losses[-20:].mean()
    print(f"training: loss {first:.4f} -> {last:.4f}")
    assert last < 0.5 * first
    cl.close()


def test_dependent_launch_same_bits(C, monkeypatch):
    """The convolutions and weight gradients launched as programmatic
    dependents (the default) and as ordinary kernels (DNSB_CNN_PDL=0, read
    when a closure is created) give the same bits: inference on a 24^3
    field, and 20 Adam steps of a training batch (losses and parameters)."""
    closure, O = C
    rng = np.random.default_rng(21)
    n = 24
    v = torch.from_numpy(rng.standard_normal((3, n, n, n))).cuda()
    data = torch.from_numpy(rng.standard_normal((3, 9, 16, 16, 16)).astype(np.float32)).cuda()
    out = []
    for flag in ("1", "0"):
        monkeypatch.setenv("DNSB_CNN_PDL", flag)
        cl = closure.Closure(batch=2, crop=8, nfield=n, seed=4)
        cl.set_scales([1.0, 2.0, 0.5], [1.0] * 6)
        tau = cl.infer_cells(v).cpu().numpy()
        cl.set_dataset(data)
        cl.train(20, lr=1e-3, seed=6)
        out.append((tau, cl.losses().copy(), cl.get_params().copy()))
        cl.close()
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)
