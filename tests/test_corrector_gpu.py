"""The corrector network's tensor-core kernels (tcgen05 implicit-GEMM 5x5
convolutions, forward and input-gradient passes, and tensor-core weight
gradients)
against the CPU restatement oracle/cnn.py, which rounds the same operands
to bfloat16: outputs within 2e-3 and parameter gradients within 2e-2
relative L2 per layer (the GPU accumulates in FP32 in another order, and an
activation that lands on a bfloat16 rounding tie may round the other way).
The gradient sums are reduced in a fixed order, so they are reproducible."""
import numpy as np
import pytest

from ouc_b200.corrector import Net
from oracle import cnn

pytestmark = pytest.mark.gpu

TOL_OUT = 2e-3
TOL_GRAD = 2e-2


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


def _params(seed):
    p = cnn.init_params(seed=seed)
    rng = np.random.default_rng(seed + 100)
    k = 0
    for ci, co in cnn.DIMS:                  # non-zero biases
        k += co * ci * cnn.TAPS
        p[k:k + co] = rng.normal(0, 0.05, co)
        k += co
    return p


@pytest.mark.parametrize("shape", [(2, 9, 150), (4, 40, 300)])
def test_forward_and_gradients_match_oracle(shape):
    import torch
    n, H, W = shape
    rng = np.random.default_rng(7)
    p = _params(11)
    x = rng.normal(size=(n, H, W, cnn.DIMS[0][0])).astype(np.float32)
    gout = rng.normal(size=(n, H, W, 8)).astype(np.float32)
    ref = cnn.Net(p)
    y_ref = ref.forward(x)
    g_ref = ref.backward(gout)
    dev = torch.device("cuda", 0)
    dx = torch.from_numpy(x).to(dev)
    dy = torch.empty((n, H, W, 8), dtype=torch.float32, device=dev)
    dg = torch.from_numpy(gout).to(dev)
    with Net(0, p) as net:
        net.zero_grad()
        net.forward_dev(n, H, W, dx.data_ptr(), dy.data_ptr())
        net.backward_dev(dg.data_ptr())
        torch.cuda.synchronize()
        g = net.grads()
        assert net.error() == 0
    y = dy.cpu().numpy()
    e_out = _rel(y, y_ref)
    e_grad = []
    k = 0
    for ci, co in cnn.DIMS:
        nw = co * ci * cnn.TAPS
        e_grad.append((_rel(g[k:k + nw], g_ref[k:k + nw]), _rel(g[k + nw:k + nw + co], g_ref[k + nw:k + nw + co])))
        k += nw + co
    print(shape, "output", e_out, "gradients (W, b) per layer", e_grad)
    assert e_out <= TOL_OUT
    assert max(max(t) for t in e_grad) <= TOL_GRAD


def test_adam_reduces_a_regression_loss():
    """A few Adam steps on a fixed batch lower the mean squared error."""
    import torch
    n, H, W = 2, 24, 130
    rng = np.random.default_rng(1)
    x = rng.normal(size=(n, H, W, cnn.DIMS[0][0])).astype(np.float32)
    target = cnn.Net(_params(3)).forward(x).astype(np.float32)   # a reachable target
    dev = torch.device("cuda", 0)
    dx = torch.from_numpy(x).to(dev)
    dt = torch.from_numpy(target).to(dev)
    dy = torch.empty_like(dt)
    losses = []
    with Net(0, _params(4)) as net:
        for it in range(30):
            net.zero_grad()
            net.forward_dev(n, H, W, dx.data_ptr(), dy.data_ptr())
            diff = dy - dt
            losses.append(float((diff * diff).mean()))
            gout = (2.0 / diff.numel()) * diff
            net.backward_dev(gout.data_ptr())
            net.adam_step(1e-3)
        torch.cuda.synchronize()
        assert net.error() == 0
    print("loss", losses[0], "->", losses[-1])
    assert losses[-1] < 0.5 * losses[0]


def test_gradients_are_reproducible():
    """Weight and bias gradients are reduced in a fixed order (per-block
    partial sums, then an ordered sum; no atomics): two backward passes on
    the same inputs give bit-identical gradients, so training runs repeat."""
    import torch
    n, H, W = 3, 33, 170
    rng = np.random.default_rng(5)
    p = _params(13)
    x = rng.normal(size=(n, H, W, cnn.DIMS[0][0])).astype(np.float32)
    gout = rng.normal(size=(n, H, W, 8)).astype(np.float32)
    dev = torch.device("cuda", 0)
    dx = torch.from_numpy(x).to(dev)
    dy = torch.empty((n, H, W, 8), dtype=torch.float32, device=dev)
    dg = torch.from_numpy(gout).to(dev)
    grads = []
    with Net(0, p) as net:
        for _ in range(2):
            net.zero_grad()
            net.forward_dev(n, H, W, dx.data_ptr(), dy.data_ptr())
            net.backward_dev(dg.data_ptr())
            torch.cuda.synchronize()
            grads.append(net.grads().copy())
        assert net.error() == 0
    assert np.array_equal(grads[0], grads[1])
    assert np.abs(grads[0]).max() > 0
