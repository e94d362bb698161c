"""The corrector network's CPU restatement (oracle/cnn.py): its backward
pass against central finite differences of its forward pass in float64,
and the bfloat16 rounding helper.  The GPU kernels are checked against it in
tests/test_corrector_gpu.py."""
import numpy as np

from oracle import cnn


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2**-8, 1.0 + 3 * 2**-9, 1.0 + 2**-9, -3.1415926], np.float32)
    r = cnn.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 + 2**-7 or r[1] == 1.0   # a tie: to even
    assert r[2] == 1.0 + 2**-7
    assert r[3] == 1.0                                             # tie, even mantissa
    assert abs(r[4] + 3.140625) < 1e-12


def test_oracle_backward_matches_finite_differences():
    rng = np.random.default_rng(3)
    p = cnn.init_params(seed=5).astype(np.float64)
    p[np.arange(len(p)) % 7 == 0] += 0.01                          # non-zero biases too
    x = rng.normal(size=(1, 7, 9, cnn.DIMS[0][0]))
    gout = rng.normal(size=(1, 7, 9, 8))
    net = cnn.Net(p, rounding=False)
    net.forward(x)
    g = net.backward(gout)
    idx = rng.choice(len(p), size=40, replace=False)
    eps = 1e-6
    for k in idx:
        q = p.copy()
        q[k] += eps
        fp = (cnn.Net(q, rounding=False).forward(x) * gout).sum()
        q[k] -= 2 * eps
        fm = (cnn.Net(q, rounding=False).forward(x) * gout).sum()
        fd = (fp - fm) / (2 * eps)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(fd)), (k, fd, g[k])


def test_parameter_count_matches_the_layout():
    assert cnn.nparams() == 65704
    assert len(cnn.init_params()) == cnn.nparams()
