"""The CPU network oracle's analytic gradient against central finite
differences (FP64, no BF16 rounding, the leaky ReLU's activation pattern
held at the base point)."""
import numpy as np
import pytest

from oracle import unet_oracle as U


@pytest.mark.parametrize("pery,extra", [(False, 0), (True, 1)])
def test_oracle_gradient_matches_finite_differences(pery, extra):
    net = U.Net(c0=16, c1=16, extra=extra, slope=0.3, pery=pery)
    shape = (16, 8, 8)
    n = 16 * 8 * 8
    rng = np.random.default_rng(7)
    p = U.init_params(net, 3)
    in4 = rng.standard_normal((5, n))
    t = rng.standard_normal(n)
    loss, g, out, masks = U.loss_grad(net, p, in4, t, shape, bf16=False, return_masks=True)
    assert out.shape == (n,) and g.shape == p.shape
    offs, ho = net.offsets()
    blocks = [(a, b + c) for (a, b), (_, c, _) in zip(offs, net.layers())] + [(ho, ho + net.c0 + 1)]
    h = 1e-5
    for a, b in blocks:   # one random direction inside each layer's parameters
        dvec = np.zeros_like(p)
        dvec[a:b] = rng.standard_normal(b - a)
        if a == 0:   # the zero-padded input channels do not enter
            dvec[:27 * 16 * 16].reshape(27, 16, 16)[:, :, U.NIN:] = 0.0
        lp, _, _ = U.loss_grad(net, p + h * dvec, in4, t, shape, bf16=False, masks=masks)
        lm, _, _ = U.loss_grad(net, p - h * dvec, in4, t, shape, bf16=False, masks=masks)
        fd = (lp - lm) / (2 * h)
        an = float(g @ dvec)
        assert abs(fd - an) <= 1e-6 * max(abs(an), 1e-3), (a, b, fd, an)


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -3.14159, 0.0])
    r = U.bf16_round(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 4 * 2 ** -8   # ties to even
    assert abs(r[3] + 3.140625) < 1e-12 and r[4] == 0.0
