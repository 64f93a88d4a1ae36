"""CPU FP64 restatement of the learned warm-start network -- test
infrastructure only (the gradient checks of the CUDA convolution, pooling,
up-sampling, head and Adam-free training kernels import it; nothing on the
product path does).

The network has no counterpart in the reference (mobydiff starts every
red-black projection from phi = 0, src/modules/pressure/pressure_redblack.f90:63-84),
so this module restates the network the C ABI documents
(include/mobydiff_b200.h, "learned warm start"):

  enc0a 16->c0, enc0b c0->c0 = s0; pool; enc1a c0->c1, enc1b = s1; pool;
  enc2a, enc2b = s2; pool; enc3a, enc3b (+ extra) = b;
  dec2 = conv(up(b) + s2) c1->c1; dec1 = conv(up(dec2) + s1) c1->c0;
  dec0 = conv(up(dec1) + s0) c0->c0; out = head(dec0) (1x1, c0->1)

3x3x3 convolutions with a leaky ReLU, periodic in x and z, zero padding
in y (periodic when y is).  Arrays are channels-last [z][y][x][c].  The flat
parameter vector is, per convolution, W[tap][cout][cin] (tap =
9*(dz+1)+3*(dy+1)+(dx+1)) then bias[cout]; then head w[c0], b.

With ``bf16=True`` values are rounded to BF16 where the CUDA kernels store
BF16 (weights, packed input, every activation, pool and up-add output and
every pre-activation gradient); sums run in FP64 here and in FP32 on the
GPU.  With ``bf16=False`` everything is FP64, which the finite-difference
check of the analytic gradient uses.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

NIN = 5
C_IN = 16


def bf16_round(a: np.ndarray) -> np.ndarray:
    """Round to the nearest BF16 (ties to even), via FP32, returned as FP64."""
    f = np.asarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


@dataclass
class Net:
    c0: int = 16
    c1: int = 32
    extra: int = 0
    slope: float = 0.1
    pery: bool = False

    def layers(self):
        """(cin, cout, level) per convolution in parameter order."""
        c0, c1 = self.c0, self.c1
        L = [(C_IN, c0, 0), (c0, c0, 0), (c0, c1, 1), (c1, c1, 1), (c1, c1, 2), (c1, c1, 2), (c1, c1, 3), (c1, c1, 3)]
        L += [(c1, c1, 3)] * self.extra
        L += [(c1, c1, 2), (c1, c0, 1), (c0, c0, 0)]
        return L

    def offsets(self):
        offs, o = [], 0
        for cin, cout, _ in self.layers():
            offs.append((o, o + 27 * cin * cout))
            o += 27 * cin * cout + cout
        return offs, o

    def nparam(self) -> int:
        _, o = self.offsets()
        return o + self.c0 + 1

    def unpack(self, p):
        offs, ho = self.offsets()
        convs = []
        for (cin, cout, _), (wo, bo) in zip(self.layers(), offs):
            convs.append((p[wo:bo].reshape(27, cout, cin), p[bo:bo + cout]))
        return convs, p[ho:ho + self.c0], p[ho + self.c0]


def _taps():
    for t in range(27):
        yield t, t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1


def _shift(x: np.ndarray, dz: int, dy: int, dx: int, pery: bool) -> np.ndarray:
    """s[z,y,x] = x[z+dz, y+dy, x+dx]; wrapped in z and x, zero beyond y walls."""
    s = np.roll(x, shift=(-dz, -dy, -dx), axis=(0, 1, 2))
    if not pery and dy != 0:
        s = s.copy()
        if dy == 1:
            s[:, -1] = 0.0
        else:
            s[:, 0] = 0.0
    return s


def conv3(x, w, pery):
    """Sum over taps of shift(x) @ w[tap].T: [z,y,x,cin] -> [z,y,x,cout]."""
    out = np.zeros(x.shape[:3] + (w.shape[1],))
    for t, dz, dy, dx in _taps():
        out += _shift(x, dz, dy, dx, pery) @ w[t].T
    return out


def conv3_data_grad(g, w, pery):
    """Gradient of conv3 with respect to x given the output gradient g."""
    out = np.zeros(g.shape[:3] + (w.shape[2],))
    for t, dz, dy, dx in _taps():
        out += _shift(g, -dz, -dy, -dx, pery) @ w[t]
    return out


def conv3_weight_grad(x, g, pery):
    """dW[tap][co][ci] = sum_v g[v,co] shift(x)[v,ci]."""
    cin, cout = x.shape[3], g.shape[3]
    dw = np.zeros((27, cout, cin))
    g2 = g.reshape(-1, cout)
    for t, dz, dy, dx in _taps():
        dw[t] = g2.T @ _shift(x, dz, dy, dx, pery).reshape(-1, cin)
    return dw


def pool(x):
    nz, ny, nx, c = x.shape
    return x.reshape(nz // 2, 2, ny // 2, 2, nx // 2, 2, c).mean(axis=(1, 3, 5))


def up(x):
    return x.repeat(2, axis=0).repeat(2, axis=1).repeat(2, axis=2)


def down_sum(x):
    nz, ny, nx, c = x.shape
    return x.reshape(nz // 2, 2, ny // 2, 2, nx // 2, 2, c).sum(axis=(1, 3, 5))


def loss_grad(net: Net, params: np.ndarray, in4: np.ndarray, target: np.ndarray, shape, bf16: bool = True,
              masks=None, return_masks: bool = False):
    """Forward and backward of the network on one field.

    in4: [NIN][n] cell inputs (x fastest), target: [n], shape = (nx, ny, nz).
    Returns (loss, grad (flat like params), out [n]).  loss = mean((out-t)^2).
    ``masks`` (one boolean array per convolution, as returned with
    ``return_masks``) fixes which pre-activations count as positive, so that
    finite differences do not cross the kinks of the leaky ReLU.
    """
    nx, ny, nz = shape
    n = nx * ny * nz
    R = bf16_round if bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    p = np.asarray(params, dtype=np.float64)
    convs, hw, hb = net.unpack(p)
    wq = [(R(w), b) for w, b in convs]
    s = net.slope
    x0 = np.zeros((nz, ny, nx, C_IN))
    x0[..., :NIN] = np.asarray(in4, dtype=np.float64).reshape(NIN, nz, ny, nx).transpose(1, 2, 3, 0)
    x0 = R(x0)

    M = [None] * len(convs)

    def fwd(i, x):
        w, b = wq[i]
        pre = conv3(x, w, net.pery) + b
        M[i] = masks[i] if masks is not None else pre > 0.0
        return R(np.where(M[i], pre, pre * s))

    def dl(i):
        return np.where(M[i], 1.0, s)

    A = [None] * len(convs)
    P = [None] * 4
    Uu = [None] * 3
    A[0] = fwd(0, x0)
    A[1] = fwd(1, A[0])
    for lv in range(1, 4):
        P[lv] = R(pool(A[2 * lv - 1]))
        A[2 * lv] = fwd(2 * lv, P[lv])
        A[2 * lv + 1] = fwd(2 * lv + 1, A[2 * lv])
    ne = 8 + net.extra
    for e in range(8, ne):
        A[e] = fwd(e, A[e - 1])
    below = A[ne - 1]
    for lv in (2, 1, 0):
        li = ne + (2 - lv)
        Uu[lv] = R(up(below) + A[2 * lv + 1])
        A[li] = fwd(li, Uu[lv])
        below = A[li]
    out = A[-1] @ hw + hb
    t = np.asarray(target, dtype=np.float64).reshape(nz, ny, nx)
    e = out - t
    loss = float(np.mean(e * e))
    dO = 2.0 * e / n

    grads = [None] * len(convs)
    G = R(dO[..., None] * hw[None, None, None, :] * dl(len(convs) - 1))
    dhw = (A[-1] * dO[..., None]).reshape(-1, net.c0).sum(axis=0)
    dhb = dO.sum()

    def wgrad(i, x, g):
        grads[i] = (conv3_weight_grad(x, g, net.pery), g.reshape(-1, g.shape[3]).sum(axis=0))

    dU = [None] * 3
    for lv in (0, 1, 2):
        li = ne + (2 - lv)
        wgrad(li, Uu[lv], G)
        dU[lv] = conv3_data_grad(G, wq[li][0], net.pery)
        bl = ne + (2 - (lv + 1)) if lv < 2 else ne - 1
        G = R(down_sum(dU[lv]) * dl(bl))
    dP3 = None
    for li in range(ne - 1, 5, -1):
        x = P[3] if li == 6 else A[li - 1]
        wgrad(li, x, G)
        d = conv3_data_grad(G, wq[li][0], net.pery)
        if li == 6:
            dP3 = d
        else:
            G = R(d * dl(li - 1))
    dP = {3: dP3}
    for lv in (2, 1, 0):
        lb, la = 2 * lv + 1, 2 * lv
        G = R((dU[lv] + up(dP[lv + 1]) / 8.0) * dl(lb))
        wgrad(lb, A[la], G)
        d = conv3_data_grad(G, wq[lb][0], net.pery)
        G = R(d * dl(la))
        xa = x0 if lv == 0 else P[lv]
        wgrad(la, xa, G)
        if lv > 0:
            dP[lv] = conv3_data_grad(G, wq[la][0], net.pery)

    flat = []
    for dw, db in grads:
        flat.append(dw.ravel())
        flat.append(db)
    flat.append(dhw)
    flat.append(np.array([dhb]))
    if return_masks:
        return loss, np.concatenate(flat), out.ravel(), M
    return loss, np.concatenate(flat), out.ravel()


def init_params(net: Net, seed: int) -> np.ndarray:
    """Seeded random parameters for tests (not the library's initialisation)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(net.nparam())
    offs, ho = net.offsets()
    for (cin, cout, _), (wo, bo) in zip(net.layers(), offs):
        fan = 27 * (NIN if wo == 0 else cin)
        w = rng.uniform(-1, 1, (27, cout, cin)) * np.sqrt(6.0 / fan)
        if wo == 0:
            w[:, :, NIN:] = 0.0
        p[wo:bo] = w.ravel()
        p[bo:bo + cout] = rng.uniform(-0.1, 0.1, cout)
    p[ho:ho + net.c0] = rng.uniform(-1, 1, net.c0) * np.sqrt(3.0 / net.c0)
    p[ho + net.c0] = 0.05
    return p
