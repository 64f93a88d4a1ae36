"""CPU model of the warp-shuffle transforms of the FFT path (k_fft.cu,
warp_fft / wout / wline / wcol): the four-step split N = P x 32 with lane l
holding x[l + 32 m], the radix-2 decimation-in-frequency stages in registers
and across the lanes (half exchanges that trade a lane bit for a register
bit), the output positions, and the shared-memory swizzles.  The model follows the
kernel's index algebra step by step in numpy and is checked against
numpy.fft; the swizzles are checked for being permutations that spread each
warp access over all bank groups."""
import numpy as np
import pytest

PS = [1, 2, 4, 8, 16]


def brev(x, bits):
    r = 0
    for b in range(bits):
        r |= ((x >> b) & 1) << (bits - 1 - b)
    return r


def wout(lane, q, P):
    """Output index of register q of lane `lane` after warp_fft (k_fft.cu wout)."""
    if P == 1:
        return brev(lane, 5)
    p = (q & ~1) | (lane >> 4)
    cl = (q & 1) | ((lane & 15) << 1)
    return p + P * brev(cl, 5)


def warp_fft_model(x, inv=False):
    """X[wout(l, q)] = v[l][q] after the kernel's steps; returns X."""
    N = x.size
    P = N // 32
    sign = 1.0 if inv else -1.0
    W = lambda t, n: np.exp(sign * 2j * np.pi * t / n)
    lanes = np.arange(32)
    v = np.array([[x[l + 32 * m] for m in range(P)] for l in lanes], dtype=np.complex128)   # v[l][m]
    # P-point DIF in registers (same loop order as warp_fft)
    LP = P.bit_length() - 1
    for s in range(LP):
        h = P >> (s + 1)
        for b in range(0, P, 2 * h):
            for r in range(h):
                a0, a1 = v[:, b + r].copy(), v[:, b + r + h].copy()
                v[:, b + r] = a0 + a1
                v[:, b + r + h] = (a0 - a1) * W(r * (N // (2 * h)), N)
    y = np.empty_like(v)
    for i in range(P):
        y[:, brev(i, LP)] = v[:, i]
    for p in range(1, P):
        y[:, p] *= W(lanes * p, N)
    # 32-point DIF across the lanes, partner = lane ^ h.  P = 1 exchanges
    # its one element; for P >= 2 a lane keeps the element of each register
    # pair (p0, p0 + 1) whose bit 0 equals its lane bit h and sends the other.
    for s in range(5):
        h = 16 >> s
        up = (lanes & h) != 0
        w = W((lanes & (h - 1)) * (N // (2 * h)), N)
        if P == 1:
            o = y[lanes ^ h]
            y = np.where(up[:, None], (o - y) * w[:, None], y + o)
            continue
        ny = y.copy()
        for p0 in range(0, P, 2):
            keep = np.where(up, y[:, p0 + 1], y[:, p0])
            send = np.where(up, y[:, p0], y[:, p0 + 1])
            o = send[lanes ^ h]
            lo = np.where(up, o, keep)
            hi = np.where(up, keep, o)
            ny[:, p0] = lo + hi
            ny[:, p0 + 1] = (lo - hi) * w
        y = ny
    X = np.empty(N, dtype=np.complex128)
    for l in lanes:
        for q in range(P):
            X[wout(l, q, P)] = y[l, q]
    return X


@pytest.mark.parametrize("P", PS)
@pytest.mark.parametrize("inv", [False, True])
def test_four_step_model_matches_numpy(P, inv):
    rng = np.random.default_rng(7 + P)
    N = 32 * P
    x = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    X = warp_fft_model(x, inv)
    ref = np.fft.ifft(x) * N if inv else np.fft.fft(x)
    assert np.max(np.abs(X - ref)) <= 1e-12 * np.max(np.abs(ref))


def wsw(k, P, G):
    return 0 if P == 1 else (k // P) & (G - 1)


def wline(k, P, G):
    return k ^ wsw(k, P, G)


def wcol(kz, P, G):
    return (kz ^ wsw(kz, P, G)) & (G - 1)


def _groups(addr, elem_bytes):
    """Shared-memory wavefronts of one warp access to element addresses
    `addr`: the largest number of distinct elements that fall on one of the
    32 four-byte banks."""
    banks = {}
    for a in addr:
        for w in range(elem_bytes // 4):
            b = (a * elem_bytes // 4 + w) % 32
            banks.setdefault(b, set()).add(a)
    return max(len(s) for s in banks.values())


@pytest.mark.parametrize("P", PS)
@pytest.mark.parametrize("elem", [16, 8])
def test_line_swizzle_is_a_conflict_free_permutation(P, elem):
    G = 128 // elem
    N = 32 * P
    perm = [wline(k, P, G) for k in range(N)]
    assert sorted(perm) == list(range(N))
    best = (32 * elem) // 128                     # wavefronts of a 32-lane access
    lanes = range(32)
    for m in range(P):                            # natural-order reads k = l + 32 m
        assert _groups([wline(l + 32 * m, P, G) for l in lanes], elem) == best
    for q in range(P):                            # the transform's writes k = wout(l, q)
        assert _groups([wline(wout(l, q, P), P, G) for l in lanes], elem) == best


@pytest.mark.parametrize("P", PS)
@pytest.mark.parametrize("elem", [16, 8])
def test_z_tile_swizzle_is_a_conflict_free_permutation(P, elem):
    G = 128 // elem
    TX = G                                        # one 128-byte row segment per kz
    NZ = 32 * P
    addr = [kz * TX + (c ^ wcol(kz, P, G)) for kz in range(NZ) for c in range(TX)]
    assert sorted(addr) == list(range(NZ * TX))
    best = (32 * elem) // 128
    for c in range(TX):                           # a warp's column reads and writes
        for m in range(P):
            assert _groups([(l + 32 * m) * TX + (c ^ wcol(l + 32 * m, P, G)) for l in range(32)], elem) == best
        for q in range(P):
            kzs = [wout(l, q, P) for l in range(32)]
            assert _groups([kz * TX + (c ^ wcol(kz, P, G)) for kz in kzs], elem) == best
    # the cp.async staging: 32 consecutive threads cover 32 / TX whole rows
    for t0 in range(0, NZ * TX, 32):
        a = [(t // TX) * TX + ((t % TX) ^ wcol(t // TX, P, G)) for t in range(t0, t0 + 32)]
        assert _groups(a, elem) == best
