"""CPU model of k_sor_sweep32v (k_sor_mixed.cu): one FP32 colour sweep with V
consecutive cells of the swept colour per thread, on the colour-split arrays
with their padded rows.  It runs the kernel thread by thread on flat arrays
laid out as the CUDA code lays them out, and logs every access, so that the
tests can check, beside the result, that
- every access stays inside its array and every vector access is aligned;
- no element is written by two threads;
- no value that feeds an update is one that another thread writes.
All threads read the state before the sweep (what a thread sees when no
other thread writes what it uses), so the model's result is the kernel's.
The arithmetic is rb32_model's (the same FP32 roundings as sweep32_update).
"""
from __future__ import annotations

import numpy as np

from tests.rb32_model import F, div_of, fma, mul


def split_stride(nx):
    return ((nx + 2) // 2 + 3) & ~3


class Layout:
    def __init__(self, nx, ny, nz):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.nyp, self.nzp = ny + 2, nz + 2
        self.hs = split_stride(nx)
        self.H = self.hs * self.nyp * self.nzp
        self.PH = self.hs * self.nyp
        self.n = 2 * self.H          # elements of one field
        self.npl = 2 * self.PH       # elements of one factor plane

    def cidx(self, i, j, k):
        return ((i + j + k) & 1) * self.H + (k * self.nyp + j) * self.hs + (i >> 1)

    def pidx2(self, i, j):
        return ((i + j) & 1) * self.PH + j * self.hs + (i >> 1)


def to_split(L, a, fill):
    """Natural [k][j][i] padded array -> colour-split flat array; positions
    that hold no element get `fill` (a NaN payload, so that a write of a
    computed value there shows)."""
    out = np.full(L.n, fill, dtype=F)
    for k in range(L.nzp):
        for j in range(L.nyp):
            for i in range(L.nx + 2):
                out[L.cidx(i, j, k)] = a[k, j, i]
    return out


def plane_to_split(L, a, fill):
    out = np.full(L.npl, fill, dtype=F)
    for j in range(L.nyp):
        for i in range(L.nx + 2):
            out[L.pidx2(i, j)] = a[j, i]
    return out


def from_split(L, s):
    out = np.zeros((L.nzp, L.nyp, L.nx + 2), dtype=F)
    for k in range(L.nzp):
        for j in range(L.nyp):
            for i in range(L.nx + 2):
                out[k, j, i] = s[L.cidx(i, j, k)]
    return out


class Log:
    def __init__(self):
        self.writes = {}      # (array, index) -> thread
        self.used = []        # (array, index, thread)
        self.errors = []

    def check(self, arr, idx, size, V, thread, what):
        if idx < 0 or idx + V > size:
            self.errors.append(f"{what} {arr}[{idx}:{idx + V}] outside 0..{size} (thread {thread})")
        if V > 1 and idx % V != 0:
            self.errors.append(f"{what} {arr}[{idx}] not aligned to {V} (thread {thread})")

    def write(self, arr, idx, V, size, thread):
        self.check(arr, idx, size, V, thread, "store")
        for e in range(V):
            key = (arr, idx + e)
            if key in self.writes and self.writes[key] != thread:
                self.errors.append(f"{arr}[{idx + e}] written by threads {self.writes[key]} and {thread}")
            self.writes[key] = thread


def vector_sweep(L, P, py, parity, V, reverse, f, mu32, fac32, log=None):
    """One colour sweep as k_sor_sweep32v<PY, V> runs it.  f: dict of the
    colour-split flat arrays du, dv, dw, dp, r (updated copies returned)."""
    old = {n: a.copy() for n, a in f.items()}    # what every thread reads
    new = {n: a.copy() for n, a in f.items()}
    log = log or Log()
    nx, ny, nz, hs = L.nx, L.ny, L.nz, L.hs
    nwin = (nx // 2 + V) // V
    per_plane = nwin * ny
    nthr = per_plane * nz
    half = nx // 2
    sizes = {"du": L.n, "dv": L.n, "dw": L.n, "dp": L.n, "r": L.n, "mu": 3 * L.npl, "fac": L.npl}
    arrays = dict(old, mu=mu32, fac=fac32)

    for g in range(nthr):
        kk = g // per_plane
        rem = g - kk * per_plane
        j = rem // nwin + 1
        p0 = V * (rem - (j - 1) * nwin)
        k = nz - kk if reverse else kk + 1
        cs = 1 - parity
        eo = (cs + j + k) & 1
        jp = 1 if (py and j == ny) else j + 1
        kp = 1 if k == nz else k + 1
        H = L.H
        own = cs * H + (k * L.nyp + j) * hs + p0
        oth = (1 - cs) * H + (k * L.nyp + j) * hs
        ojp = (1 - cs) * H + (k * L.nyp + jp) * hs + p0
        okp = (1 - cs) * H + (kp * L.nyp + j) * hs + p0
        PH, npl = L.PH, L.npl
        hp = (eo + j) & 1
        mown = hp * PH + j * hs + p0
        mox = (1 - hp) * PH + j * hs
        mjp = (1 - hp) * PH + jp * hs + p0

        def ld(arr, idx, n=V):
            log.check(arr, idx, sizes[arr], n, g, "load")
            return [arrays[arr][idx + e] for e in range(n)]

        u0, v0, w0, q = ld("du", own), ld("dv", own), ld("dw", own), ld("dp", own)
        ux, vy, wz, rr = ld("du", oth + p0), ld("dv", ojp), ld("dw", okp), ld("r", own)
        mu_u, mu_v, mu_w = ld("mu", mown), ld("mu", npl + mown), ld("mu", 2 * npl + mown)
        fc, mu_ux, mu_vy = ld("fac", mown), ld("mu", mox + p0), ld("mu", npl + mjp)
        xe = p0 + V if eo else 0
        need_xe = (p0 + V < hs) if eo else (p0 <= half < p0 + V)
        uxe = muxe = F(0.0)
        if need_xe:
            uxe, = ld("du", oth + xe, 1)
            muxe, = ld("mu", mox + xe, 1)
        v_lo, v_hi = py or j > 1, py or j < ny
        for e in range(V):
            p = p0 + e
            valid = (p < half) if eo else (1 <= p <= half)
            wrap = (not eo) and p == half
            if e + 1 < V:
                uip = ux[e + 1] if eo else (uxe if wrap else ux[e])
                muip = mu_ux[e + 1] if eo else (muxe if wrap else mu_ux[e])
                src = oth + p0 + e + 1 if eo else (oth + xe if wrap else oth + p0 + e)
            else:
                uip = uxe if (eo or wrap) else ux[e]
                muip = muxe if (eo or wrap) else mu_ux[e]
                src = oth + xe if (eo or wrap) else oth + p0 + e
            if not valid:
                continue
            for arr, idx in (("du", own + e), ("du", src), ("dv", own + e), ("dv", ojp + e), ("dw", own + e),
                             ("dw", okp + e), ("dp", own + e), ("r", own + e)):
                log.used.append((arr, idx, g))
            phi = mul(div_of(P, rr[e], u0[e], uip, v0[e], vy[e], w0[e], wz[e]), fc[e])
            q[e] = fma(phi, P["idt"], q[e])
            px, pyv, pz = mul(phi, P["idx"]), mul(phi, P["idy"]), mul(phi, P["idz"])
            u0[e] = fma(-px, mu_u[e], u0[e])
            uip = fma(px, muip, uip)
            if v_lo:
                v0[e] = fma(-pyv, mu_v[e], v0[e])
            if v_hi:
                vy[e] = fma(pyv, mu_vy[e], vy[e])
            wk, wkp = w0[e], wz[e]
            w0[e] = fma(-pz, mu_w[e], wk)
            wz[e] = fma(pz, mu_w[e], wkp)
            dst = oth + (p + 1 if eo else (0 if wrap else p))
            log.write("du", dst, 1, L.n, g)
            new["du"][dst] = uip
        for arr, base, vals in (("du", own, u0), ("dv", own, v0), ("dw", own, w0), ("dp", own, q),
                                ("dv", ojp, vy), ("dw", okp, wz)):
            log.write(arr, base, V, L.n, g)
            for e in range(V):
                new[arr][base + e] = vals[e]
    for arr, idx, g in log.used:
        w = log.writes.get((arr, idx))
        if w is not None and w != g:
            log.errors.append(f"thread {g} uses {arr}[{idx}], which thread {w} writes")
    return new, log
