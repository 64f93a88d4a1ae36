"""CPU model of the FP32 red-black correction sweeps of the mixed-precision
projection: the two colour sweeps as the kernels k_sor_sweep32 run them, and
the fused red+black pass k_rb32_fused (k_sor_mixed.cu) step by step, with its
tiles, halo threads, plane loads (the kernel stages them with cp.async in a
ring of five planes), shared-memory rings and register history.  Arrays are in
natural padded order [k][j][i] (the CUDA code's colour-split storage is an
index permutation).  Both use the same FP32 operations (one rounding per
multiply, add and fused multiply-add), so the fused pass must reproduce the
two sweeps bit for bit.
"""
from __future__ import annotations

import numpy as np

F = np.float32


def fma(a, b, c):
    """FP32 fused multiply-add: the product of two FP32 values is exact in
    FP64; one rounding of the FP64 sum to FP32 (a double rounding that both
    models share, so it cannot hide a dataflow difference)."""
    return F(np.float64(a) * np.float64(b) + np.float64(c))


def mul(a, b):
    return F(np.float64(a) * np.float64(b))


def sub(a, b):
    return F(np.float64(a) - np.float64(b))


def div_of(P, r, ui, uip, vj, vjp, wk, wkp):
    return fma(sub(wkp, wk), P["idz"], fma(sub(vjp, vj), P["idy"], fma(sub(uip, ui), P["idx"], r)))


class Grid:
    def __init__(self, nx, ny, nz, py):
        self.nx, self.ny, self.nz, self.py = nx, ny, nz, py

    def ip(self, i):
        return 1 if i == self.nx else i + 1

    def jp(self, j):
        return 1 if (self.py and j == self.ny) else j + 1

    def kp(self, k):
        return 1 if k == self.nz else k + 1


def two_sweeps(g, P, du, dv, dw, dp, r, mu_u, mu_v, mu_w, fac):
    """One red+black iteration as two colour sweeps (first colour: i+j+k odd)."""
    du, dv, dw, dp = (a.copy() for a in (du, dv, dw, dp))
    for parity in (1, 0):
        for k in range(1, g.nz + 1):
            for j in range(1, g.ny + 1):
                for i in range(1, g.nx + 1):
                    if (i + j + k) & 1 != parity:
                        continue
                    ip, jp, kp = g.ip(i), g.jp(j), g.kp(k)
                    ui, uip, vj, vjp = du[k, j, i], du[k, j, ip], dv[k, j, i], dv[k, jp, i]
                    wk, wkp = dw[k, j, i], dw[kp, j, i]
                    phi = mul(div_of(P, r[k, j, i], ui, uip, vj, vjp, wk, wkp), fac[j, i])
                    dp[k, j, i] = fma(phi, P["idt"], dp[k, j, i])
                    px, py_, pz = mul(phi, P["idx"]), mul(phi, P["idy"]), mul(phi, P["idz"])
                    du[k, j, i] = fma(-px, mu_u[j, i], ui)
                    du[k, j, ip] = fma(px, mu_u[j, ip], uip)
                    if g.py or j > 1:
                        dv[k, j, i] = fma(-py_, mu_v[j, i], vj)
                    if g.py or j < g.ny:
                        dv[k, jp, i] = fma(py_, mu_v[jp, i], vjp)
                    dw[k, j, i] = fma(-pz, mu_w[j, i], wk)
                    dw[kp, j, i] = fma(pz, mu_w[j, i], wkp)
    return du, dv, dw, dp


def fused(g, P, xu, xv, xw, dp, r, mu_u, mu_v, mu_w, fac, TI, TJ, TK):
    """The fused pass, thread by thread and phase by phase as k_rb32_fused
    runs it: reads x*, writes the returned y* (faces) and dp (in place)."""
    nx, ny, nz, PY = g.nx, g.ny, g.nz, g.py
    yu, yv, yw = (np.full_like(a, np.nan) for a in (xu, xv, xw))
    yv[:, 0, :] = xv[:, 0, :]          # wall rows are never written (they stay 0)
    yv[:, ny + 1, :] = xv[:, ny + 1, :]
    dp = dp.copy()
    PW, RW, CW = TI // 2 + 2, TJ + 3, 2 * (TI // 2 + 2)

    def cx(i):
        m = i % nx
        return nx if m == 0 else m

    def cy(j):
        return ((j - 1) % ny) + 1 if PY else j

    def cz(k):
        return ((k - 1) % nz) + 1

    def exists(j):
        return PY or 1 <= j <= ny

    for bz in range((nz + TK - 1) // TK):
        for by in range((ny + TJ - 1) // TJ):
            for bx in range((nx + TI - 1) // TI):
                i0, j0, k0 = bx * TI, 1 + by * TJ, 1 + bz * TK
                thr = [(tx, ty) for ty in range(RW) for tx in range(PW)]
                U = np.zeros((2, RW, PW + 1), F)
                PH = np.zeros((2, RW, CW + 2), F)
                st = {}
                for tx, ty in thr:
                    ie, j = i0 - 2 + 2 * tx, j0 - 2 + ty
                    ex = exists(j)
                    jc = cy(j)
                    s = {"ie": ie, "j": j, "ex": ex, "ic": (cx(ie), cx(ie + 1)), "jc": jc}
                    # per-column constants
                    if ex:
                        s["fac"] = (fac[jc, cx(ie)], fac[jc, cx(ie + 1)])
                        s["mu_u"] = (mu_u[jc, cx(ie)], mu_u[jc, cx(ie + 1)], mu_u[jc, cx(ie + 2)])
                        s["mu_w"] = (mu_w[jc, cx(ie)], mu_w[jc, cx(ie + 1)])
                        s["mu_v"] = (mu_v[jc, cx(ie)], mu_v[jc, cx(ie + 1)])
                        jn = cy(j + 1) if PY else j + 1
                        s["mu_vn"] = (mu_v[jn, cx(ie)], mu_v[jn, cx(ie + 1)]) if jn <= ny + 1 else (F(0), F(0))
                    s["p"] = [[F(0)] * 3, [F(0)] * 3]          # phi history per column: planes q, q-1, q-2
                    st[(tx, ty)] = s

                def load(s, q):
                    """Plane q: u, v, v(j+1), r, dp of the two cells and w(q+1)."""
                    j, ex = s["j"], s["ex"]
                    kc, kn = cz(q), cz(q + 1)
                    jn = cy(j + 1) if PY else j + 1
                    out = {}
                    for c in (0, 1):
                        ic = s["ic"][c]
                        out[("u", c)] = xu[kc, s["jc"], ic] if ex else F(0)
                        out[("v", c)] = xv[kc, s["jc"], ic] if ex else F(0)
                        out[("vn", c)] = xv[kc, jn, ic] if ex else F(0)
                        out[("r", c)] = r[kc, s["jc"], ic] if ex else F(0)
                        out[("dp", c)] = dp[kc, s["jc"], ic] if ex else F(0)
                        out[("w1", c)] = xw[kn, s["jc"], ic] if ex else F(0)
                    return out

                for s in st.values():               # prologue: w(k0-2), plane k0-2
                    kc = cz(k0 - 2)
                    s["w"] = [xw[kc, s["jc"], s["ic"][c]] if s["ex"] else F(0) for c in (0, 1)]
                    s["cur"] = load(s, k0 - 2)
                    s["prev"] = None
                for q in range(k0 - 2, k0 + TK + 1):
                    # A: publish this plane's u(even)
                    for (tx, ty), s in st.items():
                        U[q & 1, ty, tx] = s["cur"][("u", 0)]
                    # B: red cell of plane q
                    for (tx, ty), s in st.items():
                        j = s["j"]
                        c = 0 if (j + q) & 1 else 1
                        if not (s["ex"] and 2 * tx + c <= TI + 2 and ty <= TJ + 2):
                            continue
                        cur = s["cur"]
                        ui = cur[("u", c)]
                        uip = cur[("u", 1)] if c == 0 else U[q & 1, ty, tx + 1]
                        vj, vjp = cur[("v", c)], cur[("vn", c)]
                        wk, wkp = s["w"][c], cur[("w1", c)]
                        phi = mul(div_of(P, cur[("r", c)], ui, uip, vj, vjp, wk, wkp), s["fac"][c])
                        s["p"][c][0] = phi
                        PH[q & 1, ty, 2 * tx + c + 1] = phi
                    # C: black cell of plane q-1 (the column that was red at q)
                    if q >= k0:
                        for (tx, ty), s in st.items():
                            j = s["j"]
                            c = 0 if (j + q) & 1 else 1
                            if not (s["ex"] and 1 <= 2 * tx + c <= TI + 1 and 1 <= ty <= TJ + 1):
                                continue
                            pv, cur = s["prev"], s["cur"]
                            h = (q - 1) & 1
                            p_left = s["p"][0][1] if c == 1 else PH[h, ty, 2 * tx]
                            p_right = s["p"][1][1] if c == 0 else PH[h, ty, 2 * tx + 3]
                            mu_ui = s["mu_u"][c]
                            mu_uip = s["mu_u"][1] if c == 0 else s["mu_u"][2]
                            up_ip = pv[("u", 1)] if c == 0 else U[h, ty, tx + 1]
                            ui = fma(mul(p_left, P["idx"]), mu_ui, pv[("u", c)])
                            uip = fma(-mul(p_right, P["idx"]), mu_uip, up_ip)
                            vj = pv[("v", c)]
                            if exists(j - 1):
                                vj = fma(mul(PH[h, ty - 1, 2 * tx + c + 1], P["idy"]), s["mu_v"][c], vj)
                            vjp = pv[("vn", c)]
                            if exists(j + 1):
                                vjp = fma(-mul(PH[h, ty + 1, 2 * tx + c + 1], P["idy"]), s["mu_vn"][c], vjp)
                            wk = fma(mul(s["p"][c][2], P["idz"]), s["mu_w"][c], s["wp"][c])
                            wkp = fma(-mul(s["p"][c][0], P["idz"]), s["mu_w"][c], s["w"][c])
                            phi = mul(div_of(P, pv[("r", c)], ui, uip, vj, vjp, wk, wkp), s["fac"][c])
                            s["p"][c][1] = phi
                            PH[h, ty, 2 * tx + c + 1] = phi
                    # D: final faces and dp of plane q-1
                    if q >= k0 + 1 and q - 1 <= nz:
                        h = (q - 1) & 1
                        for (tx, ty), s in st.items():
                            j = s["j"]
                            if not (s["ex"] and 2 <= ty < TJ + 2 and j <= ny):
                                continue
                            pv = s["prev"]
                            for c in (0, 1):
                                i = s["ie"] + c
                                if not (2 <= 2 * tx + c < TI + 2 and i < nx):
                                    continue
                                red = (c + j + q - 1) & 1 == 1
                                phi = s["p"][c][1]
                                px, py_, pz = mul(phi, P["idx"]), mul(phi, P["idy"]), mul(phi, P["idz"])
                                p_left = s["p"][0][1] if c == 1 else PH[h, ty, 2 * tx]
                                pxl = mul(p_left, P["idx"])
                                mu = s["mu_u"][c]
                                if red:
                                    u2 = fma(pxl, mu, fma(-px, mu, pv[("u", c)]))
                                else:
                                    u2 = fma(-px, mu, fma(pxl, mu, pv[("u", c)]))
                                v_lo = PY or j > 1
                                down = exists(j - 1)
                                pyd = mul(PH[h, ty - 1, 2 * tx + c + 1], P["idy"]) if down else F(0)
                                mv = s["mu_v"][c]
                                v1 = pv[("v", c)]
                                if red:
                                    v1 = fma(-py_, mv, v1) if v_lo else v1
                                    v1 = fma(pyd, mv, v1) if down else v1
                                else:
                                    v1 = fma(pyd, mv, v1) if down else v1
                                    v1 = fma(-py_, mv, v1) if v_lo else v1
                                pzb = mul(s["p"][c][2], P["idz"])
                                mw = s["mu_w"][c]
                                if red:
                                    w2 = fma(pzb, mw, fma(-pz, mw, s["wp"][c]))
                                else:
                                    w2 = fma(-pz, mw, fma(pzb, mw, s["wp"][c]))
                                kc, jc, ic = cz(q - 1), s["jc"], s["ic"][c]
                                if k0 <= q - 1 < k0 + TK:
                                    yu[kc, jc, ic] = u2
                                    yv[kc, jc, ic] = v1
                                    yw[kc, jc, ic] = w2
                                    dp[kc, jc, ic] = fma(phi, P["idt"], pv[("dp", c)])
                    # shift to the next plane
                    for s in st.values():
                        s["prev"] = s["cur"]
                        s["wp"] = s["w"]
                        s["w"] = [s["cur"][("w1", c)] for c in (0, 1)]
                        s["cur"] = load(s, q + 1)
                        for c in (0, 1):
                            s["p"][c] = [F(0), s["p"][c][0], s["p"][c][1]]
    return yu, yv, yw, dp
