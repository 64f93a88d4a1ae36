"""CPU model of the potential form of the FP32 correction sweeps
(k_pot_sweep in k_sor_mixed.cu).

The red-black update of pressure_redblack.f90:117-241 moves the faces of a
cell by -+ phi/h * mu and adds phi/dt_gamma to p.  Starting from zero
corrections, every face therefore equals h^-1 mu (Phi(low cell) - Phi(high
cell)) where Phi is the sum of the phi of a cell so far, and the cell
divergence the next update needs is a 7-point stencil of Phi:

  e(c) = r~(c) + sum over the faces of c of  a_f (Phi(c) - Phi(neighbour)),
  a_f  = h^-2 mu_f  (0 for a wall face, which never moves),

so the same iteration can carry Phi alone: Phi(c) += fac(c) e(c).  The
kernel keeps Phi and r~ in a colour-split layout of its own:

  cell (i, j, k), i in 0..nx+1, lives in half (i + j + k) & 1 at
  (k (ny+2) + j) hq + 3 + (i + 1) / 2,

so a row of one half holds its nx/2 interior cells at positions 4..4+nx/2-1
(16-byte aligned), the copy of cell nx at position 3 when the row holds even
cells, and the copy of cell 1 at position 4+nx/2 when it holds odd cells.
Planes 0 and nz+1 (and rows 0 and ny+1 when y is periodic) hold copies of
planes nz and 1 (rows ny and 1).  A sweep writes those copies of the cells
it updates, so every neighbour read needs no wrap test.

This model runs the kernel thread by thread (V positions of a row per
thread, TX x TY threads per block, a march over KZ planes), logs every
access, and lets the tests check that accesses stay inside the arrays and
are aligned, that no element is written twice, that no value a thread uses
is written by another thread, and that the result equals a plain
restatement of the face-form sweeps.  Arithmetic is FP64 here; the kernel
rounds the same operations in FP32.
"""
from __future__ import annotations

import numpy as np


class PotLayout:
    def __init__(self, nx, ny, nz):
        assert nx % 2 == 0
        self.nx, self.ny, self.nz = nx, ny, nz
        self.hq = ((nx // 2 + 5) + 3) & ~3          # positions 3 .. nx/2+4, rows 16-byte aligned
        self.rowz = self.hq * (ny + 2)               # one plane of one half
        self.H = ((self.rowz * (nz + 2)) + 63) & ~63  # one half, 256-byte aligned
        self.n = 2 * self.H

    def idx(self, i, j, k):
        return ((i + j + k) & 1) * self.H + (k * (self.ny + 2) + j) * self.hq + 3 + (i + 1) // 2

    def row(self, h, j, k):
        return h * self.H + (k * (self.ny + 2) + j) * self.hq


def tables(nx, ny, nz, py, idx2, idy2, idz2, mu_u, mu_v, mu_w, fac):
    """Per (i, j) column: a_x of its low x face, a_y of its low y face (0 at
    a wall), a_z, fac; column nx+1 repeats column 1's a_x, row ny+1 holds the
    top faces (0 at a wall, row 1's a_y when y is periodic)."""
    t = np.zeros((ny + 2, nx + 2, 4))
    for j in range(1, ny + 1):
        for i in range(1, nx + 1):
            t[j, i, 0] = idx2 * mu_u[j, i]
            t[j, i, 1] = idy2 * mu_v[j, i] if (py or j > 1) else 0.0
            t[j, i, 2] = idz2 * mu_w[j, i]
            t[j, i, 3] = fac[j, i]
        t[j, nx + 1, 0] = t[j, 1, 0]
    for i in range(1, nx + 1):
        t[ny + 1, i, 1] = t[1, i, 1] if py else 0.0
    return t


def face_sweeps(nx, ny, nz, py, idx, idy, idz, idt, du, dv, dw, dp, r, mu_u, mu_v, mu_w, fac, iters):
    """The face form (sweep32_update's operations, FP64): iters red+black
    iterations, first colour i+j+k odd."""
    du, dv, dw, dp = (a.copy() for a in (du, dv, dw, dp))
    for _ in range(iters):
        for parity in (1, 0):
            for k in range(1, nz + 1):
                kp = 1 if k == nz else k + 1
                for j in range(1, ny + 1):
                    jp = 1 if (py and j == ny) else j + 1
                    for i in range(1, nx + 1):
                        if (i + j + k) & 1 != parity:
                            continue
                        ip = 1 if i == nx else i + 1
                        e = (r[k, j, i] + (du[k, j, ip] - du[k, j, i]) * idx + (dv[k, jp, i] - dv[k, j, i]) * idy
                             + (dw[kp, j, i] - dw[k, j, i]) * idz)
                        phi = e * fac[j, i]
                        dp[k, j, i] += phi * idt
                        du[k, j, i] -= phi * idx * mu_u[j, i]
                        du[k, j, ip] += phi * idx * mu_u[j, ip]
                        if py or j > 1:
                            dv[k, j, i] -= phi * idy * mu_v[j, i]
                        if py or j < ny:
                            dv[k, jp, i] += phi * idy * mu_v[jp, i]
                        dw[k, j, i] -= phi * idz * mu_w[j, i]
                        dw[kp, j, i] += phi * idz * mu_w[j, i]
    return du, dv, dw, dp


def faces_of_phi(L, py, idx, idy, idz, idt, phi, mu_u, mu_v, mu_w):
    """The face corrections and dp that Phi stands for (what k_pot_apply adds
    in FP64), as natural [k][j][i] padded arrays."""
    nx, ny, nz = L.nx, L.ny, L.nz
    shp = (nz + 2, ny + 2, nx + 2)
    du, dv, dw, dp = (np.zeros(shp) for _ in range(4))
    P = lambda i, j, k: phi[L.idx(i, j, k)]
    for k in range(1, nz + 1):
        for j in range(1, ny + 1):
            for i in range(1, nx + 1):
                c = P(i, j, k)
                du[k, j, i] = idx * mu_u[j, i] * (P(i - 1, j, k) - c)
                if py or j > 1:
                    dv[k, j, i] = idy * mu_v[j, i] * (P(i, j - 1, k) - c)
                dw[k, j, i] = idz * mu_w[j, i] * (P(i, j, k - 1) - c)
                dp[k, j, i] = c * idt
    return du, dv, dw, dp


def to_layout(L, a, fill):
    out = np.full(L.n, fill)
    for k in range(1, L.nz + 1):
        for j in range(1, L.ny + 1):
            for i in range(1, L.nx + 1):
                out[L.idx(i, j, k)] = a[k, j, i]
    return out


class Log:
    def __init__(self):
        self.reads = {}    # element -> set of threads
        self.writes = {}   # element -> list of threads

    def rd(self, t, e):
        self.reads.setdefault(e, set()).add(t)

    def wr(self, t, e):
        self.writes.setdefault(e, []).append(t)


def sweep(L, py, cs, phi, r, tab, V, TX, TY, KZ, log=None):
    """One colour sweep (cells of colour cs = (i+j+k)&1), thread by thread as
    k_pot_sweep runs it.  Every thread reads the state before the sweep,
    which is what it sees when no other thread writes what it uses (the
    tests check that from the log).  Returns the new phi."""
    nx, ny, nz, hq = L.nx, L.ny, L.nz, L.hq
    assert (nx // 2) % V == 0 and 4 % V == 0
    old = phi.copy()
    new = phi.copy()
    tabf = tab.reshape(-1, 4)
    ncol = nx + 2
    gx = (nx // 2 // V + TX - 1) // TX
    gy = (ny + TY - 1) // TY
    gz = (nz + KZ - 1) // KZ
    oh = 1 - cs

    def vld(t, base, n=V):
        assert base % V == 0 or n == 1, "misaligned vector load"
        assert 0 <= base and base + n <= L.n
        for e in range(n):
            if log:
                log.rd(t, base + e)
        return [old[base + e] for e in range(n)]

    def vst(t, base, vals):
        assert base % V == 0 and 0 <= base and base + len(vals) <= L.n
        for e, v in enumerate(vals):
            if log:
                log.wr(t, base + e)
            new[base + e] = v

    def sst(t, e, v):
        assert 0 <= e < L.n
        if log:
            log.wr(t, e)
        new[e] = v

    for bz in range(gz):
        for by in range(gy):
            for bx in range(gx):
                for ty in range(TY):
                    for tx in range(TX):
                        t = (bx, by, bz, tx, ty)
                        q0 = V * (bx * TX + tx)
                        j = 1 + by * TY + ty
                        if q0 >= nx // 2 or j > ny:
                            continue
                        k0 = 1 + bz * KZ
                        k1 = min(k0 + KZ - 1, nz)
                        # coefficients of the 2V columns 2 q0 + 1 .. 2 q0 + 2V and the
                        # a_x of column 2 q0 + 2V + 1; the a_y of row j + 1
                        c0 = j * ncol + 2 * q0 + 1
                        cr = [tabf[c0 + m] for m in range(2 * V + 1)]
                        cu = [tabf[(j + 1) * ncol + 2 * q0 + 1 + m][1] for m in range(2 * V)]
                        # odd cells 2q+1 (column m = 2e), even cells 2q+2 (m = 2e+1)
                        co = {par: [(cr[2 * e + par][0], cr[2 * e + par + 1][0], cr[2 * e + par][1],
                                     cu[2 * e + par], cr[2 * e + par][2], cr[2 * e + par][3]) for e in range(V)]
                              for par in (0, 1)}
                        zm = vld(t, L.row(oh, j, k0 - 1) + 4 + q0)
                        z0 = vld(t, L.row(oh, j, k0) + 4 + q0)
                        for k in range(k0, k1 + 1):
                            zp = vld(t, L.row(oh, j, k + 1) + 4 + q0)
                            sb = L.row(cs, j, k) + 4 + q0
                            s = vld(t, sb)
                            rr = [r[sb + e] for e in range(V)]
                            ym = vld(t, L.row(oh, j - 1, k) + 4 + q0)
                            yp = vld(t, L.row(oh, j + 1, k) + 4 + q0)
                            eo = (cs + j + k) & 1    # 1: the swept cells have odd i
                            ob = L.row(oh, j, k)
                            if eo:
                                xs = vld(t, ob + 3 + q0, 1)[0]
                                xl = [xs] + z0[:V - 1]
                                xr = z0
                                cc = co[0]
                            else:
                                xs = vld(t, ob + 4 + q0 + V, 1)[0]
                                xl = z0
                                xr = z0[1:] + [xs]
                                cc = co[1]
                            out = []
                            for e in range(V):
                                axl, axr, ayl, ayr, az, f = cc[e]
                                c = s[e]
                                E = (rr[e] + axl * (c - xl[e]) + axr * (c - xr[e]) + ayl * (c - ym[e])
                                     + ayr * (c - yp[e]) + az * ((c - zm[e]) + (c - zp[e])))
                                out.append(c + f * E)
                            vst(t, sb, out)
                            # copies of the updated cells
                            if eo and q0 == 0:
                                sst(t, L.row(cs, j, k) + 4 + nx // 2, out[0])       # cell nx+1 = cell 1
                            if not eo and q0 + V == nx // 2:
                                sst(t, L.row(cs, j, k) + 3, out[V - 1])            # cell 0 = cell nx
                            if k == nz:
                                vst(t, L.row(cs, j, 0) + 4 + q0, out)
                            if k == 1:
                                vst(t, L.row(cs, j, nz + 1) + 4 + q0, out)
                            if py and j == ny:
                                vst(t, L.row(cs, 0, k) + 4 + q0, out)
                            if py and j == 1:
                                vst(t, L.row(cs, ny + 1, k) + 4 + q0, out)
                            zm, z0 = z0, zp
    return new


def tabu_of(L, tab):
    """k_pot_tables' tabu: row j holds the a_y of column i's top face,
    cy(i, j+1), at (i - 1); rows ncu = nx rounded up to 4 apart."""
    nx, ny = L.nx, L.ny
    ncu = (nx + 3) & ~3
    tu = np.zeros((ny + 2) * ncu)
    for j in range(1, ny + 2):
        for i in range(1, nx + 1):
            tu[(j - 1) * ncu + (i - 1)] = tab[j, i, 1]
    return tu, ncu


def sweep_rows(L, py, cs, phi, r, tab, KZ):
    """One colour sweep as k_pot_sweep_w runs it: one warp per row (nx/2 =
    32 V positions), 8 rows per block, x neighbours by shuffle with the
    row's wrap, rows j-1 and j+1 through the block's shared buffer (warps 0
    and 7 load the rows just outside the block), coefficients from the
    column table and tabu, the next lane's first a_x by shuffle."""
    nx, ny, nz = L.nx, L.ny, L.nz
    half = nx // 2
    assert half % 32 == 0 and ny % 8 == 0
    V = half // 32
    NW = 8
    old = phi.copy()
    new = phi.copy()
    tabf = tab.reshape(-1, 4)
    ncol = nx + 2
    tu, ncu = tabu_of(L, tab)
    oh = 1 - cs
    for by in range(ny // NW):
        for bz in range((nz + KZ - 1) // KZ):
            j0 = 1 + by * NW
            k0 = 1 + bz * KZ
            k1 = min(k0 + KZ - 1, nz)
            # per lane coefficient sets, like the kernel's registers
            co = {}
            for w in range(NW):
                j = j0 + w
                for lane in range(32):
                    q0 = V * lane
                    cr = [tabf[j * ncol + 2 * q0 + 1 + m] for m in range(2 * V)]
                    up = [tu[j * ncu + 2 * q0 + m] for m in range(2 * V)]
                    axl = [[0.0] * V for _ in range(2)]
                    axr = [[0.0] * V for _ in range(2)]
                    ayl = [[0.0] * V for _ in range(2)]
                    ayr = [[0.0] * V for _ in range(2)]
                    az = [[0.0] * V for _ in range(2)]
                    fc = [[0.0] * V for _ in range(2)]
                    for m in range(2 * V):
                        s_, e = m & 1, m >> 1
                        axl[s_][e], ayl[s_][e], az[s_][e], fc[s_][e] = cr[m]
                        ayr[s_][e] = up[m]
                        if m > 0:
                            axr[(m - 1) & 1][(m - 1) >> 1] = cr[m][0]
                    co[(w, lane)] = [axl, axr, ayl, ayr, az, fc]
                for lane in range(32):   # the shuffle of the next lane's first a_x
                    co[(w, lane)][1][1][V - 1] = co[(w, (lane + 1) % 32)][0][0][0]
            for k in range(k0, k1 + 1):
                rows = {}
                for w in range(-1, NW + 1):
                    rows[w] = [old[L.row(oh, j0 + w, k) + 4 + q] for q in range(half)]
                for w in range(NW):
                    j = j0 + w
                    z0 = rows[w]
                    zm = [old[L.row(oh, j, k - 1) + 4 + q] for q in range(half)]
                    zp = [old[L.row(oh, j, k + 1) + 4 + q] for q in range(half)]
                    odd = (cs + j + k) & 1
                    for lane in range(32):
                        axl, axr, ayl, ayr, az, fc = co[(w, lane)]
                        st = 0 if odd else 1
                        q0 = V * lane
                        out = []
                        for e in range(V):
                            q = q0 + e
                            xl = z0[(q - 1) % half] if odd else z0[q]
                            xr = z0[q] if odd else z0[(q + 1) % half]
                            c = old[L.row(cs, j, k) + 4 + q]
                            rr = r[L.row(cs, j, k) + 4 + q]
                            E = (rr + axl[st][e] * (c - xl) + axr[st][e] * (c - xr)
                                 + ayl[st][e] * (c - rows[w - 1][q]) + ayr[st][e] * (c - rows[w + 1][q])
                                 + az[st][e] * ((c - zm[q]) + (c - zp[q])))
                            out.append(c + fc[st][e] * E)
                        sk = L.row(cs, j, k) + 4 + q0
                        for e in range(V):
                            new[sk + e] = out[e]
                        if odd and lane == 0:
                            new[sk + half] = out[0]
                        if not odd and lane == 31:
                            new[sk - q0 - 1] = out[V - 1]
                        if k == nz:
                            for e in range(V):
                                new[L.row(cs, j, 0) + 4 + q0 + e] = out[e]
                        if k == 1:
                            for e in range(V):
                                new[L.row(cs, j, nz + 1) + 4 + q0 + e] = out[e]
                        if py and j == ny:
                            for e in range(V):
                                new[L.row(cs, 0, k) + 4 + q0 + e] = out[e]
                        if py and j == 1:
                            for e in range(V):
                                new[L.row(cs, ny + 1, k) + 4 + q0 + e] = out[e]
    return new
