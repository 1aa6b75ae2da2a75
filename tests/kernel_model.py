"""Pure-Python model of the CUDA U-apply kernel (vpfhf_b200/csrc/u_apply.{cuh,cu}).

It replays the kernel's schedule -- xy tiles of 32 x TY elements, z-chunks with
one halo layer, the fixed-order node sums, the register carry between layers,
the seam partial buffers and the seam fix-up -- with bounds-checked numpy
indexing, and the modal ("mean/difference") element arithmetic.  The tests use
it to check the index arithmetic and buffer sizes on the CPU against the
oracle, independently of any GPU.
"""
from __future__ import annotations

import math

import numpy as np

TAU = math.sqrt(0.6) / 2
GT = (-TAU, 0.0, TAU)
GW = (5 / 18, 8 / 18, 5 / 18)


def modal8(f):
    a = np.empty(8)
    b = np.empty(8)
    m = np.empty(8)
    for p in range(4):
        a[2 * p] = 0.5 * (f[2 * p] + f[2 * p + 1])
        a[2 * p + 1] = f[2 * p + 1] - f[2 * p]
    for k in range(2):
        for al in range(2):
            lo, hi = a[al + 4 * k], a[al + 2 + 4 * k]
            b[al + 4 * k] = 0.5 * (lo + hi)
            b[al + 2 + 4 * k] = hi - lo
    for q in range(4):
        lo, hi = b[q], b[q + 4]
        m[q] = 0.5 * (lo + hi)
        m[q + 4] = hi - lo
    return m


def u_element_points(xn, vn, lam, mu, eta, h):
    """xn[8][3], vn[8] -> y[8][3]: the modal scheme summed point by point over the 27
    Gauss points (the reference arrangement of the row sums in u_element)."""
    ihx, ihy, ihz = 1 / h[0], 1 / h[1], 1 / h[2]
    vol = h[0] * h[1] * h[2]
    m = [modal8(xn[:, c]) for c in range(3)]
    mv = modal8(vn)
    QX = np.zeros((3, 4))
    QY = np.zeros((3, 4))
    QZ = np.zeros((3, 4))
    SZ = np.zeros((3, 3, 3))
    for gz in range(3):
        tz = GT[gz]
        SY = np.zeros((3, 3))
        for gy in range(3):
            ty = GT[gy]
            SX = np.zeros(3)
            for gx in range(3):
                tx = GT[gx]
                G = np.zeros((3, 3))
                for c in range(3):
                    G[c, 0] = (m[c][1] + m[c][3] * ty + m[c][5] * tz + m[c][7] * ty * tz) * ihx
                    G[c, 1] = (m[c][2] + m[c][3] * tx + m[c][6] * tz + m[c][7] * tx * tz) * ihy
                    G[c, 2] = (m[c][4] + m[c][5] * tx + m[c][6] * ty + m[c][7] * tx * ty) * ihz
                vg = (mv[0] + mv[1] * tx + mv[2] * ty + mv[3] * tx * ty + mv[4] * tz
                      + mv[5] * tx * tz + mv[6] * ty * tz + mv[7] * tx * ty * tz)
                ws = vol * GW[gx] * GW[gy] * GW[gz] * (vg * vg + eta)
                tr = G[0, 0] + G[1, 1] + G[2, 2]
                s = ws * (lam * tr * np.eye(3) + mu * (G + G.T))
                SX += s[:, 0]
                SY[:, gx] += s[:, 1]
                SZ[:, gy, gx] += s[:, 2]
            for c in range(3):
                QX[c] += SX[c] * np.array([1, ty, tz, ty * tz])
        for gx in range(3):
            tx = GT[gx]
            for c in range(3):
                QY[c] += SY[c, gx] * np.array([1, tx, tz, tx * tz])
    for gy in range(3):
        for gx in range(3):
            for c in range(3):
                QZ[c] += SZ[c, gy, gx] * np.array([1, GT[gx], GT[gy], GT[gx] * GT[gy]])

    def inv(Q, ih):
        A = np.empty((2, 2))
        for s1 in range(2):
            for s2 in range(2):
                a, b = 2 * s1 - 1, 2 * s2 - 1
                A[s1, s2] = (Q[0] / 4 + a * Q[1] / 2 + b * Q[2] / 2 + a * b * Q[3]) * ih
        return A

    y = np.zeros((8, 3))
    for c in range(3):
        Ax, Ay, Az = inv(QX[c], ihx), inv(QY[c], ihy), inv(QZ[c], ihz)
        for k in range(2):
            for j in range(2):
                for i in range(2):
                    y[i + 2 * j + 4 * k, c] = ((Ax[j, k] if i else -Ax[j, k])
                                               + (Ay[i, k] if j else -Ay[i, k])
                                               + (Az[i, j] if k else -Az[i, j]))
    return y


def u_element(xn, vn, lam, mu, eta, h):
    """xn[8][3], vn[8] -> y[8][3]; same arithmetic as u_element<T> in u_apply.cuh: the
    x-direction Gauss sum of every (gy, gz) row is done in closed form.  Along a row the gradient
    is G0 + t G1 (G1 has no x column) and v^2 + eta = a0 + a1 t + a2 t^2, so the
    3-point sums sum_gx w s and sum_gx w t s of the stress s = (v^2+eta) D(G) are
    Wr [(a0 + a2/12) D0 + (a1/12) D1] and Wr [(a1/12) D0 + ((a0 + 0.15 a2)/12) D1]
    with D0 = D(G0), D1 = D(G1) (sum_gx w_x t^2 = 1/12, sum_gx w_x t^4 = 0.15/12)."""
    ihx, ihy, ihz = 1 / h[0], 1 / h[1], 1 / h[2]
    vol = h[0] * h[1] * h[2]
    m = [modal8(xn[:, c]) for c in range(3)]
    mv = modal8(vn)
    QX = np.zeros((3, 4))
    QY = np.zeros((3, 4))
    QZ = np.zeros((3, 4))
    SZ0 = np.zeros((3, 3))
    SZ1 = np.zeros((3, 3))

    def D(G):
        tr = G[0, 0] + G[1, 1] + G[2, 2]
        return lam * tr * np.eye(3) + mu * (G + G.T)

    for gz in range(3):
        tz = GT[gz]
        SY0 = np.zeros(3)
        SY1 = np.zeros(3)
        for gy in range(3):
            ty = GT[gy]
            G0 = np.zeros((3, 3))
            G1 = np.zeros((3, 3))
            for c in range(3):
                G0[c, 0] = (m[c][1] + m[c][3] * ty + m[c][5] * tz + m[c][7] * ty * tz) * ihx
                G0[c, 1] = (m[c][2] + m[c][6] * tz) * ihy
                G1[c, 1] = (m[c][3] + m[c][7] * tz) * ihy
                G0[c, 2] = (m[c][4] + m[c][6] * ty) * ihz
                G1[c, 2] = (m[c][5] + m[c][7] * ty) * ihz
            q0 = mv[0] + mv[2] * ty + mv[4] * tz + mv[6] * ty * tz
            q1 = mv[1] + mv[3] * ty + mv[5] * tz + mv[7] * ty * tz
            a0, a1, a2 = q0 * q0 + eta, 2 * q0 * q1, q1 * q1
            Wr = vol * GW[gy] * GW[gz]
            D0, D1 = D(G0), D(G1)
            M0 = Wr * ((a0 + a2 / 12) * D0 + (a1 / 12) * D1)
            M1 = Wr * ((a1 / 12) * D0 + ((a0 + 0.15 * a2) / 12) * D1)
            for c in range(3):
                QX[c] += M0[c, 0] * np.array([1, ty, tz, ty * tz])
            SY0 += M0[:, 1]
            SY1 += M1[:, 1]
            SZ0[:, gy] += M0[:, 2]
            SZ1[:, gy] += M1[:, 2]
        for c in range(3):
            QY[c] += np.array([SY0[c], SY1[c], tz * SY0[c], tz * SY1[c]])
    for gy in range(3):
        for c in range(3):
            QZ[c] += np.array([SZ0[c, gy], SZ1[c, gy], GT[gy] * SZ0[c, gy], GT[gy] * SZ1[c, gy]])

    def inv(Q, ih):
        A = np.empty((2, 2))
        for s1 in range(2):
            for s2 in range(2):
                a, b = 2 * s1 - 1, 2 * s2 - 1
                A[s1, s2] = (Q[0] / 4 + a * Q[1] / 2 + b * Q[2] / 2 + a * b * Q[3]) * ih
        return A

    y = np.zeros((8, 3))
    for c in range(3):
        Ax, Ay, Az = inv(QX[c], ihx), inv(QY[c], ihy), inv(QZ[c], ihz)
        for k in range(2):
            for j in range(2):
                for i in range(2):
                    y[i + 2 * j + 4 * k, c] = ((Ax[j, k] if i else -Ax[j, k])
                                               + (Ay[i, k] if j else -Ay[i, k])
                                               + (Az[i, j] if k else -Az[i, j]))
    return y


def modal8s(f):
    """modal8 without the halvings: m'[p] = 2^(3 - popcount p) m[p]."""
    a = np.empty(8)
    b = np.empty(8)
    m = np.empty(8)
    for p in range(4):
        a[2 * p] = f[2 * p] + f[2 * p + 1]
        a[2 * p + 1] = f[2 * p + 1] - f[2 * p]
    for k in range(2):
        for al in range(2):
            lo, hi = a[al + 4 * k], a[al + 2 + 4 * k]
            b[al + 4 * k] = lo + hi
            b[al + 2 + 4 * k] = hi - lo
    for q in range(4):
        lo, hi = b[q], b[q + 4]
        m[q] = lo + hi
        m[q + 4] = hi - lo
    return m


def u_element_sums(xn, vn, lam, mu, eta, h, cubic=False):
    """The arithmetic of u_element<T, CUBIC> in u_apply.cuh: the row closed form of
    u_element on the modal sums in the doubled coordinate 2t (gradient column d =
    G'/(4 h_d), v = v'/8, moments against 2t), with W = Wr/64 and, on cubic cells,
    every 1/(4h) folded into W."""
    ihx, ihy, ihz = 1 / h[0], 1 / h[1], 1 / h[2]
    vol = h[0] * h[1] * h[2]
    assert not cubic or (ihx == ihy == ihz)
    m = [modal8s(xn[:, c]) for c in range(3)]
    mv = modal8s(vn)
    T2 = [2 * t for t in GT]
    sx, sy, sz = (1.0, 1.0, 1.0) if cubic else (ihx / 4, ihy / 4, ihz / 4)
    wsc = vol * ihx * ihx / 1024 if cubic else vol / 64
    QX = np.zeros((3, 4))
    QY = np.zeros((3, 4))
    QZ = np.zeros((3, 4))
    SZ0 = np.zeros((3, 3))
    SZ1 = np.zeros((3, 3))

    def D(G):
        tr = G[0, 0] + G[1, 1] + G[2, 2]
        return lam * tr * np.eye(3) + mu * (G + G.T)

    for gz in range(3):
        tz = T2[gz]
        SY0 = np.zeros(3)
        SY1 = np.zeros(3)
        for gy in range(3):
            ty = T2[gy]
            G0 = np.zeros((3, 3))
            G1 = np.zeros((3, 3))
            for c in range(3):
                ax = (m[c][1] + m[c][5] * tz) * sx
                bx = (m[c][3] + m[c][7] * tz) * sx
                G0[c, 0] = ax + bx * ty
                G0[c, 1] = (m[c][2] + m[c][6] * tz) * sy
                G1[c, 1] = (m[c][3] + m[c][7] * tz) * sy
                G0[c, 2] = (m[c][4] + m[c][6] * ty) * sz
                G1[c, 2] = (m[c][5] + m[c][7] * ty) * sz
            p0, p1 = mv[0] + mv[4] * tz, mv[1] + mv[5] * tz
            p2, p3 = mv[2] + mv[6] * tz, mv[3] + mv[7] * tz
            q0, q1 = p0 + p2 * ty, p1 + p3 * ty
            A0, A2, H1 = q0 * q0 + 64 * eta, q1 * q1, q0 * q1
            W = wsc * GW[gz] * GW[gy]
            C0, C1, E1 = W * (A0 + A2 / 3), W * 2 * H1 / 3, W * (A0 + 0.6 * A2) / 3
            d, e = D(G0), D(G1)
            n = C0 * d + C1 * e
            o = C1 * d + E1 * e
            for c in range(3):
                QX[c] += n[c, 0] * np.array([1, ty, tz, ty * tz])
            SY0 += n[:, 1]
            SY1 += o[:, 1]
            SZ0[:, gy] += n[:, 2]
            SZ1[:, gy] += o[:, 2]
        for c in range(3):
            QY[c] += np.array([SY0[c], SY1[c], tz * SY0[c], tz * SY1[c]])
    for gy in range(3):
        for c in range(3):
            QZ[c] += np.array([SZ0[c, gy], SZ1[c, gy], T2[gy] * SZ0[c, gy], T2[gy] * SZ1[c, gy]])

    # monomial coefficients in (s_i, s_j, s_k), then the signed 8-point butterfly
    y = np.zeros((8, 3))
    for c in range(3):
        w = np.zeros(8)
        w[1], w[2], w[4] = QX[c][0] * sx, QY[c][0] * sy, QZ[c][0] * sz
        w[3] = QX[c][1] * sx + QY[c][1] * sy
        w[5] = QX[c][2] * sx + QZ[c][1] * sz
        w[6] = QY[c][2] * sy + QZ[c][2] * sz
        w[7] = QX[c][3] * sx + QY[c][3] * sy + QZ[c][3] * sz
        for a in range(8):
            s = [1 if (a >> b) & 1 else -1 for b in range(3)]
            y[a, c] = sum(w[p] * np.prod([s[b] for b in range(3) if (p >> b) & 1]) for p in range(1, 8))
    return y


def u_element_const(xn, S, lam, mu, h, cubic=False):
    """xn[8][3] -> y[8][3] for an element whose phase field is the same at its 8 nodes
    (S = v^2 + eta at every point); same arithmetic as u_element_const<T> in u_apply.cuh.
    The stress is then the polynomial S D(G) with G bilinear per column, and its moments
    against {1, s_a, s_b, s_a s_b} (doubled coordinate s = 2t) are exact averages over the
    cell: E[s^2] = 1/3 and the odd moments vanish, which is also what the 3-point Gauss
    rule gives for these degrees.  With the modal sums m (modal8s) and k_d = 1/(4 h_d):
      T_B = sum_{e not in B} m[e][B + e] k_e                  (trace coefficient of s^B)
      R[c][d][B] = vol S 3^-|B| k_d [lambda [c == d] T_B
                   + mu (m[c][B + d] k_d + [c not in B] m[d][B + c] k_c)],
    and the node polynomial's coefficient of the monomial p (a set of axes) is
    w[p] = sum_{d in p} R[c][d][p - d]."""
    m = [modal8s(xn[:, c]) for c in range(3)]
    k = [0.25 / hh for hh in h]
    vol = h[0] * h[1] * h[2]
    T = {}
    for B in range(8):
        T[B] = sum(m[e][B | (1 << e)] * (1.0 if cubic else k[e]) for e in range(3)
                   if not (B >> e) & 1)
    y = np.zeros((8, 3))
    for c in range(3):
        w = np.zeros(8)
        for pset in range(1, 8):
            for d in range(3):
                if not (pset >> d) & 1:
                    continue
                B = pset & ~(1 << d)
                nb = bin(B).count("1")
                kd = 1.0 if cubic else k[d]
                kc = 1.0 if cubic else k[c]
                off = m[d][B | (1 << c)] * kc if not (B >> c) & 1 else 0.0
                if c == d:
                    inner = lam * T[B] + 2 * mu * m[c][B | (1 << c)] * kd
                else:
                    inner = mu * (m[c][B | (1 << d)] * kd + off)
                scale = vol * S * 3.0 ** -nb * (k[0] ** 2 if cubic else kd)
                w[pset] += scale * inner
        for a in range(8):
            sg = [1 if (a >> b) & 1 else -1 for b in range(3)]
            y[a, c] = sum(w[p] * np.prod([sg[b] for b in range(3) if (p >> b) & 1])
                          for p in range(1, 8))
    return y


def plan(nx, ny, nz, TY, zc):
    ntx = -(-(nx - 1) // 32)
    nty = -(-(ny - 1) // TY)
    nzc = -(-nz // zc)
    return dict(ntx=ntx, nty=nty, zc=zc, nzc=nzc,
                seamX=(ntx - 1) * nz * ny * 12, seamY=(nty - 1) * nz * nx * 6)


def segments(ntx, nty, nz, ncta, b):
    """Block b's share of the tile engine's work: node planes [U b / ncta, U (b+1) / ncta)
    of the U = ntx nty nz (column, plane) units, column-major, cut at column ends into
    (bx, by, z0, z1) chunks (tile_apply_kernel)."""
    U = ntx * nty * nz
    u, u1 = U * b // ncta, U * (b + 1) // ncta
    out = []
    while u < u1:
        col, z0 = u // nz, u % nz
        z1 = min(nz, z0 + (u1 - u))
        out.append((col % ntx, col // ntx, z0, z1))
        u += z1 - z0
    return out


def tile_layer_const(v, n, TY):
    """u_classify_kernel: cls[col, k] for tile col = by ntx + bx and element layer k, True
    when the tile's elements (32 x TY, clipped to the grid) in layer k all have 8 equal
    nodal v."""
    nx, ny, nz = n
    vv = v.reshape(nz, ny, nx)
    corners = [vv[kk:nz - 1 + kk, j:ny - 1 + j, i:nx - 1 + i] for kk in (0, 1) for j in (0, 1) for i in (0, 1)]
    const = np.all([c == corners[0] for c in corners[1:]], axis=0)  # [nez, ney, nex]
    ntx, nty = -(-(nx - 1) // 32), -(-(ny - 1) // TY)
    cls = np.zeros((ntx * nty, nz - 1), bool)
    for by in range(nty):
        for bx in range(ntx):
            blk = const[:, by * TY:(by + 1) * TY, bx * 32:(bx + 1) * 32]
            cls[by * ntx + bx] = blk.reshape(nz - 1, -1).all(axis=1)
    return cls


def unit_lists(cls, nz, ncta):
    """unit_lists_kernel: per list l (0: both adjacent element layers constant, 1: the
    rest) the runs (col, z0, z1, units before) in column order, the block starts (the run
    holding unit total b / ncta) and the unit totals."""
    runs, nez = [[], []], nz - 1

    def utype(f, z):
        below = z == 0 or f[z - 1]
        above = z == nez or f[z]
        return 0 if below and above else 1

    tot = [0, 0]
    for c, f in enumerate(cls):
        z0, t0 = 0, utype(f, 0)
        for z in range(1, nz + 1):
            t = utype(f, z) if z < nz else -1
            if t != t0:
                runs[t0].append((c, z0, z, tot[t0]))
                tot[t0] += z - z0
                z0, t0 = z, t
    start = [[0] * ncta, [0] * ncta]
    for l in (0, 1):
        for b in range(ncta):
            ub = tot[l] * b // ncta
            cand = [i for i, r in enumerate(runs[l]) if r[3] <= ub]
            start[l][b] = cand[-1] if cand else 0
    return runs, start, tot


def list_segments(runs, start, total, ncta, b, ntx):
    """Block b's (bx, by, z0, z1) segments of one unit list (tile_apply_kernel, list
    mode)."""
    u, u1 = total * b // ncta, total * (b + 1) // ncta
    r, out = start[b], []
    while u < u1:
        col, rz0, rz1, w = runs[r]
        r += 1
        z0, z1 = rz0 + (u - w), min(rz1, rz0 + (u1 - w))
        out.append((col % ntx, col // ntx, z0, z1))
        u += z1 - z0
    return out


def u_apply_tiled(x, v, bcbits, n, h, lam, mu, eta, TY=8, zc=5, element=None, ncta=None,
                  chunks=None):
    """Replays u_apply_kernel + u_seam_fixup_kernel; returns y (3N).  ncta: the kernel's
    balanced segments over ncta blocks instead of z-chunks of zc planes; chunks: given
    (bx, by, z0, z1, element) segments."""
    nx, ny, nz = n
    nex, ney = nx - 1, ny - 1
    P = plan(nx, ny, nz, TY, zc)
    ntx, nty = P["ntx"], P["nty"]
    N = nx * ny * nz
    y = np.full(3 * N, np.nan)
    seamX = np.full(max(P["seamX"], 1), np.nan)
    seamY = np.full(max(P["seamY"], 1), np.nan)
    written = np.zeros(3 * N, int)
    el_fn = element or (lambda xn, vn: u_element(xn, vn, lam, mu, eta, h))
    BX, BY = 33, TY + 1
    nslot = -(-(BX * BY) // (32 * TY))

    def nid(i, j, k):
        assert 0 <= i < nx and 0 <= j < ny and 0 <= k < nz
        return (k * ny + j) * nx + i

    if chunks is not None:
        pass
    elif ncta is None:  # z-chunks of zc planes per xy tile
        chunks = [(bx, by, bz * zc, min(bz * zc + zc, nz), el_fn) for bz in range(P["nzc"])
                  for by in range(nty) for bx in range(ntx) if bz * zc < nz]
    else:  # the kernel's balanced segments
        chunks = [c + (el_fn,) for b in range(ncta) for c in segments(ntx, nty, nz, ncta, b)]
    for bx, by, z0, z1, seg_el in chunks:
        X0, Y0 = 32 * bx, TY * by
        kf, kl = max(z0 - 1, 0), min(z1, nz - 1) - 1
        carry = np.zeros((32 * TY, nslot, 3))

        def emit(l, w, X, Y, z, val):
            left, right = (l == 0 and bx > 0), (l == 32 and bx < ntx - 1)
            bot, top = (w == 0 and by > 0), (w == TY and by < nty - 1)
            nn = nid(X, Y, z)
            if not (left or right or bot or top):
                for c in range(3):
                    y[3 * nn + c] = x[3 * nn + c] if (bcbits[nn] >> c) & 1 else val[c]
                    written[3 * nn + c] += 1
            elif left or right:
                i = bx if left else bx + 1
                slot = (2 if bot else 0) + (1 if left else 0)
                base = ((((i - 1) * nz + z) * ny + Y) * 4 + slot) * 3
                assert 0 <= base and base + 3 <= P["seamX"]
                assert np.isnan(seamX[base:base + 3]).all()
                seamX[base:base + 3] = val
            else:
                j = by if bot else by + 1
                base = ((((j - 1) * nz + z) * nx + X) * 2 + (1 if bot else 0)) * 3
                assert 0 <= base and base + 3 <= P["seamY"]
                assert np.isnan(seamY[base:base + 3]).all()
                seamY[base:base + 3] = val

        def plane(kz):
            sx = np.zeros((4, BY, BX))
            for w in range(BY):
                for l in range(BX):
                    X, Y = X0 + l, Y0 + w
                    if X < nx and Y < ny:
                        nn = nid(X, Y, kz)
                        sx[0:3, w, l] = x[3 * nn:3 * nn + 3]
                        sx[3, w, l] = v[nn]
            return sx

        buf = {kf: plane(kf)}
        for k in range(kf, kl + 1):
            buf[k + 1] = plane(k + 1)
            sc = np.zeros((24, TY, 32))
            for wy in range(TY):
                for lane in range(32):
                    ex, ey = X0 + lane, Y0 + wy
                    if ex < nex and ey < ney:
                        xn = np.zeros((8, 3))
                        vn = np.zeros(8)
                        for kk in range(2):
                            for j in range(2):
                                for i in range(2):
                                    a = i + 2 * j + 4 * kk
                                    xn[a] = buf[k + kk][0:3, wy + j, lane + i]
                                    vn[a] = buf[k + kk][3, wy + j, lane + i]
                        yc = seg_el(xn, vn)
                        sc[:, wy, lane] = yc.reshape(24)
            for tid in range(32 * TY):
                for si in range(nslot):
                    s = tid + si * 32 * TY
                    if s >= BX * BY:
                        continue
                    l, w = s % BX, s // BX
                    X, Y = X0 + l, Y0 + w
                    if X >= nx or Y >= ny:
                        continue
                    p0 = np.zeros(3)
                    p1 = np.zeros(3)
                    for dw in range(2):  # x-sums (left element's corner + own) per row
                        ew, j = w - 1 + dw, 1 - dw
                        if ew < 0 or ew >= TY:
                            continue
                        for kk, acc in ((0, p0), (1, p1)):
                            xs = np.zeros(3)
                            for dl in range(2):
                                el, i = l - 1 + dl, 1 - dl
                                if 0 <= el < 32:
                                    a = i + 2 * j + 4 * kk
                                    xs = xs + sc[a * 3:a * 3 + 3, ew, el]
                            acc += xs
                    if k >= z0:
                        emit(l, w, X, Y, k, carry[tid, si] + p0)
                    carry[tid, si] = p1
        if z1 == nz:
            for tid in range(32 * TY):
                for si in range(nslot):
                    s = tid + si * 32 * TY
                    if s >= BX * BY:
                        continue
                    l, w = s % BX, s // BX
                    X, Y = X0 + l, Y0 + w
                    if X < nx and Y < ny:
                        emit(l, w, X, Y, nz - 1, carry[tid, si])
    # seam fix-up
    nxs = (ntx - 1) * nz * ny
    nys = (nty - 1) * nz * nx
    for t in range(nxs + nys):
        if t < nxs:
            Y = t % ny
            r = t // ny
            z, i = r % nz, r // nz + 1
            onY = (Y % TY == 0) and Y > 0 and (Y // TY < nty)
            p = seamX[t * 12:t * 12 + 12]
            val = ((p[0:3] + p[3:6]) + p[6:9]) + p[9:12] if onY else p[0:3] + p[3:6]
            X = 32 * i
        else:
            u = t - nxs
            X = u % nx
            r = u // nx
            z, j = r % nz, r // nz + 1
            if X % 32 == 0 and X > 0 and X // 32 < ntx:
                continue
            p = seamY[u * 6:u * 6 + 6]
            val = p[0:3] + p[3:6]
            Y = TY * j
        assert not np.isnan(val).any(), "seam slot never written"
        nn = nid(X, Y, z)
        for c in range(3):
            y[3 * nn + c] = x[3 * nn + c] if (bcbits[nn] >> c) & 1 else val[c]
            written[3 * nn + c] += 1
    assert (written == 1).all(), "every dof must be written exactly once"
    return y


def v_element(xn, cg, aeps, h):
    """xn[8], cg[27] (weight-premultiplied mass coefficient) -> y[8]; the arithmetic of
    v_element<T> in ops.cuh: closed-form stiffness moments, sum-factorised mass moments."""
    ihx, ihy, ihz = 1 / h[0], 1 / h[1], 1 / h[2]
    vol = h[0] * h[1] * h[2]
    m = modal8(xn)
    av = aeps * vol
    kx, ky, kz = av * ihx * ihx, av * ihy * ihy, av * ihz * ihz

    def bfly(q0, q1, q2, q3):
        A = np.empty((2, 2))
        for s1 in range(2):
            for s2 in range(2):
                a, b = 2 * s1 - 1, 2 * s2 - 1
                A[s1, s2] = q0 + a * q1 + b * q2 + a * b * q3
        return A

    AX = bfly(kx / 4 * m[1], kx / 24 * m[3], kx / 24 * m[5], kx / 144 * m[7])
    AY = bfly(ky / 4 * m[2], ky / 24 * m[3], ky / 24 * m[6], ky / 144 * m[7])
    AZ = bfly(kz / 4 * m[4], kz / 24 * m[5], kz / 24 * m[6], kz / 144 * m[7])
    P00, P01, P10, P11 = np.zeros(3), np.zeros(3), np.zeros(3), np.zeros(3)
    for gz in range(3):
        tz = GT[gz]
        p = [m[0] + m[4] * tz, m[1] + m[5] * tz, m[2] + m[6] * tz, m[3] + m[7] * tz]
        L0, L1 = np.zeros(3), np.zeros(3)
        for gy in range(3):
            ty = GT[gy]
            q0, q1 = p[0] + p[2] * ty, p[1] + p[3] * ty
            psi = [cg[gx + 3 * gy + 9 * gz] * (q0 + q1 * GT[gx]) for gx in range(3)]
            L0[gy] = psi[0] + psi[1] + psi[2]
            L1[gy] = psi[2] - psi[0]
        P00[gz], P01[gz] = L0.sum(), L0[2] - L0[0]
        P10[gz], P11[gz] = L1.sum(), L1[2] - L1[0]
    t = GT[2]
    M = np.array([P00.sum(), t * P10.sum(), t * P01.sum(), t * t * P11.sum(),
                  t * (P00[2] - P00[0]), t * t * (P10[2] - P10[0]), t * t * (P01[2] - P01[0]),
                  t ** 3 * (P11[2] - P11[0])])
    y = np.zeros(8)
    for k in range(2):
        for j in range(2):
            for i in range(2):
                sgn = np.array([2 * i - 1, 2 * j - 1, 2 * k - 1])
                val = 0.0
                for p in range(8):  # value part: prod_d (1/2 + s_d t_d) moments
                    al, be, ga = p & 1, (p >> 1) & 1, p >> 2
                    f = 1.0
                    for d, mode in enumerate((al, be, ga)):
                        f *= sgn[d] if mode else 0.5
                    val += f * M[p]
                y[i + 2 * j + 4 * k] = ((AX[j, k] * sgn[0] + AY[i, k] * sgn[1]) + AZ[i, j] * sgn[2]) + val
    return y
