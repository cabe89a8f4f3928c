"""NumPy backend of the oracle driver: the reference's hot-path kernels restated as whole-array NumPy operations in ONE
process (NumPy's element-wise loops, no threads), for the single-process CPU baseline.

TEST INFRASTRUCTURE ONLY: the oracle driver (``oracle/model.py``, backend ``'numpy'``) runs it for the tests and the
benchmark's CPU-baseline leg; the product never imports it.

Each method restates one reference kernel over its whole domain, with the same argument list as ``oracle/oracle.c``
(the reference kernel's own, after ``rows``). Every element gets the reference's operations in the reference's order:
each binary operation rounds once (NumPy applies them one by one, as the reference's ``--fmad=false`` build does), slot
loops run slot by slot with a mask standing for the reference's ``break`` at the trailing -1 pads (``np.where``, never
an added zero, so signed zeros are kept), and neighbour sums accumulate in the reference's slot order. Results are
bit-identical to the C restatement except where ``exp`` is called (the interfacial stress and the stress term), whose
last bit NumPy and libm may round differently.
"""
import numpy as np


def _rows(a, n):
    return a.reshape(-1, n)


def _edge_h(a, b, shelf):
    """Edge thickness of a layer: the two cells' mean, or the thinner one under the shelf (reference layers.cu:41-45)."""
    mean = 0.5 * (a + b)
    if shelf > 0:
        m = np.where(a < b, a, b)
        return np.where(m < shelf, m, mean)
    return mean


def _slot(tab, m):
    """Column m of an (items, slots) index table: the index (pads clamped to 0 for the gather) and the mask of real
    entries."""
    e = tab[:, m]
    ok = e >= 0
    return np.where(ok, e, 0), ok


def _upwind(f, p, eI, eJ):
    """reference fused.cu:124-127"""
    return f * np.where(f >= 0, p[eI], p[eJ])


def _hoflux(f, ps, psf, idx, wt, eI, eJ, beta):
    """reference fused.cu:131-138: the 3rd-order edge flux from the 8-point stencil (two 4-point halves a and b)."""
    a = wt[:, 0] * psf[idx[:, 0]] + wt[:, 1] * psf[idx[:, 1]] + wt[:, 2] * psf[idx[:, 2]] + wt[:, 3] * psf[idx[:, 3]]
    b = wt[:, 4] * psf[idx[:, 4]] + wt[:, 5] * psf[idx[:, 5]] + wt[:, 6] * psf[idx[:, 6]] + wt[:, 7] * psf[idx[:, 7]]
    return f * (0.5 * (ps[eI] + ps[eJ]) - (a + b)) + np.abs(f) * ((b - a) * beta)


class NumpyKernels:
    def __init__(self):
        self._csr = {}

    def __call__(self, name, n, rows, args):
        with np.errstate(divide='ignore', invalid='ignore', over='ignore'):
            getattr(self, name)(rows, *args)

    # ---- the layers' step (reference kernels/layers.cu, fused.cu, trisk.cu) ----

    def lay_eta(self, rows, N, L, h, b, eta):
        """reference layers.cu:33-38"""
        h = _rows(h, N)
        z = b.copy()
        for k in range(L - 1, -1, -1):
            z = z + h[k]
        eta[:] = z

    def lay_ubar(self, rows, N, E, L, h, u, eI, eJ, shelf, ubar, ob):
        """reference layers.cu:64-74"""
        if ob is not None:
            raise NotImplementedError('numpy oracle: the shelf-bed option is not restated')
        h, u = _rows(h, N), _rows(u, E)
        H, U = np.zeros(E), np.zeros(E)
        for k in range(L):
            he = _edge_h(h[k][eI], h[k][eJ], shelf)
            H = H + he
            U = U + he * u[k]
        ubar[:] = U / H

    def lay_bern(self, rows, N, E, L, h, u, b, gp, cellEdge, le, de, areaCell, B, sig, zm, tide):
        """reference layers.cu:83-109, fixed-g' branch"""
        if sig is not None or zm is not None or tide is not None:
            raise NotImplementedError('numpy oracle: per-cell buoyancy and the tide are not restated')
        h, u, B = _rows(h, N), _rows(u, E), _rows(B, N)
        ce = cellEdge.reshape(N, 6)
        z = [None] * L
        s = b.copy()
        for k in range(L - 1, -1, -1):
            s = s + h[k]
            z[k] = s
        Mp = np.zeros(N)
        for k in range(L):
            if k > 0:
                Mp = Mp + gp[k - 1] * z[k]
            ke = np.zeros(N)
            for m in range(6):
                e, ok = _slot(ce, m)
                ke = np.where(ok, ke + le[e] * de[e] * 0.25 * u[k][e] * u[k][e], ke)
            B[k] = Mp + ke / areaCell

    def swe_vertex(self, rows, N, E, NV, h, u, vCell, vSlot, kite, vEdge, vEdgeSign, de, areaV, fV, q):
        """reference fused.cu:82-98 (FP64: divisions)"""
        h, u, q, kite = _rows(h, N), _rows(u, E), _rows(q, NV), kite.reshape(-1)
        vc, vs = vCell.reshape(NV, 3), vSlot.reshape(NV, 3).astype(np.int64)
        ve, vg = vEdge.reshape(NV, 3), vEdgeSign.reshape(NV, 3).astype(np.float64)
        for l in range(rows):
            hv, z = np.zeros(NV), np.zeros(NV)
            for k in range(3):
                c = vc[:, k]
                hv = hv + kite[c * 6 + vs[:, k]] * h[l][c] * 1.0
            for k in range(3):
                e = ve[:, k]
                z = z + vg[:, k] * de[e] * u[l][e]
            q[l] = (z / areaV + fV) / (hv / areaV)

    def lay_edge_hq(self, rows, N, E, NV, h, q, eI, eJ, ev1, ev2, shelf, u, he, pk, ob):
        """reference layers.cu:254-263 (pk packed [edge][layer][h_e, u, q_e])"""
        if ob is not None:
            raise NotImplementedError('numpy oracle: the shelf-bed option is not restated')
        h, q, u, he = _rows(h, N), _rows(q, NV), _rows(u, E), _rows(he, E)
        p = pk.reshape(E, rows, 3)
        for l in range(rows):
            hv = _edge_h(h[l][eI], h[l][eJ], shelf)
            he[l] = hv
            p[:, l, 0] = hv
            p[:, l, 1] = u[l]
            p[:, l, 2] = 0.5 * (q[l][ev1] + q[l][ev2])

    def _trisk_rows(self, eoeStart, eoe, E):
        """The CSR rows as a padded (E, width) table of positions into eoe, with the mask of real entries."""
        key = (eoeStart.ctypes.data, eoe.ctypes.data, E)
        if key not in self._csr:
            start = eoeStart.astype(np.int64)
            cnt = np.diff(start)
            width = int(cnt.max()) if E else 0
            pos = start[:-1, None] + np.arange(width)[None, :]
            ok = np.arange(width)[None, :] < cnt[:, None]
            self._csr[key] = (np.where(ok, pos, 0), ok)
        return self._csr[key]

    def lay_slow(self, rows, N, E, L, pk, wf, hedge, u, B, eoeStart, eoe, eI, eJ, de, drag, stress, floor_, nu4, lap4,
                 theta, pibar, dts, thin, shelf, Tp, G, He, ubs, sig, zm, ob, cd_bot, cbot):
        """reference layers.cu:269-359, Boussinesq branch"""
        if any(a is not None for a in (theta, pibar, sig, zm, ob, cbot)) or cd_bot > 0:
            raise NotImplementedError('numpy oracle: option branch of the slow tendency not restated')
        p = pk.reshape(E, L, 3)
        hedge, u, B, Tp = _rows(hedge, E), _rows(u, E), _rows(B, N), _rows(Tp, E)
        lap4 = None if lap4 is None else _rows(lap4, E)
        pos, okm = self._trisk_rows(eoeStart, eoe, E)
        nb = eoe[pos]
        T, hev = [], []
        H, U = np.zeros(E), np.zeros(E)
        for k in range(L):
            he = hedge[k]
            cap = thin * he
            qf = p[:, k, 2]
            Q = np.zeros(E)
            for m in range(pos.shape[1]):
                j = nb[:, m]
                h2 = p[j, k, 0]
                h2 = np.where(h2 > cap, cap, h2)
                F2 = h2 * p[j, k, 1]
                Q = np.where(okm[:, m], Q + wf[pos[:, m]] * F2 * 0.5 * (qf + p[j, k, 2]), Q)
            if shelf > 0:
                sq = np.where(he < shelf, np.where(he - 2 * floor_ > 0, (he - 2 * floor_) / (shelf - 2 * floor_), 0.0), 1.0)
            else:
                sq = np.ones(E)
            d = Q - (sq * (B[k][eJ] - B[k][eI])) / de - (drag[k] + (1 - sq) / 21600.0) * u[k]
            ck = stress[k]
            if ck != 0:
                r = ck / np.where(he > floor_, he, floor_)
                d = d - np.where(r * dts > 1e-8, (1 - np.exp(-r * dts)) / dts, r) * u[k]
            if nu4 != 0:
                d = d - nu4 * lap4[k]
            T.append(d)
            hev.append(he)
            H = H + he
            U = U + he * u[k]
        GT = np.zeros(E)
        for k in range(L):
            GT = GT + hev[k] * T[k]
        g = GT / H
        for k in range(L):
            Tp[k] = T[k] - g
        G[:] = g
        He[:] = H
        ubs[:] = U / H

    def cell_div(self, rows, N, E, u, cellEdge, cellSign, le, areaCell, D):
        """reference trisk.cu:14-25"""
        u, D = _rows(u, E), _rows(D, N)
        ce, cs = cellEdge.reshape(N, 6), cellSign.reshape(N, 6).astype(np.float64)
        for l in range(rows):
            s = np.zeros(N)
            for m in range(6):
                e, ok = _slot(ce, m)
                s = np.where(ok, s + cs[:, m] * le[e] * u[l][e], s)
            D[l] = s / areaCell

    def vertex_curl(self, rows, E, NV, u, vEdge, vEdgeSign, de, areaV, Z):
        """reference trisk.cu:27-37"""
        u, Z = _rows(u, E), _rows(Z, NV)
        ve, vg = vEdge.reshape(NV, 3), vEdgeSign.reshape(NV, 3).astype(np.float64)
        for l in range(rows):
            z = np.zeros(NV)
            for k in range(3):
                e = ve[:, k]
                z = z + vg[:, k] * de[e] * u[l][e]
            Z[l] = z / areaV

    def edge_lap(self, rows, N, E, NV, D, Z, eI, eJ, ev1, ev2, de, le, out):
        """reference trisk.cu:39-45"""
        D, Z, out = _rows(D, N), _rows(Z, NV), _rows(out, E)
        for l in range(rows):
            out[l] = (D[l][eJ] - D[l][eI]) / de - (Z[l][ev2] - Z[l][ev1]) / le

    def bt_eta(self, rows, N, He, ub, cellEdge, cellSign, le, areaCell, tau, eta, eta_prev):
        """reference layers.cu:366-377"""
        ce, cs = cellEdge.reshape(N, 6), cellSign.reshape(N, 6).astype(np.float64)
        eta_prev[:] = eta
        div = np.zeros(N)
        for m in range(6):
            e, ok = _slot(ce, m)
            div = np.where(ok, div + cs[:, m] * le[e] * He[e] * ub[e], div)
        eta[:] = eta - (tau * div) / areaCell

    def bt_u(self, rows, E, eta, eta_prev, gamma, G, eI, eJ, de, Gc, tau, ub, acc):
        """reference layers.cu:379-388"""
        v = ub.copy()
        acc += v
        ej = Gc[eJ] * (eta[eJ] + gamma * (eta[eJ] - eta_prev[eJ]))
        ei = Gc[eI] * (eta[eI] + gamma * (eta[eI] - eta_prev[eI]))
        ub[:] = v + tau * ((-(ej - ei)) / de + G)

    def lay_flux(self, rows, N, E, h, u, ubs, acc, inv_n, eI, eJ, shelf, F, ob):
        """reference layers.cu:392-397"""
        if ob is not None:
            raise NotImplementedError('numpy oracle: the shelf-bed option is not restated')
        h, u, F = _rows(h, N), _rows(u, E), _rows(F, E)
        for l in range(rows):
            he = _edge_h(h[l][eI], h[l][eJ], shelf)
            F[l] = he * (u[l] - ubs) + he * (acc * inv_n)

    def lay_scale(self, rows, N, E, h0, F, cellEdgeAsc, eI, le, areaCell, dts, floor_, scale):
        """reference layers.cu:401-416"""
        h0, F, scale = _rows(h0, N), _rows(F, E), _rows(scale, N)
        ca = cellEdgeAsc.reshape(N, 6)
        me = np.arange(N)
        for l in range(rows):
            out = np.zeros(N)
            for m in range(6):
                e, ok = _slot(ca, m)
                f = F[l][e] * le[e] * dts
                own = eI[e] == me
                nxt = np.where(own, np.where(f > 0, out + f, out), np.where(~(f > 0), out - f, out))
                out = np.where(ok, nxt, out)
            avail = h0[l] - floor_
            cap = np.where(avail > 0, avail, 0.0) * areaCell
            scale[l] = np.where(out > cap, cap / out, 1.0)

    def lay_limit(self, rows, N, E, eI, eJ, scale, le, dt, F, Fm):
        """reference layers.cu:418-426"""
        scale, F = _rows(scale, N), _rows(F, E)
        Fm = None if Fm is None else _rows(Fm, E)
        for l in range(rows):
            f = F[l]
            f = f * np.where(f > 0, scale[l][eI], scale[l][eJ])
            F[l] = f
            if Fm is not None:
                Fm[l] = f * le * dt

    def lay_h(self, rows, N, E, h0, F, cellEdge, cellSign, le, areaCell, cdt, hn):
        """reference layers.cu:429-441"""
        h0, F, hn = _rows(h0, N), _rows(F, E), _rows(hn, N)
        ce, cs = cellEdge.reshape(N, 6), cellSign.reshape(N, 6).astype(np.float64)
        for l in range(rows):
            div = np.zeros(N)
            for m in range(6):
                e, ok = _slot(ce, m)
                div = np.where(ok, div + cs[:, m] * le[e] * F[l][e], div)
            hn[l] = h0[l] - (cdt * div) / areaCell

    def lay_u(self, rows, E, u0, Tp, ub_end, ub0, cdt, un):
        """reference layers.cu:443-447"""
        u0, Tp, un = _rows(u0, E), _rows(Tp, E), _rows(un, E)
        for l in range(rows):
            un[l] = u0[l] + cdt * Tp[l] + (ub_end - ub0)

    def lay_vmix(self, rows, N, E, L, h, eI, eJ, c, dt, u, diss, cd):
        """reference layers.cu:575-593: interfacial stress between neighbouring layers, top down"""
        h, u = _rows(h, N), _rows(u, E)
        d = np.zeros(E)
        for k in range(L - 1):
            ha = 0.5 * (h[k][eI] + h[k][eJ])
            hb = 0.5 * (h[k + 1][eI] + h[k + 1][eJ])
            ua, ub = u[k].copy(), u[k + 1].copy()
            mean = (ha * ua + hb * ub) / (ha + hb)
            du0 = ua - ub
            du1 = du0 * np.exp(-c * (1 / ha + 1 / hb) * dt)
            if cd > 0:
                du1 = du1 / (1 + cd * np.abs(du0) * (1 / ha + 1 / hb) * dt)
            u[k] = mean + hb / (ha + hb) * du1
            u[k + 1] = mean - ha / (ha + hb) * du1
            d = d + 0.5 * ha * hb / (ha + hb) * (du0 * du0 - du1 * du1)
        diss[:] = d

    # ---- transport (reference kernels/trisk.cu, fused.cu); rows y = tracer x Lm + layer ----

    def mass_update(self, rows, N, E, M0, Fm, cellEdgeAsc, eI, M1):
        """reference trisk.cu:48-59"""
        M0, Fm, M1 = _rows(M0, N), _rows(Fm, E), _rows(M1, N)
        ca = cellEdgeAsc.reshape(N, 6)
        me = np.arange(N)
        for l in range(rows):
            m = M0[l].copy()
            for k in range(6):
                e, ok = _slot(ca, k)
                f = Fm[l][e]
                m = np.where(ok, np.where(eI[e] == me, m - f, m + f), m)
            M1[l] = m

    def tr_td(self, rows, N, E, Lm, M0, psi, Fm, M1, cellEdgeAsc, eI, eJ, td):
        """reference fused.cu:146-160"""
        M0, psi, Fm, M1, td = _rows(M0, N), _rows(psi, N), _rows(Fm, E), _rows(M1, N), _rows(td, N)
        ca = cellEdgeAsc.reshape(N, 6)
        me = np.arange(N)
        for y in range(rows):
            l = y % Lm
            t = M0[l] * psi[y]
            for k in range(6):
                e, ok = _slot(ca, k)
                f = _upwind(Fm[l][e], psi[y], eI[e], eJ[e])
                t = np.where(ok, np.where(eI[e] == me, t - f, t + f), t)
            td[y] = t / M1[l]

    def tr_hflux(self, rows, E, Lm, src, srcf, frac, Fm, idx, wt, eI, eJ, N, beta, Hf):
        """reference fused.cu:163-167"""
        src, srcf, Fm, Hf = _rows(src, N), _rows(srcf, N), _rows(Fm, E), _rows(Hf, E)
        idx, wt = idx.reshape(E, 8), wt.reshape(E, 8)
        for y in range(rows):
            Hf[y] = frac * _hoflux(Fm[y % Lm], src[y], srcf[y], idx, wt, eI, eJ, beta)

    def tr_stage(self, rows, N, E, Lm, M0, psi, Hf, frac, Fm, cellEdgeAsc, eI, out):
        """reference fused.cu:170-186"""
        M0, psi, Hf, Fm, out = _rows(M0, N), _rows(psi, N), _rows(Hf, E), _rows(Fm, E), _rows(out, N)
        ca = cellEdgeAsc.reshape(N, 6)
        me = np.arange(N)
        for y in range(rows):
            l = y % Lm
            t = M0[l] * psi[y]
            mx = M0[l].copy()
            for k in range(6):
                e, ok = _slot(ca, k)
                f = Hf[y][e]
                m = frac * Fm[l][e]
                own = ok & (eI[e] == me)
                other = ok & ~(eI[e] == me)
                t = np.where(own, t - f, np.where(other, t + f, t))
                mx = np.where(own, mx - m, np.where(other, mx + m, mx))
            out[y] = t / mx

    def tr_aflux(self, rows, E, Lm, psi, p2, p2f, Fm, idx, wt, eI, eJ, N, beta, A):
        """reference fused.cu:189-194"""
        psi, p2, p2f, Fm, A = _rows(psi, N), _rows(p2, N), _rows(p2f, N), _rows(Fm, E), _rows(A, E)
        idx, wt = idx.reshape(E, 8), wt.reshape(E, 8)
        for y in range(rows):
            f = Fm[y % Lm]
            A[y] = _hoflux(f, p2[y], p2f[y], idx, wt, eI, eJ, beta) - _upwind(f, psi[y], eI, eJ)

    def tr_ratios(self, rows, N, E, Lm, psi, td, M1, A, nbr, cellEdgeAsc, eI, Rp, Rm):
        """reference fused.cu:197-222"""
        psi, td, M1, A, Rp, Rm = _rows(psi, N), _rows(td, N), _rows(M1, N), _rows(A, E), _rows(Rp, N), _rows(Rm, N)
        nb, ca = nbr.reshape(N, 6), cellEdgeAsc.reshape(N, 6)
        me = np.arange(N)
        for y in range(rows):
            p, t = psi[y], td[y]
            hi, lo = np.fmax(p, t), np.fmin(p, t)
            for k in range(6):
                j, ok = _slot(nb, k)
                hi = np.where(ok, np.fmax(hi, np.fmax(p[j], t[j])), hi)
                lo = np.where(ok, np.fmin(lo, np.fmin(p[j], t[j])), lo)
            m1 = M1[y % Lm]
            qmax, qmin = (hi - t) * m1, (t - lo) * m1
            Pp, Pm = np.zeros(N), np.zeros(N)
            for k in range(6):
                e, ok = _slot(ca, k)
                a = A[y][e]
                own, pos = eI[e] == me, a > 0
                Pm = np.where(ok & own & pos, Pm + a, Pm)
                Pp = np.where(ok & own & ~pos, Pp - a, Pp)
                Pp = np.where(ok & ~own & pos, Pp + a, Pp)
                Pm = np.where(ok & ~own & ~pos, Pm - a, Pm)
            Rp[y] = np.where(Pp > 0, np.fmin(1.0, qmax / Pp), 0.0)
            Rm[y] = np.where(Pm > 0, np.fmin(1.0, qmin / Pm), 0.0)

    def tr_apply(self, rows, N, E, Lm, td, M1, A, Rp, Rm, cellEdgeAsc, eI, eJ, psi_out):
        """reference fused.cu:225-241"""
        td, M1, A, Rp, Rm, out = _rows(td, N), _rows(M1, N), _rows(A, E), _rows(Rp, N), _rows(Rm, N), _rows(psi_out, N)
        ca = cellEdgeAsc.reshape(N, 6)
        me = np.arange(N)
        for y in range(rows):
            l = y % Lm
            t = td[y] * M1[l]
            for k in range(6):
                e, ok = _slot(ca, k)
                a = A[y][e]
                c = np.where(a > 0, np.fmin(Rp[y][eJ[e]], Rm[y][eI[e]]), np.fmin(Rp[y][eI[e]], Rm[y][eJ[e]]))
                t = np.where(ok, np.where(eI[e] == me, t - c * a, t + c * a), t)
            out[y] = t / M1[l]

    # ---- the deterministic sum (reference kernels/trisk.cu:61-81, driven by gpu.py:111-126) ----

    def dsum(self, x, y=None):
        """Blocks of 2048 values: thread t of a block adds values t + 256 k (k = 0..7) in order, then the 256 partial
        sums halve pairwise; passes repeat until one block remains."""
        v = np.ascontiguousarray(x, dtype=np.float64).ravel()
        if y is not None:
            v = v * np.ascontiguousarray(y, dtype=np.float64).ravel()
        while True:
            n = v.size
            blocks = max(1, (n + 2047) // 2048)
            pad = np.zeros(blocks * 2048)
            pad[:n] = v
            ok = np.zeros(blocks * 2048, dtype=bool)
            ok[:n] = True
            X, OK = pad.reshape(blocks, 8, 256), ok.reshape(blocks, 8, 256)
            s = np.zeros((blocks, 256))
            for k in range(8):
                s = np.where(OK[:, k], s + X[:, k], s)
            h = 128
            while h > 0:
                s[:, :h] = s[:, :h] + s[:, h:2 * h]
                h //= 2
            v = s[:, 0].copy()
            if blocks == 1:
                return float(v[0])
