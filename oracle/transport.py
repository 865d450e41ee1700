"""CPU restatement (numpy / SuperLU) of the reference's two-phase
incompressible transport, for testing only: the transport source, the
harmonic gravity flux, the upwind residual and Jacobian, the explicit step
estimate, forward-Euler and backward-Euler (Newton + bisection line search +
substep control) transport.

Test infrastructure: the product path never imports this module.  Pinned by
tests/test_oracle.py against the reference's outputs and the MATLAB arrays
(tests/golden/transport_phase3.npz).

Follows pymrst/modules/incomp/transport/__init__.py: transport_source :33-93,
gravity_flux :96-111, _upwind_indices :114-149, two_phase_residual_jacobian
:152-229, _estimate_dt :232-282, explicit_transport :285-332,
implicit_transport :335-402, _linesearch :405-421.  The fluid is Corey
(init_simple_fluid, pymrst/modules/incomp/fluid/__init__.py:64-86):
kr = (s^n_w, (1-s)^n_o), mobility kr / mu.
"""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla


class Corey:
    def __init__(self, mu, rho, n):
        self.mu = np.asarray(mu, float)
        self.rho = np.asarray(rho, float)
        self.n = np.asarray(n, float)

    def relperm(self, s):
        s1 = np.atleast_2d(s)[:, 0]
        return np.column_stack([s1 ** self.n[0], (1.0 - s1) ** self.n[1]])

    def mobility(self, s):
        return self.relperm(s) / self.mu

    def d_mobility(self, s):
        s1 = np.atleast_2d(s)[:, 0]
        return np.column_stack([self.n[0] * s1 ** (self.n[0] - 1.0),
                                self.n[1] * (1.0 - s1) ** (self.n[1] - 1.0)]) / self.mu


def source(nc, fluid, cells, flux, compi):
    """Per-cell water source: inflow times the injected fractional flow,
    outflow total (the mixture of the producing cell is applied later)."""
    if len(cells) == 0:
        return np.zeros(nc)
    cells, flux = np.asarray(cells), np.asarray(flux, float).copy()
    inj = flux > 0
    if inj.any():
        m = fluid.mobility(np.asarray(compi)[inj])
        flux[inj] *= m[:, 0] / m.sum(axis=1)
    return np.bincount(cells, weights=flux, minlength=nc)


def gravity_flux(normals, cell_faces, cell_no, K, dg, nf):
    """2 / sum over half-faces of 1 / (n . K dg), zero where not finite."""
    if not np.linalg.norm(dg) > 0:
        return np.zeros(nf)
    nkg = np.einsum("hi,hij,j->h", normals[cell_faces], K[cell_no], dg)
    with np.errstate(divide="ignore"):
        out = 2.0 / np.bincount(cell_faces, weights=1.0 / nkg, minlength=nf)
    out[~np.isfinite(out)] = 0.0
    return out


def upwind(N, v, g, mob):
    a, b = N[:, 0], N[:, 1]
    iw = np.where(~(v > 0) & ~(g > 0), b, np.where(~(v < 0) & ~(g < 0), a, -1))
    io = np.where(~(v > 0) & ~(g < 0), b, np.where(~(v < 0) & ~(g > 0), a, -1))
    if (iw < 0).any() or (io < 0).any():
        mw = np.where(iw >= 0, mob[np.maximum(iw, 0), 0], np.nan)
        mo = np.where(io >= 0, mob[np.maximum(io, 0), 1], np.nan)
        iw = np.where(iw >= 0, iw, np.where(v + g * mo < 0, b, a))
        io = np.where(io >= 0, io, np.where(v - g * mw < 0, b, a))
    return iw, io


class Problem:
    """The frozen quantities of one transport call."""

    def __init__(self, fluid, N, flux, gflux, q, pv):
        self.fluid, self.N, self.v, self.g, self.q, self.pv = fluid, N, flux, gflux, q, pv

    def residual(self, s, s0, dt):
        f = self.fluid
        m = f.mobility(np.column_stack([s, 1.0 - s]))
        fc = m[:, 0] / m.sum(axis=1)
        qw = np.maximum(self.q, 0.0) + np.minimum(self.q, 0.0) * fc
        iw, io = upwind(self.N, self.v, self.g, m)
        mw, mo = m[iw, 0], m[io, 1]
        vw = mw / (mw + mo) * (self.v + self.g * mo)
        nc = s.size
        div = np.bincount(np.concatenate([self.N[:, 0], self.N[:, 1]]), weights=np.concatenate([vw, -vw]),
                          minlength=nc)
        return s - s0 + dt / self.pv * (div - qw)

    def jacobian(self, s, s0, dt):
        f = self.fluid
        sat = np.column_stack([s, 1.0 - s])
        m = f.mobility(sat)
        dm = f.d_mobility(sat) * np.array([1.0, -1.0])
        iw, io = upwind(self.N, self.v, self.g, m)
        mw, mo = m[iw, 0], m[io, 1]
        mt = mw + mo
        d1 = (self.v + self.g * mo) * (mo / mt * dm[iw, 0]) / mt
        d2 = -(self.v - self.g * mw) * (mw / mt * dm[io, 1]) / mt
        mtc = m.sum(axis=1)
        df = (m[:, 1] * dm[:, 0] - m[:, 0] * dm[:, 1]) / mtc ** 2
        nc = s.size
        a, b = self.N[:, 0], self.N[:, 1]
        pv = self.pv
        rows = np.concatenate([np.arange(nc), a, b, a, b])
        cols = np.concatenate([np.arange(nc), iw, iw, io, io])
        vals = np.concatenate([1.0 - dt / pv * (np.minimum(self.q, 0.0) * df), dt / pv[a] * d1, -(dt / pv[b] * d1),
                               dt / pv[a] * d2, -(dt / pv[b] * d2)])
        return sp.coo_array((vals, (rows, cols)), shape=(nc, nc)).tocsr()

    def estimate_dt(self, s, gflux_est):
        f = self.fluid
        sat = np.column_stack([s, 1.0 - s])
        m = f.mobility(sat)
        dm = f.d_mobility(sat) * np.array([1.0, -1.0])
        df = (m[:, 1] * dm[:, 0] - m[:, 0] * dm[:, 1]) / m.sum(axis=1) ** 2
        wave = np.max(np.max(np.abs(df[self.N]), axis=1) * np.abs(self.v), initial=0.0)
        s1 = np.linspace(0.0, 1.0, 101)
        ml = f.relperm(np.column_stack([s1, 1 - s1])) / f.mu.min()
        seg = ml[:, 0] * ml[:, 1] / ml.sum(axis=1)
        dg = np.max(np.abs(np.diff(seg)) / np.diff(s1))
        wave = max(wave, np.max(np.abs(dg * gflux_est * abs(f.rho[1] - f.rho[0])), initial=0.0))
        for sel, up in ((self.q > 0, True), (self.q < 0, False)):
            if not sel.any():
                continue
            grid = np.arange(s[sel].min(), 1.0 + 1e-12, 0.05) if up else np.arange(s[sel].max(), -1e-12, -0.05)
            if grid.size < 2:
                continue
            mg = f.mobility(np.column_stack([grid, 1 - grid]))
            fg = mg[:, 0] / mg.sum(axis=1)
            wave = max(wave, np.max(np.abs(self.q[sel] * np.max(np.diff(fg) / np.diff(grid)))))
        return np.inf if not wave > 0 else float(np.min(self.pv / wave))

    def explicit(self, s, tf, gflux_est, dt=None, max_dt=np.inf, dt_factor=0.5, satwarn=np.sqrt(np.finfo(float).eps)):
        s = s.copy()
        t = 0.0
        nsub = 0
        while t < tf:
            step = dt if dt is not None else min(max_dt, dt_factor * self.estimate_dt(s, gflux_est))
            step = min(tf - t, step)
            s = s - self.residual(s, s, step)
            t += step
            nsub += 1
            assert not np.any(s > 1 + satwarn) and not np.any(s < -satwarn)
            s = np.clip(s, 0.0, 1.0)
        return s, nsub

    def implicit(self, s, tf, nltol=1e-6, lstrials=20, maxnewt=25, tsref=12, resred=0.99):
        s = s.copy()
        mints = tf * 2.0 ** (-tsref)
        t, dt, dtprev, count = 0.0, tf, -tf, 0
        while t < tf and dt >= mints:
            dt = min(dt, tf - t)
            while True:
                s0 = s.copy()
                sn = np.minimum(1.0, s + 0.05)
                res = self.residual(sn, s0, dt)
                err = np.abs(res).max()
                it, fail = 0, False
                while err > nltol and not fail and it < maxnewt:
                    ds = -spla.spsolve(self.jacobian(sn, s0, dt).tocsc(), res)
                    target = resred * err
                    fail = True
                    base = sn
                    for k in range(lstrials):
                        sn = np.clip(base + ds * 2.0 ** (-k), 0.0, 1.0)
                        res = self.residual(sn, s0, dt)
                        if np.abs(res).max() < target:
                            fail = False
                            break
                    it += 1
                    err = np.abs(res).max()
                count -= 1
                if err > nltol:
                    dt = dtprev if (count > 0 and dtprev > 0) else dt / 2.0
                    count = 5
                else:
                    t += dt
                    dtprev = -dt
                    if t < tf and it <= 5 and count < 0:
                        dtprev = dt
                        dt = min(1.5 * dt, tf - t)
                        count = 5
                    break
            s = sn
        assert t >= tf
        return s
