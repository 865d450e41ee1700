"""CPU restatement (numpy) of the reference's three-phase black-oil
equations with dissolved gas, for testing only: residual values, the
convergence values, and the Newton update with the flash.

Test infrastructure: the product path never imports this module.  It is
pinned against the reference's own outputs (tests/golden/bo_assemble.npz,
made by tests/golden/make_golden.py from the reference's
ThreePhaseBlackOilModelAD).

Follows pymrst/modules/ad_blackoil/models/three_phase_black_oil_model.py:
assemble :314-381, _well :383-437, update_state :439-469, _flash :471-508,
_conv_scaling / _converged :510-539; the fluid of
pymrst/modules/ad_props/props/init_deck_adi_fluid.py:60-200 and the table
interpolations of pymrst/utils/interp_table.py:17-30 and
pymrst/modules/ad_props/utils/interp_pvt.py (`_interp1_slope`, `_get_bins`,
the 'parallel' branch of `_pvt_values`).
"""

from __future__ import annotations

import numpy as np

ETOL = np.sqrt(np.finfo(float).eps)


def _bracket(x, v):
    return np.clip(np.searchsorted(x, v, side="right") - 1, 0, x.size - 2)


def interp_w(x, f, v):
    """interp_table: f0 (1 - t) + f1 t."""
    i = _bracket(x, v)
    t = (v - x[i]) / (x[i + 1] - x[i])
    return f[i] * (1 - t) + f[i + 1] * t


def interp_s(x, f, v):
    """The slope form of the keyed tables."""
    i = _bracket(x, v)
    slope = (f[i + 1] - f[i]) / (x[i + 1] - x[i])
    return f[i] + slope * (v - x[i])


def pvt_parallel(t, f_all, p, rs, sat):
    """Keyed live-oil interpolation, 'parallel' strategy."""
    key, ptr, bp = t.key, t.branch_ptr, t.branch_p
    sat_x = bp[ptr[:-1]]
    sat_f = f_all[ptr[:-1]]
    out = np.zeros_like(p)
    sat = sat & ~(p < sat_x[0])
    if sat.any():
        out[sat] = interp_s(sat_x, sat_f, p[sat])
    u = ~sat
    if u.any():
        pu, ru = p[u], rs[u]
        lims = key.copy()
        lims[0], lims[-1] = -np.inf, np.inf
        b = np.clip(np.searchsorted(lims, ru, side="right") - 1, 0, key.size - 2)
        w = (ru - key[b]) / (key[b + 1] - key[b])
        ps = interp_s(key, sat_x, ru)
        dp = pu - ps
        fl, fr = np.zeros_like(pu), np.zeros_like(pu)
        for k in range(key.size):
            px, fx = bp[ptr[k]:ptr[k + 1]], f_all[ptr[k]:ptr[k + 1]]
            il, ir = b == k - 1, b == k
            if il.any():
                fl[il] = interp_s(px - px[0], fx, dp[il])
            if ir.any():
                fr[ir] = interp_s(px - px[0], fx, dp[ir])
        out[u] = fl * w + fr * (1.0 - w)
    return out


class Fluid:
    """Value-only fluid functions over the device table layout
    (pymrst_b200.blackoil.BlackOilTables)."""

    def __init__(self, t):
        self.t = t

    def b_w(self, p):
        t = self.t
        x = t.pvtw[2] * (p - t.pvtw[0])
        return (1.0 + x + 0.5 * x ** 2) / t.pvtw[1]

    def pv_mult(self, p):
        x = self.t.rock[1] * (p - self.t.rock[0])
        return 1.0 + x + 0.5 * x ** 2

    def b_o(self, p, rs, sat):
        return pvt_parallel(self.t, self.t.branch_b, p, rs, sat)

    def mu_o(self, p, rs, sat):
        return pvt_parallel(self.t, self.t.branch_mu, p, rs, sat)

    def b_g(self, p):
        return interp_w(self.t.gas_p, self.t.gas_b, p)

    def mu_g(self, p):
        return interp_w(self.t.gas_p, self.t.gas_mu, p)

    def rs_sat(self, p):
        return interp_w(self.t.rssat_p, self.t.rssat_rs, p)

    def kr_w(self, sw):
        return interp_w(self.t.sw, self.t.krw, sw)

    def kr_g(self, sg):
        return interp_w(self.t.sg, self.t.krg, sg)

    def kr_o(self, sw, so, sg):
        t = self.t
        swcon = np.minimum(t.swcon, sw - 1e-5)
        ww = (sw - swcon) / (sg + sw - swcon)
        return (1.0 - ww) * interp_w(t.sog, t.krog, so) + ww * interp_w(t.sow, t.krow, so)

    def pc_ow(self, sw):
        return 0.0 if self.t.pcow is None else interp_w(self.t.sw, self.t.pcow, sw)

    def pc_og(self, sg):
        return 0.0 if self.t.pcog is None else interp_w(self.t.sg, self.t.pcog, sg)


def residual(fl, N, T, gdz, pv_ref, wells, st0, st, dt):
    """Residual values in the variable-blocked order of combine_equations."""
    nc = st.pressure.size
    st1, st3 = st.status == 1, st.status == 3
    p, sw = st.pressure, st.s[:, 0]
    x = np.where(st1, st.rs, st.s[:, 2])
    rs = np.where(st1, x, fl.rs_sat(p))
    sg = np.where(st3, x, 0.0)
    so = 1.0 - sw - sg
    rhoS = fl.t.rhoS
    pw, pg = p - fl.pc_ow(sw), p + fl.pc_og(sg)
    b = [fl.b_w(pw), fl.b_o(p, rs, st3), fl.b_g(pg)]
    mu = [np.full(nc, fl.t.pvtw[3]), fl.mu_o(p, rs, st3), fl.mu_g(pg)]
    kr = [fl.kr_w(sw), fl.kr_o(sw, so, sg), fl.kr_g(sg)]
    rho = [b[0] * rhoS[0], b[1] * (rs * rhoS[2] + rhoS[1]), b[2] * rhoS[2]]
    pph = [pw, p, pg]
    a_, b_ = N[:, 0], N[:, 1]
    bv, ups = [], []
    for ph in range(3):
        rhof = 0.5 * rho[ph][a_] + 0.5 * rho[ph][b_]
        dp = (pph[ph][b_] - pph[ph][a_]) - rhof * gdz
        up = dp <= 0
        u = np.where(up, a_, b_)
        v = -(kr[ph][u] / mu[ph][u]) * T * dp
        bv.append(b[ph][u] * v)
        ups.append(u)
    bv[2] = bv[2] + rs[ups[1]] * bv[1]
    pv = pv_ref * fl.pv_mult(p)
    p0, s0, rs0 = st0.pressure, st0.s, st0.rs
    pv0 = pv_ref * fl.pv_mult(p0)
    bw0, bo0, bg0 = fl.b_w(p0), fl.b_o(p0, rs0, st0.status == 3), fl.b_g(p0)
    eq = [(1.0 / dt) * (pv * b[0] * sw - pv0 * bw0 * s0[:, 0]),
          (1.0 / dt) * (pv * b[1] * so - pv0 * bo0 * s0[:, 1]),
          (1.0 / dt) * (pv * (b[2] * sg + rs * b[1] * so) - pv0 * (bg0 * s0[:, 2] + rs0 * bo0 * s0[:, 1]))]
    for ph in range(3):
        div = np.bincount(a_, weights=bv[ph], minlength=nc) - np.bincount(b_, weights=bv[ph], minlength=nc)
        eq[ph] = eq[ph] + div
    mob = [kr[ph] / mu[ph] for ph in range(3)]
    weq, ctrl = [[], [], []], []
    for k, w in enumerate(wells):
        wc, tw, compi = w["cells"], w["WI"], w["compi"]
        q = [st.qWs[k], st.qOs[k], st.qGs[k]]
        dd = -st.bhp[k] + p[wc]
        inj = dd < 0
        prod = ~inj
        m = [x_[wc] for x_ in mob]
        bc = [x_[wc] for x_ in b]
        rc = rs[wc]
        cq_ps = None
        if prod.any():
            con = prod * tw
            cq_p = [-con * mm * dd for mm in m]
            cq_ps = [bc[0] * cq_p[0], bc[1] * cq_p[1], bc[2] * cq_p[2] + rc * (bc[1] * cq_p[1])]
            wbq = [q[ph] * float(q[ph] > 0) - cq_ps[ph].sum() for ph in range(3)]
            wbqt = wbq[0] + wbq[1] + wbq[2]
            mix = list(compi) if wbqt == 0.0 else [x_ / wbqt for x_ in wbq]
        else:
            mix = list(compi)
        if inj.any():
            mt = m[0] + m[1] + m[2]
            cqt = -(inj * tw) * (mt * dd)
            vr = mix[0] / bc[0] + mix[1] / bc[1] + (mix[2] - rc * mix[1]) / bc[2]
            cqts = cqt / vr
            cq = [cq_ps[ph] + mix[ph] * cqts for ph in range(3)] if prod.any() else [mix[ph] * cqts
                                                                                   for ph in range(3)]
        else:
            cq = cq_ps
        for ph in range(3):
            eq[ph][wc] = eq[ph][wc] - cq[ph]
            weq[ph].append(q[ph] - cq[ph].sum())
        if w["type"] == "bhp":
            ctrl.append(st.bhp[k] - w["val"])
        elif w["type"] == "rate":
            ctrl.append(q[0] + q[1] + q[2] - w["val"])
        else:
            ctrl.append(q[1] - w["val"])
    return np.concatenate(eq + [np.array(weq[0]), np.array(weq[1]), np.array(weq[2]), np.array(ctrl)])


def convergence(fl, pv_ref, wells, st, res, dt, tol_cnv=1e-3, tol_mb=1e-7, tol_well=1e-6):
    nc = st.pressure.size
    p = st.pressure
    b = [fl.b_w(p), fl.b_o(p, st.rs, st.status == 3), fl.b_g(p)]
    bavg = np.array([np.mean(1.0 / x) for x in b])
    pv = pv_ref * fl.pv_mult(p)
    cnv = np.array([bavg[i] * dt * np.abs(res[i * nc:(i + 1) * nc] / pv).max() for i in range(3)])
    mb = np.array([bavg[i] * dt * abs(res[i * nc:(i + 1) * nc].sum()) / pv.sum() for i in range(3)])
    nw = len(wells)
    q_ref = max(abs(w["val"]) for w in wells)
    wr = res[3 * nc:3 * nc + 3 * nw]
    well_ok = np.abs(wr).max() <= tol_well * q_ref
    scale = np.array([1e5 if w["type"] == "bhp" else abs(w["val"]) for w in wells])
    ctrl_ok = np.all(np.abs(res[3 * nc + 3 * nw:]) <= tol_well * scale)
    return cnv, mb, bool(cnv.max() <= tol_cnv and mb.max() <= tol_mb and well_ok and ctrl_ok)


def update_state(fl, st, upd, ds_max=0.2):
    """update_state followed by _flash; returns a new state (same type)."""
    nc, nw = st.pressure.size, st.qWs.size
    st1, st3 = st.status == 1, st.status == 3
    new = st.copy()
    dp, dsw, dx = upd[:nc], upd[nc:2 * nc], upd[2 * nc:3 * nc]
    new.pressure = st.pressure + dp
    dsg = np.where(st3, dx, 0.0)
    new.rs = np.maximum(st.rs + np.where(st1, dx, 0.0), 0.0)
    ds = np.clip(np.column_stack([dsw, -(dsg + dsw), dsg]), -ds_max, ds_max)
    new.s = st.s + ds
    o = 3 * nc
    new.qWs = st.qWs + upd[o:o + nw]
    new.qOs = st.qOs + upd[o + nw:o + 2 * nw]
    new.qGs = st.qGs + upd[o + 2 * nw:o + 3 * nw]
    new.bhp = st.bhp + upd[o + 3 * nw:o + 4 * nw]
    sw, so, sg = new.s[:, 0].copy(), new.s[:, 1].copy(), new.s[:, 2].copy()
    rs = new.rs.copy()
    rs_sat, rs_sat0 = fl.rs_sat(new.pressure), fl.rs_sat(st.pressure)
    gas = ((sg > 0) | (rs == 0)) & ~st1
    gas |= sw > 1.0 - ETOL
    gas |= (sg < 0) & (st.s[:, 2] > ETOL)
    ix2 = (rs > rs_sat * (1 + ETOL)) & st1 & (st.rs > rs_sat0 * (1 - ETOL))
    sg[ix2] = 0.0
    gas |= ix2
    ix = sg < 0
    sw[ix] /= 1.0 - sg[ix]
    so[ix] /= 1.0 - sg[ix]
    sg[ix] = 0.0
    ix = so < 0
    sw[ix] /= 1.0 - so[ix]
    sg[ix] /= 1.0 - so[ix]
    so[ix] = 0.0
    ix = sw < 0
    so[ix] /= 1.0 - sw[ix]
    sg[ix] /= 1.0 - sw[ix]
    sw[ix] = 0.0
    rs = np.where(gas, rs_sat, np.minimum(rs_sat, rs))
    new.rs = np.maximum(rs, 0.0)
    new.status = 1 + 2 * gas.astype(np.int64)
    s = np.column_stack([sw, so, sg])
    new.s = s / s.sum(axis=1, keepdims=True)
    return new
