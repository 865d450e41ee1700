"""Oracle: fully-implicit two-phase oil-water model (test infrastructure only).

A numpy restatement, with hand-derived derivatives in place of the reference's
sparse forward AD, of
  * TwoPhaseOilWaterModelAD.assemble
    (pymrst/modules/ad_blackoil/models/two_phase_oil_water_model.py:493-546),
  * _well_contributions_batched / _well_contributions (:286-491),
  * _compute_cdp_per_well / _segment_mix_fractions / _topology_cdp (:205-284),
  * _converged (:549-567) with cnv_mb_convergence
    (pymrst/modules/ad_core/utils/convergence.py:44-69),
  * step (:605-657) with the direct solve of _solve_increment (:569-603),
  * the legacy simulate_schedule_ad (pymrst/modules/ad_core/simulators/
    simulate_schedule_ad.py:16-75).
The fluid is init_simple_adi_fluid's (pymrst/modules/ad_props/
init_simple_adi_fluid.py:217-239); ad_max/ad_min pass the derivative of the
winning branch with ties to the variable (pymrst/utils/adi/operators.py:107-147).

The residual and Jacobian are returned in the reference's variable-blocked
layout: rows [water(nc), oil(nc), eq_w(nw), eq_o(nw), ctrl(nw)], columns
[p(nc), sW(nc), qWs(nw), qOs(nw), bhp(nw)] (utils/adi/operators.py:204-211).
"""

from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from . import trans as _trans

BARSA = 1.0e5


@dataclass
class WellSpec:
    cells: np.ndarray
    WI: np.ndarray
    dZ: np.ndarray
    compi: np.ndarray
    type: str
    val: float


@dataclass
class OWProblem:
    nc: int
    N: np.ndarray
    T: np.ndarray
    gdz: np.ndarray
    pv: np.ndarray
    fluid: object                   # mu, rhoS, n, c, p_ref, b0, sl, su
    wells: List[WellSpec]
    gravity: float = 0.0
    ds_max: float = 0.2
    dp_max_rel: float = 0.2
    tol_cnv: float = 1e-3
    tol_mb: float = 1e-7
    tol_well: float = 1e-6
    max_iterations: int = 25
    last_cdp: Optional[list] = None

    @property
    def nw(self):
        return len(self.wells)


@dataclass
class State:
    pressure: np.ndarray
    sW: np.ndarray
    qWs: np.ndarray
    qOs: np.ndarray
    bhp: np.ndarray

    def copy(self):
        return State(*(np.array(v, dtype=float, copy=True) for v in
                       (self.pressure, self.sW, self.qWs, self.qOs, self.bhp)))


def build_problem(g, rock, fluid, wells, gravity=0.0, T=None, **opts) -> OWProblem:
    """Model set-up (two_phase_oil_water_model.py:98-170): internal pairs,
    harmonic face T, pore volume, gdz = g * (z[N1] - z[N0])."""
    Nall = np.asarray(g.faces.neighbors, dtype=np.int64)
    internal = np.all(Nall >= 0, axis=1)
    if T is None:
        T = _trans.face_trans(g, _trans.compute_trans(g, rock))[internal]
    N = Nall[internal]
    pv = np.asarray(rock.poro, float) * np.asarray(g.cells.volumes, float)
    if getattr(rock, "ntg", None) is not None:
        pv = pv * rock.ntg
    if gravity:
        z = np.asarray(g.cells.centroids)[:, -1]
        gdz = gravity * (z[N[:, 1]] - z[N[:, 0]])
    else:
        gdz = np.zeros(N.shape[0])
    ws = [WellSpec(cells=np.asarray(w.cells, np.int64).ravel(),
                   WI=np.asarray(w.WI, float).ravel(),
                   dZ=np.asarray(w.dZ, float).ravel(),
                   compi=np.asarray(w.compi, float).ravel()[:2],
                   type=str(w.type).lower(), val=float(w.val)) for w in wells]
    return OWProblem(nc=int(g.cells.num), N=N, T=np.asarray(T, float), gdz=gdz,
                     pv=pv, fluid=fluid, wells=ws, gravity=float(gravity), **opts)


def initial_state(prob: OWProblem, p0: float, sw0: float) -> State:
    """two_phase_oil_water_model.py:191-203."""
    w = prob.wells
    return State(pressure=np.full(prob.nc, float(p0)), sW=np.full(prob.nc, float(sw0)),
                 qWs=np.array([x.val * x.compi[0] if x.type == "rate" else 0.0 for x in w]),
                 qOs=np.array([x.val * x.compi[1] if x.type == "rate" else 0.0 for x in w]),
                 bhp=np.array([x.val if x.type == "bhp" else p0 for x in w], dtype=float))


# -- fluid -------------------------------------------------------------------

def shrinkage(f, i, p):
    """b_i(p) and db_i/dp."""
    p = np.asarray(p, float)
    if f.c[i] == 0.0:
        return p * 0.0 + f.b0[i], np.zeros_like(p)
    b = f.b0[i] * np.exp(f.c[i] * (p - f.p_ref))
    return b, f.c[i] * b


def relperm(f, i, s):
    """kr_i(s) and dkr_i/ds."""
    s = np.asarray(s, float)
    n = float(f.n[i])
    sl, su = float(f.sl[i]), float(f.su[i])
    if sl == 0.0 and su == 1.0:
        return s ** n, n * s ** (n - 1.0)
    u = (s - sl) * (1.0 / (su - sl))
    m = np.minimum(u, 1.0)
    v = np.maximum(m, 0.0)
    passes = (u <= 1.0) & (m >= 0.0)
    d = np.where(passes, n * v ** (n - 1.0) * (1.0 / (su - sl)), 0.0)
    return v ** n, d


def props(f, p, sw):
    bw, dbw = shrinkage(f, 0, p)
    bo, dbo = shrinkage(f, 1, p)
    krw, dkrw = relperm(f, 0, sw)
    kro, dkro = relperm(f, 1, 1.0 - sw)
    imw, imo = 1.0 / f.mu[0], 1.0 / f.mu[1]
    return dict(bw=bw, dbw=dbw, bo=bo, dbo=dbo, mobw=krw * imw, dmobw=dkrw * imw,
                mobo=kro * imo, dmobo=-dkro * imo)


# -- wells -------------------------------------------------------------------

def _well_terms(prob, k, p, sw, P, qws, qos, bhp, cdp, want_jac=True):
    """Perforation rates of well k with derivatives.

    Returns dict with per-perforation cq_sw/cq_so, the derivative of each
    w.r.t. its own cell (p, sW) ['dcq_loc' (np, 2, 2)], w.r.t. the well's
    (qWs, qOs, bhp) ['dcq_w' (np, 2, 3)], and the mixture coupling
    U (np, 2, 2) = d cq / d(mix_w, mix_o) with V (np, 2, 2) = d mix / d(p, sW)
    of each perforated cell and dmix_w (2, 3) = d mix / d(qWs, qOs, bhp).
    """
    w = prob.wells[k]
    f = prob.fluid
    c = w.cells
    t = w.WI
    npf = c.size
    mobw, dmobw = P["mobw"][c], P["dmobw"][c]
    mobo, dmobo = P["mobo"][c], P["dmobo"][c]
    bw, dbw, bo, dbo = P["bw"][c], P["dbw"][c], P["bo"][c], P["dbo"][c]
    dd = -(bhp[k] + cdp) + p[c]
    inj = dd < 0
    prod = ~inj
    ce = prod.astype(float) * t
    # producer connections: cq_p = -ce * mob * dd, surface = b * cq_p
    cq_pw = -ce * mobw * dd
    cq_po = -ce * mobo * dd
    cq_psw = bw * cq_pw
    cq_pso = bo * cq_po
    # derivatives of surface producer rates: d/dp, d/dsw, d/dbhp
    d_psw = np.stack([dbw * cq_pw + bw * (-ce * mobw), bw * (-ce * dmobw * dd)], axis=1)
    d_pso = np.stack([dbo * cq_po + bo * (-ce * mobo), bo * (-ce * dmobo * dd)], axis=1)
    d_psw_bhp = bw * (ce * mobw)
    d_pso_bhp = bo * (ce * mobo)

    any_prod = bool(prod.any())
    pos_w = float(qws[k] > 0)
    pos_o = float(qos[k] > 0)
    wbq_w = qws[k] * pos_w - np.sum(cq_psw)
    wbq_o = qos[k] * pos_o - np.sum(cq_pso)
    wbqt = wbq_w + wbq_o
    dead = (wbqt == 0.0) or (not any_prod)
    mixV = np.zeros((npf, 2, 2))         # d mix_(w,o) / d(p, sw) of perf cell j
    dmix_w = np.zeros((2, 3))            # d mix_(w,o) / d(qws, qos, bhp)
    if dead:
        mix_w, mix_o = float(w.compi[0]), float(w.compi[1])
    else:
        inv_t = wbqt ** -1.0
        mix_w = wbq_w * inv_t
        mix_o = wbq_o * inv_t
        # d wbq_w / d x_j = -d cq_psw_j ; d wbqt = d wbq_w + d wbq_o
        dwq_w = -d_psw
        dwq_o = -d_pso
        dwq_t = dwq_w + dwq_o
        mixV[:, 0, :] = (dwq_w - mix_w * dwq_t) * inv_t
        mixV[:, 1, :] = (dwq_o - mix_o * dwq_t) * inv_t
        dq_w = np.array([pos_w, 0.0, -np.sum(d_psw_bhp)])
        dq_o = np.array([0.0, pos_o, -np.sum(d_pso_bhp)])
        dq_t = dq_w + dq_o
        dmix_w[0] = (dq_w - mix_w * dq_t) * inv_t
        dmix_w[1] = (dq_o - mix_o * dq_t) * inv_t

    mt = mobw + mobo
    dmt = dmobw + dmobo
    ci = inj.astype(float) * t
    cqt_i = -ci * (mt * dd)
    d_cqt = np.stack([-ci * mt, -ci * (dmt * dd)], axis=1)     # d/dp, d/dsw
    d_cqt_bhp = ci * mt
    vol_rat = mix_w / bw + mix_o / bo
    inv_vr = vol_rat ** -1.0
    cqt_is = cqt_i * inv_vr
    d_vr_p = -mix_w * dbw / bw ** 2 - mix_o * dbo / bo ** 2
    d_cqtis = np.stack([(d_cqt[:, 0] - cqt_is * d_vr_p) * inv_vr,
                        d_cqt[:, 1] * inv_vr], axis=1)
    d_cqtis_bhp = d_cqt_bhp * inv_vr
    d_cqtis_mix = np.stack([-cqt_is * (1.0 / bw) * inv_vr,
                            -cqt_is * (1.0 / bo) * inv_vr], axis=1)
    cq_sw = cq_psw + mix_w * cqt_is
    cq_so = cq_pso + mix_o * cqt_is
    out = dict(cq_sw=cq_sw, cq_so=cq_so, mix=(mix_w, mix_o), dead=dead)
    if not want_jac:
        return out
    dcq_loc = np.zeros((npf, 2, 2))
    dcq_loc[:, 0, :] = d_psw + mix_w * d_cqtis
    dcq_loc[:, 1, :] = d_pso + mix_o * d_cqtis
    U = np.zeros((npf, 2, 2))
    U[:, 0, 0] = cqt_is + mix_w * d_cqtis_mix[:, 0]
    U[:, 0, 1] = mix_w * d_cqtis_mix[:, 1]
    U[:, 1, 0] = mix_o * d_cqtis_mix[:, 0]
    U[:, 1, 1] = cqt_is + mix_o * d_cqtis_mix[:, 1]
    dcq_w = np.zeros((npf, 2, 3))
    dcq_w[:, 0, 2] = d_psw_bhp + mix_w * d_cqtis_bhp
    dcq_w[:, 1, 2] = d_pso_bhp + mix_o * d_cqtis_bhp
    dcq_w += np.einsum("pab,bc->pac", U, dmix_w)
    out.update(dcq_loc=dcq_loc, dcq_w=dcq_w, U=U, V=mixV, dmix_w=dmix_w)
    return out


def compute_cdp(prob: OWProblem, st0: State):
    """Per-perforation wellbore hydrostatic drop, once per timestep
    (two_phase_oil_water_model.py:205-284)."""
    if not prob.gravity:
        return [np.zeros(w.dZ.size) for w in prob.wells]
    f = prob.fluid
    P = props(f, st0.pressure, st0.sW)
    prev = prob.last_cdp if prob.last_cdp is not None else [np.zeros(w.dZ.size) for w in prob.wells]
    new = []
    for k, w in enumerate(prob.wells):
        r = _well_terms(prob, k, st0.pressure, st0.sW, P, st0.qWs, st0.qOs, st0.bhp,
                        prev[k], want_jac=False)
        seg_w = np.cumsum(r["cq_sw"][::-1])[::-1]
        seg_o = np.cumsum(r["cq_so"][::-1])[::-1]
        seg_t = seg_w + seg_o
        dead = seg_t == 0.0
        safe = np.where(dead, 1.0, seg_t)
        mix_w = np.where(dead, w.compi[0], seg_w / safe)
        mix_o = np.where(dead, w.compi[1], seg_o / safe)
        bw = P["bw"][w.cells]
        bo = P["bo"][w.cells]
        vol_rat = mix_w / bw + mix_o / bo
        rho_mix = (mix_w * f.rhoS[0] + mix_o * f.rhoS[1]) / vol_rat
        dz = np.diff(np.concatenate(([0.0], w.dZ)))
        new.append(np.cumsum(prob.gravity * rho_mix * dz))
    prob.last_cdp = new
    return new


# -- assembly ----------------------------------------------------------------

def assemble(prob: OWProblem, st0: State, st: State, dt: float, cdp=None, want_jac=True):
    """Residual (and Jacobian) in the reference's variable-blocked layout."""
    nc, nw = prob.nc, prob.nw
    f = prob.fluid
    p, sw = st.pressure, st.sW
    P = props(f, p, sw)
    bw0, _ = shrinkage(f, 0, st0.pressure)
    bo0, _ = shrinkage(f, 1, st0.pressure)
    pv, idt = prob.pv, 1.0 / dt
    so = 1.0 - sw
    water = idt * (pv * P["bw"] * sw - pv * bw0 * st0.sW)
    oil = idt * (pv * P["bo"] * so - pv * bo0 * (1.0 - st0.sW))

    rows, cols, vals = [], [], []

    def add(r, c_, v):
        rows.append(np.asarray(r).ravel())
        cols.append(np.asarray(c_).ravel())
        vals.append(np.asarray(v, float).ravel())

    cells = np.arange(nc)
    if want_jac:
        add(cells, cells, idt * pv * P["dbw"] * sw)
        add(cells, nc + cells, idt * pv * P["bw"])
        add(nc + cells, cells, idt * pv * P["dbo"] * so)
        add(nc + cells, nc + cells, -idt * pv * P["bo"])

    L, R = prob.N[:, 0], prob.N[:, 1]
    T, gdz = prob.T, prob.gdz
    dp = p[R] - p[L]
    for ph, (b, db, mob, dmob) in enumerate(((P["bw"], P["dbw"], P["mobw"], P["dmobw"]),
                                            (P["bo"], P["dbo"], P["mobo"], P["dmobo"]))):
        rhoS = f.rhoS[ph]
        rho = rhoS * b
        drho = rhoS * db
        pot = dp - (0.5 * rho[L] + 0.5 * rho[R]) * gdz
        flag = pot <= 0
        up = np.where(flag, L, R)
        v = -T * mob[up] * pot
        F = b[up] * v
        res = water if ph == 0 else oil
        res += np.bincount(L, F, minlength=nc) - np.bincount(R, F, minlength=nc)
        if want_jac:
            isL = flag.astype(float)
            isR = 1.0 - isL
            tm = -T * mob[up]
            dpot_L = -1.0 - gdz * 0.5 * drho[L]
            dpot_R = 1.0 - gdz * 0.5 * drho[R]
            dF_pL = isL * db[up] * v + b[up] * tm * dpot_L
            dF_pR = isR * db[up] * v + b[up] * tm * dpot_R
            dF_s = b[up] * (-T * dmob[up] * pot)
            dF_sL = isL * dF_s
            dF_sR = isR * dF_s
            r0 = ph * nc
            for rc, sg in ((L, 1.0), (R, -1.0)):
                add(r0 + rc, L, sg * dF_pL)
                add(r0 + rc, R, sg * dF_pR)
                add(r0 + rc, nc + L, sg * dF_sL)
                add(r0 + rc, nc + R, sg * dF_sR)

    if cdp is None:
        cdp = [np.zeros(w.dZ.size) for w in prob.wells]
    eq_w = np.zeros(nw)
    eq_o = np.zeros(nw)
    ctrl = np.zeros(nw)
    for k, w in enumerate(prob.wells):
        r = _well_terms(prob, k, p, sw, P, st.qWs, st.qOs, st.bhp, cdp[k], want_jac)
        np.subtract.at(water, w.cells, r["cq_sw"])
        np.subtract.at(oil, w.cells, r["cq_so"])
        eq_w[k] = st.qWs[k] - np.sum(r["cq_sw"])
        eq_o[k] = st.qOs[k] - np.sum(r["cq_so"])
        if w.type == "bhp":
            ctrl[k] = st.bhp[k] - w.val
        elif w.type == "rate":
            ctrl[k] = st.qWs[k] + st.qOs[k] - w.val
        else:
            raise ValueError(f"unsupported well control '{w.type}'")
        if not want_jac:
            continue
        c = w.cells
        wcol = np.array([2 * nc + k, 2 * nc + nw + k, 2 * nc + 2 * nw + k])
        # cell rows: water/oil(c_i) -= cq_i
        for a in range(2):
            ra = a * nc + c
            add(ra, c, -r["dcq_loc"][:, a, 0])
            add(ra, nc + c, -r["dcq_loc"][:, a, 1])
            for j in range(3):
                add(ra, np.full(c.size, wcol[j]), -r["dcq_w"][:, a, j])
        # mixture coupling: d cq_i / d x_cj = U_i V_j
        if not r["dead"]:
            UV = np.einsum("iab,jbc->ijac", r["U"], r["V"])
            ii, jj = np.meshgrid(np.arange(c.size), np.arange(c.size), indexing="ij")
            for a in range(2):
                add(a * nc + c[ii], c[jj], -UV[:, :, a, 0])
                add(a * nc + c[ii], nc + c[jj], -UV[:, :, a, 1])
        # well rows
        for a, row in ((0, 2 * nc + k), (1, 2 * nc + nw + k)):
            dloc = r["dcq_loc"][:, a, :].copy()
            if not r["dead"]:
                Usum = r["U"][:, a, :].sum(axis=0)           # sum_i U_i[a, :]
                dloc += np.einsum("b,jbc->jc", Usum, r["V"])
            add(np.full(c.size, row), c, -dloc[:, 0])
            add(np.full(c.size, row), nc + c, -dloc[:, 1])
            dw = -r["dcq_w"][:, a, :].sum(axis=0)
            dw[a] += 1.0
            add(np.full(3, row), wcol, dw)
        if w.type == "bhp":
            add([2 * nc + 2 * nw + k], [wcol[2]], [1.0])
        else:
            add([2 * nc + 2 * nw + k] * 2, wcol[:2], [1.0, 1.0])

    res = np.concatenate([water, oil, eq_w, eq_o, ctrl])
    if not want_jac:
        return res, None
    n = 2 * nc + 3 * nw
    J = sp.csr_array((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                     shape=(n, n))
    J.sum_duplicates()
    return res, J


# -- convergence and stepping ------------------------------------------------

def converged(prob: OWProblem, res, dt: float, st: State):
    nc, nw = prob.nc, prob.nw
    f = prob.fluid
    water, oil = res[:nc], res[nc:2 * nc]
    eq_w, eq_o, ctrl = res[2 * nc:2 * nc + nw], res[2 * nc + nw:2 * nc + 2 * nw], res[2 * nc + 2 * nw:]
    bw = np.mean(1.0 / shrinkage(f, 0, st.pressure)[0])
    bo = np.mean(1.0 / shrinkage(f, 1, st.pressure)[0])
    pv = prob.pv
    cnv = max(bw * dt * np.abs(water / pv).max(), bo * dt * np.abs(oil / pv).max())
    mb = max(bw * dt * abs(water.sum()) / pv.sum(), bo * dt * abs(oil.sum()) / pv.sum())
    rate = [abs(w.val) for w in prob.wells if w.type == "rate"]
    q_ref = max(max(rate), 1e-12) if rate else 1.0
    if nw:
        well_ok = (np.abs(eq_w).max() <= prob.tol_well * q_ref
                   and np.abs(eq_o).max() <= prob.tol_well * q_ref)
        ctrl_ok = bool(np.all(np.abs(ctrl) <= prob.tol_well *
                              np.array([BARSA if w.type == "bhp" else q_ref for w in prob.wells])))
    else:
        well_ok = ctrl_ok = True
    ok = cnv <= prob.tol_cnv and mb <= prob.tol_mb and well_ok and ctrl_ok
    return bool(ok), dict(cnv=cnv, mb=mb)


def apply_update(prob: OWProblem, st: State, upd):
    nc, nw = prob.nc, prob.nw
    dp = upd[:nc]
    ds = upd[nc:2 * nc]
    cap = prob.dp_max_rel * np.abs(st.pressure)
    dp = np.clip(dp, -cap, cap)
    ds = np.clip(ds, -prob.ds_max, prob.ds_max)
    st.pressure = st.pressure + dp
    st.sW = np.clip(st.sW + ds, 0.0, 1.0)
    st.qWs = st.qWs + upd[2 * nc:2 * nc + nw]
    st.qOs = st.qOs + upd[2 * nc + nw:2 * nc + 2 * nw]
    st.bhp = st.bhp + upd[2 * nc + 2 * nw:]


def step(prob: OWProblem, state: State, dt: float, linear_solve=None):
    """One backward-Euler step by Newton; returns (state, converged, its)."""
    st0 = state
    st = state.copy()
    cdp = compute_cdp(prob, st0)
    solve = linear_solve or (lambda A, b: spla.spsolve(A.tocsc(), b))
    for it in range(prob.max_iterations):
        res, J = assemble(prob, st0, st, dt, cdp)
        ok, _ = converged(prob, res, dt, st)
        if ok:
            return st, True, it
        upd = solve(J, -res)
        apply_update(prob, st, upd)
    res, _ = assemble(prob, st0, st, dt, cdp, want_jac=False)
    return st, converged(prob, res, dt, st)[0], prob.max_iterations


def simulate(prob: OWProblem, state0: State, timesteps: Sequence[float], max_cuts=6,
             linear_solve=None):
    """Report-step loop with halving cuts (simulate_schedule_ad.py:45-75)."""
    state = state0
    states, its_per_step = [], np.zeros(len(timesteps), dtype=np.int64)
    for i, dt_report in enumerate(timesteps):
        t_local, its, dt, cuts = 0.0, 0, float(dt_report), 0
        while t_local < dt_report - 1e-12 * dt_report:
            dt = min(dt, dt_report - t_local)
            cand, ok, nit = step(prob, state, dt, linear_solve)
            its += nit
            if ok:
                state = cand
                t_local += dt
                dt = min(2.0 * dt, dt_report - t_local) if cuts else dt
            else:
                cuts += 1
                if cuts > max_cuts:
                    raise AssertionError(f"step {i}: Newton failed after {max_cuts} timestep cuts")
                dt /= 2.0
        its_per_step[i] = its
        states.append(state)
    return states, its_per_step
