"""Incompressible TPFA pressure solve with the reference's interface
(`incomp_tpfa`, pymrst/modules/incomp/incomp_tpfa.py:55-243).

The pressure system is assembled on the host exactly as the reference
describes it: mobility-weighted one-sided T, harmonic face T, gravity /
Dirichlet / Neumann / source right-hand side, well rows, and the pin when
nothing fixes the pressure level.  It is then solved on the GPU by AMG-
preconditioned conjugate gradients (`pmb_pcg_*`), which replaces the
reference's SuperLU call (:172-184, 98% of its time); face pressures, face
fluxes and well fluxes follow (:186-211).  A caller's `LinSolve` is honoured.

Gravity is the `gravity` argument (a vector, default zero), used for both
the half-face potentials and the well pressure drop; the reference's newer
function reads a global setting for those, its earlier `incomp_tpfa_ad`
(which the MATLAB goldens are replayed with) the argument.
Not supported here: capillary pressure, periodic `bcp`, non-neighbouring
connections, `reduce`.
"""

from __future__ import annotations

import copy
import hashlib
from dataclasses import dataclass, field
from types import SimpleNamespace
from typing import Any, List, Optional

import numpy as np
import scipy.sparse as sp

from . import _native as N


@dataclass
class WellSol:
    flux: np.ndarray = field(default_factory=lambda: np.zeros(0))
    pressure: float = float("nan")
    cdp: np.ndarray = field(default_factory=lambda: np.zeros(0))


@dataclass
class State:
    pressure: np.ndarray
    flux: np.ndarray
    s: np.ndarray
    wellSol: List[WellSol] = field(default_factory=list)
    facePressure: Optional[np.ndarray] = None


def init_state(g, wells=None, p0=0.0, s0=1.0) -> State:
    """Reference `init_state` / `init_res_sol` (pymrst/solvers/)."""
    nc = g.cells.num
    st = State(pressure=np.full(nc, float(p0)), flux=np.zeros(g.faces.num),
               s=np.full((nc, 1), float(s0)))
    st.wellSol = [WellSol(flux=np.zeros(np.asarray(w.cells).size), pressure=float(p0)) for w in (wells or [])]
    return st


class SingleFluid:
    """Incompressible single-phase fluid (reference `init_single_fluid`)."""

    def __init__(self, mu, rho):
        self.mu = np.array([float(mu)])
        self.rho = np.array([float(rho)])

    def properties(self, state=None):
        return self.mu, self.rho

    def saturation(self, state):
        return np.ones((np.asarray(state.pressure).size, 1))

    def relperm(self, s):
        return np.atleast_2d(np.asarray(s, float))


def init_single_fluid(mu, rho) -> SingleFluid:
    return SingleFluid(mu, rho)


def _props(state, fluid):
    mu, rho = fluid.properties(state)
    s = fluid.saturation(state)
    kr = np.atleast_2d(fluid.relperm(s))
    return np.asarray(rho, float).ravel(), kr, np.asarray(mu, float).ravel()


# ---- device pressure solver ---------------------------------------------------

_SOLVERS = {}


class GpuLinSolve:
    """`LinSolve(A, b) -> x` on the GPU (PCG + aggregation AMG) for symmetric
    positive definite systems; usable as the reference's `LinSolve=` plug.
    Handles are cached per sparsity pattern."""

    def __init__(self, rtol=1e-12, maxiter=1000, theta=0.25, coarse=200):
        self.rtol, self.maxiter, self.theta, self.coarse = rtol, maxiter, theta, coarse
        self.last_iterations = 0

    def __call__(self, A, b):
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("GpuLinSolve needs a CUDA device")
        A = sp.csr_array(A)
        A.sum_duplicates()
        A.sort_indices()
        n = A.shape[0]
        rp = np.ascontiguousarray(A.indptr, dtype=np.int32)
        ci = np.ascontiguousarray(A.indices, dtype=np.int32)
        key = (n, hashlib.sha1(rp.tobytes() + ci.tobytes()).hexdigest())
        h = _SOLVERS.get(key)
        if h is None:
            h = N.c_vp()
            stream = torch.cuda.current_stream().cuda_stream
            N.check(N.lib().pmb_pcg_create(n, N.as_p(rp, N.C.c_int32), N.as_p(ci, N.C.c_int32),
                                           float(self.theta), int(self.coarse), stream, N.C.byref(h)))
            _SOLVERS[key] = h
        vals = torch.as_tensor(np.ascontiguousarray(A.data, dtype=np.float64), device="cuda")
        N.check(N.lib().pmb_pcg_setup(h, N.ptr(vals)))
        bd = torch.as_tensor(np.ascontiguousarray(b, dtype=np.float64), device="cuda")
        xd = torch.empty_like(bd)
        info = (N.C.c_double * 3)()
        N.check(N.lib().pmb_pcg_solve(h, N.ptr(bd), N.ptr(xd), float(self.rtol), int(self.maxiter), info))
        self.last_iterations = int(info[0])
        self.last_relres = float(info[1])
        return xd.cpu().numpy()


# ---- incomp_tpfa ----------------------------------------------------------------

def _cell_faces(G):
    cf = np.asarray(G.cells.faces, dtype=np.int64)
    cf = cf[:, 0] if cf.ndim > 1 else cf
    cell_no = np.repeat(np.arange(G.cells.num, dtype=np.int64), np.diff(np.asarray(G.cells.facePos)))
    return cell_no, cf


def incomp_tpfa(state: Any, G, T, fluid, bc=None, src=None, wells=None, gravity=None, *, W=None,
                LinSolve=None, MatrixOutput=False, use_trans=False, pc_form="nonwetting", **unsupported):
    """Incompressible TPFA pressure; returns a new state (the input is not
    modified).  Arguments as the reference's `incomp_tpfa`."""
    for k, v in unsupported.items():
        if v not in (None, False):
            raise NotImplementedError(f"incomp_tpfa option {k!r} is not supported by this path")
    wells = list(wells if wells is not None else (W or []))
    state = copy.copy(state)
    g_vec = np.zeros(3) if gravity is None else np.resize(np.asarray(gravity, float), 3)
    dim = int(G.griddim)
    nbr = np.asarray(G.faces.neighbors, dtype=np.int64)
    nf = G.faces.num
    nc = G.cells.num
    nw = len(wells)
    n = nc + nw
    cell_no, cf = _cell_faces(G)
    internal = np.all(nbr >= 0, axis=1)

    rho, kr, mu = _props(state, fluid)
    mob = kr / mu
    totmob = mob.sum(axis=1)
    omega = (mob * rho).sum(axis=1) / totmob

    # mobility-weighted transmissibilities (incomp_tpfa.py:223-243)
    T = np.asarray(T, float).ravel()
    if use_trans:
        assert T.size == nf
        cnt = (nbr >= 0).sum(axis=1)
        fmob = np.bincount(cf, totmob[cell_no], minlength=nf) / cnt
        ft = T * fmob
        Th = (ft * cnt)[cf]
    else:
        assert T.size == cf.size, "one one-sided transmissibility per half-face expected"
        Th = T * totmob[cell_no]
        with np.errstate(divide="ignore"):
            ft = 1.0 / np.bincount(cf, 1.0 / Th, minlength=nf)

    # right-hand-side pieces (compute_pressure_rhs.py:17-55)
    if np.linalg.norm(g_vec[:dim]) > 0:
        cvec = np.asarray(G.faces.centroids)[cf, :dim] - np.asarray(G.cells.centroids)[cell_no, :dim]
        grav = omega[cell_no] * (cvec @ g_vec[:dim])
    else:
        grav = np.zeros(cf.size)
    ff = np.zeros(cf.size)
    gg = np.zeros(nc)
    hh = np.zeros(nf)
    dF = np.zeros(nf, dtype=bool)
    dC = np.zeros(0)
    if src is not None and np.size(src.cell):
        cells = np.asarray(src.cell, dtype=np.int64).ravel()
        gg += np.bincount(cells, np.asarray(src.rate, float).ravel(), minlength=nc)
    if bc is not None and np.size(bc.face):
        faces = np.asarray(bc.face, dtype=np.int64).ravel()
        vals = np.asarray(bc.value, float).ravel()
        types = np.resize(np.array([str(t).lower() for t in np.atleast_1d(bc.type)]), faces.size)
        isp = types == "pressure"
        pos = np.zeros(nf, dtype=np.int64)
        pos[faces[isp]] = np.arange(isp.sum())
        dF[faces[isp]] = True
        i = dF[cf]
        ff[i] = -vals[isp][pos[cf[i]]]
        dC = vals[isp][pos[dF]]
        isf = types == "flux"
        hh[faces[isf]] = -vals[isf]

    sgn = 2.0 * (nbr[cf, 0] == cell_no) - 1.0
    j = internal[cf] | dF[cf]
    fg = np.bincount(cf[j], grav[j] * sgn[j], minlength=nf)
    rhs = np.zeros(n)
    rhs[:nc] += np.bincount(cell_no, -ft[cf] * (sgn * fg[cf] + ff), minlength=nc)
    rhs[:nc] += gg
    rhs[:nc] += np.bincount(cell_no, -hh[cf], minlength=nc)

    # wells (incomp_tpfa.py:126-148)
    d = np.zeros(nc)
    Cr, Cc, Cv = [], [], []
    D = np.zeros(nw)
    norm_g = float(np.linalg.norm(g_vec))
    well_sols = [copy.copy(ws) for ws in (getattr(state, "wellSol", None) or [])]
    while len(well_sols) < nw:
        well_sols.append(WellSol())
    for k, w in enumerate(wells):
        wc = np.asarray(w.cells, dtype=np.int64).ravel()
        wi = np.asarray(w.WI, float).ravel() * totmob[wc]
        compi = np.atleast_1d(np.asarray(w.compi, float)).ravel()
        injector = (np.all(np.asarray(getattr(w, "sign", 0)) > 0) and getattr(w, "sign", 0) != 0) or \
                   (str(w.type).lower() == "rate" and float(np.sum(w.val)) > 0)
        if injector:
            m = min(rho.size, compi.size)
            rho_mix = rho[:m] @ compi[:m]
        else:
            mw = mob[wc]
            f = mw / mw.sum(axis=1, keepdims=True)
            m = min(rho.size, mob.shape[1])
            WI = np.asarray(w.WI, float).ravel()
            rho_mix = np.sum(WI * (f[:, :m] @ rho[:m])) / np.sum(WI)
        dp = norm_g * (np.asarray(w.dZ, float).ravel() * rho_mix)
        np.add.at(d, wc, wi)
        well_sols[k].cdp = dp
        kind = str(w.type).lower()
        val = float(np.ravel(w.val)[0])
        if kind == "bhp":
            ww = wi.max()
            rhs[nc + k] += ww * val
            np.add.at(rhs, wc, wi * (val + dp))
            D[k] = ww
        elif kind == "rate":
            rhs[nc + k] += val
            np.add.at(rhs, wc, wi * dp)
            Cr.extend([k] * wc.size)
            Cc.extend(wc.tolist())
            Cv.extend((-wi).tolist())
            D[k] = wi.sum()
            rhs[nc + k] -= wi @ dp
        else:
            raise ValueError("Unsupported well type.")
    C = sp.csr_array((Cv, (Cr, Cc)), shape=(nw, nc))
    d = (d + np.bincount(cell_no[dF[cf]], Th[dF[cf]], minlength=nc)
         + np.bincount(nbr[internal].ravel(order="F"), np.tile(ft[internal], 2), minlength=nc))
    I = np.concatenate([nbr[internal, 0], nbr[internal, 1], np.arange(nc)])
    J = np.concatenate([nbr[internal, 1], nbr[internal, 0], np.arange(nc)])
    V = np.concatenate([-ft[internal], -ft[internal], d])
    A = sp.csr_array((V, (I, J)), shape=(nc, nc))
    A = sp.block_array([[A, C.T], [C, sp.diags_array(D, shape=(nw, nw))]], format="csr")
    A.sum_duplicates()
    A.sort_indices()
    if not np.any(dF) and not any(str(w.type).lower() == "bhp" for w in wells):
        diag = A.diagonal()
        jpin = 0 if diag[0] > 0 else int(np.argmax(diag))
        A = A.tolil()
        A[jpin, jpin] = 2 * A[jpin, jpin]
        A = A.tocsr()
        A.sort_indices()
    if MatrixOutput:
        state.A, state.rhs = A, rhs
    solve = LinSolve if LinSolve is not None else GpuLinSolve()
    p = np.asarray(solve(A, rhs)).ravel()

    # reconstruction (incomp_tpfa.py:186-211)
    fpress = (np.bincount(cf, (p[cell_no] + grav) * Th, minlength=nf)
              / np.bincount(cf, Th, minlength=nf))
    bnd = np.any(nbr < 0, axis=1)
    fpress[bnd] = fpress[bnd] - hh[bnd] / ft[bnd]
    fpress[dF] = dC
    ext = ~internal
    sgn_b = 2.0 * (nbr[ext, 1] < 0) - 1.0
    ni = nbr[internal]
    flux = np.zeros(nf)
    flux[internal] = -(ft[internal] * (p[ni[:, 1]] - p[ni[:, 0]] - fg[internal]))
    cext = nbr[ext].max(axis=1)
    fg_all = np.bincount(cf, grav, minlength=nf)
    flux[ext] = -sgn_b * ft[ext] * (fpress[ext] - p[cext] - fg_all[ext])
    state.pressure = p[:nc]
    state.flux = flux
    state.facePressure = fpress
    for k, w in enumerate(wells):
        wc = np.asarray(w.cells, dtype=np.int64).ravel()
        well_sols[k].flux = np.asarray(w.WI, float).ravel() * totmob[wc] * (p[nc + k] + well_sols[k].cdp - p[wc])
        well_sols[k].pressure = float(p[nc + k])
    if nw or well_sols:
        state.wellSol = well_sols
    return state


incompTPFA = incomp_tpfa
