"""Incompressible TPFA pressure solve with the reference's interface
(`incomp_tpfa`, pymrst/modules/incomp/incomp_tpfa.py:55-211).

The pressure system is assembled, solved and post-processed on the device
through the `pmb_tpfa_*` entry points (`csrc/tpfa.cu`): mobility-weighted
transmissibilities, the gravity / boundary / source right-hand side, the
well rows and the pressure pin are formed by kernels that gather per cell
row and per well; the solve is AMG-preconditioned conjugate gradients; face
pressures, face fluxes and well fluxes are reconstructed by kernels.  The host
side only evaluates the caller's fluid object (its relative permeabilities and
viscosities, which are Python callables) and converts the reference's bc / src
/ well structures into arrays.

A caller's `LinSolve(A, b)` is honoured (A is then copied to the host as a
scipy CSR matrix), and so are `MatrixOutput` and `reduce` (the Schur
complement on the well unknowns, formed on the host because it is an output
of the call, not part of the device solve).

Gravity is the `gravity` argument (a vector, default zero), used for both
the half-face potentials and the well pressure drop; the reference's newer
function reads a global setting for those, its earlier `incomp_tpfa_ad`
(which the MATLAB goldens are replayed with) the argument.
Not supported: capillary pressure, periodic `bcp`, non-neighbouring
connections (NotImplementedError).
"""

from __future__ import annotations

import copy
import hashlib
import warnings
from collections import OrderedDict
from dataclasses import dataclass, field
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


def _field(state, name):
    return state.get(name) if isinstance(state, dict) else getattr(state, name, None)


def fluid_mobilities(state, fluid):
    """Phase densities (nph) and mobilities kr / mu (nc x nph) of the fluid
    at the state, for both fluid kinds the reference's incompressible solver
    accepts (get_incomp_props.py): an incompressible fluid with
    `properties` / `saturation` / `relperm`, or an AD fluid evaluated at the
    mean pressure."""
    if hasattr(fluid, "properties"):
        mu, rho = fluid.properties(state)
        kr = np.atleast_2d(np.asarray(fluid.relperm(fluid.saturation(state)), float))
        mu = np.asarray(mu, float)
        return np.asarray(rho, float).ravel(), kr / (mu if mu.ndim == 2 else mu.ravel())
    val = lambda v: np.asarray(getattr(v, "val", v), float)
    p = _field(state, "pressure")
    p_mean = float(np.mean(p)) if p is not None else 101325.0
    rho = np.array([float(fluid.rhoWS * val(fluid.bW(p_mean))), float(fluid.rhoOS * val(fluid.bO(p_mean)))])
    mu = np.column_stack([val(fluid.muW(p)) * np.ones(np.size(p)), val(fluid.muO(p)) * np.ones(np.size(p))])
    sw = np.atleast_2d(np.asarray(_field(state, "s"), float))[:, 0]
    kro = fluid.krOW if hasattr(fluid, "krOW") else fluid.krO
    kr = np.column_stack([val(fluid.krW(sw)), val(kro(1.0 - sw))])
    return rho, kr / mu


# ---- device pressure solver (LinSolve plug) ----------------------------------------

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


# ---- the device system ----------------------------------------------------------------

def _i32(a):
    return np.ascontiguousarray(np.asarray(a).ravel(), dtype=np.int32)


def _f64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel())


def _is_injector(w) -> bool:
    """The reference's injector test for the mixture density
    (compute_incomp_well_pressure_drop.py): every sign positive, or a rate
    well with a positive target."""
    sign = getattr(w, "sign", None)
    if sign is not None and np.size(sign) > 0 and bool(np.all(np.asarray(sign) > 0)):
        return True
    return str(w.type).lower() == "rate" and float(np.sum(w.val)) > 0


class TpfaSystem:
    """One grid + well set on the device (a `pmb_tpfa` handle): the pattern
    of the pressure system and its workspaces.  `solve` assembles, solves and
    reconstructs; the arrays stay on the device until `result` copies them."""

    def __init__(self, G, wells, use_trans=False, stream=None):
        import torch
        self.torch = torch
        nc, nf = int(G.cells.num), int(G.faces.num)
        cf = np.asarray(G.cells.faces)
        cf = cf[:, 0] if cf.ndim > 1 else cf
        self.nc, self.nf, self.nhf, self.nw = nc, nf, int(cf.size), len(wells)
        self.dim = int(getattr(G, "griddim", np.asarray(G.cells.centroids).shape[1]))
        perf_ptr = np.zeros(self.nw + 1, dtype=np.int64)
        for k, w in enumerate(wells):
            perf_ptr[k + 1] = perf_ptr[k] + np.asarray(w.cells).size
        self._keep = dict(
            face_pos=_i32(G.cells.facePos), cell_faces=_i32(cf), nbr=_i32(G.faces.neighbors),
            cc=_f64(np.asarray(G.cells.centroids)[:, :self.dim]), fc=_f64(np.asarray(G.faces.centroids)[:, :self.dim]),
            perf_ptr=_i32(perf_ptr), perf_cell=_i32(np.concatenate([np.asarray(w.cells).ravel() for w in wells])
                                                    if wells else np.zeros(0)),
            well_rate=_i32([str(w.type).lower() == "rate" for w in wells]))
        k = self._keep
        d = N.TpfaDesc()
        d.nc, d.nf, d.nhf, d.dim = nc, nf, self.nhf, self.dim
        d.h_face_pos, d.h_cell_faces = N.as_p(k["face_pos"], N.C.c_int32), N.as_p(k["cell_faces"], N.C.c_int32)
        d.h_neighbors = N.as_p(k["nbr"], N.C.c_int32)
        d.h_cell_centroids, d.h_face_centroids = N.as_p(k["cc"], N.C.c_double), N.as_p(k["fc"], N.C.c_double)
        d.nw = self.nw
        d.h_perf_ptr, d.h_perf_cell = N.as_p(k["perf_ptr"], N.C.c_int32), N.as_p(k["perf_cell"], N.C.c_int32)
        d.h_well_rate = N.as_p(k["well_rate"], N.C.c_int32)
        d.use_trans = int(bool(use_trans))
        self.stream = torch.cuda.current_stream().cuda_stream if stream is None else stream
        self.handle = N.c_vp()
        N.check(N.lib().pmb_tpfa_create(N.C.byref(d), self.stream, N.C.byref(self.handle)))
        sz = (N.c_i64 * 4)()
        N.check(N.lib().pmb_tpfa_sizes(self.handle, sz))
        self.n, self.nnz, self.nperf = int(sz[0]), int(sz[1]), int(sz[2])
        self.row_ptr = np.zeros(self.n + 1, np.int32)
        self.col = np.zeros(self.nnz, np.int32)
        N.check(N.lib().pmb_tpfa_pattern(self.handle, N.as_p(self.row_ptr, N.C.c_int32),
                                         N.as_p(self.col, N.C.c_int32)))
        dev = "cuda"
        self.vals = torch.empty(self.nnz, dtype=torch.float64, device=dev)
        self.rhs = torch.empty(self.n, dtype=torch.float64, device=dev)
        self.p = torch.empty(self.n, dtype=torch.float64, device=dev)
        self.flux = torch.empty(max(nf, 1), dtype=torch.float64, device=dev)
        self.fpress = torch.empty(max(nf, 1), dtype=torch.float64, device=dev)
        self.perf_flux = torch.empty(max(self.nperf, 1), dtype=torch.float64, device=dev)
        self.perf_dp = torch.empty(max(self.nperf, 1), dtype=torch.float64, device=dev)
        self.last_iterations = 0

    def __del__(self):
        h = getattr(self, "handle", None)
        if h:
            try:
                N.lib().pmb_tpfa_destroy(h)
            except Exception:
                pass
            self.handle = None

    def assemble(self, T, mob, rho, gvec, norm_g, bc, src, wells):
        torch = self.torch
        mob = np.ascontiguousarray(np.atleast_2d(np.asarray(mob, float)))
        if mob.shape[0] != self.nc:
            mob = np.ascontiguousarray(np.broadcast_to(mob, (self.nc, mob.shape[1])))
        nph = mob.shape[1]
        if nph > 4:
            raise NotImplementedError("at most four phases")
        keep = {}
        keep["T"] = torch.as_tensor(_f64(T), device="cuda")
        keep["mob"] = torch.as_tensor(mob, device="cuda")
        keep["rho"] = _f64(np.resize(np.asarray(rho, float), nph))
        fr = N.TpfaForces()
        fr.d_T, fr.d_mob, fr.nph = N.ptr(keep["T"]), N.ptr(keep["mob"]), nph
        fr.h_rho = N.as_p(keep["rho"], N.C.c_double)
        for i in range(3):
            fr.gravity[i] = float(gvec[i])
        fr.well_gravity = float(norm_g)
        if bc is not None and np.size(bc.face):
            faces = np.asarray(bc.face, dtype=np.int64).ravel()
            types = np.resize(np.array([str(t).lower() for t in np.atleast_1d(bc.type)]), faces.size)
            code = np.where(types == "pressure", 1, np.where(types == "flux", 2, 0))
            if np.any(code == 0):
                raise ValueError("boundary condition types must be 'pressure' or 'flux'")
            keep["bcf"], keep["bct"] = _i32(faces), _i32(code)
            keep["bcv"] = _f64(np.resize(np.asarray(bc.value, float).ravel(), faces.size))
            fr.nbc = faces.size
            fr.h_bc_face, fr.h_bc_type = N.as_p(keep["bcf"], N.C.c_int32), N.as_p(keep["bct"], N.C.c_int32)
            fr.h_bc_value = N.as_p(keep["bcv"], N.C.c_double)
        if src is not None and np.size(src.cell):
            cells = np.asarray(src.cell, dtype=np.int64).ravel()
            keep["sc"], keep["sr"] = _i32(cells), _f64(np.resize(np.asarray(src.rate, float).ravel(), cells.size))
            fr.nsrc = cells.size
            fr.h_src_cell, fr.h_src_rate = N.as_p(keep["sc"], N.C.c_int32), N.as_p(keep["sr"], N.C.c_double)
        if wells:
            keep["wv"] = _f64([float(np.ravel(w.val)[0]) for w in wells])
            keep["WI"] = torch.as_tensor(np.concatenate([_f64(w.WI) for w in wells]), device="cuda")
            keep["dZ"] = torch.as_tensor(np.concatenate([_f64(np.resize(np.asarray(w.dZ, float), np.size(w.cells)))
                                                         for w in wells]), device="cuda")
            compis = [np.atleast_1d(np.asarray(w.compi, float)).ravel() for w in wells]
            nci = max(c.size for c in compis)
            ca = np.zeros((len(wells), max(nci, 1)))
            for k, c in enumerate(compis):
                ca[k, :c.size] = c
            keep["compi"] = np.ascontiguousarray(ca)
            keep["inj"] = _i32([_is_injector(w) for w in wells])
            fr.h_well_val = N.as_p(keep["wv"], N.C.c_double)
            fr.d_perf_WI, fr.d_perf_dZ = N.ptr(keep["WI"]), N.ptr(keep["dZ"])
            fr.ncompi = ca.shape[1]
            fr.h_compi = N.as_p(keep["compi"], N.C.c_double)
            fr.h_injector = N.as_p(keep["inj"], N.C.c_int32)
        N.check(N.lib().pmb_tpfa_assemble(self.handle, N.C.byref(fr), N.ptr(self.vals), N.ptr(self.rhs)))
        self._inputs = keep  # device inputs stay alive until the next assembly

    def matrix(self):
        return sp.csr_array((self.vals.cpu().numpy(), self.col, self.row_ptr), shape=(self.n, self.n))

    def solve_device(self, rtol=1e-12, maxiter=1000):
        info = (N.C.c_double * 3)()
        N.check(N.lib().pmb_tpfa_solve(self.handle, N.ptr(self.vals), N.ptr(self.rhs), N.ptr(self.p),
                                       float(rtol), int(maxiter), info))
        self.last_iterations = int(info[0])
        self.last_relres = float(info[1])

    def set_solution(self, p):
        self.p.copy_(self.torch.as_tensor(_f64(p), device="cuda"))

    def reconstruct(self):
        N.check(N.lib().pmb_tpfa_reconstruct(self.handle, N.ptr(self.p), N.ptr(self.flux), N.ptr(self.fpress),
                                             N.ptr(self.perf_flux), N.ptr(self.perf_dp)))


_SYSTEMS: "OrderedDict[tuple, TpfaSystem]" = OrderedDict()
_MAX_SYSTEMS = 4


def _system(G, wells, use_trans) -> TpfaSystem:
    """The cached device system of this grid and well set (the few most
    recently used are kept)."""
    cf = np.asarray(G.cells.faces)
    h = hashlib.sha1()
    for a in (np.asarray(G.cells.facePos), cf, np.asarray(G.faces.neighbors)):
        h.update(np.ascontiguousarray(a).tobytes())
    for w in wells:
        h.update(np.ascontiguousarray(np.asarray(w.cells, dtype=np.int64)).tobytes())
        h.update(str(w.type).lower().encode())
    key = (int(G.cells.num), int(G.faces.num), bool(use_trans), h.hexdigest(),
           hashlib.sha1(np.ascontiguousarray(np.asarray(G.cells.centroids, float)).tobytes()).hexdigest())
    s = _SYSTEMS.get(key)
    if s is None:
        s = TpfaSystem(G, wells, use_trans)
        _SYSTEMS[key] = s
        while len(_SYSTEMS) > _MAX_SYSTEMS:
            _SYSTEMS.popitem(last=False)
    else:
        _SYSTEMS.move_to_end(key)
    return s


def _driving_forces(G, gvec, bc, src, wells, MatrixOutput) -> bool:
    """Whether the solve has anything to do (checkDrivingForcesIncomp), with
    its warnings: unbalanced rates when nothing fixes the pressure level, and
    no driving force at all."""
    pressure_bc = bc is not None and any(str(t).lower() == "pressure" for t in np.atleast_1d(bc.type))
    bhp = any(str(w.type).lower() == "bhp" for w in wells)
    if not (pressure_bc or bhp):
        total = sum(float(np.sum(w.val)) for w in wells)
        total += float(np.sum(src.rate)) if src is not None else 0.0
        total += float(np.sum(bc.value)) if bc is not None else 0.0
        if abs(total) > 1e-12:
            warnings.warn("Well rates and flux bc must sum up to 0 \nwhen there are no bhp "
                          "constrained wells or pressure bc.Results may not be reliable.\n")
    grav_on = np.linalg.norm(gvec[:int(G.griddim)]) > 0
    if grav_on or bc is not None or src is not None or wells or MatrixOutput:
        return True
    warnings.warn("No external driving forces present in model--state remains unchanged.\n")
    return False


def incomp_tpfa(state: Any, G, T, fluid, bc=None, src=None, wells=None, gravity=None, *, W=None, bcp=None,
                LinSolve=None, MatrixOutput=False, Verbose=False, condition_number=False,
                pc_form="nonwetting", reduce=False, use_trans=False, rtol=1e-12, maxiter=1000):
    """Incompressible TPFA pressure; returns a new state (the input is not
    modified).  Arguments as the reference's `incomp_tpfa`; `rtol` and
    `maxiter` bound the device PCG solve (the reference solves directly)."""
    if bcp is not None:
        raise NotImplementedError("periodic boundary conditions (bcp) are not supported by this path")
    if getattr(G, "nnc", None) is not None and np.size(getattr(G.nnc, "cells", [])):
        raise NotImplementedError("non-neighbouring connections are not supported by this path")
    pc_fn = getattr(fluid, "pc", None) if hasattr(fluid, "properties") else getattr(fluid, "pcOW", None)
    if pc_fn is not None:
        pc = np.asarray(getattr(pc_fn(state), "val", pc_fn(state)) if hasattr(fluid, "properties") else
                        getattr(pc_fn(np.atleast_2d(np.asarray(state.s, float))[:, 0]), "val", 0.0), float)
        if np.any(np.abs(pc) > 0):
            raise NotImplementedError("capillary pressure is not supported by this path")
    wells = list(wells if wells is not None else (W or []))
    for w in wells:
        if str(w.type).lower() not in ("bhp", "rate"):
            raise ValueError("Unsupported well type.")
    state = copy.copy(state)
    gvec = np.zeros(3) if gravity is None else np.resize(np.asarray(gravity, float), 3)
    if not _driving_forces(G, gvec, bc, src, wells, MatrixOutput):
        return state
    nc, nw = int(G.cells.num), len(wells)
    T = np.asarray(T, float).ravel()
    cf = np.asarray(G.cells.faces)
    if use_trans:
        assert T.size == G.faces.num, (
            f"Expected one transmissibility for each interface (={G.faces.num}) but got {T.size}.")
    else:
        assert T.size == (cf.shape[0] if cf.ndim > 1 else cf.size), (
            f"Expected one one-sided transmissibility for each half face, but got {T.size}.")
    rho, mob = fluid_mobilities(state, fluid)
    syst = _system(G, wells, use_trans)
    syst.assemble(T, mob, rho, gvec, float(np.linalg.norm(gvec)), bc, src, wells)
    A = None
    if MatrixOutput or reduce or LinSolve is not None or condition_number:
        A = syst.matrix()
        rhs = syst.rhs.cpu().numpy()
    if condition_number:
        print(f"condition number of the pressure matrix: {np.linalg.cond(A.toarray()):.6e}")
    if MatrixOutput:
        state.A, state.rhs = A, rhs
    if reduce:
        # Schur complement on the well unknowns: D is diagonal
        Dinv = sp.diags_array(1.0 / A.diagonal()[nc:], shape=(nw, nw))
        C = A[nc:, :nc]
        A_r = (A[:nc, :nc] - A[:nc, nc:] @ Dinv @ C).tocsr()
        rhs_r = rhs[:nc] - A[:nc, nc:] @ (Dinv @ rhs[nc:])
        state.A, state.rhs = A_r, rhs_r
        if LinSolve is not None:
            p_r = np.asarray(LinSolve(A_r, rhs_r)).ravel()
            syst.set_solution(np.concatenate([p_r, Dinv @ (rhs[nc:] - C @ p_r)]))
        else:
            syst.solve_device(rtol, maxiter)
    elif LinSolve is not None:
        syst.set_solution(np.asarray(LinSolve(A, rhs)).ravel())
    else:
        syst.solve_device(rtol, maxiter)
    syst.reconstruct()
    p = syst.p.cpu().numpy()
    state.pressure = p[:nc]
    state.flux = syst.flux.cpu().numpy()[:G.faces.num]
    state.facePressure = syst.fpress.cpu().numpy()[:G.faces.num]
    well_sols = [copy.copy(ws) for ws in (getattr(state, "wellSol", None) or [])]
    while len(well_sols) < nw:
        well_sols.append(WellSol())
    if nw:
        pf = syst.perf_flux.cpu().numpy()
        pdp = syst.perf_dp.cpu().numpy()
        for k in range(nw):
            a, b = syst._keep["perf_ptr"][k], syst._keep["perf_ptr"][k + 1]
            well_sols[k].flux = pf[a:b].copy()
            well_sols[k].cdp = pdp[a:b].copy()
            well_sols[k].pressure = float(p[nc + k])
    if nw or well_sols:
        state.wellSol = well_sols
    return state


incompTPFA = incomp_tpfa
