"""Device oil-water model with the reference's interface.

`GpuOilWaterModel` takes the constructor arguments of
`TwoPhaseOilWaterModelAD` (pymrst/modules/ad_blackoil/models/
two_phase_oil_water_model.py:98-175) and offers its `initial_state`,
`step(state, dt) -> (state, converged, iterations)` and `assemble` methods.
Residuals, Jacobians, the Newton loop and the CPR-GMRES solve all run in
libpymrst_b200.so on the GPU; only set-up bookkeeping and layout
conversions for export happen here.

Differences from the reference, by design:
* the linear solve inside `step` is the device CPR-GMRES (the reference's
  default is SuperLU); its tolerance is `cpr_options['rtol']`;
* a linear-solver failure inside `step` is reported as a non-converged step
  (state unchanged) so that the schedule driver cuts the timestep.
"""

from __future__ import annotations

import copy
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np
import scipy.sparse as sp

from . import _native as N
from .params import fluid_params, pore_volume


@dataclass
class OWState:
    """Same fields as the reference's OWState (two_phase_oil_water_model.py:61-74)."""
    pressure: np.ndarray
    sW: np.ndarray
    qWs: np.ndarray
    qOs: np.ndarray
    bhp: np.ndarray

    def copy(self) -> "OWState":
        return OWState(*(np.array(v, dtype=float, copy=True) for v in
                         (self.pressure, self.sW, self.qWs, self.qOs, self.bhp)))


class Equation:
    """One equation block: values and the Jacobian blocks with respect to
    each primary variable (the fields of the reference's ADI)."""

    def __init__(self, val, jac):
        self.val = np.asarray(val, float)
        self.jac = list(jac)

    def __len__(self):
        return self.val.size


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("pymrst_b200 needs a CUDA device; none is visible")
    return torch


def default_cpr_options(**overrides) -> dict:
    o = N.CPROpts()
    N.check(N.lib().pmb_cpr_default_opts(N.C.byref(o)))
    d = {name: getattr(o, name) for name, _ in N.CPROpts._fields_}
    for k, v in overrides.items():
        if k not in d:
            raise ValueError(f"unknown CPR option {k!r}")
        d[k] = v
    return d


def _opts_struct(d: dict) -> N.CPROpts:
    o = N.CPROpts()
    for name, _ in N.CPROpts._fields_:
        setattr(o, name, d[name])
    return o


def face_transmissibility_device(g, rock) -> np.ndarray:
    """Harmonic face transmissibilities computed on the GPU
    (pmb_compute_trans + pmb_face_trans); returns all faces."""
    torch = _torch()
    dev = torch.device("cuda")
    nc = g.cells.num
    fp = np.asarray(g.cells.facePos, dtype=np.int64)
    cf = np.asarray(g.cells.faces, dtype=np.int64)
    cell_no = np.repeat(np.arange(nc), np.diff(fp))
    nbr = np.asarray(g.faces.neighbors, dtype=np.int64)
    perm = np.asarray(rock.perm, dtype=float)
    if perm.ndim == 1:
        perm = perm[:, None]
    if perm.shape[1] == 1:
        K9 = np.zeros((nc, 9)); K9[:, 0] = K9[:, 4] = K9[:, 8] = perm[:, 0]
    elif perm.shape[1] == 3:
        K9 = np.zeros((nc, 9)); K9[:, 0], K9[:, 4], K9[:, 8] = perm[:, 0], perm[:, 1], perm[:, 2]
    elif perm.shape[1] == 6:
        k = perm
        K9 = np.column_stack([k[:, 0], k[:, 1], k[:, 2], k[:, 1], k[:, 3], k[:, 4], k[:, 2], k[:, 4], k[:, 5]])
    else:
        raise ValueError("permeability must have 1, 3 or 6 columns")
    t = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a, dtype=dt), device=dev)
    d_cell_no = t(cell_no, np.int32)
    d_hf = t(cf, np.int32)
    d_first = t(nbr[:, 0], np.int32)
    d_cc = t(g.cells.centroids, np.float64)
    d_fc = t(g.faces.centroids, np.float64)
    d_fn = t(g.faces.normals, np.float64)
    d_K = t(K9, np.float64)
    ntg = getattr(rock, "ntg", None)
    tags = getattr(g.cells, "tags", None)
    d_ntg = t(ntg, np.float64) if ntg is not None and tags is not None else None
    d_tag = t(tags, np.int32) if ntg is not None and tags is not None else None
    th = torch.empty(cf.size, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    N.check(N.lib().pmb_compute_trans(cf.size, N.ptr(d_cell_no), N.ptr(d_hf), N.ptr(d_first), N.ptr(d_cc),
                                      N.ptr(d_fc), N.ptr(d_fn), N.ptr(d_K), N.ptr(d_ntg), N.ptr(d_tag), 1,
                                      N.ptr(th), stream))
    order = np.argsort(cf, kind="stable")
    ptr = np.zeros(g.faces.num + 1, dtype=np.int64)
    np.add.at(ptr, cf + 1, 1)
    ptr = np.cumsum(ptr)
    d_ptr = t(ptr, np.int32)
    d_idx = t(order, np.int32)
    tf = torch.empty(g.faces.num, dtype=torch.float64, device=dev)
    N.check(N.lib().pmb_face_trans(g.faces.num, N.ptr(d_ptr), N.ptr(d_idx), N.ptr(th), N.ptr(tf), stream))
    torch.cuda.current_stream().synchronize()
    return tf.cpu().numpy(), th.cpu().numpy()


class GpuOilWaterModel:
    """Fully-implicit oil-water model on the GPU (reference
    TwoPhaseOilWaterModelAD)."""

    n_phases = 2
    disgas = False
    vapoil = False

    def __init__(self, g, rock, fluid, wells: Sequence, gravity: float = 0.0, ds_max: float = 0.2,
                 dp_max_rel: float = 0.2, tol_cnv: float = 1e-3, tol_mb: float = 1e-7,
                 tol_well: float = 1e-6, max_iterations: int = 25, linear_solver=None,
                 cpr_options: Optional[dict] = None, T: Optional[np.ndarray] = None):
        torch = _torch()
        self.g = g
        self.rock = rock
        self.fluid = fluid
        self.raw_fluid = fluid
        self.wells = list(wells)
        self.gravity = float(gravity)
        self.ds_max, self.dp_max_rel = float(ds_max), float(dp_max_rel)
        self.tol_cnv, self.tol_mb, self.tol_well = float(tol_cnv), float(tol_mb), float(tol_well)
        self.max_iterations = int(max_iterations)
        self.linear_solver = linear_solver
        for w in self.wells:
            assert np.asarray(w.compi).size >= 2, "wells need 2-phase compi"
        prm = fluid_params(fluid)
        self.fluid_params = prm
        Nall = np.asarray(g.faces.neighbors, dtype=np.int64)
        internal = np.all(Nall >= 0, axis=1)
        self._internal = internal
        self.N = Nall[internal]
        if T is None:
            tf, _ = face_transmissibility_device(g, rock)
            T = tf[internal]
        self.T = np.asarray(T, dtype=float)
        self.pv = pore_volume(g, rock)
        if self.gravity:
            z = np.asarray(g.cells.centroids)[:, -1]
            self.gdz = self.gravity * (z[self.N[:, 1]] - z[self.N[:, 0]])
        else:
            self.gdz = np.zeros(self.N.shape[0])
        self.nc = int(g.cells.num)
        self.nw = len(self.wells)
        self._build_handle(prm)
        self.cpr_options = default_cpr_options(**(cpr_options or {}))
        self._cpr = None
        self._stream = torch.cuda.current_stream()

    # -- ad_core attribute contract --------------------------------------
    @property
    def G(self):
        return self.g

    @G.setter
    def G(self, grid):
        self.g = grid

    # -- set-up -----------------------------------------------------------
    def _build_handle(self, prm):
        torch = _torch()
        nw = self.nw
        perf_cells = [np.asarray(w.cells, np.int64).ravel() for w in self.wells]
        perf_ptr = np.zeros(nw + 1, dtype=np.int32)
        perf_ptr[1:] = np.cumsum([c.size for c in perf_cells]) if nw else []
        cat = lambda xs, dt: (np.ascontiguousarray(np.concatenate(xs), dtype=dt) if xs else np.zeros(1, dt))
        self._h = dict(
            N=np.ascontiguousarray(self.N, dtype=np.int32),
            T=np.ascontiguousarray(self.T, dtype=np.float64),
            gdz=np.ascontiguousarray(self.gdz, dtype=np.float64),
            pv=np.ascontiguousarray(self.pv, dtype=np.float64),
            perf_ptr=perf_ptr,
            perf_cell=cat(perf_cells, np.int32),
            perf_WI=cat([np.asarray(w.WI, float).ravel() for w in self.wells], np.float64),
            perf_dZ=cat([np.asarray(w.dZ, float).ravel() for w in self.wells], np.float64),
            compi=np.ascontiguousarray([np.asarray(w.compi, float).ravel()[:2] for w in self.wells]
                                       if nw else np.zeros((1, 2)), dtype=np.float64),
            well_type=np.array([self._well_type(w) for w in self.wells] or [0], dtype=np.int32),
            well_val=np.array([float(np.ravel(w.val)[0]) for w in self.wells] or [0.0], dtype=np.float64),
        )
        # vertical interfaces (|n_z| dominant) chain cells into the lines the
        # CPR second stage solves along
        normals = getattr(getattr(self.g, "faces", None), "normals", None)
        if getattr(self, "_line_face", None) is not None:
            self._h["line_face"] = np.ascontiguousarray(self._line_face, dtype=np.int32)
        elif normals is not None and np.asarray(normals).shape[1] == 3 and self.N.shape[0]:
            nrm = np.abs(np.asarray(normals)[self._internal])
            line = (nrm[:, 2] > nrm[:, 0]) & (nrm[:, 2] > nrm[:, 1])
            self._h["line_face"] = np.ascontiguousarray(line, dtype=np.int32)
        h = self._h
        d = N.OWDesc()
        d.nc, d.nf, d.nw = self.nc, self.N.shape[0], nw
        d.h_N = N.as_p(h["N"], N.C.c_int32)
        d.h_T = N.as_p(h["T"], N.C.c_double)
        d.h_gdz = N.as_p(h["gdz"], N.C.c_double)
        d.h_pv = N.as_p(h["pv"], N.C.c_double)
        for name, vals in (("mu", prm.mu), ("rhoS", prm.rhoS), ("n_exp", prm.n), ("c", prm.c),
                           ("b0", prm.b0), ("sl", prm.sl), ("su", prm.su)):
            arr = getattr(d, name)
            arr[0], arr[1] = float(vals[0]), float(vals[1])
        d.p_ref = float(prm.p_ref)
        d.h_perf_ptr = N.as_p(h["perf_ptr"], N.C.c_int32)
        d.h_perf_cell = N.as_p(h["perf_cell"], N.C.c_int32)
        d.h_perf_WI = N.as_p(h["perf_WI"], N.C.c_double)
        d.h_perf_dZ = N.as_p(h["perf_dZ"], N.C.c_double)
        d.h_compi = N.as_p(h["compi"], N.C.c_double)
        d.h_well_type = N.as_p(h["well_type"], N.C.c_int32)
        d.h_well_val = N.as_p(h["well_val"], N.C.c_double)
        d.gravity = self.gravity
        d.tol_cnv, d.tol_mb, d.tol_well = self.tol_cnv, self.tol_mb, self.tol_well
        d.ds_max, d.dp_max_rel = self.ds_max, self.dp_max_rel
        if "line_face" in h:
            d.h_line_face = N.as_p(h["line_face"], N.C.c_int32)
        hd = N.c_vp()
        stream = torch.cuda.current_stream().cuda_stream
        N.check(N.lib().pmb_ow_create(N.C.byref(d), stream, N.C.byref(hd)))
        self._handle = hd
        sizes = (N.C.c_int64 * 8)()
        N.check(N.lib().pmb_ow_sizes(hd, sizes))
        self.sizes = dict(zip(["nc", "nf", "nw", "nperf", "nnzb", "nvec", "well_len", "ncolors"],
                              [int(v) for v in sizes]))
        self.perf_cells = h["perf_cell"][:self.sizes["nperf"]]
        self.perf_ptr = perf_ptr

    @staticmethod
    def _well_type(w) -> int:
        t = str(w.type).lower()
        if t == "bhp":
            return 0
        if t == "rate":
            return 1
        raise ValueError(f"unsupported well control '{w.type}'")

    def __del__(self):
        try:
            if getattr(self, "_cpr", None) is not None:
                N.lib().pmb_cpr_destroy(self._cpr)
                self._cpr = None
            if getattr(self, "_handle", None) is not None:
                N.lib().pmb_ow_destroy(self._handle)
                self._handle = None
        except Exception:
            pass

    def solver_handle(self):
        if self._cpr is None:
            h = N.c_vp()
            o = _opts_struct(self.cpr_options)
            N.check(N.lib().pmb_cpr_create(self._handle, N.C.byref(o), N.C.byref(h)))
            self._cpr = h
        return self._cpr

    # -- state -------------------------------------------------------------
    def initial_state(self, p0: float, sw0: float) -> OWState:
        """two_phase_oil_water_model.py:191-203."""
        bhp = np.array([float(w.val) if str(w.type).lower() == "bhp" else p0 for w in self.wells], dtype=float)
        qws = np.array([float(w.val) * float(w.compi[0]) if str(w.type).lower() == "rate" else 0.0
                        for w in self.wells], dtype=float)
        qos = np.array([float(w.val) * float(w.compi[1]) if str(w.type).lower() == "rate" else 0.0
                        for w in self.wells], dtype=float)
        return OWState(pressure=np.full(self.nc, float(p0)), sW=np.full(self.nc, float(sw0)),
                       qWs=qws, qOs=qos, bhp=bhp)

    def pack(self, st: OWState) -> np.ndarray:
        """Host state -> device (cell-major) layout."""
        x = np.empty(2 * self.nc + 3 * self.nw)
        x[0:2 * self.nc:2] = st.pressure
        x[1:2 * self.nc:2] = st.sW
        w = x[2 * self.nc:].reshape(self.nw, 3) if self.nw else np.zeros((0, 3))
        if self.nw:
            w[:, 0], w[:, 1], w[:, 2] = st.qWs, st.qOs, st.bhp
        return x

    def unpack(self, x: np.ndarray) -> OWState:
        w = x[2 * self.nc:].reshape(self.nw, 3)
        return OWState(pressure=x[0:2 * self.nc:2].copy(), sW=x[1:2 * self.nc:2].copy(),
                       qWs=w[:, 0].copy(), qOs=w[:, 1].copy(), bhp=w[:, 2].copy())

    def to_device(self, st: OWState):
        torch = _torch()
        return torch.as_tensor(self.pack(st), device="cuda")

    def from_device(self, x) -> OWState:
        return self.unpack(x.detach().cpu().numpy())

    # -- stepping ----------------------------------------------------------
    def step_device(self, x, dt: float):
        """Newton step on a device state tensor, in place.  Returns
        (converged, iterations, stats8)."""
        stats = (N.C.c_double * 8)()
        rc = N.lib().pmb_ow_step(self._handle, self.solver_handle(), N.ptr(x), float(dt),
                                 self.max_iterations, stats)
        if rc == 5:  # linear solver failure: the state was restored; the step failed
            self.last_failure = N.lib().pmb_last_error().decode()
            return False, int(stats[0]), list(stats)
        N.check(rc)
        return bool(stats[1]), int(stats[0]), list(stats)

    def _staging(self):
        """Pinned host buffer and device state buffer reused by `step`."""
        if getattr(self, "_pin", None) is None:
            torch = _torch()
            n = self.sizes["nvec"]
            self._pin = torch.empty(n, dtype=torch.float64, pin_memory=True)
            self._xdev = torch.empty(n, dtype=torch.float64, device="cuda")
        return self._pin, self._xdev

    def step(self, state: OWState, dt: float):
        """One backward-Euler step (two_phase_oil_water_model.py:605-657):
        the state goes to the device through a pinned buffer, the Newton loop
        runs there, and the new state comes back the same way."""
        pin, x = self._staging()
        pin.numpy()[:] = self.pack(state)
        x.copy_(pin, non_blocking=True)
        ok, its, stats = self.step_device(x, dt)
        pin.copy_(x, non_blocking=True)
        _torch().cuda.current_stream().synchronize()
        self.last_stats = stats
        return self.unpack(pin.numpy().copy()), ok, its

    def set_controls(self, u) -> None:
        """New well targets, one per well (the reference's `_set_controls`,
        optimization/adjoint.py:63-65): `w.val` on the well objects and the
        device model's targets."""
        u = np.ascontiguousarray(np.asarray(u, dtype=np.float64).ravel())
        if u.size != self.nw:
            raise ValueError(f"{u.size} controls for {self.nw} wells")
        for w, v in zip(self.wells, u):
            w.val = float(v)
        if self.nw:
            N.check(N.lib().pmb_ow_set_controls(self._handle, N.as_p(u, N.C.c_double)))

    def reset_cdp(self) -> None:
        """Forget the previous timestep's well pressure drops (a fresh run)."""
        N.check(N.lib().pmb_ow_reset_cdp(self._handle))

    # -- assembly export (parity / protocol) ---------------------------------
    def compute_cdp(self, st0: OWState):
        torch = _torch()
        x0 = self.to_device(st0)
        cdp = torch.zeros(max(self.sizes["nperf"], 1), dtype=torch.float64, device="cuda")
        N.check(N.lib().pmb_ow_compute_cdp(self._handle, N.ptr(x0), N.ptr(cdp)))
        out = cdp.cpu().numpy()[:self.sizes["nperf"]]
        return [out[self.perf_ptr[k]:self.perf_ptr[k + 1]].copy() for k in range(self.nw)]

    def assemble_device(self, x, x0, dt, cdp_dev, want_jac=True):
        torch = _torch()
        res = torch.empty(self.sizes["nvec"], dtype=torch.float64, device="cuda")
        jac = torch.empty(4 * self.sizes["nnzb"], dtype=torch.float64, device="cuda")
        well = torch.zeros(max(self.sizes["well_len"], 1), dtype=torch.float64, device="cuda")
        N.check(N.lib().pmb_ow_assemble(self._handle, N.ptr(x), N.ptr(x0), float(dt), N.ptr(cdp_dev),
                                        N.ptr(res), N.ptr(jac), N.ptr(well), int(want_jac)))
        return res, jac, well

    def residual_and_jacobian(self, st0: OWState, st: OWState, dt: float, cdp=None):
        """Residual vector and Jacobian (scipy CSR) in the reference's
        variable-blocked layout (combine_equations of assemble's five
        equations)."""
        torch = _torch()
        x = self.to_device(st)
        x0 = self.to_device(st0)
        if cdp is None:
            cdp = [np.zeros(np.asarray(w.cells).size) for w in self.wells]
        cdp_flat = np.concatenate([np.asarray(c, float).ravel() for c in cdp]) if self.nw else np.zeros(1)
        cdp_dev = torch.as_tensor(np.ascontiguousarray(cdp_flat if cdp_flat.size else np.zeros(1)), device="cuda")
        res, jac, well = self.assemble_device(x, x0, dt, cdp_dev, True)
        return self.export_residual(res.cpu().numpy()), self.export_jacobian(jac.cpu().numpy(), well.cpu().numpy())

    def pattern(self):
        rp = np.zeros(self.nc + 1, dtype=np.int32)
        col = np.zeros(self.sizes["nnzb"], dtype=np.int32)
        N.check(N.lib().pmb_ow_pattern(self._handle, N.as_p(rp, N.C.c_int32), N.as_p(col, N.C.c_int32)))
        return rp, col

    def export_residual(self, r: np.ndarray) -> np.ndarray:
        nc, nw = self.nc, self.nw
        w = r[2 * nc:].reshape(nw, 3)
        return np.concatenate([r[0:2 * nc:2], r[1:2 * nc:2], w[:, 0], w[:, 1], w[:, 2]])

    def export_jacobian(self, vals: np.ndarray, well: np.ndarray) -> sp.csr_array:
        nc, nw = self.nc, self.nw
        nperf = self.sizes["nperf"]
        rp, col = self.pattern()
        rows_c = np.repeat(np.arange(nc), np.diff(rp))
        V = vals.reshape(-1, 2, 2)
        R, Cc, D = [], [], []
        for a in range(2):
            for b in range(2):
                R.append(a * nc + rows_c); Cc.append(b * nc + col); D.append(V[:, a, b])
        if nw:
            lay = self._well_layout(nperf, nw)
            B = well[lay["B"]:lay["C"]].reshape(nperf, 2, 3)
            Cp = well[lay["C"]:lay["U"]].reshape(nperf, 2, 2)
            U = well[lay["U"]:lay["V"]].reshape(nperf, 2, 2)
            Vp = well[lay["V"]:lay["D"]].reshape(nperf, 2, 2)
            Dw = well[lay["D"]:lay["M"]].reshape(nw, 3, 3)
            M = well[lay["M"]:lay["M"] + nw]
            perf_well = np.repeat(np.arange(nw), np.diff(self.perf_ptr))
            pc = self.perf_cells
            for a in range(2):
                for j in range(3):
                    R.append(a * nc + pc); Cc.append(2 * nc + j * nw + perf_well); D.append(B[:, a, j])
                for b in range(2):
                    R.append(2 * nc + a * nw + perf_well); Cc.append(b * nc + pc); D.append(Cp[:, a, b])
            for k in range(nw):
                for r in range(3):
                    for j in range(3):
                        R.append([2 * nc + r * nw + k]); Cc.append([2 * nc + j * nw + k]); D.append([Dw[k, r, j]])
                if M[k] != 0.0:
                    sl = slice(self.perf_ptr[k], self.perf_ptr[k + 1])
                    UV = np.einsum("iab,jbc->ijac", U[sl], Vp[sl])
                    ci, cj = np.meshgrid(pc[sl], pc[sl], indexing="ij")
                    for a in range(2):
                        for b in range(2):
                            R.append((a * nc + ci).ravel()); Cc.append((b * nc + cj).ravel())
                            D.append(UV[:, :, a, b].ravel())
        n = 2 * nc + 3 * nw
        J = sp.csr_array((np.concatenate(D), (np.concatenate(R), np.concatenate(Cc))), shape=(n, n))
        J.sum_duplicates()
        return J

    @staticmethod
    def _well_layout(nperf, nw):
        B = 0
        C = B + 6 * nperf
        U = C + 4 * nperf
        V = U + 4 * nperf
        D = V + 4 * nperf
        M = D + 9 * nw
        return dict(B=B, C=C, U=U, V=V, D=D, M=M)

    def convergence(self, res_dev, x_dev, dt):
        out = (N.C.c_double * 8)()
        N.check(N.lib().pmb_ow_convergence(self._handle, N.ptr(res_dev), N.ptr(x_dev), float(dt), out))
        return list(out)

    # -- the legacy nonlinear-solver protocol ------------------------------
    # What the reference's NonLinearSolver.solve_ministep calls
    # (ad_core/simulators/nonlinear_solver.py:239-381) on a model, with the
    # meaning GenericBlackOilModelAD gives them (generic_black_oil_model.py:
    # 472-684): get_equations -> the equation list, get_convergence -> (ok,
    # residual report), update_state -> the limited Newton update.  The
    # residual, Jacobian, convergence values and update are computed on the
    # device; the equation list is a host copy, because the solver combines
    # it on the host (combine_equations) before its linear solve.

    def _protocol_start(self, state0, dt):
        """Device start state and well pressure drops of the timestep that
        `state0` and `dt` open (computed once per timestep, as `step` does)."""
        torch = _torch()
        p0 = np.asarray(state0.pressure, float)
        key = (id(state0), float(dt), p0[:8].tobytes(), np.asarray(state0.sW, float)[:8].tobytes())
        if getattr(self, "_proto_key", None) != key:
            self._proto_x0 = self.to_device(state0)
            self._proto_cdp = torch.zeros(max(self.sizes["nperf"], 1), dtype=torch.float64, device="cuda")
            N.check(N.lib().pmb_ow_compute_cdp(self._handle, N.ptr(self._proto_x0), N.ptr(self._proto_cdp)))
            self._proto_key = key
        return self._proto_x0, self._proto_cdp

    def get_equations(self, state0: OWState, state: OWState, dt: float):
        """[water, oil, eq_w, eq_o, ctrl] at `state` for the step from
        `state0` over `dt`, each with its values and its Jacobian blocks with
        respect to [p, sW, qWs, qOs, bhp], as `assemble` returns them
        (two_phase_oil_water_model.py:493-546).  The objects are the
        reference's ADI type where that package is importable (so that its
        combine_equations accepts them), else `Equation`."""
        x0, cdp = self._protocol_start(state0, dt)
        x = self.to_device(state)
        res, jac, well = self.assemble_device(x, x0, dt, cdp, True)
        self._proto_eval = (x, res, float(dt))
        r = self.export_residual(res.cpu().numpy())
        J = self.export_jacobian(jac.cpu().numpy(), well.cpu().numpy()).tocsr()
        nc, nw = self.nc, self.nw
        cuts = [0, nc, 2 * nc, 2 * nc + nw, 2 * nc + 2 * nw, 2 * nc + 3 * nw]
        try:
            from pymrst.utils.adi import ADI as make
        except ImportError:
            make = Equation
        eqs = []
        for i in range(5):
            rows = J[cuts[i]:cuts[i + 1]]
            eqs.append(make(r[cuts[i]:cuts[i + 1]].copy(),
                            [sp.csr_matrix(rows[:, cuts[j]:cuts[j + 1]]) for j in range(5)]))
        return eqs

    def get_convergence(self, eqs, dt: float):
        """(converged, {"CNV", "MB", "well", "control"}) of the equations of
        the last get_equations: the device CNV / MB / well test of `step`
        (_converged, two_phase_oil_water_model.py:549-567); "control" is the
        largest control residual scaled by 1 bar (bhp) or the reference rate."""
        if getattr(self, "_proto_eval", None) is None:
            raise RuntimeError("get_convergence needs the equations of a preceding get_equations")
        x, res, _ = self._proto_eval
        out = self.convergence(res, x, dt)
        ctrl = np.abs(np.asarray(getattr(eqs[4], "val", eqs[4]), float))
        rates = [abs(float(np.ravel(w.val)[0])) for w in self.wells if str(w.type).lower() == "rate"]
        q_ref = max(max(rates), 1e-12) if rates else 1.0
        scale = np.array([1e5 if str(w.type).lower() == "bhp" else q_ref for w in self.wells])
        control = float(np.max(ctrl / scale)) if self.nw else 0.0
        return bool(out[5]), {"CNV": float(out[0]), "MB": float(out[1]), "well": float(max(out[2], out[3])),
                              "control": control}

    def update_state(self, state: OWState, increment) -> OWState:
        """The Newton update of `step` (two_phase_oil_water_model.py:641-651)
        on the device: dp limited to dp_max_rel |p|, dsW to ds_max, sW kept in
        [0, 1]; `increment` in the variable-blocked layout [p, sW, qWs, qOs,
        bhp]."""
        torch = _torch()
        dx = np.asarray(increment, float).ravel()
        nc, nw = self.nc, self.nw
        if dx.size != 2 * nc + 3 * nw:
            raise ValueError(f"increment of length {dx.size}, expected {2 * nc + 3 * nw}")
        d = self.pack(OWState(pressure=dx[:nc], sW=dx[nc:2 * nc], qWs=dx[2 * nc:2 * nc + nw],
                              qOs=dx[2 * nc + nw:2 * nc + 2 * nw], bhp=dx[2 * nc + 2 * nw:]))
        x = self.to_device(state)
        dd = torch.as_tensor(d, device="cuda")  # held until the update kernel has run
        N.check(N.lib().pmb_ow_update(self._handle, N.ptr(x), N.ptr(dd), 1.0))
        return self.from_device(x)

    def cpr_levels(self):
        sizes = (N.C.c_int64 * 64)()
        nl = N.C.c_int32()
        N.check(N.lib().pmb_cpr_levels(self.solver_handle(), 64, sizes, N.C.byref(nl)))
        return [int(sizes[i]) for i in range(min(nl.value, 64))]


TwoPhaseOilWaterModelAD = GpuOilWaterModel
