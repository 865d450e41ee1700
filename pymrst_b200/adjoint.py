"""Adjoint gradients of well-control objectives on the GPU model.

The interface of pymrst/modules/optimization/adjoint.py:
`compute_gradient_adjoint` (:163-225), `simulate_forward` (:136-147),
`evaluate_objective` (:150-160) and `npv_objective` (:228-265), with
`GpuOilWaterModel` in place of `TwoPhaseOilWaterModelAD`.  The sweep runs on
the device:

* forward: the device Newton step per timestep, the controls set before each
  step as the reference's `_set_controls` does; the state is kept only at
  checkpoints (every k-th step, with the well pressure-drop history the next
  step starts from), so device memory does not grow with the schedule;
* backward, segment by segment from the last: the segment's states are
  recomputed from its checkpoint (the same steps again), then for each step
  n, last first,
  - the Jacobian dR_n/dx_n at the states, assembled with the well pressure
    drops 0 as the reference's `_jac_wrt_current` does (:74-80), is turned
    into J_n^T in CSR form on the device (`pmb_ow_csr_values` over term lists
    built once per model),
  - the right-hand side -dJ_n/dx_n - (dR_{n+1}/dx_n)^T lambda_{n+1}
    (`pmb_ow_prev_jacobian_tmul`, the accumulation terms of
    `_jac_wrt_previous`, :83-105),
  - J_n^T lambda_n = rhs by the transposed device CPR (`pmb_csr_cpr_*`,
    transposed transfer operators; rows scaled to unit maximum), where the
    reference calls spsolve (:209),
  - dJ/du_n = -lambda_n on the control rows (dR/du = -1 there, :108-123),
  - with `perm_gradient`, lambda_n^T dR_n/d(log k) accumulated per cell
    (`pmb_ow_perm_contract`); the reference has no such gradient.

Only the objective runs on the host: it is the caller's callable
`obj(model, state, u, dt, n) -> (J_n, dJ_n/dx_n)`, given each step's state as
an `OWState`, its derivative in the variable-blocked layout [p, sW, qWs,
qOs, bhp].  `npv_objective` builds the reference's NPV.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional, Sequence

import numpy as np

from . import _native as N
from .linear_solvers import GpuCPRSolver
from .ow_model import OWState, _torch


@dataclass
class AdjointResult:
    value: float
    gradient: np.ndarray                      # nsteps x nw: dJ/du
    states: List[OWState]                     # state0 and the end state of every step
    initial_state_gradient: Optional[np.ndarray]  # dJ/dx_0, variable-blocked layout
    perm_gradient: Optional[np.ndarray] = None    # dJ/d(log k) per cell
    stats: Dict[str, float] = field(default_factory=dict)


def npv_objective(oil_price: float = 60.0, water_cost: float = 6.0, water_inj_cost: float = 6.0,
                  discount_rate: float = 0.0, dts: Optional[Sequence[float]] = None,
                  time_unit: float = 365.0 * 86400.0) -> Callable:
    """Net present value with the reference's signs: a producer (qWs + qOs
    < 0) earns -oil_price * qOs and pays water_cost * qWs, an injector pays
    -water_inj_cost * qWs, all times dt and the discount factor
    (npv_objective, optimization/adjoint.py:228-265).  Returns the term of
    step n and its derivative with respect to that step's end state."""
    if discount_rate and dts is None:
        raise ValueError("a discount rate needs the timestep sizes (dts=)")
    elapsed = np.cumsum(np.asarray(dts, float)) if dts is not None else None

    def obj(model, st: OWState, u, dt: float, n: int):
        nc, nw = model.nc, model.nw
        dj = np.zeros(2 * nc + 3 * nw)
        factor = dt * ((1.0 + discount_rate) ** (-(elapsed[n] / time_unit)) if discount_rate else 1.0)
        total = 0.0
        for k in range(nw):
            qw, qo = float(st.qWs[k]), float(st.qOs[k])
            if qw + qo < 0.0:  # producing
                total += water_cost * qw - oil_price * qo
                dj[2 * nc + k] = water_cost * factor
                dj[2 * nc + nw + k] = -oil_price * factor
            else:
                total += -water_inj_cost * qw
                dj[2 * nc + k] = -water_inj_cost * factor
        return total * factor, dj

    return obj


def simulate_forward(model, state0: OWState, dts: Sequence[float], controls) -> List[OWState]:
    """Every step's end state (host copies) under per-step controls."""
    controls = np.atleast_2d(np.asarray(controls, float))
    states = [state0]
    for n, dt in enumerate(dts):
        model.set_controls(controls[n])
        st, ok, _ = model.step(states[-1], float(dt))
        if not ok:
            raise RuntimeError(f"the forward simulation failed to converge at step {n}")
        states.append(st)
    return states


def evaluate_objective(model, objective: Callable, states: Sequence[OWState], dts: Sequence[float],
                       controls) -> float:
    controls = np.atleast_2d(np.asarray(controls, float))
    return float(sum(objective(model, states[n + 1], controls[n], float(dt), n)[0] for n, dt in enumerate(dts)))


# ---- J^T on the device ------------------------------------------------------------------

def jacobian_terms(model, transpose: bool = True):
    """CSR pattern of J (or J^T) in the reference's variable-blocked layout
    (combine_equations, utils/adi/operators.py:204-211) and, per entry, the
    Jacobian entries of the model's device layout that sum into it: the term
    lists of `pmb_ow_csr_values`.  Every perforation pair of a well gets its
    cross-flow product slots whether or not the coupling is on."""
    nc, nw = model.nc, model.nw
    rp, col = model.pattern()
    nnzb = col.size
    njac = 4 * nnzb
    nperf = model.sizes["nperf"]
    lay = model._well_layout(nperf, nw)
    rows_c = np.repeat(np.arange(nc, dtype=np.int64), np.diff(rp))
    col = col.astype(np.int64)
    kb = np.arange(nnzb, dtype=np.int64)
    R, C, T = [], [], []
    for a in range(2):
        for b in range(2):
            R.append(a * nc + rows_c)
            C.append(b * nc + col)
            T.append(4 * kb + 2 * a + b)
    if nw:
        pw = np.repeat(np.arange(nw, dtype=np.int64), np.diff(model.perf_ptr))
        pc = np.asarray(model.perf_cells, np.int64)
        pp = np.arange(nperf, dtype=np.int64)
        for a in range(2):
            for j in range(3):
                R.append(a * nc + pc)
                C.append(2 * nc + j * nw + pw)
                T.append(njac + lay["B"] + 6 * pp + 3 * a + j)
            for b in range(2):
                R.append(2 * nc + a * nw + pw)
                C.append(b * nc + pc)
                T.append(njac + lay["C"] + 4 * pp + 2 * a + b)
        kw = np.arange(nw, dtype=np.int64)
        for r in range(3):
            for j in range(3):
                R.append(2 * nc + r * nw + kw)
                C.append(2 * nc + j * nw + kw)
                T.append(njac + lay["D"] + 9 * kw + 3 * r + j)
        for k in range(nw):
            ps = np.arange(model.perf_ptr[k], model.perf_ptr[k + 1], dtype=np.int64)
            ii, jj = (v.ravel() for v in np.meshgrid(ps, ps, indexing="ij"))
            for a in range(2):
                for b in range(2):
                    R.append(a * nc + pc[ii])
                    C.append(b * nc + pc[jj])
                    T.append(-1 - ((ii * nperf + jj) * 4 + 2 * a + b))
    R, C, T = np.concatenate(R), np.concatenate(C), np.concatenate(T)
    if transpose:
        R, C = C, R
    n = 2 * nc + 3 * nw
    key = R * n + C
    order = np.argsort(key, kind="stable")
    key = key[order]
    uniq, start = np.unique(key, return_index=True)
    ptr = np.append(start, key.size).astype(np.int64)
    rows = uniq // n
    row_ptr = np.zeros(n + 1, np.int64)
    np.add.at(row_ptr, rows + 1, 1)
    return (np.cumsum(row_ptr).astype(np.int32), (uniq % n).astype(np.int32), ptr,
            np.ascontiguousarray(T[order], dtype=np.int64))


class TransposedSystem:
    """J_n^T lambda = rhs on the device for one model: the CSR pattern of
    J^T, its term lists, and transposed CPR handles (one per number of
    block-Jacobi sweeps: the first try, and a stronger retry)."""

    def __init__(self, model, rtol=1e-11, maxiter=400, restart=50, local_sweeps=1, precision="fp64",
                 amg_rebuild_interval=1_000_000):
        torch = _torch()
        self.model = model
        self.rp, self.ci, ptr, terms = jacobian_terms(model, transpose=True)
        self.n = self.rp.size - 1
        dev = "cuda"
        self.d_rp = torch.as_tensor(self.rp, device=dev)
        self.d_ptr = torch.as_tensor(ptr, device=dev)
        self.d_terms = torch.as_tensor(terms, device=dev)
        self.vals = torch.empty(max(self.ci.size, 1), dtype=torch.float64, device=dev)
        self.scale = torch.empty(self.n, dtype=torch.float64, device=dev)
        self.b = torch.empty(self.n, dtype=torch.float64, device=dev)
        self.opts = dict(rtol=float(rtol), maxiter=int(maxiter), restart=int(restart),
                         precision=1 if precision == "mixed" else 0, local_sweeps=int(local_sweeps),
                         amg_rebuild_interval=int(amg_rebuild_interval))
        self.stream = torch.cuda.current_stream().cuda_stream
        self._handles = {}
        self.iterations = 0
        self.solves = 0

    def _handle(self, sweeps):
        h = self._handles.get(sweeps)
        if h is None:
            o = N.CPROpts()
            N.check(N.lib().pmb_cpr_default_opts(N.C.byref(o)))
            for k, v in self.opts.items():
                setattr(o, k, v)
            o.local_sweeps = sweeps
            h = N.c_vp()
            N.check(N.lib().pmb_csr_cpr_create(self.n, self.model.nc, 2, N.as_p(self.rp, N.C.c_int32),
                                               N.as_p(self.ci, N.C.c_int32), 1, N.C.byref(o), self.stream,
                                               N.C.byref(h)))
            self._handles[sweeps] = h
        return h

    def __del__(self):
        for h in getattr(self, "_handles", {}).values():
            try:
                N.lib().pmb_csr_cpr_destroy(h)
            except Exception:
                pass

    def solve(self, jac, well, rhs, weights, lam):
        """lam = J^-T rhs for the Jacobian (jac, well) just assembled."""
        m = self.model
        N.check(N.lib().pmb_ow_csr_values(m._handle, N.ptr(jac), N.ptr(well), int(self.ci.size),
                                          N.ptr(self.d_ptr), N.ptr(self.d_terms), N.ptr(self.vals)))
        N.check(N.lib().pmb_csr_row_scale(self.n, N.ptr(self.d_rp), N.ptr(self.vals), N.ptr(self.scale),
                                          self.stream))
        self.b.copy_(rhs)
        self.b.mul_(self.scale)
        w = np.ascontiguousarray(weights, dtype=np.float64)
        info = (N.C.c_double * 4)()
        for sweeps in (self.opts["local_sweeps"], 3):
            h = self._handle(sweeps)
            N.check(N.lib().pmb_csr_cpr_setup(h, N.ptr(self.vals), N.as_p(w, N.C.c_double)))
            rc = N.lib().pmb_csr_cpr_solve(h, N.ptr(self.b), N.ptr(lam), info)
            self.iterations += int(info[0])
            if rc == N.PMB_OK:
                self.solves += 1
                return
            if rc != 5:
                N.check(rc)
        raise RuntimeError(f"the transposed CPR solve did not converge (relative residual {info[1]:.2e})")


# ---- the sweep ------------------------------------------------------------------------

class ForwardCheckpoints:
    """The forward run kept at every k-th step: the device state that opens
    the step, the well pressure drops its compute_cdp starts from, and the
    states of the final segment."""

    def __init__(self, model, state0: OWState, dts, controls, every: int, on_step: Optional[Callable] = None):
        torch = _torch()
        self.every = max(1, int(every))
        self.dts = [float(v) for v in dts]
        self.controls = np.atleast_2d(np.asarray(controls, float))
        nsteps = len(self.dts)
        nperf = max(model.sizes["nperf"], 1)
        self.points = {}
        self.tail = {}
        last_start = ((nsteps - 1) // self.every) * self.every if nsteps else 0
        x = model.to_device(state0)
        self.x0 = x.clone()
        for n in range(nsteps):
            if n % self.every == 0:
                cdp = torch.empty(nperf, dtype=torch.float64, device="cuda")
                have = N.C.c_int32()
                N.check(N.lib().pmb_ow_get_last_cdp(model._handle, N.ptr(cdp), N.C.byref(have)))
                self.points[n] = (x.clone(), cdp, bool(have.value))
            model.set_controls(self.controls[n])
            ok, _, _ = model.step_device(x, self.dts[n])
            if not ok:
                raise RuntimeError(f"the forward simulation failed to converge at step {n}")
            if n + 1 > last_start:
                self.tail[n + 1] = x.clone()
            if on_step is not None:
                on_step(n, x)
        if nsteps and last_start in self.points:
            self.tail[last_start] = self.points[last_start][0]

    def segments(self):
        starts = sorted(self.points)
        ends = starts[1:] + [len(self.dts)]
        return list(zip(starts, ends))

    def states(self, model, start, end, recompute_log):
        """Device states start .. end of one segment: the kept ones for the
        final segment, else recomputed from the checkpoint at `start`."""
        if all(n in self.tail for n in range(start, end + 1)):
            return {n: self.tail[n] for n in range(start, end + 1)}
        x0, cdp, have = self.points[start]
        N.check(N.lib().pmb_ow_set_last_cdp(model._handle, N.ptr(cdp) if have else None))
        x = x0.clone()
        out = {start: x0}
        for n in range(start, end):
            model.set_controls(self.controls[n])
            ok, _, _ = model.step_device(x, self.dts[n])
            if not ok:
                raise RuntimeError(f"the recomputed forward step {n} failed to converge")
            out[n + 1] = x.clone()
        recompute_log["steps"] = recompute_log.get("steps", 0) + (end - start)
        if end in self.points:  # a recomputed state that the forward run also kept
            ref = self.points[end][0]
            d = float((out[end] - ref).abs().max() / max(float(ref.abs().max()), 1e-300))
            recompute_log["max_rel_diff"] = max(recompute_log.get("max_rel_diff", 0.0), d)
        return out


def compute_gradient_adjoint(model, state0: OWState, dts: Sequence[float], controls,
                             objective: Optional[Callable] = None, states: Optional[Sequence[OWState]] = None,
                             linear_solver: Optional[GpuCPRSolver] = None, perm_gradient: bool = False,
                             checkpoint_every: Optional[int] = None,
                             forward: Optional[ForwardCheckpoints] = None) -> AdjointResult:
    """dJ/du for every control of every step, in one backward sweep
    (compute_gradient_adjoint, optimization/adjoint.py:163-225); with
    perm_gradient also dJ/d(log k) per cell.  `states` (the reference's
    argument: every step's state) skips the forward run; otherwise the
    forward run keeps a checkpoint every `checkpoint_every` steps (default
    about sqrt(nsteps)) and the backward sweep recomputes each segment from
    it.  `linear_solver` (a GpuCPRSolver) gives the options of the
    transposed solves."""
    torch = _torch()
    controls = np.atleast_2d(np.asarray(controls, float))
    nsteps, nw = controls.shape
    if len(dts) != nsteps:
        raise ValueError("one control row per timestep is needed")
    if nw != model.nw:
        raise ValueError("one control per well is needed")
    dts = [float(v) for v in dts]
    objective = objective or npv_objective()
    ls = linear_solver or GpuCPRSolver(rtol=1e-11, maxiter=400)
    system = getattr(model, "_adjoint_system", None)
    key = (ls.rtol, ls.maxiter, ls.restart, ls.local_sweeps, ls.precision)
    if system is None or getattr(model, "_adjoint_key", None) != key:
        system = TransposedSystem(model, rtol=ls.rtol, maxiter=ls.maxiter, restart=ls.restart,
                                  local_sweeps=ls.local_sweeps, precision=ls.precision)
        model._adjoint_system, model._adjoint_key = system, key
    if states is not None:
        if len(states) != nsteps + 1:
            raise ValueError("states must hold state0 and the end state of every step")
        dev_states = None
    else:
        if forward is None:
            every = checkpoint_every or max(1, int(round(math.sqrt(nsteps))))
            forward = ForwardCheckpoints(model, state0, dts, controls, every)
    nc = model.nc
    nperf = max(model.sizes["nperf"], 1)
    ctrl = slice(2 * nc + 2 * nw, 2 * nc + 3 * nw)
    cdp0 = torch.zeros(nperf, dtype=torch.float64, device="cuda")
    lam = torch.zeros(2 * nc + 3 * nw, dtype=torch.float64, device="cuda")
    y = torch.empty_like(lam)
    rhs = torch.empty_like(lam)
    grad = np.zeros((nsteps, nw))
    host_states: List[Optional[OWState]] = [None] * (nsteps + 1)
    host_states[0] = state0
    if perm_gradient:
        t0, t1 = _half_transmissibilities(model)
        gperm = torch.zeros(nc, dtype=torch.float64, device="cuda")
        ff = torch.empty(2 * max(model.N.shape[0], 1), dtype=torch.float64, device="cuda")
        pr = torch.empty(2 * nperf, dtype=torch.float64, device="cuda")
    log = {}
    jtotal = 0.0
    have_lam = False
    segs = forward.segments() if states is None else [(0, nsteps)]
    for start, end in reversed(segs):
        if states is None:
            xs = forward.states(model, start, end, log)
        else:
            xs = {n: model.to_device(states[n]) for n in range(start, end + 1)}
        for n in reversed(range(start, end)):
            model.set_controls(controls[n])
            x_prev, x = xs[n], xs[n + 1]
            st = model.from_device(x) if states is None else states[n + 1]
            host_states[n + 1] = st
            jn, djdx = objective(model, st, controls[n], dts[n], n)
            jtotal += jn
            rhs.copy_(torch.as_tensor(np.asarray(djdx, float), device="cuda"))
            rhs.neg_()
            if have_lam:
                # dR_{n+1}/dx_n couples this step to the one after it
                N.check(N.lib().pmb_ow_prev_jacobian_tmul(model._handle, N.ptr(x), dts[n + 1], N.ptr(lam),
                                                          N.ptr(y)))
                rhs.sub_(y)
            _, jac, well = model.assemble_device(x, x_prev, dts[n], cdp0, True)
            w = GpuCPRSolver.weights(model, {"pressure": st.pressure})
            system.solve(jac, well, rhs, w, lam)
            have_lam = True
            grad[n] = -lam[ctrl].cpu().numpy()
            if perm_gradient:
                N.check(N.lib().pmb_ow_perm_contract(model._handle, N.ptr(x), N.ptr(lam), N.ptr(t0), N.ptr(t1),
                                                     N.ptr(ff), N.ptr(pr), N.ptr(gperm)))
    dx0 = None
    if nsteps:
        x0 = forward.x0 if states is None else model.to_device(states[0])
        N.check(N.lib().pmb_ow_prev_jacobian_tmul(model._handle, N.ptr(x0), dts[0], N.ptr(lam), N.ptr(y)))
        dx0 = y.cpu().numpy()
    stats = {"transposed_solves": system.solves, "krylov_iterations": system.iterations,
             "recomputed_steps": log.get("steps", 0), "recompute_max_rel_diff": log.get("max_rel_diff", 0.0),
             "checkpoint_every": forward.every if states is None else 0}
    return AdjointResult(value=float(jtotal), gradient=grad, states=host_states, initial_state_gradient=dx0,
                         perm_gradient=gperm.cpu().numpy() if perm_gradient else None, stats=stats)


def _half_transmissibilities(model):
    """Device arrays t0, t1: the half-face transmissibility of N[f,0] and of
    N[f,1] for every interior interface (for dT_f/d(log k))."""
    from .ow_model import face_transmissibility_device
    torch = _torch()
    cached = getattr(model, "_half_t", None)
    if cached is not None:
        return cached
    g = model.g
    _, th = face_transmissibility_device(g, model.rock)
    fp = np.asarray(g.cells.facePos).ravel()
    cf = np.asarray(g.cells.faces)
    cf = cf[:, 0] if cf.ndim > 1 else cf
    cell_no = np.repeat(np.arange(model.nc), np.diff(fp))
    internal = np.flatnonzero(model._internal)
    pos = np.full(np.asarray(g.faces.neighbors).shape[0], -1)
    pos[internal] = np.arange(internal.size)
    k = pos[cf]
    keep = k >= 0
    t0 = np.zeros(max(internal.size, 1))
    t1 = np.zeros(max(internal.size, 1))
    on0 = keep & (cell_no == model.N[np.maximum(k, 0), 0])
    on1 = keep & ~on0
    t0[k[on0]] = np.asarray(th)[on0]
    t1[k[on1]] = np.asarray(th)[on1]
    model._half_t = (torch.as_tensor(t0, device="cuda"), torch.as_tensor(t1, device="cuda"))
    return model._half_t


def adjoint_objective(factory: Callable, state0: OWState, dts: Sequence[float],
                      objective: Optional[Callable] = None, linear_solver: Optional[GpuCPRSolver] = None,
                      checkpoint_every: Optional[int] = None) -> Callable:
    """J(log_k, controls) as a torch function whose backward is the adjoint
    sweep.  `factory(perm) -> GpuOilWaterModel` builds the model for a
    permeability field (the wells' indices computed from it); `log_k` is a
    torch tensor of per-cell log-permeabilities, `controls` (nsteps x nw)
    the well targets.  The forward pass simulates on the device keeping
    checkpoints only, evaluating the objective step by step; backward runs
    the adjoint sweep from those checkpoints and returns dJ/d(log k) and
    dJ/du."""
    torch = _torch()
    objective = objective or npv_objective()
    nsteps = len(dts)

    class _OWAdjoint(torch.autograd.Function):
        @staticmethod
        def forward(ctx, log_k, controls):
            model = factory(np.exp(log_k.detach().cpu().numpy().astype(np.float64)))
            u = np.atleast_2d(controls.detach().cpu().numpy().astype(np.float64))
            every = checkpoint_every or max(1, int(round(math.sqrt(nsteps))))
            terms = []
            fwd = ForwardCheckpoints(model, state0, dts, u, every, on_step=lambda n, x: terms.append(
                objective(model, model.from_device(x), u[n], float(dts[n]), n)[0]))
            # summed last step first, as the adjoint sweep sums them
            value = float(sum(reversed(terms)))
            ctx.model, ctx.u, ctx.fwd = model, u, fwd
            return torch.tensor(value, dtype=torch.float64)

        @staticmethod
        def backward(ctx, grad_out):
            res = compute_gradient_adjoint(ctx.model, state0, dts, ctx.u, objective, linear_solver=linear_solver,
                                           perm_gradient=True, forward=ctx.fwd)
            g = grad_out.detach().cpu().double()
            return (g * torch.as_tensor(res.perm_gradient), g * torch.as_tensor(res.gradient))

    return _OWAdjoint.apply
