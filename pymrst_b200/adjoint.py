"""Adjoint gradients of well-control objectives on the GPU model.

Mirrors pymrst/modules/optimization/adjoint.py: `compute_gradient_adjoint`
(:161-225), `simulate_forward` (:140-151), `evaluate_objective` (:154-158)
and `npv_objective` (:228-265), with `GpuOilWaterModel` in place of
`TwoPhaseOilWaterModelAD`.

  * forward: the device Newton step per timestep, controls set before each
    step as `_set_controls` does;
  * backward, per step n: the Jacobian dR_n/dx_n at the stored states is
    assembled on the device with the well pressure drops cdp = 0, as the
    reference's `_jac_wrt_current` calls `assemble` without them (:74-80),
    and J_n^T lambda_n = rhs is solved by the device CPR with transposed
    transfer operators (`GpuCPRSolver.solve_transposed`) where the reference
    calls spsolve (:209);
  * dR_{n+1}/dx_n touches only the accumulation terms (:83-105) and dR/du is
    -1 on each control row (:108-123): both are formed in closed form on the
    host, as is the objective derivative.

With `perm_gradient=True` the sweep also returns dJ/d(log k) per cell, for
which the reference has no counterpart (it is checked against finite
differences).  The residual is linear in every interface transmissibility
T_f and in every perforation's well index: R = R_0 + sum_f T_f G_f, so
lambda^T dR/dT_f = (flux of f) . (lambda[N0] - lambda[N1]) / T_f with the
phase fluxes exported by the device (pmb_ow_fluxes), and
dT_f/d(log k_c) = T_f^2 / t_{c,f} for the half-face transmissibility t_{c,f};
a perforation's rates scale with its well index, which scales with the
permeability of its cell.  Wells whose perforations cross-flow are outside
this (their mixture is not linear in one well index).

Objectives are callables `obj(model, state, u, dt, n) -> (J_n, dJ_n/dx_n)`
with the derivative in the reference's variable-blocked layout [p, sW, qWs,
qOs, bhp]; `npv_objective` builds the reference's NPV.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Callable, List, Optional, Sequence

import numpy as np
import scipy.sparse as sp

from .linear_solvers import GpuCPRSolver
from .ow_model import OWState, _torch


@dataclass
class AdjointResult:
    value: float
    gradient: np.ndarray                      # nsteps x nw: dJ/du
    states: List[OWState]                     # state0 and the end state of every step
    initial_state_gradient: Optional[np.ndarray]  # dJ/dx_0, variable-blocked layout
    perm_gradient: Optional[np.ndarray] = None    # dJ/d(log k) per cell


def npv_objective(oil_price: float = 60.0, water_cost: float = 6.0, water_inj_cost: float = 6.0,
                  discount_rate: float = 0.0, dts: Optional[Sequence[float]] = None,
                  time_unit: float = 365.0 * 86400.0) -> Callable:
    """Net present value with the reference's signs: a producer (qWs + qOs
    < 0) earns -oil_price * qOs and pays water_cost * qWs, an injector pays
    -water_inj_cost * qWs, all times dt and the discount factor
    (npv_objective, optimization/adjoint.py:228-265)."""
    if discount_rate and dts is None:
        raise ValueError("discounting needs the timestep sizes; pass dts=")
    elapsed = np.cumsum(np.asarray(dts, float)) if dts is not None else None

    def obj(model, st: OWState, u, dt: float, n: int):
        nc, nw = model.nc, model.nw
        dj = np.zeros(2 * nc + 3 * nw)
        disc = (1.0 + discount_rate) ** (-(elapsed[n] / time_unit)) if discount_rate else 1.0
        scale = dt * disc
        j = 0.0
        for k in range(nw):
            qw, qo = float(st.qWs[k]), float(st.qOs[k])
            if qo + qw < 0.0:
                term = (-oil_price) * qo + water_cost * qw
                dj[2 * nc + k] = water_cost * scale
                dj[2 * nc + nw + k] = -oil_price * scale
            else:
                term = (-water_inj_cost) * qw
                dj[2 * nc + k] = -water_inj_cost * scale
            j = term if k == 0 else j + term
        return j * scale, dj

    return obj


def simulate_forward(model, state0: OWState, dts: Sequence[float], controls) -> List[OWState]:
    """Run the schedule with per-step controls, keeping every state."""
    controls = np.atleast_2d(np.asarray(controls, float))
    states = [state0]
    for n, dt in enumerate(dts):
        model.set_controls(controls[n])
        st, ok, _ = model.step(states[-1], float(dt))
        if not ok:
            raise RuntimeError(f"forward step {n} did not converge")
        states.append(st)
    return states


def evaluate_objective(model, objective: Callable, states: Sequence[OWState], dts: Sequence[float],
                       controls) -> float:
    controls = np.atleast_2d(np.asarray(controls, float))
    return float(sum(objective(model, states[n + 1], controls[n], float(dt), n)[0] for n, dt in enumerate(dts)))


def jac_wrt_previous(model, st_prev: OWState, dt: float) -> sp.csr_array:
    """dR_n/dx_{n-1} (_jac_wrt_previous, optimization/adjoint.py:83-105): the
    accumulation terms (pv b_w s - pv b_w(p0) s0)/dt and
    (pv b_o (1-s) - pv b_o(p0) (1-s0))/dt differentiated in (p0, s0)."""
    f = model.fluid_params
    nc, nw = model.nc, model.nw
    p0 = np.asarray(st_prev.pressure, float)
    s0 = np.asarray(st_prev.sW, float)

    def shrink(i):
        if f.c[i] == 0.0:
            return np.full(nc, f.b0[i]), np.zeros(nc)
        b = f.b0[i] * np.exp(f.c[i] * (p0 - f.p_ref))
        return b, f.c[i] * b

    bw0, dbw0 = shrink(0)
    bo0, dbo0 = shrink(1)
    pv, idt = model.pv, 1.0 / dt
    cells = np.arange(nc)
    rows = np.concatenate([cells, cells, nc + cells, nc + cells])
    cols = np.concatenate([cells, nc + cells, cells, nc + cells])
    vals = np.concatenate([-idt * pv * dbw0 * s0, -idt * pv * bw0, -idt * pv * dbo0 * (1.0 - s0), idt * pv * bo0])
    n = 2 * nc + 3 * nw
    return sp.csr_array((vals, (rows, cols)), shape=(n, n))


class _PermSensitivity:
    """lambda^T dR/d(log k) for a model: interface geometry and the device
    flux export."""

    def __init__(self, model):
        from . import _native as N
        from .ow_model import face_transmissibility_device
        self.N = N
        self.model = model
        g = model.g
        tf, th = face_transmissibility_device(g, model.rock)
        fp = np.asarray(g.cells.facePos).ravel()
        cf = np.asarray(g.cells.faces)
        cf = cf[:, 0] if cf.ndim > 1 else cf
        cell_no = np.repeat(np.arange(model.nc), np.diff(fp))
        internal = np.flatnonzero(model._internal)
        pos = np.full(np.asarray(g.faces.neighbors).shape[0], -1)
        pos[internal] = np.arange(internal.size)
        k = pos[cf]
        keep = k >= 0
        self.t0 = np.zeros(internal.size)
        self.t1 = np.zeros(internal.size)
        on0 = keep & (cell_no == model.N[np.maximum(k, 0), 0])
        on1 = keep & ~on0
        self.t0[k[on0]] = np.asarray(th)[on0]
        self.t1[k[on1]] = np.asarray(th)[on1]
        self.T = np.asarray(model.T, float)
        self.perf_cell = np.asarray(model.perf_cells, np.int64)
        self.perf_well = np.repeat(np.arange(model.nw), np.diff(model.perf_ptr))

    def contract(self, st: OWState, lam: np.ndarray) -> np.ndarray:
        torch = _torch()
        m, N = self.model, self.N
        nc, nw = m.nc, m.nw
        x = m.to_device(st)
        nf = self.T.size
        flux = torch.empty(2 * max(nf, 1), dtype=torch.float64, device="cuda")
        nperf = max(self.perf_cell.size, 1)
        rates = torch.empty(2 * nperf, dtype=torch.float64, device="cuda")
        cdp = torch.zeros(nperf, dtype=torch.float64, device="cuda")
        N.check(N.lib().pmb_ow_fluxes(m._handle, N.ptr(x), N.ptr(cdp), N.ptr(flux), N.ptr(rates)))
        F = flux.cpu().numpy()[:2 * nf].reshape(-1, 2)
        q = rates.cpu().numpy()[:2 * self.perf_cell.size].reshape(-1, 2)
        lw, lo = lam[:nc], lam[nc:2 * nc]
        n0, n1 = m.N[:, 0], m.N[:, 1]
        gf = F[:, 0] * (lw[n0] - lw[n1]) + F[:, 1] * (lo[n0] - lo[n1])  # lambda^T dR/dT_f * T_f
        out = np.zeros(nc)
        with np.errstate(divide="ignore", invalid="ignore"):
            np.add.at(out, n0, np.where(self.t0 > 0, gf * self.T / self.t0, 0.0))
            np.add.at(out, n1, np.where(self.t1 > 0, gf * self.T / self.t1, 0.0))
        if nw:
            lqw, lqo = lam[2 * nc:2 * nc + nw], lam[2 * nc + nw:2 * nc + 2 * nw]
            c, k = self.perf_cell, self.perf_well
            gp = -(lw[c] + lqw[k]) * q[:, 0] - (lo[c] + lqo[k]) * q[:, 1]
            np.add.at(out, c, gp)
        return out


def compute_gradient_adjoint(model, state0: OWState, dts: Sequence[float], controls,
                             objective: Optional[Callable] = None, states: Optional[Sequence[OWState]] = None,
                             linear_solver: Optional[GpuCPRSolver] = None,
                             perm_gradient: bool = False) -> AdjointResult:
    """dJ/du for every control of every step, in one backward sweep
    (compute_gradient_adjoint, optimization/adjoint.py:161-225); with
    perm_gradient also dJ/d(log k) per cell."""
    controls = np.atleast_2d(np.asarray(controls, float))
    nsteps, nw = controls.shape
    if len(dts) != nsteps:
        raise ValueError("one control row per timestep")
    if nw != model.nw:
        raise ValueError("one control per well")
    objective = objective or npv_objective()
    solver = linear_solver or GpuCPRSolver(rtol=1e-11, maxiter=400)
    if states is None:
        states = simulate_forward(model, state0, dts, controls)
    nc = model.nc
    ctrl_rows = 2 * nc + 2 * nw + np.arange(nw)
    grad = np.zeros((nsteps, nw))
    sens = _PermSensitivity(model) if perm_gradient else None
    gperm = np.zeros(nc) if perm_gradient else None
    jtotal = 0.0
    lam = None
    for n in reversed(range(nsteps)):
        model.set_controls(controls[n])
        st_prev, st = states[n], states[n + 1]
        dt = float(dts[n])
        jn, djdx = objective(model, st, controls[n], dt, n)
        jtotal += jn
        rhs = -djdx
        if lam is not None:
            rhs = rhs - jac_wrt_previous(model, st, float(dts[n + 1])).T @ lam
        _, a = model.residual_and_jacobian(st_prev, st, dt, None)
        lam = solver.solve_transposed(a, rhs, model, {"pressure": st.pressure})
        grad[n] = -lam[ctrl_rows]
        if sens is not None:
            gperm += sens.contract(st, lam)
    dx0 = jac_wrt_previous(model, state0, float(dts[0])).T @ lam if nsteps else None
    return AdjointResult(value=float(jtotal), gradient=grad, states=list(states), initial_state_gradient=dx0,
                         perm_gradient=gperm)


def adjoint_objective(factory: Callable, state0: OWState, dts: Sequence[float],
                      objective: Optional[Callable] = None,
                      linear_solver: Optional[GpuCPRSolver] = None) -> Callable:
    """J(log_k, controls) as a torch function whose backward is the adjoint
    sweep.  `factory(perm) -> GpuOilWaterModel` builds the model for a
    permeability field (the wells' indices computed from it); `log_k` is a
    torch tensor of per-cell log-permeabilities, `controls` (nsteps x nw)
    the well targets.  The forward pass simulates on the device and keeps
    every step's state on the host (a checkpoint per timestep); backward runs
    compute_gradient_adjoint on those states and returns dJ/d(log k) and
    dJ/du."""
    torch = _torch()
    objective = objective or npv_objective()

    class _OWAdjoint(torch.autograd.Function):
        @staticmethod
        def forward(ctx, log_k, controls):
            model = factory(np.exp(log_k.detach().cpu().numpy().astype(np.float64)))
            u = np.atleast_2d(controls.detach().cpu().numpy().astype(np.float64))
            states = simulate_forward(model, state0, dts, u)
            ctx.model, ctx.u, ctx.states = model, u, states
            value = evaluate_objective(model, objective, states, dts, u)
            return torch.tensor(value, dtype=torch.float64)

        @staticmethod
        def backward(ctx, grad_out):
            res = compute_gradient_adjoint(ctx.model, state0, dts, ctx.u, objective, states=ctx.states,
                                           linear_solver=linear_solver, perm_gradient=True)
            g = grad_out.detach().cpu().double()
            return (g * torch.as_tensor(res.perm_gradient), g * torch.as_tensor(res.gradient))

    return _OWAdjoint.apply
