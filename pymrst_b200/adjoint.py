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
from .ow_model import OWState


@dataclass
class AdjointResult:
    value: float
    gradient: np.ndarray                      # nsteps x nw: dJ/du
    states: List[OWState]                     # state0 and the end state of every step
    initial_state_gradient: Optional[np.ndarray]  # dJ/dx_0, variable-blocked layout


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


def compute_gradient_adjoint(model, state0: OWState, dts: Sequence[float], controls,
                             objective: Optional[Callable] = None, states: Optional[Sequence[OWState]] = None,
                             linear_solver: Optional[GpuCPRSolver] = None) -> AdjointResult:
    """dJ/du for every control of every step, in one backward sweep
    (compute_gradient_adjoint, optimization/adjoint.py:161-225)."""
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
    dx0 = jac_wrt_previous(model, state0, float(dts[0])).T @ lam if nsteps else None
    return AdjointResult(value=float(jtotal), gradient=grad, states=list(states), initial_state_gradient=dx0)
