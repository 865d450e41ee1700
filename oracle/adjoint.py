"""Oracle: adjoint gradient of a well-control objective (test infrastructure only).

A numpy restatement, over the oracle oil-water model (oracle/ow.py), of
  * compute_gradient_adjoint (pymrst/modules/optimization/adjoint.py:161-225),
  * simulate_forward (:140-151) and _set_controls (:63-65),
  * _jac_wrt_current (:74-80): the forward Jacobian, assembled with cdp = None
    (zeros), as the reference's call does,
  * _jac_wrt_previous (:83-105): only the accumulation terms see x_{n-1},
  * _jac_wrt_controls (:108-123): -1 on each well's control row,
  * npv_objective (:228-265) without discounting, with its derivative.
The accumulation derivatives are written out by hand in place of the
reference's forward AD.
"""

from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from . import ow


@dataclass
class AdjointResult:
    value: float
    gradient: np.ndarray               # nsteps x nw
    states: List[ow.State]             # state0 and every step's end state
    initial_state_gradient: Optional[np.ndarray]


def set_controls(prob: ow.OWProblem, u) -> None:
    for w, v in zip(prob.wells, np.asarray(u, float).ravel()):
        w.val = float(v)


def npv(prob: ow.OWProblem, st: ow.State, dt: float, oil_price=60.0, water_cost=6.0, water_inj_cost=6.0):
    """J_n of npv_objective at the end-of-step state, and dJ_n/dx_n in the
    variable-blocked layout [p, sW, qWs, qOs, bhp]."""
    nc, nw = prob.nc, prob.nw
    dj = np.zeros(2 * nc + 3 * nw)
    j = 0.0
    for k in range(nw):
        qw, qo = float(st.qWs[k]), float(st.qOs[k])
        if qo + qw < 0.0:
            term = (-oil_price) * qo + water_cost * qw
            dj[2 * nc + k] = water_cost * dt
            dj[2 * nc + nw + k] = -oil_price * dt
        else:
            term = (-water_inj_cost) * qw
            dj[2 * nc + k] = -water_inj_cost * dt
        j = term if k == 0 else j + term
    return j * dt, dj


def jac_wrt_previous(prob: ow.OWProblem, st_prev: ow.State, dt: float) -> sp.csr_array:
    """dR_n/dx_{n-1}: water = (pv b_w s - pv b_w(p0) s0)/dt and
    oil = (pv b_o (1-s) - pv b_o(p0) (1-s0))/dt differentiated in (p0, s0);
    the well rows are zero."""
    nc, nw = prob.nc, prob.nw
    f = prob.fluid
    bw0, dbw0 = ow.shrinkage(f, 0, st_prev.pressure)
    bo0, dbo0 = ow.shrinkage(f, 1, st_prev.pressure)
    pv, idt = prob.pv, 1.0 / dt
    s0 = st_prev.sW
    cells = np.arange(nc)
    rows = np.concatenate([cells, cells, nc + cells, nc + cells])
    cols = np.concatenate([cells, nc + cells, cells, nc + cells])
    vals = np.concatenate([-idt * pv * dbw0 * s0, -idt * pv * bw0,
                           -idt * pv * dbo0 * (1.0 - s0), idt * pv * bo0])
    n = 2 * nc + 3 * nw
    return sp.csr_array((vals, (rows, cols)), shape=(n, n))


def jac_wrt_controls(prob: ow.OWProblem) -> sp.csr_array:
    nc, nw = prob.nc, prob.nw
    n = 2 * nc + 3 * nw
    return sp.csr_array((-np.ones(nw), (2 * nc + 2 * nw + np.arange(nw), np.arange(nw))), shape=(n, nw))


def simulate_forward(prob: ow.OWProblem, state0: ow.State, dts: Sequence[float], controls) -> List[ow.State]:
    states = [state0]
    for n, dt in enumerate(dts):
        set_controls(prob, controls[n])
        st, ok, _ = ow.step(prob, states[-1], float(dt))
        if not ok:
            raise RuntimeError(f"forward step {n} did not converge")
        states.append(st)
    return states


def compute_gradient_adjoint(prob: ow.OWProblem, state0: ow.State, dts: Sequence[float], controls,
                             objective=npv, states=None) -> AdjointResult:
    controls = np.atleast_2d(np.asarray(controls, float))
    nsteps, nw = controls.shape
    assert len(dts) == nsteps and nw == prob.nw
    if states is None:
        states = simulate_forward(prob, state0, dts, controls)
    dRdu = jac_wrt_controls(prob)
    grad = np.zeros((nsteps, nw))
    jtotal = 0.0
    lam = None
    for n in reversed(range(nsteps)):
        set_controls(prob, controls[n])
        st_prev, st = states[n], states[n + 1]
        dt = float(dts[n])
        jn, djdx = objective(prob, st, dt)
        jtotal += jn
        rhs = -djdx
        if lam is not None:
            b = jac_wrt_previous(prob, st, float(dts[n + 1]))
            rhs = rhs - b.T @ lam
        _, a = ow.assemble(prob, st_prev, st, dt, None)
        lam = spla.spsolve(sp.csc_matrix(a.T), rhs)
        grad[n] = dRdu.T @ lam
    dx0 = jac_wrt_previous(prob, state0, float(dts[0])).T @ lam if nsteps else None
    return AdjointResult(value=jtotal, gradient=grad, states=list(states), initial_state_gradient=dx0)
