"""Adjoint gradients on the GPU model against the reference's own
compute_gradient_adjoint (optimization/adjoint.py:161-225), golden fixtures
made by tests/golden/make_golden.py.

Tolerances: forward states as the Newton-history tests (p 1e-8 relative,
sW 1e-7); objective 1e-9 relative; gradients 1e-6 of each control column's
largest entry (the bhp-control column is ~1e-6 in magnitude and carries the
cancellation); dJ/dx0 1e-6 of its largest entry.  The device transposed
CPR runs at rtol 1e-11 where the reference solves directly.
"""

import numpy as np
import pytest

from fixtures import load, ow_case

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from pymrst_b200.adjoint import compute_gradient_adjoint, npv_objective  # noqa: E402
from pymrst_b200.build import build  # noqa: E402
from pymrst_b200.ow_model import GpuOilWaterModel, OWState  # noqa: E402

build()


@pytest.mark.parametrize("name", ["adjoint_grav.npz", "adjoint_nograv.npz"])
def test_adjoint_gradient_matches_reference(name):
    d = load(name)
    g, rock, fluid, wells = ow_case(d)
    m = GpuOilWaterModel(g, rock, fluid, wells, gravity=float(d["gravity"]),
                         cpr_options=dict(rtol=1e-12, maxiter=400))
    st0 = OWState(pressure=d["p0"].copy(), sW=d["sw0"].copy(), qWs=d["qws0"].copy(), qOs=d["qos0"].copy(),
                  bhp=d["bhp0"].copy())
    res = compute_gradient_adjoint(m, st0, d["dts"], d["controls"], npv_objective())
    for k, s in enumerate(res.states[1:]):
        assert np.abs(s.pressure - d["p_hist"][k]).max() <= 1e-8 * np.abs(d["p_hist"][k]).max()
        assert np.abs(s.sW - d["sw_hist"][k]).max() <= 1e-7
    assert abs(res.value - float(d["value"])) <= 1e-9 * abs(float(d["value"]))
    for j in range(d["gradient"].shape[1]):
        ref = d["gradient"][:, j]
        assert np.abs(res.gradient[:, j] - ref).max() <= 1e-6 * np.abs(ref).max()
    assert np.abs(res.initial_state_gradient - d["dx0"]).max() <= 1e-6 * np.abs(d["dx0"]).max()


def test_adjoint_gradient_matches_finite_differences():
    """Central differences of the objective in one injector rate of one step."""
    d = load("adjoint_nograv.npz")
    g, rock, fluid, wells = ow_case(d)
    m = GpuOilWaterModel(g, rock, fluid, wells, gravity=float(d["gravity"]),
                         cpr_options=dict(rtol=1e-12, maxiter=400))
    st0 = OWState(pressure=d["p0"].copy(), sW=d["sw0"].copy(), qWs=d["qws0"].copy(), qOs=d["qos0"].copy(),
                  bhp=d["bhp0"].copy())
    u = d["controls"].copy()
    obj = npv_objective()
    res = compute_gradient_adjoint(m, st0, d["dts"], u, obj)
    from pymrst_b200.adjoint import evaluate_objective, simulate_forward
    h = 1e-4 * abs(u[1, 0])
    vals = []
    for sgn in (1.0, -1.0):
        up = u.copy()
        up[1, 0] += sgn * h
        vals.append(evaluate_objective(m, obj, simulate_forward(m, st0, d["dts"], up), d["dts"], up))
    fd = (vals[0] - vals[1]) / (2 * h)
    assert abs(fd - res.gradient[1, 0]) <= 1e-4 * abs(res.gradient[1, 0])


def test_log_permeability_gradient_matches_finite_differences():
    """dJ/d(log k_c) from the adjoint sweep against central differences of the
    objective (h = 1e-5 in log k) at a few cells, a perforated one among
    them; the reference has no such gradient.  A cell's perturbation scales
    its half-transmissibilities and its perforations' well indices (Peaceman
    indices are proportional to the permeability)."""
    from types import SimpleNamespace
    from pymrst_b200.adjoint import evaluate_objective, simulate_forward
    from pymrst_b200.params import make_rock
    d = load("adjoint_nograv.npz")
    g, rock, fluid, wells = ow_case(d)
    opts = dict(rtol=1e-12, maxiter=400)
    tight = dict(tol_cnv=1e-9, tol_mb=1e-12, tol_well=1e-10, max_iterations=60)
    st0 = OWState(pressure=d["p0"].copy(), sW=d["sw0"].copy(), qWs=d["qws0"].copy(), qOs=d["qos0"].copy(),
                  bhp=d["bhp0"].copy())
    obj = npv_objective()
    m = GpuOilWaterModel(g, rock, fluid, wells, gravity=float(d["gravity"]), cpr_options=opts, **tight)
    res = compute_gradient_adjoint(m, st0, d["dts"], d["controls"], obj, perm_gradient=True)
    perf_cell = int(np.asarray(wells[2].cells).ravel()[0])
    cells = [perf_cell, 7, int(g.cells.num) // 2 + 3]
    h = 1e-5
    for c in cells:
        vals = []
        for sgn in (1.0, -1.0):
            perm = d["perm"].copy()
            perm[c] *= np.exp(sgn * h)
            ws = []
            for w in wells:
                wi = np.asarray(w.WI, float).copy()
                wi[np.asarray(w.cells).ravel() == c] *= np.exp(sgn * h)
                ws.append(SimpleNamespace(**{**vars(w), "WI": wi}))
            mp = GpuOilWaterModel(g, make_rock(g, perm[:, None], float(d["poro"])), fluid, ws,
                                  gravity=float(d["gravity"]), cpr_options=opts, **tight)
            sts = simulate_forward(mp, st0, d["dts"], d["controls"])
            vals.append(evaluate_objective(mp, obj, sts, d["dts"], d["controls"]))
        fd = (vals[0] - vals[1]) / (2 * h)
        scale = np.abs(res.perm_gradient).max()
        assert abs(fd - res.perm_gradient[c]) <= 1e-4 * scale + 1e-3 * abs(fd), (c, fd, res.perm_gradient[c])


def test_torch_autograd_wrapper_returns_the_adjoint_gradients():
    from pymrst_b200.adjoint import adjoint_objective
    from pymrst_b200.params import make_rock
    d = load("adjoint_nograv.npz")
    g, rock, fluid, wells = ow_case(d)
    opts = dict(rtol=1e-12, maxiter=400)
    st0 = OWState(pressure=d["p0"].copy(), sW=d["sw0"].copy(), qWs=d["qws0"].copy(), qOs=d["qos0"].copy(),
                  bhp=d["bhp0"].copy())
    k0 = d["perm"].copy()

    def factory(perm):
        from types import SimpleNamespace
        ws = []
        for w in wells:  # Peaceman indices scale with the perforated cell's permeability
            c = np.asarray(w.cells).ravel()
            ws.append(SimpleNamespace(**{**vars(w), "WI": np.asarray(w.WI, float) * perm[c] / k0[c]}))
        return GpuOilWaterModel(g, make_rock(g, perm[:, None], float(d["poro"])), fluid, ws,
                                gravity=float(d["gravity"]), cpr_options=opts)

    J = adjoint_objective(factory, st0, d["dts"])
    log_k = torch.tensor(np.log(k0), dtype=torch.float64, requires_grad=True)
    u = torch.tensor(d["controls"], dtype=torch.float64, requires_grad=True)
    val = J(log_k, u)
    val.backward()
    assert abs(float(val) - float(d["value"])) <= 1e-9 * abs(float(d["value"]))
    ref = compute_gradient_adjoint(factory(k0), st0, d["dts"], d["controls"], npv_objective(), perm_gradient=True)
    np.testing.assert_allclose(u.grad.numpy(), ref.gradient, rtol=1e-8, atol=1e-12 * np.abs(ref.gradient).max())
    np.testing.assert_allclose(log_k.grad.numpy(), ref.perm_gradient, rtol=1e-8,
                               atol=1e-12 * np.abs(ref.perm_gradient).max())


# ---- the device pieces of the sweep ------------------------------------------------------

def _xflow_model_and_jacobian():
    d = load("ow_assemble_xflow.npz")
    g, rock, fluid, wells = ow_case(d)
    m = GpuOilWaterModel(g, rock, fluid, wells, gravity=float(d["gravity"]))
    st = OWState(pressure=d["p"].copy(), sW=d["sw"].copy(), qWs=d["qws"].copy(), qOs=d["qos"].copy(),
                 bhp=d["bhp"].copy())
    st0 = OWState(pressure=d["p0"].copy(), sW=d["sw0"].copy(), qWs=d["qws0"].copy(), qOs=d["qos0"].copy(),
                  bhp=d["bhp0"].copy())
    x, x0 = m.to_device(st), m.to_device(st0)
    res, jac, well = m.assemble_device(x, x0, float(d["dt"]), torch.as_tensor(d["cdp"], device="cuda"))
    return d, m, st, st0, x, x0, jac, well


@pytest.mark.parametrize("transpose", [False, True])
def test_device_csr_jacobian_equals_the_exported_one(transpose):
    """J and J^T in the reference's layout built on the device from the term
    lists, on the cross-flow fixture (the mixture products are on)."""
    import scipy.sparse as sp
    from pymrst_b200 import _native as N
    from pymrst_b200.adjoint import jacobian_terms
    d, m, st, st0, x, x0, jac, well = _xflow_model_and_jacobian()
    rp, ci, ptr, terms = jacobian_terms(m, transpose=transpose)
    vals = torch.empty(ci.size, dtype=torch.float64, device="cuda")
    d_ptr, d_terms = torch.as_tensor(ptr, device="cuda"), torch.as_tensor(terms, device="cuda")
    N.check(N.lib().pmb_ow_csr_values(m._handle, N.ptr(jac), N.ptr(well), ci.size, N.ptr(d_ptr), N.ptr(d_terms),
                                      N.ptr(vals)))
    n = rp.size - 1
    A = sp.csr_array((vals.cpu().numpy(), ci, rp), shape=(n, n))
    J = m.export_jacobian(jac.cpu().numpy(), well.cpu().numpy())
    ref = sp.csr_array(J.T) if transpose else J
    assert abs(A - ref).max() <= 1e-15 * abs(ref).max()


def test_previous_step_coupling_equals_the_oracle():
    """(dR_{n+1}/dx_n)^T lambda on the device against the oracle's
    jac_wrt_previous (the reference's _jac_wrt_previous restated)."""
    from oracle import adjoint as oadj
    from oracle import ow as oow
    from pymrst_b200 import _native as N
    d, m, st, st0, x, x0, jac, well = _xflow_model_and_jacobian()
    g, rock, fluid, wells = ow_case(d)
    prob = oow.build_problem(g, rock, fluid.params, wells, gravity=float(d["gravity"]))
    lam = np.random.default_rng(3).normal(size=2 * m.nc + 3 * m.nw)
    y = torch.empty(lam.size, dtype=torch.float64, device="cuda")
    dt = float(d["dt"])
    d_lam = torch.as_tensor(lam, device="cuda")
    N.check(N.lib().pmb_ow_prev_jacobian_tmul(m._handle, N.ptr(x0), dt, N.ptr(d_lam),
                                              N.ptr(y)))
    st0o = oow.State(pressure=d["p0"].copy(), sW=d["sw0"].copy(), qWs=d["qws0"].copy(), qOs=d["qos0"].copy(),
                     bhp=d["bhp0"].copy())
    ref = oadj.jac_wrt_previous(prob, st0o, dt).T @ lam
    np.testing.assert_allclose(y.cpu().numpy(), ref, rtol=1e-12, atol=1e-14 * np.abs(ref).max())


def test_checkpointed_sweep_equals_the_stored_state_sweep():
    """Checkpoints every 2 steps with recomputed segments give the gradients
    of the sweep over stored states; the recomputed states equal the forward
    run's (the model's aggregates are kept for the run)."""
    d = load("adjoint_grav.npz")
    g, rock, fluid, wells = ow_case(d)
    m = GpuOilWaterModel(g, rock, fluid, wells, gravity=float(d["gravity"]),
                         cpr_options=dict(rtol=1e-12, maxiter=400, amg_rebuild_interval=1_000_000))
    st0 = OWState(pressure=d["p0"].copy(), sW=d["sw0"].copy(), qWs=d["qws0"].copy(), qOs=d["qos0"].copy(),
                  bhp=d["bhp0"].copy())
    a = compute_gradient_adjoint(m, st0, d["dts"], d["controls"], npv_objective(), perm_gradient=True,
                                 checkpoint_every=2)
    assert a.stats["recomputed_steps"] > 0 and a.stats["recompute_max_rel_diff"] == 0.0
    m2 = GpuOilWaterModel(g, rock, fluid, wells, gravity=float(d["gravity"]),
                          cpr_options=dict(rtol=1e-12, maxiter=400, amg_rebuild_interval=1_000_000))
    b = compute_gradient_adjoint(m2, st0, d["dts"], d["controls"], npv_objective(), perm_gradient=True,
                                 states=a.states)
    assert a.value == b.value
    np.testing.assert_allclose(a.gradient, b.gradient, rtol=1e-10, atol=1e-14 * np.abs(b.gradient).max())
    np.testing.assert_allclose(a.perm_gradient, b.perm_gradient, rtol=1e-10,
                               atol=1e-14 * np.abs(b.perm_gradient).max())


def test_adjoint_at_64x64x4_matches_reference_over_30_steps():
    """Benchmark config 4: the 16,384-cell five-spot, 30 steps of 10 days,
    cumulative produced oil, controls held at the wells' targets; value and
    control gradients against the reference's compute_gradient_adjoint."""
    from pymrst_b200 import cases
    d = load("cfg4_adjoint_64x64x4.npz")
    c = cases.five_spot(dims=(64, 64, 4), seed=4, nsteps=30)
    assert np.isclose(np.sum(c.rock.perm), float(d["perm_sum"]), rtol=1e-14)
    m = GpuOilWaterModel(c.grid, c.rock, c.fluid, c.wells, gravity=c.gravity,
                         cpr_options=dict(rtol=1e-12, maxiter=400, amg_rebuild_interval=1_000_000))
    obj = npv_objective(oil_price=1.0, water_cost=0.0, water_inj_cost=0.0)
    res = compute_gradient_adjoint(m, m.initial_state(c.p0, c.sw0), d["dts"], d["controls"], obj)
    assert abs(res.value - float(d["value"])) <= 1e-8 * abs(float(d["value"]))
    for j in range(d["gradient"].shape[1]):
        ref = d["gradient"][:, j]
        assert np.abs(res.gradient[:, j] - ref).max() <= 1e-6 * np.abs(ref).max(), j
    assert np.abs(res.states[-1].pressure - d["p_final"]).max() <= 1e-8 * np.abs(d["p_final"]).max()
    assert np.abs(res.states[-1].sW - d["sw_final"]).max() <= 1e-7
