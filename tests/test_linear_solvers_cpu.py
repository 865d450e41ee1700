"""Host logic of the drop-in CPR solver (no GPU needed): the reference's
constructor validation and model contract (linear_solvers.py:113-140,
396-424), the decoupling weights (:155-190), and the C-ABI's pattern checks,
which reject a bad matrix before any device work."""

from types import SimpleNamespace

import numpy as np
import pytest

from pymrst_b200 import _native as N
from pymrst_b200.build import build
from pymrst_b200.grid import cartesian_grid
from pymrst_b200.linear_solvers import GpuCPRSolver
from pymrst_b200.params import BARSA, CENTI, POISE, init_simple_adi_fluid


@pytest.fixture(scope="module")
def lib():
    build()
    return N.lib()


def _fluid():
    return init_simple_adi_fluid(mu=np.array([1.0, 5.0]) * CENTI * POISE, rho=[1000.0, 800.0], n=[2, 2],
                                 c=[1e-5 / BARSA, 1e-4 / BARSA], p_ref=200 * BARSA)


@pytest.mark.parametrize("kwargs,match", [
    (dict(local_stage="lu"), "unknown local_stage"),
    (dict(local_stage="ilu"), "no ILU"),
    (dict(amg_rebuild_interval=0), "amg_rebuild_interval"),
    (dict(amg_cycles=2), "amg_cycles"),
    (dict(elliptic_solver=object()), "elliptic_solver"),
    (dict(precision="fp16"), "precision"),
    (dict(restart=61), "restart"),
])
def test_constructor_rejects_what_the_device_path_cannot_do(kwargs, match):
    with pytest.raises(ValueError, match=match):
        GpuCPRSolver(**kwargs)


def test_reference_defaults():
    s = GpuCPRSolver()
    assert (s.rtol, s.maxiter, s.restart, s.amg_rebuild_interval) == (1e-8, 200, 50, 8)
    assert s.last_iterations == 0 and s.last_local_stage is None


def test_missing_model_contract_is_loud():
    g = cartesian_grid([3, 2, 1], [3.0, 2.0, 1.0])
    J = np.eye(12)
    with pytest.raises(ValueError, match="no model was supplied"):
        GpuCPRSolver().solve(J, np.ones(12))
    with pytest.raises(ValueError, match=r"has no \.G.*it has \.g"):
        GpuCPRSolver().solve(J, np.ones(12), SimpleNamespace(g=g, fluid=_fluid(), n_phases=2))
    with pytest.raises(ValueError, match=r"fluid has no \.b"):
        GpuCPRSolver().solve(J, np.ones(12), SimpleNamespace(G=g, fluid=SimpleNamespace(disgas=False, vapoil=False),
                                                             n_phases=2))


def test_weights_are_inverse_shrinkage_at_mean_pressure():
    fl = _fluid()
    model = SimpleNamespace(G=None, fluid=fl, n_phases=2)
    p = np.array([150.0, 210.0, 240.0]) * BARSA
    w = GpuCPRSolver.weights(model, {"pressure": p})
    pm = p.mean()
    expect = [1.0 / float(fl.b_w(np.array([pm]))[0]), 1.0 / float(fl.b_o(np.array([pm]))[0])]
    np.testing.assert_allclose(w, expect, rtol=1e-15)
    # attribute-style states work too
    w2 = GpuCPRSolver.weights(model, SimpleNamespace(pressure=p))
    np.testing.assert_array_equal(w, w2)


def _create(lib, n, nc, nph, rp, ci):
    o = N.CPROpts()
    N.check(lib.pmb_cpr_default_opts(N.C.byref(o)))
    h = N.c_vp()
    rp = np.asarray(rp, dtype=np.int32)
    ci = np.asarray(ci, dtype=np.int32)
    rc = lib.pmb_csr_cpr_create(n, nc, nph, N.as_p(rp, N.C.c_int32), N.as_p(ci, N.C.c_int32), 0, N.C.byref(o),
                                None, N.C.byref(h))
    return rc, lib.pmb_last_error().decode()


def test_csr_create_rejects_bad_patterns(lib):
    rc, msg = _create(lib, 2, 1, 2, [0, 2, 3], [1, 0, 1])
    assert rc == 2 and "strictly increasing" in msg
    rc, msg = _create(lib, 2, 1, 2, [0, 1, 2], [0, 5])
    assert rc == 2 and "out of range" in msg
    rc, msg = _create(lib, 3, 2, 2, [0, 1, 2, 3], [0, 1, 2])
    assert rc == 2 and "nph * nc" in msg
    rc, msg = _create(lib, 4, 1, 4, [0, 1, 2, 3, 4], [0, 1, 2, 3])
    assert rc == 2 and "nph must be" in msg


def test_linearized_problem_assembly_sign_and_increment_split():
    """The AD-OO protocol's host logic: a LinearizedProblemAD stores the
    residual (its right-hand side is -b), MRST's LinearizedProblem the
    right-hand side itself; the solution splits by the first equation's
    Jacobian block widths."""
    from types import SimpleNamespace

    import scipy.sparse as sp
    from pymrst_b200.linear_solvers import GpuCPRSolver

    class LinearizedProblem:
        def __init__(self, eqs):
            self.equations = eqs
            self.A = None
            self.b = None
            self.num_vars = None

        def assemble_system(self):
            self.A = sp.bmat([[sp.csr_array(j) for j in e.jac] for e in self.equations], format="csr")
            self.b = np.concatenate([e.val for e in self.equations])
            return self

    class LinearizedProblemAD(LinearizedProblem):
        pass

    eqs = [SimpleNamespace(val=np.array([1.0, 2.0]), jac=[np.eye(2), np.zeros((2, 1))]),
           SimpleNamespace(val=np.array([3.0]), jac=[np.zeros((1, 2)), np.ones((1, 1))])]
    _, A, b = GpuCPRSolver._assembled_system(LinearizedProblem(eqs))
    assert A.shape == (3, 3) and np.array_equal(b, [1.0, 2.0, 3.0])
    _, _, b = GpuCPRSolver._assembled_system(LinearizedProblemAD(eqs))
    assert np.array_equal(b, [-1.0, -2.0, -3.0])
    parts = GpuCPRSolver.store_increments(LinearizedProblem(eqs), np.arange(3.0))
    assert [p.tolist() for p in parts] == [[0.0, 1.0], [2.0]]


def _reference_adoo_problem():
    """A linearized problem of the reference's AD-OO oil-water model (its own
    get_equations through its FacilityModel), from the reference package
    installed under baseline/_ref; skipped where that install is absent."""
    import sys
    from pathlib import Path
    ref = Path(__file__).resolve().parents[1] / "baseline" / "_ref"
    if not (ref / "pymrst").is_dir():
        pytest.skip("the reference package is not installed under baseline/_ref")
    if str(ref) not in sys.path:
        sys.path.insert(0, str(ref))
    from pymrst.gridprocessing import cart_grid, compute_geometry
    from pymrst.modules.ad_blackoil.models.two_phase_oil_water_model import TwoPhaseOilWaterModel
    from pymrst.modules.ad_core.utils.schedule import simple_schedule
    from pymrst.modules.ad_props import init_simple_adi_fluid as ref_fluid
    from pymrst.params import make_rock
    from pymrst.params.wells_and_bc.vertical_well import vertical_well
    from pymrst.solvers.init_res_sol import init_res_sol
    from pymrst.utils.units import BARSA as B, CENTI as C_, DARCY, DAY, MILLI, POISE as P_
    G = compute_geometry(cart_grid([10, 8, 3], [100.0, 80.0, 6.0]))
    rng = np.random.default_rng(0)
    rock = make_rock(G, np.exp(rng.normal(np.log(100), 0.5, G.cells.num))[:, None] * MILLI * DARCY, 0.2)
    fluid = ref_fluid(mu=np.array([1, 5]) * C_ * P_, rho=np.array([1000.0, 800.0]), n=[2, 2],
                      c=[1e-5 / B, 1e-5 / B], p_ref=200 * B, phases="wo")
    rate = 0.2 * float(np.sum(0.2 * G.cells.volumes)) / (100 * DAY)
    W = vertical_well([], G, rock, 0, 0, None, val=rate, well_type="rate", compi=np.array([1.0, 0.0]), name="I")
    W = vertical_well(W, G, rock, 9, 7, None, val=150 * B, well_type="bhp", compi=np.array([0.0, 1.0]), name="P")
    schedule = simple_schedule(np.full(1, 10 * DAY), W=W)
    model = TwoPhaseOilWaterModel(G, rock, fluid)
    state = init_res_sol(G, 200 * B, np.array([0.1, 0.9]))
    forces = model.get_driving_forces(schedule.controls[0])
    model = model.validate_model(forces)
    state = model.validate_state(state)
    dt = float(schedule.step_val[0])
    model, st = model.prepare_timestep(state, state, dt, forces)
    model.FacilityModel = model.FacilityModel.validate_model(forces)
    model, st = model.prepare_report_step(st, state, dt, forces)
    model, st = model.prepare_timestep(st, state, dt, forces)
    st["pressure"] = st["pressure"] + np.linspace(0.0, 3.0 * B, G.cells.num)
    problem, _ = model.get_equations(state, st, dt, forces, iteration=1)
    return model, problem


def test_cpr_ad_decoupling_keeps_the_solution_of_the_reference_problem():
    """GpuCPRSolverAD's dynamic row-sum decoupling is an invertible row
    transformation (plus a pressure column scaling): solving the decoupled
    system gives the increments of the reference problem's own direct solve
    and of the reference's CPRSolverAD."""
    import scipy.sparse.linalg as spla
    model, problem = _reference_adoo_problem()
    from pymrst.modules.ad_core.solvers.concrete_solvers import BackslashSolverAD
    from pymrst.modules.ad_core.solvers.cpr_solver_ad import CPRSolverAD
    from pymrst_b200.linear_solvers import GpuCPRSolverAD
    A, b, colscale, widths, p, ncell, nc = GpuCPRSolverAD().decoupled_system(problem, model)
    assert p == 0 and ncell == 2 and A.shape[0] == sum(widths)
    x = spla.spsolve(A.tocsc(), b) * colscale
    _, ref, _ = BackslashSolverAD().solve_linear_problem(problem, model)
    np.testing.assert_allclose(x, ref, rtol=1e-9, atol=1e-12 * np.abs(ref).max())
    _, ref_cpr, _ = CPRSolverAD(tolerance=1e-12, maxIterations=200).solve_linear_problem(problem, model)
    np.testing.assert_allclose(x, ref_cpr, rtol=1e-6, atol=1e-9 * np.abs(ref).max())
