"""The reference's own drivers and models with this package's GPU pieces
plugged in, through the reference's public objects, against the reference's
own Newton histories (ow_newton_grav.npz: 8 x 6 x 4 cells with gravity, four
10-day steps, made by the reference's TwoPhaseOilWaterModelAD and
simulate_schedule_ad with its direct solver):

* the reference's TwoPhaseOilWaterModelAD with `linear_solver=GpuCPRSolver()`,
  driven by the reference's simulate_schedule_ad;
* GpuOilWaterModel, built from the reference's grid, rock, fluid and wells,
  driven by the reference's simulate_schedule_ad (its `step`);
* GpuOilWaterModel driven by the reference's legacy NonLinearSolver through
  get_equations / get_convergence / update_state, with the solver's own
  direct solve and with GpuCPRSolver.

The reference package comes from its install under baseline/_ref; the module
is skipped where that install is absent."""

import sys
from pathlib import Path

import numpy as np
import pytest
import scipy.sparse as sp

from fixtures import load

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

REF = Path(__file__).resolve().parents[1] / "baseline" / "_ref"
if not (REF / "pymrst").is_dir():
    pytest.skip("the reference package is not installed under baseline/_ref", allow_module_level=True)
sys.path.insert(0, str(REF))

from pymrst.gridprocessing import cart_grid, compute_geometry  # noqa: E402
from pymrst.modules.ad_blackoil import TwoPhaseOilWaterModelAD  # noqa: E402
from pymrst.modules.ad_core import simulate_schedule_ad  # noqa: E402
from pymrst.modules.ad_core.simulators.nonlinear_solver import NonLinearSolver  # noqa: E402
from pymrst.modules.ad_props import init_simple_adi_fluid  # noqa: E402
from pymrst.params import add_well, make_rock  # noqa: E402
from pymrst.utils.adi import combine_equations  # noqa: E402
from pymrst.utils.units import BARSA, CENTI, DAY, POISE  # noqa: E402

from pymrst_b200.build import build  # noqa: E402
from pymrst_b200.linear_solvers import GpuCPRSolver  # noqa: E402
from pymrst_b200.ow_model import GpuOilWaterModel  # noqa: E402

build()


def _reference_case():
    """The fixture's model, built from the reference's own constructors (as
    tests/golden/make_golden.py's newton_fixture builds it)."""
    d = load("ow_newton_grav.npz")
    dims = [int(v) for v in d["dims"]]
    g = compute_geometry(cart_grid(dims, [float(v) for v in d["phys"]]))
    rock = make_rock(g, d["perm"][:, None], 0.2)
    fluid = init_simple_adi_fluid(mu=np.array([1.0, 5.0]) * CENTI * POISE, rho=[1000.0, 800.0], n=[2, 2],
                                  c=[1e-5 / BARSA, 1e-5 / BARSA], p_ref=200 * BARSA, smin=[0.1, 0.1])
    nx, ny, nz = dims
    col = lambda i, j: i + nx * (j + ny * np.arange(nz))
    grav = float(d["gravity"])
    gvec = np.array([0, 0, grav])
    nsteps, dt_days = int(d["nsteps"]), float(d["dt_days"])
    rate = 0.25 * float(np.sum(0.2 * g.cells.volumes)) / (nsteps * dt_days * DAY) / 2
    w = add_well(None, g, rock, col(0, 0), well_type="rate", val=rate, compi=np.array([1.0, 0.0]), sign=1,
                 gravity=gvec)
    w = add_well(w, g, rock, col(nx - 1, 0), well_type="rate", val=rate, compi=np.array([1.0, 0.0]), sign=1,
                 gravity=gvec)
    w = add_well(w, g, rock, col(nx // 2, ny - 1), well_type="bhp", val=150 * BARSA, compi=np.array([0.0, 1.0]),
                 sign=-1, gravity=gvec)
    return d, g, rock, fluid, w, grav, np.full(nsteps, dt_days * DAY)


def _check_history(d, states, its):
    assert list(np.asarray(its)) == list(d["its"])
    for k, st in enumerate(states):
        p, sw = np.asarray(st.pressure), np.asarray(st.sW)
        assert np.abs(p - d["p_hist"][k]).max() <= 1e-8 * np.abs(d["p_hist"][k]).max()
        assert np.abs(sw - d["sw_hist"][k]).max() <= 1e-7


def test_reference_model_with_the_gpu_linear_solver():
    d, g, rock, fluid, w, grav, dts = _reference_case()
    model = TwoPhaseOilWaterModelAD(g, rock, fluid, w, gravity=grav, linear_solver=GpuCPRSolver(rtol=1e-12))
    states, its = simulate_schedule_ad(model.initial_state(200 * BARSA, 0.1), model, dts, verbose=False)
    _check_history(d, states, its)


def test_reference_driver_runs_the_gpu_model():
    d, g, rock, fluid, w, grav, dts = _reference_case()
    model = GpuOilWaterModel(g, rock, fluid, w, gravity=grav, cpr_options=dict(rtol=1e-12, maxiter=400))
    states, its = simulate_schedule_ad(model.initial_state(200 * BARSA, 0.1), model, dts, verbose=False)
    _check_history(d, states, its)


@pytest.mark.parametrize("solver", ["direct", "gpu_cpr"])
def test_reference_nonlinear_solver_drives_the_gpu_model(solver):
    d, g, rock, fluid, w, grav, dts = _reference_case()
    model = GpuOilWaterModel(g, rock, fluid, w, gravity=grav)
    nls = NonLinearSolver(max_iterations=25, verbose=False,
                          linear_solver=None if solver == "direct" else GpuCPRSolver(rtol=1e-12))
    states, report = nls.simulate_schedule(model, model.initial_state(200 * BARSA, 0.1), dts)
    assert all(r.converged for r in report.steps)
    _check_history(d, states, [r.iterations for r in report.steps])


@pytest.mark.parametrize("kind", ["LinearizedProblem", "LinearizedProblemAD"])
def test_reference_linearized_problem_solved_by_the_gpu_solver(kind):
    """solve_linear_problem on the reference's own problem objects built from
    the GPU model's equations (MRST's LinearizedProblem, whose b is the
    right-hand side, and LinearizedProblemAD, which stores the residual):
    the increments per primary variable equal a direct solve."""
    import scipy.sparse.linalg as spla
    from pymrst.modules.ad_core.solvers.linear_solver_ad import LinearizedProblemAD
    from pymrst.modules.ad_core.solvers.linearized_problem import LinearizedProblem
    d, g, rock, fluid, w, grav, dts = _reference_case()
    model = GpuOilWaterModel(g, rock, fluid, w, gravity=grav)
    st0 = model.initial_state(200 * BARSA, 0.1)
    st = st0.copy()
    st.pressure = st.pressure + np.linspace(0.0, 5.0 * BARSA, st.pressure.size)
    eqs = model.get_equations(st0, st, float(dts[0]))
    names = ["water", "oil", "waterWells", "oilWells", "closure"]
    types = ["cell", "cell", "well", "well", "well"]
    pvars = ["pressure", "sW", "qWs", "qOs", "bhp"]
    state = {"pressure": st.pressure}
    if kind == "LinearizedProblem":
        problem = LinearizedProblem(eqs, types, names, pvars, state, float(dts[0]))
    else:
        problem = LinearizedProblemAD.from_equations(eqs, types, names, pvars, state, float(dts[0]))
    dx, result, report = GpuCPRSolver(rtol=1e-12).solve_linear_problem(problem, model)
    A = combine_equations(*eqs)
    ref = spla.spsolve(A.jac[0].tocsc(), -A.val)
    assert np.abs(result - ref).max() <= 1e-7 * np.abs(ref).max()
    assert [x.size for x in dx] == [model.nc, model.nc, model.nw, model.nw, model.nw]
    assert report["Iterations"] > 0


def test_reference_adoo_simulation_with_the_gpu_cpr_solver_ad():
    """The reference's AD-OO oil-water model (its own equations through its
    FacilityModel) and AD-OO simulate_schedule_ad, with GpuCPRSolverAD as the
    linear solver: the same Newton iterations per step and the same states
    (p 1e-8, sW 1e-7) as with the reference's direct solver."""
    from pymrst.modules.ad_blackoil.models.two_phase_oil_water_model import TwoPhaseOilWaterModel
    from pymrst.modules.ad_core.ad_oo.simulate_schedule_ad import simulate_schedule_ad as sim_adoo
    from pymrst.modules.ad_core.solvers.concrete_solvers import BackslashSolverAD
    from pymrst.modules.ad_core.utils.schedule import simple_schedule
    from pymrst.params.wells_and_bc.vertical_well import vertical_well
    from pymrst.solvers.init_res_sol import init_res_sol
    from pymrst.utils.units import DARCY, MILLI
    from pymrst_b200.linear_solvers import GpuCPRSolverAD
    G = compute_geometry(cart_grid([10, 8, 3], [100.0, 80.0, 6.0]))
    rng = np.random.default_rng(0)
    rock = make_rock(G, np.exp(rng.normal(np.log(100), 0.5, G.cells.num))[:, None] * MILLI * DARCY, 0.2)
    fluid = init_simple_adi_fluid(mu=np.array([1, 5]) * CENTI * POISE, rho=np.array([1000.0, 800.0]), n=[2, 2],
                                  c=[1e-5 / BARSA, 1e-5 / BARSA], p_ref=200 * BARSA, phases="wo")
    rate = 0.2 * float(np.sum(0.2 * G.cells.volumes)) / (100 * DAY)
    W = vertical_well([], G, rock, 0, 0, None, val=rate, well_type="rate", compi=np.array([1.0, 0.0]), name="I")
    W = vertical_well(W, G, rock, 9, 7, None, val=150 * BARSA, well_type="bhp", compi=np.array([0.0, 1.0]),
                      name="P")
    schedule = simple_schedule(np.full(3, 10 * DAY), W=W)
    runs = {}
    for name, ls in (("direct", BackslashSolverAD()), ("gpu", GpuCPRSolverAD(tolerance=1e-12))):
        model = TwoPhaseOilWaterModel(G, rock, fluid)
        _, states, rep = sim_adoo(init_res_sol(G, 200 * BARSA, np.array([0.1, 0.9])), model, schedule,
                                  LinearSolver=ls)
        runs[name] = (states, [r["Iterations"] for r in rep["ControlstepReports"]])
    (sd, itd), (sg, itg) = runs["direct"], runs["gpu"]
    assert itd == itg
    for a, b in zip(sg, sd):
        pa, pb = np.asarray(a["pressure"]), np.asarray(b["pressure"])
        assert np.abs(pa - pb).max() <= 1e-8 * np.abs(pb).max()
        assert np.abs(np.asarray(a["s"])[:, 0] - np.asarray(b["s"])[:, 0]).max() <= 1e-7


def _adoo_case(gravity_on):
    from pymrst.modules.ad_blackoil.models.two_phase_oil_water_model import TwoPhaseOilWaterModel
    from pymrst.modules.ad_core.utils.schedule import simple_schedule
    from pymrst.params.wells_and_bc.vertical_well import vertical_well
    from pymrst.solvers.init_res_sol import init_res_sol
    from pymrst.utils.units import DARCY, MILLI
    G = compute_geometry(cart_grid([10, 8, 3], [100.0, 80.0, 6.0]))
    rng = np.random.default_rng(0)
    rock = make_rock(G, np.exp(rng.normal(np.log(100), 0.5, G.cells.num))[:, None] * MILLI * DARCY, 0.2)
    fluid = init_simple_adi_fluid(mu=np.array([1, 5]) * CENTI * POISE, rho=np.array([1000.0, 800.0]), n=[2, 2],
                                  c=[1e-5 / BARSA, 1e-5 / BARSA], p_ref=200 * BARSA, phases="wo")
    rate = 0.2 * float(np.sum(0.2 * G.cells.volumes)) / (100 * DAY)
    W = vertical_well([], G, rock, 0, 0, None, val=rate, well_type="rate", compi=np.array([1.0, 0.0]), name="I")
    W = vertical_well(W, G, rock, 9, 7, None, val=150 * BARSA, well_type="bhp", compi=np.array([0.0, 1.0]),
                      name="P")
    schedule = simple_schedule(np.full(3, 10 * DAY), W=W)

    def model():
        m = TwoPhaseOilWaterModel(G, rock, fluid)
        if gravity_on:
            m.gravity = np.array([0.0, 0.0, 9.80665])
        return m
    return G, model, schedule, init_res_sol(G, 200 * BARSA, np.array([0.1, 0.9]))


@pytest.mark.parametrize("gravity_on", [False, True])
def test_adoo_model_with_device_cell_equations(gravity_on):
    """The reference's AD-OO oil-water model with its cell equations from
    the device (use_device_cell_equations): one get_equations call gives the
    reference's equations (values and every Jacobian block to 1e-12 of the
    block's largest entry), and the reference's AD-OO simulate_schedule_ad
    with its direct solver takes the same Newton iterations to the same
    states as with the reference's own equations."""
    from pymrst.modules.ad_core.ad_oo.simulate_schedule_ad import simulate_schedule_ad as sim_adoo
    from pymrst.modules.ad_core.solvers.concrete_solvers import BackslashSolverAD
    from pymrst_b200.adoo import use_device_cell_equations
    G, model, schedule, init = _adoo_case(gravity_on)
    runs = {}
    for name in ("reference", "device"):
        m = model() if name == "reference" else use_device_cell_equations(model())
        _, states, rep = sim_adoo(init, m, schedule, LinearSolver=BackslashSolverAD())
        runs[name] = (m, states, [r["Iterations"] for r in rep["ControlstepReports"]])
    (mr, sr, ir), (md, sd, idev) = runs["reference"], runs["device"]
    assert ir == idev
    for a, b in zip(sd, sr):
        pa, pb = np.asarray(a["pressure"]), np.asarray(b["pressure"])
        assert np.abs(pa - pb).max() <= 1e-9 * np.abs(pb).max()
        assert np.abs(np.asarray(a["s"])[:, 0] - np.asarray(b["s"])[:, 0]).max() <= 1e-9
    # one call at a perturbed mid-run state, the facility model prepared for
    # the control step as the reference's nonlinear solver prepares it
    from pymrst.modules.ad_core.ad_oo.physical_model import copy_state
    base = model()
    forces = dict(base.get_valid_driving_forces())
    forces.update(base.get_driving_forces(schedule.controls[0]))

    def prepared(mm):
        mm = mm.validate_model(forces)
        st = copy_state(sr[1])
        st["pressure"] = np.asarray(st["pressure"]) + np.linspace(-2.0, 2.0, G.cells.num) * BARSA
        mm, st = mm.prepare_report_step(st, sr[0], 10 * DAY, forces)
        mm, st = mm.prepare_timestep(st, sr[0], 10 * DAY, forces)
        return mm, st
    mr, st_r = prepared(model())
    md, st_d = prepared(use_device_cell_equations(model()))
    pr, _ = mr.get_equations(sr[0], st_r, 10 * DAY, forces, iteration=1)
    pd, _ = md.get_equations(sr[0], st_d, 10 * DAY, forces, iteration=1)
    assert pr.equationNames == pd.equationNames and pr.primaryVariables == pd.primaryVariables
    for er, ed in zip(pr.equations, pd.equations):
        vr, vd = np.asarray(er.val), np.asarray(ed.val)
        assert np.abs(vr - vd).max() <= 1e-12 * max(np.abs(vr).max(), 1e-300)
        for jr, jd in zip(er.jac, ed.jac):
            jr, jd = sp.csr_array(jr), sp.csr_array(jd)
            scale = abs(jr).max() if jr.nnz else 1.0
            assert (abs(jr - jd).max() if (jr - jd).nnz else 0.0) <= 1e-12 * max(scale, 1e-300)
