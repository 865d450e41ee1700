"""GPU parity of the oil-water path against the reference's own outputs
(golden fixtures) and the CPU oracle.

Tolerances: residuals and Jacobians 1e-12 (blockwise relative, as in the
oracle pin); states after each timestep p <= 1e-8 relative to the field
maximum and sW <= 1e-7 absolute, with the CPR-GMRES tolerance tightened to
1e-12 so that the Newton paths coincide.
"""

import numpy as np
import pytest
import scipy.sparse as sp

from compare import blockwise_error, ow_splits, segment_error
from fixtures import load, ow_case, ow_fluid, wells_from

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from pymrst_b200 import cases  # noqa: E402
from pymrst_b200.build import build  # noqa: E402
from pymrst_b200.grid import cartesian_grid  # noqa: E402
from pymrst_b200.ow_model import GpuOilWaterModel, OWState, face_transmissibility_device  # noqa: E402
from pymrst_b200.params import add_well, make_rock  # noqa: E402
from pymrst_b200.schedule import simulate_schedule_ad  # noqa: E402

from oracle import ow as oow  # noqa: E402

build()

TIGHT = dict(rtol=1e-12, maxiter=400)


def _state(d, sfx=""):
    return OWState(pressure=d["p" + sfx].copy(), sW=d["sw" + sfx].copy(), qWs=d["qws" + sfx].copy(),
                   qOs=d["qos" + sfx].copy(), bhp=d["bhp" + sfx].copy())


def test_device_transmissibilities_match_reference():
    d = load("grid_trans.npz")
    g = cartesian_grid([4, 3, 2], [40.0, 30.0, 4.0])
    for key, permkey in (("1", "perm"), ("3", "perm3")):
        perm = d[permkey]
        rock = make_rock(g, perm[:, None] if perm.ndim == 1 else perm, 0.2)
        tf, th = face_transmissibility_device(g, rock)
        np.testing.assert_allclose(th, d["hT" + key], rtol=1e-13)
        np.testing.assert_allclose(tf, d["T" + key], rtol=1e-13)


@pytest.mark.parametrize("name", ["ow_assemble_nograv.npz", "ow_assemble_grav.npz", "ow_assemble_xflow.npz"])
def test_residual_jacobian_cdp_match_reference(name):
    d = load(name)
    g, rock, fluid, wells = ow_case(d)
    m = GpuOilWaterModel(g, rock, fluid, wells, gravity=float(d["gravity"]))
    np.testing.assert_allclose(m.T, d["T"], rtol=1e-13)
    st0, st = _state(d, "0"), _state(d)
    cdp = m.compute_cdp(st0)
    np.testing.assert_allclose(np.concatenate(cdp), d["cdp"], rtol=1e-12, atol=1e-9)
    res, J = m.residual_and_jacobian(st0, st, float(d["dt"]), cdp)
    splits = ow_splits(m.nc, m.nw)
    assert segment_error(res, d["res"], splits) < 1e-12
    Jref = sp.csr_array((d["J_data"], d["J_indices"], d["J_indptr"]), shape=tuple(d["J_shape"]))
    assert blockwise_error(J, Jref, splits) < 1e-12


def test_assembly_is_bit_reproducible_and_spmv_matches_the_exported_matrix():
    d = load("ow_assemble_xflow.npz")
    g, rock, fluid, wells = ow_case(d)
    m = GpuOilWaterModel(g, rock, fluid, wells, gravity=float(d["gravity"]))
    x = m.to_device(_state(d))
    x0 = m.to_device(_state(d, "0"))
    cdp = torch.as_tensor(d["cdp"], device="cuda")
    r1, j1, w1 = m.assemble_device(x, x0, float(d["dt"]), cdp)
    r2, j2, w2 = m.assemble_device(x, x0, float(d["dt"]), cdp)
    assert torch.equal(r1, r2) and torch.equal(j1, j2) and torch.equal(w1, w2)
    J = m.export_jacobian(j1.cpu().numpy(), w1.cpu().numpy())
    rng = np.random.default_rng(0)
    v = rng.standard_normal(m.sizes["nvec"])
    y = torch.empty_like(x)
    from pymrst_b200 import _native as N
    dv = torch.as_tensor(v, device="cuda")
    N.check(N.lib().pmb_ow_spmv(m._handle, N.ptr(j1), N.ptr(w1), N.ptr(dv), N.ptr(y)))
    # export is in the reference layout: permute v and y
    vref = m.export_residual(v)
    yref = J @ vref
    yd = m.export_residual(y.cpu().numpy())
    assert np.abs(yd - yref).max() <= 1e-12 * np.abs(yref).max()


def test_cpr_gmres_solves_the_reference_jacobian():
    d = load("ow_assemble_grav.npz")
    g, rock, fluid, wells = ow_case(d)
    m = GpuOilWaterModel(g, rock, fluid, wells, gravity=float(d["gravity"]), cpr_options=dict(rtol=1e-10))
    x = m.to_device(_state(d))
    x0 = m.to_device(_state(d, "0"))
    cdp = torch.as_tensor(d["cdp"], device="cuda")
    res, jac, well = m.assemble_device(x, x0, float(d["dt"]), cdp)
    from pymrst_b200 import _native as N
    s = m.solver_handle()
    N.check(N.lib().pmb_cpr_setup(s, N.ptr(jac), N.ptr(well), N.ptr(x)))
    dx = torch.empty_like(res)
    info = (N.C.c_double * 4)()
    N.check(N.lib().pmb_cpr_solve(s, N.ptr(res), N.ptr(dx), info))
    J = m.export_jacobian(jac.cpu().numpy(), well.cpu().numpy())
    r = m.export_residual(res.cpu().numpy())
    ref = sp.linalg.spsolve(J.tocsc(), r)
    got = m.export_residual(dx.cpu().numpy())
    assert info[2] == 1.0 and info[1] <= 1e-10
    assert np.abs(got - ref).max() <= 1e-6 * np.abs(ref).max()


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("name", ["ow_newton_grav.npz", "ow_newton_nograv.npz"])
def test_newton_history_matches_reference(name, precision):
    d = load(name)
    g, rock, fluid, wells = ow_case(d)
    m = GpuOilWaterModel(g, rock, fluid, wells, gravity=float(d["gravity"]),
                         cpr_options=dict(TIGHT, precision=precision))
    st0 = m.initial_state(float(d["p0"][0]), float(d["sw0"][0]))
    states, its = simulate_schedule_ad(st0, m, np.full(int(d["nsteps"]), float(d["dt_days"]) * 86400.0),
                                       verbose=False)
    np.testing.assert_array_equal(its, d["its"])
    for k, s in enumerate(states):
        assert np.abs(s.pressure - d["p_hist"][k]).max() <= 1e-8 * np.abs(d["p_hist"][k]).max()
        assert np.abs(s.sW - d["sw_hist"][k]).max() <= 1e-7
        np.testing.assert_allclose(s.bhp, d["bhp_hist"][k], rtol=1e-8)


def test_phase5_matches_reference_and_matlab():
    d = load("ow_phase5.npz")
    g = cartesian_grid([15, 15, 1], [300.0, 300.0, 10.0])
    rock = make_rock(g, d["perm"][:, None], 0.25)
    w = add_well(None, g, rock, np.array([0]), well_type="rate", val=2e-3, compi=np.array([1.0, 0.0]), sign=1)
    w = add_well(w, g, rock, np.array([g.cells.num - 1]), well_type="bhp", val=150e5,
                 compi=np.array([0.0, 1.0]), sign=-1)
    m = GpuOilWaterModel(g, rock, ow_fluid("p5"), w, cpr_options=TIGHT)
    states, its = simulate_schedule_ad(m.initial_state(200e5, 0.2), m, np.full(8, 30.0 * 86400.0),
                                       verbose=False)
    np.testing.assert_array_equal(its, d["its"])
    p = np.vstack([s.pressure for s in states])
    sw = np.vstack([s.sW for s in states])
    assert np.abs(p - d["p_hist"]).max() <= 1e-8 * np.abs(d["p_hist"]).max()
    assert np.abs(sw - d["sw_hist"]).max() <= 1e-7
    assert np.abs(p - d["mat_p_hist"]).max() <= 5e-6 * np.abs(d["mat_p_hist"]).max()
    assert np.abs(sw.ravel() - d["mat_sw_hist"].ravel()).max() <= 5e-6 * np.abs(d["mat_sw_hist"]).max()


@pytest.mark.parametrize("precision", [0, 1])
def test_five_spot_step_matches_oracle(precision):
    case = cases.five_spot(dims=(16, 14, 4), nsteps=4, dt_days=10.0)
    m = GpuOilWaterModel(case.grid, case.rock, case.fluid, case.wells, gravity=case.gravity,
                         cpr_options=dict(TIGHT, precision=precision))
    prob = oow.build_problem(case.grid, case.rock, case.fluid.params, case.wells, gravity=case.gravity)
    st_o = oow.initial_state(prob, case.p0, case.sw0)
    st_g = m.initial_state(case.p0, case.sw0)
    for _ in range(2):
        st_o, ok_o, it_o = oow.step(prob, st_o, case.dt)
        st_g, ok_g, it_g = m.step(st_g, case.dt)
        assert ok_o and ok_g and it_o == it_g
        assert np.abs(st_g.pressure - st_o.pressure).max() <= 1e-8 * np.abs(st_o.pressure).max()
        assert np.abs(st_g.sW - st_o.sW).max() <= 1e-7


def test_nonfinite_state_fails_the_step_without_a_device_fault():
    case = cases.five_spot(dims=(8, 8, 2), nsteps=2)
    m = GpuOilWaterModel(case.grid, case.rock, case.fluid, case.wells, gravity=case.gravity)
    st = m.initial_state(case.p0, case.sw0)
    st.pressure[3] = np.nan
    new, ok, its = m.step(st, case.dt)
    assert not ok
    # the handle is still usable afterwards
    new, ok, its = m.step(m.initial_state(case.p0, case.sw0), case.dt)
    assert ok


def test_config1_first_step_matches_reference_at_100x100x10():
    """Benchmark config 1 at its own size: the 100,000-cell five-spot with
    gravity, the first 10-day report step under the schedule driver (the
    reference's timestep cuts), against the reference's own
    simulate_schedule_ad with its direct solver (cfg1_ow_100x100x10.npz).
    The reference needs 83 Newton iterations over five ministeps (10 and 5
    days rejected after 25 iterations each, then 2.5, 5 and 2.5 days);
    an iterative solve to rtol 1e-12 cannot reproduce SuperLU's iterates
    bit for bit at this size, so the bar is the same ministeps accepted and
    rejected, each within 2 Newton iterations of the reference's, and the
    converged state within the Newton tolerance: p <= 1e-6 relative,
    sW <= 1e-5."""
    d = load("cfg1_ow_100x100x10.npz")
    c = cases.five_spot(dims=(100, 100, 10), seed=1)
    assert np.isclose(np.sum(c.rock.perm), float(d["perm_sum"]), rtol=1e-14)
    assert np.isclose(sum(np.sum(w.WI) for w in c.wells), float(d["wi_sum"]), rtol=1e-12)
    m = GpuOilWaterModel(c.grid, c.rock, c.fluid, c.wells, gravity=c.gravity,
                         cpr_options=dict(rtol=1e-12, maxiter=600, amg_rebuild_interval=1_000_000))
    events = []
    states, its = simulate_schedule_ad(m.initial_state(c.p0, c.sw0), m, [c.dt], verbose=False,
                                       observer=lambda ev, p: events.append((ev, p.get("dt"), p.get("iterations"))))
    mine = [(round(dt), int(it), ev == "step_accepted") for ev, dt, it in events
            if ev in ("step_accepted", "step_rejected")]
    ref = [(round(a), int(b), bool(c_)) for a, b, c_ in d["ministeps"]]
    assert [(a, c_) for a, _, c_ in mine] == [(a, c_) for a, _, c_ in ref], (mine, ref)
    assert all(abs(x[1] - y[1]) <= 2 for x, y in zip(mine, ref)), (mine, ref)
    p_ref = d["p_hist"][0]
    assert np.abs(states[0].pressure - p_ref).max() <= 1e-6 * np.abs(p_ref).max()
    assert np.abs(states[0].sW - d["sw_hist"][0]).max() <= 1e-5
