"""Pin the CPU oracle against the reference's own outputs (golden fixtures
made by tests/golden/make_golden.py) and the reference's MATLAB goldens."""

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import ow as oow
from oracle import trans as otrans
from pymrst_b200.grid import cartesian_grid
from pymrst_b200.params import make_rock

from compare import blockwise_error, ow_splits, segment_error
from fixtures import load, ow_case


def test_cartesian_grid_matches_reference_numbering_and_geometry():
    d = load("grid_trans.npz")
    g = cartesian_grid([4, 3, 2], [40.0, 30.0, 4.0])
    np.testing.assert_array_equal(g.faces.neighbors, d["neighbors"])
    np.testing.assert_array_equal(g.cells.faces, d["cell_faces"])
    np.testing.assert_array_equal(g.cells.facePos, d["facePos"])
    np.testing.assert_allclose(g.cells.centroids, d["cell_centroids"], rtol=1e-14, atol=1e-13)
    np.testing.assert_allclose(g.faces.centroids, d["face_centroids"], rtol=1e-14, atol=1e-13)
    np.testing.assert_allclose(g.faces.normals, d["normals"], rtol=1e-14, atol=1e-13)
    np.testing.assert_allclose(g.cells.volumes, d["volumes"], rtol=1e-14)


@pytest.mark.parametrize("key,permkey", [("1", "perm"), ("3", "perm3")])
def test_oracle_trans_matches_reference(key, permkey):
    d = load("grid_trans.npz")
    g = cartesian_grid([4, 3, 2], [40.0, 30.0, 4.0])
    perm = d[permkey]
    rock = make_rock(g, perm[:, None] if perm.ndim == 1 else perm, 0.2)
    ht = otrans.compute_trans(g, rock)
    np.testing.assert_allclose(ht, d["hT" + key], rtol=1e-13)
    np.testing.assert_allclose(otrans.face_trans(g, ht), d["T" + key], rtol=1e-13)


def _state(d, sfx=""):
    return oow.State(pressure=d["p" + sfx].copy(), sW=d["sw" + sfx].copy(),
                     qWs=d["qws" + sfx].copy(), qOs=d["qos" + sfx].copy(), bhp=d["bhp" + sfx].copy())


@pytest.mark.parametrize("name", ["ow_assemble_nograv.npz", "ow_assemble_grav.npz",
                                  "ow_assemble_xflow.npz"])
def test_oracle_residual_and_jacobian_match_reference_adi(name):
    d = load(name)
    g, rock, fluid, wells = ow_case(d)
    prob = oow.build_problem(g, rock, fluid.params, wells, gravity=float(d["gravity"]))
    np.testing.assert_allclose(prob.T, d["T"], rtol=1e-13)
    np.testing.assert_allclose(prob.pv, d["pv"], rtol=1e-14)
    st0, st = _state(d, "0"), _state(d)
    cdp = oow.compute_cdp(prob, st0)
    np.testing.assert_allclose(np.concatenate(cdp), d["cdp"], rtol=1e-12, atol=1e-9)
    res, J = oow.assemble(prob, st0, st, float(d["dt"]), cdp)
    splits = ow_splits(prob.nc, prob.nw)
    assert segment_error(res, d["res"], splits) < 1e-12
    Jref = sp.csr_array((d["J_data"], d["J_indices"], d["J_indptr"]), shape=tuple(d["J_shape"]))
    assert blockwise_error(J, Jref, splits) < 1e-12
    assert oow.converged(prob, res, float(d["dt"]), st)[0] == bool(d["converged"])


def test_crossflow_fixture_exercises_mixture_coupling():
    d = load("ow_assemble_xflow.npz")
    g, rock, fluid, wells = ow_case(d)
    prob = oow.build_problem(g, rock, fluid.params, wells, gravity=float(d["gravity"]))
    st = _state(d)
    P = oow.props(prob.fluid, st.pressure, st.sW)
    r = oow._well_terms(prob, 3, st.pressure, st.sW, P, st.qWs, st.qOs, st.bhp,
                        np.zeros(wells[3].cells.size))
    assert not r["dead"] and np.abs(r["U"]).max() > 0


@pytest.mark.parametrize("name", ["ow_newton_grav.npz", "ow_newton_nograv.npz"])
def test_oracle_newton_history_matches_reference(name):
    d = load(name)
    g, rock, fluid, wells = ow_case(d)
    prob = oow.build_problem(g, rock, fluid.params, wells, gravity=float(d["gravity"]))
    st0 = oow.initial_state(prob, float(d["p0"][0]), float(d["sw0"][0]))
    states, its = oow.simulate(prob, st0, np.full(int(d["nsteps"]), float(d["dt_days"]) * 86400.0))
    np.testing.assert_array_equal(its, d["its"])
    for k, s in enumerate(states):
        assert np.abs(s.pressure - d["p_hist"][k]).max() <= 1e-10 * np.abs(d["p_hist"][k]).max()
        assert np.abs(s.sW - d["sw_hist"][k]).max() <= 1e-9
        np.testing.assert_allclose(s.bhp, d["bhp_hist"][k], rtol=1e-10)


def test_oracle_phase5_matches_reference_and_matlab():
    d = load("ow_phase5.npz")
    from types import SimpleNamespace
    from pymrst_b200.params import add_well
    from fixtures import ow_fluid
    g = cartesian_grid([15, 15, 1], [300.0, 300.0, 10.0])
    rock = make_rock(g, d["perm"][:, None], 0.25)
    w = add_well(None, g, rock, np.array([0]), well_type="rate", val=2e-3,
                 compi=np.array([1.0, 0.0]), sign=1)
    w = add_well(w, g, rock, np.array([g.cells.num - 1]), well_type="bhp", val=150e5,
                 compi=np.array([0.0, 1.0]), sign=-1)
    np.testing.assert_allclose(np.concatenate([w[0].WI, w[1].WI]), d["mat_WI"], rtol=1e-12)
    prob = oow.build_problem(g, rock, ow_fluid("p5").params, w)
    st0 = oow.initial_state(prob, 200e5, 0.2)
    states, its = oow.simulate(prob, st0, np.full(8, 30.0 * 86400.0))
    np.testing.assert_array_equal(its, d["its"])
    p = np.vstack([s.pressure for s in states])
    sw = np.vstack([s.sW for s in states])
    assert np.abs(p - d["p_hist"]).max() <= 1e-10 * np.abs(d["p_hist"]).max()
    assert np.abs(sw - d["sw_hist"]).max() <= 1e-9
    # MATLAB MRST goldens, at validate_phase5.py's tolerance (5e-6 of field max)
    for mine, ref in ((p, d["mat_p_hist"]), (sw, d["mat_sw_hist"]),
                      (np.vstack([s.bhp for s in states]), d["mat_bhp"])):
        mine = np.asarray(mine).ravel()
        ref = np.asarray(ref).ravel()
        assert np.abs(mine - ref).max() <= 5e-6 * np.abs(ref).max()


@pytest.mark.parametrize("name", ["adjoint_grav.npz", "adjoint_nograv.npz"])
def test_oracle_adjoint_matches_reference(name):
    """compute_gradient_adjoint (optimization/adjoint.py:161-225) restated over
    the oracle model, against the reference's own run."""
    from oracle import adjoint as oadj
    d = load(name)
    g, rock, fluid, wells = ow_case(d)
    prob = oow.build_problem(g, rock, fluid.params, wells, gravity=float(d["gravity"]))
    st0 = oow.State(pressure=d["p0"].copy(), sW=d["sw0"].copy(), qWs=d["qws0"].copy(), qOs=d["qos0"].copy(),
                    bhp=d["bhp0"].copy())
    res = oadj.compute_gradient_adjoint(prob, st0, d["dts"], d["controls"])
    for k, s in enumerate(res.states[1:]):
        assert np.abs(s.pressure - d["p_hist"][k]).max() <= 1e-8 * np.abs(d["p_hist"][k]).max()
        assert np.abs(s.sW - d["sw_hist"][k]).max() <= 1e-7
    assert abs(res.value - float(d["value"])) <= 1e-9 * abs(float(d["value"]))
    for j in range(d["gradient"].shape[1]):
        ref = d["gradient"][:, j]
        assert np.abs(res.gradient[:, j] - ref).max() <= 1e-6 * np.abs(ref).max()
    assert np.abs(res.initial_state_gradient - d["dx0"]).max() <= 1e-6 * np.abs(d["dx0"]).max()


# ---- incompressible TPFA -----------------------------------------------------------

def _incomp_close(mine, ref, rtol=1e-9):
    mine = np.asarray(mine, float).ravel()
    ref = np.asarray(ref, float).ravel()
    np.testing.assert_allclose(mine, ref, rtol=rtol, atol=rtol * max(np.abs(ref).max(), 1e-300) + 1e-15)


def _incomp_matlab_cases():
    """The four MATLAB incompTPFA golden cases (validate_phase2's setups):
    name -> (grid, half-face T, bc, src, wells, gravity vector)."""
    from pymrst_b200.params import BARSA, DARCY, MILLI, add_bc, add_source, add_well
    gz = np.array([0.0, 0.0, 9.80665])
    out = {}
    g = cartesian_grid([32, 32, 1], [500.0, 500.0, 10.0])
    rock = make_rock(g, ((10 + (7 * np.arange(g.cells.num)) % 100) * MILLI * DARCY)[:, None], 0.2)
    src = add_source(add_source(None, [0], 1e-3), [g.cells.num - 1], -1e-3)
    out["qfs"] = (g, otrans.compute_trans(g, rock), None, src, [], None)
    g = cartesian_grid([20, 10, 5], [200.0, 100.0, 50.0])
    rock = make_rock(g, ((1 + (3 * np.arange(g.cells.num)) % 50) * MILLI * DARCY)[:, None], 0.25)
    bd = np.any(g.faces.neighbors == -1, axis=1)
    fc = g.faces.centroids
    bc = add_bc(None, np.flatnonzero(bd & (fc[:, 0] < 1e-10)), "pressure", 200 * BARSA)
    bc = add_bc(bc, np.flatnonzero(bd & (fc[:, 0] > 200 - 1e-10)), "pressure", 100 * BARSA)
    bc = add_bc(bc, np.flatnonzero(bd & (fc[:, 1] < 1e-10)), "flux", 1e-6)
    out["bc"] = (g, otrans.compute_trans(g, rock), bc, None, [], None)
    g = cartesian_grid([10, 10, 3], [1000.0, 1000.0, 30.0])
    rock = make_rock(g, np.tile(np.array([100.0, 100.0, 10.0]) * MILLI * DARCY, (g.cells.num, 1)), 0.3)
    w = add_well(None, g, rock, [0, 100, 200], well_type="rate", val=5e-3, radius=0.1,
                 compi=np.array([1.0]), gravity=gz)
    w = add_well(w, g, rock, [99, 199, 299], well_type="bhp", val=100 * BARSA, radius=0.1,
                 compi=np.array([1.0]), gravity=gz)
    out["wells"] = (g, otrans.compute_trans(g, rock), None, None, w, gz)
    g = cartesian_grid([1, 1, 30], [1.0, 1.0, 300.0])
    rock = make_rock(g, 100 * MILLI * DARCY, 0.2)
    bd = np.any(g.faces.neighbors == -1, axis=1)
    bc = add_bc(None, np.flatnonzero(bd & (g.faces.centroids[:, 2] < 1e-10)), "pressure", 100 * BARSA)
    out["gravity"] = (g, otrans.compute_trans(g, rock), bc, None, [], gz)
    return out


@pytest.mark.parametrize("case", ["qfs", "bc", "wells", "gravity"])
def test_oracle_incomp_matches_matlab(case):
    from oracle import incomp as oinc
    from pymrst_b200.params import CENTI, POISE
    m = load("incomp_matlab.npz")
    g, ht, bc, src, wells, gz = _incomp_matlab_cases()[case]
    mob = np.full((g.cells.num, 1), 1.0 / (1 * CENTI * POISE))
    p, bhp, fp, flux, wflux = oinc.incomp_tpfa(g, ht, mob, [1000.0], gz, bc, src, wells)
    _incomp_close(p, m[case + "__p"])
    _incomp_close(flux, m[case + "__flux"])
    if case in ("qfs", "bc"):
        _incomp_close(fp, m[case + "__fp"])
    if case == "wells":
        _incomp_close(wflux[0], m["wells__wflux1"])
        _incomp_close(wflux[1], m["wells__wflux2"])
        _incomp_close(bhp, np.concatenate([m["wells__bhp1"], m["wells__bhp2"]]))


def test_oracle_incomp_matches_reference_at_64x64x8():
    """Benchmark config 0 (32,768 cells), against the reference's own
    incomp_tpfa output."""
    from oracle import incomp as oinc
    from pymrst_b200 import cases
    from pymrst_b200.params import CENTI, DARCY, MILLI, POISE
    from fixtures import wells_from
    d = load("cfg0_incomp_64x64x8.npz")
    g = cartesian_grid([64, 64, 8], [640.0, 640.0, 16.0])
    perm = np.exp(cases.lognormal_logperm((64, 64, 8), np.random.default_rng(0))).ravel(order="F") * MILLI * DARCY
    assert np.isclose(perm.sum(), float(d["perm_sum"]), rtol=1e-14)
    ht = otrans.compute_trans(g, make_rock(g, perm[:, None], 0.2))
    assert np.isclose(ht.sum(), float(d["hT_sum"]), rtol=1e-13)
    wells = wells_from(d)
    mob = np.full((g.cells.num, 1), 1.0 / (1 * CENTI * POISE))
    p, bhp, fp, flux, wflux = oinc.incomp_tpfa(g, ht, mob, [1000.0], None, None, None, wells)
    _incomp_close(p, d["p"])
    _incomp_close(bhp, d["bhp"])
    _incomp_close(flux, d["flux"])
    _incomp_close(fp, d["facePressure"])
    _incomp_close(wflux[0], d["wflux0"])
    _incomp_close(wflux[1], d["wflux1"])


# ---- black-oil ------------------------------------------------------------------------------

def _bo_oracle_problem(d):
    from oracle import blackoil as obo
    from pymrst_b200.blackoil import BlackOilTables
    from pymrst_b200.params import pore_volume
    from fixtures import bo_case
    g, rock, deck, wells = bo_case(d)
    fl = obo.Fluid(BlackOilTables.from_deck(deck))
    Nall = np.asarray(g.faces.neighbors)
    internal = np.all(Nall >= 0, axis=1)
    Nn = Nall[internal]
    T = otrans.face_trans(g, otrans.compute_trans(g, rock))[internal]
    z = np.asarray(g.cells.centroids)[:, 2]
    gdz = 9.80665 * (z[Nn[:, 1]] - z[Nn[:, 0]])
    ws = [dict(cells=w.cells, WI=w.WI, compi=np.asarray(w.compi, float)[:3], type=w.type, val=w.val) for w in wells]
    return fl, Nn, T, gdz, pore_volume(g, rock), ws


@pytest.mark.parametrize("tag", ["a", "b"])
def test_oracle_blackoil_residual_update_and_convergence_match_reference(tag):
    """The numpy restatement of the black-oil equations against the
    reference's assemble (saturated and undersaturated cells, a cross-flowing
    bhp well, every control type), its update_state + flash and _converged."""
    from oracle import blackoil as obo
    from fixtures import bo_state
    d = load("bo_assemble.npz")
    fl, Nn, T, gdz, pv, ws = _bo_oracle_problem(d)
    st0, st = bo_state(d, tag + "0_"), bo_state(d, tag + "_")
    dt = float(d[tag + "_dt"])
    r = obo.residual(fl, Nn, T, gdz, pv, ws, st0, st, dt)
    ref = d[tag + "_res"]
    nc = st.pressure.size
    for lo, hi in ((0, nc), (nc, 2 * nc), (2 * nc, 3 * nc), (3 * nc, ref.size)):
        scale = np.abs(ref[lo:hi]).max()
        assert np.abs(r[lo:hi] - ref[lo:hi]).max() <= 1e-11 * scale
    assert obo.convergence(fl, pv, ws, st, ref, dt)[2] == bool(d[tag + "_converged"])
    new = obo.update_state(fl, st, d[tag + "_upd"])
    want = bo_state(d, tag + "_new_")
    np.testing.assert_array_equal(new.status, want.status)
    np.testing.assert_allclose(new.s, want.s, rtol=0, atol=1e-15)
    np.testing.assert_allclose(new.rs, want.rs, rtol=1e-14)
    np.testing.assert_allclose(new.pressure, want.pressure, rtol=1e-15)
    np.testing.assert_allclose(new.bhp, want.bhp, rtol=1e-15)


def test_blackoil_fixture_exercises_switching_and_crossflow():
    d = load("bo_assemble.npz")
    assert set(np.unique(d["a_status"])) == {1, 3}
    assert (d["a_new_status"] != d["a_status"]).any()
    p = d["a_p"]
    xf = d["w2_cells"]
    assert (p[xf] < d["a_bhp"][2]).any() and (p[xf] > d["a_bhp"][2]).any()
    n = load("bo_newton.npz")
    assert (n["hist_status"][-1] == 3).sum() > (n["init_status"] == 3).sum()


# ---- incompressible transport ------------------------------------------------------------------

def transport_problem(case, flux=None):
    """The phase-3 transport cases: (problem, initial s, gravity-estimate
    flux) for the oracle, from the grid, rock, sources and flux of
    validate_phase3's setups."""
    from oracle import transport as otr
    from pymrst_b200.params import CENTI, DARCY, DAY, MILLI, POISE
    d = load("transport_phase3.npz")
    if case == "bl":
        g = cartesian_grid([100, 1, 1], [100.0, 1.0, 1.0])
        k, poro, fl = 100 * MILLI * DARCY, 0.2, otr.Corey(np.array([1.0, 10.0]) * CENTI * POISE, [1000.0, 700.0], [2, 2])
        rate = float(d["bl_rate"])
        srcs = ([0, 99], [rate, -rate], [[1.0, 0.0], [0.0, 1.0]])
        gvec = np.zeros(3)
        flux = d["bl_flux0"] if flux is None else flux
        s0 = np.zeros(g.cells.num)
    elif case == "qfs":
        g = cartesian_grid([32, 32, 1], [500.0, 500.0, 10.0])
        k = ((10 + (7 * np.arange(g.cells.num)) % 100) * MILLI * DARCY)
        poro, fl = 0.2, otr.Corey(np.array([1.0, 10.0]) * CENTI * POISE, [1000.0, 700.0], [2, 2])
        srcs = ([0, g.cells.num - 1], [5e-3, -5e-3], [[1.0, 0.0], [0.0, 1.0]])
        gvec = np.zeros(3)
        s0 = np.zeros(g.cells.num)
    else:
        g = cartesian_grid([1, 1, 20], [1.0, 1.0, 20.0])
        k, poro, fl = 1000 * MILLI * DARCY, 0.3, otr.Corey([1e-3, 1e-3], [1000.0, 700.0], [2, 2])
        srcs = ([], [], np.zeros((0, 2)))
        gvec = np.array([0.0, 0.0, 9.80665])
        flux = np.zeros(g.faces.num)
        s0 = np.full(g.cells.num, 0.5)
    nc = g.cells.num
    Nall = np.asarray(g.faces.neighbors)
    internal = np.all(Nall >= 0, axis=1)
    cf = np.asarray(g.cells.faces)
    cell_no = np.repeat(np.arange(nc), np.diff(g.cells.facePos))
    K = np.zeros((nc, 3, 3))
    K[:, 0, 0] = K[:, 1, 1] = K[:, 2, 2] = k
    normals = np.asarray(g.faces.normals)
    gf = otr.gravity_flux(normals, cf, cell_no, K, gvec * (fl.rho[0] - fl.rho[1]), g.faces.num)[internal]
    gf_est = otr.gravity_flux(normals, cf, cell_no, K, -gvec, g.faces.num)[internal]
    q = otr.source(nc, fl, *srcs)
    pv = poro * np.asarray(g.cells.volumes)
    prob = otr.Problem(fl, Nall[internal], None if flux is None else np.asarray(flux)[internal], gf, q, pv)
    return prob, s0, gf_est, g, internal


def test_oracle_explicit_transport_matches_reference_and_matlab():
    d = load("transport_phase3.npz")
    DAY = 86400.0
    prob, s0, gf_est, _, _ = transport_problem("bl")
    s, nsub = prob.explicit(s0, 30 * DAY, gf_est, dt=0.25 * DAY)
    assert nsub == 120
    np.testing.assert_allclose(s, d["bl_sE"], rtol=0, atol=1e-13)
    np.testing.assert_allclose(s, d["bl_mat_sE"], rtol=0, atol=1e-10)
    s, _ = prob.explicit(s0, 30 * DAY, gf_est)
    np.testing.assert_allclose(s, d["bl_sE_auto"], rtol=0, atol=1e-12)
    prob, s0, gf_est, _, _ = transport_problem("grav")
    s, _ = prob.explicit(s0, 5 * DAY, gf_est)
    np.testing.assert_allclose(s, d["grav_sE_auto"], rtol=0, atol=1e-12)


def test_oracle_implicit_transport_matches_reference_and_matlab():
    d = load("transport_phase3.npz")
    DAY = 86400.0
    prob, s0, _, _, _ = transport_problem("bl")
    s = prob.implicit(s0, 30 * DAY)
    np.testing.assert_allclose(s, d["bl_sI"], rtol=0, atol=1e-10)
    np.testing.assert_allclose(s, d["bl_mat_sI"], rtol=0, atol=5e-6)
    prob, s0, _, _, _ = transport_problem("grav")
    s = prob.implicit(s0, 50 * DAY)
    np.testing.assert_allclose(s, d["grav_sG"], rtol=0, atol=1e-10)
    np.testing.assert_allclose(s, d["grav_mat_sG"], rtol=0, atol=5e-6)


def test_oracle_sequential_quarter_five_spot_matches_reference_and_matlab():
    """Two incomp_tpfa + implicit transport cycles (validate_phase3's qfs)."""
    from oracle import incomp as oinc
    from pymrst_b200.params import DARCY, MILLI, add_source
    d = load("transport_phase3.npz")
    prob, s, _, g, internal = transport_problem("qfs")
    rock = make_rock(g, ((10 + (7 * np.arange(g.cells.num)) % 100) * MILLI * DARCY)[:, None], 0.2)
    ht = otrans.compute_trans(g, rock)
    src = add_source(add_source(None, [0], 5e-3, sat=[[1.0, 0.0]]), [g.cells.num - 1], -5e-3, sat=[[0.0, 1.0]])
    for _ in range(2):
        mob = prob.fluid.mobility(np.column_stack([s, 1.0 - s]))
        p, _, _, flux, _ = oinc.incomp_tpfa(g, ht, mob, [1000.0, 700.0], None, None, src, [])
        prob.v = np.asarray(flux)[internal]
        s = prob.implicit(s, 100 * 86400.0)
    np.testing.assert_allclose(s, d["qfs_sQ"], rtol=0, atol=1e-9)
    np.testing.assert_allclose(p, d["qfs_pQ"], rtol=1e-9)
    np.testing.assert_allclose(s, d["qfs_mat_sQ"], rtol=0, atol=2e-5)
