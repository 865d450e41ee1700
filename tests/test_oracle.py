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
