"""GPU parity of the black-oil path (three phases, dissolved gas, variable
switching) against the reference's own outputs and the CPU oracle.

Fixtures (tests/golden/make_golden.py, from the reference's
ThreePhaseBlackOilModelAD on a synthetic deck): bo_assemble.npz holds the
residual, Jacobian, update + flash and convergence flag at iterates with
saturated and undersaturated cells, cells at their bubble point and a
cross-flowing bhp well; bo_newton.npz the Newton histories of seven steps
with gas injection (rate), an oil-rate producer (orat) and a bhp producer.

Tolerances: residuals 1e-11 and Jacobians 1e-10 blockwise relative;
updates to rounding; states after each step p <= 1e-8 relative, s and rs
<= 1e-7 (rs relative), equal Newton counts and phase states, with the
CPR-GMRES tolerance at 1e-12 so that the Newton paths coincide.
"""

import sys
from pathlib import Path

import numpy as np
import pytest
import scipy.sparse as sp

from compare import blockwise_error, segment_error
from fixtures import bo_case, bo_state, load

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from oracle import blackoil as obo  # noqa: E402
from pymrst_b200.blackoil import BlackOilTables, GpuBlackOilModel  # noqa: E402
from pymrst_b200.build import build  # noqa: E402

build()

TIGHT = dict(rtol=1e-12, maxiter=400)


def _splits(nc, nw):
    return np.array([0, nc, 2 * nc, 3 * nc, 3 * nc + nw, 3 * nc + 2 * nw, 3 * nc + 3 * nw, 3 * nc + 4 * nw])


def _model(d, **kw):
    g, rock, deck, wells = bo_case(d)
    return GpuBlackOilModel(g, rock, deck, wells, **kw), deck


def test_fluid_tables_match_the_oracle_inside_and_outside_the_tables():
    d = load("bo_assemble.npz")
    m, deck = _model(d)
    fl = obo.Fluid(BlackOilTables.from_deck(deck))
    rng = np.random.default_rng(0)
    p = rng.uniform(-20e5, 450e5, 4000)
    rs = rng.uniform(-10.0, 220.0, p.size)
    for sat in (False, True):
        flag = np.full(p.size, sat)
        got = m.pvt_points(p, rs, flag)
        want = [fl.b_w(p), fl.b_o(p, rs, flag), fl.mu_o(p, rs, flag), fl.b_g(p), fl.mu_g(p), fl.rs_sat(p),
                fl.pv_mult(p)]
        for a, b in zip(got, want):
            np.testing.assert_allclose(a, b, rtol=1e-13, atol=0)
    sw = rng.uniform(-0.1, 1.1, 4000)
    sg = rng.uniform(-0.1, 1.0, sw.size)
    kr = m.relperm_points(sw, sg)
    so = 1.0 - sw - sg
    for a, b in zip(kr, [fl.kr_w(sw), fl.kr_o(sw, so, sg), fl.kr_g(sg), fl.pc_ow(sw), fl.pc_og(sg)]):
        np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-15)


@pytest.mark.parametrize("tag", ["a", "b"])
def test_residual_jacobian_update_and_convergence_match_reference(tag):
    d = load("bo_assemble.npz")
    m, _ = _model(d)
    st0, st = bo_state(d, tag + "0_"), bo_state(d, tag + "_")
    dt = float(d[tag + "_dt"])
    res, jac = m.assemble_system(st0, st, dt)
    nc, nw = m.nc, m.nw
    sp_ = _splits(nc, nw)
    assert segment_error(res, d[tag + "_res"], sp_) <= 1e-11
    ref = sp.csr_array((d[tag + "_jac_data"], d[tag + "_jac_indices"], d[tag + "_jac_indptr"]), shape=jac.shape)
    assert blockwise_error(jac, ref, sp_) <= 1e-10
    assert m.convergence(st0, st, dt)["converged"] == bool(d[tag + "_converged"])
    new = m.update_state(st, d[tag + "_upd"])
    want = bo_state(d, tag + "_new_")
    np.testing.assert_array_equal(new.status, want.status)
    np.testing.assert_allclose(new.s, want.s, rtol=0, atol=1e-15)
    np.testing.assert_allclose(new.rs, want.rs, rtol=1e-14)
    np.testing.assert_allclose(new.pressure, want.pressure, rtol=1e-15)
    for f in ("qWs", "qOs", "qGs", "bhp"):
        np.testing.assert_allclose(getattr(new, f), getattr(want, f), rtol=1e-15)


def test_jacobian_is_the_derivative_of_the_residual():
    """Central differences of the device residual along a random direction
    of the primary variables (phase states fixed) equal J v."""
    d = load("bo_assemble.npz")
    m, _ = _model(d)
    st0, st = bo_state(d, "a0_"), bo_state(d, "a_")
    # the well-stream mixture takes q * (q > 0): a rate of exactly 0 is a kink,
    # where a central difference averages the two one-sided slopes
    st.qWs = np.where(st.qWs == 0.0, -1e-6, st.qWs)
    st.qOs = np.where(st.qOs == 0.0, -1e-6, st.qOs)
    dt = float(d["a_dt"])
    res, jac = m.assemble_system(st0, st, dt)
    nc, nw = m.nc, m.nw
    rng = np.random.default_rng(5)
    v = np.concatenate([rng.normal(size=nc) * 1e3, rng.normal(size=nc) * 1e-4,
                        np.where(st.status == 1, 1e-2, 1e-4) * rng.normal(size=nc),
                        rng.normal(size=3 * nw) * 1e-4, rng.normal(size=nw) * 1e3])

    def shifted(h):
        s = st.copy()
        s.pressure = s.pressure + h * v[:nc]
        dsw = h * v[nc:2 * nc]
        dx = h * v[2 * nc:3 * nc]
        sat = s.status == 3
        s.s = s.s + np.column_stack([dsw, -dsw - np.where(sat, dx, 0.0), np.where(sat, dx, 0.0)])
        s.rs = np.where(sat, s.rs, s.rs + dx)
        s.qWs, s.qOs, s.qGs = (s.qWs + h * v[3 * nc:3 * nc + nw], s.qOs + h * v[3 * nc + nw:3 * nc + 2 * nw],
                               s.qGs + h * v[3 * nc + 2 * nw:3 * nc + 3 * nw])
        s.bhp = s.bhp + h * v[3 * nc + 3 * nw:]
        return s

    # the tables are piecewise linear and the upwind / injection choices switch:
    # a step small enough to stay on one linear piece of every function
    h = 1e-7
    fd = (m.assemble_system(st0, shifted(h), dt)[0] - m.assemble_system(st0, shifted(-h), dt)[0]) / (2 * h)
    jv = jac @ v
    assert segment_error(jv, fd, _splits(nc, nw)) <= 1e-4


def test_newton_history_matches_reference():
    d = load("bo_newton.npz")
    m, _ = _model(d, cpr_options=TIGHT)
    st = bo_state(d, "init_")
    for k, dt in enumerate(d["dts"]):
        st, ok, its = m.step(st, float(dt))
        assert ok and its == int(d["its"][k]), (k, its, int(d["its"][k]))
        np.testing.assert_array_equal(st.status, d["hist_status"][k])
        p_ref = d["hist_pressure"][k]
        assert np.abs(st.pressure - p_ref).max() <= 1e-8 * np.abs(p_ref).max()
        assert np.abs(st.s - d["hist_s"][k]).max() <= 1e-7
        assert np.abs(st.rs - d["hist_rs"][k]).max() <= 1e-7 * np.abs(d["hist_rs"][k]).max()
        for f in ("qWs", "qOs", "qGs"):
            r = d["hist_" + f][k]
            assert np.abs(getattr(st, f) - r).max() <= 1e-7 * max(np.abs(r).max(), 1e-3)
        assert np.abs(st.bhp - d["hist_bhp"][k]).max() <= 1e-8 * np.abs(d["hist_bhp"][k]).max()


def test_invalid_inputs_are_rejected_on_the_host():
    d = load("bo_assemble.npz")
    g, rock, deck, wells = bo_case(d)
    bad = dict(deck)
    bad["pvtg"] = []
    with pytest.raises(ValueError):
        GpuBlackOilModel(g, rock, bad, wells)
    twice = list(wells) + [wells[0]]
    from pymrst_b200._native import PMBError
    with pytest.raises(PMBError):
        GpuBlackOilModel(g, rock, deck, twice)


REF = Path(__file__).resolve().parents[1] / "baseline" / "_ref"


@pytest.mark.skipif(not (REF / "pymrst").is_dir(), reason="the reference package is not installed under baseline/_ref")
def test_reference_fluid_and_wells_drive_the_gpu_model():
    """The reference's own BlackOilFluid (tables read from its functions and
    checked against them) and wells: the same Newton history as the
    reference's ThreePhaseBlackOilModelAD."""
    sys.path.insert(0, str(REF))
    from pymrst.gridprocessing import cart_grid, compute_geometry
    from pymrst.modules.ad_blackoil.models.three_phase_black_oil_model import BOState, ThreePhaseBlackOilModelAD
    from pymrst.modules.ad_props.props.init_deck_adi_fluid import init_deck_blackoil_fluid
    from pymrst.params import add_well, make_rock
    from fixtures import bo_deck
    d = load("bo_newton.npz")
    deck = bo_deck(d)
    g = compute_geometry(cart_grid([int(v) for v in d["dims"]], [float(v) for v in d["phys"]]))
    rock = make_rock(g, d["perm"][:, None], 0.3)
    fluid = init_deck_blackoil_fluid(deck)
    wells = None
    for k in range(int(d["wcount"])):
        wells = add_well(wells, g, rock, d[f"w{k}_cells"], well_type=str(d[f"w{k}_type"]),
                         val=float(d[f"w{k}_val"]), radius=0.1, compi=d[f"w{k}_compi"])
    ref_model = ThreePhaseBlackOilModelAD(g, rock, fluid, wells)
    gpu = GpuBlackOilModel(g, rock, fluid, wells, cpr_options=TIGHT)
    init = bo_state(d, "init_")
    st_ref = BOState(*(np.array(getattr(init, f)) for f in ("pressure", "s", "rs", "status", "qWs", "qOs",
                                                            "qGs", "bhp")))
    st_gpu = st_ref.copy()
    for dt in d["dts"][:3]:
        st_ref, ok_r, it_r = ref_model.step(st_ref, float(dt))
        st_gpu, ok_g, it_g = gpu.step(st_gpu, float(dt))
        assert isinstance(st_gpu, BOState)
        assert ok_r and ok_g and it_r == it_g
        np.testing.assert_array_equal(st_gpu.status, st_ref.status)
        assert np.abs(st_gpu.pressure - st_ref.pressure).max() <= 1e-8 * np.abs(st_ref.pressure).max()
        assert np.abs(st_gpu.s - st_ref.s).max() <= 1e-7
