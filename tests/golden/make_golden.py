"""Generate the golden fixtures in this folder by running the reference.

Run once, where the reference's Python package is importable:

    python tests/golden/make_golden.py <reference checkout> [--only NAME,...]

NAME selects fixture groups: small (the toy-grid fixtures), cfg0 (incomp_tpfa
at 64x64x8), cfg1 (the first oil-water steps at 100x100x10), cfg4 (the
adjoint at 64x64x4), transport (the phase-3 transport cases), bo (the three-phase black-oil model on a synthetic
deck: residuals and Jacobians, and Newton histories), geometry (compute_geometry on a perturbed 3-D grid).  Without --only every
group is written.

It writes small .npz files holding inputs and the reference's own outputs
(grid arrays, transmissibilities, oil-water residuals and Jacobians, Newton
histories, incompressible pressure solves, adjoint gradients) plus the reference's MATLAB golden
arrays (examples/validation/ref_p2_*.mat, ref_p5_ow.mat) copied as data.  The
tests read only the .npz files, so they run without the reference.
"""

import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).parent
if len(sys.argv) < 2 or sys.argv[1].startswith("-"):
    sys.exit(__doc__)
REF = Path(sys.argv[1])
ONLY = None
if "--only" in sys.argv:
    ONLY = set(sys.argv[sys.argv.index("--only") + 1].split(","))
sys.path.insert(0, str(REF))
sys.path.insert(1, str(HERE.parent.parent))  # the repository: the seeded case generators

import scipy.io  # noqa: E402
from scipy.ndimage import uniform_filter  # noqa: E402

from pymrst.gridprocessing import cart_grid, compute_geometry  # noqa: E402
from pymrst.modules.ad_blackoil import TwoPhaseOilWaterModelAD  # noqa: E402
from pymrst.modules.ad_core import simulate_schedule_ad  # noqa: E402
from pymrst.modules.ad_props import init_simple_adi_fluid  # noqa: E402
from pymrst.params import add_well, make_rock  # noqa: E402
from pymrst.solvers import compute_trans  # noqa: E402
from pymrst.solvers.get_face_transmissibility import get_face_transmissibility  # noqa: E402
from pymrst.utils.adi import combine_equations, init_variables_adi  # noqa: E402
from pymrst.utils.units import BARSA, CENTI, DARCY, DAY, MILLI, POISE  # noqa: E402


def lognormal_perm(dims, seed, sigma=1.0, mean_md=100.0):
    rng = np.random.default_rng(seed)
    logk = rng.normal(np.log(mean_md), sigma, size=tuple(dims))
    logk = uniform_filter(logk, size=3, mode="nearest")
    return np.exp(logk).ravel(order="F") * MILLI * DARCY


def save(name, **arrays):
    np.savez_compressed(HERE / name, **arrays)
    print("wrote", name, sum(np.asarray(v).nbytes for v in arrays.values()), "bytes raw")


def wells_arrays(prefix, wells):
    out = {}
    out[prefix + "count"] = np.array(len(wells))
    for k, w in enumerate(wells):
        out[f"{prefix}{k}_cells"] = np.asarray(w.cells)
        out[f"{prefix}{k}_WI"] = np.asarray(w.WI)
        out[f"{prefix}{k}_dZ"] = np.asarray(w.dZ)
        out[f"{prefix}{k}_compi"] = np.asarray(w.compi)
        out[f"{prefix}{k}_type"] = np.array(w.type)
        out[f"{prefix}{k}_val"] = np.array(w.val)
        out[f"{prefix}{k}_refDepth"] = np.array(w.refDepth)
    return out


def grid_fixture():
    g = compute_geometry(cart_grid([4, 3, 2], [40.0, 30.0, 4.0]))
    perm = lognormal_perm([4, 3, 2], 11)
    rock1 = make_rock(g, perm[:, None], 0.2)
    perm3 = np.column_stack([perm, 2 * perm, 0.1 * perm])
    rock3 = make_rock(g, perm3, 0.2)
    t1 = compute_trans(g, rock1)
    t3 = compute_trans(g, rock3)
    save("grid_trans.npz",
         neighbors=g.faces.neighbors, cell_faces=g.cells.faces, facePos=g.cells.facePos,
         cell_centroids=g.cells.centroids, face_centroids=g.faces.centroids,
         normals=g.faces.normals, areas=g.faces.areas, volumes=g.cells.volumes,
         perm=perm, perm3=perm3, hT1=t1, hT3=t3,
         T1=get_face_transmissibility(g, rock1), T3=get_face_transmissibility(g, rock3))


def ow_fluid(kind):
    if kind == "cfg":
        return init_simple_adi_fluid(mu=np.array([1.0, 5.0]) * CENTI * POISE,
                                     rho=[1000.0, 800.0], n=[2, 2],
                                     c=[1e-5 / BARSA, 1e-5 / BARSA], p_ref=200 * BARSA,
                                     smin=[0.1, 0.1])
    return init_simple_adi_fluid(mu=np.array([1.0, 5.0]) * CENTI * POISE,
                                 rho=[1000.0, 800.0], n=[2, 2],
                                 c=[1e-6 / BARSA, 1e-4 / BARSA], p_ref=200 * BARSA)


def assemble_fixture(name, dims, phys, seed, fluid_kind, gravity, crossflow):
    rng = np.random.default_rng(seed)
    g = compute_geometry(cart_grid(dims, phys))
    nc = g.cells.num
    perm = lognormal_perm(dims, seed)
    rock = make_rock(g, perm[:, None], 0.2)
    fluid = ow_fluid(fluid_kind)
    nx, ny, nz = dims
    col = lambda i, j: i + nx * (j + ny * np.arange(nz))
    gvec = np.array([0, 0, gravity]) if gravity else None
    w = add_well(None, g, rock, col(0, 0), well_type="rate", val=2e-3,
                 compi=np.array([1.0, 0.0]), sign=1, gravity=gvec)
    w = add_well(w, g, rock, col(nx - 1, 0), well_type="rate", val=1e-3,
                 compi=np.array([1.0, 0.0]), sign=1, gravity=gvec)
    w = add_well(w, g, rock, col(nx - 1, ny - 1), well_type="bhp", val=150 * BARSA,
                 compi=np.array([0.0, 1.0]), sign=-1, gravity=gvec)
    if crossflow:
        w = add_well(w, g, rock, col(nx // 2, ny // 2), well_type="bhp", val=200 * BARSA,
                     compi=np.array([0.0, 1.0]), sign=-1, gravity=gvec)
    model = TwoPhaseOilWaterModelAD(g, rock, fluid, w, gravity=gravity)
    st0 = model.initial_state(200 * BARSA, 0.2)
    st0.pressure = 200 * BARSA + rng.normal(0, 2 * BARSA, nc)
    st0.sW = rng.uniform(0.1, 0.8, nc)
    st0.sW[::7] = 0.1
    st0.qWs = np.array([2e-3, 1e-3, 0.0] + ([0.0] if crossflow else []))
    st0.qOs = np.array([0.0, 0.0, -1.5e-3] + ([-1e-4] if crossflow else []))
    st = st0.copy()
    st.pressure = st0.pressure + rng.normal(0, 1 * BARSA, nc)
    st.sW = np.clip(st0.sW + rng.normal(0, 0.05, nc), 0.0, 1.0)
    st.sW[::5] = 0.1
    st.sW[3::11] = 0.9
    st.bhp = np.array([230 * BARSA, 225 * BARSA, 150 * BARSA] + ([200 * BARSA] if crossflow else []))
    st.qWs = np.array([1.9e-3, 1.1e-3, -2e-4] + ([1e-5] if crossflow else []))
    st.qOs = np.array([1e-6, 0.0, -1.2e-3] + ([-2e-4] if crossflow else []))
    if crossflow:
        c4 = w[3].cells
        st.pressure[c4] = 200 * BARSA + np.linspace(-3, 3, c4.size) * BARSA
    dt = 10 * DAY
    cdp = model._compute_cdp_per_well(st0)
    v = init_variables_adi(st.pressure, st.sW, st.qWs, st.qOs, st.bhp)
    eqs = model.assemble(st0, *v, dt, cdp)
    eq = combine_equations(*eqs)
    J = eq.jac[0].tocsr()
    conv = model._converged(eqs, dt, st)
    save(name, dims=np.array(dims), phys=np.array(phys, float), perm=perm, poro=np.array(0.2),
         gravity=np.array(float(gravity)), fluid_kind=np.array(fluid_kind),
         p0=st0.pressure, sw0=st0.sW, qws0=st0.qWs, qos0=st0.qOs, bhp0=st0.bhp,
         p=st.pressure, sw=st.sW, qws=st.qWs, qos=st.qOs, bhp=st.bhp, dt=np.array(dt),
         cdp=np.concatenate(cdp) if cdp else np.zeros(0),
         res=eq.val, J_data=J.data, J_indices=J.indices, J_indptr=J.indptr,
         J_shape=np.array(J.shape), converged=np.array(conv),
         T=model.ops.T, pv=model.pv, **wells_arrays("w", w))


def newton_fixture(name, dims, phys, seed, fluid_kind, gravity, nsteps, dt_days):
    g = compute_geometry(cart_grid(dims, phys))
    perm = lognormal_perm(dims, seed)
    rock = make_rock(g, perm[:, None], 0.2)
    fluid = ow_fluid(fluid_kind)
    nx, ny, nz = dims
    col = lambda i, j: i + nx * (j + ny * np.arange(nz))
    gvec = np.array([0, 0, gravity]) if gravity else None
    pvtot = float(np.sum(0.2 * g.cells.volumes))
    rate = 0.25 * pvtot / (nsteps * dt_days * DAY) / 2
    w = add_well(None, g, rock, col(0, 0), well_type="rate", val=rate,
                 compi=np.array([1.0, 0.0]), sign=1, gravity=gvec)
    w = add_well(w, g, rock, col(nx - 1, 0), well_type="rate", val=rate,
                 compi=np.array([1.0, 0.0]), sign=1, gravity=gvec)
    w = add_well(w, g, rock, col(nx // 2, ny - 1), well_type="bhp", val=150 * BARSA,
                 compi=np.array([0.0, 1.0]), sign=-1, gravity=gvec)
    model = TwoPhaseOilWaterModelAD(g, rock, fluid, w, gravity=gravity)
    st0 = model.initial_state(200 * BARSA, 0.1 if fluid_kind == "cfg" else 0.2)
    states, its = simulate_schedule_ad(st0, model, np.full(nsteps, dt_days * DAY), verbose=False)
    save(name, dims=np.array(dims), phys=np.array(phys, float), perm=perm, poro=np.array(0.2),
         gravity=np.array(float(gravity)), fluid_kind=np.array(fluid_kind),
         p0=st0.pressure, sw0=st0.sW, dt_days=np.array(float(dt_days)), nsteps=np.array(nsteps),
         its=its, p_hist=np.vstack([s.pressure for s in states]),
         sw_hist=np.vstack([s.sW for s in states]),
         qws_hist=np.vstack([s.qWs for s in states]), qos_hist=np.vstack([s.qOs for s in states]),
         bhp_hist=np.vstack([s.bhp for s in states]), **wells_arrays("w", w))


def phase5_fixture():
    """validate_phase5.py's case, run by the reference, with the MATLAB arrays."""
    g = compute_geometry(cart_grid([15, 15, 1], [300.0, 300.0, 10.0]))
    kvals = (50 + (11 * np.arange(g.cells.num)) % 200) * MILLI * DARCY
    rock = make_rock(g, kvals[:, None], 0.25)
    fluid = ow_fluid("p5")
    w = add_well(None, g, rock, np.array([0]), well_type="rate", val=2e-3,
                 compi=np.array([1.0, 0.0]), sign=1)
    w = add_well(w, g, rock, np.array([g.cells.num - 1]), well_type="bhp",
                 val=150 * BARSA, compi=np.array([0.0, 1.0]), sign=-1)
    model = TwoPhaseOilWaterModelAD(g, rock, fluid, w)
    st0 = model.initial_state(200 * BARSA, 0.2)
    states, its = simulate_schedule_ad(st0, model, np.full(8, 30.0) * DAY, verbose=False)
    m = scipy.io.loadmat(REF / "examples/validation/ref_p5_ow.mat", squeeze_me=True)
    save("ow_phase5.npz", perm=kvals, its=its,
         p_hist=np.vstack([s.pressure for s in states]), sw_hist=np.vstack([s.sW for s in states]),
         qws_hist=np.vstack([s.qWs for s in states]), qos_hist=np.vstack([s.qOs for s in states]),
         bhp_hist=np.vstack([s.bhp for s in states]),
         mat_p_hist=np.asarray(m["p_hist"], float), mat_sw_hist=np.asarray(m["sw_hist"], float),
         mat_qWs=np.asarray(m["qWs"], float), mat_qOs=np.asarray(m["qOs"], float),
         mat_bhp=np.asarray(m["bhp"], float),
         mat_WI=np.concatenate([np.atleast_1d(m["WI1"]), np.atleast_1d(m["WI2"])]).astype(float),
         **wells_arrays("w", w))


def incomp_fixtures():
    """The MATLAB incompTPFA goldens (validate_phase2.py cases) as data, plus
    the reference's own incomp_tpfa on a five-spot-like case with wells."""
    out = {}
    for case in ("qfs", "bc", "wells", "gravity"):
        m = scipy.io.loadmat(REF / f"examples/validation/ref_p2_{case}.mat", squeeze_me=True)
        for k, v in m.items():
            if k.startswith("__"):
                continue
            out[f"{case}__{k}"] = np.atleast_1d(np.asarray(v, dtype=float))
    save("incomp_matlab.npz", **out)

    from pymrst.modules.incomp import incomp_tpfa, init_single_fluid
    from pymrst.solvers import init_state
    dims = [16, 16, 4]
    g = compute_geometry(cart_grid(dims, [160.0, 160.0, 8.0]))
    perm = lognormal_perm(dims, 0)
    rock = make_rock(g, perm[:, None], 0.2)
    ht = compute_trans(g, rock)
    fl = init_single_fluid(1 * CENTI * POISE, 1000.0)
    nx, ny, nz = dims
    w = add_well(None, g, rock, 0 + nx * (0 + ny * np.arange(nz)), well_type="rate", val=1e-3,
                 radius=0.1, compi=np.array([1.0]))
    w = add_well(w, g, rock, (nx - 1) + nx * ((ny - 1) + ny * np.arange(nz)), well_type="bhp",
                 val=100 * BARSA, radius=0.1, compi=np.array([1.0]))
    st = incomp_tpfa(init_state(g, w, 0.0), g, ht, fl, wells=w)
    save("incomp_wells.npz", dims=np.array(dims), perm=perm, hT=ht, p=st.pressure, flux=st.flux,
         facePressure=st.facePressure, bhp=np.array([ws.pressure for ws in st.wellSol]),
         wflux0=st.wellSol[0].flux, wflux1=st.wellSol[1].flux, **wells_arrays("w", w))


def adjoint_fixture(name, dims, phys, seed, fluid_kind, gravity, nsteps, dt_days):
    """compute_gradient_adjoint (optimization/adjoint.py:161-225) with the NPV
    objective on a small model with per-step well controls."""
    from pymrst.modules.optimization.adjoint import compute_gradient_adjoint, npv_objective
    g = compute_geometry(cart_grid(dims, phys))
    perm = lognormal_perm(dims, seed)
    rock = make_rock(g, perm[:, None], 0.2)
    fluid = ow_fluid(fluid_kind)
    nx, ny, nz = dims
    col = lambda i, j: i + nx * (j + ny * np.arange(nz))
    gvec = np.array([0, 0, gravity]) if gravity else None
    pvtot = float(np.sum(0.2 * g.cells.volumes))
    rate = 0.3 * pvtot / (nsteps * dt_days * DAY) / 2
    w = add_well(None, g, rock, col(0, 0), well_type="rate", val=rate,
                 compi=np.array([1.0, 0.0]), sign=1, gravity=gvec)
    w = add_well(w, g, rock, col(nx - 1, 0), well_type="rate", val=rate,
                 compi=np.array([1.0, 0.0]), sign=1, gravity=gvec)
    w = add_well(w, g, rock, col(nx // 2, ny - 1), well_type="bhp", val=150 * BARSA,
                 compi=np.array([0.0, 1.0]), sign=-1, gravity=gvec)
    model = TwoPhaseOilWaterModelAD(g, rock, fluid, w, gravity=gravity)
    st0 = model.initial_state(200 * BARSA, 0.1 if fluid_kind == "cfg" else 0.2)
    rng = np.random.default_rng(seed)
    controls = np.column_stack([rate * rng.uniform(0.7, 1.3, nsteps), rate * rng.uniform(0.7, 1.3, nsteps),
                                BARSA * rng.uniform(140.0, 160.0, nsteps)])
    dts = np.full(nsteps, dt_days * DAY)
    wells0 = wells_arrays("w", w)  # before the sweep sets w.val to each step's controls
    res = compute_gradient_adjoint(model, st0, dts, controls, npv_objective())
    save(name, dims=np.array(dims), phys=np.array(phys, float), perm=perm, poro=np.array(0.2),
         gravity=np.array(float(gravity)), fluid_kind=np.array(fluid_kind),
         p0=st0.pressure, sw0=st0.sW, qws0=st0.qWs, qos0=st0.qOs, bhp0=st0.bhp, dts=dts, controls=controls,
         value=np.array(res.value), gradient=res.gradient, dx0=res.initial_state_gradient,
         p_hist=np.vstack([s.pressure for s in res.states[1:]]),
         sw_hist=np.vstack([s.sW for s in res.states[1:]]),
         qws_hist=np.vstack([s.qWs for s in res.states[1:]]),
         qos_hist=np.vstack([s.qOs for s in res.states[1:]]),
         bhp_hist=np.vstack([s.bhp for s in res.states[1:]]), **wells0)


def _sample_idx(n, k, seed):
    """k sorted distinct indices of range(n), seeded (the entries a fixture keeps
    of an array too large to store whole)."""
    return np.sort(np.random.default_rng(seed).choice(n, size=min(k, n), replace=False))


def cfg0_fixture():
    """Benchmark config 0: incomp_tpfa on 64x64x8 cells of 10x10x2 m, the
    seeded lognormal permeability, rate injector 1e-3 m^3/s down column
    (0, 0), bhp producer at 100 bar down column (63, 63), gravity off."""
    from pymrst.modules.incomp import incomp_tpfa, init_single_fluid
    from pymrst.solvers import init_state
    from pymrst_b200 import cases
    dims = [64, 64, 8]
    g = compute_geometry(cart_grid(dims, [640.0, 640.0, 16.0]))
    perm = np.exp(cases.lognormal_logperm(dims, np.random.default_rng(0))).ravel(order="F") * MILLI * DARCY
    rock = make_rock(g, perm[:, None], 0.2)
    ht = compute_trans(g, rock)
    fl = init_single_fluid(1 * CENTI * POISE, 1000.0)
    nx, ny, nz = dims
    w = add_well(None, g, rock, 0 + nx * (0 + ny * np.arange(nz)), well_type="rate", val=1e-3,
                 radius=0.1, compi=np.array([1.0]))
    w = add_well(w, g, rock, (nx - 1) + nx * ((ny - 1) + ny * np.arange(nz)), well_type="bhp",
                 val=100 * BARSA, radius=0.1, compi=np.array([1.0]))
    st = incomp_tpfa(init_state(g, w, 0.0), g, ht, fl, wells=w)
    save("cfg0_incomp_64x64x8.npz", dims=np.array(dims), perm_sum=np.array(perm.sum()),
         hT_sum=np.array(ht.sum()), p=st.pressure, flux=st.flux, facePressure=st.facePressure,
         bhp=np.array([ws.pressure for ws in st.wellSol]),
         wflux0=st.wellSol[0].flux, wflux1=st.wellSol[1].flux, **wells_arrays("w", w))


def _five_spot_reference(case):
    """The reference's model for a seeded five-spot case of the repository's
    generator: same grid, rock, wells (the reference's add_well) and fluid."""
    g = compute_geometry(cart_grid(list(case.grid.cartDims), list(np.asarray(case.grid.cartDims)
                                                                   * _cell_size(case))))
    rock = make_rock(g, np.asarray(case.rock.perm, float).reshape(g.cells.num, -1), np.asarray(case.rock.poro))
    gvec = np.array([0.0, 0.0, case.gravity]) if case.gravity else None
    w = None
    for wc in case.wells:
        w = add_well(w, g, rock, np.asarray(wc.cells), well_type=wc.type, val=float(np.ravel(wc.val)[0]),
                     compi=np.asarray(wc.compi, float), sign=int(wc.sign), gravity=gvec)
    model = TwoPhaseOilWaterModelAD(g, rock, ow_fluid("cfg"), w, gravity=case.gravity)
    return g, rock, w, model


def _cell_size(case):
    c = np.asarray(case.grid.cells.centroids)
    dims = case.grid.cartDims
    return np.array([2 * c[0, 0], 2 * c[0, 1], 2 * c[0, 2]]) if np.prod(dims) else np.ones(3)


def cfg1_fixture(nsteps=1):
    """Benchmark config 1: the oil-water five-spot on 100x100x10 cells with
    gravity, the first `nsteps` 10-day step(s) of the reference's own
    simulate_schedule_ad with its default (direct) linear solver."""
    import time
    from pymrst_b200 import cases
    case = cases.five_spot(dims=(100, 100, 10), seed=1)
    g, rock, w, model = _five_spot_reference(case)
    st0 = model.initial_state(case.p0, case.sw0)
    events = []
    t0 = time.perf_counter()
    states, its = simulate_schedule_ad(st0, model, np.full(nsteps, case.dt), verbose=False,
                                       observer=lambda ev, p: events.append((ev, p.get("dt", 0.0),
                                                                             p.get("iterations", -1))))
    el = time.perf_counter() - t0
    ministeps = np.array([[dt, it, 1.0 if ev == "step_accepted" else 0.0] for ev, dt, it in events
                          if ev in ("step_accepted", "step_rejected")])
    save("cfg1_ow_100x100x10.npz", dims=np.array(case.grid.cartDims), perm_sum=np.array(np.sum(rock.perm)),
         ministeps=ministeps,
         wi_sum=np.array(sum(np.sum(x.WI) for x in w)), its=np.asarray(its),
         p_hist=np.vstack([s.pressure for s in states]), sw_hist=np.vstack([s.sW for s in states]),
         qws_hist=np.vstack([s.qWs for s in states]), qos_hist=np.vstack([s.qOs for s in states]),
         bhp_hist=np.vstack([s.bhp for s in states]), seconds=np.array(el))


def cfg4_fixture(nsteps=30):
    """Benchmark config 4: compute_gradient_adjoint on the 64x64x4 five-spot,
    30 steps of 10 days, objective cumulative produced oil
    (npv_objective(oil_price=1, water_cost=0, water_inj_cost=0)), controls the
    wells' own targets held over the schedule."""
    import time
    from pymrst.modules.optimization.adjoint import compute_gradient_adjoint, npv_objective
    from pymrst_b200 import cases
    case = cases.five_spot(dims=(64, 64, 4), seed=4, nsteps=nsteps)
    g, rock, w, model = _five_spot_reference(case)
    st0 = model.initial_state(case.p0, case.sw0)
    controls = np.tile([float(np.ravel(x.val)[0]) for x in w], (nsteps, 1))
    dts = np.full(nsteps, case.dt)
    t0 = time.perf_counter()
    res = compute_gradient_adjoint(model, st0, dts, controls,
                                   npv_objective(oil_price=1.0, water_cost=0.0, water_inj_cost=0.0))
    el = time.perf_counter() - t0
    save("cfg4_adjoint_64x64x4.npz", dims=np.array(case.grid.cartDims), perm_sum=np.array(np.sum(rock.perm)),
         controls=controls, dts=dts, value=np.array(res.value), gradient=res.gradient,
         p_final=res.states[-1].pressure, sw_final=res.states[-1].sW, seconds=np.array(el))



def _bo_deck_arrays(deck):
    """The deck's tables as flat arrays (pvto rows stacked with their key)."""
    keys = np.array([k for k, _ in deck["pvto"]])
    nrows = np.array([len(r) for _, r in deck["pvto"]])
    rows = np.vstack([r for _, r in deck["pvto"]])
    w, r = deck["pvtw"], deck["rock_cp"]
    return dict(pvtw=np.array([w["p_ref"], w["b_ref"], w["c"], w["mu_ref"], w["viscosibility"]]),
                rock_cp=np.array([r["p_ref"], r["c"]]), pvdg=deck["pvdg"], pvto_keys=keys,
                pvto_nrows=nrows, pvto_rows=rows, swof=deck["swof"], sgof=deck["sgof"], rhoS=deck["rhoS"])


def _bo_model(dims, phys, seed, wells_spec):
    """The reference's ThreePhaseBlackOilModelAD on a box grid with the
    synthetic deck; layered lognormal permeability."""
    from pymrst.modules.ad_blackoil.models.three_phase_black_oil_model import ThreePhaseBlackOilModelAD
    from pymrst.modules.ad_props.props.init_deck_adi_fluid import init_deck_blackoil_fluid
    from pymrst_b200.cases import synthetic_blackoil_deck
    deck = synthetic_blackoil_deck()
    g = compute_geometry(cart_grid(dims, phys))
    layer = np.array([500.0, 50.0, 200.0, 120.0])[np.arange(dims[2]) % 4]
    perm = lognormal_perm(dims, seed, sigma=0.5, mean_md=1.0) * np.repeat(layer, dims[0] * dims[1])
    rock = make_rock(g, perm[:, None], 0.3)
    fluid = init_deck_blackoil_fluid(deck)
    nx, ny = dims[0], dims[1]
    wells = None
    for (i, j, ks, wtype, val, compi) in wells_spec:
        cells = np.array([i + nx * (j + ny * k) for k in ks])
        wells = add_well(wells, g, rock, cells, well_type=wtype, val=val, radius=0.1,
                         compi=np.asarray(compi, float), sign=1 if compi[2] > 0 or compi[0] > 0 else -1)
    model = ThreePhaseBlackOilModelAD(g, rock, fluid, wells)
    return deck, g, rock, perm, model


def _bo_initial_state(model, g, p_top=300.0 * BARSA, sw=0.2, rs=120.0):
    from pymrst.modules.ad_blackoil.models.three_phase_black_oil_model import BOState
    nc, nw = g.cells.num, len(model.wells)
    z = g.cells.centroids[:, 2]
    p = p_top + 840.0 * 1.1 * 9.80665 * z
    s = np.column_stack([np.full(nc, sw), np.full(nc, 1.0 - sw), np.zeros(nc)])
    qws, qos, qgs, bhp = np.zeros(nw), np.zeros(nw), np.zeros(nw), np.zeros(nw)
    for k, w in enumerate(model.wells):
        if w.type == "orat":
            qos[k], bhp[k] = w.val, p.mean() - 10 * BARSA
        elif w.type == "rate":
            qws[k], qgs[k], bhp[k] = w.val * w.compi[0], w.val * w.compi[2], p.mean() + 10 * BARSA
        else:
            bhp[k] = w.val
    return BOState(pressure=p, s=s, rs=np.full(nc, rs), status=np.ones(nc, dtype=np.int64),
                   qWs=qws, qOs=qos, qGs=qgs, bhp=bhp)


def _bo_save_common(out, deck, dims, phys, perm, model):
    out.update(_bo_deck_arrays(deck))
    out.update(dims=np.array(dims), phys=np.array(phys), perm=perm, poro=np.array(0.3))
    out.update(wells_arrays("w", model.wells))
    return out


def _bo_state_arrays(prefix, st):
    return {prefix + "p": st.pressure, prefix + "s": st.s, prefix + "rs": st.rs, prefix + "status": st.status,
            prefix + "qWs": st.qWs, prefix + "qOs": st.qOs, prefix + "qGs": st.qGs, prefix + "bhp": st.bhp}


BO_WELLS = [(0, 0, (0, 1), "rate", 5.0, (0.0, 0.0, 1.0)),
            (9, 9, (1, 2), "orat", -0.012, (0.0, 1.0, 0.0)),
            (9, 0, (2,), "bhp", 250.0 * BARSA, (0.0, 1.0, 0.0))]


def bo_assemble_fixture():
    """Residual and Jacobian of the reference's assemble at an iterate with
    saturated and undersaturated cells, a cross-flowing bhp well (its top
    perforation injects, its bottom one produces) and every control type."""
    from pymrst.modules.ad_blackoil.models.three_phase_black_oil_model import BOState
    dims, phys = [6, 5, 4], [180.0, 150.0, 40.0]
    spec = [(0, 0, (0, 1), "rate", 5.0, (0.0, 0.0, 1.0)),
            (5, 4, (2, 3), "orat", -0.012, (0.0, 1.0, 0.0)),
            (5, 0, (0, 1, 2, 3), "bhp", 0.0, (0.0, 1.0, 0.0))]
    deck, g, rock, perm, model = _bo_model(dims, phys, 21, spec)
    st0 = _bo_initial_state(model, g)
    rng = np.random.default_rng(22)
    nc = g.cells.num
    xf = model.wells[2]
    pw = st0.pressure[xf.cells]
    xf.val = float(0.5 * (pw[1] + pw[2]))      # between the 2nd and 3rd perforation pressures
    st0.bhp[2] = xf.val
    st = st0.copy()
    st.pressure = st.pressure + rng.uniform(-2, 2, nc) * BARSA
    sat = rng.random(nc) < 0.4
    st.status = np.where(sat, 3, 1).astype(np.int64)
    sg = np.where(sat, rng.uniform(0.01, 0.2, nc), 0.0)
    swv = st.s[:, 0] + rng.uniform(-0.03, 0.05, nc)
    st.s = np.column_stack([swv, 1.0 - swv - sg, sg])
    rs_sat = np.asarray(model.fluid.rs_sat(st.pressure))
    st.rs = np.where(sat, rs_sat, 120.0 + rng.uniform(-20, 5, nc))
    bub = ~sat & (rng.random(nc) < 0.4)           # undersaturated cells at their bubble point
    st.rs[bub] = rs_sat[bub]
    st.qWs = np.array([0.0, 0.0, 0.0])
    st.qOs = np.array([0.0, -0.011, -0.004])
    st.qGs = np.array([4.8, -0.9, -0.3])
    st.bhp = np.array([st0.pressure.mean() + 12 * BARSA, st0.pressure.mean() - 9 * BARSA, xf.val])
    out = _bo_save_common({}, deck, dims, phys, perm, model)
    for tag, (a, b, dt) in {"a": (st0, st, 5 * DAY), "b": (st, st0, 2 * DAY)}.items():
        x_val = np.where(b.status == 1, b.rs, b.s[:, 2])
        ad = init_variables_adi(b.pressure, b.s[:, 0], x_val, b.qWs, b.qOs, b.qGs, b.bhp)
        eqs = model.assemble(a, b, *ad, dt)
        eq = combine_equations(*eqs)
        jac = eq.jac[0].tocsr()
        jac.sort_indices()
        out.update(_bo_state_arrays(tag + "0_", a))
        out.update(_bo_state_arrays(tag + "_", b))
        out[tag + "_dt"] = np.array(dt)
        out[tag + "_res"] = np.asarray(eq.val)
        out[tag + "_jac_data"], out[tag + "_jac_indices"], out[tag + "_jac_indptr"] = jac.data, jac.indices, jac.indptr
        out[tag + "_converged"] = np.array(model._converged(eqs, dt, b))
        upd = np.linspace(-1.0, 1.0, jac.shape[0]) * np.concatenate(
            [np.full(nc, 3 * BARSA), np.full(nc, 0.05), np.where(b.status == 1, 5.0, 0.04),
             np.full(4 * len(model.wells), 0.01)])
        new = model.update_state(b, upd)
        out[tag + "_upd"] = upd
        out.update(_bo_state_arrays(tag + "_new_", new))
    save("bo_assemble.npz", **out)


def bo_newton_fixture(nsteps_days=(0.5, 1.0, 2.0, 5.0, 10.0, 10.0, 20.0)):
    """Newton histories of the reference's step on a 10x10x3 box with a gas
    injector (rate), an oil-rate producer (orat) and a bhp producer."""
    dims, phys = [10, 10, 3], [300.0, 300.0, 30.0]
    deck, g, rock, perm, model = _bo_model(dims, phys, 23, BO_WELLS)
    st = _bo_initial_state(model, g)
    out = _bo_save_common({}, deck, dims, phys, perm, model)
    out.update(_bo_state_arrays("init_", st))
    its, hist = [], []
    for dt in np.asarray(nsteps_days) * DAY:
        st, ok, it = model.step(st, float(dt))
        assert ok, "reference step did not converge"
        its.append(it)
        hist.append(st.copy())
    out["dts"] = np.asarray(nsteps_days) * DAY
    out["its"] = np.array(its)
    for name in ("pressure", "rs", "qWs", "qOs", "qGs", "bhp"):
        out["hist_" + name] = np.array([getattr(h, name) for h in hist])
    out["hist_s"] = np.array([h.s for h in hist])
    out["hist_status"] = np.array([h.status for h in hist])
    save("bo_newton.npz", **out)


def transport_fixture():
    """validate_phase3.py's three cases (Buckley-Leverett 100x1x1 with fixed
    and computed explicit substeps and implicit transport; two sequential
    incomp_tpfa + implicit cycles on a 32x32 quarter five-spot; gravity
    segregation in a 20-cell column) run by the reference, with the MATLAB
    arrays (ref_p3_bl.mat, ref_p3_qfs.mat, ref_p3_gravity.mat)."""
    from pymrst.modules.incomp import explicit_transport, implicit_transport, incomp_tpfa_ad, init_simple_fluid
    from pymrst.params import add_source, gravity_vector, pore_volume
    from pymrst.solvers import init_res_sol
    fluid = init_simple_fluid(mu=np.array([1.0, 10.0]) * CENTI * POISE, rho=[1000.0, 700.0], n=[2.0, 2.0])
    out = {}
    # Buckley-Leverett
    mb = scipy.io.loadmat(REF / "examples/validation/ref_p3_bl.mat", squeeze_me=True)
    g = compute_geometry(cart_grid([100, 1, 1], [100.0, 1.0, 1.0]))
    rock = make_rock(g, 100 * MILLI * DARCY, 0.2)
    ht = compute_trans(g, rock)
    rate = float(pore_volume(g, rock).sum()) / (100 * DAY)
    src = add_source(None, np.array([0]), rate, sat=np.array([[1.0, 0.0]]))
    src = add_source(src, np.array([99]), -rate, sat=np.array([[0.0, 1.0]]))
    new = lambda: incomp_tpfa_ad(init_res_sol(g, 0.0, s0=np.array([[0.0, 1.0]])), g, ht, fluid, src=src)
    st = new()
    out.update(bl_rate=np.array(rate), bl_p0=st.pressure, bl_flux0=st.flux)
    out["bl_sE"] = explicit_transport(new(), g, 30 * DAY, rock, fluid, src=src, dt=0.25 * DAY).s[:, 0]
    out["bl_sE_auto"] = explicit_transport(new(), g, 30 * DAY, rock, fluid, src=src).s[:, 0]
    out["bl_sI"] = implicit_transport(new(), g, 30 * DAY, rock, fluid, src=src).s[:, 0]
    for k in ("p0", "flux0", "sE", "sI"):
        out["bl_mat_" + k] = np.asarray(mb[k], float).ravel()
    # quarter five-spot, two sequential cycles
    mq = scipy.io.loadmat(REF / "examples/validation/ref_p3_qfs.mat", squeeze_me=True)
    g = compute_geometry(cart_grid([32, 32, 1], [500.0, 500.0, 10.0]))
    kvals = (10 + (7 * np.arange(g.cells.num)) % 100) * MILLI * DARCY
    rock = make_rock(g, kvals[:, None], 0.2)
    ht = compute_trans(g, rock)
    src = add_source(None, np.array([0]), 5e-3, sat=np.array([[1.0, 0.0]]))
    src = add_source(src, np.array([g.cells.num - 1]), -5e-3, sat=np.array([[0.0, 1.0]]))
    st = init_res_sol(g, 0.0, s0=np.array([[0.0, 1.0]]))
    for _ in range(2):
        st = incomp_tpfa_ad(st, g, ht, fluid, src=src)
        st = implicit_transport(st, g, 100 * DAY, rock, fluid, src=src)
    out.update(qfs_sQ=st.s[:, 0], qfs_pQ=st.pressure, qfs_mat_sQ=np.asarray(mq["sQ"], float).ravel(),
               qfs_mat_pQ=np.asarray(mq["pQ"], float).ravel())
    # gravity segregation, implicit (the MATLAB case) and explicit with computed substeps
    mg = scipy.io.loadmat(REF / "examples/validation/ref_p3_gravity.mat", squeeze_me=True)
    g = compute_geometry(cart_grid([1, 1, 20], [1.0, 1.0, 20.0]))
    rock = make_rock(g, 1000 * MILLI * DARCY, 0.3)
    gfluid = init_simple_fluid(mu=[1e-3, 1e-3], rho=[1000.0, 700.0], n=[2.0, 2.0])

    def col():
        s0 = init_res_sol(g, 0.0, s0=np.array([[0.5, 0.5]]))
        s0.flux = np.zeros(g.faces.num)
        return s0
    out["grav_sG"] = implicit_transport(col(), g, 50 * DAY, rock, gfluid, gravity=gravity_vector(3)).s[:, 0]
    out["grav_sE_auto"] = explicit_transport(col(), g, 5 * DAY, rock, gfluid, gravity=gravity_vector(3)).s[:, 0]
    out["grav_mat_sG"] = np.asarray(mg["sG"], float).ravel()
    save("transport_phase3.npz", **out)


def geometry_fixture():
    """compute_geometry on a 5x4x3 grid with seeded perturbed nodes
    (non-planar faces), without and with hinge points on four faces: the
    topology arrays and the reference's face and cell geometry."""
    g = cart_grid([5, 4, 3], [50.0, 40.0, 6.0])
    rng = np.random.default_rng(11)
    g.nodes.coords = g.nodes.coords + rng.uniform(-0.15, 0.15, g.nodes.coords.shape) * np.array([10.0, 10.0, 2.0])
    out = dict(coords=g.nodes.coords, node_pos=g.faces.nodePos, nodes=g.faces.nodes, face_pos=g.cells.facePos,
               cell_faces=g.cells.faces, neighbors=g.faces.neighbors)
    hf = np.array([0, 7, 31, 50])
    hn = np.array([g.nodes.coords[g.faces.nodes[g.faces.nodePos[f]:g.faces.nodePos[f + 1]]].mean(axis=0)
                   for f in hf]) + np.array([0.3, -0.2, 0.1])
    for tag, hinge in (("plain", None), ("hinge", {"faces": hf, "nodes": hn})):
        r = compute_geometry(g, hinge_nodes=hinge)
        out.update({f"{tag}_face_areas": r.faces.areas, f"{tag}_face_normals": r.faces.normals,
                    f"{tag}_face_centroids": r.faces.centroids, f"{tag}_cell_volumes": r.cells.volumes,
                    f"{tag}_cell_centroids": r.cells.centroids})
    out.update(hinge_faces=hf, hinge_nodes=hn)
    save("geometry3d.npz", **out)


if __name__ == "__main__":
    def want(name):
        return ONLY is None or name in ONLY

    if want("small"):
        grid_fixture()
        assemble_fixture("ow_assemble_nograv.npz", [6, 5, 3], [60.0, 50.0, 6.0], 3, "p5", 0.0, False)
        assemble_fixture("ow_assemble_grav.npz", [6, 5, 4], [60.0, 50.0, 8.0], 4, "cfg", 9.80665, False)
        assemble_fixture("ow_assemble_xflow.npz", [5, 5, 6], [50.0, 50.0, 30.0], 5, "cfg", 9.80665, True)
        newton_fixture("ow_newton_grav.npz", [8, 6, 4], [80.0, 60.0, 8.0], 6, "cfg", 9.80665, 4, 10.0)
        newton_fixture("ow_newton_nograv.npz", [10, 8, 3], [100.0, 80.0, 6.0], 7, "p5", 0.0, 4, 20.0)
        phase5_fixture()
        incomp_fixtures()
        adjoint_fixture("adjoint_grav.npz", [7, 6, 3], [70.0, 60.0, 6.0], 8, "cfg", 9.80665, 4, 15.0)
        adjoint_fixture("adjoint_nograv.npz", [8, 5, 2], [80.0, 50.0, 4.0], 9, "p5", 0.0, 3, 20.0)
    if want("cfg0"):
        cfg0_fixture()
    if want("cfg4"):
        cfg4_fixture()
    if want("cfg1"):
        cfg1_fixture()
    if want("transport"):
        transport_fixture()
    if want("bo"):
        bo_assemble_fixture()
        bo_newton_fixture()
    if want("geometry"):
        geometry_fixture()
