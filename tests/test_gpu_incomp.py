"""Incompressible TPFA on the GPU against the reference's MATLAB goldens
(the validate_phase2 cases, tolerance rtol 1e-9 with atol 1e-9 of the field
maximum, as the reference checks them) and the reference's own incomp_tpfa
on a case with wells."""

import numpy as np
import pytest

from fixtures import load, wells_from

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from pymrst_b200.build import build  # noqa: E402
from pymrst_b200.grid import cartesian_grid  # noqa: E402
from pymrst_b200.incomp import GpuLinSolve, incomp_tpfa, init_single_fluid, init_state  # noqa: E402
from pymrst_b200.ow_model import face_transmissibility_device  # noqa: E402
from pymrst_b200.params import (BARSA, CENTI, DARCY, MILLI, POISE, add_bc, add_source, add_well,  # noqa: E402
                                make_rock)

build()
FLUID = init_single_fluid(1 * CENTI * POISE, 1000.0)
GVEC = np.array([0.0, 0.0, 9.80665])
SOLVE = GpuLinSolve(rtol=1e-14, maxiter=2000)


def close(mine, ref, rtol=1e-9):
    mine = np.asarray(mine, float).ravel()
    ref = np.asarray(ref, float).ravel()
    scale = max(np.abs(ref).max(), 1e-300)
    np.testing.assert_allclose(mine, ref, rtol=rtol, atol=rtol * scale + 1e-15)


def half_trans(g, rock):
    return face_transmissibility_device(g, rock)[1]


def test_qfs_sources_match_matlab():
    m = load("incomp_matlab.npz")
    g = cartesian_grid([32, 32, 1], [500.0, 500.0, 10.0])
    k = (10 + (7 * np.arange(g.cells.num)) % 100) * MILLI * DARCY
    rock = make_rock(g, k[:, None], 0.2)
    ht = half_trans(g, rock)
    close(ht, m["qfs__hT"], 1e-12)
    src = add_source(None, [0], 1e-3)
    src = add_source(src, [g.cells.num - 1], -1e-3)
    st = incomp_tpfa(init_state(g, None, 0.0), g, ht, FLUID, src=src, LinSolve=SOLVE)
    close(st.pressure, m["qfs__p"])
    close(st.flux, m["qfs__flux"])
    close(st.facePressure, m["qfs__fp"])


def test_pressure_and_flux_bc_match_matlab():
    m = load("incomp_matlab.npz")
    g = cartesian_grid([20, 10, 5], [200.0, 100.0, 50.0])
    k = (1 + (3 * np.arange(g.cells.num)) % 50) * MILLI * DARCY
    rock = make_rock(g, k[:, None], 0.25)
    ht = half_trans(g, rock)
    bd = np.any(g.faces.neighbors == -1, axis=1)
    fc = g.faces.centroids
    bc = add_bc(None, np.flatnonzero(bd & (fc[:, 0] < 1e-10)), "pressure", 200 * BARSA)
    bc = add_bc(bc, np.flatnonzero(bd & (fc[:, 0] > 200 - 1e-10)), "pressure", 100 * BARSA)
    bc = add_bc(bc, np.flatnonzero(bd & (fc[:, 1] < 1e-10)), "flux", 1e-6)
    st = incomp_tpfa(init_state(g, None, 0.0), g, ht, FLUID, bc=bc, LinSolve=SOLVE)
    close(st.pressure, m["bc__p"])
    close(st.flux, m["bc__flux"])
    close(st.facePressure, m["bc__fp"])


def test_wells_with_gravity_match_matlab():
    m = load("incomp_matlab.npz")
    g = cartesian_grid([10, 10, 3], [1000.0, 1000.0, 30.0])
    k = np.tile(np.array([100.0, 100.0, 10.0]) * MILLI * DARCY, (g.cells.num, 1))
    rock = make_rock(g, k, 0.3)
    ht = half_trans(g, rock)
    w = add_well(None, g, rock, [0, 100, 200], well_type="rate", val=5e-3, radius=0.1,
                 compi=np.array([1.0]), gravity=GVEC)
    w = add_well(w, g, rock, [99, 199, 299], well_type="bhp", val=100 * BARSA, radius=0.1,
                 compi=np.array([1.0]), gravity=GVEC)
    close(w[0].WI, m["wells__wi1"], 1e-12)
    close(w[0].dZ, m["wells__dz1"], 1e-12)
    st = incomp_tpfa(init_state(g, w, 0.0), g, ht, FLUID, wells=w, gravity=GVEC, LinSolve=SOLVE)
    close(st.pressure, m["wells__p"])
    close(st.flux, m["wells__flux"])
    close(st.wellSol[0].flux, m["wells__wflux1"])
    close(st.wellSol[1].flux, m["wells__wflux2"])
    close([st.wellSol[0].pressure], m["wells__bhp1"])
    close([st.wellSol[1].pressure], m["wells__bhp2"])


def test_gravity_column_matches_matlab():
    m = load("incomp_matlab.npz")
    g = cartesian_grid([1, 1, 30], [1.0, 1.0, 300.0])
    rock = make_rock(g, 100 * MILLI * DARCY, 0.2)
    ht = half_trans(g, rock)
    bd = np.any(g.faces.neighbors == -1, axis=1)
    top = np.flatnonzero(bd & (g.faces.centroids[:, 2] < 1e-10))
    bc = add_bc(None, top, "pressure", 100 * BARSA)
    st = incomp_tpfa(init_state(g, None, 0.0), g, ht, FLUID, bc=bc, gravity=GVEC, LinSolve=SOLVE)
    close(st.pressure, m["gravity__p"])
    close(st.flux, m["gravity__flux"])


def test_default_device_solve_matches_reference_incomp_tpfa():
    d = load("incomp_wells.npz")
    g = cartesian_grid(d["dims"], [160.0, 160.0, 8.0])
    rock = make_rock(g, d["perm"][:, None], 0.2)
    ht = half_trans(g, rock)
    np.testing.assert_allclose(ht, d["hT"], rtol=1e-13)
    wells = wells_from(d)
    st = incomp_tpfa(init_state(g, wells, 0.0), g, ht, FLUID, wells=wells)
    close(st.pressure, d["p"], 1e-8)
    close(st.flux, d["flux"], 1e-8)
    close([ws.pressure for ws in st.wellSol], d["bhp"], 1e-8)
