"""Incompressible TPFA on the GPU against the reference's MATLAB goldens
(the validate_phase2 cases, tolerance rtol 1e-9 with atol 1e-9 of the field
maximum, as the reference checks them), the reference's own incomp_tpfa on
a case with wells and on the 64x64x8 benchmark case, and the oracle's
matrix and right-hand side (device assembly, entry by entry)."""

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


# ---- the device assembly and reconstruction (pmb_tpfa_*) -------------------------------

from oracle import incomp as oinc  # noqa: E402
from test_oracle import _incomp_matlab_cases  # noqa: E402


@pytest.mark.parametrize("case", ["qfs", "bc", "wells", "gravity"])
def test_device_path_matches_matlab(case):
    """Assembly, PCG solve and reconstruction all on the device."""
    m = load("incomp_matlab.npz")
    g, ht, bc, src, wells, gz = _incomp_matlab_cases()[case]
    st = incomp_tpfa(init_state(g, wells, 0.0), g, ht, FLUID, bc=bc, src=src, wells=wells, gravity=gz,
                     rtol=1e-14, maxiter=3000)
    close(st.pressure, m[case + "__p"])
    close(st.flux, m[case + "__flux"])
    if case in ("qfs", "bc"):
        close(st.facePressure, m[case + "__fp"])
    if case == "wells":
        close(st.wellSol[0].flux, m["wells__wflux1"])
        close(st.wellSol[1].flux, m["wells__wflux2"])
        close([ws.pressure for ws in st.wellSol], np.concatenate([m["wells__bhp1"], m["wells__bhp2"]]))


def _matrix_vs_oracle(g, ht, bc, src, wells, gz, use_trans=False, mob=None, rho=(1000.0,), fluid=FLUID):
    st = incomp_tpfa(init_state(g, wells, 0.0), g, ht, fluid, bc=bc, src=src, wells=wells, gravity=gz,
                     MatrixOutput=True, use_trans=use_trans, rtol=1e-13, maxiter=3000)
    if mob is None:
        mob = np.full((g.cells.num, 1), 1.0 / (1 * CENTI * POISE))
    A, rhs, aux = oinc.pressure_system(g, ht, mob, rho, gz, bc, src, wells, use_trans)
    D = (st.A - A).tocsr()
    scale = np.abs(A.data).max()
    assert (np.abs(D.data).max() if D.nnz else 0.0) <= 1e-13 * scale
    np.testing.assert_allclose(st.rhs, rhs, rtol=1e-12, atol=1e-13 * np.abs(rhs).max())
    p = np.linalg.solve(A.toarray(), rhs) if A.shape[0] < 4000 else None
    return st, p, aux


@pytest.mark.parametrize("case", ["qfs", "bc", "wells", "gravity"])
def test_device_matrix_and_rhs_equal_oracle(case):
    g, ht, bc, src, wells, gz = _incomp_matlab_cases()[case]
    _matrix_vs_oracle(g, ht, bc, src, wells, gz)


def test_interface_transmissibilities_two_phases_and_pin():
    """use_trans (one T per interface), a two-phase incompressible fluid with
    per-cell mobilities, sources only (the pressure pin), and a rate well
    whose mixture density follows the fractional flow of its cells."""
    from types import SimpleNamespace
    g = cartesian_grid([7, 5, 3], [70.0, 50.0, 6.0])
    rng = np.random.default_rng(5)
    k = np.exp(rng.normal(np.log(100.0), 0.5, g.cells.num)) * MILLI * DARCY
    rock = make_rock(g, k[:, None], 0.2)
    T = face_transmissibility_device(g, rock)[0]
    sw = rng.uniform(0.0, 1.0, g.cells.num)
    mu = np.array([1.0, 4.0]) * CENTI * POISE

    class TwoPhase:
        def properties(self, state=None):
            return mu, np.array([1000.0, 850.0])

        def saturation(self, state):
            return np.column_stack([sw, 1 - sw])

        def relperm(self, s):
            return s ** 2

    w = add_well(None, g, rock, [3, 38, 73], well_type="rate", val=-2e-4, radius=0.1,
                 compi=np.array([0.0, 1.0]), gravity=GVEC)
    src = add_source(None, [0, 104], [1e-4, 1e-4])
    mob = np.column_stack([sw, 1 - sw]) ** 2 / mu
    st, p, aux = _matrix_vs_oracle(g, T, None, src, w, GVEC, use_trans=True, mob=mob, rho=(1000.0, 850.0),
                                   fluid=TwoPhase())
    fp, flux, wflux = oinc.reconstruct(g, p, aux, w)
    close(st.pressure, p[:g.cells.num], 1e-8)
    close(st.flux, flux, 1e-8)
    close(st.wellSol[0].flux, wflux[0], 1e-8)


def test_reduce_gives_the_same_pressures_and_the_schur_system():
    m = load("incomp_matlab.npz")
    g, ht, bc, src, wells, gz = _incomp_matlab_cases()["wells"]
    st = incomp_tpfa(init_state(g, wells, 0.0), g, ht, FLUID, wells=wells, gravity=gz, reduce=True,
                     rtol=1e-14, maxiter=3000)
    close(st.pressure, m["wells__p"])
    assert st.A.shape == (g.cells.num, g.cells.num) and st.rhs.shape == (g.cells.num,)
    p_r = np.linalg.solve(st.A.toarray(), st.rhs)
    close(p_r, m["wells__p"])


def test_assembly_is_bitwise_repeatable():
    g, ht, bc, src, wells, gz = _incomp_matlab_cases()["wells"]
    a = incomp_tpfa(init_state(g, wells, 0.0), g, ht, FLUID, wells=wells, gravity=gz, MatrixOutput=True)
    b = incomp_tpfa(init_state(g, wells, 0.0), g, ht, FLUID, wells=wells, gravity=gz, MatrixOutput=True)
    assert np.array_equal(a.A.data, b.A.data) and np.array_equal(a.rhs, b.rhs)
    assert np.array_equal(a.pressure, b.pressure) and np.array_equal(a.flux, b.flux)


def test_benchmark_case_64x64x8_matches_reference():
    """Benchmark config 0: 32,768 cells, rate injector and bhp producer down
    opposite corner columns, gravity off; against the reference's own
    incomp_tpfa (SuperLU) output."""
    from pymrst_b200 import cases
    d = load("cfg0_incomp_64x64x8.npz")
    g = cartesian_grid([64, 64, 8], [640.0, 640.0, 16.0])
    perm = np.exp(cases.lognormal_logperm((64, 64, 8), np.random.default_rng(0))).ravel(order="F") * MILLI * DARCY
    rock = make_rock(g, perm[:, None], 0.2)
    ht = half_trans(g, rock)
    np.testing.assert_allclose(ht.sum(), d["hT_sum"], rtol=1e-13)
    wells = wells_from(d)
    st = incomp_tpfa(init_state(g, wells, 0.0), g, ht, FLUID, wells=wells, rtol=1e-14, maxiter=3000)
    close(st.pressure, d["p"])
    close(st.flux, d["flux"])
    close(st.facePressure, d["facePressure"])
    close([ws.pressure for ws in st.wellSol], d["bhp"])
    close(st.wellSol[0].flux, d["wflux0"])
    close(st.wellSol[1].flux, d["wflux1"])
