"""The drop-in CPR solver (`GpuCPRSolver`, the reference's `CPRSolver.solve`
protocol) on the reference's own Jacobians.

The pin is the reference's: CPR with rtol 1e-10 equals the direct solve to
1e-7 of the solution's maximum (linear_solvers.py test
`test_cpr_reproduces_the_direct_solution`).  Newton histories driven through
the drop-in with rtol 1e-12 reproduce the reference's iteration counts and
states (p 1e-8 relative, sW 1e-7).
"""

from types import SimpleNamespace

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from fixtures import load, ow_case

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from pymrst_b200 import _native as N  # noqa: E402
from pymrst_b200.build import build  # noqa: E402
from pymrst_b200.linear_solvers import GpuCPRSolver  # noqa: E402

from oracle import ow as oow  # noqa: E402

build()


def _jacobian(d):
    J = sp.csr_array((d["J_data"], d["J_indices"], d["J_indptr"]), shape=tuple(d["J_shape"]))
    return J, -d["res"]


def _model(d):
    g, rock, fluid, wells = ow_case(d)
    return SimpleNamespace(G=g, n_phases=2, fluid=fluid), (g, rock, fluid, wells)


@pytest.mark.parametrize("name", ["ow_assemble_grav.npz", "ow_assemble_nograv.npz", "ow_assemble_xflow.npz"])
def test_spmv_matches_the_reference_jacobian(name):
    d = load(name)
    J, _ = _jacobian(d)
    J = J.copy()
    J.sum_duplicates()  # the C-ABI takes canonical CSR (the reference's may be unsorted)
    n = J.shape[0]
    model, _ = _model(d)
    rp = np.ascontiguousarray(J.indptr, dtype=np.int32)
    ci = np.ascontiguousarray(J.indices, dtype=np.int32)
    o = N.CPROpts()
    N.check(N.lib().pmb_cpr_default_opts(N.C.byref(o)))
    h = N.c_vp()
    N.check(N.lib().pmb_csr_cpr_create(n, model.G.cells.num, 2, N.as_p(rp, N.C.c_int32), N.as_p(ci, N.C.c_int32),
                                       0, N.C.byref(o), None, N.C.byref(h)))
    try:
        x = np.random.default_rng(0).standard_normal(n)
        vals = torch.as_tensor(J.data, device="cuda")
        xd = torch.as_tensor(x, device="cuda")
        yd = torch.empty_like(xd)
        N.check(N.lib().pmb_csr_spmv(h, N.ptr(vals), N.ptr(xd), N.ptr(yd)))
        torch.cuda.synchronize()
        ref = J @ x
        assert np.abs(yd.cpu().numpy() - ref).max() <= 1e-13 * np.abs(ref).max()
    finally:
        N.lib().pmb_csr_cpr_destroy(h)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", ["ow_assemble_grav.npz", "ow_assemble_nograv.npz", "ow_assemble_xflow.npz"])
def test_cpr_reproduces_the_direct_solution(name, precision):
    d = load(name)
    J, rhs = _jacobian(d)
    model, _ = _model(d)
    solver = GpuCPRSolver(rtol=1e-10, precision=precision)
    got = solver.solve(J, rhs, model, {"pressure": d["p"]}, float(d["dt"]))
    exact = spla.spsolve(J.tocsc(), rhs)
    err = np.abs(got - exact).max() / np.abs(exact).max()
    assert err < 1e-7, f"CPR is not the direct solution: {err:.2e}"
    assert solver.last_iterations > 0 and solver.last_relres <= 1e-10
    assert solver.last_local_stage == "block_jacobi"
    assert solver.last_fallback == ()


def test_pattern_reuse_and_duplicate_entries():
    d = load("ow_assemble_grav.npz")
    J, rhs = _jacobian(d)
    model, _ = _model(d)
    solver = GpuCPRSolver(rtol=1e-10)
    x1 = solver.solve(J, rhs, model, {"pressure": d["p"]})
    h1 = dict(solver._handles)
    # the same matrix with every entry split into two halves (a non-canonical CSR)
    coo = J.tocoo()
    dup = sp.coo_array((np.concatenate([coo.data * 0.5, coo.data * 0.5]),
                        (np.concatenate([coo.row, coo.row]), np.concatenate([coo.col, coo.col]))),
                       shape=J.shape).tocsr()
    x2 = solver.solve(dup, rhs, model, {"pressure": d["p"]})
    assert solver._handles == h1  # same pattern after summing duplicates: handles kept
    assert np.abs(x2 - x1).max() <= 1e-8 * np.abs(x1).max()


def test_singular_cell_block_is_an_error_not_a_fault():
    d = load("ow_assemble_nograv.npz")
    J, rhs = _jacobian(d)
    model, _ = _model(d)
    nc = model.G.cells.num
    J = J.tolil()
    c = 3
    for i in (c, nc + c):
        for j in (c, nc + c):
            J[i, j] = 0.0
    J = sp.csr_array(J)
    with pytest.raises(RuntimeError, match="singular cell block"):
        GpuCPRSolver(rtol=1e-10).solve(J, rhs, model, {"pressure": d["p"]})


@pytest.mark.parametrize("name", ["ow_newton_grav.npz", "ow_newton_nograv.npz"])
def test_newton_through_the_drop_in_matches_reference(name):
    """The reference's Newton loop (oracle restatement) with the linear solve
    plugged through GpuCPRSolver, as `TwoPhaseOilWaterModelAD(linear_solver=...)`
    does it (two_phase_oil_water_model.py:599-603)."""
    d = load(name)
    model, (g, rock, fluid, wells) = _model(d)
    prob = oow.build_problem(g, rock, fluid.params, wells, gravity=float(d["gravity"]))
    solver = GpuCPRSolver(rtol=1e-12, maxiter=400)
    st = oow.initial_state(prob, float(d["p0"][0]), float(d["sw0"][0]))
    dt = float(d["dt_days"]) * 86400.0
    for k in range(int(d["nsteps"])):
        st0 = st
        st = st0.copy()
        cdp = oow.compute_cdp(prob, st0)
        its = None
        for it in range(prob.max_iterations):
            res, J = oow.assemble(prob, st0, st, dt, cdp)
            if oow.converged(prob, res, dt, st)[0]:
                its = it
                break
            upd = solver.solve(J, -res, model, {"pressure": st.pressure})
            oow.apply_update(prob, st, upd)
        assert its == int(d["its"][k])
        assert np.abs(st.pressure - d["p_hist"][k]).max() <= 1e-8 * np.abs(d["p_hist"][k]).max()
        assert np.abs(st.sW - d["sw_hist"][k]).max() <= 1e-7


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", ["ow_assemble_grav.npz", "ow_assemble_nograv.npz", "ow_assemble_xflow.npz"])
def test_transposed_solve_matches_the_direct_adjoint_solve(name, precision):
    """J^T x = b, the adjoint solve that compute_gradient_adjoint does with
    spsolve (optimization/adjoint.py:209), to the same 1e-7 bar."""
    d = load(name)
    J, rhs = _jacobian(d)
    model, _ = _model(d)
    solver = GpuCPRSolver(rtol=1e-10, precision=precision)
    got = solver.solve_transposed(J, rhs, model, {"pressure": d["p"]})
    exact = spla.spsolve(sp.csc_matrix(J.T), rhs)
    err = np.abs(got - exact).max() / np.abs(exact).max()
    assert err < 1e-7, f"transposed CPR is not the direct solution: {err:.2e}"
    assert solver.last_relres <= 1e-10
