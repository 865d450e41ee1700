"""GPU parity of the incompressible transport path against the reference's
outputs and the phase-3 MATLAB arrays (tests/golden/transport_phase3.npz)
and against the oracle.

Tolerances follow the reference's own validation (validate_phase3.py): the
explicit saturations with fixed substeps 1e-10 against MATLAB and 1e-12
against the reference; implicit 5e-6 against MATLAB (2e-5 for the two
sequential cycles) and 1e-8 against the reference; residuals and Jacobians
1e-12 against the oracle.
"""

import numpy as np
import pytest
import scipy.sparse as sp

from fixtures import load

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from pymrst_b200 import _native as N  # noqa: E402
from pymrst_b200.build import build  # noqa: E402
from pymrst_b200.grid import cartesian_grid  # noqa: E402
from pymrst_b200.incomp import State, incomp_tpfa  # noqa: E402
from pymrst_b200.ow_model import face_transmissibility_device  # noqa: E402
from pymrst_b200.params import CENTI, DARCY, DAY, MILLI, POISE, add_source, make_rock  # noqa: E402
from pymrst_b200.transport import (explicit_transport, implicit_transport, init_simple_fluid,  # noqa: E402
                                   _prepare)

from test_oracle import transport_problem  # noqa: E402

build()

FLUID = init_simple_fluid(mu=np.array([1.0, 10.0]) * CENTI * POISE, rho=[1000.0, 700.0], n=[2.0, 2.0])
GRAV = np.array([0.0, 0.0, 9.80665])


def _two_phase_state(g, sw, flux=None):
    nc = g.cells.num
    s = np.column_stack([np.full(nc, sw), np.full(nc, 1.0 - sw)])
    return State(pressure=np.zeros(nc), flux=np.zeros(g.faces.num) if flux is None else np.array(flux, float), s=s)


def _bl():
    g = cartesian_grid([100, 1, 1], [100.0, 1.0, 1.0])
    rock = make_rock(g, 100 * MILLI * DARCY, 0.2)
    d = load("transport_phase3.npz")
    rate = float(d["bl_rate"])
    src = add_source(add_source(None, [0], rate, sat=[[1.0, 0.0]]), [99], -rate, sat=[[0.0, 1.0]])
    return g, rock, src, d


def test_buckley_leverett_explicit_fixed_and_computed_substeps():
    g, rock, src, d = _bl()
    st = explicit_transport(_two_phase_state(g, 0.0, d["bl_flux0"]), g, 30 * DAY, rock, FLUID, src=src,
                            dt=0.25 * DAY)
    np.testing.assert_allclose(st.s[:, 0], d["bl_sE"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(st.s[:, 0], d["bl_mat_sE"], rtol=0, atol=1e-10)
    st = explicit_transport(_two_phase_state(g, 0.0, d["bl_flux0"]), g, 30 * DAY, rock, FLUID, src=src)
    np.testing.assert_allclose(st.s[:, 0], d["bl_sE_auto"], rtol=0, atol=1e-12)


def test_buckley_leverett_pressure_then_transport_on_the_device():
    """incomp_tpfa (the device pressure solve) then transport, as
    validate_phase3 runs them: p0, flux0, and both saturations."""
    g, rock, src, d = _bl()
    ht = face_transmissibility_device(g, rock)[1]
    st = incomp_tpfa(_two_phase_state(g, 0.0), g, ht, FLUID, src=src)
    np.testing.assert_allclose(st.pressure, d["bl_mat_p0"], rtol=0, atol=1e-9 * 2e7)
    np.testing.assert_allclose(st.flux, d["bl_mat_flux0"], rtol=0, atol=1e-9 * float(d["bl_rate"]))
    se = explicit_transport(st, g, 30 * DAY, rock, FLUID, src=src, dt=0.25 * DAY).s[:, 0]
    np.testing.assert_allclose(se, d["bl_mat_sE"], rtol=0, atol=1e-10)
    st = incomp_tpfa(_two_phase_state(g, 0.0), g, ht, FLUID, src=src)
    si = implicit_transport(st, g, 30 * DAY, rock, FLUID, src=src).s[:, 0]
    np.testing.assert_allclose(si, d["bl_sI"], rtol=0, atol=1e-8)
    np.testing.assert_allclose(si, d["bl_mat_sI"], rtol=0, atol=5e-6)


def test_gravity_segregation_implicit_and_explicit():
    d = load("transport_phase3.npz")
    g = cartesian_grid([1, 1, 20], [1.0, 1.0, 20.0])
    rock = make_rock(g, 1000 * MILLI * DARCY, 0.3)
    fluid = init_simple_fluid(mu=[1e-3, 1e-3], rho=[1000.0, 700.0], n=[2.0, 2.0])
    st = implicit_transport(_two_phase_state(g, 0.5), g, 50 * DAY, rock, fluid, gravity=GRAV)
    np.testing.assert_allclose(st.s[:, 0], d["grav_sG"], rtol=0, atol=1e-8)
    np.testing.assert_allclose(st.s[:, 0], d["grav_mat_sG"], rtol=0, atol=5e-6)
    st = explicit_transport(_two_phase_state(g, 0.5), g, 5 * DAY, rock, fluid, gravity=GRAV)
    np.testing.assert_allclose(st.s[:, 0], d["grav_sE_auto"], rtol=0, atol=1e-12)


def test_sequential_quarter_five_spot_two_cycles():
    d = load("transport_phase3.npz")
    g = cartesian_grid([32, 32, 1], [500.0, 500.0, 10.0])
    rock = make_rock(g, ((10 + (7 * np.arange(g.cells.num)) % 100) * MILLI * DARCY)[:, None], 0.2)
    ht = face_transmissibility_device(g, rock)[1]
    src = add_source(add_source(None, [0], 5e-3, sat=[[1.0, 0.0]]), [g.cells.num - 1], -5e-3, sat=[[0.0, 1.0]])
    st = _two_phase_state(g, 0.0)
    for _ in range(2):
        st = incomp_tpfa(st, g, ht, FLUID, src=src)
        st = implicit_transport(st, g, 100 * DAY, rock, FLUID, src=src)
    np.testing.assert_allclose(st.s[:, 0], d["qfs_sQ"], rtol=0, atol=1e-7)
    np.testing.assert_allclose(st.s[:, 0], d["qfs_mat_sQ"], rtol=0, atol=2e-5)
    np.testing.assert_allclose(st.pressure, d["qfs_mat_pQ"], rtol=0, atol=1e-6 * np.abs(d["qfs_mat_pQ"]).max())


@pytest.mark.parametrize("case", ["bl", "qfs", "grav"])
def test_residual_and_jacobian_match_the_oracle(case):
    """At random saturations (both flow directions of every phase occur on
    the gravity column), with a random previous state and step."""
    rng = np.random.default_rng(7)
    prob, s0, _, g, internal = transport_problem(case)
    if prob.v is None:
        prob.v = rng.normal(size=int(internal.sum())) * 1e-4
    nc = g.cells.num
    s = rng.uniform(0.0, 1.0, nc)
    sprev = rng.uniform(0.0, 1.0, nc)
    dt = 3.0 * DAY
    rock = make_rock(g, 100 * MILLI * DARCY, 0.2)
    fluid = init_simple_fluid(prob.fluid.mu, prob.fluid.rho, prob.fluid.n)
    flux = np.zeros(g.faces.num)
    flux[internal] = prob.v
    st = _two_phase_state(g, 0.0, flux)
    st.s = np.column_stack([sprev, 1 - sprev])
    hd, d_s, params, gvec, _, keep = _prepare(st, g, rock, fluid, None, None, None, None)
    # the oracle problem's own q, gravity flux and pore volumes, on the device
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda")
    d_v, d_gf, d_q = dev(prob.v), dev(prob.g), dev(prob.q)
    N.check(N.lib().pmb_transport_set_flow(hd, N.ptr(d_v), N.ptr(d_gf), N.ptr(d_q), N.as_p(params, N.C.c_double)))
    # pore volumes differ between rock above and the oracle's: use a handle built on the oracle's
    hd2 = N.c_vp()
    Nn = np.ascontiguousarray(prob.N, dtype=np.int32)
    pv = np.ascontiguousarray(prob.pv, dtype=np.float64)
    N.check(N.lib().pmb_transport_create(nc, Nn.shape[0], N.as_p(Nn, N.C.c_int32), N.as_p(pv, N.C.c_double),
                                         torch.cuda.current_stream().cuda_stream, N.C.byref(hd2)))
    try:
        N.check(N.lib().pmb_transport_set_flow(hd2, N.ptr(d_v), N.ptr(d_gf), N.ptr(d_q),
                                               N.as_p(params, N.C.c_double)))
        ds, ds0, res = dev(s), dev(sprev), torch.empty(nc, dtype=torch.float64, device="cuda")
        amax = N.C.c_double()
        N.check(N.lib().pmb_transport_residual(hd2, N.ptr(ds), N.ptr(ds0), dt, N.ptr(res), N.C.byref(amax)))
        r = res.cpu().numpy()
        want = prob.residual(s, sprev, dt)
        np.testing.assert_allclose(r, want, rtol=0, atol=1e-12 * np.abs(want).max())
        assert amax.value == np.abs(r).max()
        nnz = N.C.c_int64()
        N.check(N.lib().pmb_transport_pattern(hd2, N.C.byref(nnz), None, None))
        rp = np.empty(nc + 1, np.int32)
        ci = np.empty(nnz.value, np.int32)
        N.check(N.lib().pmb_transport_pattern(hd2, N.C.byref(nnz), N.as_p(rp, N.C.c_int32), N.as_p(ci, N.C.c_int32)))
        vals = torch.empty(nnz.value, dtype=torch.float64, device="cuda")
        N.check(N.lib().pmb_transport_jacobian(hd2, N.ptr(ds), dt, N.ptr(vals)))
        J = sp.csr_array((vals.cpu().numpy(), ci, rp), shape=(nc, nc))
        ref = prob.jacobian(s, sprev, dt)
        assert abs(J - ref).max() <= 1e-12 * abs(ref).max()
    finally:
        N.lib().pmb_transport_destroy(hd2)


def test_explicit_out_of_range_is_reported():
    """A substep far beyond the stable one overshoots [0, 1]: the device
    flags it and the call raises, as the reference's check does."""
    g, rock, src, d = _bl()
    with pytest.raises(AssertionError):
        explicit_transport(_two_phase_state(g, 0.0, d["bl_flux0"]), g, 30 * DAY, rock, FLUID, src=src, dt=30 * DAY)
