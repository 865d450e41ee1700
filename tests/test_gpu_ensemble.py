"""Batched realisations (GpuOilWaterEnsemble) against single runs of each
member on its own model: the per-member Newton counts equal and the states
after every step within the parity bars (p 1e-8 relative, sW 1e-7), with
the CPR-GMRES tolerance at 1e-12 in both runs."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from pymrst_b200 import cases  # noqa: E402
from pymrst_b200.build import build  # noqa: E402
from pymrst_b200.ensemble import GpuOilWaterEnsemble  # noqa: E402
from pymrst_b200.ow_model import GpuOilWaterModel  # noqa: E402
from pymrst_b200.schedule import simulate_schedule_ad  # noqa: E402

build()

TIGHT = dict(rtol=1e-12, maxiter=400)


def test_batched_members_match_single_runs():
    reals = cases.ensemble_realisations(n=6, seed=5, nx_range=(6, 14), nz_range=(2, 4), nsteps=3, dt_days=30.0)
    fluid = reals[0].fluid
    ens = GpuOilWaterEnsemble([(c.grid, c.rock, c.wells) for c in reals], fluid, gravity=reals[0].gravity,
                              cpr_options=TIGHT)
    st0 = [ens.member_initial_state(k, c.p0, c.sw0) for k, c in enumerate(reals)]
    dts = np.full(3, reals[0].dt)
    states, its = ens.simulate(st0, dts)
    for k, c in enumerate(reals):
        m = GpuOilWaterModel(c.grid, c.rock, c.fluid, c.wells, gravity=c.gravity, cpr_options=TIGHT)
        ref_states, ref_its = simulate_schedule_ad(m.initial_state(c.p0, c.sw0), m, dts, verbose=False)
        np.testing.assert_array_equal(its[k], ref_its)
        for s, r in zip(states[k], ref_states):
            assert np.abs(s.pressure - r.pressure).max() <= 1e-8 * np.abs(r.pressure).max()
            assert np.abs(s.sW - r.sW).max() <= 1e-7
            np.testing.assert_allclose(s.bhp, r.bhp, rtol=1e-8)


def test_a_frozen_member_is_left_exactly_as_it_was():
    reals = cases.ensemble_realisations(n=3, seed=6, nx_range=(6, 10), nz_range=(2, 3), nsteps=2, dt_days=30.0)
    ens = GpuOilWaterEnsemble([(c.grid, c.rock, c.wells) for c in reals], reals[0].fluid,
                              gravity=reals[0].gravity, cpr_options=TIGHT)
    st0 = ens.join([ens.member_initial_state(k, c.p0, c.sw0) for k, c in enumerate(reals)])
    x = ens.to_device(st0)
    before = x.clone()
    state, its, _ = ens.step_members(x, reals[0].dt, np.array([True, False, True]))
    assert state[1] == -1 and state[0] == 1 and state[2] == 1
    c0, c1 = ens.cell_ptr[1], ens.cell_ptr[2]
    assert torch.equal(x[2 * c0:2 * c1], before[2 * c0:2 * c1])
    w0, w1 = ens.well_ptr[1], ens.well_ptr[2]
    nc = ens.nc
    assert torch.equal(x[2 * nc + 3 * w0:2 * nc + 3 * w1], before[2 * nc + 3 * w0:2 * nc + 3 * w1])


def test_concurrent_members_equal_single_runs_bitwise():
    """Members stepped concurrently on their own streams follow exactly the
    single-run path, so their states equal single runs bit for bit."""
    from pymrst_b200.ensemble import simulate_members_concurrently
    reals = cases.ensemble_realisations(n=5, seed=7, nx_range=(6, 12), nz_range=(2, 3), nsteps=2, dt_days=30.0)
    dts = np.full(2, reals[0].dt)
    st0 = []
    for c in reals:
        m = GpuOilWaterModel(c.grid, c.rock, c.fluid, c.wells, gravity=c.gravity)
        st0.append(m.initial_state(c.p0, c.sw0))
    states, its = simulate_members_concurrently([(c.grid, c.rock, c.wells) for c in reals], reals[0].fluid, st0, dts,
                                                gravity=reals[0].gravity, workers=3)
    for k, c in enumerate(reals):
        m = GpuOilWaterModel(c.grid, c.rock, c.fluid, c.wells, gravity=c.gravity)
        ref, ref_its = simulate_schedule_ad(st0[k], m, dts, verbose=False)
        np.testing.assert_array_equal(its[k], ref_its)
        for s, r in zip(states[k], ref):
            np.testing.assert_array_equal(s.pressure, r.pressure)
            np.testing.assert_array_equal(s.sW, r.sW)


def test_concurrent_members_with_graph_replay_equal_single_runs_bitwise():
    """The concurrent runner with every model built up front and each
    member's preconditioner replayed as a CUDA graph: still each member's
    single run, bit for bit."""
    from pymrst_b200.ensemble import simulate_members_concurrently
    reals = cases.ensemble_realisations(n=6, seed=8, nx_range=(6, 12), nz_range=(2, 3), nsteps=2, dt_days=30.0)
    dts = np.full(2, reals[0].dt)
    st0 = []
    for c in reals:
        m = GpuOilWaterModel(c.grid, c.rock, c.fluid, c.wells, gravity=c.gravity)
        st0.append(m.initial_state(c.p0, c.sw0))
    states, its = simulate_members_concurrently([(c.grid, c.rock, c.wells) for c in reals], reals[0].fluid, st0, dts,
                                                gravity=reals[0].gravity, workers=3, replay_graph=True)
    for k, c in enumerate(reals):
        m = GpuOilWaterModel(c.grid, c.rock, c.fluid, c.wells, gravity=c.gravity)
        ref, ref_its = simulate_schedule_ad(st0[k], m, dts, verbose=False)
        np.testing.assert_array_equal(its[k], ref_its)
        for s, r in zip(states[k], ref):
            np.testing.assert_array_equal(s.pressure, r.pressure)
            np.testing.assert_array_equal(s.sW, r.sW)
