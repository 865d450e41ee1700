"""The allocation-free convergence check against the handle-based one.

Callers that cannot allocate device memory where they run the check (inside
another framework's memory pool, or where cudaMalloc's implicit
synchronisation is not allowed) use pmb_ow_cnv_mb_noalloc, whose scratch is
a fixed array inside the library.  Its CNV and MB must equal those of
pmb_ow_convergence, on two calls in a row (the second call reuses the
scratch the first one left behind).  This file is collected last.
"""

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from fixtures import load, ow_case  # noqa: E402
from pymrst_b200 import _native as N  # noqa: E402
from pymrst_b200.build import build  # noqa: E402
from pymrst_b200.ow_model import GpuOilWaterModel, OWState  # noqa: E402

build()


def _state(d, sfx=""):
    return OWState(pressure=d["p" + sfx].copy(), sW=d["sw" + sfx].copy(), qWs=d["qws" + sfx].copy(),
                   qOs=d["qos" + sfx].copy(), bhp=d["bhp" + sfx].copy())


@pytest.mark.parametrize("name", ["ow_assemble_grav.npz", "ow_assemble_xflow.npz"])
def test_noalloc_cnv_mb_matches_handle_convergence_twice(name):
    d = load(name)
    g, rock, fluid, wells = ow_case(d)
    m = GpuOilWaterModel(g, rock, fluid, wells, gravity=float(d["gravity"]))
    dt = float(d["dt"])
    x = m.to_device(_state(d))
    x0 = m.to_device(_state(d, "0"))
    cdp = torch.as_tensor(d["cdp"], device="cuda")
    res, _, _ = m.assemble_device(x, x0, dt, cdp, want_jac=False)
    ref = m.convergence(res, x, dt)
    prm = m.fluid_params
    fl = (C.c_double * 5)(prm.c[0], prm.c[1], prm.b0[0], prm.b0[1], prm.p_ref)
    pv = torch.as_tensor(m.pv, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        out = torch.full((4,), -1.0, dtype=torch.float64, device="cuda")
        N.check(N.lib().pmb_ow_cnv_mb_noalloc(m.nc, N.ptr(res), N.ptr(x), N.ptr(pv), float(m.pv.sum()), fl, dt,
                                              N.ptr(out), stream))
        got = out.cpu().numpy()
        np.testing.assert_allclose(got[:2], ref[:2], rtol=1e-12)
        assert got[2] == 0.0


def test_noalloc_rejects_sizes_beyond_its_scratch():
    fl = (C.c_double * 5)(0.0, 0.0, 1.0, 1.0, 0.0)
    dummy = torch.zeros(4, dtype=torch.float64, device="cuda")
    rc = N.lib().pmb_ow_cnv_mb_noalloc(16_777_217, N.ptr(dummy), N.ptr(dummy), N.ptr(dummy), 1.0, fl, 1.0,
                                       N.ptr(dummy), 0)
    assert rc == 2 and "exceeds" in N.lib().pmb_last_error().decode()


def _cnv_mb_numpy(res, x, pv, fl, dt):
    """CNV and MB of the reference's _converged (two_phase_oil_water_model.py:
    549-567) on the cell part, in numpy."""
    cw, co, b0w, b0o, p_ref = fl
    p = x[0::2]
    bw = np.mean(1.0 / (b0w * np.exp(cw * (p - p_ref))))
    bo = np.mean(1.0 / (b0o * np.exp(co * (p - p_ref))))
    rw, ro = res[0::2], res[1::2]
    cnv = max(bw * dt * np.max(np.abs(rw / pv)), bo * dt * np.max(np.abs(ro / pv)))
    mb = max(bw * dt * abs(rw.sum()) / pv.sum(), bo * dt * abs(ro.sum()) / pv.sum())
    return cnv, mb


def test_noalloc_many_blocks_larger_then_smaller_and_nonfinite():
    """Millions of cells, so that thousands of per-block partial sums go
    through the static array and its final reduction: a size that is not a
    multiple of the 2048 cells of a block, then a smaller size on the same
    scratch (slots beyond the second call's blocks hold the first call's
    values and must be ignored), then a NaN residual, counted as one
    non-finite cell."""
    rng = np.random.default_rng(7)
    fl = (1e-9, 2e-9, 1.02, 0.98, 2e7)
    flc = (C.c_double * 5)(*fl)
    dt = 864000.0
    stream = torch.cuda.current_stream().cuda_stream
    n_big = 3_000_001
    res = rng.normal(0.3, 1.0, 2 * n_big) * 1e-3
    x = np.empty(2 * n_big)
    x[0::2] = rng.uniform(1.5e7, 2.5e7, n_big)
    x[1::2] = rng.uniform(0.1, 0.9, n_big)
    pv = rng.uniform(5.0, 50.0, n_big)
    d_res, d_x, d_pv = (torch.as_tensor(a, device="cuda") for a in (res, x, pv))
    for nc in (n_big, 1_000_003):
        out = torch.full((4,), -1.0, dtype=torch.float64, device="cuda")
        N.check(N.lib().pmb_ow_cnv_mb_noalloc(nc, N.ptr(d_res), N.ptr(d_x), N.ptr(d_pv), float(pv[:nc].sum()),
                                              flc, dt, N.ptr(out), stream))
        got = out.cpu().numpy()
        cnv, mb = _cnv_mb_numpy(res[:2 * nc], x[:2 * nc], pv[:nc], fl, dt)
        np.testing.assert_allclose(got[0], cnv, rtol=1e-12)
        np.testing.assert_allclose(got[1], mb, rtol=1e-10)
        assert got[2] == 0.0
    res[2 * 123_457 + 1] = np.nan
    d_res = torch.as_tensor(res, device="cuda")
    out = torch.full((4,), -1.0, dtype=torch.float64, device="cuda")
    N.check(N.lib().pmb_ow_cnv_mb_noalloc(n_big, N.ptr(d_res), N.ptr(d_x), N.ptr(d_pv), float(pv.sum()), flc, dt,
                                          N.ptr(out), stream))
    assert out.cpu().numpy()[2] == 1.0


def test_noalloc_rejects_misaligned_pointers():
    fl = (C.c_double * 5)(0.0, 0.0, 1.0, 1.0, 0.0)
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    base = N.ptr(buf)
    rc = N.lib().pmb_ow_cnv_mb_noalloc(2, base, base, base + 4, 1.0, fl, 1.0, base + 64, 0)
    assert rc == 2 and "aligned" in N.lib().pmb_last_error().decode()
