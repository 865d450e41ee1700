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
