"""The slot-major ELL copy of the large AMG levels (one thread per row)
(its diagonal form, and the column form that PMB_AMG_ELL=1 forces)
against the CSR kernels (PMB_AMG_ELL=0): the CPR-FGMRES solve of the same
Newton system, run in two processes, reaches the same solution to the
tolerance, in FP64 and in mixed precision, with Krylov counts within 2%
(FP64) and 10% (mixed): the two layouts differ only in the order of each
row's sum."""

import json
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

ROOT = Path(__file__).resolve().parents[1]

SNIPPET = r"""
import json, sys
import numpy as np
import torch
sys.path.insert(0, sys.argv[1])
from pymrst_b200 import cases, _native as N
from pymrst_b200.ow_model import GpuOilWaterModel
precision = int(sys.argv[3])
case = cases.channelised(dims=(40, 60, 30), n_smooth=10)
m = GpuOilWaterModel(case.grid, case.rock, case.fluid, case.wells, gravity=case.gravity,
                     cpr_options=dict(amg_cycle=3, precision=precision, rtol=1e-11, maxiter=600,
                                      amg_smoother_degree=3, amg_coarse_degree=2, local_sweeps=4))
x = m.to_device(m.initial_state(case.p0, case.sw0))
x0 = x.clone()
cdp = torch.zeros(max(m.sizes["nperf"], 1), dtype=torch.float64, device="cuda")
N.check(N.lib().pmb_ow_compute_cdp(m._handle, N.ptr(x0), N.ptr(cdp)))
res, jac, well = m.assemble_device(x, x0, case.dt, cdp, True)
s = m.solver_handle()
N.check(N.lib().pmb_cpr_setup(s, N.ptr(jac), N.ptr(well), N.ptr(x)))
dx = torch.zeros_like(res)
info = (N.C.c_double * 4)()
N.check(N.lib().pmb_cpr_solve(s, N.ptr(res), N.ptr(dx), info))
cb = (N.C.c_double * 8)()
N.check(N.lib().pmb_cpr_bytes(s, cb))
np.save(sys.argv[2], dx.cpu().numpy())
print(json.dumps({"krylov": info[0], "relres": info[1], "cycle_bytes": cb[0], "levels": m.cpr_levels(),
                  "nc": int(m.nc)}))
"""


def _run(tmp_path, mode, precision):
    env = dict(os.environ)
    env.pop("PMB_AMG_ELL", None)
    if mode != "diagonal":
        env["PMB_AMG_ELL"] = "1" if mode == "column" else "0"
    env["PMB_AMG_ELL_MIN_ROWS"] = "65537"  # a small model, so that level 0 takes the ELL copy
    out = tmp_path / f"state_{mode}_{precision}.npy"
    r = subprocess.run([sys.executable, "-c", SNIPPET, str(ROOT), str(out), str(precision)], env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return json.loads(r.stdout.strip().splitlines()[-1]), np.load(out)


@pytest.mark.parametrize("mode", ["diagonal", "column"])
@pytest.mark.parametrize("precision", [0, 1])
def test_ell_levels_match_the_csr_kernels(tmp_path, precision, mode):
    ell, xe = _run(tmp_path, mode, precision)
    csr, xc = _run(tmp_path, "csr", precision)
    assert csr["levels"][0] > 65536  # level 0 is large enough to take the ELL copy
    assert ell["relres"] <= 1e-11 and csr["relres"] <= 1e-11
    assert abs(ell["krylov"] - csr["krylov"]) <= (0.02 if precision == 0 else 0.1) * csr["krylov"] + 1
    # the byte model sees the ELL layout (no row starts, padded slots)
    assert ell["cycle_bytes"] != csr["cycle_bytes"]
    # both solve the same Newton system to the tolerance
    assert np.abs(xe - xc).max() <= 1e-6 * np.abs(xc).max()
