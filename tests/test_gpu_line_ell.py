"""The line smoother on its line-ordered operator copy (the default) against
the block-CSR line kernel (PMB_LINE_ELL=0): the same Newton step, run in two
processes, converges in the same Newton iterations to the same state; the
summation order of the smoother's residual differs and, in mixed precision,
the line-ordered r and z are FP32."""

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
sys.path.insert(0, sys.argv[1])
from pymrst_b200 import cases
from pymrst_b200.ow_model import GpuOilWaterModel
case = cases.five_spot(dims=(40, 40, 12))
m = GpuOilWaterModel(case.grid, case.rock, case.fluid, case.wells, gravity=case.gravity,
                     cpr_options=dict(rtol=1e-10, maxiter=400, precision=int(sys.argv[3])))
st = m.initial_state(case.p0, case.sw0)
st1, ok, its = m.step(st, case.dt)
np.save(sys.argv[2], np.stack([st1.pressure, st1.sW]))
print(json.dumps({"ok": bool(ok), "its": int(its), "krylov": float(m.last_stats[2])}))
"""


def _run(tmp_path, ell, precision):
    env = dict(os.environ)
    env.pop("PMB_LINE_ELL", None)
    if not ell:
        env["PMB_LINE_ELL"] = "0"
    out = tmp_path / f"state_{int(ell)}_{precision}.npy"
    r = subprocess.run([sys.executable, "-c", SNIPPET, str(ROOT), str(out), str(precision)], env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return json.loads(r.stdout.strip().splitlines()[-1]), np.load(out)


@pytest.mark.parametrize("precision", [0, 1])
def test_line_ordered_smoother_matches_the_block_csr_kernel(tmp_path, precision):
    ell, xe = _run(tmp_path, True, precision)
    csr, xc = _run(tmp_path, False, precision)
    assert ell["ok"] and csr["ok"]
    assert ell["its"] == csr["its"]
    assert abs(ell["krylov"] - csr["krylov"]) <= 0.1 * csr["krylov"] + 1
    assert np.abs(xe[0] - xc[0]).max() <= 1e-7 * np.abs(xc[0]).max()
    assert np.abs(xe[1] - xc[1]).max() <= 1e-6
