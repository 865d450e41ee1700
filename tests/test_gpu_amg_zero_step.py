"""The first pre-smoothing step of every AMG level below the first, taken
by the kernel that writes that level's right-hand side (the restriction,
or the K-cycle's axpy) instead of a launch of its own: the same Newton
step, run in two processes with and without it (PMB_AMG_FUSE_ZERO_STEP=0),
gives bitwise the same states and the same Newton and Krylov counts, in
FP64 and in mixed precision, with fewer kernel launches."""

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
from pymrst_b200 import cases, _native as N
from pymrst_b200.ow_model import GpuOilWaterModel
precision = int(sys.argv[3])
case = cases.channelised(dims=(40, 60, 30), n_smooth=10)
m = GpuOilWaterModel(case.grid, case.rock, case.fluid, case.wells, gravity=case.gravity,
                     cpr_options=dict(amg_cycle=3, precision=precision, rtol=1e-9, maxiter=400,
                                      amg_smoother_degree=3, amg_coarse_degree=2, local_sweeps=4,
                                      replay_graph=0),
                     max_iterations=6)
st = m.initial_state(case.p0, case.sw0)
l0 = N.launch_count()
st1, ok, its = m.step(st, case.dt)
launches = N.launch_count() - l0
np.save(sys.argv[2], np.concatenate([st1.pressure, st1.sW, st1.qWs, st1.qOs, st1.bhp]))
print(json.dumps({"its": int(its), "krylov": float(m.last_stats[2]), "launches": int(launches)}))
"""


def _run(tmp_path, fused, precision):
    env = dict(os.environ)
    env["PMB_AMG_FUSE_ZERO_STEP"] = "1" if fused else "0"
    out = tmp_path / f"state_{int(fused)}_{precision}.npy"
    r = subprocess.run([sys.executable, "-c", SNIPPET, str(ROOT), str(out), str(precision)], env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return json.loads(r.stdout.strip().splitlines()[-1]), np.load(out)


@pytest.mark.parametrize("precision", [0, 1])
def test_fused_zero_steps_are_bitwise_the_separate_launches(tmp_path, precision):
    fused, xf = _run(tmp_path, True, precision)
    plain, xp = _run(tmp_path, False, precision)
    assert fused["its"] == plain["its"] and fused["krylov"] == plain["krylov"]
    assert np.array_equal(xf, xp)
    assert fused["launches"] < plain["launches"]
