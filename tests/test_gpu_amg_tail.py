"""The cluster tail cycle (the AMG levels below the K-cycle levels as one
thread-block-cluster launch per visit) against the per-step kernels
(the default): the same Newton step, run in two processes, gives bitwise
the same states and the same Newton and Krylov iteration counts, in FP64 and
in mixed precision, with fewer kernel launches."""

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
precision, cycle = int(sys.argv[3]), int(sys.argv[4])
case = cases.channelised(dims=(40, 60, 24), n_smooth=10)
m = GpuOilWaterModel(case.grid, case.rock, case.fluid, case.wells, gravity=case.gravity,
                     cpr_options=dict(amg_cycle=cycle, precision=precision, rtol=1e-9, maxiter=400,
                                      amg_smoother_degree=3, amg_coarse_degree=2, local_sweeps=4),
                     max_iterations=8)
st = m.initial_state(case.p0, case.sw0)
l0 = N.launch_count()
st1, ok, its = m.step(st, case.dt)
launches = N.launch_count() - l0
np.save(sys.argv[2], np.concatenate([st1.pressure, st1.sW, st1.qWs, st1.qOs, st1.bhp]))
print(json.dumps({"its": int(its), "krylov": float(m.last_stats[2]), "launches": int(launches),
                  "levels": m.cpr_levels()}))
"""


def _run(tmp_path, tail, precision, cycle):
    env = dict(os.environ)
    env.pop("PMB_FUSED_COARSE", None)
    env["PMB_AMG_TAIL_ROWS"] = "65536" if tail else "0"
    out = tmp_path / f"state_{int(tail)}_{precision}_{cycle}.npy"
    r = subprocess.run([sys.executable, "-c", SNIPPET, str(ROOT), str(out), str(precision), str(cycle)], env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return json.loads(r.stdout.strip().splitlines()[-1]), np.load(out)


@pytest.mark.parametrize("precision,cycle", [(1, 3), (0, 3), (1, 0)])
def test_tail_cycle_is_bitwise_the_per_step_cycle(tmp_path, precision, cycle):
    tail, xt = _run(tmp_path, True, precision, cycle)
    plain, xp = _run(tmp_path, False, precision, cycle)
    assert len(plain["levels"]) >= cycle + 2  # there are levels below the K-cycle levels
    assert tail["its"] == plain["its"] and tail["krylov"] == plain["krylov"]
    assert np.array_equal(xt, xp)
    assert tail["launches"] < plain["launches"]
