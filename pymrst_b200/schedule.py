"""Report-step driver with timestep cuts (legacy simulate_schedule_ad,
pymrst/modules/ad_core/simulators/simulate_schedule_ad.py:16-75).

With a `GpuOilWaterModel` the state stays on the device for the whole
schedule; one host copy of the state is made per report step for the
returned list.  Other models (the reference's own included) are driven
through their `step(state, dt)` method exactly as the reference does.
"""

from __future__ import annotations

from typing import List, Sequence, Tuple

import numpy as np


def simulate_schedule_ad(state0, model, timesteps: Sequence[float], max_cuts: int = 6,
                         verbose: bool = True, *, observer=None) -> Tuple[List, np.ndarray]:
    def _observe(event, **payload):
        if observer is None:
            return
        try:
            observer(event, payload)
        except Exception:
            pass

    device = hasattr(model, "step_device")
    if device:
        x = model.to_device(state0)
        backup = x.clone()
    state = state0
    states: List = []
    its_per_step = np.zeros(len(timesteps), dtype=np.int64)
    for i, dt_report in enumerate(timesteps):
        _observe("report_step_started", report_step=int(i), dt=float(dt_report))
        t_local, its = 0.0, 0
        dt, cuts = float(dt_report), 0
        while t_local < dt_report - 1e-12 * dt_report:
            dt = min(dt, dt_report - t_local)
            _observe("ministep_started", report_step=int(i), dt=float(dt))
            if device:
                backup.copy_(x)
                ok, nit, _ = model.step_device(x, dt)
            else:
                candidate, ok, nit = model.step(state, dt)
            its += nit
            _observe("step_accepted" if ok else "step_rejected", report_step=int(i), dt=float(dt),
                     iterations=int(nit))
            if ok:
                if not device:
                    state = candidate
                t_local += dt
                dt = min(2.0 * dt, dt_report - t_local) if cuts else dt
            else:
                if device:
                    x.copy_(backup)
                cuts += 1
                if cuts > max_cuts:
                    raise AssertionError(f"step {i}: Newton failed after {max_cuts} timestep cuts")
                dt /= 2.0
                _observe("timestep_cut", report_step=int(i), cut=int(cuts), dt=float(dt))
                if verbose:
                    print(f"  step {i}: cutting dt to {dt:.3e}")
        its_per_step[i] = its
        states.append(model.from_device(x) if device else state)
        if verbose:
            print(f"step {i + 1}/{len(timesteps)}: {its} iterations")
    return states, its_per_step
