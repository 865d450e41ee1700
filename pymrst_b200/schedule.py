"""Report-step driver with timestep cuts, for the legacy
`simulate_schedule_ad(state0, model, timesteps, max_cuts, verbose, observer=)`
interface (pymrst/modules/ad_core/simulators/simulate_schedule_ad.py:16-75).

The time-step rule is the reference's: a report step is first tried whole; a
failed attempt halves the substep (at most `max_cuts` times per report step);
after the first cut, every accepted substep doubles the next one, never past
the end of the report step.  `MinistepControl` holds that rule, so the
benchmark and the drivers here share one implementation of it.

With a `GpuOilWaterModel` the state stays on the device for the whole
schedule (a failed attempt restores it from a device copy); one host copy is
made per report step for the returned list.  Any other model, the
reference's own included, is driven through its `step(state, dt)`.
"""

from __future__ import annotations

from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np

# Observer event names of the reference's solvers (interface: handlers
# written for the reference read these unchanged).
EVENTS = ("report_step_started", "ministep_started", "step_accepted", "step_rejected", "timestep_cut")


class MinistepControl:
    """Substep sizes inside one report step of length `dt_report`."""

    def __init__(self, dt_report: float, max_cuts: int = 6):
        self.total = float(dt_report)
        self.done = 0.0
        self.dt = float(dt_report)
        self.cuts = 0
        self.max_cuts = int(max_cuts)

    def finished(self) -> bool:
        return self.done >= self.total - 1e-12 * self.total

    def next(self) -> float:
        """The next substep: the current size, clipped to what remains."""
        self.dt = min(self.dt, self.total - self.done)
        return self.dt

    def accepted(self) -> None:
        self.done += self.dt
        if self.cuts:
            self.dt = min(2.0 * self.dt, self.total - self.done)

    def rejected(self) -> bool:
        """Halve the substep; False once the cut budget is spent."""
        self.cuts += 1
        self.dt *= 0.5
        return self.cuts <= self.max_cuts


def _notify(observer: Optional[Callable], event: str, **payload) -> None:
    """Call the observer; a failing observer never stops the simulation."""
    if observer is not None:
        try:
            observer(event, payload)
        except Exception:
            pass


def run_report_step(attempt: Callable[[float], Tuple[bool, int]], dt_report: float, max_cuts: int = 6,
                    observer=None, report_step: int = 0, verbose: bool = False) -> Tuple[int, int]:
    """Advance one report step.  `attempt(dt)` tries one substep and returns
    (accepted, Newton iterations); on rejection it must leave the state as it
    was.  Returns (Newton iterations, cuts).  Raises AssertionError when the
    cut budget is spent (the reference's failure mode)."""
    ctl = MinistepControl(dt_report, max_cuts)
    its = 0
    while not ctl.finished():
        dt = ctl.next()
        _notify(observer, "ministep_started", report_step=report_step, dt=float(dt))
        ok, nit = attempt(dt)
        its += nit
        _notify(observer, "step_accepted" if ok else "step_rejected", report_step=report_step, dt=float(dt),
                iterations=int(nit))
        if ok:
            ctl.accepted()
            continue
        if not ctl.rejected():
            raise AssertionError(f"report step {report_step}: no convergence within {max_cuts} timestep halvings")
        _notify(observer, "timestep_cut", report_step=report_step, cut=int(ctl.cuts), dt=float(ctl.dt))
        if verbose:
            print(f"  report step {report_step}: substep reduced to {ctl.dt:.3e} s")
    return its, ctl.cuts


def simulate_schedule_ad(state0, model, timesteps: Sequence[float], max_cuts: int = 6,
                         verbose: bool = True, *, observer=None) -> Tuple[List, np.ndarray]:
    """(states after each report step, Newton iterations per report step)."""
    on_device = hasattr(model, "step_device")
    holder = {"state": state0}
    if on_device:
        x = model.to_device(state0)
        saved = x.clone()

        def attempt(dt):
            saved.copy_(x)
            ok, nit, _ = model.step_device(x, dt)
            if not ok:
                x.copy_(saved)
            return ok, nit
    else:
        def attempt(dt):
            new, ok, nit = model.step(holder["state"], dt)
            if ok:
                holder["state"] = new
            return ok, nit

    states: List = []
    its = np.zeros(len(timesteps), dtype=np.int64)
    for i, dt_report in enumerate(timesteps):
        _notify(observer, "report_step_started", report_step=int(i), dt=float(dt_report))
        its[i], _ = run_report_step(attempt, float(dt_report), max_cuts, observer, int(i), verbose)
        states.append(model.from_device(x) if on_device else holder["state"])
        if verbose:
            print(f"report step {i + 1} of {len(timesteps)}: {its[i]} Newton iterations")
    return states, its
