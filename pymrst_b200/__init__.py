"""pymrst_b200: PyMRST's fully-implicit TPFA oil-water hot path on B200.

Public API (reference names):
  GpuOilWaterModel / TwoPhaseOilWaterModelAD   device oil-water model
  simulate_schedule_ad                         report-step driver
  cartesian_grid, make_rock, add_well, init_simple_adi_fluid   host inputs
The CUDA library is libpymrst_b200.so in this folder (python -m
pymrst_b200.build); there is no CPU fallback.
"""

from .grid import cartesian_grid
from .params import (BARSA, CENTI, DARCY, DAY, MILLI, POISE, add_well, init_simple_adi_fluid,
                     make_rock)


def __getattr__(name):
    # device-dependent modules load lazily so that host-only use needs no GPU
    if name in ("GpuOilWaterModel", "TwoPhaseOilWaterModelAD", "OWState"):
        from . import ow_model
        return getattr(ow_model, name)
    if name == "simulate_schedule_ad":
        from .schedule import simulate_schedule_ad
        return simulate_schedule_ad
    raise AttributeError(name)
