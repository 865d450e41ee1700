"""Host-side behaviour of `adoo.use_device_cell_equations` on the reference's
AD-OO oil-water model, with no GPU: the model keeps its identity and gets a
subclass once (copies keep the method, other instances are untouched), and
the cases the device equations do not cover are refused before any device
work: residual-only and reverse (adjoint) assembly, and a gravity vector
that is not vertical.

The reference package comes from its install under baseline/_ref; the module
is skipped where that install is absent."""

import copy
import sys
from pathlib import Path

import numpy as np
import pytest

REF = Path(__file__).resolve().parents[1] / "baseline" / "_ref"
if not (REF / "pymrst").is_dir():
    pytest.skip("the reference package is not installed under baseline/_ref", allow_module_level=True)
sys.path.insert(0, str(REF))

from pymrst.gridprocessing import cart_grid, compute_geometry  # noqa: E402
from pymrst.modules.ad_blackoil.models.two_phase_oil_water_model import TwoPhaseOilWaterModel  # noqa: E402
from pymrst.modules.ad_core.ad_oo.physical_model import copy_state  # noqa: E402
from pymrst.modules.ad_core.utils.schedule import simple_schedule  # noqa: E402
from pymrst.modules.ad_props import init_simple_adi_fluid  # noqa: E402
from pymrst.params import make_rock  # noqa: E402
from pymrst.params.wells_and_bc.vertical_well import vertical_well  # noqa: E402
from pymrst.solvers.init_res_sol import init_res_sol  # noqa: E402
from pymrst.utils.units import BARSA, CENTI, DARCY, DAY, MILLI, POISE  # noqa: E402

from pymrst_b200 import adoo  # noqa: E402


def _case():
    G = compute_geometry(cart_grid([6, 5, 2], [60.0, 50.0, 4.0]))
    rock = make_rock(G, 100 * MILLI * DARCY, 0.2)
    fluid = init_simple_adi_fluid(mu=np.array([1, 5]) * CENTI * POISE, rho=np.array([1000.0, 800.0]), n=[2, 2],
                                  c=[1e-5 / BARSA, 1e-5 / BARSA], p_ref=200 * BARSA, phases="wo")
    rate = 0.1 * float(np.sum(0.2 * G.cells.volumes)) / (100 * DAY)
    W = vertical_well([], G, rock, 0, 0, None, val=rate, well_type="rate", compi=np.array([1.0, 0.0]), name="I")
    W = vertical_well(W, G, rock, 5, 4, None, val=150 * BARSA, well_type="bhp", compi=np.array([0.0, 1.0]),
                      name="P")
    schedule = simple_schedule(np.full(1, 10 * DAY), W=W)
    return G, rock, fluid, schedule, init_res_sol(G, 200 * BARSA, np.array([0.1, 0.9]))


def test_conversion_keeps_the_model_and_subclasses_once():
    G, rock, fluid, _, _ = _case()
    m = TwoPhaseOilWaterModel(G, rock, fluid)
    other = TwoPhaseOilWaterModel(G, rock, fluid)
    out = adoo.use_device_cell_equations(m)
    assert out is m
    cls = type(m)
    assert cls is not TwoPhaseOilWaterModel and issubclass(cls, TwoPhaseOilWaterModel)
    assert type(other) is TwoPhaseOilWaterModel  # other instances keep the reference's equations
    adoo.use_device_cell_equations(m)
    assert type(m) is cls  # converting again adds no second subclass
    c = copy.copy(m)
    assert type(c) is cls and c.get_equations.__func__ is cls.get_equations


@pytest.mark.parametrize("mode", ["resOnly", "reverseMode"])
def test_residual_only_and_reverse_assembly_are_refused(mode):
    G, rock, fluid, schedule, init = _case()
    m = adoo.use_device_cell_equations(TwoPhaseOilWaterModel(G, rock, fluid))
    forces = dict(m.get_valid_driving_forces())
    forces.update(m.get_driving_forces(schedule.controls[0]))
    m = m.validate_model(forces)
    state0 = m.validate_state(init)
    m, st = m.prepare_report_step(copy_state(state0), state0, 10 * DAY, forces)
    m, st = m.prepare_timestep(st, state0, 10 * DAY, forces)
    with pytest.raises(NotImplementedError, match="device cell equations"):
        m.get_equations(state0, st, 10 * DAY, forces, **{mode: True})


def test_a_tilted_gravity_vector_is_refused():
    G, rock, fluid, _, _ = _case()
    m = TwoPhaseOilWaterModel(G, rock, fluid)
    m.gravity = np.array([0.5, 0.0, 9.8])
    with pytest.raises(ValueError, match="vertical"):
        adoo._device_model(m)
