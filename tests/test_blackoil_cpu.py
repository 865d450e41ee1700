"""Host side of the black-oil path, no GPU: the tables taken from a parsed
deck equal the tables the reference's init_deck_blackoil_fluid builds (read
back from its fluid object), and the oracle's fluid functions equal the
reference fluid's at points inside and outside the tables.  Runs where the
reference package is installed under baseline/_ref."""

import sys
from pathlib import Path

import numpy as np
import pytest

from fixtures import bo_deck, load
from oracle import blackoil as obo
from pymrst_b200.blackoil import BlackOilTables

REF = Path(__file__).resolve().parents[1] / "baseline" / "_ref"
needs_ref = pytest.mark.skipif(not (REF / "pymrst").is_dir(),
                               reason="the reference package is not installed under baseline/_ref")


def _reference_fluid(deck):
    sys.path.insert(0, str(REF))
    from pymrst.modules.ad_props.props.init_deck_adi_fluid import init_deck_blackoil_fluid
    return init_deck_blackoil_fluid(deck)


def test_tables_from_deck_have_the_device_layout():
    t = BlackOilTables.from_deck(bo_deck(load("bo_newton.npz")))
    assert t.branch_ptr[0] == 0 and t.branch_ptr[-1] == t.branch_p.size
    for x in (t.gas_p, t.rssat_p, t.key, t.sw, t.sow, t.sg, t.sog):
        assert np.all(np.diff(x) > 0)
    assert t.sw[0] == t.swcon - 1.0 and t.sw[-1] == 2.0


@needs_ref
def test_tables_read_from_the_reference_fluid_equal_the_deck_tables():
    deck = bo_deck(load("bo_newton.npz"))
    a = BlackOilTables.from_deck(deck)
    b = BlackOilTables.from_fluid(_reference_fluid(deck))
    for name in a.__dataclass_fields__:
        x, y = getattr(a, name), getattr(b, name)
        if x is None or y is None:
            assert x is None and y is None, name
            continue
        np.testing.assert_array_equal(np.asarray(x, float), np.asarray(y, float), err_msg=name)


@needs_ref
def test_oracle_fluid_equals_the_reference_fluid():
    deck = bo_deck(load("bo_newton.npz"))
    ref = _reference_fluid(deck)
    fl = obo.Fluid(BlackOilTables.from_deck(deck))
    rng = np.random.default_rng(1)
    p = rng.uniform(-20e5, 450e5, 2000)
    rs = rng.uniform(-10.0, 220.0, p.size)
    for sat in (False, True):
        flag = np.full(p.size, sat)
        np.testing.assert_array_equal(fl.b_o(p, rs, flag), ref.b_o(p, rs, flag))
        np.testing.assert_array_equal(fl.mu_o(p, rs, flag), ref.mu_o(p, rs, flag))
    np.testing.assert_array_equal(fl.b_g(p), ref.b_g(p))
    np.testing.assert_array_equal(fl.mu_g(p), ref.mu_g(p))
    np.testing.assert_array_equal(fl.rs_sat(p), ref.rs_sat(p))
    np.testing.assert_array_equal(fl.b_w(p), ref.b_w(p))
    np.testing.assert_array_equal(fl.pv_mult(p), ref.pv_mult(p))
    sw = rng.uniform(-0.1, 1.1, 2000)
    sg = rng.uniform(-0.1, 1.0, sw.size)
    so = 1.0 - sw - sg
    np.testing.assert_array_equal(fl.kr_w(sw), ref.kr_w(sw))
    np.testing.assert_array_equal(fl.kr_g(sg), ref.kr_g(sg))
    np.testing.assert_array_equal(fl.kr_o(sw, so, sg), ref.kr_o(sw, so, sg))
    np.testing.assert_array_equal(fl.pc_ow(sw), ref.pc_ow(sw))
    np.testing.assert_array_equal(fl.pc_og(sg), ref.pc_og(sg))
