"""Loaders that turn the golden .npz fixtures back into model inputs, built
with this package's own host-side grid/rock/well/fluid mirrors."""

from pathlib import Path
from types import SimpleNamespace

import numpy as np

from pymrst_b200.grid import cartesian_grid
from pymrst_b200.params import BARSA, CENTI, POISE, init_simple_adi_fluid, make_rock

GOLDEN = Path(__file__).parent / "golden"


def load(name):
    with np.load(GOLDEN / name, allow_pickle=False) as z:
        return {k: z[k] for k in z.files}


def ow_fluid(kind):
    if str(kind) == "cfg":
        return init_simple_adi_fluid(mu=np.array([1.0, 5.0]) * CENTI * POISE, rho=[1000.0, 800.0],
                                     n=[2, 2], c=[1e-5 / BARSA, 1e-5 / BARSA], p_ref=200 * BARSA,
                                     smin=[0.1, 0.1])
    return init_simple_adi_fluid(mu=np.array([1.0, 5.0]) * CENTI * POISE, rho=[1000.0, 800.0],
                                 n=[2, 2], c=[1e-6 / BARSA, 1e-4 / BARSA], p_ref=200 * BARSA)


def wells_from(d, prefix="w"):
    out = []
    for k in range(int(d[prefix + "count"])):
        out.append(SimpleNamespace(
            cells=d[f"{prefix}{k}_cells"].astype(np.int64), WI=d[f"{prefix}{k}_WI"],
            dZ=d[f"{prefix}{k}_dZ"], compi=d[f"{prefix}{k}_compi"],
            type=str(d[f"{prefix}{k}_type"]), val=float(d[f"{prefix}{k}_val"]),
            refDepth=float(d[f"{prefix}{k}_refDepth"])))
    return out


def ow_case(d):
    g = cartesian_grid(d["dims"], d["phys"])
    rock = make_rock(g, d["perm"][:, None], float(d["poro"]))
    fluid = ow_fluid(d["fluid_kind"])
    return g, rock, fluid, wells_from(d)


def bo_deck(d):
    """The synthetic deck stored in a black-oil fixture, in the parsed-deck
    layout (pvtw, rock_cp, pvdg, pvto, swof, sgof, rhoS)."""
    w, r = d["pvtw"], d["rock_cp"]
    rows, nrows, keys = d["pvto_rows"], d["pvto_nrows"], d["pvto_keys"]
    starts = np.concatenate([[0], np.cumsum(nrows)])
    pvto = [(float(k), rows[starts[i]:starts[i + 1]]) for i, k in enumerate(keys)]
    return dict(pvtw=dict(p_ref=w[0], b_ref=w[1], c=w[2], mu_ref=w[3], viscosibility=w[4]),
                rock_cp=dict(p_ref=r[0], c=r[1]), pvdg=d["pvdg"], pvto=pvto, swof=d["swof"], sgof=d["sgof"],
                rhoS=d["rhoS"])


def bo_case(d):
    """Grid, rock, deck and wells of a black-oil fixture."""
    g = cartesian_grid(d["dims"], d["phys"])
    rock = make_rock(g, d["perm"][:, None], float(d["poro"]))
    return g, rock, bo_deck(d), wells_from(d)


def bo_state(d, prefix):
    from pymrst_b200.blackoil import BOState
    return BOState(pressure=d[prefix + "p"].copy(), s=d[prefix + "s"].copy(), rs=d[prefix + "rs"].copy(),
                   status=d[prefix + "status"].copy(), qWs=d[prefix + "qWs"].copy(), qOs=d[prefix + "qOs"].copy(),
                   qGs=d[prefix + "qGs"].copy(), bhp=d[prefix + "bhp"].copy())
