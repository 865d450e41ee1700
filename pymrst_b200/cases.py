"""Seeded synthetic oil-water workloads of the benchmark shapes.

The reference measures on its own examples and on SPE10; neither dataset is
available here, so these generators stand in with the stated shapes, sizes and
value distributions (all seeded with numpy's default_rng):

* `five_spot(dims, cell_size, seed)`: lognormal permeability, log k ~
  N(ln(100 mD), sigma) smoothed by a 3x3x3 box filter; porosity 0.2; four rate
  water injectors at the corner columns (compi [1, 0]) and one BHP producer
  (100 bar) at the centre column; initial p = 200 bar, sW = 0.1.
* `channelised(dims=(60, 220, 85), cell_size=(6.1, 3.05, 0.61), seed)`: the
  upper 35 layers smooth lognormal (sigma 1.5), the lower layers binary
  sinusoidal channels (2000 mD in 1 mD) with amplitude, wavelength and width
  drawn per layer; porosity 0.05 + 0.30 * normalised log-permeability; same
  well pattern.
* `incompressible_quarter_five_spot(dims=(64, 64, 8), cell_size=(10, 10, 2),
  seed)`: the lognormal permeability (sigma 1) of `five_spot`, porosity 0.2,
  one rate injector of 1e-3 m^3/s down column (0, 0) and one bhp producer at
  100 bar down the opposite corner column, a single-phase fluid of 1 cP and
  1000 kg/m^3; gravity off.
* `ow_fluid()`: Corey n = 2 with Swc = Sor = 0.1, mu_w = 1 cP, mu_o = 5 cP,
  rho 1000 / 800 kg/m^3, compressibility 1e-5 / bar for both phases,
  p_ref = 200 bar.
* `synthetic_blackoil_deck()`: a live-oil / dry-gas black-oil description in
  the layout of a parsed deck (PVTW, ROCK, PVDG, PVTO, SWOF, SGOF, surface
  densities; SI units), with smooth analytic tables of the usual shapes: six
  PVTO keys (Rs 10 .. 160 sm^3/sm^3, bubble points 15 .. 240 bar), each with
  an undersaturated branch of four rows; gas FVF ~ 1/p; Corey-like relative
  permeabilities with Swc = 0.15 and small capillary pressures.
* `blackoil_box(dims, cell_size, seed, spacing)`: that deck on a box;
  permeability lognormal (sigma 0.5, smoothed) times a layer factor cycling
  through 500, 50, 200, 120 mD; porosity 0.3; a lattice of gas injectors and
  bhp producers plus one oil-rate producer (see the function); initial p =
  300 bar at the top plus an oil gradient, sW = 0.2, undersaturated with
  Rs = 120.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import List

import numpy as np

from .grid import Grid, cartesian_grid, cell_index
from .params import (BARSA, CENTI, DARCY, DAY, MILLI, POISE, Rock, SimpleFluid, Well,
                     add_well, init_simple_adi_fluid, make_rock)

MD = MILLI * DARCY


@dataclass
class OWCase:
    name: str
    grid: Grid
    rock: Rock
    fluid: SimpleFluid
    wells: List[Well]
    p0: float
    sw0: float
    dt: float
    nsteps: int
    gravity: float


def hydrostatic_pressure(case: "OWCase", p_top: float = None) -> np.ndarray:
    """Cell pressures in oil-hydrostatic equilibrium below `p_top` (at the
    shallowest cell centre), integrating dp/dz = rho_o b_o(p) g cell by cell
    down each column."""
    p_top = case.p0 if p_top is None else float(p_top)
    z = np.asarray(case.grid.cells.centroids)[:, 2]
    if not case.gravity:
        return np.full(z.size, p_top)
    prm = case.fluid.params
    rho = prm.rhoS[1]
    p = np.empty_like(z)
    zmin = z.min()
    # fixed-point on the compressible density (converges in a few sweeps)
    p[:] = p_top + rho * case.gravity * (z - zmin)
    for _ in range(5):
        b = prm.b0[1] * np.exp(prm.c[1] * (0.5 * (p + p_top) - prm.p_ref))
        p = p_top + rho * b * case.gravity * (z - zmin)
    return p


def ow_fluid() -> SimpleFluid:
    return init_simple_adi_fluid(mu=np.array([1.0, 5.0]) * CENTI * POISE, rho=[1000.0, 800.0],
                                 n=[2, 2], c=[1e-5 / BARSA, 1e-5 / BARSA], p_ref=200 * BARSA,
                                 smin=[0.1, 0.1])


def _box_smooth(a: np.ndarray) -> np.ndarray:
    """3x3x3 box filter with 'nearest' edges."""
    from scipy.ndimage import uniform_filter
    return uniform_filter(a, size=3, mode="nearest")


def lognormal_logperm(dims, rng, sigma=1.0, mean_md=100.0) -> np.ndarray:
    return _box_smooth(rng.normal(np.log(mean_md), sigma, size=tuple(dims)))


def _five_spot_wells(g: Grid, rock: Rock, rate: float, bhp: float, gravity: float):
    nx, ny, nz = g.cartDims
    k = np.arange(nz)
    gvec = np.array([0.0, 0.0, gravity]) if gravity else None
    wells = None
    for (i, j) in ((0, 0), (nx - 1, 0), (0, ny - 1), (nx - 1, ny - 1)):
        wells = add_well(wells, g, rock, cell_index(g, i, j, k), well_type="rate", val=rate,
                         compi=np.array([1.0, 0.0]), sign=1, gravity=gvec)
    wells = add_well(wells, g, rock, cell_index(g, nx // 2, ny // 2, k), well_type="bhp",
                     val=bhp, compi=np.array([0.0, 1.0]), sign=-1, gravity=gvec)
    return wells


def five_spot(dims=(100, 100, 10), cell_size=(10.0, 10.0, 2.0), seed=1, sigma=1.0,
              nsteps=20, dt_days=10.0, gravity=9.80665, pv_fraction=0.25) -> OWCase:
    rng = np.random.default_rng(seed)
    dims = tuple(int(v) for v in dims)
    g = cartesian_grid(dims, [d * s for d, s in zip(dims, cell_size)])
    logk = lognormal_logperm(dims, rng, sigma)
    perm = np.exp(logk).ravel(order="F") * MD
    rock = make_rock(g, perm[:, None], 0.2)
    pvtot = float(np.sum(rock.poro * g.cells.volumes))
    rate = pv_fraction * pvtot / (nsteps * dt_days * DAY) / 4.0
    wells = _five_spot_wells(g, rock, rate, 100 * BARSA, gravity)
    return OWCase(f"five_spot_{dims[0]}x{dims[1]}x{dims[2]}", g, rock, ow_fluid(), wells,
                  200 * BARSA, 0.1, dt_days * DAY, nsteps, gravity)


def channelised(dims=(60, 220, 85), cell_size=(6.1, 3.05, 0.61), seed=2, n_smooth=35,
                nsteps=20, dt_days=10.0, gravity=9.80665, pv_fraction=0.25) -> OWCase:
    rng = np.random.default_rng(seed)
    nx, ny, nz = (int(v) for v in dims)
    g = cartesian_grid((nx, ny, nz), [nx * cell_size[0], ny * cell_size[1], nz * cell_size[2]])
    logk = np.empty((nx, ny, nz))
    top = min(n_smooth, nz)
    if top:
        logk[:, :, :top] = lognormal_logperm((nx, ny, top), rng, sigma=1.5)
    xs = np.arange(nx)[:, None]
    ys = np.arange(ny)[None, :]
    for k in range(top, nz):
        mask = np.zeros((nx, ny), dtype=bool)
        for _ in range(int(rng.integers(2, 5))):
            amp = rng.uniform(2.0, 0.2 * nx)
            wav = rng.uniform(0.3 * ny, 1.5 * ny)
            wid = rng.uniform(2.0, max(2.0, 0.12 * nx))
            x0 = rng.uniform(0, nx)
            ph = rng.uniform(0, 2 * np.pi)
            centre = x0 + amp * np.sin(2 * np.pi * ys / wav + ph)
            mask |= np.abs(xs - centre) <= 0.5 * wid
        logk[:, :, k] = np.where(mask, np.log(2000.0), np.log(1.0))
    perm = np.exp(logk).ravel(order="F") * MD
    lk = logk.ravel(order="F")
    poro = 0.05 + 0.30 * (lk - lk.min()) / max(lk.max() - lk.min(), 1e-300)
    rock = make_rock(g, perm[:, None], poro)
    pvtot = float(np.sum(rock.poro * g.cells.volumes))
    rate = pv_fraction * pvtot / (nsteps * dt_days * DAY) / 4.0
    wells = _five_spot_wells(g, rock, rate, 100 * BARSA, gravity)
    return OWCase(f"channelised_{nx}x{ny}x{nz}", g, rock, ow_fluid(), wells,
                  200 * BARSA, 0.1, dt_days * DAY, nsteps, gravity)


def ensemble_realisations(n: int = 256, seed: int = 3, nx_range=(16, 64), nz_range=(2, 8),
                          cell_size=(10.0, 10.0, 2.0), nsteps: int = 15, dt_days: float = 30.0,
                          gravity: float = 9.80665, pv_fraction: float = 0.25) -> list:
    """Oil-water realisations of varying size: nx, ny uniform in nx_range and
    nz in nz_range (seeded), an independent lognormal permeability each, a
    five-spot each, the shared fluid; 15 steps of 30 days by default."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        nx, ny = (int(v) for v in rng.integers(nx_range[0], nx_range[1] + 1, size=2))
        nz = int(rng.integers(nz_range[0], nz_range[1] + 1))
        out.append(five_spot(dims=(nx, ny, nz), cell_size=cell_size, seed=int(rng.integers(1 << 30)),
                             nsteps=nsteps, dt_days=dt_days, gravity=gravity, pv_fraction=pv_fraction))
    return out


@dataclass
class IncompCase:
    name: str
    grid: Grid
    rock: Rock
    wells: List[Well]
    mu: float
    rho: float


def incompressible_quarter_five_spot(dims=(64, 64, 8), cell_size=(10.0, 10.0, 2.0), seed=0) -> IncompCase:
    rng = np.random.default_rng(seed)
    dims = tuple(int(v) for v in dims)
    g = cartesian_grid(dims, [d * s for d, s in zip(dims, cell_size)])
    perm = np.exp(lognormal_logperm(dims, rng, 1.0)).ravel(order="F") * MD
    rock = make_rock(g, perm[:, None], 0.2)
    nx, ny, nz = dims
    k = np.arange(nz)
    wells = add_well(None, g, rock, cell_index(g, 0, 0, k), well_type="rate", val=1e-3, radius=0.1,
                     compi=np.array([1.0]))
    wells = add_well(wells, g, rock, cell_index(g, nx - 1, ny - 1, k), well_type="bhp", val=100 * BARSA,
                     radius=0.1, compi=np.array([1.0]))
    return IncompCase(f"incomp_{nx}x{ny}x{nz}", g, rock, wells, 1 * CENTI * POISE, 1000.0)


def synthetic_blackoil_deck() -> dict:
    """Black-oil tables in the layout of a parsed deck (SI units): keys
    pvtw, rock_cp, pvdg, pvto (list of (Rs, rows [p, Bo, mu_o])), swof
    (sw, krw, krow, pcow), sgof (sg, krg, krog, pcog) and rhoS (water, oil,
    gas).  Analytic, smooth and monotone; no field data."""
    bar, cp = BARSA, CENTI * POISE
    pg = np.array([10.0, 30.0, 60.0, 100.0, 150.0, 200.0, 260.0, 330.0, 400.0])
    pvdg = np.column_stack([pg * bar, (0.95 + 3e-4 * pg) / pg, (0.012 + 4.5e-5 * pg) * cp])
    keys = np.array([10.0, 40.0, 70.0, 100.0, 130.0, 160.0])
    p_bub = np.array([15.0, 60.0, 105.0, 150.0, 195.0, 240.0])
    pvto = []
    for rs, pb in zip(keys, p_bub):
        dp = np.array([0.0, 80.0, 160.0, 240.0])
        bo_sat, mu_sat = 1.05 + 0.0025 * rs, 1.6 - 0.006 * rs
        rows = np.column_stack([(pb + dp) * bar, bo_sat * np.exp(-1.5e-4 * dp), mu_sat * (1.0 + 1e-3 * dp) * cp])
        pvto.append((float(rs), rows))
    sw = np.linspace(0.15, 1.0, 12)
    u = (sw - 0.15) / 0.85
    swof = np.column_stack([sw, 0.6 * u ** 2.5, (1.0 - u) ** 2, 0.2 * bar * (1.0 - u) ** 2])
    sg = np.linspace(0.0, 0.85, 12)
    v = sg / 0.85
    sgof = np.column_stack([sg, 0.8 * v ** 2, (1.0 - v) ** 3, 0.05 * bar * v])
    return dict(
        pvtw=dict(p_ref=250.0 * bar, b_ref=1.03, c=4.5e-10, mu_ref=0.4 * cp, viscosibility=0.0),
        rock_cp=dict(p_ref=250.0 * bar, c=6e-10),
        pvdg=pvdg, pvto=pvto, swof=swof, sgof=sgof,
        rhoS=np.array([1020.0, 840.0, 0.95]),
    )


@dataclass
class BlackOilCase:
    name: str
    grid: Grid
    rock: Rock
    deck: dict
    wells: List[Well]
    state: object
    dts: np.ndarray


def blackoil_box(dims=(10, 10, 3), cell_size=(30.0, 30.0, 10.0), seed=23, spacing=10, gas_rate=1.0,
                 dt_days=(0.5, 1.0, 2.0, 5.0, 10.0, 10.0, 20.0)) -> BlackOilCase:
    """Gas injection into an undersaturated live-oil box (see the module
    docstring).  Wells on a lattice: gas injectors (total surface rate) down
    the upper half of columns (s/2 + s a, s/2 + s b), bhp producers (250 bar)
    down the lower half of columns (s a, s b), s = `spacing`, and an oil-rate
    producer down the lower half of column (nx-1, ny-1).  Each injector takes
    `gas_rate` sm^3/s and the oil producer 0.012 sm^3/s per 5,400 m^3 of
    perforated pore volume, which liberates gas around the injectors within
    a few steps."""
    from .blackoil import BOState
    rng = np.random.default_rng(seed)
    dims = tuple(int(v) for v in dims)
    nx, ny, nz = dims
    g = cartesian_grid(dims, [d * s for d, s in zip(dims, cell_size)])
    logk = _box_smooth(rng.normal(0.0, 0.5, size=dims))
    layer = np.array([500.0, 50.0, 200.0, 120.0])[np.arange(nz) % 4]
    perm = (np.exp(logk) * layer[None, None, :]).ravel(order="F") * MD
    rock = make_rock(g, perm[:, None], 0.3)
    deck = synthetic_blackoil_deck()
    pv = 0.3 * np.asarray(g.cells.volumes)
    top = np.arange(max(1, nz // 2))
    bottom = np.arange(nz // 2, nz) if nz > 1 else np.arange(1)
    wells, gas, oil, bhp_val = None, [], [], []
    h = spacing // 2
    for i in range(h, nx, spacing):
        for j in range(h, ny, spacing):
            cells = cell_index(g, i, j, top)
            q = gas_rate * float(pv[cells].sum()) / 5400.0
            wells = add_well(wells, g, rock, cells, well_type="rate", val=q, radius=0.1,
                             compi=np.array([0.0, 0.0, 1.0]))
            gas.append(q); oil.append(0.0); bhp_val.append(None)
    for i in range(0, nx, spacing):
        for j in range(0, ny, spacing):
            if (i, j) == (nx - 1, ny - 1):
                continue
            wells = add_well(wells, g, rock, cell_index(g, i, j, bottom), well_type="bhp", val=250.0 * BARSA,
                             radius=0.1, compi=np.array([0.0, 1.0, 0.0]))
            gas.append(0.0); oil.append(0.0); bhp_val.append(250.0 * BARSA)
    cells = cell_index(g, nx - 1, ny - 1, bottom)
    qo = -0.012 * float(pv[cells].sum()) / 5400.0
    wells = add_well(wells, g, rock, cells, well_type="orat", val=qo, radius=0.1, compi=np.array([0.0, 1.0, 0.0]))
    gas.append(0.0); oil.append(qo); bhp_val.append(None)
    nc, nw = g.cells.num, len(wells)
    z = np.asarray(g.cells.centroids)[:, 2]
    p = 300.0 * BARSA + 840.0 * 1.1 * 9.80665 * z
    bhp = np.array([b if b is not None else (p.mean() + 10 * BARSA if q > 0 else p.mean() - 10 * BARSA)
                    for b, q in zip(bhp_val, gas)])
    st = BOState(pressure=p, s=np.column_stack([np.full(nc, 0.2), np.full(nc, 0.8), np.zeros(nc)]),
                 rs=np.full(nc, 120.0), status=np.ones(nc, dtype=np.int64), qWs=np.zeros(nw),
                 qOs=np.array(oil), qGs=np.array(gas), bhp=bhp)
    return BlackOilCase(f"blackoil_{nx}x{ny}x{nz}", g, rock, deck, wells, st,
                        np.asarray(dt_days, dtype=float) * DAY)
