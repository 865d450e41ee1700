"""Host-side model inputs with the reference's field names: units, rock,
wells and the simple AD fluid.

These are inputs, built once on the host; none of them is on the hot path.
They exist so that workloads can be built where the reference is not
installed.  Reference objects with the same attribute names are accepted
everywhere these are.

* `make_rock` mirrors pymrst/params/rock/make_rock.py:14-41.
* `add_well` mirrors pymrst/params/wells_and_bc/add_well.py:16-130 for
  vertical (`dir='z'`) Peaceman wells (pymrst/utils/compute_well_index.py:64-125)
  with the reference's reference-depth rule (add_well.py:240-272).
* `init_simple_adi_fluid` mirrors
  pymrst/modules/ad_props/init_simple_adi_fluid.py:94-260 for two phases and
  also records the parameters (`p_ref`, end points) that the device kernels
  need; `fluid_params` recovers the same parameters from a reference
  `ADFluid`, whose curves are closures.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

# Units (pymrst/utils/units.py), SI base.
BARSA = 1.0e5
DAY = 86400.0
DARCY = 9.869232667160128e-13
MILLI = 1.0e-3
CENTI = 1.0e-2
POISE = 0.1
PEACEMAN_TPF_CONSTANT = 0.14


@dataclass
class Rock:
    perm: np.ndarray
    poro: np.ndarray
    ntg: Optional[np.ndarray] = None


def make_rock(g, perm, poro, ntg=None) -> Rock:
    nc = g.cells.num

    def expand(v):
        a = np.asarray(v, dtype=np.float64)
        if a.ndim == 0:
            return np.full((nc, 1), float(a))
        if a.ndim == 1:
            return np.tile(a, (nc, 1)) if a.size != nc else a.reshape(nc, 1)
        return a.reshape(nc, -1)

    p = expand(perm)
    if p.shape[1] not in (1, 3, 6):
        raise ValueError("permeability must have 1, 3 or 6 columns in 3D")
    rock = Rock(perm=p, poro=expand(poro).ravel())
    if ntg is not None:
        rock.ntg = expand(ntg).ravel()
    return rock


def pore_volume(g, rock) -> np.ndarray:
    pv = np.asarray(rock.poro, dtype=float) * np.asarray(g.cells.volumes, dtype=float)
    if getattr(rock, "ntg", None) is not None:
        pv = pv * rock.ntg
    return pv


@dataclass
class Well:
    cells: np.ndarray
    type: str
    val: float
    r: np.ndarray
    dir: str
    WI: np.ndarray
    dZ: np.ndarray
    name: str
    compi: np.ndarray
    refDepth: float
    sign: int = 0
    status: bool = True


def _perm_diag(rock, cells) -> np.ndarray:
    perm = np.asarray(rock.perm, dtype=float)
    if perm.ndim == 1:
        perm = perm[:, None]
    perm = perm[cells]
    if perm.shape[1] == 1:
        return np.repeat(perm, 3, axis=1)
    if perm.shape[1] == 3:
        return perm
    return perm[:, [0, 3, 5]]


def _cell_dims(g, cells) -> np.ndarray:
    """Bounding-box extents of Cartesian cells from their face centroids."""
    out = np.zeros((cells.size, 3))
    fp = np.asarray(g.cells.facePos)
    cf = np.asarray(g.cells.faces)
    fc = np.asarray(g.faces.centroids)
    for n, c in enumerate(cells):
        pts = fc[cf[fp[c]:fp[c + 1]]]
        out[n] = pts.max(axis=0) - pts.min(axis=0)
    return out


def add_well(wells: Optional[List[Well]], g, rock, cells, well_type="bhp",
             val=0.0, radius=0.1, well_dir="z", name=None, skin=0.0,
             compi=None, ref_depth=None, sign=0, gravity=None, wi=None) -> List[Well]:
    """Append a vertical Peaceman well perforating `cells`."""
    wells = list(wells) if wells is not None else []
    cells = np.asarray(cells, dtype=np.int64).ravel()
    if cells.size == 0:
        return wells
    if cells.min() < 0 or cells.max() >= g.cells.num:
        raise IndexError("well completion cell index out of range")
    if str(well_dir).lower() != "z":
        raise ValueError("only vertical (z) wells are built here; pass WI for others")
    well_type = str(well_type).lower()
    radius_arr = np.broadcast_to(np.asarray(radius, float), cells.shape).astype(float)
    skin_arr = np.broadcast_to(np.asarray(skin, float), cells.shape).astype(float)
    if wi is None:
        dims = _cell_dims(g, cells)
        perm = _perm_diag(rock, cells)
        d1, d2, ell = dims[:, 0], dims[:, 1], dims[:, 2]
        k1, k2 = perm[:, 0], perm[:, 1]
        with np.errstate(divide="ignore", invalid="ignore"):
            k21 = np.where(k1 > 0, k2 / k1, 0.0)
            k12 = np.where(k2 > 0, k1 / k2, 0.0)
        numerator = 2 * PEACEMAN_TPF_CONSTANT * np.sqrt(d1**2 * np.sqrt(k21) + d2**2 * np.sqrt(k12))
        re = numerator / (k21**0.25 + k12**0.25)
        re[~np.isfinite(re)] = 0.0
        kh = ell * np.sqrt(k1 * k2)
        wi_arr = 2 * np.pi * kh / (np.log(re / radius_arr) + skin_arr)
    else:
        wi_arr = np.broadcast_to(np.asarray(wi, float), cells.shape).astype(float)
    compi_arr = np.array([1.0, 0.0, 0.0]) if compi is None else np.asarray(compi, float).ravel()
    down = np.array([0.0, 0.0, 1.0])
    if gravity is not None and np.linalg.norm(np.ravel(gravity)[:3]) > 0:
        down = np.ravel(gravity)[:3] / np.linalg.norm(np.ravel(gravity)[:3])
    depth = np.asarray(g.cells.centroids)[cells] @ down
    if ref_depth is None:
        if gravity is not None and np.linalg.norm(np.ravel(gravity)[:3]) > 0:
            ref_depth = float((np.asarray(g.nodes.coords) @ down).min())
        else:
            ref_depth = 0.0
    if well_type == "rate" and val != 0.0:
        sign = int(np.sign(val))
    wells.append(Well(cells=cells, type=well_type, val=float(val), r=radius_arr,
                      dir="z", WI=wi_arr, dZ=depth - float(ref_depth),
                      name=f"W{len(wells) + 1}" if name is None else name,
                      compi=compi_arr, refDepth=float(ref_depth), sign=int(sign)))
    return wells


@dataclass
class FluidParams:
    """Parameters of a two-phase simple AD fluid, water first.

    b_i(p) = b0_i * exp(c_i * (p - p_ref)) (b0_i when c_i == 0);
    kr_i(s) = clamp((s - sl_i) / (su_i - sl_i), 0, 1) ** n_i, or s ** n_i when
    sl_i == 0 and su_i == 1 (init_simple_adi_fluid.py:217-239).
    """
    mu: np.ndarray
    rhoS: np.ndarray
    n: np.ndarray
    c: np.ndarray
    p_ref: float
    b0: np.ndarray
    sl: np.ndarray
    su: np.ndarray

    @property
    def plain_kr(self) -> np.ndarray:
        return (self.sl == 0.0) & (self.su == 1.0)


class SimpleFluid:
    """Two-phase simple AD fluid with numpy-callable curves (the reference
    `ADFluid` contract used by the oil-water model and CPR: `b_w`, `b_o`,
    `kr_w`, `kr_o`, `mu`, `rhoS`, `b(p)`, `disgas`, `vapoil`)."""

    disgas = False
    vapoil = False
    pc_ow = None

    def __init__(self, params: FluidParams):
        self.params = params
        self.mu = params.mu.copy()
        self.rhoS = params.rhoS.copy()
        self.n = params.n.copy()
        self.c = params.c.copy()
        self.n_phases_declared = 2

    def _b(self, i, p):
        prm = self.params
        p = np.asarray(p, dtype=float)
        if prm.c[i] == 0.0:
            return p * 0.0 + prm.b0[i]
        return prm.b0[i] * np.exp(prm.c[i] * (p - prm.p_ref))

    def _kr(self, i, s):
        prm = self.params
        s = np.asarray(s, dtype=float)
        if prm.plain_kr[i]:
            return s ** prm.n[i]
        u = (s - prm.sl[i]) / (prm.su[i] - prm.sl[i])
        return np.maximum(np.minimum(u, 1.0), 0.0) ** prm.n[i]

    def b_w(self, p):
        return self._b(0, p)

    def b_o(self, p):
        return self._b(1, p)

    def kr_w(self, s):
        return self._kr(0, s)

    def kr_o(self, s):
        return self._kr(1, s)

    def b(self, p, *unused):
        return [self.b_w(p), self.b_o(p)]


def init_simple_adi_fluid(mu, rho, n=(1.0, 1.0), c=(0.0, 0.0), p_ref=0.0,
                          b=None, smin=None) -> SimpleFluid:
    """Two-phase (water, oil) simple fluid."""
    mu = np.asarray(mu, float).ravel()
    rho = np.asarray(rho, float).ravel()
    n = np.asarray(n, float).ravel()
    c = np.asarray(c, float).ravel()
    if not (mu.size == rho.size == n.size == c.size == 2):
        raise ValueError("this fluid has exactly two phases (water, oil)")
    if np.any(c < 0):
        raise ValueError("compressibilities must be non-negative")
    b0 = np.ones(2) if b is None else np.asarray(b, float).ravel()[:2]
    smin = np.zeros(2) if smin is None else np.asarray(smin, float).ravel()[:2]
    if smin.sum() >= 0.99:
        raise ValueError("sum of connate/critical saturations must be < 1")
    sl = smin.copy()
    su = 1.0 - smin.sum() + smin
    return SimpleFluid(FluidParams(mu=mu, rhoS=rho, n=n, c=c, p_ref=float(p_ref),
                                   b0=b0, sl=sl, su=su))


def fluid_params(fluid) -> FluidParams:
    """Parameters of `fluid`: read directly from a `SimpleFluid`, or recovered
    from a reference `ADFluid` by evaluating its closures and checking the
    recovered model against them.  Anything that is not the simple
    exponential-b / power-law-kr fluid is rejected."""
    if isinstance(fluid, SimpleFluid):
        return fluid.params
    if getattr(fluid, "disgas", False) or getattr(fluid, "vapoil", False):
        raise ValueError("dissolved-gas / vaporised-oil fluids are not supported by this path")
    if getattr(fluid, "pc_ow", None) is not None:
        raise ValueError("capillary pressure is not supported by this path")
    mu = np.asarray(fluid.mu, float).ravel()[:2]
    rhoS = np.asarray(fluid.rhoS, float).ravel()[:2]
    n = np.asarray(getattr(fluid, "n"), float).ravel()[:2]
    c = np.asarray(getattr(fluid, "c"), float).ravel()[:2]
    p_probe = np.array([0.0, 1.0e7, 3.0e7])
    b_w = np.asarray(fluid.b_w(p_probe), float)
    b_o = np.asarray(fluid.b_o(p_probe), float)
    # b(p) = exp(c p + beta): with unit scale, p_ref = -beta / c.
    b0 = np.ones(2)
    p_ref = 0.0
    for i, bb in enumerate((b_w, b_o)):
        if c[i] == 0.0:
            b0[i] = bb[0]
    ci = [i for i in range(2) if c[i] != 0.0]
    if ci:
        refs = [-np.log((b_w, b_o)[i][0]) / c[i] for i in ci]
        p_ref = float(refs[0])
        if len(refs) == 2 and not np.isclose(refs[0], refs[1], rtol=1e-9, atol=1e-3):
            raise ValueError("phases with different reference pressures are not supported")
    kr_pts = getattr(fluid, "krPts", None) or {}
    sl, su = np.zeros(2), np.ones(2)
    for i, key in enumerate(("w", "o")):
        pts = kr_pts.get(key)
        if pts is not None:
            pts = np.asarray(pts, float).reshape(-1, 4)[0]
            sl[i], su[i] = pts[0], pts[2]
    prm = FluidParams(mu=mu, rhoS=rhoS, n=n, c=c, p_ref=p_ref, b0=b0, sl=sl, su=su)
    probe = SimpleFluid(prm)
    s_probe = np.linspace(0.0, 1.0, 11)
    checks = [
        (probe.b_w(p_probe), b_w), (probe.b_o(p_probe), b_o),
        (probe.kr_w(s_probe), np.asarray(fluid.kr_w(s_probe), float)),
        (probe.kr_o(s_probe), np.asarray(fluid.kr_o(s_probe), float)),
    ]
    for mine, theirs in checks:
        if not np.allclose(mine, theirs, rtol=1e-12, atol=1e-300):
            raise ValueError("fluid is not a simple exponential-b / power-law-kr fluid")
    return prm


@dataclass
class BoundaryCondition:
    """Boundary conditions on faces (reference params/wells_and_bc/types.py);
    `sat` the saturations of what flows in (transport)."""
    face: np.ndarray = field(default_factory=lambda: np.zeros(0, dtype=np.int64))
    type: List[str] = field(default_factory=list)
    value: np.ndarray = field(default_factory=lambda: np.zeros(0))
    sat: np.ndarray = field(default_factory=lambda: np.zeros((0, 0)))


@dataclass
class Source:
    """Volumetric cell sources, injection positive; `sat` the saturations of
    what is injected (transport)."""
    cell: np.ndarray = field(default_factory=lambda: np.zeros(0, dtype=np.int64))
    rate: np.ndarray = field(default_factory=lambda: np.zeros(0))
    sat: np.ndarray = field(default_factory=lambda: np.zeros((0, 0)))


def _sat_rows(sat, n):
    if sat is None:
        return np.zeros((n, 0))
    a = np.atleast_2d(np.asarray(sat, float))
    return np.ascontiguousarray(np.broadcast_to(a, (n, a.shape[1])))


def _append_rows(old, new):
    if old.size == 0:
        return new
    if new.shape[1] != old.shape[1]:
        raise ValueError("saturation columns do not match the existing ones")
    return np.vstack([old, new])


def add_bc(bc, faces, bctype, values, sat=None) -> BoundaryCondition:
    """Append boundary conditions of one type (reference add_bc.py:13-41)."""
    faces = np.asarray(faces, dtype=np.int64).ravel()
    if faces.size == 0:
        return bc
    bc = BoundaryCondition() if bc is None else bc
    vals = np.broadcast_to(np.asarray(values, float), faces.shape).astype(float)
    if np.isin(faces, bc.face).any():
        raise ValueError("new boundary condition overlaps with existing conditions")
    bc.face = np.concatenate([bc.face, faces])
    bc.type = list(bc.type) + [str(bctype).lower()] * faces.size
    bc.value = np.concatenate([bc.value, vals])
    bc.sat = _append_rows(bc.sat, _sat_rows(sat, faces.size))
    return bc


def add_source(src, cells, rates, sat=None) -> Source:
    """Append cell sources (reference add_source)."""
    cells = np.asarray(cells, dtype=np.int64).ravel()
    src = Source() if src is None else src
    if np.isin(cells, src.cell).any():
        raise ValueError("new source terms conflict with existing source terms")
    src.cell = np.concatenate([src.cell, cells])
    src.rate = np.concatenate([src.rate, np.broadcast_to(np.asarray(rates, float), cells.shape)])
    src.sat = _append_rows(src.sat, _sat_rows(sat, cells.size))
    return src
