"""Two-phase incompressible transport on the GPU with the interface of the
reference's explicit_transport / implicit_transport
(pymrst/modules/incomp/transport/__init__.py:285-402): `explicit_transport(
state, g, tf, rock, fluid, wells, src, bc, gravity, dt, max_dt, dt_factor,
satwarn)` and `implicit_transport(state, g, tf, rock, fluid, wells, src, bc,
gravity, nltol, lstrials, maxnewt, tsref, resred)`, each returning the state
with `state.s` advanced by tf seconds.

The substeps (explicit: the residual, the stable-step estimate and the
clock; implicit: residual, Jacobian, the FGMRES solve preconditioned by a
Gauss-Seidel sweep in flow order, and line-search trials)
run on the device through the `pmb_transport_*` entry points
(`csrc/transport.cu`).  The host forms what the reference freezes for a
call: the water source of every cell (`transport_source`), the gravity flux
of every interface (`gravity_flux`) and the constant gravity part of the
step estimate; and for the implicit loop, reads one residual norm per Newton
trial.

The fluid is Corey (kr = s^n_w, (1-s)^n_o): `init_simple_fluid` of this
module, or the reference's init_simple_fluid / init_corey_fluid without
residual saturations (its exponents are read from the fluid and checked
against its relative permeabilities).  Capillary pressure is not part of the
reference's transport either.
"""

from __future__ import annotations

import math
from typing import Optional, Sequence

import numpy as np

from . import _native as N
from .ow_model import _opts_struct, _torch, default_cpr_options
from .params import pore_volume


class CoreyFluid:
    """Two incompressible phases with Corey relative permeabilities
    s^n[0], (1-s)^n[1] (the reference's init_simple_fluid)."""

    def __init__(self, mu, rho, n=(1.0, 1.0)):
        self.mu = np.asarray(mu, dtype=float).ravel()
        self.rho = np.asarray(rho, dtype=float).ravel()
        self.n = np.asarray(n, dtype=float).ravel()
        if not (self.mu.size == self.rho.size == self.n.size == 2):
            raise ValueError("mu, rho and the Corey exponents need two entries each")

    @property
    def n_phases(self):
        return 2

    def properties(self, state=None):
        return self.mu, self.rho

    def saturation(self, state):
        return state.s

    def relperm(self, s):
        s1 = np.atleast_2d(np.asarray(s, dtype=float))[:, 0]
        return np.column_stack([s1 ** self.n[0], (1.0 - s1) ** self.n[1]])

    def d_relperm(self, s):
        s1 = np.atleast_2d(np.asarray(s, dtype=float))[:, 0]
        return np.column_stack([self.n[0] * s1 ** (self.n[0] - 1.0), self.n[1] * (1.0 - s1) ** (self.n[1] - 1.0)])

    def mobility(self, s):
        return self.relperm(s) / self.mu

    def d_mobility(self, s):
        return self.d_relperm(s) / self.mu


def init_simple_fluid(mu, rho, n=(1.0, 1.0)) -> CoreyFluid:
    return CoreyFluid(mu, rho, n)


def _corey_params(fluid):
    """(mu_w, mu_o, n_w, n_o) of a Corey fluid, checked against its own
    relative permeabilities."""
    mu = np.asarray(fluid.mu, dtype=float).ravel()
    if mu.size != 2:
        raise ValueError("transport needs a two-phase fluid")
    if isinstance(fluid, CoreyFluid):
        n = fluid.n
    else:
        fn = fluid.relperm
        env = dict(zip(fn.__code__.co_freevars, (c.cell_contents for c in fn.__closure__ or ()))) \
            if hasattr(fn, "__code__") else {}
        if "n" not in env:
            raise ValueError("transport on the device needs a Corey fluid (init_simple_fluid)")
        n = np.asarray(env["n"], dtype=float).ravel()
    s = np.linspace(0.0, 1.0, 41)
    want = np.column_stack([s ** n[0], (1.0 - s) ** n[1]])
    got = np.asarray(fluid.relperm(np.column_stack([s, 1.0 - s])), dtype=float)
    if got.shape != want.shape or not np.allclose(got, want, rtol=1e-14, atol=0.0):
        raise ValueError("transport on the device needs a Corey fluid s^n_w, (1-s)^n_o without residual "
                         "saturations")
    return np.array([mu[0], mu[1], n[0], n[1]], dtype=float)


def transport_source(state, g, fluid, wells=None, src=None, bc=None) -> np.ndarray:
    """Water source per cell (m^3/s): inflow scaled by the fractional flow
    of its injected composition, outflow total (transport_source,
    :33-93)."""
    nc = g.cells.num
    cells, flux, comp = [], [], []
    for k, w in enumerate(wells or []):
        wc = np.asarray(w.cells, dtype=np.int64).ravel()
        cells.append(wc)
        flux.append(np.asarray(state.wellSol[k].flux, dtype=float).ravel())
        comp.append(np.tile(np.asarray(w.compi, dtype=float).ravel()[:2], (wc.size, 1)))
    if src is not None and np.size(src.cell) > 0:
        cells.append(np.asarray(src.cell, dtype=np.int64).ravel())
        flux.append(np.asarray(src.rate, dtype=float).ravel())
        comp.append(np.atleast_2d(np.asarray(src.sat, dtype=float))[:, :2])
    if bc is not None and np.size(bc.face) > 0:
        faces = np.asarray(bc.face, dtype=np.int64).ravel()
        if np.size(getattr(bc, "sat", [])) == 0:
            raise ValueError("transport needs bc saturations")
        nb = np.asarray(g.faces.neighbors)[faces]
        if not np.all(np.sum(nb == -1, axis=1) == 1):
            raise ValueError("boundary condition supplied on internal face")
        cell = nb.sum(axis=1) + 1
        sign = np.where(nb[:, 0] == -1, 1.0, -1.0)
        types = np.array(bc.type)
        sat = np.atleast_2d(np.asarray(bc.sat, dtype=float))[:, :2]
        dirichlet, neumann = types == "pressure", types == "flux"
        cells += [cell[dirichlet], cell[neumann]]
        flux += [sign[dirichlet] * np.asarray(state.flux, dtype=float)[faces[dirichlet]],
                 np.asarray(bc.value, dtype=float)[neumann]]
        comp += [sat[dirichlet], sat[neumann]]
    if not cells:
        return np.zeros(nc)
    cells, flux, comp = np.concatenate(cells), np.concatenate(flux), np.vstack(comp)
    inj = np.zeros(nc, dtype=bool)
    prod = np.zeros(nc, dtype=bool)
    inj[cells[flux > 0]] = True
    prod[cells[flux < 0]] = True
    if np.any(inj & prod):
        raise ValueError("injection and production in the same cell is unsupported")
    inflow = flux > 0
    if inflow.any():
        m = fluid.mobility(comp[inflow])
        flux = flux.copy()
        flux[inflow] *= m[:, 0] / m.sum(axis=1)
    return np.bincount(cells, weights=flux, minlength=nc)


def _perm3(rock, nc):
    k = np.asarray(rock.perm, dtype=float)
    if k.ndim == 1:
        k = k[:, None]
    K = np.zeros((nc, 3, 3))
    if k.shape[1] == 1:
        K[:, 0, 0] = K[:, 1, 1] = K[:, 2, 2] = k[:, 0]
    elif k.shape[1] == 3:
        K[:, 0, 0], K[:, 1, 1], K[:, 2, 2] = k[:, 0], k[:, 1], k[:, 2]
    elif k.shape[1] == 6:
        K[:, 0, 0], K[:, 0, 1], K[:, 0, 2] = k[:, 0], k[:, 1], k[:, 2]
        K[:, 1, 0], K[:, 1, 1], K[:, 1, 2] = k[:, 1], k[:, 3], k[:, 4]
        K[:, 2, 0], K[:, 2, 1], K[:, 2, 2] = k[:, 2], k[:, 4], k[:, 5]
    else:
        raise ValueError("permeability must have 1, 3 or 6 columns")
    return K


def gravity_flux(g, rock, delta_rho_g) -> np.ndarray:
    """Per face: 2 / the sum over its half-faces of 1 / (n . K delta_rho_g),
    0 where that is not finite (gravity_flux, :96-111)."""
    dg = np.asarray(delta_rho_g, dtype=float).ravel()
    nf = g.faces.num
    if not np.linalg.norm(dg) > 0:
        return np.zeros(nf)
    dim = np.asarray(g.faces.normals).shape[1]
    nc = g.cells.num
    cf = np.asarray(g.cells.faces, dtype=np.int64).ravel()
    cell_no = np.repeat(np.arange(nc), np.diff(np.asarray(g.cells.facePos)))
    K = _perm3(rock, nc)[:, :dim, :dim]
    nkg = np.einsum("hi,hij,j->h", np.asarray(g.faces.normals, dtype=float)[cf], K[cell_no], dg[:dim])
    with np.errstate(divide="ignore"):
        out = 2.0 / np.bincount(cf, weights=1.0 / nkg, minlength=nf)
    out[~np.isfinite(out)] = 0.0
    return out


def _gravity_vector(gravity, dim):
    if gravity is None:
        return np.zeros(dim)
    gv = np.asarray(gravity, dtype=float).ravel()
    return gv[:dim] if gv.size >= dim else np.concatenate([gv, np.zeros(dim - gv.size)])


_HANDLES = {}


def _handle(g, pv):
    """A device handle per grid (interfaces and pore volumes), cached."""
    Nall = np.asarray(g.faces.neighbors, dtype=np.int64)
    internal = np.all(Nall >= 0, axis=1)
    Nn = np.ascontiguousarray(Nall[internal], dtype=np.int32)
    key = (id(g), g.cells.num, hash(Nn.tobytes()), hash(pv.tobytes()))
    h = _HANDLES.get(key)
    if h is None:
        torch = _torch()
        hd = N.c_vp()
        pvc = np.ascontiguousarray(pv, dtype=np.float64)
        N.check(N.lib().pmb_transport_create(int(g.cells.num), int(Nn.shape[0]), N.as_p(Nn, N.C.c_int32),
                                             N.as_p(pvc, N.C.c_double), torch.cuda.current_stream().cuda_stream,
                                             N.C.byref(hd)))
        h = (hd, internal)
        if len(_HANDLES) > 8:
            for k, (old, _) in list(_HANDLES.items())[:4]:
                N.lib().pmb_transport_destroy(old)
                del _HANDLES[k]
        _HANDLES[key] = h
    return h


def _prepare(state, g, rock, fluid, wells, src, bc, gravity):
    """Device handle with the call's frozen flow; the water saturations on
    the device; the Corey parameters; the gravity-estimate flux."""
    torch = _torch()
    params = _corey_params(fluid)
    pv = np.asarray(pore_volume(g, rock), dtype=float)
    hd, internal = _handle(g, pv)
    q = transport_source(state, g, fluid, wells=wells, src=src, bc=bc)
    gvec = _gravity_vector(gravity, int(np.asarray(g.faces.normals).shape[1]))
    rho = np.asarray(fluid.rho, dtype=float).ravel()
    gflux = gravity_flux(g, rock, gvec * (rho[0] - rho[1]))[internal]
    flux = np.asarray(state.flux, dtype=float).ravel()[internal]
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda")
    d_flux, d_g, d_q = dev(flux), dev(gflux), dev(q)
    N.check(N.lib().pmb_transport_set_flow(hd, N.ptr(d_flux), N.ptr(d_g), N.ptr(d_q),
                                           N.as_p(params, N.C.c_double)))
    s = dev(np.asarray(state.s, dtype=float)[:, 0])
    return hd, s, params, gvec, internal, (d_flux, d_g, d_q)


def explicit_transport(state, g, tf: float, rock, fluid, wells: Optional[Sequence] = None, src=None, bc=None,
                       gravity=None, dt: Optional[float] = None, max_dt: float = np.inf, dt_factor: float = 0.5,
                       satwarn: float = math.sqrt(np.finfo(float).eps)):
    """Forward-Euler transport over tf seconds (fixed substeps dt, or the
    stable-step estimate)."""
    hd, s, params, gvec, internal, keep = _prepare(state, g, rock, fluid, wells, src, bc, gravity)
    # the constant gravity part of the estimate: the segregation slope over
    # a saturation sweep times the gravity flux of a unit density difference
    rho = np.asarray(fluid.rho, dtype=float).ravel()
    gf_est = gravity_flux(g, rock, -gvec)[internal]
    s1 = np.linspace(0.0, 1.0, 101)
    ml = fluid.relperm(np.column_stack([s1, 1 - s1])) / np.asarray(fluid.mu, dtype=float).min()
    seg = ml[:, 0] * ml[:, 1] / ml.sum(axis=1)
    dgs = np.max(np.abs(np.diff(seg)) / np.diff(s1))
    gwave = float(np.max(np.abs(dgs * gf_est * abs(rho[1] - rho[0])), initial=0.0))
    out = (N.C.c_double * 4)()
    N.check(N.lib().pmb_transport_explicit(hd, N.ptr(s), float(tf), float(dt) if dt is not None else 0.0,
                                           float(max_dt), float(dt_factor), float(satwarn), gwave, out))
    if out[2]:
        raise AssertionError("explicit_transport: saturation outside [0, 1] beyond satwarn")
    if out[3]:
        raise AssertionError("explicit_transport: transport failed")
    sw = s.cpu().numpy()
    state.s = np.column_stack([sw, 1.0 - sw])
    explicit_transport.last_stats = dict(substeps=int(out[0]))
    return state


def implicit_transport(state, g, tf: float, rock, fluid, wells: Optional[Sequence] = None, src=None, bc=None,
                       gravity=None, nltol: float = 1e-6, lstrials: int = 20, maxnewt: int = 25, tsref: int = 12,
                       resred: float = 0.99, cpr_options: Optional[dict] = None):
    """Backward-Euler transport over tf seconds: Newton with a bisection
    line search and substep halving / growth."""
    hd, s, params, gvec, internal, keep = _prepare(state, g, rock, fluid, wells, src, bc, gravity)
    opts = _opts_struct(default_cpr_options(**({"rtol": 1e-12, "maxiter": 500} | dict(cpr_options or {}))))
    out = (N.C.c_double * 6)()
    N.check(N.lib().pmb_transport_implicit(hd, N.ptr(s), float(tf), float(nltol), int(lstrials), int(maxnewt),
                                           int(tsref), float(resred), N.C.byref(opts), out))
    sw = s.cpu().numpy()
    if not (out[0] >= tf) or np.any(np.isnan(sw)):
        raise AssertionError(f"implicit_transport failed: t={out[0]:.3e} of {tf:.3e}, "
                             f"minimum substep {tf * 2.0 ** (-tsref):.3e} reached")
    state.s = np.column_stack([sw, 1.0 - sw])
    implicit_transport.last_stats = dict(substeps=int(out[1]), newton=int(out[2]), krylov=int(out[3]),
                                         missed_tolerance=int(out[4]))
    return state
