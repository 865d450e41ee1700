"""Oracle: incompressible TPFA pressure system (test infrastructure only).

A numpy restatement of incomp_tpfa (pymrst/modules/incomp/incomp_tpfa.py:
55-211) for single- or multi-phase incompressible fluids on grids without
non-neighbouring connections, solved with SuperLU like the reference.  It
works face by face: each interior interface adds the two-point coupling
ft (p_i - p_j - fg) to its two cells, each Dirichlet face the one-sided
coupling to its cell, each perforation the coupling WI totmob (p_cell - bhp -
dp) to its cell and well.  Checked against the reference's MATLAB goldens and
its own outputs (tests/test_oracle.py).
"""

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla


def _injector(w):
    sign = getattr(w, "sign", None)
    if sign is not None and np.size(sign) and np.all(np.asarray(sign) > 0):
        return True
    return str(w.type).lower() == "rate" and float(np.sum(w.val)) > 0


def pressure_system(G, T, mob, rho, gvec=None, bc=None, src=None, wells=(), use_trans=False):
    """(A, rhs, aux): the (nc + nw)-unknown system and what the flux
    reconstruction needs.  `mob` is nc x nph (kr / mu), `rho` nph."""
    nc, nf = G.cells.num, G.faces.num
    nbr = np.asarray(G.faces.neighbors, dtype=np.int64)
    cf = np.asarray(G.cells.faces, dtype=np.int64)
    cf = cf[:, 0] if cf.ndim > 1 else cf
    hc = np.repeat(np.arange(nc), np.diff(np.asarray(G.cells.facePos)))
    mob = np.atleast_2d(np.asarray(mob, float))
    rho = np.asarray(rho, float).ravel()
    lam = mob.sum(axis=1)
    omega = (mob * rho[: mob.shape[1]]).sum(axis=1) / lam
    gvec = np.zeros(3) if gvec is None else np.resize(np.asarray(gvec, float), 3)
    dim = G.griddim
    interior = (nbr[:, 0] >= 0) & (nbr[:, 1] >= 0)
    side = np.where(nbr[cf, 0] == hc, 1.0, -1.0)
    T = np.asarray(T, float).ravel()
    if use_trans:
        cnt = (nbr >= 0).sum(axis=1)
        ft = T * np.bincount(cf, lam[hc], minlength=nf) / cnt
        th = (ft * cnt)[cf]
    else:
        th = T * lam[hc]
        with np.errstate(divide="ignore"):
            ft = 1.0 / np.bincount(cf, 1.0 / th, minlength=nf)
    dxf = np.asarray(G.faces.centroids)[cf, :dim] - np.asarray(G.cells.centroids)[hc, :dim]
    gp = omega[hc] * (dxf @ gvec[:dim]) if np.any(gvec[:dim]) else np.zeros(cf.size)

    kind = np.zeros(nf, dtype=int)   # 1 pressure, 2 flux
    bval = np.zeros(nf)
    if bc is not None and np.size(bc.face):
        faces = np.asarray(bc.face, dtype=np.int64).ravel()
        types = np.resize(np.array([str(t).lower() for t in np.atleast_1d(bc.type)]), faces.size)
        kind[faces] = np.where(types == "pressure", 1, 2)
        bval[faces] = np.resize(np.asarray(bc.value, float).ravel(), faces.size)
    dirichlet = kind == 1
    # signed gravity sum of interior and Dirichlet faces
    use = interior[cf] | dirichlet[cf]
    fg = np.zeros(nf)
    np.add.at(fg, cf[use], gp[use] * side[use])

    nw = len(wells)
    n = nc + nw
    rows, cols, vals = [], [], []
    rhs = np.zeros(n)
    # interior interfaces: flux out of N0 is ft (p0 - p1 + fg)
    f = np.flatnonzero(interior)
    i, j = nbr[f, 0], nbr[f, 1]
    rows += [i, j, i, j]
    cols += [i, j, j, i]
    vals += [ft[f], ft[f], -ft[f], -ft[f]]
    np.add.at(rhs, i, -ft[f] * fg[f])
    np.add.at(rhs, j, ft[f] * fg[f])
    # Dirichlet faces: one-sided coupling to the prescribed pressure
    hd = np.flatnonzero(dirichlet[cf])
    rows.append(hc[hd])
    cols.append(hc[hd])
    vals.append(th[hd])
    np.add.at(rhs, hc[hd], ft[cf[hd]] * (bval[cf[hd]] - side[hd] * fg[cf[hd]]))
    # Neumann faces: prescribed flux out of the cell
    hn = np.flatnonzero(kind[cf] == 2)
    np.add.at(rhs, hc[hn], bval[cf[hn]])
    if src is not None and np.size(src.cell):
        np.add.at(rhs, np.asarray(src.cell, dtype=np.int64).ravel(), np.asarray(src.rate, float).ravel())
    # wells
    norm_g = float(np.linalg.norm(gvec))
    perf = []
    for k, w in enumerate(wells):
        wc = np.asarray(w.cells, dtype=np.int64).ravel()
        WI = np.asarray(w.WI, float).ravel()
        wi = WI * lam[wc]
        compi = np.atleast_1d(np.asarray(w.compi, float)).ravel()
        if _injector(w):
            m = min(rho.size, compi.size)
            rmix = float(rho[:m] @ compi[:m])
        else:
            frac = mob[wc] / lam[wc, None]
            rmix = float(np.sum(WI * (frac @ rho[: mob.shape[1]])) / np.sum(WI))
        dp = norm_g * np.asarray(w.dZ, float).ravel() * rmix
        target = float(np.ravel(w.val)[0])
        rows.append(wc)
        cols.append(wc)
        vals.append(wi)
        if str(w.type).lower() == "bhp":
            np.add.at(rhs, wc, wi * (target + dp))
            rows.append([nc + k])
            cols.append([nc + k])
            vals.append([wi.max()])
            rhs[nc + k] = wi.max() * target
        else:
            np.add.at(rhs, wc, wi * dp)
            rows += [wc, np.full(wc.size, nc + k), [nc + k]]
            cols += [np.full(wc.size, nc + k), wc, [nc + k]]
            vals += [-wi, -wi, [wi.sum()]]
            rhs[nc + k] = target - wi @ dp
        perf.append((wi, dp))
    A = sp.coo_array((np.concatenate([np.asarray(v, float) for v in vals]),
                      (np.concatenate([np.asarray(r) for r in rows]), np.concatenate([np.asarray(c) for c in cols]))),
                     shape=(n, n)).tocsr()
    A.sum_duplicates()
    A.sort_indices()
    if not dirichlet.any() and not any(str(w.type).lower() == "bhp" for w in wells):
        dg = A.diagonal()
        pin = 0 if dg[0] > 0 else int(np.argmax(dg))
        A = A.tolil()
        A[pin, pin] = 2 * A[pin, pin]
        A = A.tocsr()
    aux = dict(nbr=nbr, cf=cf, hc=hc, th=th, ft=ft, gp=gp, fg=fg, kind=kind, bval=bval, perf=perf,
               interior=interior)
    return A, rhs, aux


def reconstruct(G, p, aux, wells=()):
    """Face pressures, face fluxes and per-well perforation fluxes."""
    nc, nf = G.cells.num, G.faces.num
    nbr, cf, hc, th, ft = aux["nbr"], aux["cf"], aux["hc"], aux["th"], aux["ft"]
    gp, fg, kind, bval, interior = aux["gp"], aux["fg"], aux["kind"], aux["bval"], aux["interior"]
    fp = np.bincount(cf, (p[hc] + gp) * th, minlength=nf) / np.bincount(cf, th, minlength=nf)
    ext = ~interior
    neu = np.where(kind == 2, bval, 0.0)
    fp[ext] = fp[ext] + neu[ext] / ft[ext]
    fp[kind == 1] = bval[kind == 1]
    flux = np.zeros(nf)
    f = np.flatnonzero(interior)
    flux[f] = ft[f] * (p[nbr[f, 0]] - p[nbr[f, 1]] + fg[f])
    e = np.flatnonzero(ext)
    c = nbr[e].max(axis=1)
    outward = np.where(nbr[e, 1] < 0, 1.0, -1.0)
    gsum = np.bincount(cf, gp, minlength=nf)
    flux[e] = outward * ft[e] * (p[c] + gsum[e] - fp[e])
    wflux = [wi * (p[nc + k] + dp - p[np.asarray(w.cells, dtype=np.int64).ravel()])
             for k, (w, (wi, dp)) in enumerate(zip(wells, aux["perf"]))]
    return fp, flux, wflux


def incomp_tpfa(G, T, mob, rho, gvec=None, bc=None, src=None, wells=(), use_trans=False):
    """(p, bhp, face pressure, flux, well fluxes) by a direct solve."""
    A, rhs, aux = pressure_system(G, T, mob, rho, gvec, bc, src, wells, use_trans)
    p = spla.spsolve(A.tocsc(), rhs)
    fp, flux, wflux = reconstruct(G, p, aux, wells)
    return p[:G.cells.num], p[G.cells.num:], fp, flux, wflux
