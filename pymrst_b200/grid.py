"""Host-side Cartesian grid with the reference's `Grid` field layout.

The TPFA path only reads topology and geometry from a grid: the cell count,
`cells.faces`/`cells.facePos` (half-faces), `faces.neighbors` (-1 outside),
cell and face centroids, face normals (area-weighted) and cell volumes.  The
reference builds these with `cart_grid` + `compute_geometry`
(pymrst/gridprocessing/tensor_grid.py:118-206,
pymrst/gridprocessing/compute_geometry.py:16).  This module writes the same
arrays in the same numbering for uniform Cartesian boxes, analytically, so a
GPU box without the reference can build the workloads.  Any object exposing
those attribute names (a reference `Grid` included) is accepted by the rest of
the package.

Numbering (reference `_tensor_grid_3d`): cells in Fortran order (i fastest),
faces as all x-faces, then y-faces, then z-faces, each block in Fortran order
over its (nx+1, ny, nz) / (nx, ny+1, nz) / (nx, ny, nz+1) index box; every
cell lists its faces as W, E, S, N, T, B.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Optional, Sequence, Tuple

import numpy as np


@dataclass
class Cells:
    num: int
    facePos: np.ndarray
    faces: np.ndarray
    indexMap: np.ndarray
    tags: Optional[np.ndarray] = None
    volumes: Optional[np.ndarray] = None
    centroids: Optional[np.ndarray] = None


@dataclass
class Faces:
    num: int
    neighbors: np.ndarray
    areas: Optional[np.ndarray] = None
    normals: Optional[np.ndarray] = None
    centroids: Optional[np.ndarray] = None
    tag: Optional[np.ndarray] = None


@dataclass
class Nodes:
    num: int
    coords: np.ndarray


@dataclass
class Grid:
    cells: Cells
    faces: Faces
    nodes: Nodes
    griddim: int
    cartDims: Optional[Tuple[int, ...]] = None
    type: Tuple[str, ...] = ("tensorGrid", "cartGrid")

    def cell_no(self) -> np.ndarray:
        return np.repeat(np.arange(self.cells.num, dtype=np.int64),
                         np.diff(self.cells.facePos))


def cartesian_grid(celldim: Sequence[int],
                   physdims: Optional[Sequence[float]] = None) -> Grid:
    """Uniform 3-D box of `celldim` cells spanning `physdims` metres
    (reference `cart_grid(celldim, physdims)` followed by
    `compute_geometry`)."""
    nx, ny, nz = (int(v) for v in celldim)
    if min(nx, ny, nz) < 1:
        raise ValueError("every grid dimension needs at least one cell")
    if physdims is None:
        physdims = (float(nx), float(ny), float(nz))
    Lx, Ly, Lz = (float(v) for v in physdims)
    dx, dy, dz = Lx / nx, Ly / ny, Lz / nz
    xs = np.linspace(0.0, Lx, nx + 1)
    ys = np.linspace(0.0, Ly, ny + 1)
    zs = np.linspace(0.0, Lz, nz + 1)
    nc = nx * ny * nz
    nfx, nfy, nfz = (nx + 1) * ny * nz, nx * (ny + 1) * nz, nx * ny * (nz + 1)
    nf = nfx + nfy + nfz

    def F(a):
        return np.asarray(a).ravel(order="F")

    ci = np.arange(nc, dtype=np.int64).reshape((nx, ny, nz), order="F")
    pad = -np.ones((nx + 2, ny + 2, nz + 2), dtype=np.int64)
    pad[1:-1, 1:-1, 1:-1] = ci
    neighbors = np.vstack([
        np.column_stack([F(pad[:nx + 1, 1:ny + 1, 1:nz + 1]), F(pad[1:, 1:ny + 1, 1:nz + 1])]),
        np.column_stack([F(pad[1:nx + 1, :ny + 1, 1:nz + 1]), F(pad[1:nx + 1, 1:, 1:nz + 1])]),
        np.column_stack([F(pad[1:nx + 1, 1:ny + 1, :nz + 1]), F(pad[1:nx + 1, 1:ny + 1, 1:])]),
    ])

    fx = np.arange(nfx, dtype=np.int64).reshape((nx + 1, ny, nz), order="F")
    fy = nfx + np.arange(nfy, dtype=np.int64).reshape((nx, ny + 1, nz), order="F")
    fz = nfx + nfy + np.arange(nfz, dtype=np.int64).reshape((nx, ny, nz + 1), order="F")
    cell_faces = np.column_stack([
        F(fx[:nx]), F(fx[1:]), F(fy[:, :ny]), F(fy[:, 1:]),
        F(fz[:, :, :nz]), F(fz[:, :, 1:]),
    ]).ravel()

    xc = 0.5 * (xs[:-1] + xs[1:])
    yc = 0.5 * (ys[:-1] + ys[1:])
    zc = 0.5 * (zs[:-1] + zs[1:])
    CX, CY, CZ = np.meshgrid(xc, yc, zc, indexing="ij")
    cell_centroids = np.column_stack([F(CX), F(CY), F(CZ)])
    volumes = np.full(nc, dx * dy * dz)

    # Face centroids and area-weighted normals pointing from neighbors[:,0]
    # to neighbors[:,1] (+x, +y, +z).
    X, Y, Z = np.meshgrid(xs, yc, zc, indexing="ij")
    cx = np.column_stack([F(X), F(Y), F(Z)])
    X, Y, Z = np.meshgrid(xc, ys, zc, indexing="ij")
    cy = np.column_stack([F(X), F(Y), F(Z)])
    X, Y, Z = np.meshgrid(xc, yc, zs, indexing="ij")
    cz = np.column_stack([F(X), F(Y), F(Z)])
    face_centroids = np.vstack([cx, cy, cz])
    ax, ay, az = dy * dz, dx * dz, dx * dy
    normals = np.zeros((nf, 3))
    normals[:nfx, 0] = ax
    normals[nfx:nfx + nfy, 1] = ay
    normals[nfx + nfy:, 2] = az
    areas = np.concatenate([np.full(nfx, ax), np.full(nfy, ay), np.full(nfz, az)])

    NX, NY, NZ = np.meshgrid(xs, ys, zs, indexing="ij")
    coords = np.column_stack([F(NX), F(NY), F(NZ)])

    return Grid(
        cells=Cells(num=nc, facePos=6 * np.arange(nc + 1, dtype=np.int64),
                    faces=cell_faces, indexMap=np.arange(nc, dtype=np.int64),
                    tags=np.tile(np.arange(6, dtype=np.int64), nc),
                    volumes=volumes, centroids=cell_centroids),
        faces=Faces(num=nf, neighbors=neighbors, areas=areas, normals=normals,
                    centroids=face_centroids, tag=np.zeros(nf, dtype=np.int64)),
        nodes=Nodes(num=coords.shape[0], coords=coords),
        griddim=3,
        cartDims=(nx, ny, nz),
    )


def cell_index(grid: Grid, i, j, k) -> np.ndarray:
    """Linear (Fortran-order) cell index of Cartesian subscripts."""
    nx, ny, _ = grid.cartDims
    return np.asarray(i) + nx * (np.asarray(j) + ny * np.asarray(k))


def internal_neighbors(grid) -> Tuple[np.ndarray, np.ndarray]:
    """Internal interface cell pairs and the mask selecting them from all
    faces (reference `setup_operators_tpfa._grid_based_trans`,
    pymrst/modules/ad_core/utils/setup_operators_tpfa.py:99-110)."""
    N = np.asarray(grid.faces.neighbors, dtype=np.int64)
    mask = np.all(N >= 0, axis=1)
    return N[mask], mask
