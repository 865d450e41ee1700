"""Grid geometry on the GPU: a drop-in for the reference's `compute_geometry`
(pymrst/gridprocessing/compute_geometry.py:16-58) on 3-D grids, through
`pmb_compute_geometry3d` (csrc/geometry.cu): face areas, normals and
centroids, then cell volumes and centroids, from the grid's nodes and its
face/cell topology (`faces.nodePos`/`faces.nodes`, `cells.facePos`/
`cells.faces`, `faces.neighbors` with -1 outside).

Grids of dimension 1 and 2, neighbour reconstruction (`find_neighbors`, or
a grid without `faces.neighbors`) and the corner-point nominal geometry
(`cp_geometry`) are the reference's: they raise NotImplementedError here.
"""

from __future__ import annotations

import numpy as np

from . import _native as N


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("pymrst_b200.geometry needs a CUDA device")
    return torch


def hinge_array(nf: int, hinge_nodes) -> np.ndarray | None:
    """MRST's `hingenodes` (a mapping or object with `faces`, zero-based face
    indices, and `nodes`, one 3-D point per face) as an nf x 3 array of
    pivots, NaN for the faces that keep the mean of their nodes; None when
    there are none.  Invalid input raises ValueError, as the reference's
    validation does (compute_geometry.py:86-123)."""
    if hinge_nodes is None:
        return None
    try:
        faces = hinge_nodes["faces"] if isinstance(hinge_nodes, dict) else hinge_nodes.faces
        nodes = hinge_nodes["nodes"] if isinstance(hinge_nodes, dict) else hinge_nodes.nodes
    except (KeyError, AttributeError) as exc:
        raise ValueError("hinge_nodes must define faces and nodes") from exc
    faces = np.asarray(faces)
    if faces.ndim > 2 or (faces.ndim == 2 and 1 not in faces.shape):
        raise ValueError("hinge_nodes.faces must be a vector")
    faces = faces.reshape(-1)
    if faces.size and not np.issubdtype(faces.dtype, np.integer):
        if not (np.issubdtype(faces.dtype, np.number) and np.all(np.isfinite(faces))
                and np.all(faces == np.floor(faces))):
            raise ValueError("hinge_nodes.faces must contain integer indices")
    faces = faces.astype(np.int64)
    nodes = np.asarray(nodes, dtype=float)
    if faces.size == 0:
        return None
    if nodes.ndim == 1 and faces.size == 1:
        nodes = nodes.reshape(1, -1)
    if nodes.shape != (faces.size, 3):
        raise ValueError("hinge_nodes.nodes must have shape (number of faces, 3)")
    if np.any((faces < 0) | (faces >= nf)):
        raise ValueError("hinge_nodes.faces contains an out-of-range face index")
    if not np.all(np.isfinite(nodes)):
        raise ValueError("hinge_nodes.nodes must contain finite coordinates")
    out = np.full((nf, 3), np.nan)
    out[faces] = nodes  # a face listed twice takes its last point, as the reference's loop does
    return out


def geometry_arrays(coords, node_pos, nodes, face_pos, cell_faces, neighbors, hinge=None):
    """Face areas (nf), normals (nf x 3), centroids (nf x 3), cell volumes
    (nc) and centroids (nc x 3) of a 3-D grid given as plain arrays."""
    torch = _torch()
    coords = np.ascontiguousarray(coords, dtype=np.float64)
    if coords.ndim != 2 or coords.shape[1] != 3:
        raise ValueError("node coordinates must be n x 3")
    node_pos = np.asarray(node_pos, dtype=np.int64)
    face_pos = np.asarray(face_pos, dtype=np.int64)
    nf, nc = node_pos.size - 1, face_pos.size - 1
    nodes = np.asarray(nodes, dtype=np.int64)
    cell_faces = np.asarray(cell_faces, dtype=np.int64).reshape(-1)
    neighbors = np.asarray(neighbors, dtype=np.int64).reshape(nf, 2)
    if node_pos[-1] != nodes.size or face_pos[-1] != cell_faces.size:
        raise ValueError("inconsistent face-node or cell-face arrays")
    if np.any(np.diff(node_pos) < 3) and nf:
        raise ValueError("every face of a 3-D grid needs at least three nodes")
    if nodes.size and (nodes.min() < 0 or nodes.max() >= coords.shape[0]):
        raise ValueError("a face node index is out of range")
    if cell_faces.size and (cell_faces.min() < 0 or cell_faces.max() >= nf):
        raise ValueError("a cell face index is out of range")
    if np.any(np.diff(face_pos) < 1) and nc:
        raise ValueError("every cell needs at least one face")
    if max(nodes.size, cell_faces.size, 2 * nf) >= 2 ** 31:
        raise ValueError("the grid is too large for 32-bit indices")
    dev = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a, dtype=dt), device="cuda")
    d_coords = dev(coords, np.float64)
    d_npos, d_nodes = dev(node_pos, np.int32), dev(nodes, np.int32)
    d_fpos, d_cf = dev(face_pos, np.int32), dev(cell_faces, np.int32)
    d_nb = dev(neighbors, np.int32)
    d_hinge = dev(hinge, np.float64) if hinge is not None else None
    f64 = dict(dtype=torch.float64, device="cuda")
    areas, normals, fcent = torch.empty(max(nf, 1), **f64), torch.empty(max(nf, 1), 3, **f64), \
        torch.empty(max(nf, 1), 3, **f64)
    vols, ccent = torch.empty(max(nc, 1), **f64), torch.empty(max(nc, 1), 3, **f64)
    N.check(N.lib().pmb_compute_geometry3d(
        nf, nc, N.ptr(d_coords), N.ptr(d_npos), N.ptr(d_nodes), N.ptr(d_hinge), N.ptr(d_fpos), N.ptr(d_cf),
        N.ptr(d_nb), N.ptr(areas), N.ptr(normals), N.ptr(fcent), N.ptr(vols), N.ptr(ccent),
        torch.cuda.current_stream().cuda_stream))
    return (areas.cpu().numpy()[:nf], normals.cpu().numpy()[:nf], fcent.cpu().numpy()[:nf],
            vols.cpu().numpy()[:nc], ccent.cpu().numpy()[:nc])


def compute_geometry(g, *, cp_geometry: bool = False, find_neighbors: bool = False, hinge_nodes=None,
                     max_block_size=None, verbose: bool = False):
    """The reference's compute_geometry (same signature, the same fields set
    on `g`) for 3-D grids; returns `g`.  `max_block_size` and `verbose` are
    accepted and have no effect (the device pass needs no blocking)."""
    if getattr(g, "griddim", 3) != 3:
        raise NotImplementedError("device geometry is for 3-D grids; use the reference's for 1-D and 2-D")
    if find_neighbors or getattr(g.faces, "neighbors", None) is None:
        raise NotImplementedError("neighbour reconstruction is the reference's")
    if cp_geometry:
        raise NotImplementedError("corner-point nominal geometry is the reference's")
    nf = int(np.asarray(g.faces.nodePos).size - 1)
    hinge = hinge_array(nf, hinge_nodes)
    areas, normals, fcent, vols, ccent = geometry_arrays(g.nodes.coords, g.faces.nodePos, g.faces.nodes,
                                                         g.cells.facePos, g.cells.faces, g.faces.neighbors, hinge)
    g.faces.areas = areas
    g.faces.normals = normals
    g.faces.centroids = fcent
    g.cells.volumes = vols
    g.cells.centroids = ccent
    if hasattr(g, "type"):
        g.type = list(g.type) + ["computeGeometry"]
    return g
