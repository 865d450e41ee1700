"""Oracle: one-sided and face transmissibilities (test infrastructure only).

Restates pymrst/solvers/compute_trans.py:11-53 and
pymrst/solvers/get_face_transmissibility.py:12-31.
"""

import numpy as np


def _perm_tensor(perm: np.ndarray) -> np.ndarray:
    """Row-wise full 3x3 tensor entries (pymrst/params/rock/perm_tensor.py:31-66)."""
    perm = np.asarray(perm, dtype=float)
    if perm.ndim == 1:
        perm = perm[:, None]
    nc, nk = perm.shape
    if nk == 1:
        sym = perm * np.array([1.0, 0.0, 0.0, 1.0, 0.0, 1.0])
    elif nk == 3:
        z = np.zeros(nc)
        sym = np.column_stack([perm[:, 0], z, z, perm[:, 1], z, perm[:, 2]])
    elif nk == 6:
        sym = perm
    else:
        raise ValueError("unsupported permeability layout")
    return sym[:, [0, 1, 2, 1, 3, 4, 2, 4, 5]]


def compute_trans(g, rock, fix_negative=True) -> np.ndarray:
    """Half-face T = (c . K n) / (c . c) per half-face (compute_trans.py:11-29)."""
    fp = np.asarray(g.cells.facePos)
    cell_no = np.repeat(np.arange(g.cells.num), np.diff(fp))
    cf = np.asarray(g.cells.faces, dtype=np.int64)
    c = np.asarray(g.faces.centroids)[cf] - np.asarray(g.cells.centroids)[cell_no]
    sgn = np.where(np.asarray(g.faces.neighbors)[cf, 0] == cell_no, 1.0, -1.0)
    nrm = sgn[:, None] * np.asarray(g.faces.normals)[cf]
    K = _perm_tensor(rock.perm)
    rows = np.array([0, 0, 0, 1, 1, 1, 2, 2, 2])
    cols = np.array([0, 1, 2, 0, 1, 2, 0, 1, 2])
    t = np.zeros(cf.size)
    for idx in range(9):
        t += c[:, rows[idx]] * K[cell_no, idx] * nrm[:, cols[idx]]
    t /= np.sum(c * c, axis=1)
    if fix_negative and np.any(t < 0):
        t = np.abs(t)
    ntg = getattr(rock, "ntg", None)
    tags = getattr(g.cells, "tags", None)
    if ntg is not None and tags is not None:
        mult = np.asarray(ntg)[cell_no].copy()
        mult[np.asarray(tags) // 2 == 2] = 1.0
        t = mult * t
    return t


def face_trans(g, t_half: np.ndarray) -> np.ndarray:
    """Harmonic reduction 1 / sum(1 / T_hf) per face
    (get_face_transmissibility.py:22-31)."""
    with np.errstate(divide="ignore"):
        return 1.0 / np.bincount(np.asarray(g.cells.faces), weights=1.0 / t_half,
                                 minlength=g.faces.num)
