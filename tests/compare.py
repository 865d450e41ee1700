"""Comparison helpers shared by the parity tests."""

import numpy as np
import scipy.sparse as sp


def ow_splits(nc, nw):
    """Variable-block boundaries of the reference layout:
    [water|p, oil|sW, eq_w|qWs, eq_o|qOs, ctrl|bhp]."""
    return np.array([0, nc, 2 * nc, 2 * nc + nw, 2 * nc + 2 * nw, 2 * nc + 3 * nw])


def blockwise_error(A, B, splits):
    """Largest blockwise relative difference between sparse matrices A and B:
    for every (row-block, column-block) pair, max|A - B| over that block
    divided by max|B| over it (blocks where B is all zero compare against
    max|B| of the whole matrix, so structural zeros must stay zero)."""
    A = sp.csr_array(A)
    B = sp.csr_array(B)
    D = (A - B).tocsr()
    Bmax = np.abs(B.data).max() if B.nnz else 1.0
    worst = 0.0
    for i in range(len(splits) - 1):
        for j in range(len(splits) - 1):
            sl = (slice(splits[i], splits[i + 1]), slice(splits[j], splits[j + 1]))
            d = D[sl]
            if d.nnz == 0:
                continue
            dmax = np.abs(d.data).max()
            b = B[sl]
            scale = np.abs(b.data).max() if b.nnz and np.abs(b.data).max() > 0 else Bmax
            worst = max(worst, dmax / scale)
    return worst


def segment_error(a, b, splits):
    """Largest segment-relative difference between vectors: per segment,
    max|a - b| / max(max|b|, tiny)."""
    worst = 0.0
    for i in range(len(splits) - 1):
        x = np.asarray(a[splits[i]:splits[i + 1]], float)
        y = np.asarray(b[splits[i]:splits[i + 1]], float)
        if x.size == 0:
            continue
        scale = max(np.abs(y).max(), 1e-300)
        worst = max(worst, np.abs(x - y).max() / scale)
    return worst
