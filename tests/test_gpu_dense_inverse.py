"""The AMG coarsest-level solver, `pmb_dense_inverse` (in-place Gauss-Jordan
with row pivoting in one CTA, or on a cluster of CTAs when the working
matrix outgrows one CTA's shared memory), against numpy: sizes whose working
matrix fits in shared memory, sizes that take a cluster, sizes that spill
rows to global memory, matrices that need pivoting, and a singular matrix,
which is an error, not a fault."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from pymrst_b200 import _native as N  # noqa: E402
from pymrst_b200.build import build  # noqa: E402

build()


def _inverse(a):
    d_a = torch.as_tensor(np.ascontiguousarray(a), device="cuda")
    d_inv = torch.empty_like(d_a)
    rc = N.lib().pmb_dense_inverse(a.shape[0], N.ptr(d_a), N.ptr(d_inv), torch.cuda.current_stream().cuda_stream)
    return rc, d_inv.cpu().numpy()


@pytest.mark.parametrize("n", [1, 2, 7, 64, 190, 300, 700])
@pytest.mark.parametrize("kind", ["general", "zero_diagonal", "pressure_like"])
def test_dense_inverse_matches_numpy(n, kind):
    rng = np.random.default_rng(n)
    if kind == "pressure_like":
        # a weakly diagonally dominant M-matrix (a Galerkin pressure operator)
        off = -rng.uniform(0.0, 1.0, (n, n)) * (rng.uniform(size=(n, n)) < 0.05)
        np.fill_diagonal(off, 0.0)
        a = off + np.diag(-off.sum(axis=1) + 1e-3)
    else:
        a = rng.standard_normal((n, n))
        if kind == "zero_diagonal" and n > 1:
            np.fill_diagonal(a, 0.0)
    rc, inv = _inverse(a)
    assert rc == N.PMB_OK
    ref = np.linalg.inv(a)
    assert np.abs(inv - ref).max() <= 1e-9 * np.abs(ref).max()


def test_singular_matrix_is_an_error_not_a_fault():
    a = np.ones((5, 5))
    rc, _ = _inverse(a)
    assert rc == 4  # PMB_ERR_PIVOT
    # the library stays usable
    rc, inv = _inverse(np.eye(3) * 2.0)
    assert rc == N.PMB_OK and np.allclose(inv, np.eye(3) * 0.5)


@pytest.mark.parametrize("n", [190, 300])
def test_cluster_inverse_is_bitwise_the_one_cta_inverse(n, monkeypatch):
    """Matrices too large for one CTA's shared memory are inverted on a
    cluster (rows split over the CTAs' distributed shared memory); the
    result equals the one-CTA kernel's (rows spilled to global memory) bit
    for bit."""
    rng = np.random.default_rng(100 + n)
    a = rng.standard_normal((n, n))
    rc, inv_cluster = _inverse(a)
    assert rc == N.PMB_OK
    monkeypatch.setenv("PMB_GJ_CLUSTER", "0")
    rc, inv_one = _inverse(a)
    assert rc == N.PMB_OK
    assert np.array_equal(inv_cluster, inv_one)
