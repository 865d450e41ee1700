"""Host-side checks of the C-ABI library (no GPU needed)."""

import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest
import scipy.sparse as sp

from pymrst_b200 import _native as N
from pymrst_b200.build import build

HEADER = Path(__file__).resolve().parents[1] / "include" / "pymrst_b200.h"


@pytest.fixture(scope="module")
def lib():
    build()
    return N.lib()


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"\b(pmb_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(lib):
    names = declared_symbols()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
    # and the ctypes table covers all of them
    assert set(names) <= set(N.SIGNATURES)


def test_default_options_match_reference_cpr_defaults(lib):
    o = N.CPROpts()
    N.check(lib.pmb_cpr_default_opts(C.byref(o)))
    # CPRSolver(rtol=1e-8, maxiter=200, restart=50, amg_rebuild_interval=8)
    assert (o.rtol, o.maxiter, o.restart, o.amg_rebuild_interval) == (1e-8, 200, 50, 8)


def poisson3d(nx, ny, nz, aniso=(1.0, 1.0, 1.0)):
    def lap(n, a):
        return sp.diags([-a * np.ones(n - 1), 2 * a * np.ones(n), -a * np.ones(n - 1)], [-1, 0, 1])
    I = lambda n: sp.eye(n)
    A = (sp.kron(I(nz), sp.kron(I(ny), lap(nx, aniso[0]))) + sp.kron(I(nz), sp.kron(lap(ny, aniso[1]), I(nx)))
         + sp.kron(lap(nz, aniso[2]), sp.kron(I(ny), I(nx))))
    A = sp.csr_array(A + 1e-3 * sp.eye(nx * ny * nz))
    A.sort_indices()
    return A


@pytest.mark.parametrize("aniso", [(1.0, 1.0, 1.0), (1.0, 4.0, 100.0)])
def test_amg_host_aggregation_coarsens_to_the_dense_size(lib, aniso):
    A = poisson3d(20, 18, 10, aniso)
    n = A.shape[0]
    rp = A.indptr.astype(np.int32)
    ci = A.indices.astype(np.int32)
    v = A.data.astype(np.float64)
    sizes = (C.c_int64 * 64)()
    nl = C.c_int32()
    N.check(lib.pmb_amg_hierarchy_host(n, N.as_p(rp, C.c_int32), N.as_p(ci, C.c_int32), N.as_p(v, C.c_double),
                                       0.25, 200, 64, sizes, C.byref(nl)))
    s = [sizes[i] for i in range(nl.value)]
    assert s[0] == n and s[-1] <= 200
    # every level shrinks by at least 2x (two pairwise passes)
    assert all(b <= a / 2 for a, b in zip(s[:-1], s[1:]))


def test_invalid_arguments_report_an_error_not_a_crash(lib):
    rc = lib.pmb_ow_sizes(None, None)
    assert rc == 2
    assert "NULL" in lib.pmb_last_error().decode()
