"""The device geometry's per-face and per-cell arithmetic
(pymrst_b200/csrc/geometry_core.cuh), built for the host from the same
source, against the reference's compute_geometry
(pymrst/gridprocessing/compute_geometry.py:211-325) on 3-D grids: a
Cartesian grid, a tensor grid, a grid with perturbed (non-planar) faces, and
the same with hinge points on some faces (bitwise equal); and the drop-in's
hinge-point checks.

The reference package comes from its install under baseline/_ref; the
module is skipped where that install, or g++, is absent."""

import ctypes as C
import shutil
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
REF = ROOT / "baseline" / "_ref"
if not (REF / "pymrst").is_dir():
    pytest.skip("the reference package is not installed under baseline/_ref", allow_module_level=True)
if shutil.which("g++") is None:
    pytest.skip("no g++", allow_module_level=True)
sys.path.insert(0, str(REF))

from pymrst.gridprocessing import cart_grid, compute_geometry  # noqa: E402
from pymrst.gridprocessing.tensor_grid import tensor_grid  # noqa: E402

from pymrst_b200.geometry import hinge_array  # noqa: E402


@pytest.fixture(scope="module")
def host_lib(tmp_path_factory):
    out = tmp_path_factory.mktemp("geom") / "libgeom_host.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I", str(ROOT / "pymrst_b200" / "csrc"),
                    str(ROOT / "tests" / "native" / "geometry_host.cpp"), "-o", str(out)], check=True)
    return C.CDLL(str(out))


def _host_geometry(lib, g, hinge=None):
    i32 = lambda a: np.ascontiguousarray(np.asarray(a).reshape(-1), dtype=np.int32)
    coords = np.ascontiguousarray(g.nodes.coords, dtype=np.float64)
    npos, nodes = i32(g.faces.nodePos), i32(g.faces.nodes)
    fpos, cf, nb = i32(g.cells.facePos), i32(g.cells.faces), i32(g.faces.neighbors)
    nf, nc = npos.size - 1, fpos.size - 1
    piv, areas, normals, fc = np.empty((nf, 3)), np.empty(nf), np.empty((nf, 3)), np.empty((nf, 3))
    vols, cc = np.empty(nc), np.empty((nc, 3))
    p = lambda a: a.ctypes.data_as(C.c_void_p) if a is not None else None
    h = np.ascontiguousarray(hinge, dtype=np.float64) if hinge is not None else None
    lib.geom_host(C.c_int(nf), C.c_int(nc), p(coords), p(npos), p(nodes), p(h), p(fpos), p(cf), p(nb), p(piv),
                  p(areas), p(normals), p(fc), p(vols), p(cc))
    return areas, normals, fc, vols, cc


def _perturbed(seed):
    g = cart_grid([5, 4, 3], [50.0, 40.0, 6.0])
    rng = np.random.default_rng(seed)
    g.nodes.coords = g.nodes.coords + rng.uniform(-0.15, 0.15, g.nodes.coords.shape) * np.array([10.0, 10.0, 2.0])
    return g


def _compare(lib, g, hinge_nodes=None):
    nf = g.faces.num
    got = _host_geometry(lib, g, hinge_array(nf, hinge_nodes))
    ref = compute_geometry(g, hinge_nodes=hinge_nodes)
    want = (ref.faces.areas, ref.faces.normals, ref.faces.centroids, ref.cells.volumes, ref.cells.centroids)
    # the same operations in the same order as the reference's numpy code:
    # bitwise equal on the host build (the device build may contract a
    # multiply-add and differ in the last bits)
    for a, b in zip(got, want):
        assert np.array_equal(a, np.asarray(b, dtype=float).reshape(a.shape))


def test_cartesian_and_tensor_grids(host_lib):
    _compare(host_lib, cart_grid([4, 3, 2], [40.0, 30.0, 4.0]))
    _compare(host_lib, tensor_grid(np.array([0.0, 1.0, 3.0, 7.0]), np.array([0.0, 2.0, 2.5]),
                                   np.array([-1.0, 0.0, 0.5, 4.0])))


@pytest.mark.parametrize("seed", [0, 1])
def test_perturbed_nonplanar_faces(host_lib, seed):
    _compare(host_lib, _perturbed(seed))


def test_hinge_points(host_lib):
    g = _perturbed(2)
    faces = np.array([0, 7, 31, 50])
    nodes = np.array([g.nodes.coords[g.faces.nodes[g.faces.nodePos[f]:g.faces.nodePos[f + 1]]].mean(axis=0)
                      for f in faces]) + np.array([0.3, -0.2, 0.1])
    _compare(host_lib, g, {"faces": faces, "nodes": nodes})


def test_hinge_input_is_checked():
    with pytest.raises(ValueError):
        hinge_array(10, {"faces": [11], "nodes": [[0.0, 0.0, 0.0]]})
    with pytest.raises(ValueError):
        hinge_array(10, {"faces": [1, 2], "nodes": [[0.0, 0.0, 0.0]]})
    with pytest.raises(ValueError):
        hinge_array(10, {"faces": [1.5], "nodes": [[0.0, 0.0, 0.0]]})
    with pytest.raises(ValueError):
        hinge_array(10, {"faces": [1], "nodes": [[0.0, np.nan, 0.0]]})
    with pytest.raises(ValueError):
        hinge_array(10, object())
    h = hinge_array(4, {"faces": [2], "nodes": [1.0, 2.0, 3.0]})
    assert np.isnan(h[[0, 1, 3]]).all() and np.array_equal(h[2], [1.0, 2.0, 3.0])
    assert hinge_array(4, None) is None
