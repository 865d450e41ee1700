"""Device compute_geometry (pmb_compute_geometry3d, pymrst_b200.geometry)
against the reference's own output on a 3-D grid with perturbed
(non-planar) faces, without and with hinge points (tests/golden/
geometry3d.npz, made by the reference's compute_geometry,
compute_geometry.py:211-325): face areas, normals and centroids, cell
volumes and centroids to 1e-12 of each field's largest entry (the host
build of the same arithmetic is bitwise the reference's; the device may
contract a multiply-add).  Also the drop-in on a grid object, and its
refusals."""

from types import SimpleNamespace

import numpy as np
import pytest

from fixtures import load

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from pymrst_b200.build import build  # noqa: E402
from pymrst_b200.geometry import compute_geometry, geometry_arrays, hinge_array  # noqa: E402

build()

FIELDS = ("face_areas", "face_normals", "face_centroids", "cell_volumes", "cell_centroids")


def _check(got, d, tag):
    for name, a in zip(FIELDS, got):
        want = np.asarray(d[f"{tag}_{name}"], dtype=float).reshape(a.shape)
        assert np.abs(a - want).max() <= 1e-12 * max(np.abs(want).max(), 1.0), name


@pytest.mark.parametrize("tag", ["plain", "hinge"])
def test_device_geometry_matches_the_reference(tag):
    d = load("geometry3d.npz")
    nf = d["node_pos"].size - 1
    hinge = hinge_array(nf, {"faces": d["hinge_faces"], "nodes": d["hinge_nodes"]}) if tag == "hinge" else None
    got = geometry_arrays(d["coords"], d["node_pos"], d["nodes"], d["face_pos"], d["cell_faces"], d["neighbors"],
                          hinge)
    _check(got, d, tag)


def test_drop_in_sets_the_grid_fields():
    d = load("geometry3d.npz")
    g = SimpleNamespace(griddim=3, type=["tensorGrid"],
                        nodes=SimpleNamespace(coords=d["coords"]),
                        faces=SimpleNamespace(nodePos=d["node_pos"], nodes=d["nodes"], neighbors=d["neighbors"]),
                        cells=SimpleNamespace(facePos=d["face_pos"], faces=d["cell_faces"]))
    assert compute_geometry(g) is g
    _check((g.faces.areas, g.faces.normals, g.faces.centroids, g.cells.volumes, g.cells.centroids), d, "plain")
    assert g.type[-1] == "computeGeometry"
    with pytest.raises(NotImplementedError):
        compute_geometry(g, cp_geometry=True)
    g.griddim = 2
    with pytest.raises(NotImplementedError):
        compute_geometry(g)
