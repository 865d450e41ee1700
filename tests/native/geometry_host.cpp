// Host build of the device geometry's per-face and per-cell code
// (pymrst_b200/csrc/geometry_core.cuh, the arithmetic geom_face_kernel and
// geom_cell_kernel run), so that tests check it against the reference's
// compute_geometry on the CPU.  Built by tests/test_geometry_cpu.py.
#include <cmath>

#include "geometry_core.cuh"

extern "C" void geom_host(int nf, int nc, const double* coords, const int* node_pos, const int* nodes,
                          const double* hinge, const int* face_pos, const int* cell_faces, const int* neighbors,
                          double* pivots, double* areas, double* normals, double* fcent, double* vols,
                          double* ccent) {
  using pmb::geom::V3;
  for (int f = 0; f < nf; ++f) {
    const double* h = (hinge && std::isfinite(hinge[3LL * f])) ? hinge + 3LL * f : nullptr;
    V3 p, N, C;
    double A = 0.0;
    pmb::geom::face(coords, nodes, node_pos[f], node_pos[f + 1], h, &p, &A, &N, &C);
    pivots[3LL * f] = p.x;
    pivots[3LL * f + 1] = p.y;
    pivots[3LL * f + 2] = p.z;
    areas[f] = A;
    normals[3LL * f] = N.x;
    normals[3LL * f + 1] = N.y;
    normals[3LL * f + 2] = N.z;
    fcent[3LL * f] = C.x;
    fcent[3LL * f + 1] = C.y;
    fcent[3LL * f + 2] = C.z;
  }
  for (int c = 0; c < nc; ++c) {
    double V = 0.0;
    V3 C;
    pmb::geom::cell(c, coords, node_pos, nodes, cell_faces, face_pos[c], face_pos[c + 1], neighbors, pivots, normals,
                    fcent, &V, &C);
    vols[c] = V;
    ccent[3LL * c] = C.x;
    ccent[3LL * c + 1] = C.y;
    ccent[3LL * c + 2] = C.z;
  }
}
