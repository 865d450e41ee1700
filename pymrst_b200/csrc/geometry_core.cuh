// Polyhedral grid geometry, one face or one cell at a time: the arithmetic
// of the device kernels in geometry.cu, written so that it also compiles as
// plain C++ (a host build checks it against the reference's compute_geometry
// on the CPU).
//
// Follows compute_geometry.py:211-325 (MRST's computeGeometry for 3-D
// grids).  A face is split into the triangles (n_k, n_{k+1}, p) of a fan
// around its pivot p (the mean of its nodes, or a given hinge point); a
// triangle's area vector is t_k = (n_{k+1} - n_k) x (p - n_k) / 2.  The face
// normal is the sum of the t_k, its area the sum of their lengths, its
// centroid their length-weighted centroid.  A cell is split into the
// tetrahedra joining its centre c (the mean of its face centroids) to every
// face triangle, oriented outwards: each triangle's sign is that of t_k . N
// (N the face normal), times +1 where the cell is the face's first neighbour
// and -1 where it is the second.  Sums run in node and face order.
#pragma once

#include <cmath>

#ifdef __CUDACC__
#define PMB_GEOM_FN __host__ __device__ inline
#else
#define PMB_GEOM_FN inline
#endif

namespace pmb {
namespace geom {

struct V3 {
  double x, y, z;
};

PMB_GEOM_FN V3 at(const double* c, long long i) { return V3{c[3 * i], c[3 * i + 1], c[3 * i + 2]}; }
PMB_GEOM_FN V3 sub(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
PMB_GEOM_FN double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// The fan triangle between nodes a, b and the pivot p: its area vector and
// its centroid.
PMB_GEOM_FN void triangle(V3 a, V3 b, V3 p, V3* t, V3* centroid) {
  const V3 u = sub(b, a), w = sub(p, a);
  *t = V3{(u.y * w.z - u.z * w.y) / 2.0, (u.z * w.x - u.x * w.z) / 2.0, (u.x * w.y - u.y * w.x) / 2.0};
  *centroid = V3{(a.x + b.x + p.x) / 3.0, (a.y + b.y + p.y) / 3.0, (a.z + b.z + p.z) / 3.0};
}

PMB_GEOM_FN double norm(V3 t) { return std::sqrt(t.x * t.x + t.y * t.y + t.z * t.z); }

PMB_GEOM_FN double sign(double v) { return v > 0.0 ? 1.0 : (v < 0.0 ? -1.0 : 0.0); }

// Face f with nodes nodes[p0 .. p1): pivot (the mean of the nodes unless
// hinge is given), area, normal and centroid (the pivot where the area is
// not positive).
PMB_GEOM_FN void face(const double* coords, const int* nodes, int p0, int p1, const double* hinge, V3* pivot,
                      double* area, V3* normal, V3* centroid) {
  V3 p{0.0, 0.0, 0.0};
  if (hinge) {
    p = V3{hinge[0], hinge[1], hinge[2]};
  } else {
    for (int k = p0; k < p1; ++k) {
      const V3 n = at(coords, nodes[k]);
      p.x += n.x;
      p.y += n.y;
      p.z += n.z;
    }
    const double m = (double)(p1 - p0);
    p = V3{p.x / m, p.y / m, p.z / m};
  }
  double A = 0.0;
  V3 N{0.0, 0.0, 0.0}, C{0.0, 0.0, 0.0};
  for (int k = p0; k < p1; ++k) {
    const int kn = k + 1 < p1 ? k + 1 : p0;
    V3 t, c;
    triangle(at(coords, nodes[k]), at(coords, nodes[kn]), p, &t, &c);
    const double a = norm(t);
    N.x += t.x;
    N.y += t.y;
    N.z += t.z;
    A += a;
    C.x += a * c.x;
    C.y += a * c.y;
    C.z += a * c.z;
  }
  *pivot = p;
  *area = A;
  *normal = N;
  *centroid = A > 0.0 ? V3{C.x / A, C.y / A, C.z / A} : p;
}

// Cell `cell` with half-faces cell_faces[q0 .. q1): volume and centroid from
// the faces' pivots, normals and centroids of face().
PMB_GEOM_FN void cell(int cell_index, const double* coords, const int* node_pos, const int* nodes, const int* cell_faces,
                      int q0, int q1, const int* neighbors, const double* pivots, const double* normals,
                      const double* fcentroids, double* volume, V3* centroid) {
  V3 c{0.0, 0.0, 0.0};
  for (int q = q0; q < q1; ++q) {
    const V3 fc = at(fcentroids, cell_faces[q]);
    c.x += fc.x;
    c.y += fc.y;
    c.z += fc.z;
  }
  const double m = (double)(q1 - q0);
  c = V3{c.x / m, c.y / m, c.z / m};
  double V = 0.0;
  V3 R{0.0, 0.0, 0.0};
  for (int q = q0; q < q1; ++q) {
    const int f = cell_faces[q];
    const double side = neighbors[2LL * f] == cell_index ? 1.0 : -1.0;
    const V3 p = at(pivots, f), N = at(normals, f);
    const int p0 = node_pos[f], p1 = node_pos[f + 1];
    for (int k = p0; k < p1; ++k) {
      const int kn = k + 1 < p1 ? k + 1 : p0;
      V3 t, tc;
      triangle(at(coords, nodes[k]), at(coords, nodes[kn]), p, &t, &tc);
      const double s = sign(dot(t, N)) * side;
      const V3 out{t.x * s, t.y * s, t.z * s};
      const V3 rel = sub(tc, c);
      const double tv = dot(rel, out) / 3.0;
      V += tv;
      R.x += tv * (0.75 * rel.x);
      R.y += tv * (0.75 * rel.y);
      R.z += tv * (0.75 * rel.z);
    }
  }
  *volume = V;
  *centroid = V3{R.x / V + c.x, R.y / V + c.y, R.z / V + c.z};
}

}  // namespace geom
}  // namespace pmb
