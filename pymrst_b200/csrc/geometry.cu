// Grid geometry on the device: compute_geometry for 3-D grids
// (pymrst/gridprocessing/compute_geometry.py:211-325), one thread per face,
// then one thread per cell.  The arithmetic lives in geometry_core.cuh.
#include "geometry_core.cuh"
#include "pmb_common.cuh"

namespace pmb {

// Face f: pivot (kept for the cell pass), area, normal, centroid.  A face
// whose hinge row holds a finite x takes that point as its pivot.
__global__ void geom_face_kernel(int nf, const double* __restrict__ coords, const int* __restrict__ node_pos,
                                 const int* __restrict__ nodes, const double* __restrict__ hinge,
                                 double* __restrict__ pivots, double* __restrict__ areas,
                                 double* __restrict__ normals, double* __restrict__ centroids) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nf) return;
  const double* h = (hinge && isfinite(hinge[3LL * f])) ? hinge + 3LL * f : nullptr;
  geom::V3 p, N, C;
  double A = 0.0;
  geom::face(coords, nodes, node_pos[f], node_pos[f + 1], h, &p, &A, &N, &C);
  pivots[3LL * f] = p.x;
  pivots[3LL * f + 1] = p.y;
  pivots[3LL * f + 2] = p.z;
  areas[f] = A;
  normals[3LL * f] = N.x;
  normals[3LL * f + 1] = N.y;
  normals[3LL * f + 2] = N.z;
  centroids[3LL * f] = C.x;
  centroids[3LL * f + 1] = C.y;
  centroids[3LL * f + 2] = C.z;
}

__global__ void geom_cell_kernel(int nc, const double* __restrict__ coords, const int* __restrict__ node_pos,
                                 const int* __restrict__ nodes, const int* __restrict__ face_pos,
                                 const int* __restrict__ cell_faces, const int* __restrict__ neighbors,
                                 const double* __restrict__ pivots, const double* __restrict__ normals,
                                 const double* __restrict__ fcentroids, double* __restrict__ volumes,
                                 double* __restrict__ centroids) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  double V = 0.0;
  geom::V3 C;
  geom::cell(c, coords, node_pos, nodes, cell_faces, face_pos[c], face_pos[c + 1], neighbors, pivots, normals,
             fcentroids, &V, &C);
  volumes[c] = V;
  centroids[3LL * c] = C.x;
  centroids[3LL * c + 1] = C.y;
  centroids[3LL * c + 2] = C.z;
}

void compute_geometry3d(int nf, int nc, const double* coords, const int* node_pos, const int* nodes,
                        const double* hinge, const int* face_pos, const int* cell_faces, const int* neighbors,
                        double* areas, double* normals, double* fcentroids, double* volumes, double* ccentroids,
                        cudaStream_t s) {
  DArray<double> pivots;
  pivots.resize(3LL * std::max(nf, 1));
  if (nf > 0) {
    geom_face_kernel<<<grid_for(nf, 128), 128, 0, s>>>(nf, coords, node_pos, nodes, hinge, pivots.get(), areas,
                                                       normals, fcentroids);
    PMB_CHECK_LAUNCH();
  }
  if (nc > 0) {
    geom_cell_kernel<<<grid_for(nc, 128), 128, 0, s>>>(nc, coords, node_pos, nodes, face_pos, cell_faces, neighbors,
                                                       pivots.get(), normals, fcentroids, volumes, ccentroids);
    PMB_CHECK_LAUNCH();
  }
  PMB_CUDA(cudaStreamSynchronize(s));  // the pivots are freed on return
}

}  // namespace pmb

extern "C" int pmb_compute_geometry3d(int32_t nf, int32_t nc, const double* d_coords, const int32_t* d_node_pos,
                                      const int32_t* d_nodes, const double* d_hinge, const int32_t* d_face_pos,
                                      const int32_t* d_cell_faces, const int32_t* d_neighbors, double* d_face_areas,
                                      double* d_face_normals, double* d_face_centroids, double* d_cell_volumes,
                                      double* d_cell_centroids, void* stream) {
  return pmb::guarded([&] {
    PMB_REQUIRE(nf >= 0 && nc >= 0, "negative face or cell count");
    if (nf == 0 && nc == 0) return;
    PMB_REQUIRE(d_coords && d_node_pos && d_nodes && d_face_areas && d_face_normals && d_face_centroids,
                "NULL argument");
    PMB_REQUIRE(nc == 0 || (d_face_pos && d_cell_faces && d_neighbors && d_cell_volumes && d_cell_centroids),
                "NULL argument");
    pmb::compute_geometry3d(nf, nc, d_coords, d_node_pos, d_nodes, d_hinge, d_face_pos, d_cell_faces, d_neighbors,
                            d_face_areas, d_face_normals, d_face_centroids, d_cell_volumes, d_cell_centroids,
                            (cudaStream_t)stream);
  });
}
