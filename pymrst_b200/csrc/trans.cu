// One-sided and face transmissibilities (compute_trans,
// pymrst/solvers/compute_trans.py:11-53; get_face_transmissibility,
// pymrst/solvers/get_face_transmissibility.py:12-31).
#include "pmb_common.cuh"

namespace pmb {

// T_hf = sum_{r,c} cvec_r K_rc n_c / |cvec|^2 over the full 3x3 tensor,
// summed in the reference's row-major order, n oriented out of the cell.
__global__ void __launch_bounds__(256) half_trans_kernel(long long nh, const int* __restrict__ cell_no,
                                                         const int* __restrict__ hface,
                                                         const int* __restrict__ first_cell,
                                                         const double* __restrict__ cc,
                                                         const double* __restrict__ fc,
                                                         const double* __restrict__ fn,
                                                         const double* __restrict__ K9,
                                                         const double* __restrict__ ntg,
                                                         const int* __restrict__ tag, int fix_negative,
                                                         double* __restrict__ out) {
  const long long h = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (h >= nh) return;
  const int c = cell_no[h], f = hface[h];
  const double sg = first_cell[f] == c ? 1.0 : -1.0;
  double cv[3], nv[3];
  for (int d = 0; d < 3; ++d) {
    cv[d] = fc[3LL * f + d] - cc[3LL * c + d];
    nv[d] = sg * fn[3LL * f + d];
  }
  double t = 0.0;
  for (int r = 0; r < 3; ++r)
    for (int q = 0; q < 3; ++q) t += cv[r] * K9[9LL * c + 3 * r + q] * nv[q];
  t /= (cv[0] * cv[0] + cv[1] * cv[1] + cv[2] * cv[2]);
  if (fix_negative && t < 0.0) t = -t;
  if (ntg && tag) {
    const double m = (tag[h] / 2 == 2) ? 1.0 : ntg[c];
    t = m * t;
  }
  out[h] = t;
}

__global__ void __launch_bounds__(256) face_trans_kernel(long long nf, const int* __restrict__ ptr,
                                                         const int* __restrict__ idx,
                                                         const double* __restrict__ th,
                                                         double* __restrict__ tf) {
  const long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (f >= nf) return;
  double s = 0.0;
  for (int k = ptr[f]; k < ptr[f + 1]; ++k) s += 1.0 / th[idx[k]];
  tf[f] = 1.0 / s;
}

void compute_trans(long long nh, const int* cell_no, const int* hface, const int* first_cell, const double* cc,
                   const double* fc, const double* fn, const double* K9, const double* ntg, const int* tag,
                   int fix_negative, double* out, cudaStream_t s) {
  if (nh <= 0) return;
  half_trans_kernel<<<grid_for(nh, 256), 256, 0, s>>>(nh, cell_no, hface, first_cell, cc, fc, fn, K9, ntg, tag,
                                                      fix_negative, out);
  PMB_CHECK_LAUNCH();
}

void face_trans(long long nf, const int* ptr, const int* idx, const double* th, double* tf, cudaStream_t s) {
  if (nf <= 0) return;
  face_trans_kernel<<<grid_for(nf, 256), 256, 0, s>>>(nf, ptr, idx, th, tf);
  PMB_CHECK_LAUNCH();
}

}  // namespace pmb
