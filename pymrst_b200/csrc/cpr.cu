// CPR two-stage preconditioner and flexible GMRES, FP64.
//
// Replaces CPRSolver.solve (pymrst/modules/ad_core/solvers/linear_solvers.py:
// 426-545).  The decoupling is the reference's quasi-IMPES weighting
// (1/b_i at the mean pressure, linear_solvers.py:155-190) and the two-stage
// form x = P solve_p(W r); x += local(r - A x) (:510-517).  The pressure
// stage is an aggregation-AMG V-cycle instead of pyamg / spilu; the local
// stage is red-black block Gauss-Seidel on the whole system started from the
// pressure correction (so it contains the "r - A x" of the second stage), in
// place of one block-Jacobi application.
#include <algorithm>
#include <cstdlib>
#include <cmath>

#include "pmb_cpr.cuh"

namespace pmb {

constexpr int kRedBlocks = 2 * kNumSM;

// ---- CPR pieces -----------------------------------------------------------

__global__ void __launch_bounds__(256) psum_kernel(int nc, const double2* __restrict__ x, double* part) {
  __shared__ double sh[32];
  double s = 0.0;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) s += x[c].x;
  s = block_sum(s, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// Quasi-IMPES weights 1/b_w, 1/b_o at the mean cell pressure.
__global__ void weights_kernel(OWView v, int G, const double* part, double* w) {
  if (threadIdx.x != 0) return;
  double s = 0.0;
  for (int b = 0; b < G; ++b) s += part[b];
  const double pm = s / v.nc;
  for (int i = 0; i < 2; ++i) {
    const double b = v.fl.c[i] == 0.0 ? v.fl.b0[i] : v.fl.b0[i] * exp(v.fl.c[i] * (pm - v.fl.p_ref));
    w[i] = 1.0 / b;
  }
}

// Pressure matrix A_p = W A P over the cell blocks: column 0 (d/dp) of
// each block, the two rows combined with the weights.
__global__ void ap_kernel(long long nnzb, const double4* __restrict__ A, const double* __restrict__ w,
                          double* __restrict__ ap) {
  const double ww = w[0], wo = w[1];
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nnzb;
       k += (long long)gridDim.x * blockDim.x) {
    const double4 a = A[k];
    ap[k] = ww * a.x + wo * a.z;
  }
}

__global__ void to_f32_kernel(long long n, const double* __restrict__ a, float* __restrict__ b) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}

template <class T>
__global__ void restrict_p_kernel(int nc, const double2* __restrict__ r, const double* __restrict__ w,
                                  T* __restrict__ bp) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  const double2 rr = r[c];
  bp[c] = w[0] * rr.x + w[1] * rr.y;
}

// ---- pressure system with well bhp unknowns --------------------------------
//
// Pressure unknowns [p_cells, bhp_wells].  For well k, with D its 3x3 block
// (rows eq_w, eq_o, ctrl; columns qWs, qOs, bhp) and D2 = D[0:2, 0:2], the
// rate unknowns are eliminated exactly from the control row and from the
// weighted cell rows:
//   well row:  a = D[2,0:2] D2^{-1};  diagonal D[2,2] - a D[0:2,2];
//              cell columns -a C_i[:, p]
//   cell rows: g_i = (w B_i[:, 0:2]) D2^{-1};  bhp column w B_i[:, 2] - g_i D[0:2,2]
// (the coupling between perforated cells that the elimination would add is
// left out of the preconditioner).

__global__ void ext_cells_kernel(long long nnzb, const double4* __restrict__ A, const double* __restrict__ w,
                                 const int* __restrict__ bsr2ext, double* __restrict__ ext) {
  const double ww = w[0], wo = w[1];
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nnzb;
       k += (long long)gridDim.x * blockDim.x) {
    const double4 a = A[k];
    ext[bsr2ext[k]] = ww * a.x + wo * a.z;
  }
}

__global__ void ext_wells_kernel(OWView v, const double* __restrict__ wj, const double* __restrict__ w,
                                 const int* __restrict__ perf_cw, const int* __restrict__ perf_wc,
                                 const int* __restrict__ well_diag, double* __restrict__ ext,
                                 double* __restrict__ g_perf, double* __restrict__ a_well) {
  const double ww = w[0], wo = w[1];
  for (int k = threadIdx.x; k < v.nw; k += blockDim.x) {
    const double* D = wj + v.wl.D + 9LL * k;
    const double det = D[0] * D[4] - D[1] * D[3];
    const bool ok = det != 0.0 && isfinite(det);
    const double id = ok ? 1.0 / det : 0.0;
    const double i00 = id * D[4], i01 = -id * D[1], i10 = -id * D[3], i11 = id * D[0];
    const double a0 = D[6] * i00 + D[7] * i10, a1 = D[6] * i01 + D[7] * i11;
    a_well[2 * k] = a0;
    a_well[2 * k + 1] = a1;
    const int i0 = v.perf_ptr[k], i1 = v.perf_ptr[k + 1];
    for (int i = i0; i < i1; ++i) {
      ext[perf_cw[i]] = 0.0;
      ext[perf_wc[i]] = 0.0;
    }
    ext[well_diag[k]] = D[8] - (a0 * D[2] + a1 * D[5]);
    for (int i = i0; i < i1; ++i) {
      const double* C = wj + v.wl.C + 4LL * i;
      ext[perf_wc[i]] += -(a0 * C[0] + a1 * C[2]);
      const double* B = wj + v.wl.B + 6LL * i;
      const double wb0 = ww * B[0] + wo * B[3], wb1 = ww * B[1] + wo * B[4], wb2 = ww * B[2] + wo * B[5];
      const double g0 = wb0 * i00 + wb1 * i10, g1 = wb0 * i01 + wb1 * i11;
      g_perf[2 * i] = g0;
      g_perf[2 * i + 1] = g1;
      ext[perf_cw[i]] += wb2 - (g0 * D[2] + g1 * D[5]);
    }
  }
}

// ext_wells_kernel with a thread per perforation (and one per well for the
// well's diagonal), for wells that perforate each cell once, so that every
// perforation owns its two entries: the same values as the serial loop.
__global__ void ext_wells_par_kernel(OWView v, const double* __restrict__ wj, const double* __restrict__ w,
                                     const int* __restrict__ perf_cw, const int* __restrict__ perf_wc,
                                     const int* __restrict__ well_diag, double* __restrict__ ext,
                                     double* __restrict__ g_perf, double* __restrict__ a_well) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const double ww = w[0], wo = w[1];
  auto well_inverse = [&](int k, double& i00, double& i01, double& i10, double& i11, double& a0, double& a1) {
    const double* D = wj + v.wl.D + 9LL * k;
    const double det = D[0] * D[4] - D[1] * D[3];
    const bool ok = det != 0.0 && isfinite(det);
    const double id = ok ? 1.0 / det : 0.0;
    i00 = id * D[4];
    i01 = -id * D[1];
    i10 = -id * D[3];
    i11 = id * D[0];
    a0 = D[6] * i00 + D[7] * i10;
    a1 = D[6] * i01 + D[7] * i11;
  };
  if (i < v.nperf) {
    const int k = v.perf_well[i];
    double i00, i01, i10, i11, a0, a1;
    well_inverse(k, i00, i01, i10, i11, a0, a1);
    const double* D = wj + v.wl.D + 9LL * k;
    const double* C = wj + v.wl.C + 4LL * i;
    ext[perf_wc[i]] = 0.0 + -(a0 * C[0] + a1 * C[2]);
    const double* B = wj + v.wl.B + 6LL * i;
    const double wb0 = ww * B[0] + wo * B[3], wb1 = ww * B[1] + wo * B[4], wb2 = ww * B[2] + wo * B[5];
    const double g0 = wb0 * i00 + wb1 * i10, g1 = wb0 * i01 + wb1 * i11;
    g_perf[2 * i] = g0;
    g_perf[2 * i + 1] = g1;
    ext[perf_cw[i]] = 0.0 + (wb2 - (g0 * D[2] + g1 * D[5]));
  }
  if (i < v.nw) {
    double i00, i01, i10, i11, a0, a1;
    well_inverse(i, i00, i01, i10, i11, a0, a1);
    const double* D = wj + v.wl.D + 9LL * i;
    a_well[2 * i] = a0;
    a_well[2 * i + 1] = a1;
    ext[well_diag[i]] = D[8] - (a0 * D[2] + a1 * D[5]);
  }
}

// Right-hand side of the well-augmented pressure system: perforated cells
// lose g_i r_w[0:2]; well rows get r_ctrl - a r_w[0:2].  Cell rows were
// written by restrict_p_kernel.
template <class T>
__global__ void restrict_wells_kernel(OWView v, const double* __restrict__ r, const double* __restrict__ g_perf,
                                      const double* __restrict__ a_well, T* __restrict__ bp) {
  const double* rwb = r + 2LL * v.nc;
  for (int q = threadIdx.x; q < v.npc; q += blockDim.x) {
    const int c = v.pcell[q];
    double s = bp[c];
    for (int j = v.pc_ptr[q]; j < v.pc_ptr[q + 1]; ++j) {
      const int i = v.pc_perf[j];
      const double* rw = rwb + 3LL * v.perf_well[i];
      s -= g_perf[2 * i] * rw[0] + g_perf[2 * i + 1] * rw[1];
    }
    bp[c] = s;
  }
  for (int k = threadIdx.x; k < v.nw; k += blockDim.x) {
    const double* rw = rwb + 3LL * k;
    bp[v.nc + k] = rw[2] - (a_well[2 * k] * rw[0] + a_well[2 * k + 1] * rw[1]);
  }
}

// z = P xp with well bhp: cells (xp, 0); wells (0, 0, xp[nc + k]).
template <class T>
__global__ void prolong_pw_kernel(int nc, int nw, const T* __restrict__ xp, double* __restrict__ z) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < nc) reinterpret_cast<double2*>(z)[t] = make_double2(xp[t], 0.0);
  if (t < nw) {
    z[2LL * nc + 3LL * t] = 0.0;
    z[2LL * nc + 3LL * t + 1] = 0.0;
    z[2LL * nc + 3LL * t + 2] = xp[nc + t];
  }
}

// z = P xp (cells: (xp, 0); wells: 0)
template <class T>
__global__ void prolong_p_kernel(int nc, int nwv, const T* __restrict__ xp, double* __restrict__ z) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < nc) reinterpret_cast<double2*>(z)[t] = make_double2(xp ? xp[t] : 0.0, 0.0);
  if (t < nwv) z[2LL * nc + t] = 0.0;
}

// One colour of block Gauss-Seidel on J z = r: for each cell of the colour,
// z_c += inv(B_cc) (r_c - sum_k B_ck z_col(k) - well columns).  Cells of one
// colour are never neighbours, so each thread writes only its own z_c.
__global__ void __launch_bounds__(256) gs_color_kernel(OWView v, int cstart, int cend,
                                                       const int* __restrict__ ccells,
                                                       const double4* __restrict__ A,
                                                       const double* __restrict__ wj,
                                                       const double* __restrict__ r,
                                                       double* __restrict__ z, int* status) {
  const int t = cstart + blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= cend) return;
  const int c = ccells[t];
  const double2* z2 = reinterpret_cast<const double2*>(z);
  double2 rc = reinterpret_cast<const double2*>(r)[c];
  double4 D = make_double4(0, 0, 0, 0);
  for (int k = v.row_ptr[c]; k < v.row_ptr[c + 1]; ++k) {
    const double4 a = A[k];
    const int j = v.col[k];
    const double2 zj = z2[j];
    rc.x -= a.x * zj.x + a.y * zj.y;
    rc.y -= a.z * zj.x + a.w * zj.y;
    if (j == c) D = a;
  }
  const int q = v.cell_pc[c];
  if (q >= 0) {
    const double* zw = z + 2LL * v.nc;
    for (int jj = v.pc_ptr[q]; jj < v.pc_ptr[q + 1]; ++jj) {
      const int i = v.pc_perf[jj];
      const int k = v.perf_well[i];
      const double* B = wj + v.wl.B + 6LL * i;
      rc.x -= B[0] * zw[3 * k] + B[1] * zw[3 * k + 1] + B[2] * zw[3 * k + 2];
      rc.y -= B[3] * zw[3 * k] + B[4] * zw[3 * k + 1] + B[5] * zw[3 * k + 2];
    }
  }
  const double det = D.x * D.w - D.y * D.z;
  if (det == 0.0 || !isfinite(det)) {
    atomicExch(status, PMB_ERR_PIVOT);
    return;
  }
  const double id = 1.0 / det;
  double2 zc = z2[c];
  zc.x += id * (D.w * rc.x - D.y * rc.y);
  zc.y += id * (-D.z * rc.x + D.x * rc.y);
  reinterpret_cast<double2*>(z)[c] = zc;
}

__device__ __forceinline__ double4 inv2(double4 D, bool& ok) {
  const double det = D.x * D.w - D.y * D.z;
  ok = det != 0.0 && isfinite(det);
  const double id = ok ? 1.0 / det : 0.0;
  return make_double4(id * D.w, -id * D.y, -id * D.z, id * D.x);
}
__device__ __forceinline__ double4 mul2(double4 a, double4 b) {
  return make_double4(a.x * b.x + a.y * b.z, a.x * b.y + a.y * b.w, a.z * b.x + a.w * b.z, a.z * b.y + a.w * b.w);
}
__device__ __forceinline__ double2 mv2(double4 a, double2 v) {
  return make_double2(a.x * v.x + a.y * v.y, a.z * v.x + a.w * v.y);
}
// Block loads in FP64 arithmetic from FP64 or FP32 storage.
__device__ __forceinline__ double4 ld4(const double4& a) { return a; }
__device__ __forceinline__ double4 ld4(const float4& a) { return make_double4(a.x, a.y, a.z, a.w); }

// rc -= sum over the cell's block row [kb, ke) of A[k] z[col[k]], in row
// order.  The column indices, z values and blocks of the first kRowPrefetch
// entries are all loaded before any is used, so that a row costs two
// dependent memory round trips (column, then z) rather than one per block.
constexpr int kRowPrefetch = 8;
template <class BT>
__device__ __forceinline__ void sub_row(const int* __restrict__ col, const BT* __restrict__ A,
                                        const double2* __restrict__ z2, int kb, int ke, double2& rc) {
  int cj[kRowPrefetch];
#pragma unroll
  for (int q = 0; q < kRowPrefetch; ++q) cj[q] = kb + q < ke ? col[kb + q] : 0;
  double2 zq[kRowPrefetch];
  double4 aq[kRowPrefetch];
#pragma unroll
  for (int q = 0; q < kRowPrefetch; ++q) {
    zq[q] = make_double2(0.0, 0.0);
    aq[q] = make_double4(0.0, 0.0, 0.0, 0.0);
    if (kb + q < ke) {
      zq[q] = z2[cj[q]];
      aq[q] = ld4(A[kb + q]);
    }
  }
#pragma unroll
  for (int q = 0; q < kRowPrefetch; ++q)
    if (kb + q < ke) {
      const double2 t = mv2(aq[q], zq[q]);
      rc.x -= t.x;
      rc.y -= t.y;
    }
  for (int k = kb + kRowPrefetch; k < ke; ++k) {
    const double2 t = mv2(ld4(A[k]), z2[col[k]]);
    rc.x -= t.x;
    rc.y -= t.y;
  }
}

// Line Gauss-Seidel for one colour of vertical lines, one warp per line:
// the lanes form the block residual r - J z of the line's cells, then lane 0
// solves the line's block-tridiagonal system (its couplings to the previous
// and next cell of the line) by block Thomas elimination and adds the
// correction to z.  Lines of one colour never touch, so every warp writes
// only its own cells.  `ys` / `gs` are per-line-position scratch (the
// forward-eliminated right-hand side and the inverted pivots).
// Lines of up to kLineSmem cells are staged in shared memory (pivot blocks,
// couplings and right-hand side), so that lane 0's sequential recurrence reads
// shared memory instead of waiting on global loads; longer lines use the
// global scratch.
constexpr int kLineSmem = 96;
constexpr int kLineWarps = 2;

template <class BT>
__global__ void __launch_bounds__(32 * kLineWarps) line_gs_kernel(OWView v, int lstart, int lend,
                                                      const int* __restrict__ clines,
                                                      const int* __restrict__ lptr,
                                                      const int* __restrict__ lcells,
                                                      const int* __restrict__ llo,
                                                      const int* __restrict__ lup,
                                                      const BT* __restrict__ A,
                                                      const double* __restrict__ wj,
                                                      const double* __restrict__ r, double* __restrict__ z,
                                                      double2* __restrict__ ys, double4* __restrict__ gs,
                                                      int* status) {
  __shared__ double4 sD[kLineWarps][kLineSmem], sL[kLineWarps][kLineSmem], sU[kLineWarps][kLineSmem];
  __shared__ double2 sY[kLineWarps][kLineSmem];
  __shared__ int sBad[kLineWarps];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int li = lstart + (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5);
  if (li >= lend) return;  // uniform across the warp
  const int L = clines[li];
  const int t0 = lptr[L], t1 = lptr[L + 1];
  const double2* z2 = reinterpret_cast<const double2*>(z);
  if (t1 - t0 <= kLineSmem) {
    const int len = t1 - t0;
    const double4 zero4 = make_double4(0, 0, 0, 0);
    for (int u = lane; u < len; u += 32) {
      const int t = t0 + u;
      const int c = lcells[t];
      double2 rc = reinterpret_cast<const double2*>(r)[c];
      sub_row(v.col, A, z2, v.row_ptr[c], v.row_ptr[c + 1], rc);
      const int q = v.cell_pc[c];
      if (q >= 0) {
        const double* zw = z + 2LL * v.nc;
        for (int jj = v.pc_ptr[q]; jj < v.pc_ptr[q + 1]; ++jj) {
          const int i = v.pc_perf[jj];
          const int kw = v.perf_well[i];
          const double* B = wj + v.wl.B + 6LL * i;
          rc.x -= B[0] * zw[3 * kw] + B[1] * zw[3 * kw + 1] + B[2] * zw[3 * kw + 2];
          rc.y -= B[3] * zw[3 * kw] + B[4] * zw[3 * kw + 1] + B[5] * zw[3 * kw + 2];
        }
      }
      sY[wib][u] = rc;
      sD[wib][u] = ld4(A[v.diag_pos[c]]);
      sL[wib][u] = llo[t] >= 0 ? ld4(A[llo[t]]) : zero4;
      sU[wib][u] = lup[t] >= 0 ? ld4(A[lup[t]]) : zero4;
    }
    __syncwarp();
    if (lane == 0) {
      int bad = 0;
      double4 Gp = zero4;
      double2 yp = make_double2(0, 0);
      for (int u = 0; u < len && !bad; ++u) {
        double4 D = sD[wib][u];
        double2 y = sY[wib][u];
        if (u > 0) {
          const double4 LG = mul2(sL[wib][u], Gp);
          const double4 LGU = mul2(LG, sU[wib][u - 1]);
          D.x -= LGU.x; D.y -= LGU.y; D.z -= LGU.z; D.w -= LGU.w;
          const double2 qq = mv2(LG, yp);
          y.x -= qq.x;
          y.y -= qq.y;
        }
        bool ok;
        const double4 G = inv2(D, ok);
        if (!ok) bad = 1;
        sD[wib][u] = G;
        sY[wib][u] = y;
        Gp = G;
        yp = y;
      }
      if (!bad) {
        double2 dn = make_double2(0, 0);
        for (int u = len - 1; u >= 0; --u) {
          double2 y = sY[wib][u];
          if (u + 1 < len) {
            const double2 qq = mv2(sU[wib][u], dn);
            y.x -= qq.x;
            y.y -= qq.y;
          }
          dn = mv2(sD[wib][u], y);
          sY[wib][u] = dn;
        }
      } else {
        atomicExch(status, PMB_ERR_PIVOT);
      }
      sBad[wib] = bad;
    }
    __syncwarp();
    if (sBad[wib]) return;
    for (int u = lane; u < len; u += 32) {
      const int c = lcells[t0 + u];
      double2 zc = z2[c];
      zc.x += sY[wib][u].x;
      zc.y += sY[wib][u].y;
      reinterpret_cast<double2*>(z)[c] = zc;
    }
    return;
  }
  for (int t = t0 + lane; t < t1; t += 32) {
    const int c = lcells[t];
    double2 rc = reinterpret_cast<const double2*>(r)[c];
    sub_row(v.col, A, z2, v.row_ptr[c], v.row_ptr[c + 1], rc);
    const int q = v.cell_pc[c];
    if (q >= 0) {
      const double* zw = z + 2LL * v.nc;
      for (int jj = v.pc_ptr[q]; jj < v.pc_ptr[q + 1]; ++jj) {
        const int i = v.pc_perf[jj];
        const int kw = v.perf_well[i];
        const double* B = wj + v.wl.B + 6LL * i;
        rc.x -= B[0] * zw[3 * kw] + B[1] * zw[3 * kw + 1] + B[2] * zw[3 * kw + 2];
        rc.y -= B[3] * zw[3 * kw] + B[4] * zw[3 * kw + 1] + B[5] * zw[3 * kw + 2];
      }
    }
    ys[t] = rc;
  }
  __syncwarp();
  if (lane != 0) return;
  // forward elimination
  double4 Gp = make_double4(0, 0, 0, 0);
  double2 yp = make_double2(0, 0);
  for (int t = t0; t < t1; ++t) {
    const int c = lcells[t];
    double4 D = ld4(A[v.diag_pos[c]]);
    double2 y = ys[t];
    if (t > t0 && llo[t] >= 0 && lup[t - 1] >= 0) {
      const double4 LG = mul2(ld4(A[llo[t]]), Gp);
      const double4 LGU = mul2(LG, ld4(A[lup[t - 1]]));
      D.x -= LGU.x; D.y -= LGU.y; D.z -= LGU.z; D.w -= LGU.w;
      const double2 q = mv2(LG, yp);
      y.x -= q.x;
      y.y -= q.y;
    }
    bool ok;
    const double4 G = inv2(D, ok);
    if (!ok) {
      atomicExch(status, PMB_ERR_PIVOT);
      return;
    }
    gs[t] = G;
    ys[t] = y;
    Gp = G;
    yp = y;
  }
  // back substitution
  double2 dn = make_double2(0, 0);
  for (int t = t1 - 1; t >= t0; --t) {
    double2 y = ys[t];
    if (t + 1 < t1 && lup[t] >= 0) {
      const double2 q = mv2(ld4(A[lup[t]]), dn);
      y.x -= q.x;
      y.y -= q.y;
    }
    dn = mv2(gs[t], y);
    const int c = lcells[t];
    double2 zc = z2[c];
    zc.x += dn.x;
    zc.y += dn.y;
    reinterpret_cast<double2*>(z)[c] = zc;
  }
}

// Line Gauss-Seidel for one colour of vertical lines by parallel cyclic
// reduction: one CTA per line, one thread per cell of the line.  Each thread
// forms its cell's block residual r - J z (the whole block row and the well
// columns) and loads its diagonal block and its couplings to the previous and
// next cell of the line; the CTA then solves the line's block-tridiagonal
// system
//   L_u x_{u-1} + D_u x_u + U_u x_{u+1} = y_u
// in ceil(log2(len)) steps, each eliminating the couplings at distance s from
// every equation at once:
//   a = -L_u inv(D_{u-s}),  g = -U_u inv(D_{u+s}),
//   D_u += a U_{u-s} + g L_{u+s},  L_u = a L_{u-s},  U_u = g U_{u+s},
//   y_u += a y_{u-s} + g y_{u+s},
// after which x_u = inv(D_u) y_u is added to z.  Lines of one colour never
// touch, so every CTA writes only its own cells.  Needs blockDim.x >= the
// line's length; shared memory 144 B per thread.
constexpr int kPcrMaxLen = 256;

// 2x2 block (row-major) and 2-vector in the arithmetic type of the line solve.
template <class CT>
struct alignas(4 * sizeof(CT)) Blk2 {
  CT x, y, z, w;
};
template <class CT>
struct alignas(2 * sizeof(CT)) Vec2 {
  CT x, y;
};
template <class CT>
__device__ __forceinline__ Blk2<CT> blk_of(double4 a) {
  return Blk2<CT>{(CT)a.x, (CT)a.y, (CT)a.z, (CT)a.w};
}
template <class CT>
__device__ __forceinline__ Blk2<CT> bmul(Blk2<CT> a, Blk2<CT> b) {
  return Blk2<CT>{a.x * b.x + a.y * b.z, a.x * b.y + a.y * b.w, a.z * b.x + a.w * b.z, a.z * b.y + a.w * b.w};
}
template <class CT>
__device__ __forceinline__ Vec2<CT> bmv(Blk2<CT> a, Vec2<CT> v) {
  return Vec2<CT>{a.x * v.x + a.y * v.y, a.z * v.x + a.w * v.y};
}
template <class CT>
__device__ __forceinline__ Blk2<CT> badd(Blk2<CT> a, Blk2<CT> b) {
  return Blk2<CT>{a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w};
}
template <class CT>
__device__ __forceinline__ Blk2<CT> bneg(Blk2<CT> a) {
  return Blk2<CT>{-a.x, -a.y, -a.z, -a.w};
}
template <class CT>
__device__ __forceinline__ Blk2<CT> binv(Blk2<CT> D, bool& ok) {
  const CT det = D.x * D.w - D.y * D.z;
  ok = det != CT(0) && isfinite(det);
  const CT id = ok ? CT(1) / det : CT(0);
  return Blk2<CT>{id * D.w, -id * D.y, -id * D.z, id * D.x};
}

// The cyclic reduction of one line: thread u holds row u of the line's
// block-tridiagonal system (D, Lb, Ub, y; Lb of the first row and Ub of the
// last are zero); on a true return x is its solution.  Every thread of the CTA
// takes part (act false for threads past the line's end); a singular pivot
// sets *status and returns false.  `raw` is the CTA's shared memory,
// 3 blocks and one vector per thread; `bad` a shared flag zeroed by thread 0
// before the first barrier.
template <class CT>
__device__ __forceinline__ bool pcr_line(unsigned char* raw, int u, int len, bool act, Blk2<CT> D, Blk2<CT> Lb,
                                         Blk2<CT> Ub, Vec2<CT> y, int* bad, int* status, Vec2<CT>& x) {
  const int nb = blockDim.x;
  Blk2<CT>* sL = reinterpret_cast<Blk2<CT>*>(raw);
  Blk2<CT>* sU = sL + nb;
  Blk2<CT>* sI = sL + 2 * nb;
  Vec2<CT>* sY = reinterpret_cast<Vec2<CT>*>(sL + 3 * nb);
  const Blk2<CT> zero = {CT(0), CT(0), CT(0), CT(0)};
  for (int s = 1; s < len; s <<= 1) {
    bool ok = true;
    const Blk2<CT> I = binv(D, ok);
    if (act && !ok) *bad = 1;
    if (act) {
      sL[u] = Lb;
      sU[u] = Ub;
      sI[u] = I;
      sY[u] = y;
    }
    __syncthreads();
    if (*bad) break;  // uniform: read after the barrier by every thread
    if (act) {
      Blk2<CT> nD = D, nL = zero, nU = zero;
      Vec2<CT> ny = y;
      if (u - s >= 0) {
        const Blk2<CT> a = bneg(bmul(Lb, sI[u - s]));
        nD = badd(nD, bmul(a, sU[u - s]));
        nL = bmul(a, sL[u - s]);
        const Vec2<CT> q = bmv(a, sY[u - s]);
        ny.x += q.x;
        ny.y += q.y;
      }
      if (u + s < len) {
        const Blk2<CT> g = bneg(bmul(Ub, sI[u + s]));
        nD = badd(nD, bmul(g, sL[u + s]));
        nU = bmul(g, sU[u + s]);
        const Vec2<CT> q = bmv(g, sY[u + s]);
        ny.x += q.x;
        ny.y += q.y;
      }
      D = nD;
      Lb = nL;
      Ub = nU;
      y = ny;
    }
    __syncthreads();
  }
  if (*bad) {
    if (u == 0) atomicExch(status, PMB_ERR_PIVOT);
    return false;
  }
  if (!act) return false;
  bool ok = true;
  const Blk2<CT> I = binv(D, ok);
  if (!ok) {
    atomicExch(status, PMB_ERR_PIVOT);
    return false;
  }
  x = bmv(I, y);
  return true;
}

// rc -= the well columns of a cell's row: B blocks of its perforations (pc
// its index among the perforated cells, -1 for none) times the well unknowns.
__device__ __forceinline__ void sub_wells(const OWView& v, const double* __restrict__ wj,
                                          const double* __restrict__ z, int pc, double2& rc) {
  if (pc < 0) return;
  const double* zw = z + 2LL * v.nc;
  for (int jj = v.pc_ptr[pc]; jj < v.pc_ptr[pc + 1]; ++jj) {
    const int i = v.pc_perf[jj];
    const int kw = v.perf_well[i];
    const double* B = wj + v.wl.B + 6LL * i;
    rc.x -= B[0] * zw[3 * kw] + B[1] * zw[3 * kw + 1] + B[2] * zw[3 * kw + 2];
    rc.y -= B[3] * zw[3 * kw] + B[4] * zw[3 * kw + 1] + B[5] * zw[3 * kw + 2];
  }
}

// CT is the arithmetic of the cyclic reduction: double, or float when the
// smoother blocks are FP32 (mixed precision); the residual is formed in FP64.
template <class BT, class CT>
__global__ void __launch_bounds__(kPcrMaxLen) line_pcr_kernel(OWView v, int lstart, const int* __restrict__ clines,
                                                              const int* __restrict__ lptr,
                                                              const int* __restrict__ lcells,
                                                              const int* __restrict__ llo,
                                                              const int* __restrict__ lup,
                                                              const BT* __restrict__ A,
                                                              const double* __restrict__ wj,
                                                              const double* __restrict__ r, double* __restrict__ z,
                                                              int* status) {
  extern __shared__ __align__(16) unsigned char pcr_raw[];
  __shared__ int sBad;
  const int line = clines[lstart + blockIdx.x];
  const int t0 = lptr[line];
  const int len = lptr[line + 1] - t0;
  const int u = threadIdx.x;
  const bool act = u < len;
  if (u == 0) sBad = 0;
  const Blk2<CT> zero = {CT(0), CT(0), CT(0), CT(0)};
  const double2* z2 = reinterpret_cast<const double2*>(z);
  Blk2<CT> D = {CT(1), CT(0), CT(0), CT(1)}, Lb = zero, Ub = zero;
  Vec2<CT> y = {CT(0), CT(0)};
  int c = 0;
  if (act) {
    const int t = t0 + u;
    c = lcells[t];
    double2 rc = reinterpret_cast<const double2*>(r)[c];
    // the line blocks first, so that their loads overlap the row gather
    const int kl = u > 0 ? llo[t] : -1;
    const int ku = u + 1 < len ? lup[t] : -1;
    D = blk_of<CT>(ld4(A[v.diag_pos[c]]));
    if (kl >= 0) Lb = blk_of<CT>(ld4(A[kl]));
    if (ku >= 0) Ub = blk_of<CT>(ld4(A[ku]));
    sub_row(v.col, A, z2, v.row_ptr[c], v.row_ptr[c + 1], rc);
    sub_wells(v, wj, z, v.cell_pc[c], rc);
    y = Vec2<CT>{(CT)rc.x, (CT)rc.y};
  }
  Vec2<CT> x;
  if (!pcr_line<CT>(pcr_raw, u, len, act, D, Lb, Ub, y, &sBad, status, x)) return;
  double2 zc = z2[c];
  zc.x += (double)x.x;
  zc.y += (double)x.y;
  reinterpret_cast<double2*>(z)[c] = zc;
}

// ---- the line smoother on a line-ordered copy of its operator ----------------
//
// Position t of the line order is the t-th cell of the concatenated lines, so
// the cells of one line are consecutive.  Blocks are stored slot-major,
// blk[slot * nc + t]: slot 0 the diagonal, 1 and 2 the couplings to the
// previous and next cell of the line (zero at a line end or where the cells
// do not couple), 3.. the row's other blocks (zero-padded, their column the
// position t itself).  Thread u of a line's CTA then reads blk[slot * nc +
// t0 + u], rl / zl at t0 + u and, in a grid whose neighbouring lines have the
// same cells, zl of the lateral neighbours at t0' + u: every load of a warp is
// one contiguous run.
constexpr int kEllMaxSlots = 12;  // diagonal, two line couplings, up to nine others
constexpr int kEllPrefetch = 4;   // lateral entries loaded before the first is used

template <class BT>
__device__ __forceinline__ BT blk_store(double4 a);
template <>
__device__ __forceinline__ double4 blk_store<double4>(double4 a) {
  return a;
}
template <>
__device__ __forceinline__ float4 blk_store<float4>(double4 a) {
  return make_float4((float)a.x, (float)a.y, (float)a.z, (float)a.w);
}

// blk[i] = A[src[i]] (zero where src is -1), in the smoother's storage type.
template <class BT>
__global__ void ell_gather_kernel(long long n, const int* __restrict__ src, const double4* __restrict__ A,
                                  BT* __restrict__ blk) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int k = src[i];
  blk[i] = blk_store<BT>(k >= 0 ? A[k] : make_double4(0.0, 0.0, 0.0, 0.0));
}

// Into line order: rl[t] = r of the t-th cell, zl[t] = its z (from_z) or the
// prolonged pressure correction (xp_c, 0) (xp null: zero).  Without from_z
// the well part of z is prolonged as well: (0, 0, xp[nc + k]) when the
// pressure system has bhp unknowns (pw), else zero.
// The line-ordered r and z of the smoother: FP64, or FP32 in mixed precision
// (their residual is still formed and summed in FP64).
__device__ __forceinline__ double2 lv_load(const double* p, long long t) {
  return reinterpret_cast<const double2*>(p)[t];
}
__device__ __forceinline__ double2 lv_load(const float* p, long long t) {
  const float2 v = reinterpret_cast<const float2*>(p)[t];
  return make_double2((double)v.x, (double)v.y);
}
// The raw pair, converted only where it is used (fewer registers in FP32).
template <class LV>
struct LvPair;
template <>
struct LvPair<double> {
  using type = double2;
};
template <>
struct LvPair<float> {
  using type = float2;
};
template <class LV>
__device__ __forceinline__ typename LvPair<LV>::type lv_raw(const LV* p, long long t) {
  return reinterpret_cast<const typename LvPair<LV>::type*>(p)[t];
}
__device__ __forceinline__ double2 lv_d2(double2 v) { return v; }
__device__ __forceinline__ double2 lv_d2(float2 v) { return make_double2((double)v.x, (double)v.y); }

__device__ __forceinline__ void lv_store(double* p, long long t, double2 v) {
  reinterpret_cast<double2*>(p)[t] = v;
}
__device__ __forceinline__ void lv_store(float* p, long long t, double2 v) {
  reinterpret_cast<float2*>(p)[t] = make_float2((float)v.x, (float)v.y);
}

template <class T, class LV>
__global__ void line_enter_kernel(int nc, int nw, bool from_z, bool pw, const int* __restrict__ lcells,
                                  const T* __restrict__ xp, const double* __restrict__ r, double* __restrict__ z,
                                  LV* __restrict__ rl, LV* __restrict__ zl) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < nc) {
    const int c = lcells[t];
    lv_store(rl, t, reinterpret_cast<const double2*>(r)[c]);
    lv_store(zl, t, from_z ? reinterpret_cast<const double2*>(z)[c] : make_double2(xp ? (double)xp[c] : 0.0, 0.0));
  }
  if (from_z) return;
  if (t < nw) {
    z[2LL * nc + 3LL * t] = 0.0;
    z[2LL * nc + 3LL * t + 1] = 0.0;
    z[2LL * nc + 3LL * t + 2] = pw && xp ? (double)xp[nc + t] : 0.0;
  }
}

// line_pcr_kernel on the line-ordered copy: one CTA per line of the colour,
// thread u on position t0 + u.  zl is updated in place; with OUT (the last
// sweep) the cell's new z is also written to z in cell order.  The well
// unknowns are read from z (they stay in cell order).
template <class BT, class CT, bool OUT, class LV>
__global__ void __launch_bounds__(kPcrMaxLen, sizeof(CT) == 4 ? 4 : 3)
    line_pcr_ell_kernel(OWView v, int lstart, const int2* __restrict__ crange, const int* __restrict__ lcells,
                        int nslots, const BT* __restrict__ blk, const int* __restrict__ ecol,
                        const int* __restrict__ epc, const double* __restrict__ wj, const LV* __restrict__ rl,
                        LV* __restrict__ zl, double* __restrict__ z, int* status) {
  extern __shared__ __align__(16) unsigned char pcr_raw[];
  __shared__ int sBad;
  const int2 lr = crange[lstart + blockIdx.x];  // (first position, length) of the CTA's line
  const int t0 = lr.x, len = lr.y;
  const int u = threadIdx.x;
  const bool act = u < len;
  if (u == 0) sBad = 0;
  const long long n = v.nc;
  const int t = t0 + u;
  const Blk2<CT> zero = {CT(0), CT(0), CT(0), CT(0)};
  const double2 z0 = make_double2(0.0, 0.0);
  Blk2<CT> D = {CT(1), CT(0), CT(0), CT(1)}, Lb = zero, Ub = zero;
  Vec2<CT> y = {CT(0), CT(0)};
  double2 zs = z0;
  // the lateral columns and the perforation index (written at the set-up,
  // never inside a solve) are loaded before the wait on the predecessor
  // grid, so that after it the blocks, r, z and the lateral z gathers all go
  // out together
  const int nlat = nslots - 3;
  const BT bz = blk_store<BT>(make_double4(0.0, 0.0, 0.0, 0.0));
  int cj[kEllPrefetch];
  int pc = -1;
#pragma unroll
  for (int q = 0; q < kEllPrefetch; ++q) cj[q] = t;
  if (act) {
#pragma unroll
    for (int q = 0; q < kEllPrefetch; ++q)
      if (q < nlat) cj[q] = ecol[q * n + t];
    pc = epc[t];
  }
  pdl_enter();
  if (act) {
    BT aq[kEllPrefetch];
#pragma unroll
    for (int q = 0; q < kEllPrefetch; ++q) aq[q] = q < nlat ? blk[(3 + q) * n + t] : bz;
    const BT Dr = blk[t];
    const BT Lr = u > 0 ? blk[n + t] : bz;
    const BT Ur = u + 1 < len ? blk[2 * n + t] : bz;
    zs = lv_load(zl, t);
    const double2 zlo = u > 0 ? lv_load(zl, t - 1) : z0;
    const double2 zup = u + 1 < len ? lv_load(zl, t + 1) : z0;
    typename LvPair<LV>::type zq[kEllPrefetch];
#pragma unroll
    for (int q = 0; q < kEllPrefetch; ++q) zq[q] = lv_raw(zl, q < nlat ? cj[q] : t);
    double2 rc = lv_load(rl, t);
    double2 m = mv2(ld4(Dr), zs);
    rc.x -= m.x;
    rc.y -= m.y;
    m = mv2(ld4(Lr), zlo);
    rc.x -= m.x;
    rc.y -= m.y;
    m = mv2(ld4(Ur), zup);
    rc.x -= m.x;
    rc.y -= m.y;
#pragma unroll
    for (int q = 0; q < kEllPrefetch; ++q) {
      m = mv2(ld4(aq[q]), lv_d2(zq[q]));  // a zero block where q >= nlat
      rc.x -= m.x;
      rc.y -= m.y;
    }
    for (int q = kEllPrefetch; q < nlat; ++q) {
      m = mv2(ld4(blk[(3 + q) * n + t]), lv_load(zl, ecol[q * n + t]));
      rc.x -= m.x;
      rc.y -= m.y;
    }
    sub_wells(v, wj, z, pc, rc);
    D = blk_of<CT>(ld4(Dr));
    Lb = blk_of<CT>(ld4(Lr));
    Ub = blk_of<CT>(ld4(Ur));
    y = Vec2<CT>{(CT)rc.x, (CT)rc.y};
  }
  Vec2<CT> x;
  if (!pcr_line<CT>(pcr_raw, u, len, act, D, Lb, Ub, y, &sBad, status, x)) return;
  zs.x += (double)x.x;
  zs.y += (double)x.y;
  lv_store(zl, t, zs);
  if (OUT) reinterpret_cast<double2*>(z)[lcells[t]] = zs;
}

// Well unknowns: z_w += inv(D_k) (r_w - C z_cells - D_k z_w); one warp per
// well, the lanes over its perforations.  The cells' z is read from zc at the
// perforated cell (ppos null) or at its line position ppos[i]; the wells' z
// and r are in z and r.
template <class ZT>
__global__ void __launch_bounds__(256) gs_well_kernel(OWView v, const double* __restrict__ wj,
                                                      const double* __restrict__ r, double* __restrict__ z,
                                                      const ZT* __restrict__ zc, const int* __restrict__ ppos) {
  pdl_enter();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  for (int k = warp; k < v.nw; k += nwarp) {
    double s0 = 0.0, s1 = 0.0;
    for (int i = v.perf_ptr[k] + lane; i < v.perf_ptr[k + 1]; i += 32) {
      const int c = ppos ? ppos[i] : v.perf_cell[i];
      const double* C = wj + v.wl.C + 4LL * i;
      const double zp = (double)zc[2LL * c], zs = (double)zc[2LL * c + 1];
      s0 += C[0] * zp + C[1] * zs;
      s1 += C[2] * zp + C[3] * zs;
    }
    s0 = warp_sum(s0);
    s1 = warp_sum(s1);
    if (lane != 0) continue;
    const double* D = wj + v.wl.D + 9LL * k;
    double* zw = z + 2LL * v.nc + 3LL * k;
    const double* rw = r + 2LL * v.nc + 3LL * k;
    double e0 = rw[0] - s0, e1 = rw[1] - s1, e2 = rw[2];
    e0 -= D[0] * zw[0] + D[1] * zw[1] + D[2] * zw[2];
    e1 -= D[3] * zw[0] + D[4] * zw[1] + D[5] * zw[2];
    e2 -= D[6] * zw[0] + D[7] * zw[1] + D[8] * zw[2];
    // 3x3 inverse by cofactors
    const double a = D[0], b = D[1], c = D[2], d = D[3], e = D[4], f = D[5], g = D[6], h = D[7], i9 = D[8];
    const double A0 = e * i9 - f * h, A1 = -(d * i9 - f * g), A2 = d * h - e * g;
    const double det = a * A0 + b * A1 + c * A2;
    if (det == 0.0 || !isfinite(det)) continue;
    const double id = 1.0 / det;
    const double B0 = -(b * i9 - c * h), B1 = a * i9 - c * g, B2 = -(a * h - b * g);
    const double C0 = b * f - c * e, C1 = -(a * f - c * d), C2 = a * e - b * d;
    zw[0] += id * (A0 * e0 + B0 * e1 + C0 * e2);
    zw[1] += id * (A1 * e0 + B1 * e1 + C1 * e2);
    zw[2] += id * (A2 * e0 + B2 * e1 + C2 * e2);
  }
}

// ---- host -------------------------------------------------------------------

CPRSolver::CPRSolver(OWModel& m, const pmb_cpr_opts& o) : m_(m), o_(o), s_(m.stream()) {
  PMB_REQUIRE(o_.restart >= 1 && o_.restart <= kMaxRestart, "restart must be in 1..60");
  PMB_REQUIRE(o_.maxiter >= 1, "maxiter must be positive");
  PMB_REQUIRE(o_.rtol > 0.0, "rtol must be positive");
  PMB_REQUIRE(o_.precision == 0 || o_.precision == 1, "precision must be 0 (FP64) or 1 (FP32 preconditioner)");
  f32_ = o_.precision == 1;
  graph_.enabled = o_.replay_graph != 0;
  kry_.init(m.nvec(), o_.restart, s_);
  w_.resize(2);
  part_.resize((size_t)kRedBlocks);
  status_.resize(1);  // device error status
  status_.zero(s_);
  np_ = m.nc();
  if (m.nw() > 0) build_pressure_pattern();
  bp_.resize(np_);
  xp_.resize(np_);
  if (m.has_lines()) build_line_ell();
  if (m.has_lines() && !use_ell_) {
    line_y_.resize(2LL * m.nc());
    line_g_.resize(4LL * m.nc());
  }
  ap_.resize(np_ > m.nc() ? h_ecol_.size() : (size_t)m.nnzb());
  st_pin_.resize(1);
  st_pin_[0] = 0;
  amg_.degree = amg32_.degree = std::max(1, o_.amg_smoother_degree);
  amg_.coarse_degree = amg32_.coarse_degree = std::max(0, o_.amg_coarse_degree);
  amg_.k_levels = amg32_.k_levels = std::max(0, o_.amg_cycle);
  if (f32_) {
    if (m.has_lines() && !use_ell_) jac32_.resize(4LL * m.nnzb());
    bp32_.resize(np_);
    xp32_.resize(np_);
  }
  PMB_CUDA(cudaStreamSynchronize(s_));
}

// CSR pattern of the well-augmented pressure system: cell rows keep their
// block-CSR columns (in order) followed by the bhp columns of the wells that
// perforate them; well rows list their perforated cells, then themselves.
void CPRSolver::build_pressure_pattern() {
  const OWView v = m_.view();
  const int nc = v.nc, nw = v.nw;
  const auto& rp = m_.h_row_ptr();
  const auto& col = m_.h_col();
  std::vector<int> perf_ptr(nw + 1), perf_cell(v.nperf);
  PMB_CUDA(cudaMemcpy(perf_ptr.data(), v.perf_ptr, sizeof(int) * (nw + 1), cudaMemcpyDeviceToHost));
  if (v.nperf)
    PMB_CUDA(cudaMemcpy(perf_cell.data(), v.perf_cell, sizeof(int) * v.nperf, cudaMemcpyDeviceToHost));
  std::vector<std::vector<int>> cell_wells(nc);
  std::vector<std::vector<int>> well_cells(nw);
  for (int k = 0; k < nw; ++k)
    for (int i = perf_ptr[k]; i < perf_ptr[k + 1]; ++i) {
      cell_wells[perf_cell[i]].push_back(k);
      well_cells[k].push_back(perf_cell[i]);
    }
  for (auto& s : cell_wells) { std::sort(s.begin(), s.end()); s.erase(std::unique(s.begin(), s.end()), s.end()); }
  for (auto& s : well_cells) { std::sort(s.begin(), s.end()); s.erase(std::unique(s.begin(), s.end()), s.end()); }
  np_ = nc + nw;
  h_erp_.assign(np_ + 1, 0);
  h_ecol_.clear();
  std::vector<int> bsr2ext(rp[nc]);
  for (int c = 0; c < nc; ++c) {
    for (int k = rp[c]; k < rp[c + 1]; ++k) {
      bsr2ext[k] = (int)h_ecol_.size();
      h_ecol_.push_back(col[k]);
    }
    for (int k : cell_wells[c]) h_ecol_.push_back(nc + k);
    h_erp_[c + 1] = (int)h_ecol_.size();
  }
  std::vector<int> well_diag(nw);
  for (int k = 0; k < nw; ++k) {
    for (int c : well_cells[k]) h_ecol_.push_back(c);
    well_diag[k] = (int)h_ecol_.size();
    h_ecol_.push_back(nc + k);
    h_erp_[nc + k + 1] = (int)h_ecol_.size();
  }
  std::vector<int> perf_cw(v.nperf), perf_wc(v.nperf);
  for (int k = 0; k < nw; ++k)
    for (int i = perf_ptr[k]; i < perf_ptr[k + 1]; ++i) {
      const int c = perf_cell[i];
      const int ncell_cols = rp[c + 1] - rp[c];
      const auto& cw = cell_wells[c];
      perf_cw[i] = h_erp_[c] + ncell_cols + (int)(std::lower_bound(cw.begin(), cw.end(), k) - cw.begin());
      const auto& wc = well_cells[k];
      perf_wc[i] = h_erp_[nc + k] + (int)(std::lower_bound(wc.begin(), wc.end(), c) - wc.begin());
    }
  erp_.upload(h_erp_, s_);
  ecol_.upload(h_ecol_, s_);
  bsr2ext_.upload(bsr2ext, s_);
  {
    std::vector<int> e(perf_cw);
    std::sort(e.begin(), e.end());
    ext_par_ = std::adjacent_find(e.begin(), e.end()) == e.end();  // no cell perforated twice by one well
  }
  perf_cw_.upload(perf_cw, s_);
  perf_wc_.upload(perf_wc, s_);
  well_diag_.upload(well_diag, s_);
  g_perf_.resize(2LL * std::max(v.nperf, 1));
  a_well_.resize(2LL * nw);
}

// The line-ordered copy of the smoother's operator (the layout is described
// above line_pcr_ell_kernel).  Left unbuilt, so that the block-CSR kernels
// run, when a line is longer than one CTA, a row has too many blocks, or
// PMB_LINE_ELL=0.
void CPRSolver::build_line_ell() {
  static const bool off = [] {
    const char* e = std::getenv("PMB_LINE_ELL");
    return e && e[0] == '0';
  }();
  const auto& Ls = m_.lines();
  const int nc = m_.nc();
  if (off || Ls.max_len > kPcrMaxLen) return;
  const auto& rp = m_.h_row_ptr();
  const auto& col = m_.h_col();
  const OWView v = m_.view();
  std::vector<int> cells(nc), lo(nc), up(nc), cell_pc(nc), perf_cell(v.nperf);
  PMB_CUDA(cudaMemcpy(cells.data(), Ls.line_cells.get(), sizeof(int) * nc, cudaMemcpyDeviceToHost));
  PMB_CUDA(cudaMemcpy(lo.data(), Ls.line_lo.get(), sizeof(int) * nc, cudaMemcpyDeviceToHost));
  PMB_CUDA(cudaMemcpy(up.data(), Ls.line_up.get(), sizeof(int) * nc, cudaMemcpyDeviceToHost));
  PMB_CUDA(cudaMemcpy(cell_pc.data(), v.cell_pc, sizeof(int) * nc, cudaMemcpyDeviceToHost));
  if (v.nperf)
    PMB_CUDA(cudaMemcpy(perf_cell.data(), v.perf_cell, sizeof(int) * v.nperf, cudaMemcpyDeviceToHost));
  std::vector<int> pos(nc);
  for (int t = 0; t < nc; ++t) pos[cells[t]] = t;
  int slots = 3;
  for (int t = 0; t < nc; ++t) {
    const int c = cells[t];
    const int others = (rp[c + 1] - rp[c]) - 1 - (lo[t] >= 0) - (up[t] >= 0);
    slots = std::max(slots, 3 + others);
  }
  if (slots > kEllMaxSlots) return;
  const long long n = nc;
  std::vector<int> src((size_t)slots * n, -1), ecol((size_t)std::max(slots - 3, 1) * n, 0), pc(nc);
  for (int t = 0; t < nc; ++t) {
    const int c = cells[t];
    int q = 0;
    for (int k = rp[c]; k < rp[c + 1]; ++k) {
      if (col[k] == c) {
        src[t] = k;
      } else if (k == lo[t]) {
        src[n + t] = k;
      } else if (k == up[t]) {
        src[2 * n + t] = k;
      } else {
        src[(3 + q) * n + t] = k;
        ecol[q * n + t] = pos[col[k]];
        ++q;
      }
    }
    PMB_REQUIRE(src[t] >= 0, "a cell's block row has no diagonal block");
    for (; q < slots - 3; ++q) ecol[q * n + t] = t;
    pc[t] = cell_pc[c];
  }
  std::vector<int> perf_pos(std::max(v.nperf, 1), 0);
  for (int i = 0; i < v.nperf; ++i) perf_pos[i] = pos[perf_cell[i]];
  ell_.slots = slots;
  ell_.src.upload(src, s_);
  ell_.col.upload(ecol, s_);
  ell_.pc.upload(pc, s_);
  ell_.perf_pos.upload(perf_pos, s_);
  if (f32_)
    ell_.blk32.resize(4LL * slots * n);
  else
    ell_.blk64.resize(4LL * slots * n);
  if (f32_) {
    ell_.rl32.resize(2 * n);
    ell_.zl32.resize(2 * n);
  } else {
    ell_.rl.resize(2 * n);
    ell_.zl.resize(2 * n);
  }
  use_ell_ = true;
}

// The second stage's copy of the Jacobian: the line-ordered blocks, or the
// FP32 block-CSR for the line kernels of mixed precision.
void CPRSolver::prepare_local(const double* jac) {
  const long long nnzb = m_.nnzb();
  if (use_ell_) {
    const long long n = (long long)ell_.slots * m_.nc();
    if (f32_)
      ell_gather_kernel<<<grid_for(n, 256), 256, 0, s_>>>(n, ell_.src.get(), reinterpret_cast<const double4*>(jac),
                                                          reinterpret_cast<float4*>(ell_.blk32.get()));
    else
      ell_gather_kernel<<<grid_for(n, 256), 256, 0, s_>>>(n, ell_.src.get(), reinterpret_cast<const double4*>(jac),
                                                          reinterpret_cast<double4*>(ell_.blk64.get()));
    PMB_CHECK_LAUNCH();
  } else if (f32_ && m_.has_lines()) {
    to_f32_kernel<<<grid_for(4 * nnzb, 256), 256, 0, s_>>>(4 * nnzb, jac, jac32_.get());
    PMB_CHECK_LAUNCH();
  }
}

void CPRSolver::pressure_values(double* ext) {
  const OWView v = m_.view();
  const long long nnzb = m_.nnzb();
  ext_cells_kernel<<<grid_for(nnzb, 256), 256, 0, s_>>>(nnzb, reinterpret_cast<const double4*>(jac_), w_.get(),
                                                         bsr2ext_.get(), ext);
  PMB_CHECK_LAUNCH();
  if (ext_par_)
    ext_wells_par_kernel<<<grid_for(std::max(v.nperf, v.nw), 128), 128, 0, s_>>>(
        v, well_, w_.get(), perf_cw_.get(), perf_wc_.get(), well_diag_.get(), ext, g_perf_.get(), a_well_.get());
  else
    ext_wells_kernel<<<1, 128, 0, s_>>>(v, well_, w_.get(), perf_cw_.get(), perf_wc_.get(), well_diag_.get(), ext,
                                      g_perf_.get(), a_well_.get());
  PMB_CHECK_LAUNCH();
}

void CPRSolver::check_status() {
  PMB_CUDA(cudaMemcpyAsync(st_pin_.get(), status_.get(), sizeof(int), cudaMemcpyDeviceToHost, s_));
  PMB_CUDA(cudaStreamSynchronize(s_));
  if (st_pin_[0] != 0) {
    const int code = st_pin_[0];
    st_pin_[0] = 0;
    PMB_CUDA(cudaMemsetAsync(status_.get(), 0, sizeof(int), s_));
    throw Error(code, code == PMB_ERR_PIVOT ? "zero pivot in the CPR preconditioner"
                                            : "device error in the CPR preconditioner");
  }
}

void CPRSolver::setup(const double* jac, const double* well, const double* x) {
  jac_ = jac;
  well_ = well;
  const OWView v = m_.view();
  ++setups_;
  {
    PhaseTimer pt("cpr.setup.local", s_);
    prepare_local(jac);
  }
  if (!o_.use_pressure_stage) return;
  PhaseTimer pt_values("cpr.setup.weights_values", s_);
  psum_kernel<<<kRedBlocks, 256, 0, s_>>>(v.nc, reinterpret_cast<const double2*>(x), part_.get());
  PMB_CHECK_LAUNCH();
  weights_kernel<<<1, 32, 0, s_>>>(v, kRedBlocks, part_.get(), w_.get());
  PMB_CHECK_LAUNCH();
  const long long nnzb = m_.nnzb();
  const bool with_wells = np_ > v.nc;
  auto values = [&](double* dst) {
    if (with_wells) {
      pressure_values(dst);
    } else {
      ap_kernel<<<grid_for(nnzb, 256), 256, 0, s_>>>(nnzb, reinterpret_cast<const double4*>(jac), w_.get(), dst);
      PMB_CHECK_LAUNCH();
    }
  };
  const bool built = f32_ ? amg32_.built() : amg_.built();
  const bool rebuild = !built || since_build_ >= std::max(1, o_.amg_rebuild_interval);
  auto build = [&](auto& amg) {
    if (with_wells)
      amg.build(np_, h_erp_, h_ecol_, erp_.get(), ecol_.get(), h_ap_, o_.amg_theta,
                std::max(16, o_.amg_coarse_size), s_);
    else
      amg.build(v.nc, m_.h_row_ptr(), m_.h_col(), v.row_ptr, v.col, h_ap_, o_.amg_theta,
                std::max(16, o_.amg_coarse_size), s_);
  };
  if (rebuild || f32_) values(ap_.get());
  if (rebuild) {
    PhaseTimer pt("cpr.setup.aggregate", s_);
    const size_t nnz = ap_.size();
    h_ap_.resize(nnz);
    PMB_CUDA(cudaMemcpyAsync(h_ap_.data(), ap_.get(), sizeof(double) * nnz, cudaMemcpyDeviceToHost, s_));
    PMB_CUDA(cudaStreamSynchronize(s_));
    if (f32_)
      build(amg32_);
    else
      build(amg_);
    since_build_ = 0;
    graph_.invalidate();  // the hierarchy's buffers are new
  }
  PhaseTimer pt("cpr.setup.refresh", s_);
  if (f32_) {
    const long long nnz = (long long)ap_.size();
    to_f32_kernel<<<grid_for(nnz, 256), 256, 0, s_>>>(nnz, ap_.get(), amg32_.level0_val());
    PMB_CHECK_LAUNCH();
    amg32_.refresh(s_, status_.get());
  } else {
    values(amg_.level0_val());
    amg_.refresh(s_, status_.get());
  }
  ++since_build_;
}

template <class T>
void CPRSolver::enter_lines(const T* xp, const double* r, double* z, bool from_z, bool pw) {
  const OWView v = m_.view();
  const int g = grid_for(std::max(v.nc, v.nw), 256);
  if (f32_)
    line_enter_kernel<T, float><<<g, 256, 0, s_>>>(v.nc, v.nw, from_z, pw, m_.lines().line_cells.get(), xp, r, z,
                                                    ell_.rl32.get(), ell_.zl32.get());
  else
    line_enter_kernel<T, double><<<g, 256, 0, s_>>>(v.nc, v.nw, from_z, pw, m_.lines().line_cells.get(), xp, r, z,
                                                     ell_.rl.get(), ell_.zl.get());
  PMB_CHECK_LAUNCH();
}

void CPRSolver::local_stage(const double* r, double* z, bool entered) {
  const OWView v = m_.view();
  const auto& cp = m_.h_color_ptr();
  const double4* A = reinterpret_cast<const double4*>(jac_);
  if (use_ell_) {
    const auto& Ls = m_.lines();
    if (!entered) enter_lines((const double*)nullptr, r, z, true, false);
    const int nb = std::max(32, (Ls.max_len + 31) / 32 * 32);
    const int sweeps = std::max(1, o_.local_sweeps);
    for (int sweep = 0; sweep < sweeps; ++sweep) {
      const bool out = sweep + 1 == sweeps;
      for (int q = 0; q + 1 < (int)Ls.h_color_ptr.size(); ++q) {
        const int cnt = Ls.h_color_ptr[q + 1] - Ls.h_color_ptr[q];
        if (cnt <= 0) continue;
        auto go = [&](auto kernel, auto* blk, size_t smem, auto* rl, auto* zl) {
          launch_pdl(kernel, cnt, nb, (size_t)nb * smem, s_, v, Ls.h_color_ptr[q], Ls.color_range.get(),
                     Ls.line_cells.get(), ell_.slots, blk, ell_.col.get(), ell_.pc.get(), well_, rl, zl, z,
                     status_.get());
        };
        const size_t smem32 = 3 * sizeof(Blk2<float>) + sizeof(Vec2<float>);
        const size_t smem64 = 3 * sizeof(Blk2<double>) + sizeof(Vec2<double>);
        const float4* b32 = reinterpret_cast<const float4*>(ell_.blk32.get());
        const double4* b64 = reinterpret_cast<const double4*>(ell_.blk64.get());
        float* rl32 = ell_.rl32.get();
        float* zl32 = ell_.zl32.get();
        double* rl64 = ell_.rl.get();
        double* zl64 = ell_.zl.get();
        if (f32_)
          out ? go(line_pcr_ell_kernel<float4, float, true, float>, b32, smem32, rl32, zl32)
              : go(line_pcr_ell_kernel<float4, float, false, float>, b32, smem32, rl32, zl32);
        else
          out ? go(line_pcr_ell_kernel<double4, double, true, double>, b64, smem64, rl64, zl64)
              : go(line_pcr_ell_kernel<double4, double, false, double>, b64, smem64, rl64, zl64);
      }
      if (v.nw) {
        if (f32_)
          launch_pdl(gs_well_kernel<float>, 1, 256, 0, s_, v, well_, r, z, (const float*)ell_.zl32.get(),
                     (const int*)ell_.perf_pos.get());
        else
          launch_pdl(gs_well_kernel<double>, 1, 256, 0, s_, v, well_, r, z, (const double*)ell_.zl.get(),
                     (const int*)ell_.perf_pos.get());
      }
    }
    return;
  }
  if (m_.has_lines()) {
    const auto& Ls = m_.lines();
    for (int sweep = 0; sweep < std::max(1, o_.local_sweeps); ++sweep) {
      for (int q = 0; q + 1 < (int)Ls.h_color_ptr.size(); ++q) {
        const int cnt = Ls.h_color_ptr[q + 1] - Ls.h_color_ptr[q];
        if (cnt <= 0) continue;
        if (Ls.max_len <= kPcrMaxLen) {
          const int nb = std::max(32, (Ls.max_len + 31) / 32 * 32);
          if (f32_)
            line_pcr_kernel<float4, float><<<cnt, nb, (size_t)nb * (3 * sizeof(Blk2<float>) + sizeof(Vec2<float>)),
                                             s_>>>(v, Ls.h_color_ptr[q], Ls.color_lines.get(), Ls.line_ptr.get(),
                                                   Ls.line_cells.get(), Ls.line_lo.get(), Ls.line_up.get(),
                                                   reinterpret_cast<const float4*>(jac32_.get()), well_, r, z,
                                                   status_.get());
          else
            line_pcr_kernel<double4, double>
                <<<cnt, nb, (size_t)nb * (3 * sizeof(Blk2<double>) + sizeof(Vec2<double>)), s_>>>(
                    v, Ls.h_color_ptr[q], Ls.color_lines.get(), Ls.line_ptr.get(), Ls.line_cells.get(),
                    Ls.line_lo.get(), Ls.line_up.get(), A, well_, r, z, status_.get());
          PMB_CHECK_LAUNCH();
          continue;
        }
        if (f32_)
          line_gs_kernel<<<grid_for(32LL * cnt, 32 * kLineWarps), 32 * kLineWarps, 0, s_>>>(
              v, Ls.h_color_ptr[q], Ls.h_color_ptr[q + 1], Ls.color_lines.get(), Ls.line_ptr.get(),
              Ls.line_cells.get(), Ls.line_lo.get(), Ls.line_up.get(),
              reinterpret_cast<const float4*>(jac32_.get()), well_, r, z,
              reinterpret_cast<double2*>(line_y_.get()), reinterpret_cast<double4*>(line_g_.get()), status_.get());
        else
          line_gs_kernel<<<grid_for(32LL * cnt, 32 * kLineWarps), 32 * kLineWarps, 0, s_>>>(
              v, Ls.h_color_ptr[q], Ls.h_color_ptr[q + 1], Ls.color_lines.get(), Ls.line_ptr.get(),
              Ls.line_cells.get(), Ls.line_lo.get(), Ls.line_up.get(), A, well_, r, z,
              reinterpret_cast<double2*>(line_y_.get()), reinterpret_cast<double4*>(line_g_.get()), status_.get());
        PMB_CHECK_LAUNCH();
      }
      if (v.nw) {
        gs_well_kernel<double><<<1, 256, 0, s_>>>(v, well_, r, z, z, nullptr);
        PMB_CHECK_LAUNCH();
      }
    }
    return;
  }
  for (int sweep = 0; sweep < std::max(1, o_.local_sweeps); ++sweep) {
    for (int q = 0; q + 1 < (int)cp.size(); ++q) {
      const int cnt = cp[q + 1] - cp[q];
      if (cnt <= 0) continue;
      gs_color_kernel<<<grid_for(cnt, 256), 256, 0, s_>>>(v, cp[q], cp[q + 1], m_.color_cells(), A, well_, r, z,
                                                          status_.get());
      PMB_CHECK_LAUNCH();
    }
    if (v.nw) {
      gs_well_kernel<double><<<1, 256, 0, s_>>>(v, well_, r, z, z, nullptr);
      PMB_CHECK_LAUNCH();
    }
  }
}

void CPRSolver::precond(const double* r, double* z) {
  // the graph holds the operator's buffer addresses: re-capture when they move
  if (pg_jac_ != jac_ || pg_well_ != well_) {
    graph_.invalidate();
    pg_jac_ = jac_;
    pg_well_ = well_;
  }
  graph_.run(m_.nvec(), r, z, s_, [this](const double* a, double* b) { precond_body(a, b); });
}

void CPRSolver::precond_body(const double* r, double* z) {
  const OWView v = m_.view();
  const int gpro = grid_for(std::max<long long>(v.nc, 3LL * v.nw), 256);
  auto pressure_stage = [&](auto* bp, auto* xp, auto& amg) {
    restrict_p_kernel<<<grid_for(v.nc, 256), 256, 0, s_>>>(v.nc, reinterpret_cast<const double2*>(r), w_.get(),
                                                           bp);
    PMB_CHECK_LAUNCH();
    if (np_ > v.nc) {
      restrict_wells_kernel<<<1, 256, 0, s_>>>(v, r, g_perf_.get(), a_well_.get(), bp);
      PMB_CHECK_LAUNCH();
    }
    {
      PhaseTimer pt("cpr.amg_cycle", s_);
      amg.apply(bp, xp, s_);
    }
    if (use_ell_) {
      // prolongation straight into line order, with r
      enter_lines(xp, r, z, false, np_ > v.nc);
    } else if (np_ > v.nc) {
      prolong_pw_kernel<<<gpro, 256, 0, s_>>>(v.nc, v.nw, xp, z);
    } else {
      prolong_p_kernel<<<gpro, 256, 0, s_>>>(v.nc, 3 * v.nw, xp, z);
    }
    PMB_CHECK_LAUNCH();
  };
  if (o_.use_pressure_stage) {
    if (f32_)
      pressure_stage(bp32_.get(), xp32_.get(), amg32_);
    else
      pressure_stage(bp_.get(), xp_.get(), amg_);
  } else if (use_ell_) {
    enter_lines((const double*)nullptr, r, z, false, false);
  } else {
    prolong_p_kernel<double><<<gpro, 256, 0, s_>>>(v.nc, 3 * v.nw, nullptr, z);
    PMB_CHECK_LAUNCH();
  }
  PhaseTimer pt("cpr.local_stage", s_);
  local_stage(r, z, use_ell_);
}

double CPRSolver::time_stage(int stage, const double* r, double* z, int reps) {
  PMB_REQUIRE(jac_ != nullptr, "pmb_cpr_setup must run before timing a stage");
  PMB_REQUIRE(stage != 1 || o_.use_pressure_stage, "the pressure stage is switched off");
  const OWView v = m_.view();
  auto amg_once = [&]() {
    if (f32_)
      amg32_.apply(bp32_.get(), xp32_.get(), s_);
    else
      amg_.apply(bp_.get(), xp_.get(), s_);
  };
  if (stage == 1) {
    if (f32_)
      restrict_p_kernel<<<grid_for(v.nc, 256), 256, 0, s_>>>(v.nc, reinterpret_cast<const double2*>(r), w_.get(),
                                                             bp32_.get());
    else
      restrict_p_kernel<<<grid_for(v.nc, 256), 256, 0, s_>>>(v.nc, reinterpret_cast<const double2*>(r), w_.get(),
                                                             bp_.get());
    PMB_CHECK_LAUNCH();
  }
  auto once = [&]() {
    if (stage == 0) local_stage(r, z);
    else if (stage == 1) amg_once();
    else if (stage == 2) precond_body(r, z);
    else precond(r, z);  // as the solver applies it (graph replay)
  };
  once();
  cudaEvent_t e0, e1;
  PMB_CUDA(cudaEventCreate(&e0));
  PMB_CUDA(cudaEventCreate(&e1));
  PMB_CUDA(cudaEventRecord(e0, s_));
  for (int i = 0; i < reps; ++i) once();
  PMB_CUDA(cudaEventRecord(e1, s_));
  PMB_CUDA(cudaEventSynchronize(e1));
  float ms = 0.f;
  PMB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  check_status();
  return ms / reps;
}

void CPRSolver::bytes(double* out) const {
  const double nc = m_.nc(), nnzb = (double)m_.nnzb(), nvec = (double)m_.nvec();
  const double vb = f32_ ? 4.0 : 8.0, blk = 4.0 * vb;
  for (int i = 0; i < 8; ++i) out[i] = 0.0;
  out[0] = o_.use_pressure_stage ? (f32_ ? amg32_.cycle_bytes() : amg_.cycle_bytes()) : 0.0;
  // one sweep of the second stage (both colours and the well update): every
  // block once, the index of every block off the line (the line-ordered copy
  // needs none for the diagonal and the two line couplings; the block-CSR one
  // per block plus row pointers), r, z read and written, perforation index
  // (the line-ordered r and z are FP32 in mixed precision)
  const double lv = f32_ ? 8.0 : 16.0;
  out[1] = use_ell_ ? nnzb * blk + std::max(nnzb - 3.0 * nc, 0.0) * 4.0 + nc * (lv + 2.0 * lv + 4.0)
                    : nnzb * (blk + 4.0) + (nc + 1.0) * 4.0 + nc * (16.0 + 32.0 + 4.0);
  // y = J x: blocks, column indices, row pointers, x read, y written
  out[2] = nnzb * 36.0 + (nc + 1.0) * 4.0 + nvec * 16.0;
  // restriction (r read, weights, pressure right-hand side written) and the
  // prolongation into line order (pressure correction, r, the line's cell
  // index read; r and z in line order written)
  out[3] = o_.use_pressure_stage
               ? nc * (16.0 + vb) + nc * (vb + 16.0 + 4.0 + (use_ell_ ? 2.0 * lv : 32.0))
               : 0.0;
  // setup: the second stage's copy of the Jacobian (gather index, FP64 block
  // read, block written), the weights (pressures read), the pressure values
  // (blocks read, values written), FP32 conversion of level 0
  double setup = use_ell_ ? (double)ell_.slots * nc * (4.0 + 32.0 + blk) : (f32_ ? nnzb * (32.0 + 16.0) : 0.0);
  if (o_.use_pressure_stage) {
    setup += nc * 16.0 + nnzb * (32.0 + 4.0 + 8.0);
    if (f32_) setup += (double)ap_.size() * (8.0 + 4.0);
  }
  out[4] = setup;
  out[5] = nvec;
  out[6] = o_.use_pressure_stage ? (f32_ ? amg32_.refresh_bytes() : amg_.refresh_bytes()) : 0.0;
}

bool CPRSolver::solve(const double* b, double* x, double* info) {
  PMB_REQUIRE(jac_ != nullptr, "pmb_cpr_setup must run before pmb_cpr_solve");
  auto op = [this](const double* in, double* out) {
    PhaseTimer pt("gmres.spmv", s_);
    m_.spmv(jac_, well_, in, out);
  };
  auto pc = [this](const double* in, double* out) { precond(in, out); };
  const bool ok = kry_.solve(op, pc, b, x, o_.rtol, o_.maxiter, info, status_.get(), [this] { check_status(); });
  total_its_ += (long long)info[0];
  info[3] = (double)setups_;
  return ok;
}

}  // namespace pmb
