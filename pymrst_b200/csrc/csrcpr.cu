// CPR-preconditioned FGMRES on a caller's CSR matrix: the drop-in for
// CPRSolver.solve(jac, rhs, model, state)
// (pymrst/modules/ad_core/solvers/linear_solvers.py:426-545).
//
// The matrix is in the reference's variable-blocked ordering: rows and
// columns [var_0 of all nc cells, var_1 of all cells, ..., var_{nph-1},
// then nt facility (well) unknowns].  Nothing is permuted: the kernels index
// the blocks in place.  The preconditioner is the reference's two-stage form
//   x = P solve_p(W r);  z = x + local(r - A x)         (:510-517)
// with W the caller's per-phase weights (1/b_i at the mean pressure,
// :155-190), P the injection of the first nc columns (pressure), solve_p an
// aggregation-AMG cycle on A_p = W A P (:471-473), and local() the
// block-Jacobi stage (:316-363): each cell's nph x nph block inverted, the
// facility block inverted group by group, a group being a connected component
// of the facility block's own pattern (a well's unknowns, where wells do not
// couple one another), each regularised by sqrt(eps) where it is exactly
// singular, as the reference does after equilibration, :345-357).
// In transposed mode the caller passes A' = J^T (the adjoint system,
// optimization/adjoint.py:209) and the transfer operators are the
// transposes of the forward ones: restriction P^T (the pressure rows of r),
// prolongation W^T (x[i*nc + c] = w_i xp[c]), so that the pressure matrix is
// P^T J^T W^T = (W J P)^T.
// The Ruiz equilibration the reference applies before its factorisations
// (:206-224) is not applied: block inverses are invariant under it, and the
// AMG's strength measure and Jacobi-scaled smoother are invariant under the
// row scaling of A_p.
#include <algorithm>
#include <cmath>
#include <functional>
#include <memory>
#include <numeric>
#include <type_traits>
#include <vector>

#include "pmb_amg.cuh"
#include "pmb_krylov.cuh"

namespace pmb {

constexpr int kMaxPhases = 3;
constexpr int kMaxTail = 4096;

// ---- kernels --------------------------------------------------------------------

// y = A x, 8 lanes per row.
__global__ void __launch_bounds__(256) csr8_spmv_kernel(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                                                        const double* __restrict__ a, const double* __restrict__ x,
                                                        double* __restrict__ y) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long row = t >> 3;
  const int sub = threadIdx.x & 7;
  double s = 0.0;
  if (row < n)
    for (int k = rp[row] + sub; k < rp[row + 1]; k += 8) s += a[k] * x[ci[k]];
  s += __shfl_xor_sync(0xffffffffu, s, 4);
  s += __shfl_xor_sync(0xffffffffu, s, 2);
  s += __shfl_xor_sync(0xffffffffu, s, 1);
  if (row < n && sub == 0) y[row] = s;
}

// A_p values: ap[e] = sum over the entry's sources of w[phase] * A[pos].
template <class T>
__global__ void csr_pressure_values_kernel(int nnz, const int* __restrict__ gptr, const int* __restrict__ gsrc,
                                           const unsigned char* __restrict__ gph, const double* __restrict__ a,
                                           const double* __restrict__ w, T* __restrict__ ap) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int k = gptr[e]; k < gptr[e + 1]; ++k) s += w[gph[k]] * a[gsrc[k]];
    ap[e] = (T)s;
  }
}

// Inverse of each cell's nph x nph block (Gauss-Jordan with partial pivoting
// in registers).  blk_pos[c * nph^2 + i * nph + j] is the CSR position of
// (row i*nc+c, column j*nc+c), or -1 for a structural zero.
__global__ void csr_block_inv_kernel(int nc, int nph, const int* __restrict__ blk_pos, const double* __restrict__ a,
                                     double* __restrict__ inv, int* __restrict__ status) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  double M[kMaxPhases][kMaxPhases], I[kMaxPhases][kMaxPhases];
  const int m2 = nph * nph;
  for (int i = 0; i < nph; ++i)
    for (int j = 0; j < nph; ++j) {
      const int p = blk_pos[(long long)c * m2 + i * nph + j];
      M[i][j] = p >= 0 ? a[p] : 0.0;
      I[i][j] = i == j ? 1.0 : 0.0;
    }
  bool ok = true;
  for (int k = 0; k < nph; ++k) {
    int p = k;
    for (int i = k + 1; i < nph; ++i)
      if (fabs(M[i][k]) > fabs(M[p][k])) p = i;
    if (!(fabs(M[p][k]) > 0.0) || !isfinite(M[p][k])) { ok = false; break; }
    if (p != k)
      for (int j = 0; j < nph; ++j) {
        double t = M[k][j]; M[k][j] = M[p][j]; M[p][j] = t;
        t = I[k][j]; I[k][j] = I[p][j]; I[p][j] = t;
      }
    const double d = 1.0 / M[k][k];
    for (int j = 0; j < nph; ++j) { M[k][j] *= d; I[k][j] *= d; }
    for (int i = 0; i < nph; ++i) {
      if (i == k) continue;
      const double f = M[i][k];
      for (int j = 0; j < nph; ++j) { M[i][j] -= f * M[k][j]; I[i][j] -= f * I[k][j]; }
    }
  }
  if (!ok) atomicExch(status, PMB_ERR_PIVOT);
  for (int i = 0; i < nph; ++i)
    for (int j = 0; j < nph; ++j) inv[(long long)c * m2 + i * nph + j] = ok ? I[i][j] : 0.0;
}

// Facility block.  Its unknowns fall into independent groups (the connected
// components of its own pattern: one group per well when wells do not couple
// one another); group g has m_g unknowns, listed ascending at
// gmem[gptr[g] ..), and a dense m_g x m_g block at goff[g] in tM / tInv.
__global__ void csr_tail_zero_kernel(long long n, double* __restrict__ M) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
    M[e] = 0.0;
}

__global__ void csr_tail_scatter_kernel(int cnt, const int* __restrict__ pos, const long long* __restrict__ dst,
                                        const double* __restrict__ a, double* __restrict__ M) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < cnt; e += gridDim.x * blockDim.x) M[dst[e]] = a[pos[e]];
}

// One CTA per group: scale each row of the group's block to unit max norm
// (rs = 1 / max|row|), Gauss-Jordan inverse with row pivoting, an exactly
// zero pivot column replaced by sqrt(eps) on the diagonal, and finally
// Inv <- Inv diag(rs), the inverse of the unscaled block.
__global__ void __launch_bounds__(128) csr_tail_invert_kernel(const int* __restrict__ gptr,
                                                              const long long* __restrict__ goff,
                                                              double* __restrict__ Mall, double* __restrict__ Invall,
                                                              double* __restrict__ rsall, int* __restrict__ status) {
  __shared__ int piv;
  __shared__ double pval;
  const int g = blockIdx.x;
  const int nt = gptr[g + 1] - gptr[g];
  double* M = Mall + goff[g];
  double* Inv = Invall + goff[g];
  double* rs = rsall + gptr[g];
  const int t = threadIdx.x, nthr = blockDim.x;
  const double shift = 1.4901161193847656e-08;  // sqrt(2^-52)
  for (int r = t; r < nt; r += nthr) {
    double m = 0.0;
    for (int j = 0; j < nt; ++j) m = fmax(m, fabs(M[(long long)r * nt + j]));
    const double sc = m > 0.0 && isfinite(m) ? 1.0 / m : 1.0;
    rs[r] = sc;
    for (int j = 0; j < nt; ++j) M[(long long)r * nt + j] *= sc;
  }
  for (int idx = t; idx < nt * nt; idx += nthr) Inv[idx] = (idx / nt == idx % nt) ? 1.0 : 0.0;
  __syncthreads();
  for (int c = 0; c < nt; ++c) {
    if (t == 0) {
      int p = c;
      double best = fabs(M[(long long)c * nt + c]);
      for (int r = c + 1; r < nt; ++r) {
        const double v = fabs(M[(long long)r * nt + c]);
        if (v > best) { best = v; p = r; }
      }
      if (!isfinite(best)) atomicExch(status, PMB_ERR_NONFINITE);
      if (best == 0.0) {
        p = c;
        M[(long long)c * nt + c] = shift;
      }
      piv = p;
      pval = M[(long long)p * nt + c];
    }
    __syncthreads();
    const int p = piv;
    const double pv = isfinite(pval) && pval != 0.0 ? pval : 1.0;
    if (p != c) {
      for (int j = t; j < nt; j += nthr) {
        double a = M[(long long)c * nt + j];
        M[(long long)c * nt + j] = M[(long long)p * nt + j];
        M[(long long)p * nt + j] = a;
        a = Inv[(long long)c * nt + j];
        Inv[(long long)c * nt + j] = Inv[(long long)p * nt + j];
        Inv[(long long)p * nt + j] = a;
      }
    }
    __syncthreads();
    for (int j = t; j < nt; j += nthr) {
      M[(long long)c * nt + j] /= pv;
      Inv[(long long)c * nt + j] /= pv;
    }
    __syncthreads();
    for (long long idx = t; idx < (long long)nt * nt; idx += nthr) {
      const int r = (int)(idx / nt), j = (int)(idx % nt);
      if (r == c || j == c) continue;
      const double f = M[(long long)r * nt + c];
      M[idx] -= f * M[(long long)c * nt + j];
      Inv[idx] -= f * Inv[(long long)c * nt + j];
    }
    __syncthreads();
    for (int r = t; r < nt; r += nthr) {
      if (r == c) continue;
      const double f = M[(long long)r * nt + c];
      Inv[(long long)r * nt + c] -= f * Inv[(long long)c * nt + c];
      M[(long long)r * nt + c] = 0.0;
    }
    __syncthreads();
  }
  for (long long idx = t; idx < (long long)nt * nt; idx += nthr) Inv[idx] *= rs[idx % nt];
}

// bp[c] = sum_i rw[i] r[i*nc + c]  (rw = w, or (1, 0, ..) when transposed)
template <class T>
__global__ void csr_restrict_kernel(int nc, int nph, const double* __restrict__ r, const double* __restrict__ rw,
                                    T* __restrict__ bp) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  double s = 0.0;
  for (int i = 0; i < nph; ++i) s += rw[i] * r[(long long)i * nc + c];
  bp[c] = (T)s;
}

// Per-cell decoupling weights: row 0 of the inverse of the cell's diagonal
// block, so that the weighted sum of the cell's rows has a unit derivative
// with respect to its own pressure and none with respect to its other
// unknowns (true-IMPES on the full diagonal block).
__global__ void csr_cell_weights_kernel(int nc, int nph, const double* __restrict__ inv, double* __restrict__ wc) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  for (int j = 0; j < nph; ++j) wc[(long long)c * nph + j] = inv[(long long)c * nph * nph + j];
}

// A_p values with per-cell weights: row c sums w_c[phase] * A over the
// sources of each of its entries.
template <class T>
__global__ void csr_pressure_values_cell_kernel(int nc, int nph, const int* __restrict__ prp,
                                                const int* __restrict__ gptr, const int* __restrict__ gsrc,
                                                const unsigned char* __restrict__ gph, const double* __restrict__ a,
                                                const double* __restrict__ wc, T* __restrict__ ap) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  const double* w = wc + (long long)c * nph;
  for (int e = prp[c]; e < prp[c + 1]; ++e) {
    double s = 0.0;
    for (int k = gptr[e]; k < gptr[e + 1]; ++k) s += w[gph[k]] * a[gsrc[k]];
    ap[e] = (T)s;
  }
}

// bp[c] = sum_i w_c[i] r[i*nc + c]
template <class T>
__global__ void csr_restrict_cell_kernel(int nc, int nph, const double* __restrict__ r, const double* __restrict__ wc,
                                         T* __restrict__ bp) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  double s = 0.0;
  for (int i = 0; i < nph; ++i) s += wc[(long long)c * nph + i] * r[(long long)i * nc + c];
  bp[c] = (T)s;
}

// x = Q xp evaluated at column j: the injection into the pressure block
// (Q = P), or the weighted spread into every cell block (Q = W^T).
template <bool TR, class T>
__device__ __forceinline__ double prolonged(int j, int nc, int nph, const T* __restrict__ xp,
                                            const double* __restrict__ pw) {
  if (!TR) return j < nc ? (double)xp[j] : 0.0;
  if (j >= nph * nc) return 0.0;
  const int blk = j / nc;
  return pw[blk] * (double)xp[j - blk * nc];
}

// Cell rows of the second stage in one pass: with x = Q xp (zero when xp is
// null), t_i = r_i - (A x)_i for the cell's nph rows, then
// z_i = x_i + inv_c t.
template <bool TR, class T>
__global__ void __launch_bounds__(256) csr_local_cells_kernel(int nc, int nph, const int* __restrict__ rp,
                                                              const int* __restrict__ ci,
                                                              const double* __restrict__ a,
                                                              const double* __restrict__ r,
                                                              const T* __restrict__ xp,
                                                              const double* __restrict__ pw,
                                                              const double* __restrict__ inv,
                                                              double* __restrict__ z) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  double t[kMaxPhases];
  for (int i = 0; i < nph; ++i) {
    const long long row = (long long)i * nc + c;
    double s = r[row];
    if (xp)
      for (int k = rp[row]; k < rp[row + 1]; ++k) s -= a[k] * prolonged<TR>(ci[k], nc, nph, xp, pw);
    t[i] = s;
  }
  const double* B = inv + (long long)c * nph * nph;
  for (int i = 0; i < nph; ++i) {
    double s = xp ? prolonged<TR>(i * nc + c, nc, nph, xp, pw) : 0.0;
    for (int j = 0; j < nph; ++j) s += B[i * nph + j] * t[j];
    z[(long long)i * nc + c] = s;
  }
}

// Facility rows of the second stage, one CTA per facility group: t = r - A x
// over the group's rows, z = Inv_g t (x is zero there).
template <bool TR, class T>
__global__ void __launch_bounds__(128) csr_local_tail_kernel(int nc, int nph, const int* __restrict__ gptr,
                                                             const int* __restrict__ gmem,
                                                             const long long* __restrict__ goff,
                                                             const int* __restrict__ rp,
                                                             const int* __restrict__ ci,
                                                             const double* __restrict__ a,
                                                             const double* __restrict__ r,
                                                             const T* __restrict__ xp,
                                                             const double* __restrict__ pw,
                                                             const double* __restrict__ Invall,
                                                             double* __restrict__ z) {
  extern __shared__ double ts[];
  const int base = nph * nc;
  const int g = blockIdx.x, g0 = gptr[g], m = gptr[g + 1] - g0;
  const double* Inv = Invall + goff[g];
  for (int q = threadIdx.x; q < m; q += blockDim.x) {
    const int row = base + gmem[g0 + q];
    double s = r[row];
    if (xp)
      for (int k = rp[row]; k < rp[row + 1]; ++k) s -= a[k] * prolonged<TR>(ci[k], nc, nph, xp, pw);
    ts[q] = s;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < m; q += blockDim.x) {
    double s = 0.0;
    for (int j = 0; j < m; ++j) s += Inv[(long long)q * m + j] * ts[j];
    z[base + gmem[g0 + q]] = s;
  }
}

// One more block-Jacobi sweep: z += D^{-1} (r - y) with y = A z.
__global__ void __launch_bounds__(256) csr_jacobi_cells_kernel(int nc, int nph, const double* __restrict__ r,
                                                               const double* __restrict__ y,
                                                               const double* __restrict__ inv,
                                                               double* __restrict__ z) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  double t[kMaxPhases];
  for (int i = 0; i < nph; ++i) {
    const long long row = (long long)i * nc + c;
    t[i] = r[row] - y[row];
  }
  const double* B = inv + (long long)c * nph * nph;
  for (int i = 0; i < nph; ++i) {
    double s = 0.0;
    for (int j = 0; j < nph; ++j) s += B[i * nph + j] * t[j];
    z[(long long)i * nc + c] += s;
  }
}

__global__ void __launch_bounds__(128) csr_jacobi_tail_kernel(int base, const int* __restrict__ gptr,
                                                              const int* __restrict__ gmem,
                                                              const long long* __restrict__ goff,
                                                              const double* __restrict__ r,
                                                              const double* __restrict__ y,
                                                              const double* __restrict__ Invall,
                                                              double* __restrict__ z) {
  extern __shared__ double ts[];
  const int g = blockIdx.x, g0 = gptr[g], m = gptr[g + 1] - g0;
  const double* Inv = Invall + goff[g];
  for (int q = threadIdx.x; q < m; q += blockDim.x) {
    const int row = base + gmem[g0 + q];
    ts[q] = r[row] - y[row];
  }
  __syncthreads();
  for (int q = threadIdx.x; q < m; q += blockDim.x) {
    double s = 0.0;
    for (int j = 0; j < m; ++j) s += Inv[(long long)q * m + j] * ts[j];
    z[base + gmem[g0 + q]] += s;
  }
}

// ---- solver ---------------------------------------------------------------------

class CsrCPR {
 public:
  CsrCPR(int n, int nc, int nph, const int* h_rp, const int* h_col, bool transposed, const pmb_cpr_opts& o,
         cudaStream_t s);
  void setup(const double* d_val, const double* h_w);
  bool solve(const double* b, double* x, double* info);
  void spmv(const double* val, const double* x, double* y);
  // 1: per-cell weights from the diagonal blocks instead of the caller's
  // phase weights (non-transposed systems)
  void set_cell_weights(bool on) {
    PMB_REQUIRE(!on || !tr_, "per-cell weights are for the non-transposed system");
    cell_w_ = on;
    if (on) wcell_.resize((size_t)nc_ * nph_);
    since_build_ = 1 << 30;  // rebuild the hierarchy on the next setup
  }
  int num_levels() const { return f32_ ? amg32_.num_levels() : amg_.num_levels(); }
  int level_size(int l) const { return f32_ ? amg32_.level_size(l) : amg_.level_size(l); }

 private:
  void precond_body(const double* r, double* z);
  void check_status();

  int n_, nc_, nph_, nt_ = 0, nnz_ = 0;
  bool tr_ = false;
  pmb_cpr_opts o_;
  cudaStream_t s_;
  bool f32_ = false;
  const double* val_ = nullptr;
  const double* pg_val_ = nullptr;
  DArray<int> rp_, col_;
  // pressure system A_p = W A P: pattern and, per entry, its sources in A
  std::vector<int> h_prp_, h_pcol_;
  DArray<int> prp_, pcol_, gptr_, gsrc_;
  DArray<unsigned char> gph_;
  DArray<double> ap_, w_, rw_, pw_;  // weights; restriction and prolongation weights
  DArray<double> bp_, xp_;
  DArray<float> bp32_, xp32_;
  AMG<double> amg_;
  AMG<float> amg32_;
  int since_build_ = 0;
  std::vector<double> h_ap_;
  // local stage
  DArray<int> blk_pos_, tail_pos_, tg_ptr_, tg_mem_;
  DArray<long long> tail_dst_, tg_off_;
  int tail_cnt_ = 0, ngroups_ = 0, max_group_ = 0;
  long long tail_dense_ = 0;
  DArray<double> inv_, tM_, tInv_, trs_, ytmp_, wcell_;
  bool cell_w_ = false;
  DArray<int> status_;
  PinnedArray<int> st_pin_;
  PinnedArray<double> w_pin_;
  Fgmres kry_;
  GraphedApply graph_;
  long long setups_ = 0;
};

CsrCPR::CsrCPR(int n, int nc, int nph, const int* h_rp, const int* h_col, bool transposed, const pmb_cpr_opts& o,
               cudaStream_t s)
    : n_(n), nc_(nc), nph_(nph), tr_(transposed), o_(o), s_(s) {
  PMB_REQUIRE(h_rp && h_col, "row_ptr and col are required");
  PMB_REQUIRE(nph >= 1 && nph <= kMaxPhases, "nph must be 1, 2 or 3");
  PMB_REQUIRE(nc >= 1 && (long long)nph * nc <= n, "need 1 <= nc and nph * nc <= n");
  nt_ = n - nph * nc;
  PMB_REQUIRE(o_.restart >= 1 && o_.restart <= kMaxRestart, "restart must be in 1..60");
  PMB_REQUIRE(o_.maxiter >= 1, "maxiter must be positive");
  PMB_REQUIRE(o_.rtol > 0.0, "rtol must be positive");
  PMB_REQUIRE(o_.precision == 0 || o_.precision == 1, "precision must be 0 (FP64) or 1 (FP32 preconditioner)");
  f32_ = o_.precision == 1;
  graph_.enabled = o_.replay_graph != 0;
  PMB_REQUIRE(h_rp[0] == 0, "row_ptr[0] must be 0");
  for (int i = 0; i < n; ++i) {
    PMB_REQUIRE(h_rp[i + 1] >= h_rp[i], "row_ptr must be non-decreasing");
    for (int k = h_rp[i]; k < h_rp[i + 1]; ++k) {
      PMB_REQUIRE(h_col[k] >= 0 && h_col[k] < n, "column index out of range");
      PMB_REQUIRE(k == h_rp[i] || h_col[k] > h_col[k - 1],
                  "columns must be strictly increasing within a row (canonical CSR)");
    }
  }
  nnz_ = h_rp[n];
  auto find = [&](int row, int c) -> int {
    const int* b = h_col + h_rp[row];
    const int* e = h_col + h_rp[row + 1];
    const int* it = std::lower_bound(b, e, c);
    return (it != e && *it == c) ? (int)(it - h_col) : -1;
  };
  // pressure pattern: union of the pressure columns of a cell's nph rows
  h_prp_.assign(nc + 1, 0);
  std::vector<int> gptr(1, 0), gsrc;
  std::vector<unsigned char> gph;
  std::vector<std::pair<int, std::pair<int, int>>> ent;  // (column, (position, phase))
  for (int c = 0; c < nc; ++c) {
    ent.clear();
    if (!tr_) {
      // W A P: the pressure columns of the cell's nph rows, weighted by row phase
      for (int i = 0; i < nph; ++i) {
        const int row = i * nc + c;
        for (int k = h_rp[row]; k < h_rp[row + 1] && h_col[k] < nc; ++k) ent.push_back({h_col[k], {k, i}});
      }
    } else {
      // P^T A' W^T: the cell's pressure row, every cell column, weighted by column phase
      for (int k = h_rp[c]; k < h_rp[c + 1] && h_col[k] < nph * nc; ++k)
        ent.push_back({h_col[k] % nc, {k, h_col[k] / nc}});
    }
    ent.push_back({c, {-1, 0}});  // the diagonal is always in the pattern
    std::sort(ent.begin(), ent.end());
    for (size_t q = 0; q < ent.size();) {
      const int cc = ent[q].first;
      h_pcol_.push_back(cc);
      for (; q < ent.size() && ent[q].first == cc; ++q)
        if (ent[q].second.first >= 0) {
          gsrc.push_back(ent[q].second.first);
          gph.push_back((unsigned char)ent[q].second.second);
        }
      gptr.push_back((int)gsrc.size());
    }
    h_prp_[c + 1] = (int)h_pcol_.size();
  }
  std::vector<int> blk((size_t)nc * nph * nph);
  for (int c = 0; c < nc; ++c)
    for (int i = 0; i < nph; ++i)
      for (int j = 0; j < nph; ++j) blk[(size_t)c * nph * nph + i * nph + j] = find(i * nc + c, j * nc + c);
  // facility groups: connected components of the facility-facility pattern
  std::vector<int> tp, tgp(1, 0), tgm;
  std::vector<long long> tdst, tgo(1, 0);
  if (nt_ > 0) {
    const int base = nph * nc;
    std::vector<int> parent(nt_);
    std::iota(parent.begin(), parent.end(), 0);
    std::function<int(int)> root = [&](int q) {
      while (parent[q] != q) q = parent[q] = parent[parent[q]];
      return q;
    };
    for (int q = 0; q < nt_; ++q)
      for (int k = h_rp[base + q]; k < h_rp[base + q + 1]; ++k)
        if (h_col[k] >= base) {
          const int a = root(q), b = root(h_col[k] - base);
          if (a != b) parent[std::max(a, b)] = std::min(a, b);
        }
    std::vector<int> gid(nt_, -1), lid(nt_), gsize;
    std::vector<int> rid(nt_, -1);
    for (int q = 0; q < nt_; ++q) {
      const int r0 = root(q);
      if (rid[r0] < 0) {
        rid[r0] = (int)gsize.size();
        gsize.push_back(0);
      }
      gid[q] = rid[r0];
      lid[q] = gsize[gid[q]]++;
    }
    ngroups_ = (int)gsize.size();
    std::vector<int> fill(ngroups_, 0);
    for (int g = 0; g < ngroups_; ++g) {
      tgp.push_back(tgp.back() + gsize[g]);
      tgo.push_back(tgo.back() + (long long)gsize[g] * gsize[g]);
      max_group_ = std::max(max_group_, gsize[g]);
    }
    tgm.assign(nt_, 0);
    for (int q = 0; q < nt_; ++q) tgm[tgp[gid[q]] + fill[gid[q]]++] = q;  // ascending within a group
    for (int q = 0; q < nt_; ++q)
      for (int k = h_rp[base + q]; k < h_rp[base + q + 1]; ++k)
        if (h_col[k] >= base) {
          const int j = h_col[k] - base, g = gid[q];
          tp.push_back(k);
          tdst.push_back(tgo[g] + (long long)lid[q] * gsize[g] + lid[j]);
        }
    tail_dense_ = tgo.back();
    PMB_REQUIRE(max_group_ <= kMaxTail, "at most 4096 coupled facility unknowns in one group");
  }
  // device arrays (everything above is host-only validation and analysis)
  rp_.upload(h_rp, n + 1, s_);
  col_.upload(h_col, std::max(nnz_, 1), s_);
  prp_.upload(h_prp_, s_);
  pcol_.upload(h_pcol_, s_);
  gptr_.upload(gptr, s_);
  gsrc_.upload(gsrc.empty() ? std::vector<int>{0} : gsrc, s_);
  gph_.upload(gph.empty() ? std::vector<unsigned char>{0} : gph, s_);
  ap_.resize(h_pcol_.size());
  blk_pos_.upload(blk, s_);
  inv_.resize((size_t)nc * nph * nph);
  if (nt_ > 0) {
    tail_cnt_ = (int)tp.size();
    tail_pos_.upload(tp.empty() ? std::vector<int>{0} : tp, s_);
    tail_dst_.upload(tdst.empty() ? std::vector<long long>{0} : tdst, s_);
    tg_ptr_.upload(tgp, s_);
    tg_mem_.upload(tgm, s_);
    tg_off_.upload(tgo, s_);
    tM_.resize((size_t)tail_dense_);
    tInv_.resize((size_t)tail_dense_);
    trs_.resize(nt_);
  }
  w_.resize(nph);
  rw_.resize(nph);
  pw_.resize(nph);
  w_pin_.resize(3 * nph);
  bp_.resize(nc);
  xp_.resize(nc);
  if (f32_) {
    bp32_.resize(nc);
    xp32_.resize(nc);
  }
  ytmp_.resize(n);
  status_.resize(1);
  status_.zero(s_);
  st_pin_.resize(1);
  st_pin_[0] = 0;
  amg_.degree = amg32_.degree = std::max(1, o_.amg_smoother_degree);
  amg_.coarse_degree = amg32_.coarse_degree = std::max(0, o_.amg_coarse_degree);
  amg_.k_levels = amg32_.k_levels = std::max(0, o_.amg_cycle);
  kry_.init(n, o_.restart, s_);
  PMB_CUDA(cudaStreamSynchronize(s_));
}

void CsrCPR::check_status() {
  PMB_CUDA(cudaMemcpyAsync(st_pin_.get(), status_.get(), sizeof(int), cudaMemcpyDeviceToHost, s_));
  PMB_CUDA(cudaStreamSynchronize(s_));
  if (st_pin_[0] != 0) {
    const int code = st_pin_[0];
    st_pin_[0] = 0;
    PMB_CUDA(cudaMemsetAsync(status_.get(), 0, sizeof(int), s_));
    throw Error(code, code == PMB_ERR_PIVOT ? "singular cell block in the CPR preconditioner"
                                            : "device error in the CPR preconditioner");
  }
}

void CsrCPR::spmv(const double* val, const double* x, double* y) {
  csr8_spmv_kernel<<<grid_for(8LL * n_, 256), 256, 0, s_>>>(n_, rp_.get(), col_.get(), val, x, y);
  PMB_CHECK_LAUNCH();
}

void CsrCPR::setup(const double* d_val, const double* h_w) {
  PMB_REQUIRE(d_val != nullptr, "matrix values are required");
  val_ = d_val;
  ++setups_;
  // cell blocks and facility block
  csr_block_inv_kernel<<<grid_for(nc_, 128), 128, 0, s_>>>(nc_, nph_, blk_pos_.get(), val_, inv_.get(),
                                                            status_.get());
  PMB_CHECK_LAUNCH();
  if (nt_ > 0) {
    const int zb = (int)std::min<long long>(2LL * kNumSM, (tail_dense_ + 255) / 256);
    csr_tail_zero_kernel<<<std::max(zb, 1), 256, 0, s_>>>(tail_dense_, tM_.get());
    PMB_CHECK_LAUNCH();
    if (tail_cnt_ > 0) {
      csr_tail_scatter_kernel<<<std::min(2 * kNumSM, (tail_cnt_ + 255) / 256), 256, 0, s_>>>(
          tail_cnt_, tail_pos_.get(), tail_dst_.get(), val_, tM_.get());
      PMB_CHECK_LAUNCH();
    }
    csr_tail_invert_kernel<<<ngroups_, 128, 0, s_>>>(tg_ptr_.get(), tg_off_.get(), tM_.get(), tInv_.get(),
                                                     trs_.get(), status_.get());
    PMB_CHECK_LAUNCH();
  }
  if (o_.use_pressure_stage && cell_w_) {
    csr_cell_weights_kernel<<<grid_for(nc_, 256), 256, 0, s_>>>(nc_, nph_, inv_.get(), wcell_.get());
    PMB_CHECK_LAUNCH();
  }
  if (o_.use_pressure_stage) {
    PMB_REQUIRE(h_w != nullptr || cell_w_, "the pressure stage needs the phase weights");
    static const double kUnit[kMaxPhases] = {1.0, 0.0, 0.0};
    if (cell_w_) h_w = kUnit;
    for (int i = 0; i < nph_; ++i) {
      PMB_REQUIRE(std::isfinite(h_w[i]), "non-finite phase weight");
      w_pin_[i] = h_w[i];
      w_pin_[nph_ + i] = tr_ ? (i == 0 ? 1.0 : 0.0) : h_w[i];   // restriction
      w_pin_[2 * nph_ + i] = tr_ ? h_w[i] : (i == 0 ? 1.0 : 0.0);  // prolongation
    }
    PMB_CUDA(cudaMemcpyAsync(w_.get(), w_pin_.get(), sizeof(double) * nph_, cudaMemcpyHostToDevice, s_));
    PMB_CUDA(cudaMemcpyAsync(rw_.get(), w_pin_.get() + nph_, sizeof(double) * nph_, cudaMemcpyHostToDevice, s_));
    PMB_CUDA(cudaMemcpyAsync(pw_.get(), w_pin_.get() + 2 * nph_, sizeof(double) * nph_, cudaMemcpyHostToDevice,
                             s_));
    const int pn = (int)h_pcol_.size();
    const int g = grid_for(pn, 256);
    const bool built = f32_ ? amg32_.built() : amg_.built();
    if (!built || since_build_ >= std::max(1, o_.amg_rebuild_interval)) {
      if (cell_w_)
        csr_pressure_values_cell_kernel<double><<<grid_for(nc_, 128), 128, 0, s_>>>(
            nc_, nph_, prp_.get(), gptr_.get(), gsrc_.get(), gph_.get(), val_, wcell_.get(), ap_.get());
      else
        csr_pressure_values_kernel<double><<<g, 256, 0, s_>>>(pn, gptr_.get(), gsrc_.get(), gph_.get(), val_,
                                                             w_.get(), ap_.get());
      PMB_CHECK_LAUNCH();
      h_ap_.resize(pn);
      PMB_CUDA(cudaMemcpyAsync(h_ap_.data(), ap_.get(), sizeof(double) * pn, cudaMemcpyDeviceToHost, s_));
      PMB_CUDA(cudaStreamSynchronize(s_));
      for (double v : h_ap_) PMB_REQUIRE(std::isfinite(v), "non-finite entry in the pressure system");
      const int cs = std::max(16, o_.amg_coarse_size);
      if (f32_)
        amg32_.build(nc_, h_prp_, h_pcol_, prp_.get(), pcol_.get(), h_ap_, o_.amg_theta, cs, s_);
      else
        amg_.build(nc_, h_prp_, h_pcol_, prp_.get(), pcol_.get(), h_ap_, o_.amg_theta, cs, s_);
      since_build_ = 0;
      graph_.invalidate();
    }
    if (f32_) {
      if (cell_w_)
        csr_pressure_values_cell_kernel<float><<<grid_for(nc_, 128), 128, 0, s_>>>(
            nc_, nph_, prp_.get(), gptr_.get(), gsrc_.get(), gph_.get(), val_, wcell_.get(), amg32_.level0_val());
      else
        csr_pressure_values_kernel<float><<<g, 256, 0, s_>>>(pn, gptr_.get(), gsrc_.get(), gph_.get(), val_,
                                                            w_.get(), amg32_.level0_val());
      PMB_CHECK_LAUNCH();
      amg32_.refresh(s_, status_.get());
    } else {
      if (cell_w_)
        csr_pressure_values_cell_kernel<double><<<grid_for(nc_, 128), 128, 0, s_>>>(
            nc_, nph_, prp_.get(), gptr_.get(), gsrc_.get(), gph_.get(), val_, wcell_.get(), amg_.level0_val());
      else
        csr_pressure_values_kernel<double><<<g, 256, 0, s_>>>(pn, gptr_.get(), gsrc_.get(), gph_.get(), val_,
                                                             w_.get(), amg_.level0_val());
      PMB_CHECK_LAUNCH();
      amg_.refresh(s_, status_.get());
    }
    ++since_build_;
  }
  check_status();
}

void CsrCPR::precond_body(const double* r, double* z) {
  auto second_stage = [&](auto* xp) {
    using T = std::remove_const_t<std::remove_pointer_t<decltype(xp)>>;
    auto launch = [&](auto trc) {
      constexpr bool TR = decltype(trc)::value;
      csr_local_cells_kernel<TR, T><<<grid_for(nc_, 256), 256, 0, s_>>>(nc_, nph_, rp_.get(), col_.get(), val_, r,
                                                                        xp, pw_.get(), inv_.get(), z);
      PMB_CHECK_LAUNCH();
      if (nt_ > 0) {
        csr_local_tail_kernel<TR, T><<<ngroups_, 128, sizeof(double) * max_group_, s_>>>(
            nc_, nph_, tg_ptr_.get(), tg_mem_.get(), tg_off_.get(), rp_.get(), col_.get(), val_, r, xp, pw_.get(),
            tInv_.get(), z);
        PMB_CHECK_LAUNCH();
      }
    };
    if (tr_)
      launch(std::true_type{});
    else
      launch(std::false_type{});
  };
  if (o_.use_pressure_stage) {
    auto pressure_stage = [&](auto* bp, auto* xp, auto& amg) {
      if (cell_w_)
        csr_restrict_cell_kernel<<<grid_for(nc_, 256), 256, 0, s_>>>(nc_, nph_, r, wcell_.get(), bp);
      else
        csr_restrict_kernel<<<grid_for(nc_, 256), 256, 0, s_>>>(nc_, nph_, r, rw_.get(), bp);
      PMB_CHECK_LAUNCH();
      {
        PhaseTimer pt("cpr.amg_cycle", s_);
        amg.apply(bp, xp, s_);
      }
      second_stage(static_cast<const std::remove_pointer_t<decltype(xp)>*>(xp));
    };
    if (f32_)
      pressure_stage(bp32_.get(), xp32_.get(), amg32_);
    else
      pressure_stage(bp_.get(), xp_.get(), amg_);
  } else {
    second_stage(static_cast<const double*>(nullptr));
  }
  // further block-Jacobi sweeps on the whole system
  for (int sweep = 1; sweep < std::max(1, o_.local_sweeps); ++sweep) {
    spmv(val_, z, ytmp_.get());
    csr_jacobi_cells_kernel<<<grid_for(nc_, 256), 256, 0, s_>>>(nc_, nph_, r, ytmp_.get(), inv_.get(), z);
    PMB_CHECK_LAUNCH();
    if (nt_ > 0) {
      csr_jacobi_tail_kernel<<<ngroups_, 128, sizeof(double) * max_group_, s_>>>(
          nph_ * nc_, tg_ptr_.get(), tg_mem_.get(), tg_off_.get(), r, ytmp_.get(), tInv_.get(), z);
      PMB_CHECK_LAUNCH();
    }
  }
}

bool CsrCPR::solve(const double* b, double* x, double* info) {
  PMB_REQUIRE(val_ != nullptr, "pmb_csr_cpr_setup must run before pmb_csr_cpr_solve");
  if (pg_val_ != val_) {
    graph_.invalidate();
    pg_val_ = val_;
  }
  auto op = [this](const double* in, double* out) {
    PhaseTimer pt("gmres.spmv", s_);
    spmv(val_, in, out);
  };
  auto pc = [this](const double* in, double* out) {
    graph_.run(n_, in, out, s_, [this](const double* a, double* c) { precond_body(a, c); });
  };
  const bool ok = kry_.solve(op, pc, b, x, o_.rtol, o_.maxiter, info, status_.get(), [this] { check_status(); });
  info[3] = (double)setups_;
  return ok;
}

}  // namespace pmb

// ---- C ABI ------------------------------------------------------------------------

struct pmb_csr_cpr {
  std::unique_ptr<pmb::CsrCPR> impl;
};

extern "C" {

int pmb_csr_cpr_create(int32_t n, int32_t nc, int32_t nph, const int32_t* h_row_ptr, const int32_t* h_col,
                       int32_t transposed, const pmb_cpr_opts* opts, void* stream, pmb_csr_cpr** out) {
  return pmb::guarded([&] {
    PMB_REQUIRE(out != nullptr && opts != nullptr, "NULL argument");
    *out = nullptr;
    auto h = std::make_unique<pmb_csr_cpr>();
    h->impl = std::make_unique<pmb::CsrCPR>(n, nc, nph, h_row_ptr, h_col, transposed != 0, *opts,
                                            (cudaStream_t)stream);
    *out = h.release();
  });
}

int pmb_csr_cpr_destroy(pmb_csr_cpr* h) {
  return pmb::guarded([&] { delete h; });
}

int pmb_csr_cpr_setup(pmb_csr_cpr* h, const double* d_val, const double* h_weights) {
  return pmb::guarded([&] {
    PMB_REQUIRE(h != nullptr, "NULL argument");
    h->impl->setup(d_val, h_weights);
  });
}

int pmb_csr_cpr_solve(pmb_csr_cpr* h, const double* d_b, double* d_x, double* info4) {
  return pmb::guarded([&] {
    PMB_REQUIRE(h != nullptr && d_b != nullptr && d_x != nullptr && info4 != nullptr, "NULL argument");
    PMB_REQUIRE(d_b != d_x, "b and x must not alias");
    if (!h->impl->solve(d_b, d_x, info4))
      throw pmb::Error(PMB_ERR_NOCONV, "CPR-GMRES did not reach its tolerance (relres " +
                                           std::to_string(info4[1]) + " after " +
                                           std::to_string((long long)info4[0]) + " iterations)");
  });
}

int pmb_csr_cpr_set_cell_weights(pmb_csr_cpr* h, int32_t on) {
  return pmb::guarded([&] {
    PMB_REQUIRE(h != nullptr, "NULL argument");
    h->impl->set_cell_weights(on != 0);
  });
}

int pmb_csr_spmv(pmb_csr_cpr* h, const double* d_val, const double* d_x, double* d_y) {
  return pmb::guarded([&] {
    PMB_REQUIRE(h != nullptr && d_val != nullptr && d_x != nullptr && d_y != nullptr, "NULL argument");
    h->impl->spmv(d_val, d_x, d_y);
  });
}

int pmb_csr_cpr_levels(const pmb_csr_cpr* h, int32_t max_levels, int64_t* sizes, int32_t* n_levels) {
  return pmb::guarded([&] {
    PMB_REQUIRE(h != nullptr && n_levels != nullptr, "NULL argument");
    const int L = h->impl->num_levels();
    *n_levels = L;
    for (int l = 0; l < std::min<int>(L, max_levels); ++l) sizes[l] = h->impl->level_size(l);
  });
}

}  // extern "C"
