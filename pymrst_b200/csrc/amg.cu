// Aggregation AMG: host aggregation, device Galerkin refresh, Chebyshev
// smoothing, V-cycle, dense coarsest solve.
#include <algorithm>
#include <string>
#include <cmath>
#include <cstdlib>
#include <numeric>
#include <type_traits>
#include <unordered_map>

#include <cooperative_groups.h>

#include "pmb_amg.cuh"

namespace pmb {

namespace cg = cooperative_groups;

// ---------------------------------------------------------------------------
// host: pairwise aggregation and Galerkin structure
// ---------------------------------------------------------------------------

// Greedy pairwise matching: each unmatched unknown i (in order) is paired
// with its strongest unmatched neighbour j, strength s_ij = -a_ij, among
// those with s_ij >= theta * max_k s_ik; otherwise it stays alone.
// Rows without any negative coupling (possible after upwinding with gravity,
// and on Galerkin coarse levels) use |a_ij| as strength instead.  With
// `attach`, an unknown left alone joins the aggregate of its strongest
// neighbour, so every connected unknown is coarsened; a row whose couplings
// are all exactly zero (a transport Jacobian where no phase is mobile) is
// then paired with, or attached to, its first neighbour in the pattern, so
// that the coarsening does not stall on it (the smoother solves such rows
// exactly).
static int pairwise_match(int n, const int* rp, const int* ci, const double* v, double theta,
                          std::vector<int>& agg, bool attach) {
  agg.assign(n, -1);
  std::vector<int> alone;
  int na = 0;
  for (int i = 0; i < n; ++i) {
    if (agg[i] >= 0) continue;
    double mx = 0.0;
    for (int k = rp[i]; k < rp[i + 1]; ++k)
      if (ci[k] != i) mx = std::max(mx, -v[k]);
    const bool use_abs = !(mx > 0.0);
    if (use_abs)
      for (int k = rp[i]; k < rp[i + 1]; ++k)
        if (ci[k] != i) mx = std::max(mx, std::fabs(v[k]));
    int best = -1;
    double bv = -1.0;
    if (mx > 0.0) {
      for (int k = rp[i]; k < rp[i + 1]; ++k) {
        const int j = ci[k];
        if (j == i || agg[j] >= 0) continue;
        const double s = use_abs ? std::fabs(v[k]) : -v[k];
        if (s >= theta * mx && s > bv) { bv = s; best = j; }
      }
    } else if (attach) {
      for (int k = rp[i]; k < rp[i + 1] && best < 0; ++k)
        if (ci[k] != i && agg[ci[k]] < 0) best = ci[k];
    }
    agg[i] = na;
    if (best >= 0) agg[best] = na;
    else alone.push_back(i);
    ++na;
  }
  if (!attach || alone.empty()) return na;
  // move singletons into a neighbour's aggregate, then renumber densely
  for (int i : alone) {
    int best = -1;
    double bv = 0.0;
    for (int k = rp[i]; k < rp[i + 1]; ++k) {
      const int j = ci[k];
      if (j == i) continue;
      const double s = std::fabs(v[k]);
      if (s > bv) { bv = s; best = j; }
    }
    for (int k = rp[i]; k < rp[i + 1] && best < 0; ++k)
      if (ci[k] != i) best = ci[k];
    if (best >= 0) agg[i] = agg[best];
  }
  std::vector<int> ren(na, -1);
  int m = 0;
  for (int i = 0; i < n; ++i) {
    if (ren[agg[i]] < 0) ren[agg[i]] = m++;
    agg[i] = ren[agg[i]];
  }
  return m;
}

struct HostCSR {
  int n = 0;
  std::vector<int> rp, ci;
  std::vector<double> v;
};

// Coarse pattern of P^T A P for aggregation `agg` (n -> nc) and, for every
// coarse entry, the fine entries that sum into it (in increasing order).
static void galerkin_structure(int n, const int* rp, const int* ci, const std::vector<int>& agg, int nc,
                               std::vector<int>& crp, std::vector<int>& cci, std::vector<int>& gptr,
                               std::vector<int>& gidx, std::vector<int>& cptr, std::vector<int>& cmem) {
  cptr.assign(nc + 1, 0);
  for (int i = 0; i < n; ++i) ++cptr[agg[i] + 1];
  for (int I = 0; I < nc; ++I) cptr[I + 1] += cptr[I];
  cmem.assign(n, 0);
  {
    std::vector<int> fill(cptr.begin(), cptr.end() - 1);
    for (int i = 0; i < n; ++i) cmem[fill[agg[i]]++] = i;
  }
  crp.assign(nc + 1, 0);
  cci.clear();
  std::vector<std::pair<int, int>> ent;      // (coarse col, fine nnz)
  std::vector<std::pair<int, int>> all_map;  // (coarse nnz, fine nnz)
  all_map.reserve(rp[n]);
  for (int I = 0; I < nc; ++I) {
    ent.clear();
    for (int m = cptr[I]; m < cptr[I + 1]; ++m) {
      const int i = cmem[m];
      for (int k = rp[i]; k < rp[i + 1]; ++k) ent.emplace_back(agg[ci[k]], k);
    }
    std::sort(ent.begin(), ent.end());
    for (size_t e = 0; e < ent.size(); ++e) {
      if (e == 0 || ent[e].first != ent[e - 1].first) cci.push_back(ent[e].first);
      all_map.emplace_back((int)cci.size() - 1, ent[e].second);
    }
    crp[I + 1] = (int)cci.size();
  }
  const int nnzc = (int)cci.size();
  gptr.assign(nnzc + 1, 0);
  for (auto& p : all_map) ++gptr[p.first + 1];
  for (int K = 0; K < nnzc; ++K) gptr[K + 1] += gptr[K];
  gidx.assign(all_map.size(), 0);
  std::vector<int> fill(gptr.begin(), gptr.end() - 1);
  for (auto& p : all_map) gidx[fill[p.first]++] = p.second;
}

static void galerkin_values(const std::vector<int>& gptr, const std::vector<int>& gidx,
                            const std::vector<double>& fv, std::vector<double>& cv) {
  const int nnzc = (int)gptr.size() - 1;
  cv.assign(nnzc, 0.0);
  for (int K = 0; K < nnzc; ++K) {
    double s = 0.0;
    for (int g = gptr[K]; g < gptr[K + 1]; ++g) s += fv[gidx[g]];
    cv[K] = s;
  }
}

std::vector<AMGHostLevel> amg_build_hierarchy(int n, const int* row_ptr, const int* col,
                                              const double* val, double theta, int passes,
                                              int coarse_size, int max_levels, int aggressive_below) {
  std::vector<AMGHostLevel> out;
  HostCSR cur;
  cur.n = n;
  cur.rp.assign(row_ptr, row_ptr + n + 1);
  cur.ci.assign(col, col + row_ptr[n]);
  cur.v.assign(val, val + row_ptr[n]);
  while (cur.n > coarse_size && (int)out.size() < max_levels) {
    std::vector<int> agg(cur.n);
    std::iota(agg.begin(), agg.end(), 0);
    int na = cur.n;
    HostCSR work = cur;
    const int level_passes = cur.n < aggressive_below ? passes + 1 : passes;
    for (int p = 0; p < level_passes; ++p) {
      std::vector<int> a2;
      int na2 = pairwise_match(work.n, work.rp.data(), work.ci.data(), work.v.data(), theta, a2, false);
      if (na2 > 0.7 * work.n)
        na2 = pairwise_match(work.n, work.rp.data(), work.ci.data(), work.v.data(), 0.0, a2, true);
      for (int i = 0; i < cur.n; ++i) agg[i] = a2[agg[i]];
      na = na2;
      if (p + 1 < level_passes) {
        HostCSR next;
        std::vector<int> gp, gi, cp, cm;
        galerkin_structure(work.n, work.rp.data(), work.ci.data(), a2, na2, next.rp, next.ci, gp, gi, cp, cm);
        next.n = na2;
        galerkin_values(gp, gi, work.v, next.v);
        work = std::move(next);
      }
    }
    if (na >= 0.95 * cur.n) break;  // coarsening stalled
    AMGHostLevel L;
    L.n = cur.n;
    L.row_ptr = cur.rp;
    L.col = cur.ci;
    L.agg = agg;
    HostCSR next;
    galerkin_structure(cur.n, cur.rp.data(), cur.ci.data(), agg, na, next.rp, next.ci, L.gptr, L.gidx,
                       L.cptr, L.cmem);
    next.n = na;
    galerkin_values(L.gptr, L.gidx, cur.v, next.v);
    out.push_back(std::move(L));
    cur = std::move(next);
  }
  AMGHostLevel last;
  last.n = cur.n;
  last.row_ptr = cur.rp;
  last.col = cur.ci;
  out.push_back(std::move(last));
  return out;
}

// ---------------------------------------------------------------------------
// device kernels
// ---------------------------------------------------------------------------

// Inverse diagonal and the Gershgorin bound max_i sum_j |a_ij| / |a_ii| of
// D^{-1} A (positive doubles order like their bit patterns, so the maximum
// is an integer atomicMax and independent of the order of arrival).
template <class T>
__global__ void diag_kernel(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                            const T* __restrict__ a, T* __restrict__ dinv,
                            unsigned long long* __restrict__ lmax_bits, int* status) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double d = 0.0, s = 0.0;
  for (int k = rp[i]; k < rp[i + 1]; ++k) {
    const double v = (double)a[k];
    s += fabs(v);
    if (ci[k] == i) d = v;
  }
  if (d == 0.0 || !isfinite(d)) {
    atomicExch(status, PMB_ERR_PIVOT);
    d = 1.0;
  }
  dinv[i] = (T)(1.0 / d);
  const double g = s / fabs(d);
  atomicMax(lmax_bits, (unsigned long long)__double_as_longlong(g));
}

// The Chebyshev table of a level, after its Gershgorin bound: tab[0] = the
// bound, tab[1 + 2k], tab[2 + 2k] = the coefficients (c1, c2) of step k.
// Computed once per refresh, so that a step kernel loads its two
// coefficients instead of deriving them (a chain of FP64 divisions before
// its first row could finish).
constexpr int kMaxChebSteps = 16;
constexpr int kChebTable = 1 + 2 * kMaxChebSteps;

__device__ __forceinline__ void cheb_coeffs(double lm, int step, double& c1, double& c2);

__global__ void cheb_table_kernel(const unsigned long long* bits, double* tab) {
  const double lm = __longlong_as_double((long long)bits[0]);
  const int k = threadIdx.x;
  if (k == 0) tab[0] = lm;
  if (k < kMaxChebSteps) cheb_coeffs(lm, k, tab[1 + 2 * k], tab[2 + 2 * k]);
}

template <class T>
__global__ void galerkin_kernel(int nnzc, const int* __restrict__ gptr, const int* __restrict__ gidx,
                                const T* __restrict__ fv, T* __restrict__ cv) {
  const int K = blockIdx.x * blockDim.x + threadIdx.x;
  if (K >= nnzc) return;
  double s = 0.0;
  for (int g = gptr[K]; g < gptr[K + 1]; ++g) s += (double)fv[gidx[g]];
  cv[K] = (T)s;
}

// Sum over a group of LANES consecutive lanes (a power of two); every lane of
// the warp must take part.
template <int LANES>
__device__ __forceinline__ double group_sum(double v) {
#pragma unroll
  for (int o = LANES / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// A lane's first two entries of a CSR row (entries rp[i] + sub,
// + LANES, ...), loaded before the kernel waits on its predecessor grid: a
// level's matrix is written only when the hierarchy is refreshed, never
// inside a cycle, so its loads may overlap the predecessor's tail; only the
// iterate has to wait.  row_sum then folds the row in the same entry order
// as a plain loop over k.
template <class T>
struct RowPre {
  int k = 0, end = 0, c0 = 0, c1 = 0;
  T v0 = T(0), v1 = T(0);
};

template <class T, int LANES>
__device__ __forceinline__ RowPre<T> row_prefetch(long long i, int sub, const int* __restrict__ rp,
                                                  const int* __restrict__ ci, const T* __restrict__ a) {
  RowPre<T> p;
  p.k = rp[i] + sub;
  p.end = rp[i + 1];
  if (p.k < p.end) {
    p.c0 = ci[p.k];
    p.v0 = a[p.k];
  }
  if (p.k + LANES < p.end) {
    p.c1 = ci[p.k + LANES];
    p.v1 = a[p.k + LANES];
  }
  return p;
}

template <class T, int LANES, class F>
__device__ __forceinline__ double row_sum(const RowPre<T> p, const int* __restrict__ ci, const T* __restrict__ a,
                                          double acc, F f) {
  if (p.k < p.end) acc = f(acc, (double)p.v0, p.c0);
  if (p.k + LANES < p.end) acc = f(acc, (double)p.v1, p.c1);
  for (int k = p.k + 2 * LANES; k < p.end; k += LANES) acc = f(acc, (double)a[k], ci[k]);
  return acc;
}

// Calls f(std::integral_constant<int, L>) with L the row-group width.
template <class F>
void with_lanes(int lanes, F&& f) {
  switch (lanes) {
    case 32: f(std::integral_constant<int, 32>{}); break;
    case 16: f(std::integral_constant<int, 16>{}); break;
    case 8: f(std::integral_constant<int, 8>{}); break;
    case 4: f(std::integral_constant<int, 4>{}); break;
    case 2: f(std::integral_constant<int, 2>{}); break;
    default: f(std::integral_constant<int, 1>{}); break;
  }
}

// Row-group width for a level: about two entries of the row per lane.
// Measured on the channelised model: one entry per lane left the finest
// level latency-bound (20 of 32 threads active, scoreboard stalls); two per
// lane made the AMG cycle 11% faster, four per lane 9% slower.
inline int lanes_for(long long n, long long nnz) {
  const double avg = n > 0 ? (double)nnz / (double)n : 0.0;
  if (avg > 48.0) return 32;
  if (avg > 24.0) return 16;
  if (avg > 12.0) return 8;
  if (avg > 5.0) return 4;
  return 2;
}

// Coefficients of step `step` of the Chebyshev recurrence on [lm/10, lm].
__device__ __forceinline__ void cheb_coeffs(double lm, int step, double& c1, double& c2) {
  // explicit roundings: the per-step and the cluster tail kernels must agree
  const double lo = __ddiv_rn(lm, 10.0);
  const double theta = __dmul_rn(0.5, __dadd_rn(lm, lo)), delta = __dmul_rn(0.5, __dsub_rn(lm, lo));
  const double sigma = __ddiv_rn(theta, delta);
  double rho = __ddiv_rn(1.0, sigma);
  c1 = 0.0;
  c2 = __ddiv_rn(1.0, theta);
  for (int k = 1; k <= step; ++k) {
    const double rho1 = __ddiv_rn(1.0, __dsub_rn(__dmul_rn(2.0, sigma), rho));
    c1 = __dmul_rn(rho1, rho);
    c2 = __ddiv_rn(__dmul_rn(2.0, rho1), delta);
    rho = rho1;
  }
}

// The arithmetic of one Chebyshev row update, shared by the per-step kernels
// and the cluster tail kernel below so that both produce the same bits:
// explicit roundings leave the compiler no choice of contraction.
__device__ __forceinline__ double cheb_res(double b, double ax, double dinv) {
  return __dmul_rn(__dsub_rn(b, ax), dinv);
}
__device__ __forceinline__ double cheb_dir(int step, double c1, double c2, double d_old, double r) {
  const double t = __dmul_rn(c2, r);
  return step == 0 ? t : __fma_rn(c1, d_old, t);
}

// ZeroStep (pmb_amg.cuh): the arithmetic of cheb_step_kernel<T, true>.
template <class T>
__device__ __forceinline__ void zero_step(const ZeroStep<T>& z, long long i, T b) {
  const double r = cheb_res((double)b, 0.0, (double)z.dinv[i]);
  const double dn = cheb_dir(0, z.tab[1], z.tab[2], 0.0, r);
  z.d[i] = (T)dn;
  z.x[i] = (T)__dadd_rn(0.0, dn);
}

// Chebyshev on D^{-1} A over [lmax/10, lmax]: step `step` of the
// three-term recurrence; x_out = x_in + d, d = c1 d + c2 D^{-1}(b - A x_in).
// LANES threads share a row.
// With PRO, x_in is first corrected by the coarse-level correction, read as
// x_in[j] + xc[agg[j]] rounded to T exactly as prolong_add_kernel would store
// it: the prolongation and the first post-smoothing step in one launch.
template <class T, bool PRO>
__device__ __forceinline__ double cheb_x(const T* __restrict__ xin, const int* __restrict__ agg,
                                         const T* __restrict__ xc, int j) {
  if (!PRO) return (double)xin[j];
  return (double)(T)__dadd_rn((double)xin[j], (double)xc[agg[j]]);
}

template <class T, bool ZERO, int LANES, bool PRO = false>
__global__ void __launch_bounds__(256) cheb_step_kernel(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                                                        const T* __restrict__ a, const T* __restrict__ dinv,
                                                        const T* __restrict__ b, const T* __restrict__ xin,
                                                        T* __restrict__ xout, T* __restrict__ d, const double* lmax,
                                                        int step, const int* __restrict__ agg = nullptr,
                                                        const T* __restrict__ xc = nullptr) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long i = t / LANES;
  const int sub = (int)(t % LANES);
  RowPre<T> p;
  double di = 0.0;
  if (i < n) {
    if (!ZERO) p = row_prefetch<T, LANES>(i, sub, rp, ci, a);
    if (sub == 0) di = (double)dinv[i];
  }
  const double c1 = lmax[1 + 2 * step], c2 = lmax[2 + 2 * step];  // written at the refresh
  pdl_enter();
  // the row's own values first, so that they travel with the gathers below
  double bi = 0.0, dold = 0.0, xi = 0.0;
  if (i < n && sub == 0) {
    bi = (double)b[i];
    if (step != 0) dold = (double)d[i];
    if (!ZERO) xi = cheb_x<T, PRO>(xin, agg, xc, (int)i);
  }
  double ax = 0.0;
  if (!ZERO) {
    if (i < n)
      ax = row_sum<T, LANES>(p, ci, a, 0.0, [=](double acc, double v, int j) {
        return __fma_rn(v, cheb_x<T, PRO>(xin, agg, xc, j), acc);
      });
    ax = group_sum<LANES>(ax);
  }
  if (i >= n || sub != 0) return;
  const double r = cheb_res(bi, ax, di);
  const double dn = cheb_dir(step, c1, c2, dold, r);
  d[i] = (T)dn;
  xout[i] = (T)__dadd_rn(xi, dn);
}

// b_c[I] = sum over members i of (b_i - (A x)_i); LANES threads per aggregate
// share each member row.
template <class T, int LANES>
__global__ void __launch_bounds__(256) restrict_residual_kernel(int nc, const int* __restrict__ cptr,
                                                                const int* __restrict__ cmem,
                                                                const int* __restrict__ rp, const int* __restrict__ ci,
                                                                const T* __restrict__ a, const T* __restrict__ b,
                                                                const T* __restrict__ x, T* __restrict__ bc) {
  pdl_enter();
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long I = t / LANES;
  const int sub = (int)(t % LANES);
  double s = 0.0;
  if (I < nc)
    for (int m = cptr[I]; m < cptr[I + 1]; ++m) {
      const int i = cmem[m];
      if (sub == 0) s += (double)b[i];
      for (int k = rp[i] + sub; k < rp[i + 1]; k += LANES) s -= (double)a[k] * (double)x[ci[k]];
    }
  s = group_sum<LANES>(s);
  if (I < nc && sub == 0) bc[I] = (T)s;
}

// The same restricted residual, parallel over member rows: CTA b takes the
// aggregates [blk[b], blk[b+1]) of the restriction plan; each lane group
// forms the residual b_i - (A x)_i of one member row (looping over the
// members only when one aggregate has more rows than the CTA has groups),
// keeps it in shared memory, and one thread per aggregate then sums its
// members in member order.  The member loop of restrict_residual_kernel
// waits on a chain of dependent loads (member, row start, column, x) per
// member; here the chains of all members overlap.
template <class T, int LANES>
__global__ void __launch_bounds__(256) restrict_rows_kernel(const int* __restrict__ blk, const int* __restrict__ cptr,
                                                            const int* __restrict__ cmem,
                                                            const int* __restrict__ rp, const int* __restrict__ ci,
                                                            const T* __restrict__ a, const T* __restrict__ b,
                                                            const T* __restrict__ x, T* __restrict__ bc,
                                                            ZeroStep<T> zs) {
  extern __shared__ double rr_smem[];
  // the plan, the member lists and the first member rows: loaded before the
  // wait (none is written inside a cycle)
  const int I0 = blk[blockIdx.x], I1 = blk[blockIdx.x + 1];
  const int m0 = cptr[I0], m1 = cptr[I1];
  const int groups = blockDim.x / LANES;
  const int g = threadIdx.x / LANES, sub = threadIdx.x % LANES;
  RowPre<T> p;
  int i = 0;
  if (m0 + g < m1) {
    i = cmem[m0 + g];
    p = row_prefetch<T, LANES>(i, sub, rp, ci, a);
  }
  pdl_enter();
  for (int mb = m0; mb < m1; mb += groups) {  // the same trip count for every thread
    const int m = mb + g;
    double s = 0.0, bi = 0.0;
    if (m < m1) {
      if (mb != m0) {
        i = cmem[m];
        p = row_prefetch<T, LANES>(i, sub, rp, ci, a);
      }
      if (sub == 0) bi = (double)b[i];
      s = row_sum<T, LANES>(p, ci, a, 0.0,
                            [=](double acc, double v, int j) { return __fma_rn(-v, (double)x[j], acc); });
    }
    s = group_sum<LANES>(s);
    if (m < m1 && sub == 0) rr_smem[m - m0] = __dadd_rn(bi, s);
  }
  __syncthreads();
  for (int I = I0 + threadIdx.x; I < I1; I += blockDim.x) {
    double v = 0.0;
    for (int m = cptr[I]; m < cptr[I + 1]; ++m) v = __dadd_rn(v, rr_smem[m - m0]);
    bc[I] = (T)v;
    if (zs.dinv) zero_step(zs, I, (T)v);
  }
}

template <class T>
__global__ void prolong_add_kernel(int n, const int* __restrict__ agg, const T* __restrict__ xc,
                                   T* __restrict__ x) {
  pdl_enter();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  x[i] = (T)__dadd_rn((double)x[i], (double)xc[agg[i]]);
}

template <class T>
__global__ void copy_kernel(int n, const T* __restrict__ a, T* __restrict__ b) {
  pdl_enter();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = a[i];
}

// ELL levels (AMGLevel::ell_k > 0) ------------------------------------------
//
// One thread per row: the row's slots are loaded together, then the iterate
// at every column, so a thread has all its loads in flight at once instead
// of the CSR kernels' chain of row start -> column -> iterate.  In the
// diagonal form (a level whose entries lie on a few column offsets, as a
// structured grid's do) slot k of row i is column i + off[k], so the iterate
// gathers need no column load at all.  The row is summed in slot order,
// then its overflow entries.

// A row's slots, loaded before the kernel waits on its predecessor (the
// ELL copy is written only at a refresh); ovf >= 0 names its overflow row.
template <class T>
struct EllPre {
  int c[kEllMaxK];
  T v[kEllMaxK];
  int ovf;
};

template <class T>
__device__ __forceinline__ void ell_load(EllPre<T>& e, int i, const EllView<T>& E) {
  const long long n = E.n;
  const int K = E.K;
#pragma unroll
  for (int k = 0; k < kEllMaxK; ++k) e.v[k] = k < K ? E.val[k * n + i] : T(0);
  if (E.col == nullptr) {
    // padded slots hold zero: any column in range will do for them
#pragma unroll
    for (int k = 0; k < kEllMaxK; ++k) e.c[k] = k < K ? min(max(i + E.off[k], 0), E.n - 1) : i;
    e.ovf = E.orow[i];
    return;
  }
#pragma unroll
  for (int k = 0; k < kEllMaxK; ++k) e.c[k] = k < K ? E.col[k * n + i] : i;
  e.ovf = -1;
#pragma unroll
  for (int k = 0; k < kEllMaxK; ++k)
    if (k == K - 1 && e.c[k] < 0) {
      e.ovf = -1 - e.c[k];
      e.c[k] = i;  // its value is zero
    }
}

template <class T, bool PRO, bool NEG>
__device__ __forceinline__ double ell_sum(const EllPre<T>& e, const EllView<T>& E, const T* __restrict__ xin,
                                          const int* __restrict__ agg, const T* __restrict__ xc) {
  const int K = E.K;
  double xv[kEllMaxK];
#pragma unroll
  for (int k = 0; k < kEllMaxK; ++k)
    if (k < K) xv[k] = cheb_x<T, PRO>(xin, agg, xc, e.c[k]);
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < kEllMaxK; ++k)
    if (k < K) s = __fma_rn(NEG ? -(double)e.v[k] : (double)e.v[k], xv[k], s);
  if (e.ovf >= 0)
    for (int q = E.optr[e.ovf]; q < E.optr[e.ovf + 1]; ++q)
      s = __fma_rn(NEG ? -(double)E.oval[q] : (double)E.oval[q], cheb_x<T, PRO>(xin, agg, xc, E.ocol[q]), s);
  return s;
}

// cheb_step_kernel (non-zero start) on an ELL level: the same row update.
template <class T, bool PRO>
__global__ void __launch_bounds__(256) cheb_ell_kernel(EllView<T> E, const T* __restrict__ dinv,
                                                       const T* __restrict__ b, const T* __restrict__ xin,
                                                       T* __restrict__ xout, T* __restrict__ d, const double* lmax,
                                                       int step, const int* __restrict__ agg,
                                                       const T* __restrict__ xc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = E.n;
  EllPre<T> e;
  double di = 0.0;
  if (i < n) {
    ell_load(e, i, E);
    di = (double)dinv[i];
  }
  const double c1 = lmax[1 + 2 * step], c2 = lmax[2 + 2 * step];
  pdl_enter();
  if (i >= n) return;
  const double bi = (double)b[i];
  const double dold = step == 0 ? 0.0 : (double)d[i];
  const double xi = cheb_x<T, PRO>(xin, agg, xc, i);
  const double ax = ell_sum<T, PRO, false>(e, E, xin, agg, xc);
  const double r = cheb_res(bi, ax, di);
  const double dn = cheb_dir(step, c1, c2, dold, r);
  d[i] = (T)dn;
  xout[i] = (T)__dadd_rn(xi, dn);
}

// rr[i] = b_i - (A x)_i on an ELL level, accumulated as the restriction
// kernels do (the negated products, then b).
template <class T>
__global__ void __launch_bounds__(256) ell_residual_kernel(EllView<T> E, const T* __restrict__ b,
                                                           const T* __restrict__ x, double* __restrict__ rr) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  EllPre<T> e;
  if (i < E.n) ell_load(e, i, E);
  pdl_enter();
  if (i >= E.n) return;
  const double bi = (double)b[i];
  const double s = ell_sum<T, false, true>(e, E, x, nullptr, nullptr);
  rr[i] = __dadd_rn(bi, s);
}

// bc[I] = the sum of rr over the members of aggregate I, in member order.
template <class T>
__global__ void __launch_bounds__(256) aggregate_sum_kernel(int nc, const int* __restrict__ cptr,
                                                            const int* __restrict__ cmem,
                                                            const double* __restrict__ rr, T* __restrict__ bc,
                                                            ZeroStep<T> zs) {
  pdl_enter();
  const int I = blockIdx.x * blockDim.x + threadIdx.x;
  if (I >= nc) return;
  double v = 0.0;
  for (int m = cptr[I]; m < cptr[I + 1]; ++m) v = __dadd_rn(v, rr[cmem[m]]);
  bc[I] = (T)v;
  if (zs.dinv) zero_step(zs, I, (T)v);
}

// dst[k] = val[src[k]] (zero where src is -1): the ELL copy's values after a
// refresh of the CSR values.
template <class T>
__global__ void ell_values_kernel(long long total, const int* __restrict__ src, const T* __restrict__ val,
                                  T* __restrict__ dst) {
  const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (k >= total) return;
  const int j = src[k];
  dst[k] = j >= 0 ? val[j] : T(0);
}

// Dense coarsest level (FP64): assemble, invert by Gauss-Jordan with
// partial pivoting in one CTA, apply as a dense product.
template <class T>
__global__ void dense_assemble_kernel(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                                      const T* __restrict__ a, double* __restrict__ M) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int j = 0; j < n; ++j) M[(size_t)i * n + j] = 0.0;
  for (int k = rp[i]; k < rp[i + 1]; ++k) M[(size_t)i * n + ci[k]] = (double)a[k];
}

// Dense coarsest inverse: in-place Gauss-Jordan elimination with row
// pivoting in one CTA.  Step k takes the largest |A[i][k]|, i >= k, as pivot
// (ties to the lowest row), swaps it into row k, scales row k by 1/pivot
// (A[k][k] becomes 1/pivot) and subtracts A[i][k] times the new row k from
// every other row i (A[i][k] becomes -A[i][k]/pivot).  The row interchanges
// are undone at the end by the same column interchanges in reverse order.
// The first m rows of the working matrix live in shared memory, the others
// in Inv itself (L2-resident at these sizes); the pivot row and the
// multipliers of each step are staged in shared memory, so every step is
// four barriers and one parallel pass over the matrix.  Dynamic shared
// memory: (2n + m n) doubles and n ints.  A zero or non-finite pivot sets
// PMB_ERR_PIVOT in *status (the elimination goes on with pivot 1).
constexpr int kGJThreads = 1024;

__global__ void __launch_bounds__(kGJThreads) gauss_jordan_kernel(int n, int m, const double* __restrict__ M,
                                                                  double* __restrict__ Inv,
                                                                  int* __restrict__ status) {
  extern __shared__ __align__(16) double gj_smem[];
  double* prow = gj_smem;
  double* fcol = prow + n;
  double* srows = fcol + n;
  int* piv = reinterpret_cast<int*>(srows + (size_t)m * n);
  __shared__ double w_best[kGJThreads / 32];
  __shared__ int w_idx[kGJThreads / 32];
  __shared__ int s_p;
  const int t = threadIdx.x, nt = blockDim.x, lane = t & 31, warp = t >> 5;
  auto row = [&](int r) -> double* { return r < m ? srows + (size_t)r * n : Inv + (size_t)r * n; };
  const int nwarps = nt >> 5;
  for (int i = warp; i < n; i += nwarps) {
    double* ri = row(i);
    for (int j = lane; j < n; j += 32) ri[j] = M[(size_t)i * n + j];
  }
  __syncthreads();
  for (int k = 0; k < n; ++k) {
    // pivot: the largest |A[i][k]| over i >= k, lowest row on ties
    double best = -1.0;
    int bi = n;
    for (int i = k + t; i < n; i += nt) {
      const double v = fabs(row(i)[k]);
      if (v > best) {  // rows are visited in increasing order: ties keep the lower
        best = v;
        bi = i;
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const double ob = __shfl_down_sync(0xffffffffu, best, o);
      const int oi = __shfl_down_sync(0xffffffffu, bi, o);
      if (ob > best || (ob == best && oi < bi)) {
        best = ob;
        bi = oi;
      }
    }
    if (lane == 0) {
      w_best[warp] = best;
      w_idx[warp] = bi;
    }
    __syncthreads();
    if (warp == 0) {
      const int nw = nt >> 5;
      best = lane < nw ? w_best[lane] : -1.0;
      bi = lane < nw ? w_idx[lane] : n;
      for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_down_sync(0xffffffffu, best, o);
        const int oi = __shfl_down_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi < bi)) {
          best = ob;
          bi = oi;
        }
      }
      if (lane == 0) {
        if (!(best > 0.0) || !isfinite(best) || bi >= n) {
          atomicExch(status, PMB_ERR_PIVOT);
          bi = k;
        }
        s_p = bi;
        piv[k] = bi;
      }
    }
    __syncthreads();
    const int p = s_p;
    if (p != k) {
      double* rk = row(k);
      double* rp = row(p);
      for (int j = t; j < n; j += nt) {
        const double a = rk[j];
        rk[j] = rp[j];
        rp[j] = a;
      }
    }
    __syncthreads();
    {
      const double d = row(k)[k];
      const double inv_d = (d != 0.0 && isfinite(d)) ? 1.0 / d : 1.0;
      const double* rk = row(k);
      for (int j = t; j < n; j += nt) prow[j] = j == k ? inv_d : rk[j] * inv_d;
      for (int i = t; i < n; i += nt) fcol[i] = i == k ? 0.0 : row(i)[k];
    }
    __syncthreads();
    for (int i = warp; i < n; i += nwarps) {
      double* ri = row(i);
      if (i == k) {
        for (int j = lane; j < n; j += 32) ri[j] = prow[j];
      } else {
        const double f = fcol[i];
        for (int j = lane; j < n; j += 32) ri[j] = (j == k ? 0.0 : ri[j]) - f * prow[j];
      }
    }
    __syncthreads();
  }
  for (int k = n - 1; k >= 0; --k) {
    const int p = piv[k];
    if (p != k)
      for (int r = t; r < n; r += nt) {
        double* rr = row(r);
        const double a = rr[k];
        rr[k] = rr[p];
        rr[p] = a;
      }
    __syncthreads();
  }
  for (int i = warp; i < m; i += nwarps)
    for (int j = lane; j < n; j += 32) Inv[(size_t)i * n + j] = srows[(size_t)i * n + j];
}

// The same Gauss-Jordan inverse on a thread-block cluster of C CTAs when the
// working matrix does not fit one CTA's shared memory: CTA c holds rows
// [c R, c R + R) in its own shared memory and reads the others' through
// distributed shared memory.  Every step does what gauss_jordan_kernel does,
// with the same operations on every element (the pivot is the largest |a|
// of the column, the lowest row on ties, so the cluster agrees on it), so
// the inverse is bitwise that kernel's.  The cluster barriers are taken by
// every thread of every CTA in the same order (the branches around them
// depend only on the pivot, which all CTAs compute alike).
__global__ void __launch_bounds__(kGJThreads) gauss_jordan_cluster_kernel(int n, int R, const double* __restrict__ M,
                                                                          double* __restrict__ Inv,
                                                                          int* __restrict__ status) {
  extern __shared__ __align__(16) double gjc_smem[];
  cg::cluster_group cl = cg::this_cluster();
  const int me = (int)cl.block_rank(), C = (int)cl.num_blocks();
  double* rows = gjc_smem;                    // R x n, the CTA's rows
  double* prow = rows + (size_t)R * n;        // n: the scaled pivot row
  double* tmp = prow + n;                     // n: a row arriving in a swap
  double* fcol = tmp + n;                     // R: column k of the CTA's rows
  double* cand = fcol + R;                    // 2: this CTA's pivot candidate (value, row)
  int* piv = reinterpret_cast<int*>(cand + 2);  // n
  __shared__ double w_best[kGJThreads / 32];
  __shared__ int w_idx[kGJThreads / 32];
  __shared__ int s_p;
  const int t = threadIdx.x, nt = blockDim.x, lane = t & 31, warp = t >> 5, nwarps = nt >> 5;
  const int r0 = me * R, r1 = min(n, r0 + R);
  auto row_of = [&](int r) -> double* {  // row r of the matrix, wherever it lives
    return cl.map_shared_rank(rows + (size_t)(r % R) * n, r / R);
  };
  for (int i = r0 + warp; i < r1; i += nwarps)
    for (int j = lane; j < n; j += 32) rows[(size_t)(i - r0) * n + j] = M[(size_t)i * n + j];
  cl.sync();
  for (int k = 0; k < n; ++k) {
    // the CTA's candidate: the largest |A[i][k]| over its rows i >= k
    double best = -1.0;
    int bi = n;
    for (int i = max(k, r0) + t; i < r1; i += nt) {
      const double v = fabs(rows[(size_t)(i - r0) * n + k]);
      if (v > best) {
        best = v;
        bi = i;
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const double ob = __shfl_down_sync(0xffffffffu, best, o);
      const int oi = __shfl_down_sync(0xffffffffu, bi, o);
      if (ob > best || (ob == best && oi < bi)) {
        best = ob;
        bi = oi;
      }
    }
    if (lane == 0) {
      w_best[warp] = best;
      w_idx[warp] = bi;
    }
    __syncthreads();
    if (warp == 0) {
      best = lane < nwarps ? w_best[lane] : -1.0;
      bi = lane < nwarps ? w_idx[lane] : n;
      for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_down_sync(0xffffffffu, best, o);
        const int oi = __shfl_down_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi < bi)) {
          best = ob;
          bi = oi;
        }
      }
      if (lane == 0) {
        cand[0] = best;
        cand[1] = (double)bi;
      }
    }
    cl.sync();
    // every CTA reduces the candidates alike
    if (t == 0) {
      double b = -1.0;
      int p = n;
      for (int c = 0; c < C; ++c) {
        const double* oc = cl.map_shared_rank(cand, c);
        const double ob = oc[0];
        const int oi = (int)oc[1];
        if (ob > b || (ob == b && oi < p)) {
          b = ob;
          p = oi;
        }
      }
      if (!(b > 0.0) || !isfinite(b) || p >= n) {
        if (me == 0) atomicExch(status, PMB_ERR_PIVOT);
        p = k;
      }
      s_p = p;
      piv[k] = p;
    }
    __syncthreads();
    const int p = s_p;
    if (p != k) {
      // the owners of rows k and p each copy in the other row, then store it
      const bool own_k = k >= r0 && k < r1, own_p = p >= r0 && p < r1;
      if (own_k) {
        const double* src = row_of(p);
        for (int j = t; j < n; j += nt) tmp[j] = src[j];
      }
      if (own_p && !own_k) {
        const double* src = row_of(k);
        for (int j = t; j < n; j += nt) tmp[j] = src[j];
      }
      cl.sync();
      if (own_k && own_p) {
        double* rk = rows + (size_t)(k - r0) * n;
        double* rp = rows + (size_t)(p - r0) * n;
        for (int j = t; j < n; j += nt) {
          rp[j] = rk[j];
          rk[j] = tmp[j];
        }
      } else if (own_k) {
        double* rk = rows + (size_t)(k - r0) * n;
        for (int j = t; j < n; j += nt) rk[j] = tmp[j];
      } else if (own_p) {
        double* rp = rows + (size_t)(p - r0) * n;
        for (int j = t; j < n; j += nt) rp[j] = tmp[j];
      }
      cl.sync();
    }
    {
      const double* rk = row_of(k);
      const double d = rk[k];
      const double inv_d = (d != 0.0 && isfinite(d)) ? 1.0 / d : 1.0;
      for (int j = t; j < n; j += nt) prow[j] = j == k ? inv_d : rk[j] * inv_d;
      for (int i = r0 + t; i < r1; i += nt) fcol[i - r0] = i == k ? 0.0 : rows[(size_t)(i - r0) * n + k];
    }
    cl.sync();  // row k is read by every CTA before its owner overwrites it
    for (int i = r0 + warp; i < r1; i += nwarps) {
      double* ri = rows + (size_t)(i - r0) * n;
      if (i == k) {
        for (int j = lane; j < n; j += 32) ri[j] = prow[j];
      } else {
        const double f = fcol[i - r0];
        for (int j = lane; j < n; j += 32) ri[j] = (j == k ? 0.0 : ri[j]) - f * prow[j];
      }
    }
    __syncthreads();
  }
  for (int k = n - 1; k >= 0; --k) {
    const int p = piv[k];
    if (p != k)
      for (int r = r0 + t; r < r1; r += nt) {
        double* rr = rows + (size_t)(r - r0) * n;
        const double a = rr[k];
        rr[k] = rr[p];
        rr[p] = a;
      }
    __syncthreads();
  }
  for (int i = r0 + warp; i < r1; i += nwarps)
    for (int j = lane; j < n; j += 32) Inv[(size_t)i * n + j] = rows[(size_t)(i - r0) * n + j];
  cl.sync();  // no CTA leaves while another may still read its rows
}

// Cluster size and shared memory of gauss_jordan_cluster_kernel for n, or 0
// when one CTA holds the whole matrix or no cluster of at most 8 does.
static int gj_cluster_layout(int n, size_t& smem) {
  const char* e = std::getenv("PMB_GJ_CLUSTER");
  if (e && e[0] == '0') return 0;
  int dev = 0, optin = 0;
  PMB_CUDA(cudaGetDevice(&dev));
  PMB_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  const long long budget = (long long)optin - 1024;
  if (3LL * n * sizeof(double) + (long long)n * n * sizeof(double) + (long long)n * sizeof(int) <= budget)
    return 0;  // one CTA holds it
  for (int C : {2, 4, 8}) {
    const int R = (n + C - 1) / C;
    const long long need = ((long long)R * n + 2LL * n + R + 2) * sizeof(double) + (long long)n * sizeof(int);
    if (need > budget) continue;
    if (cudaFuncSetAttribute(gauss_jordan_cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)budget) != cudaSuccess) {
      (void)cudaGetLastError();
      return 0;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(C);
    cfg.blockDim = dim3(kGJThreads);
    cfg.dynamicSmemBytes = (size_t)need;
    cudaLaunchAttribute a[1];
    a[0].id = cudaLaunchAttributeClusterDimension;
    a[0].val.clusterDim.x = C;
    a[0].val.clusterDim.y = 1;
    a[0].val.clusterDim.z = 1;
    cfg.attrs = a;
    cfg.numAttrs = 1;
    int active = 0;
    if (cudaOccupancyMaxActiveClusters(&active, gauss_jordan_cluster_kernel, &cfg) != cudaSuccess || active < 1) {
      (void)cudaGetLastError();
      continue;
    }
    smem = (size_t)need;
    return C;
  }
  return 0;
}

static void gj_cluster_launch(int C, size_t smem, int n, const double* a, double* inv, int* d_status,
                              cudaStream_t s) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(C);
  cfg.blockDim = dim3(kGJThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = C;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  const int R = (n + C - 1) / C;
  PMB_CUDA(cudaLaunchKernelEx(&cfg, gauss_jordan_cluster_kernel, n, R, a, inv, d_status));
  PMB_CHECK_LAUNCH();
}

// Rows of an n x n Gauss-Jordan working matrix that fit in shared memory, and
// the kernel's dynamic shared memory for them.  The kernel's limit is raised
// once to the whole opt-in budget (the same value for every caller), so that
// hierarchies with different coarsest sizes never lower it for one another.
static void gj_layout(int n, int& rows, size_t& smem) {
  int dev = 0, optin = 0;
  PMB_CUDA(cudaGetDevice(&dev));
  PMB_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  const long long budget = (long long)optin - 1024;  // the kernel's static shared memory
  const long long fixed = 2LL * n * sizeof(double) + (long long)n * sizeof(int);
  PMB_REQUIRE(n >= 1 && fixed <= budget, "dense matrix too large for the one-CTA inverse");
  rows = (int)std::min<long long>(n, (budget - fixed) / ((long long)n * sizeof(double)));
  smem = (size_t)(fixed + (long long)rows * n * sizeof(double));
  PMB_CUDA(cudaFuncSetAttribute(gauss_jordan_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)budget));
}

void dense_inverse(int n, const double* a, double* inv, int* d_status, cudaStream_t s) {
  size_t csmem = 0;
  const int C = gj_cluster_layout(n, csmem);
  if (C > 0) {
    gj_cluster_launch(C, csmem, n, a, inv, d_status, s);
    return;
  }
  int rows = 0;
  size_t smem = 0;
  gj_layout(n, rows, smem);
  gauss_jordan_kernel<<<1, kGJThreads, smem, s>>>(n, rows, a, inv, d_status);
  PMB_CHECK_LAUNCH();
}

template <class T>
__global__ void dense_apply_kernel(int n, const double* __restrict__ Inv, const T* __restrict__ b,
                                   T* __restrict__ x) {
  pdl_enter();
  const int lane = threadIdx.x & 31;
  const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (row >= n) return;
  double s = 0.0;
  for (int j = lane; j < n; j += 32) s = __fma_rn(Inv[(size_t)row * n + j], (double)b[j], s);
  s = warp_sum(s);
  if (lane == 0) x[row] = (T)s;
}

// Sum over a group of `lanes` consecutive lanes (a power of two <= 32), the
// order of group_sum<LANES>.
__device__ __forceinline__ double group_sum_rt(double v, int lanes) {
  for (int o = lanes >> 1; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Cluster tail cycle --------------------------------------------------------
//
// The V-cycle from level `first` (a level below the K-cycle levels) down to
// the dense coarsest solve, as ONE launch of one thread-block cluster whose
// shared memory holds those levels.  Every level's rows are split into
// contiguous chunks, one per CTA; a CTA keeps its rows' matrix entries,
// vectors and restriction lists in its own shared memory, and reads the
// other chunks' vector entries through distributed shared memory.  A column
// (or a member row, or an aggregate) is stored packed as (owning CTA << 16)
// | row within that CTA's chunk.  The steps of the per-step path (Chebyshev
// steps, member residuals, aggregate sums, the dense coarsest product, the
// prolongation and post-smoothing) are separated by the hardware cluster
// barrier instead of kernel boundaries, with the same row grouping, sum
// order and explicit roundings as the per-step kernels, so the result is
// bitwise that of the per-step path.  On these levels a launch per step
// costs more than its work, and under the K-cycle every cycle visits them 8
// times; here every dependent load of a step is a shared-memory access.
constexpr int kTailThreads = 1024;
constexpr int kTailMaxRows = 65536;
constexpr int kFusedMaxRows = 65536;  // the largest level of the fused coarse cycle
constexpr int kEllMinRows = 262144;   // the smallest level with an ELL copy

template <class T>
__device__ __forceinline__ T* ct_sec(unsigned char* base, int off) {
  return reinterpret_cast<T*>(base + off);
}

// The entry `p` (packed) of the section at offset `off`, in its owner's
// shared memory.
template <class V>
__device__ __forceinline__ V ct_remote(cg::cluster_group& cl, unsigned char* base, int off, unsigned p) {
  V* loc = reinterpret_cast<V*>(base + off) + (p & 0xffffu);
  return *cl.map_shared_rank(loc, (int)(p >> 16));
}

// One Chebyshev step of level L on the CTA's rows: xout = xin + d,
// d = c1 d + c2 D^-1 (b - A xin); ZERO: from xin = 0 (no product).
template <class T, bool ZERO>
__device__ void ct_step(cg::cluster_group& cl, unsigned char* sm, const CtLevel<T>& L, const CtPart& P, int sin,
                        int sout, int step) {
  const double c1 = L.tab[1 + 2 * step], c2 = L.tab[2 + 2 * step];
  const int LN = L.lanes;
  const int* rp = ct_sec<int>(sm, L.s_rp);
  const unsigned* col = ct_sec<unsigned>(sm, L.s_col);
  const T* val = ct_sec<T>(sm, L.s_val);
  const T* dinv = ct_sec<T>(sm, L.s_dinv);
  const T* b = ct_sec<T>(sm, L.s_b);
  const T* xin = ct_sec<T>(sm, sin);
  T* xout = ct_sec<T>(sm, sout);
  T* d = ct_sec<T>(sm, L.s_d);
  const int total = (P.nr * LN + 31) / 32 * 32;
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    const int i = t / LN, sub = t % LN;
    double ax = 0.0;
    if (!ZERO) {
      if (i < P.nr)
        for (int k = rp[i] + sub; k < rp[i + 1]; k += LN)
          ax = __fma_rn((double)val[k], (double)ct_remote<T>(cl, sm, sin, col[k]), ax);
      ax = group_sum_rt(ax, LN);
    }
    if (i < P.nr && sub == 0) {
      const double r = cheb_res((double)b[i], ax, (double)dinv[i]);
      const double dn = cheb_dir(step, c1, c2, step == 0 ? 0.0 : (double)d[i], r);
      d[i] = (T)dn;
      xout[i] = (T)__dadd_rn(ZERO ? 0.0 : (double)xin[i], dn);
    }
  }
  cl.sync();
}

// AMG<T>::smooth on the CTA's rows, buffer for buffer.
template <class T>
__device__ void ct_smooth(cg::cluster_group& cl, unsigned char* sm, const CtLevel<T>& L, const CtPart& P,
                          bool zero_start) {
  const int steps = L.steps;
  int cur = L.s_x;
  int step = 0;
  if (zero_start) {
    const int out = (steps % 2 == 1) ? L.s_x : L.s_t;
    ct_step<T, true>(cl, sm, L, P, L.s_x, out, 0);
    cur = out;
    step = 1;
  }
  for (; step < steps; ++step) {
    int out = ((steps - 1 - step) % 2 == 0) ? L.s_x : L.s_t;
    if (out == cur) out = L.s_u;
    ct_step<T, false>(cl, sm, L, P, cur, out, step);
    cur = out;
  }
  if (cur != L.s_x) {
    T* x = ct_sec<T>(sm, L.s_x);
    const T* c = ct_sec<T>(sm, cur);
    for (int i = threadIdx.x; i < P.nr; i += blockDim.x) x[i] = c[i];
    cl.sync();
  }
}

template <class T>
__global__ void __launch_bounds__(kTailThreads, 1)
    amg_ctail_kernel(const CtLevel<T>* __restrict__ lv, const CtPart* __restrict__ parts, int nlev, CtCoarse co,
                     const T* b_top, T* x_top) {
  extern __shared__ __align__(16) unsigned char sm[];
  cg::cluster_group cl = cg::this_cluster();
  const int me = (int)cl.block_rank();
  const CtPart* my = parts + (size_t)me * (nlev + 1);  // nlev levels, then the coarsest rows
  // the hierarchy's entries (written at a refresh, never inside a cycle):
  // loaded before the wait on the predecessor grid
  for (int j = 0; j < nlev; ++j) {
    const CtLevel<T>& L = lv[j];
    const CtPart P = my[j];
    int* rp = ct_sec<int>(sm, L.s_rp);
    for (int k = threadIdx.x; k <= P.nr; k += blockDim.x) rp[k] = L.rp[P.r0 + k] - P.z0;
    unsigned* col = ct_sec<unsigned>(sm, L.s_col);
    T* val = ct_sec<T>(sm, L.s_val);
    for (int k = threadIdx.x; k < P.nz; k += blockDim.x) {
      col[k] = L.pcol[P.z0 + k];
      val[k] = L.val[P.z0 + k];
    }
    T* dinv = ct_sec<T>(sm, L.s_dinv);
    unsigned* agg = ct_sec<unsigned>(sm, L.s_agg);
    for (int k = threadIdx.x; k < P.nr; k += blockDim.x) {
      dinv[k] = L.dinv[P.r0 + k];
      agg[k] = L.pagg[P.r0 + k];
    }
    int* cptr = ct_sec<int>(sm, L.s_cptr);
    for (int k = threadIdx.x; k <= P.ncr; k += blockDim.x) cptr[k] = L.cptr[P.R0 + k] - P.m0;
    unsigned* mem = ct_sec<unsigned>(sm, L.s_mem);
    for (int k = threadIdx.x; k < P.nm; k += blockDim.x) mem[k] = L.pmem[P.m0 + k];
  }
  const CtPart PC = my[nlev];  // coarsest rows [r0, r0 + nr)
  {
    double* inv = ct_sec<double>(sm, co.s_inv);
    const long long cnt = (long long)PC.nr * co.nco;
    const double* src = co.inv + (long long)PC.r0 * co.nco;
    for (long long k = threadIdx.x; k < cnt; k += blockDim.x) inv[k] = src[k];
    unsigned* pco = ct_sec<unsigned>(sm, co.s_pco);
    for (int k = threadIdx.x; k < co.nco; k += blockDim.x) pco[k] = co.pco[k];
  }
  pdl_enter();
  {
    const CtLevel<T>& L = lv[0];
    const CtPart P = my[0];
    T* b = ct_sec<T>(sm, L.s_b);
    for (int k = threadIdx.x; k < P.nr; k += blockDim.x) b[k] = b_top[P.r0 + k];
  }
  cl.sync();
  for (int j = 0; j < nlev; ++j) {
    const CtLevel<T>& L = lv[j];
    const CtPart P = my[j];
    ct_smooth(cl, sm, L, P, true);
    // restrict_rows_kernel: member residuals b_i - (A x)_i of the CTA's rows ...
    {
      const int LN = L.lanes;
      const int* rp = ct_sec<int>(sm, L.s_rp);
      const unsigned* col = ct_sec<unsigned>(sm, L.s_col);
      const T* val = ct_sec<T>(sm, L.s_val);
      const T* b = ct_sec<T>(sm, L.s_b);
      double* rr = ct_sec<double>(sm, L.s_rr);
      const int total = (P.nr * LN + 31) / 32 * 32;
      for (int t = threadIdx.x; t < total; t += blockDim.x) {
        const int i = t / LN, sub = t % LN;
        double s = 0.0;
        if (i < P.nr)
          for (int k = rp[i] + sub; k < rp[i + 1]; k += LN)
            s = __fma_rn(-(double)val[k], (double)ct_remote<T>(cl, sm, L.s_x, col[k]), s);
        s = group_sum_rt(s, LN);
        if (i < P.nr && sub == 0) rr[i] = __dadd_rn((double)b[i], s);
      }
      cl.sync();
    }
    // ... summed per aggregate in member order into the next level's b
    {
      const int* cptr = ct_sec<int>(sm, L.s_cptr);
      const unsigned* mem = ct_sec<unsigned>(sm, L.s_mem);
      T* bc = j + 1 < nlev ? ct_sec<T>(sm, lv[j + 1].s_b) : ct_sec<T>(sm, co.s_b);
      for (int I = threadIdx.x; I < P.ncr; I += blockDim.x) {
        double v = 0.0;
        for (int m = cptr[I]; m < cptr[I + 1]; ++m) v = __dadd_rn(v, ct_remote<double>(cl, sm, L.s_rr, mem[m]));
        bc[I] = (T)v;
      }
      cl.sync();
    }
  }
  // dense_apply_kernel: one warp per row of the coarsest inverse, on the
  // whole coarse right-hand side gathered into every CTA
  {
    const unsigned* pco = ct_sec<unsigned>(sm, co.s_pco);
    T* bfull = ct_sec<T>(sm, co.s_bfull);
    for (int k = threadIdx.x; k < co.nco; k += blockDim.x) bfull[k] = ct_remote<T>(cl, sm, co.s_b, pco[k]);
    __syncthreads();
    const double* inv = ct_sec<double>(sm, co.s_inv);
    T* cx = ct_sec<T>(sm, co.s_x);
    const int lane = threadIdx.x & 31, nwarp = blockDim.x >> 5;
    for (int r = threadIdx.x >> 5; r < PC.nr; r += nwarp) {
      double s = 0.0;
      for (int k = lane; k < co.nco; k += 32) s = __fma_rn(inv[(long long)r * co.nco + k], (double)bfull[k], s);
      s = warp_sum(s);
      if (lane == 0) cx[r] = (T)s;
    }
    cl.sync();
  }
  // post-smoothing from the prolonged correction, back up to the first level
  for (int j = nlev - 1; j >= 0; --j) {
    const CtLevel<T>& L = lv[j];
    const CtPart P = my[j];
    {
      // prolong_add_kernel: x += P xc (the folded first step of the
      // per-step path reads these same values)
      const int sxc = j + 1 < nlev ? lv[j + 1].s_x : co.s_x;
      T* x = ct_sec<T>(sm, L.s_x);
      const unsigned* agg = ct_sec<unsigned>(sm, L.s_agg);
      for (int i = threadIdx.x; i < P.nr; i += blockDim.x)
        x[i] = (T)__dadd_rn((double)x[i], (double)ct_remote<T>(cl, sm, sxc, agg[i]));
      cl.sync();
    }
    ct_smooth(cl, sm, L, P, false);
  }
  {
    const CtLevel<T>& L = lv[0];
    const CtPart P = my[0];
    const T* x = ct_sec<T>(sm, L.s_x);
    for (int k = threadIdx.x; k < P.nr; k += blockDim.x) x_top[P.r0 + k] = x[k];
  }
}

// Fused coarse cycle (opt-in) ----------------------------------------------
//
// The V-cycle from level `first` down to the dense coarsest solve in one
// cooperative launch, the steps separated by a grid barrier: the same
// arithmetic, row grouping and buffer order as the per-step kernels, so the
// result is the same; what goes is one launch per step on levels of a few
// thousand rows.

constexpr long long kBarrierSpins = 1LL << 25;  // polls of an L2 line: a second or so

// Grid barrier for a cooperative launch.  Bounded: a block that waits too
// long records PMB_ERR_INTERNAL in *status and goes on; once the status is
// set, every later barrier returns at once, so a fault cannot hang the GPU.
__device__ __forceinline__ void grid_barrier(unsigned int* bar, int* status) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned int* gen = bar + 1;
    volatile int* st = status;
    if (*st == 0) {
      const unsigned int g = *gen;
      __threadfence();
      if (atomicAdd(bar, 1u) == gridDim.x - 1) {
        bar[0] = 0;
        __threadfence();
        atomicAdd(bar + 1, 1u);
      } else {
        long long spins = 0;
        while (*gen == g) {
          if (*st != 0) break;
          if (++spins > kBarrierSpins) {
            atomicExch(status, PMB_ERR_INTERNAL);
            break;
          }
        }
      }
      __threadfence();
    }
  }
  __syncthreads();
}


template <class T, bool ZERO>
__device__ void fused_cheb_rows(const CoopLevel<T>& L, const T* b, const T* xin, T* xout, int step, long long tid,
                                long long nthr) {
  const double c1 = L.lmax[1 + 2 * step], c2 = L.lmax[2 + 2 * step];
  const long long total = ((long long)L.n * L.lanes + 31) / 32 * 32;
  for (long long t = tid; t < total; t += nthr) {
    const long long i = t / L.lanes;
    const int sub = (int)(t % L.lanes);
    double ax = 0.0;
    if (!ZERO) {
      if (i < L.n)
        for (int k = L.rp[i] + sub; k < L.rp[i + 1]; k += L.lanes) ax += (double)L.val[k] * (double)xin[L.ci[k]];
      ax = group_sum_rt(ax, L.lanes);
    }
    if (i < L.n && sub == 0) {
      const double r = ((double)b[i] - ax) * (double)L.dinv[i];
      const double dn = (step == 0 ? 0.0 : c1 * (double)L.d[i]) + c2 * r;
      L.d[i] = (T)dn;
      xout[i] = (T)((ZERO ? 0.0 : (double)xin[i]) + dn);
    }
  }
}

template <class T>
__device__ void fused_smooth(const CoopLevel<T>& L, const T* b, T* x, bool zero_start, int degree, long long tid,
                             long long nthr, unsigned int* bar, int* status) {
  const int steps = degree < 1 ? 1 : degree;
  T* cur = x;
  int step = 0;
  if (zero_start) {
    T* out = (steps % 2 == 1) ? x : L.t;
    fused_cheb_rows<T, true>(L, b, nullptr, out, 0, tid, nthr);
    grid_barrier(bar, status);
    cur = out;
    step = 1;
  }
  for (; step < steps; ++step) {
    T* out = (cur == x) ? L.t : x;
    fused_cheb_rows<T, false>(L, b, cur, out, step, tid, nthr);
    grid_barrier(bar, status);
    cur = out;
  }
  if (cur != x) {
    for (long long i = tid; i < L.n; i += nthr) x[i] = cur[i];
    grid_barrier(bar, status);
  }
}

template <class T>
__global__ void __launch_bounds__(256) amg_fused_cycle_kernel(const CoopLevel<T>* __restrict__ lv, int nlev,
                                                              int degree, int nco, const double* __restrict__ co_inv,
                                                              T* co_b, T* co_x, const T* b_top, T* x_top,
                                                              unsigned int* bar, int* status) {
  const long long nthr = (long long)gridDim.x * blockDim.x;
  const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  for (int j = 0; j < nlev; ++j) {
    const CoopLevel<T> L = lv[j];
    const T* b = j == 0 ? b_top : L.b;
    T* x = j == 0 ? x_top : L.x;
    fused_smooth(L, b, x, true, degree, tid, nthr, bar, status);
    // residual restricted to the next level
    T* bc = j + 1 < nlev ? lv[j + 1].b : co_b;
    const int nn = j + 1 < nlev ? lv[j + 1].n : nco;
    const long long total = ((long long)nn * L.lanes + 31) / 32 * 32;
    for (long long t = tid; t < total; t += nthr) {
      const long long I = t / L.lanes;
      const int sub = (int)(t % L.lanes);
      double sres = 0.0;
      if (I < nn)
        for (int m = L.cptr[I]; m < L.cptr[I + 1]; ++m) {
          const int i = L.cmem[m];
          if (sub == 0) sres += (double)b[i];
          for (int k = L.rp[i] + sub; k < L.rp[i + 1]; k += L.lanes) sres -= (double)L.val[k] * (double)x[L.ci[k]];
        }
      sres = group_sum_rt(sres, L.lanes);
      if (I < nn && sub == 0) bc[I] = (T)sres;
    }
    grid_barrier(bar, status);
  }
  // dense coarsest solve: one warp per row
  {
    const long long lane = tid & 31, nwarp = nthr >> 5;
    for (long long row = tid >> 5; row < nco; row += nwarp) {
      double sv = 0.0;
      for (long long jj = lane; jj < nco; jj += 32) sv += co_inv[row * nco + jj] * (double)co_b[jj];
      sv = warp_sum(sv);
      if (lane == 0) co_x[row] = (T)sv;
    }
    grid_barrier(bar, status);
  }
  for (int j = nlev - 1; j >= 0; --j) {
    const CoopLevel<T> L = lv[j];
    const T* b = j == 0 ? b_top : L.b;
    T* x = j == 0 ? x_top : L.x;
    const T* xc = j + 1 < nlev ? lv[j + 1].x : co_x;
    for (long long i = tid; i < L.n; i += nthr) x[i] = (T)((double)x[i] + (double)xc[L.agg[i]]);
    grid_barrier(bar, status);
    fused_smooth(L, b, x, false, degree, tid, nthr, bar, status);
  }
}

// K-cycle pieces ------------------------------------------------------------

template <class T, int LANES>
__global__ void __launch_bounds__(256) csr_spmv_kernel(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                                                       const T* __restrict__ a, const T* __restrict__ x,
                                                       T* __restrict__ y) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long i = t / LANES;
  const int sub = (int)(t % LANES);
  RowPre<T> p;
  if (i < n) p = row_prefetch<T, LANES>(i, sub, rp, ci, a);  // the matrix, before the wait
  pdl_enter();
  double s = 0.0;
  if (i < n) s = row_sum<T, LANES>(p, ci, a, 0.0, [=](double acc, double v, int j) {
      return __fma_rn(v, (double)x[j], acc);
    });
  s = group_sum<LANES>(s);
  if (i < n && sub == 0) y[i] = (T)s;
}

// NDOT = 2: [v1.v1, v1.rc]; NDOT = 5: [v1.v1, v1.v2, v2.v2, v1.rc, v2.rc]
template <class T, int NDOT>
__global__ void __launch_bounds__(256) kdots_kernel(int n, const T* __restrict__ v1, const T* __restrict__ v2,
                                                    const T* __restrict__ rc, double* __restrict__ part) {
  pdl_enter();
  __shared__ double sh[32];
  double d[NDOT];
  for (int q = 0; q < NDOT; ++q) d[q] = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double a = (double)v1[i], r = (double)rc[i];
    if (NDOT == 2) {
      d[0] += a * a;
      d[1] += a * r;
    } else {
      const double b = (double)v2[i];
      d[0] += a * a;
      d[1] += a * b;
      d[2] += b * b;
      d[3] += a * r;
      d[4] += b * r;
    }
  }
  for (int q = 0; q < NDOT; ++q) {
    const double s = block_sum(d[q], sh);
    if (threadIdx.x == 0) part[q * gridDim.x + blockIdx.x] = s;
  }
}

// The coefficients of one K-cycle step from the kdots partials, into c
// (shared memory): mode 0: c[0] = (v1.rc)/(v1.v1); mode 1: the least-squares
// pair [c[1], c[2]] minimising |rc - y0 v1 - y1 v2|.  One warp sums each
// dot's G block partials, in the same order in every CTA, so that every CTA
// gets the same values.  Needs at least 5 warps.
__device__ __forceinline__ void kcoef_block(int G, int mode, const double* __restrict__ part, double* c) {
  __shared__ double d[5];
  const int nd = mode == 0 ? 2 : 5;
  const int lane = threadIdx.x & 31, q = threadIdx.x >> 5;
  if (q < nd) {
    double s = 0.0;
    for (int b = lane; b < G; b += 32) s += part[q * G + b];
    s = warp_sum(s);
    if (lane == 0) d[q] = s;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (mode == 0) {
      c[0] = d[0] > 0.0 ? d[1] / d[0] : 0.0;
    } else {
      const double a11 = d[0], a12 = d[1], a22 = d[2], r1 = d[3], r2 = d[4];
      const double det = a11 * a22 - a12 * a12;
      if (det > 1e-14 * a11 * a22 && isfinite(det)) {
        c[1] = (a22 * r1 - a12 * r2) / det;
        c[2] = (a11 * r2 - a12 * r1) / det;
      } else {
        c[1] = a11 > 0.0 ? r1 / a11 : 0.0;
        c[2] = 0.0;
      }
    }
  }
  __syncthreads();
}

// out = a - c0 b, c0 = (v1.rc)/(v1.v1) from the kdots partials
template <class T>
__global__ void __launch_bounds__(256) kaxpy_kernel(int n, const T* __restrict__ a, const T* __restrict__ b, int G,
                                                    const double* __restrict__ part, T* __restrict__ out,
                                                    ZeroStep<T> zs) {
  pdl_enter();
  __shared__ double c[3];
  kcoef_block(G, 0, part, c);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const T o = (T)((double)a[i] - c[0] * (double)b[i]);
    out[i] = o;
    if (zs.dinv) zero_step(zs, i, o);
  }
}

// out = y0 c1 + y1 c2, (y0, y1) the least-squares pair from the kdots partials
template <class T>
__global__ void __launch_bounds__(256) kcombine_kernel(int n, const T* __restrict__ c1, const T* __restrict__ c2,
                                                       int G, const double* __restrict__ part, T* __restrict__ out) {
  pdl_enter();
  __shared__ double c[3];
  kcoef_block(G, 1, part, c);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = (T)(c[1] * (double)c1[i] + c[2] * (double)c2[i]);
}

// ---------------------------------------------------------------------------
// host class
// ---------------------------------------------------------------------------

template <class T>
void AMG<T>::build(int n, const std::vector<int>& h_row_ptr, const std::vector<int>& h_col,
                   const int* d_row_ptr, const int* d_col, const std::vector<double>& h_val,
                   double theta, int coarse_size, cudaStream_t s) {
  static const int aggressive = [] {
    const char* e = std::getenv("PMB_AMG_AGGRESSIVE_BELOW");
    return e ? std::atoi(e) : 0;
  }();
  PMB_REQUIRE(degree >= 0 && degree <= kMaxChebSteps && coarse_degree >= 0 && coarse_degree <= kMaxChebSteps,
              "the AMG smoother degree must be at most 16");
  auto H = amg_build_hierarchy(n, h_row_ptr.data(), h_col.data(), h_val.data(), theta, 2, coarse_size, 40,
                               aggressive);
  levels_.clear();
  levels_.resize(H.size() - 1);
  for (size_t l = 0; l + 1 < H.size(); ++l) {
    AMGLevel<T>& L = levels_[l];
    const AMGHostLevel& h = H[l];
    L.n = h.n;
    L.nnz = (int)h.col.size();
    if (l == 0) {
      L.row_ptr = d_row_ptr;
      L.col = d_col;
    } else {
      L.own_row_ptr.upload(h.row_ptr, s);
      L.own_col.upload(h.col, s);
      L.row_ptr = L.own_row_ptr.get();
      L.col = L.own_col.get();
    }
    L.lanes = lanes_for(L.n, L.nnz);
    L.degree = ((int)l >= k_levels && coarse_degree > 0) ? coarse_degree : 0;
    {
      // restriction plan: consecutive aggregates while their members fit
      // one per lane group
      const int groups = 256 / L.lanes;
      std::vector<int> blk(1, 0);
      size_t most = 0;
      const int nag = (int)h.cptr.size() - 1;
      PMB_REQUIRE(nag >= 1, "an AMG level without aggregates");
      for (int I = 0; I < nag;) {
        int J = I + 1;
        while (J < nag && h.cptr[J + 1] - h.cptr[I] <= groups) ++J;
        most = std::max<size_t>(most, (size_t)(h.cptr[J] - h.cptr[I]));
        blk.push_back(J);
        I = J;
      }
      L.rblocks = (int)blk.size() - 1;
      L.rsmem = std::max<size_t>(most, 1) * sizeof(double);
      PMB_REQUIRE(L.rsmem <= 48 * 1024, "an AMG aggregate has too many members for the restriction kernel");
      L.rblk.upload(blk, s);
    }
    L.val.resize(L.nnz);
    L.dinv.resize(L.n);
    L.x.resize(L.n);
    L.b.resize(L.n);
    L.r.resize(L.n);
    L.t.resize(L.n);
    L.u.resize(L.n);
    L.agg.upload(h.agg, s);
    L.cptr.upload(h.cptr, s);
    L.cmem.upload(h.cmem, s);
    L.gptr.upload(h.gptr, s);
    L.gidx.upload(h.gidx, s);
    L.lmax.resize(kChebTable);
    build_ell(L, h, s);
    if (l >= 1) {  // K-cycle work vectors of a coarse level
      L.kc1.resize(L.n);
      L.kc2.resize(L.n);
      L.kv1.resize(L.n);
      L.kv2.resize(L.n);
      L.kr2.resize(L.n);
      L.kpart.resize(5 * 2 * kNumSM);
    }
  }
  const AMGHostLevel& c = H.back();
  nco_ = c.n;
  PMB_REQUIRE(nco_ <= 4096, "coarsest AMG level too large for the dense solve");
  if (levels_.empty()) {
    // the whole matrix is the coarsest level: its pattern is the operator's
    co_row_ptr_.upload(c.row_ptr, s);
    co_col_.upload(c.col, s);
  } else {
    co_row_ptr_.upload(c.row_ptr, s);
    co_col_.upload(c.col, s);
  }
  co_nnz_ = (int)c.col.size();
  co_val_.resize(std::max(co_nnz_, 1));
  co_dense_.resize((size_t)nco_ * nco_);
  co_inv_.resize((size_t)nco_ * nco_);
  co_x_.resize(nco_);
  co_b_.resize(nco_);
  gj_layout(nco_, gj_rows_, gj_smem_);
  gj_cluster_ = gj_cluster_layout(nco_, gj_csmem_);
  bits_.resize(std::max<size_t>(levels_.size(), 1));
  build_fused(s);
  build_tail(H, s);
  PMB_CUDA(cudaStreamSynchronize(s));
}

template <class T>
static EllView<T> ell_view(const AMGLevel<T>& L) {
  EllView<T> E;
  E.n = L.n;
  E.K = L.ell_k;
  E.col = L.ell_dia ? nullptr : L.ell_col.get();
  E.val = L.ell_val.get();
  E.orow = L.ell_dia ? L.ell_orow.get() : nullptr;
  E.optr = L.ell_optr.get();
  E.ocol = L.ell_ovf > 0 ? L.ell_ocol.get() : nullptr;
  E.oval = L.ell_ovf > 0 ? L.ell_oval.get() : nullptr;
  for (int k = 0; k < kEllMaxK; ++k) E.off[k] = L.ell_off[k];
  return E;
}

// The ELL copy of a level, where it pays: rows of nearly equal length (at
// most 0.1% longer than the slot count, which is at most kEllMaxK, and the
// padding at most 30% of the entries), on levels of at least kEllMinRows
// rows (one thread per row needs a few waves of threads to hide its
// latency; PMB_AMG_ELL_MIN_ROWS changes the bound, never below the sizes the
// cluster tail and the fused cycle take: those read the CSR arrays and must
// give the per-step path's bits).  The diagonal form is taken where it fits, the
// column form otherwise.  PMB_AMG_ELL=0 keeps every level in CSR,
// PMB_AMG_ELL=1 allows only the column form.
template <class T>
void AMG<T>::build_ell(AMGLevel<T>& L, const AMGHostLevel& h, cudaStream_t s) {
  L.ell_k = 0;
  L.ell_ovf = 0;
  L.ell_dia = false;
  const char* e = std::getenv("PMB_AMG_ELL");
  const char* em = std::getenv("PMB_AMG_ELL_MIN_ROWS");
  const long long min_rows = std::max<long long>(em ? std::atoll(em) : kEllMinRows,
                                                 std::max(kTailMaxRows, kFusedMaxRows) + 1LL);
  if ((e && e[0] == '0') || L.n < min_rows) return;
  const int n = L.n;
  const long long nnz = h.row_ptr[n];
  if (!(e && e[0] == '1')) {
    // diagonal form: the fewest column offsets, most frequent first, that
    // hold all but 1% of the entries, with at most 1% of the rows reaching
    // off them (through the overflow list) and at most 30% padding
    std::unordered_map<int, long long> freq;
    for (int i = 0; i < n; ++i)
      for (int k = h.row_ptr[i]; k < h.row_ptr[i + 1]; ++k) ++freq[h.col[k] - i];
    std::vector<std::pair<long long, int>> byf;
    for (const auto& kv : freq) byf.push_back({kv.second, kv.first});
    std::sort(byf.begin(), byf.end(), [](const std::pair<long long, int>& a, const std::pair<long long, int>& b) {
      return a.first != b.first ? a.first > b.first : a.second < b.second;
    });
    long long covered = 0;
    for (int K = 1; K <= std::min<int>(kEllMaxK, (int)byf.size()); ++K) {
      covered += byf[K - 1].first;
      if ((nnz - covered) * 100 > nnz || (double)K * n > 1.3 * (double)nnz) continue;
      std::vector<int> off(K);
      for (int k = 0; k < K; ++k) off[k] = byf[k].second;
      std::sort(off.begin(), off.end());
      std::vector<int> src((size_t)K * n, -1), orow(n, -1), optr(1, 0), ocol, osrc;
      for (int i = 0; i < n; ++i) {
        bool extra = false;
        for (int q = h.row_ptr[i]; q < h.row_ptr[i + 1]; ++q) {
          const int d = h.col[q] - i;
          const int slot = (int)(std::find(off.begin(), off.end(), d) - off.begin());
          if (slot < K) {
            src[(size_t)slot * n + i] = q;
          } else {
            ocol.push_back(h.col[q]);
            osrc.push_back(q);
            extra = true;
          }
        }
        if (extra) {
          orow[i] = (int)optr.size() - 1;
          optr.push_back((int)ocol.size());
        }
      }
      if ((long long)(optr.size() - 1) * 100 > n) break;  // too many rows off the diagonals
      L.ell_src.upload(src, s);
      L.ell_val.resize((size_t)K * n);
      L.ell_orow.upload(orow, s);
      L.ell_optr.upload(optr, s);
      L.ell_ovf = (long long)ocol.size();
      if (!ocol.empty()) {
        L.ell_ocol.upload(ocol, s);
        L.ell_osrc.upload(osrc, s);
        L.ell_oval.resize(ocol.size());
      }
      for (int k = 0; k < kEllMaxK; ++k) L.ell_off[k] = k < K ? off[k] : 0;
      L.ell_rr.resize(n);
      L.ell_k = K;
      L.ell_dia = true;
      return;
    }
  }
  std::vector<long long> count(kEllMaxK + 2, 0);  // rows of each length, the last bin longer
  for (int i = 0; i < n; ++i) ++count[std::min(h.row_ptr[i + 1] - h.row_ptr[i], kEllMaxK + 1)];
  int K = 0;
  long long over = 0;  // rows longer than k
  for (int q = 1; q <= kEllMaxK + 1; ++q) over += count[q];
  for (int k = 1; k <= kEllMaxK; ++k) {
    over -= count[k];
    if (over * 1000 <= n) {
      K = k;
      break;
    }
  }
  if (K < 2 || (double)K * n > 1.3 * (double)L.nnz) return;
  std::vector<int> col((size_t)K * n), src((size_t)K * n), optr(1, 0), ocol, osrc;
  for (int i = 0; i < n; ++i) {
    const int a = h.row_ptr[i], len = h.row_ptr[i + 1] - a;
    const int in_slots = len > K ? K - 1 : len;
    for (int k = 0; k < K; ++k) {
      const size_t at = (size_t)k * n + i;
      if (k < in_slots) {
        col[at] = h.col[a + k];
        src[at] = a + k;
      } else {
        col[at] = i;
        src[at] = -1;
      }
    }
    if (len > K) {
      col[(size_t)(K - 1) * n + i] = -1 - ((int)optr.size() - 1);
      for (int q = in_slots; q < len; ++q) {
        ocol.push_back(h.col[a + q]);
        osrc.push_back(a + q);
      }
      optr.push_back((int)ocol.size());
    }
  }
  L.ell_col.upload(col, s);
  L.ell_src.upload(src, s);
  L.ell_val.resize((size_t)K * n);
  L.ell_optr.upload(optr, s);
  L.ell_ovf = (long long)ocol.size();
  if (!ocol.empty()) {
    L.ell_ocol.upload(ocol, s);
    L.ell_osrc.upload(osrc, s);
    L.ell_oval.resize(ocol.size());
  }
  L.ell_rr.resize(n);
  L.ell_k = K;
}

// The cluster tail's layout: from the first level below the K-cycle levels
// with at most PMB_AMG_TAIL_ROWS rows (at most 65,536; unset or 0: the
// per-step kernels) whose levels, down to the coarsest, fit the shared
// memory of a cluster of 16 (else 8) CTAs; a level that does not fit moves
// the start one level down.
template <class T>
void AMG<T>::build_tail(const std::vector<AMGHostLevel>& H, cudaStream_t s) {
  tail_start_ = -1;
  tail_cluster_ = 0;
  const char* e = std::getenv("PMB_AMG_TAIL_ROWS");
  const int max_rows = e ? std::min(std::atoi(e), kTailMaxRows) : 0;
  const int L = (int)levels_.size();
  if (max_rows <= 0 || L == 0 || nco_ < 1) return;
  int dev = 0, smem_max = 0;
  PMB_CUDA(cudaGetDevice(&dev));
  PMB_CUDA(cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  for (int first = std::max(0, k_levels); first < L; ++first) {
    if (levels_[first].n > max_rows) continue;
    for (int C : {16, 8}) {
      // row chunks: level rows balanced by entries, coarsest rows evenly
      const int nq = L - first;
      std::vector<std::vector<int>> cut(nq + 1, std::vector<int>(C + 1, 0));
      for (int q = 0; q < nq; ++q) {
        const AMGHostLevel& h = H[first + q];
        const long long nnz = h.row_ptr[h.n];
        int r = 0;
        for (int c = 1; c < C; ++c) {
          const long long want = nnz * c / C;
          while (r < h.n && h.row_ptr[r] < want) ++r;
          cut[q][c] = r;
        }
        cut[q][C] = h.n;
      }
      for (int c = 0; c <= C; ++c) cut[nq][c] = (int)((long long)nco_ * c / C);
      bool ok = true;
      for (int q = 0; q <= nq && ok; ++q)
        for (int c = 0; c < C; ++c)
          if (cut[q][c + 1] - cut[q][c] > 65535) ok = false;
      if (!ok) continue;
      auto pack = [&](int q, int g) -> unsigned {
        const std::vector<int>& k = cut[q];
        const int c = (int)(std::upper_bound(k.begin(), k.end(), g) - k.begin()) - 1;
        return ((unsigned)c << 16) | (unsigned)(g - k[c]);
      };
      // shared-memory layout (the largest chunk of every section)
      size_t off = 0;
      auto take = [&](size_t bytes) {
        const size_t at = off;
        off += (bytes + 15) / 16 * 16;
        return (int)at;
      };
      std::vector<CtLevel<T>> lv(nq);
      std::vector<CtPart> parts((size_t)C * (nq + 1));
      for (int q = 0; q < nq; ++q) {
        const AMGHostLevel& h = H[first + q];
        int NR = 0, NZ = 0, NC = 0, NM = 0;
        for (int c = 0; c < C; ++c) {
          CtPart& P = parts[(size_t)c * (nq + 1) + q];
          P.r0 = cut[q][c];
          P.nr = cut[q][c + 1] - P.r0;
          P.z0 = h.row_ptr[P.r0];
          P.nz = h.row_ptr[P.r0 + P.nr] - P.z0;
          P.R0 = cut[q + 1][c];
          P.ncr = cut[q + 1][c + 1] - P.R0;
          P.m0 = h.cptr[P.R0];
          P.nm = h.cptr[P.R0 + P.ncr] - P.m0;
          NR = std::max(NR, P.nr);
          NZ = std::max(NZ, P.nz);
          NC = std::max(NC, P.ncr);
          NM = std::max(NM, P.nm);
        }
        CtLevel<T>& t = lv[q];
        const AMGLevel<T>& V = levels_[first + q];
        t.lanes = V.lanes;
        t.steps = std::max(1, V.degree > 0 ? V.degree : degree);
        t.s_rp = take(4 * (size_t)(NR + 1));
        t.s_col = take(4 * (size_t)NZ);
        t.s_val = take(sizeof(T) * (size_t)NZ);
        t.s_dinv = take(sizeof(T) * (size_t)NR);
        t.s_b = take(sizeof(T) * (size_t)NR);
        t.s_x = take(sizeof(T) * (size_t)NR);
        t.s_t = take(sizeof(T) * (size_t)NR);
        t.s_u = take(sizeof(T) * (size_t)NR);
        t.s_d = take(sizeof(T) * (size_t)NR);
        t.s_rr = take(8 * (size_t)NR);
        t.s_agg = take(4 * (size_t)NR);
        t.s_cptr = take(4 * (size_t)(NC + 1));
        t.s_mem = take(4 * (size_t)NM);
      }
      int NRC = 0;
      for (int c = 0; c < C; ++c) {
        CtPart& P = parts[(size_t)c * (nq + 1) + nq];
        P = CtPart{cut[nq][c], cut[nq][c + 1] - cut[nq][c], 0, 0, 0, 0, 0, 0};
        NRC = std::max(NRC, P.nr);
      }
      CtCoarse co{};
      co.nco = nco_;
      co.s_inv = take(8 * (size_t)NRC * nco_);
      co.s_b = take(sizeof(T) * (size_t)NRC);
      co.s_x = take(sizeof(T) * (size_t)NRC);
      co.s_pco = take(4 * (size_t)nco_);
      co.s_bfull = take(sizeof(T) * (size_t)nco_);
      if (off > (size_t)smem_max) continue;
      // the cluster must be schedulable with this shared memory
      if (C > 8 && cudaFuncSetAttribute(amg_ctail_kernel<T>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
                       cudaSuccess) {
        (void)cudaGetLastError();
        continue;
      }
      if (cudaFuncSetAttribute(amg_ctail_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)off) !=
          cudaSuccess) {
        (void)cudaGetLastError();
        continue;
      }
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(C);
      cfg.blockDim = dim3(kTailThreads);
      cfg.dynamicSmemBytes = off;
      cudaLaunchAttribute a[1];
      a[0].id = cudaLaunchAttributeClusterDimension;
      a[0].val.clusterDim.x = C;
      a[0].val.clusterDim.y = 1;
      a[0].val.clusterDim.z = 1;
      cfg.attrs = a;
      cfg.numAttrs = 1;
      int active = 0;
      if (cudaOccupancyMaxActiveClusters(&active, amg_ctail_kernel<T>, &cfg) != cudaSuccess || active < 1) {
        (void)cudaGetLastError();
        continue;
      }
      // packed indices on the device
      for (int q = 0; q < nq; ++q) {
        const AMGHostLevel& h = H[first + q];
        AMGLevel<T>& V = levels_[first + q];
        std::vector<unsigned> pcol(h.col.size()), pagg(h.n), pmem(h.cmem.size());
        for (size_t k = 0; k < h.col.size(); ++k) pcol[k] = pack(q, h.col[k]);
        for (int i = 0; i < h.n; ++i) pagg[i] = pack(q + 1, h.agg[i]);
        for (size_t m = 0; m < h.cmem.size(); ++m) pmem[m] = pack(q, h.cmem[m]);
        V.ct_pcol.upload(pcol, s);
        V.ct_pagg.upload(pagg, s);
        V.ct_pmem.upload(pmem, s);
        CtLevel<T>& t = lv[q];
        t.val = V.val.get();
        t.dinv = V.dinv.get();
        t.pcol = V.ct_pcol.get();
        t.rp = V.row_ptr;
        t.pagg = V.ct_pagg.get();
        t.cptr = V.cptr.get();
        t.pmem = V.ct_pmem.get();
        t.tab = V.lmax.get();
      }
      std::vector<unsigned> pco(nco_);
      for (int g = 0; g < nco_; ++g) pco[g] = pack(nq, g);
      ct_pco_.upload(pco, s);
      co.inv = co_inv_.get();
      co.pco = ct_pco_.get();
      tail_levels_.resize(sizeof(CtLevel<T>) * lv.size());
      PMB_CUDA(cudaMemcpyAsync(tail_levels_.get(), lv.data(), sizeof(CtLevel<T>) * lv.size(),
                               cudaMemcpyHostToDevice, s));
      tail_parts_.upload(parts, s);
      tail_co_ = co;
      tail_smem_ = off;
      tail_start_ = first;
      tail_cluster_ = C;
      return;
    }
  }
}

template <class T>
void AMG<T>::launch_tail(const T* b, T* x, cudaStream_t s) {
  const CtLevel<T>* lv = reinterpret_cast<const CtLevel<T>*>(tail_levels_.get());
  const int nlev = (int)levels_.size() - tail_start_;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(tail_cluster_);
  cfg.blockDim = dim3(kTailThreads);
  cfg.dynamicSmemBytes = tail_smem_;
  cfg.stream = s;
  cudaLaunchAttribute attr[2];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = tail_cluster_;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[1].val.programmaticStreamSerializationAllowed = pdl_enabled() ? 1 : 0;
  cfg.attrs = attr;
  cfg.numAttrs = 2;
  const CtPart* parts = tail_parts_.get();
  PMB_CUDA(cudaLaunchKernelEx(&cfg, amg_ctail_kernel<T>, lv, parts, nlev, tail_co_, b, x));
  PMB_CHECK_LAUNCH();
}

template <class T>
void AMG<T>::refresh(cudaStream_t s, int* d_status) {
  coop_status_ = d_status;
  for (size_t l = 0; l < levels_.size(); ++l) {
    AMGLevel<T>& L = levels_[l];
    if (L.ell_k > 0) {
      const long long tot = (long long)L.ell_k * L.n;
      ell_values_kernel<T><<<grid_for(tot, 256), 256, 0, s>>>(tot, L.ell_src.get(), L.val.get(), L.ell_val.get());
      PMB_CHECK_LAUNCH();
      if (L.ell_ovf > 0) {
        ell_values_kernel<T><<<grid_for(L.ell_ovf, 256), 256, 0, s>>>(L.ell_ovf, L.ell_osrc.get(), L.val.get(),
                                                                       L.ell_oval.get());
        PMB_CHECK_LAUNCH();
      }
    }
    PMB_CUDA(cudaMemsetAsync(bits_.get() + l, 0, sizeof(unsigned long long), s));
    diag_kernel<T><<<grid_for(L.n, 256), 256, 0, s>>>(L.n, L.row_ptr, L.col, L.val.get(), L.dinv.get(),
                                                       bits_.get() + l, d_status);
    PMB_CHECK_LAUNCH();
    cheb_table_kernel<<<1, 32, 0, s>>>(bits_.get() + l, L.lmax.get());
    PMB_CHECK_LAUNCH();
    const bool last = (l + 1 == levels_.size());
    T* cval = last ? co_val_.get() : levels_[l + 1].val.get();
    const int nnzc = last ? co_nnz_ : levels_[l + 1].nnz;
    galerkin_kernel<T><<<grid_for(nnzc, 256), 256, 0, s>>>(nnzc, L.gptr.get(), L.gidx.get(), L.val.get(), cval);
    PMB_CHECK_LAUNCH();
  }
  PhaseTimer pt("amg.refresh.coarse_inverse", s);
  dense_assemble_kernel<T><<<grid_for(nco_, 128), 128, 0, s>>>(nco_, co_row_ptr_.get(), co_col_.get(),
                                                                co_val_.get(), co_dense_.get());
  PMB_CHECK_LAUNCH();
  if (gj_cluster_ > 0) {
    gj_cluster_launch(gj_cluster_, gj_csmem_, nco_, co_dense_.get(), co_inv_.get(), d_status, s);
  } else {
    gauss_jordan_kernel<<<1, kGJThreads, gj_smem_, s>>>(nco_, gj_rows_, co_dense_.get(), co_inv_.get(), d_status);
    PMB_CHECK_LAUNCH();
  }
}

template <class T>
void AMG<T>::smooth(AMGLevel<T>& L, const T* b, T* x, cudaStream_t s, bool zero_start, const T* xc,
                    bool first_done) {
  // degree steps ping-pong between x and L.t, ordered so that the last one
  // writes x; the first step of an odd count from a non-zero start, which
  // would overwrite its own input, writes L.u instead.  Only a single step
  // from a non-zero start needs a copy.
  const int steps = std::max(1, L.degree > 0 ? L.degree : degree);
  T* t = L.t.get();
  T* u = L.u.get();
  auto out_for = [&](int k) -> T* { return ((steps - 1 - k) % 2 == 0) ? x : t; };
  T* cur = x;
  int step = 0;
  with_lanes(L.lanes, [&](auto ln) {
    constexpr int LN = decltype(ln)::value;
    const int g = grid_for((long long)L.n * LN, 256);
    if (zero_start) {
      T* out = (steps % 2 == 1) ? x : t;  // zero_step_for() names the same buffer
      if (!first_done)
        launch_pdl(cheb_step_kernel<T, true, LN>, g, 256, 0, s, L.n, L.row_ptr, L.col, (const T*)L.val.get(),
                   (const T*)L.dinv.get(), b, (const T*)nullptr, out, L.r.get(), (const double*)L.lmax.get(), 0,
                   (const int*)nullptr, (const T*)nullptr);
      cur = out;
      step = 1;
    }
    for (; step < steps; ++step) {
      T* out = out_for(step);
      if (out == cur) out = u;
      if (L.ell_k > 0) {
        const int ge = grid_for(L.n, 256);
        const EllView<T> E = ell_view(L);
        if (xc && step == 0)
          launch_pdl(cheb_ell_kernel<T, true>, ge, 256, 0, s, E, (const T*)L.dinv.get(), b, (const T*)cur, out,
                     L.r.get(), (const double*)L.lmax.get(), step, (const int*)L.agg.get(), xc);
        else
          launch_pdl(cheb_ell_kernel<T, false>, ge, 256, 0, s, E, (const T*)L.dinv.get(), b, (const T*)cur, out,
                     L.r.get(), (const double*)L.lmax.get(), step, (const int*)nullptr, (const T*)nullptr);
      } else if (xc && step == 0)  // x + P xc, folded into the first step
        launch_pdl(cheb_step_kernel<T, false, LN, true>, g, 256, 0, s, L.n, L.row_ptr, L.col, (const T*)L.val.get(),
                   (const T*)L.dinv.get(), b, (const T*)cur, out, L.r.get(), (const double*)L.lmax.get(), step,
                   (const int*)L.agg.get(), xc);
      else
        launch_pdl(cheb_step_kernel<T, false, LN>, g, 256, 0, s, L.n, L.row_ptr, L.col, (const T*)L.val.get(),
                   (const T*)L.dinv.get(), b, (const T*)cur, out, L.r.get(), (const double*)L.lmax.get(), step,
                   (const int*)nullptr, (const T*)nullptr);
      cur = out;
    }
  });
  if (cur != x) {
    launch_pdl(copy_kernel<T>, grid_for(L.n, 256), 256, 0, s, L.n, (const T*)cur, x);
  }
}

// Levels below this size fold the prolongation into the first post-smoothing
// step (one launch less per visit); on larger levels the extra gathers of agg
// and the correction cost more than the launch.
constexpr int kFoldProlongRows = 200000;

template <class T>
void AMG<T>::build_fused(cudaStream_t s) {
  coop_start_ = -1;
  // Off unless PMB_FUSED_COARSE=1: measured on the channelised model (528,000
  // cells, mixed precision) the fused cycle made a step 26% slower than the
  // per-step kernels replayed from the preconditioner's CUDA graph, with 1, 2
  // or 4 blocks per SM, although it launched 2.4x fewer kernels.
  static const bool enabled = [] {
    const char* e = std::getenv("PMB_FUSED_COARSE");
    return e && e[0] == '1';
  }();
  if (!fused_coarse || !enabled) return;
  const int L = (int)levels_.size();
  for (int l = std::max(0, k_levels); l < L; ++l)
    if (levels_[l].n <= kFusedMaxRows) {
      coop_start_ = l;
      break;
    }
  if (coop_start_ < 0) return;
  std::vector<CoopLevel<T>> h;
  for (int l = coop_start_; l < L; ++l) {
    AMGLevel<T>& V = levels_[l];
    CoopLevel<T> c;
    c.n = V.n;
    c.lanes = V.lanes;
    c.rp = V.row_ptr;
    c.ci = V.col;
    c.val = V.val.get();
    c.dinv = V.dinv.get();
    c.lmax = V.lmax.get();
    c.x = V.x.get();
    c.b = V.b.get();
    c.d = V.r.get();
    c.t = V.t.get();
    c.cptr = V.cptr.get();
    c.cmem = V.cmem.get();
    c.agg = V.agg.get();
    h.push_back(c);
  }
  coop_levels_.resize(sizeof(CoopLevel<T>) * h.size());
  PMB_CUDA(cudaMemcpyAsync(coop_levels_.get(), h.data(), sizeof(CoopLevel<T>) * h.size(), cudaMemcpyHostToDevice, s));
  coop_bar_.resize(2);
  coop_bar_.zero(s);
  int dev = 0, sms = 0, per_sm = 0;
  PMB_CUDA(cudaGetDevice(&dev));
  PMB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  PMB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, amg_fused_cycle_kernel<T>, 256, 0));
  static const int blocks_per_sm = [] {
    const char* e = std::getenv("PMB_FUSED_BLOCKS_PER_SM");
    const int v = e ? std::atoi(e) : 1;
    return v < 1 ? 1 : v;
  }();
  coop_grid_ = std::min(per_sm, blocks_per_sm) * sms;
  if (coop_grid_ < 1) coop_start_ = -1;
}

template <class T>
void AMG<T>::launch_fused(const T* b, T* x, cudaStream_t s) {
  PMB_REQUIRE(coop_status_ != nullptr, "AMG refresh must run before a cycle");
  PMB_CUDA(cudaMemsetAsync(coop_bar_.get(), 0, 2 * sizeof(unsigned int), s));
  const CoopLevel<T>* lv = reinterpret_cast<const CoopLevel<T>*>(coop_levels_.get());
  int nlev = (int)levels_.size() - coop_start_;
  int deg = degree;
  int nco = nco_;
  const double* inv = co_inv_.get();
  T* cob = co_b_.get();
  T* cox = co_x_.get();
  unsigned int* bar = coop_bar_.get();
  int* st = coop_status_;
  // cooperative: every block resident at once, which the grid barrier needs
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(coop_grid_);
  cfg.blockDim = dim3(256);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  PMB_CUDA(cudaLaunchKernelEx(&cfg, amg_fused_cycle_kernel<T>, lv, nlev, deg, nco, inv, cob, cox, b, x, bar, st));
  PMB_CHECK_LAUNCH();
}

// Names of the per-level phase timers (active under PMB_PROFILE=1 only):
// kind 0 pre-smoothing, 1 residual restriction, 2 prolongation and
// post-smoothing, 3 the K-cycle's own kernels on that level.
static const char* level_phase(int l, int kind) {
  static const std::vector<std::string> names = [] {
    static const char* kinds[] = {"pre", "restrict", "post", "kcycle"};
    std::vector<std::string> v;
    for (int i = 0; i < 32; ++i)
      for (const char* k : kinds) v.push_back("amg.L" + std::string(i < 10 ? "0" : "") + std::to_string(i) + "." + k);
    return v;
  }();
  return names[(size_t)std::min(l, 31) * 4 + kind].c_str();
}

// The first step of level m's pre-smoothing on right-hand side into x, for
// the kernel that writes that right-hand side to take over, where level m
// runs the per-step smoothing (not the coarsest, the cluster tail or the
// fused cycle).
template <class T>
ZeroStep<T> AMG<T>::zero_step_for(int m, T* x) {
  ZeroStep<T> z;
  if (m >= (int)levels_.size() || (tail_start_ >= 0 && m >= tail_start_) || (coop_start_ >= 0 && m >= coop_start_))
    return z;
  static const bool enabled = [] {
    const char* e = std::getenv("PMB_AMG_FUSE_ZERO_STEP");
    return !(e && e[0] == '0');
  }();
  if (!enabled) return z;
  AMGLevel<T>& L = levels_[m];
  const int steps = std::max(1, L.degree > 0 ? L.degree : degree);
  z.dinv = L.dinv.get();
  z.tab = L.lmax.get();
  z.d = L.r.get();
  z.x = (steps % 2 == 1) ? x : L.t.get();
  return z;
}

template <class T>
void AMG<T>::cycle(int l, const T* b, T* x, cudaStream_t s, bool zero_done) {
  if (tail_start_ >= 0 && l == tail_start_) {
    PhaseTimer pt("amg.tail", s);
    launch_tail(b, x, s);
    return;
  }
  if (coop_start_ >= 0 && l == coop_start_) {
    launch_fused(b, x, s);
    return;
  }
  if (l == (int)levels_.size()) {
    PhaseTimer pt("amg.coarsest", s);
    launch_pdl(dense_apply_kernel<T>, grid_for(32LL * nco_, 256), 256, 0, s, nco_, (const double*)co_inv_.get(), b,
               x);
    return;
  }
  AMGLevel<T>& L = levels_[l];
  const bool next_is_coarsest = (l + 1 == (int)levels_.size());
  const int nc = next_is_coarsest ? nco_ : levels_[l + 1].n;
  T* bc = next_is_coarsest ? co_b_.get() : levels_[l + 1].b.get();
  T* xc = next_is_coarsest ? co_x_.get() : levels_[l + 1].x.get();
  {
    PhaseTimer pt(level_phase(l, 0), s);
    smooth(L, b, x, s, true, nullptr, zero_done);
  }
  // the next level's first pre-smoothing step rides on the restriction: its
  // first visit smooths bc into xc (a plain correction) or into kc1 (K-cycle)
  const bool kc = l < k_levels && l + 1 < (int)levels_.size();
  ZeroStep<T> zs = zero_step_for(l + 1, kc ? levels_[l + 1].kc1.get() : xc);
  {
    PhaseTimer pt(level_phase(l, 1), s);
    static const bool by_rows = [] {
      const char* e = std::getenv("PMB_RESTRICT_ROWS");
      return !(e && e[0] == '0');
    }();
    if (!by_rows && L.ell_k == 0) zs = ZeroStep<T>();  // restrict_residual_kernel does not take it
    if (L.ell_k > 0) {
      launch_pdl(ell_residual_kernel<T>, grid_for(L.n, 256), 256, 0, s, ell_view(L), b, (const T*)x,
                 L.ell_rr.get());
      launch_pdl(aggregate_sum_kernel<T>, grid_for(nc, 256), 256, 0, s, nc, (const int*)L.cptr.get(),
                 (const int*)L.cmem.get(), (const double*)L.ell_rr.get(), bc, zs);
    } else {
      with_lanes(L.lanes, [&](auto ln) {
        constexpr int LN = decltype(ln)::value;
        if (by_rows)
          launch_pdl(restrict_rows_kernel<T, LN>, L.rblocks, 256, L.rsmem, s, (const int*)L.rblk.get(),
                     (const int*)L.cptr.get(), (const int*)L.cmem.get(), L.row_ptr, L.col, (const T*)L.val.get(), b,
                     (const T*)x, bc, zs);
        else
          launch_pdl(restrict_residual_kernel<T, LN>, grid_for((long long)nc * LN, 256), 256, 0, s, nc,
                     (const int*)L.cptr.get(), (const int*)L.cmem.get(), L.row_ptr, L.col, (const T*)L.val.get(), b,
                     (const T*)x, bc);
      });
    }
  }
  coarse_correction(l, bc, xc, s, zs.dinv != nullptr);
  PhaseTimer pt(level_phase(l, 2), s);
  if (L.n < kFoldProlongRows && degree >= 1) {
    smooth(L, b, x, s, false, xc);  // prolongation folded into the first smoothing step
  } else {
    launch_pdl(prolong_add_kernel<T>, grid_for(L.n, 256), 256, 0, s, L.n, (const int*)L.agg.get(), (const T*)xc,
               x);
    smooth(L, b, x, s, false);
  }
}

// Coarse correction of level l: a plain recursive cycle, or on the first
// k_levels levels two Krylov-accelerated cycles (K-cycle):
//   c1 = B rc, v1 = A c1, r2 = rc - (v1.rc / v1.v1) v1,
//   c2 = B r2, v2 = A c2, ec = y0 c1 + y1 c2 with y minimising |rc - y0 v1 - y1 v2|.
template <class T>
void AMG<T>::coarse_correction(int l, const T* rc, T* ec, cudaStream_t s, bool first_done) {
  const bool kc = l < k_levels && l + 1 < (int)levels_.size();
  if (!kc) {
    cycle(l + 1, rc, ec, s, first_done);
    return;
  }
  AMGLevel<T>& C = levels_[l + 1];
  const int n = C.n, g = grid_for(n, 256);
  const int G = std::min(2 * kNumSM, g);
  cycle(l + 1, rc, C.kc1.get(), s, first_done);
  const ZeroStep<T> zs2 = zero_step_for(l + 1, C.kc2.get());  // rides on the kaxpy below
  {
    PhaseTimer pt(level_phase(l + 1, 3), s);
    with_lanes(C.lanes, [&](auto ln) {
      constexpr int LN = decltype(ln)::value;
      launch_pdl(csr_spmv_kernel<T, LN>, grid_for((long long)n * LN, 256), 256, 0, s, n, C.row_ptr, C.col,
                 (const T*)C.val.get(), (const T*)C.kc1.get(), C.kv1.get());
    });
    launch_pdl(kdots_kernel<T, 2>, G, 256, 0, s, n, (const T*)C.kv1.get(), (const T*)nullptr, rc, C.kpart.get());
    launch_pdl(kaxpy_kernel<T>, G, 256, 0, s, n, rc, (const T*)C.kv1.get(), G, (const double*)C.kpart.get(),
               C.kr2.get(), zs2);
  }
  cycle(l + 1, C.kr2.get(), C.kc2.get(), s, zs2.dinv != nullptr);
  PhaseTimer pt(level_phase(l + 1, 3), s);
  with_lanes(C.lanes, [&](auto ln) {
    constexpr int LN = decltype(ln)::value;
    launch_pdl(csr_spmv_kernel<T, LN>, grid_for((long long)n * LN, 256), 256, 0, s, n, C.row_ptr, C.col,
               (const T*)C.val.get(), (const T*)C.kc2.get(), C.kv2.get());
  });
  launch_pdl(kdots_kernel<T, 5>, G, 256, 0, s, n, (const T*)C.kv1.get(), (const T*)C.kv2.get(), rc,
             C.kpart.get());
  launch_pdl(kcombine_kernel<T>, G, 256, 0, s, n, (const T*)C.kc1.get(), (const T*)C.kc2.get(), G,
             (const double*)C.kpart.get(), ec);
}

template <class T>
void AMG<T>::apply(const T* b, T* x, cudaStream_t s) {
  cycle(0, b, x, s);
}

template <class T>
double AMG<T>::time_visit(int l, int reps, cudaStream_t s) {
  PMB_REQUIRE(l >= 0 && l <= (int)levels_.size(), "level out of range");
  PMB_REQUIRE(reps >= 1, "reps must be positive");
  const bool co = l == (int)levels_.size();
  T* bw = co ? co_b_.get() : levels_[l].b.get();
  // level 0's own vectors are not written by a cycle: a zero right-hand side
  if (l == 0) PMB_CUDA(cudaMemsetAsync(bw, 0, sizeof(T) * levels_[0].n, s));
  const T* b = bw;
  T* x = co ? co_x_.get() : levels_[l].x.get();
  cudaGraph_t g = nullptr;
  cudaGraphExec_t ge = nullptr;
  // captured on a private stream (the legacy default stream cannot be
  // captured), replayed on s
  cudaStream_t cap = nullptr;
  PMB_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
  cudaError_t ce = cudaStreamSynchronize(s);
  if (ce == cudaSuccess) ce = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
  if (ce == cudaSuccess) {
    try {
      cycle(l, b, x, cap);
    } catch (...) {
      cudaStreamEndCapture(cap, &g);
      if (g) cudaGraphDestroy(g);
      cudaStreamDestroy(cap);
      throw;
    }
    ce = cudaStreamEndCapture(cap, &g);
  }
  cudaStreamDestroy(cap);
  PMB_CUDA(ce);
  const cudaError_t ie = cudaGraphInstantiate(&ge, g, 0);
  cudaGraphDestroy(g);
  PMB_CUDA(ie);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  float ms = 0.f;
  cudaError_t err = cudaGraphLaunch(ge, s);
  if (err == cudaSuccess) err = cudaEventCreate(&e0);
  if (err == cudaSuccess) err = cudaEventCreate(&e1);
  if (err == cudaSuccess) err = cudaEventRecord(e0, s);
  for (int i = 0; i < reps && err == cudaSuccess; ++i) err = cudaGraphLaunch(ge, s);
  if (err == cudaSuccess) err = cudaEventRecord(e1, s);
  if (err == cudaSuccess) err = cudaEventSynchronize(e1);
  if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaGraphExecDestroy(ge);
  PMB_CUDA(err);
  return ms / reps;
}

// Byte model of the launches of cycle() and coarse_correction() above.
template <class T>
double AMG<T>::cycle_bytes_from(int l) const {
  const double vb = sizeof(T);
  if (l == (int)levels_.size()) return (double)nco_ * nco_ * 8.0 + 2.0 * nco_ * vb;  // dense_apply_kernel
  const AMGLevel<T>& L = levels_[l];
  const double n = L.n;
  // the matrix as stored: CSR (values, columns, row starts) or the ELL slots
  // (padding included; the diagonal form has no columns but a per-row
  // overflow index) and the overflow entries
  const double mat = L.ell_k > 0 ? (L.ell_dia ? (double)L.ell_k * n * vb + n * 4.0 + (double)L.ell_ovf * (vb + 4.0)
                                              : ((double)L.ell_k * n + (double)L.ell_ovf) * (vb + 4.0))
                                 : (double)L.nnz * (vb + 4.0) + (n + 1.0) * 4.0;
  const int steps = std::max(1, L.degree > 0 ? L.degree : degree);
  const double nc = (l + 1 == (int)levels_.size()) ? nco_ : levels_[l + 1].n;
  // pre-smoothing from zero: the first step reads b and D^-1 and writes d, x
  // (no matrix); each further step reads the matrix, b, D^-1, x, d and writes
  // x, d
  const double step = mat + 6.0 * n * vb;
  double bytes = 4.0 * n * vb + (steps - 1) * step;
  // restriction: matrix, b and x of every member row, the member lists, the
  // coarse right-hand side written
  // (ELL: the member residuals written in FP64 and read back by the
  // aggregate sums)
  bytes += mat + 2.0 * n * vb + n * 4.0 + (nc + 1.0) * 4.0 + nc * vb + (L.ell_k > 0 ? 16.0 * n : 0.0);
  bytes += coarse_bytes(l);
  // post-smoothing from the prolonged correction: agg and the coarse
  // correction once (folded into the first step, or a separate launch that
  // also reads and writes x)
  bytes += steps * step + n * 4.0 + nc * vb + (L.n < kFoldProlongRows ? 0.0 : 2.0 * n * vb);
  return bytes;
}

template <class T>
double AMG<T>::coarse_bytes(int l) const {
  const bool kc = l < k_levels && l + 1 < (int)levels_.size();
  if (!kc) return cycle_bytes_from(l + 1);
  const AMGLevel<T>& C = levels_[l + 1];
  const double vb = sizeof(T), n = C.n;
  const double spmv = (double)C.nnz * (vb + 4.0) + (n + 1.0) * 4.0 + 2.0 * n * vb;
  // two cycles, two products, kdots<2> (v1, rc), kaxpy (rc, v1 -> r2),
  // kdots<5> (v1, v2, rc), kcombine (c1, c2 -> ec)
  return 2.0 * cycle_bytes_from(l + 1) + 2.0 * spmv + (2.0 + 3.0 + 3.0 + 3.0) * n * vb;
}

template <class T>
double AMG<T>::refresh_bytes() const {
  const double vb = sizeof(T);
  double bytes = 0.0;
  for (size_t l = 0; l < levels_.size(); ++l) {
    const AMGLevel<T>& L = levels_[l];
    const double nnz_next = (l + 1 < levels_.size()) ? (double)levels_[l + 1].nnz : (double)co_nnz_;
    // diagonal and Gershgorin bound: matrix read, D^-1 written
    bytes += (double)L.nnz * (vb + 4.0) + (L.n + 1.0) * 4.0 + L.n * vb;
    // Galerkin gather: every fine value once through its index, the coarse
    // values and their index ranges
    bytes += (double)L.nnz * (vb + 4.0) + nnz_next * (vb + 4.0);
    // the ELL copy's values: the source index and value of every slot read
    // (padding: the index only), the slot written
    if (L.ell_k > 0)
      bytes += ((double)L.ell_k * L.n + (double)L.ell_ovf) * (4.0 + vb) + (double)L.nnz * vb;
  }
  // dense coarsest matrix assembled and inverted in place
  bytes += (double)co_nnz_ * (vb + 4.0) + 3.0 * (double)nco_ * nco_ * 8.0;
  return bytes;
}

template class AMG<double>;
template class AMG<float>;

}  // namespace pmb
