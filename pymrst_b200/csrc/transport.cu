// Two-phase incompressible transport on the device: the sequential
// saturation step of the reference's explicit_transport and
// implicit_transport (pymrst/modules/incomp/transport/__init__.py:152-402)
// for a Corey fluid (kr = s^n_w, (1-s)^n_o; mobility kr / mu).
//
// The Darcy flux v and the gravity flux g of every interior interface and
// the water source q of every cell are frozen for a call, as in the
// reference.  Kernels gather per cell (no atomics):
//   tr_residual / the explicit substep: r = (s - s0) + dt / pv (div - q_w),
//     div summed as np.bincount sums it (the cell's interfaces where it is
//     N[f,0], ascending, then those where it is N[f,1]);
//   tr_jacobian: dr/ds on a fixed pattern (the cell and its neighbours),
//     upwind cells chosen per interface as _upwind_indices chooses them;
//   tr_estimate_* / tr_control: the explicit step estimate (_estimate_dt)
//     and the substep clock, entirely on the device, so that a chunk of
//     substeps runs with no host round trip.
// Values are formed with explicit roundings in the reference's order of
// operations.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "pmb_common.cuh"
#include "pmb_krylov.cuh"

namespace pmb {
namespace tr {

__device__ __forceinline__ double ad(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sb(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double ml(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dv(double a, double b) { return __ddiv_rn(a, b); }

struct Fluid {
  double mu[2], n[2];
};

// x ** n as numpy evaluates an array to a scalar power (squares and the
// identity exactly).
__device__ __forceinline__ double powi(double x, double n) {
  if (n == 2.0) return ml(x, x);
  if (n == 1.0) return x;
  if (n == 0.0) return 1.0;
  return pow(x, n);
}

// Mobilities (kr / mu) at water saturation s.
__device__ __forceinline__ void mobility(const Fluid& f, double s, double* mw, double* mo) {
  *mw = dv(powi(s, f.n[0]), f.mu[0]);
  *mo = dv(powi(sb(1.0, s), f.n[1]), f.mu[1]);
}
// d(mobility)/d(own saturation): n s^(n-1) / mu for each phase.
__device__ __forceinline__ void dmobility(const Fluid& f, double s, double* dw, double* dox) {
  *dw = dv(ml(f.n[0], powi(s, f.n[0] - 1.0)), f.mu[0]);
  *dox = dv(ml(f.n[1], powi(sb(1.0, s), f.n[1] - 1.0)), f.mu[1]);
}

// The fractional-flow slope df/ds_w of the estimate.
__device__ __forceinline__ double dfrac(const Fluid& f, double s) {
  double mw, mo, dw, dox;
  mobility(f, s, &mw, &mo);
  dmobility(f, s, &dw, &dox);
  const double dmo = -dox;
  const double mt = ad(mw, mo);
  return dv(sb(ml(mo, dw), ml(mw, dmo)), ml(mt, mt));
}

struct View {
  int nc, nf;
  const int* N;        // nf x 2
  const double* pv;    // nc
  const int* adj_ptr;  // nc + 1
  const int* adj;      // f where the cell is N[f,0] (listed first), -(f+1) where it is N[f,1]
  const int* adj_rank; // rank of the cell across in the cell's Jacobian row
  const int* diag_rank;
  const int* row_ptr;  // nc + 1
  const double* v;     // nf Darcy flux
  const double* g;     // nf gravity flux
  const double* q;     // nc source
  const double* fmax;  // nc: max |v| over the cell's interfaces
  Fluid fl;
};

// Upwind cells of interface f for water (*iw) and oil (*io)
// (_upwind_indices): the sign of a phase flux is decided by v and g where
// they agree for that phase; otherwise by v + g m_o (water) or v - g m_w
// (oil) with the other phase's mobility at its own upwind cell.
__device__ __forceinline__ void upwind(const View& w, int f, const double* s, int* iw, int* io) {
  const int a = w.N[2 * f], b = w.N[2 * f + 1];
  const double v = w.v[f], g = w.g[f];
  int uw = -1, uo = -1;
  if (!(v > 0.0) && !(g > 0.0)) uw = b;
  else if (!(v < 0.0) && !(g < 0.0)) uw = a;
  if (!(v > 0.0) && !(g < 0.0)) uo = b;
  else if (!(v < 0.0) && !(g > 0.0)) uo = a;
  if (uw < 0) {  // oil decided
    double mw_, mo_;
    mobility(w.fl, s[uo], &mw_, &mo_);
    uw = ad(v, ml(g, mo_)) < 0.0 ? b : a;
  } else if (uo < 0) {  // water decided
    double mw_, mo_;
    mobility(w.fl, s[uw], &mw_, &mo_);
    uo = sb(v, ml(g, mw_)) < 0.0 ? b : a;
  }
  *iw = uw;
  *io = uo;
}

// Water flux through interface f: f_w (v + g m_o) with upwind mobilities.
__device__ __forceinline__ double water_flux(const View& w, int f, const double* s) {
  int iw, io;
  upwind(w, f, s, &iw, &io);
  double mw, mo, t;
  mobility(w.fl, s[iw], &mw, &t);
  mobility(w.fl, s[io], &t, &mo);
  const double ff = dv(mw, ad(mw, mo));
  return ml(ff, ad(w.v[f], ml(w.g[f], mo)));
}

// r_c = (s_c - s0_c) + dt / pv_c (div_c - q_w,c).
__device__ __forceinline__ double residual_at(const View& w, int c, const double* s, double s0c, double dt) {
  double div = 0.0;
  for (int k = w.adj_ptr[c]; k < w.adj_ptr[c + 1]; ++k) {
    const int code = w.adj[k];
    if (code >= 0) div = ad(div, water_flux(w, code, s));
    else div = ad(div, -water_flux(w, -code - 1, s));
  }
  double mw, mo;
  mobility(w.fl, s[c], &mw, &mo);
  const double fc = dv(mw, ad(mw, mo));
  const double q = w.q[c];
  const double qw = ad(q > 0.0 ? q : 0.0, ml(q < 0.0 ? q : 0.0, fc));
  return ad(sb(s[c], s0c), ml(dv(dt, w.pv[c]), sb(div, qw)));
}

__global__ void tr_fmax_kernel(View w, double* __restrict__ fmax) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= w.nc) return;
  double m = 0.0;
  for (int k = w.adj_ptr[c]; k < w.adj_ptr[c + 1]; ++k) {
    const int code = w.adj[k];
    const double a = fabs(w.v[code >= 0 ? code : -code - 1]);
    m = (a > m || a != a) ? a : m;
  }
  fmax[c] = m;
}

__global__ void tr_residual_kernel(View w, const double* __restrict__ s, const double* __restrict__ s0, double dt,
                                   double* __restrict__ res) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= w.nc) return;
  res[c] = residual_at(w, c, s, s0[c], dt);
}

// Jacobian values on the pattern (two_phase_residual_jacobian's jacobian):
// the diagonal 1 - dt / pv min(q, 0) df/ds, and per interface the
// derivatives of its water flux with respect to the saturations of its water
// and oil upwind cells, added to the row of N[f,0] and subtracted from the
// row of N[f,1].
__global__ void tr_jacobian_kernel(View w, const double* __restrict__ s, double dt, double* __restrict__ vals) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= w.nc) return;
  const int base = w.row_ptr[c], len = w.row_ptr[c + 1] - base;
  for (int k = 0; k < len; ++k) vals[base + k] = 0.0;
  const double q = w.q[c];
  const double diag = sb(1.0, ml(dv(dt, w.pv[c]), ml(q < 0.0 ? q : 0.0, dfrac(w.fl, s[c]))));
  vals[base + w.diag_rank[c]] += diag;
  const double h = dv(dt, w.pv[c]);
  for (int k = w.adj_ptr[c]; k < w.adj_ptr[c + 1]; ++k) {
    const int code = w.adj[k];
    const bool first = code >= 0;
    const int f = first ? code : -code - 1;
    int iw, io;
    upwind(w, f, s, &iw, &io);
    double mw, mo, t, dmw, dmo_raw, t2;
    mobility(w.fl, s[iw], &mw, &t);
    mobility(w.fl, s[io], &t, &mo);
    dmobility(w.fl, s[iw], &dmw, &t2);
    dmobility(w.fl, s[io], &t2, &dmo_raw);
    const double dmo = -dmo_raw;
    const double mt = ad(mw, mo);
    const double fw = dv(mw, mt), fo = dv(mo, mt);
    const double d1 = dv(ml(ad(w.v[f], ml(w.g[f], mo)), ml(fo, dmw)), mt);
    const double d2 = dv(-ml(sb(w.v[f], ml(w.g[f], mw)), ml(fw, dmo)), mt);
    const double sg = first ? 1.0 : -1.0;
    const int rk = w.adj_rank[k], dr = w.diag_rank[c];
    vals[base + (iw == c ? dr : rk)] += sg * ml(h, d1);
    vals[base + (io == c ? dr : rk)] += sg * ml(h, d2);
  }
}

// ---- explicit transport on a device clock ---------------------------------------
constexpr int kEstBlocks = 2 * kNumSM;
constexpr int kEstThreads = 256;

// Device clock of an explicit call (one per handle).
struct Clock {
  double t, tf, step, fixed_dt, max_dt, dt_factor, satwarn;
  double gwave, pvmin, qpos, qneg;  // the constant parts of the estimate
  int nsub, done, bad, nan_seen, has_pos, has_neg, nparts, pad;
};

// Per-block partials of the estimate: max |df| fmax, min s over q > 0,
// max s over q < 0.
__global__ void __launch_bounds__(kEstThreads) tr_estimate_partial_kernel(View w, const double* __restrict__ s,
                                                                           const Clock* __restrict__ ck,
                                                                           double* __restrict__ part) {
  if (ck->done) return;
  double wv = 0.0, smin = INFINITY, smax = -INFINITY;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < w.nc; c += gridDim.x * blockDim.x) {
    const double a = ml(fabs(dfrac(w.fl, s[c])), w.fmax[c]);
    wv = (a > wv || a != a) ? a : wv;
    const double q = w.q[c];
    if (q > 0.0) smin = fmin(smin, s[c]);
    if (q < 0.0) smax = fmax(smax, s[c]);
  }
  for (int o = 16; o; o >>= 1) {
    const double a = __shfl_xor_sync(0xffffffffu, wv, o);
    wv = (a > wv || a != a) ? a : wv;
    smin = fmin(smin, __shfl_xor_sync(0xffffffffu, smin, o));
    smax = fmax(smax, __shfl_xor_sync(0xffffffffu, smax, o));
  }
  __shared__ double sh[kEstThreads / 32][3];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) {
    sh[wid][0] = wv;
    sh[wid][1] = smin;
    sh[wid][2] = smax;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < kEstThreads / 32; ++k) {
      wv = (sh[k][0] > wv || sh[k][0] != sh[k][0]) ? sh[k][0] : wv;
      smin = fmin(smin, sh[k][1]);
      smax = fmax(smax, sh[k][2]);
    }
    part[3 * blockIdx.x] = wv;
    part[3 * blockIdx.x + 1] = smin;
    part[3 * blockIdx.x + 2] = smax;
  }
}

// The largest fractional-flow slope over a saturation sweep starting at s0
// in steps of +0.05 up to 1 (up) or -0.05 down to 0, the sweep laid out as
// numpy.arange lays it out (start, start + step, then start + i delta).
// Returns -inf when the sweep has fewer than two points.
__device__ double sweep_slope(const Fluid& f, double s0, bool up) {
  const double step = up ? 0.05 : -0.05;
  const double stop = up ? 1.0 + 1e-12 : -1e-12;
  const double len = ceil(dv(sb(stop, s0), step));
  if (!(len >= 2.0)) return -INFINITY;
  const long long n = (long long)len;
  const double delta = sb(ad(s0, step), s0);
  double best = -INFINITY, prev_s = s0, prev_f = 0.0;
  {
    double mw, mo;
    mobility(f, s0, &mw, &mo);
    prev_f = dv(mw, ad(mw, mo));
  }
  for (long long i = 1; i < n; ++i) {
    const double si = i == 1 ? ad(s0, step) : ad(s0, ml((double)i, delta));
    double mw, mo;
    mobility(f, si, &mw, &mo);
    const double fi = dv(mw, ad(mw, mo));
    const double d = dv(sb(fi, prev_f), sb(si, prev_s));
    best = (d > best || d != d) ? d : best;
    prev_s = si;
    prev_f = fi;
  }
  return best;
}

// One thread: the next substep (the step estimate when no fixed dt is
// given), the clock, and the stop conditions.
__global__ void tr_control_kernel(View w, Clock* __restrict__ ck, const double* __restrict__ part) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (ck->done) return;
  if (ck->bad || ck->nan_seen || !(ck->t < ck->tf)) {
    ck->done = 1;
    return;
  }
  double step;
  if (ck->fixed_dt > 0.0) {
    step = ck->fixed_dt;
  } else {
    double wave = 0.0, smin = INFINITY, smax = -INFINITY;
    for (int b = 0; b < ck->nparts; ++b) {
      const double a = part[3 * b];
      wave = (a > wave || a != a) ? a : wave;
      smin = fmin(smin, part[3 * b + 1]);
      smax = fmax(smax, part[3 * b + 2]);
    }
    wave = (ck->gwave > wave || ck->gwave != ck->gwave) ? ck->gwave : wave;
    if (ck->has_pos) {
      const double d = sweep_slope(w.fl, smin, true);
      if (d > -INFINITY) {
        const double a = fabs(ml(ck->qpos, d));
        wave = (a > wave || a != a) ? a : wave;
      }
    }
    if (ck->has_neg) {
      const double d = sweep_slope(w.fl, smax, false);
      if (d > -INFINITY) {
        const double a = fabs(ml(ck->qneg, d));
        wave = (a > wave || a != a) ? a : wave;
      }
    }
    const double est = wave > 0.0 ? dv(ck->pvmin, wave) : INFINITY;
    step = fmin(ck->max_dt, ml(ck->dt_factor, est));
  }
  step = fmin(sb(ck->tf, ck->t), step);
  ck->step = step;
  ck->t = ad(ck->t, step);
  ck->nsub += 1;
}

// One forward-Euler substep: s_out = clip(s - r(s, s, step), 0, 1), with the
// range and NaN flags of the reference's checks.
__global__ void tr_explicit_kernel(View w, const double* __restrict__ s, double* __restrict__ s_out,
                                   Clock* __restrict__ ck) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= w.nc) return;
  if (ck->done) return;
  const double step = ck->step;
  const double sn = sb(s[c], residual_at(w, c, s, s[c], step));
  if (sn > 1.0 + ck->satwarn || sn < -ck->satwarn) atomicExch(&ck->bad, 1);
  if (sn != sn) atomicExch(&ck->nan_seen, 1);
  s_out[c] = sn < 0.0 ? 0.0 : (sn > 1.0 ? 1.0 : sn);
}

// ---- implicit helpers ---------------------------------------------------------------------
constexpr int kMaxBlocks = 2 * kNumSM;

__global__ void __launch_bounds__(256) tr_absmax_kernel(int n, const double* __restrict__ x, double* __restrict__ part) {
  double m = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double a = fabs(x[i]);
    m = (a > m || a != a) ? a : m;
  }
  for (int o = 16; o; o >>= 1) {
    const double a = __shfl_xor_sync(0xffffffffu, m, o);
    m = (a > m || a != a) ? a : m;
  }
  __shared__ double sh[8];
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < (int)(blockDim.x >> 5); ++k) m = (sh[k] > m || sh[k] != sh[k]) ? sh[k] : m;
    part[blockIdx.x] = m;
  }
}

__global__ void tr_absmax_final_kernel(int nparts, const double* __restrict__ part, double* __restrict__ out) {
  if (threadIdx.x != 0) return;
  double m = 0.0;
  for (int b = 0; b < nparts; ++b) m = (part[b] > m || part[b] != part[b]) ? part[b] : m;
  *out = m;
}

// out = min(1, s + 0.05): the Newton start of a substep.
__global__ void tr_start_kernel(int n, const double* __restrict__ s, double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    const double a = ad(s[i], 0.05);
    out[i] = a > 1.0 ? 1.0 : a;  // np.minimum(1.0, a)
    if (a != a) out[i] = a;
  }
}

// out = clip(base + ds * scale, 0, 1): one line-search trial.
__global__ void tr_trial_kernel(int n, const double* __restrict__ base, const double* __restrict__ ds, double scale,
                                double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    const double a = ad(base[i], ml(ds[i], scale));
    out[i] = a < 0.0 ? 0.0 : (a > 1.0 ? 1.0 : a);
  }
}

__global__ void tr_neg_kernel(int n, const double* __restrict__ a, double* __restrict__ b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = -a[i];
}

// y = A x for the scalar CSR Jacobian, a thread per row.
__global__ void tr_spmv_kernel(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                               const double* __restrict__ a, const double* __restrict__ x, double* __restrict__ y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s = 0.0;
  for (int k = rp[i]; k < rp[i + 1]; ++k) s += a[k] * x[ci[k]];
  y[i] = s;
}

// One level of the flow-ordered Gauss-Seidel sweep: for the cells
// perm[lo .. hi), x_c = (r_c - sum of a_cj x_j over the kept couplings) /
// a_cc; every kept coupling points at a cell of an earlier level.
__global__ void tr_flow_gs_level_kernel(int lo, int hi, const int* __restrict__ perm, const int* __restrict__ rp,
                                        const int* __restrict__ ci, const double* __restrict__ a,
                                        const unsigned char* __restrict__ keep, const int* __restrict__ dpos,
                                        const double* __restrict__ r, double* __restrict__ x) {
  const int t = lo + blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= hi) return;
  const int c = perm[t];
  double s = r[c];
  for (int k = rp[c]; k < rp[c + 1]; ++k)
    if (keep[k]) s -= a[k] * x[ci[k]];
  const double d = a[dpos[c]];
  x[c] = d != 0.0 ? s / d : s;
}

}  // namespace tr
}  // namespace pmb

// ---- host ---------------------------------------------------------------------------------
namespace pmb {

class Transport {
 public:
  Transport(int nc, int nf, const int* h_N, const double* h_pv, cudaStream_t s);
  ~Transport() {
    if (cpr_) pmb_csr_cpr_destroy(cpr_);
  }
  int nc() const { return w_.nc; }
  int64_t nnz() const { return h_rp_.back(); }
  const std::vector<int>& row_ptr() const { return h_rp_; }
  const std::vector<int>& col() const { return h_col_; }
  void set_flow(const double* d_v, const double* d_g, const double* d_q, const double* h_fluid4);
  void residual(const double* s, const double* s0, double dt, double* res);
  double absmax(int n, const double* x);
  void jacobian(const double* s, double dt, double* vals);
  void explicit_run(double* s, double tf, double dt, double max_dt, double dt_factor, double satwarn,
                    double gwave, double* h_out4);
  void implicit_run(double* s, double tf, double nltol, int lstrials, int maxnewt, int tsref, double resred,
                    const pmb_cpr_opts& o, double* h_out6);

 private:
  cudaStream_t s_;
  tr::View w_{};
  std::vector<int> h_rp_, h_col_;
  std::vector<double> h_pv_;
  double pvmin_ = 0.0;
  DArray<int> N_, adj_ptr_, adj_, adj_rank_, diag_rank_, rp_, col_;
  DArray<double> pv_, v_, g_, q_, fmax_, part_, sbuf_, res_, vals_, ds_, rhs_, s0_, base_, out1_;
  DArray<tr::Clock> clock_;
  PinnedArray<tr::Clock> h_clock_;
  PinnedArray<double> h_scalar_;
  double qpos_ = 0.0, qneg_ = 0.0;
  int has_pos_ = 0, has_neg_ = 0;
  bool flow_set_ = false;
  pmb_csr_cpr* cpr_ = nullptr;
  pmb_cpr_opts cpr_opts_{};
  // flow-ordered Gauss-Seidel preconditioner of the implicit solves
  std::vector<int> h_dpos_;
  DArray<int> dpos_, gs_perm_;
  DArray<unsigned char> gs_keep_;
  const double* gs_vals_ = nullptr;
  std::vector<int> gs_level_ptr_;
  std::vector<double> h_vals_;
  Fgmres kry_;
  void flow_order(const double* d_vals);
  void flow_gs(const double* r, double* z);
  bool solve_flow(const double* d_vals, const double* b, double* x, const pmb_cpr_opts& o, double* info);
};

Transport::Transport(int nc, int nf, const int* h_N, const double* h_pv, cudaStream_t s) : s_(s) {
  PMB_REQUIRE(nc > 0 && nf >= 0 && h_pv && (nf == 0 || h_N), "transport: bad sizes or NULL arrays");
  std::vector<int> N(h_N, h_N + 2LL * nf);
  for (int f = 0; f < nf; ++f)
    PMB_REQUIRE(N[2 * f] >= 0 && N[2 * f] < nc && N[2 * f + 1] >= 0 && N[2 * f + 1] < nc &&
                    N[2 * f] != N[2 * f + 1],
                "transport: interface neighbours must be two distinct cells in [0, nc)");
  h_pv_.assign(h_pv, h_pv + nc);
  for (double v : h_pv_) PMB_REQUIRE(v > 0.0 && std::isfinite(v), "transport: pore volumes must be positive");
  pvmin_ = *std::min_element(h_pv_.begin(), h_pv_.end());
  // adjacency in the order np.bincount sums: first the interfaces where the
  // cell is N[f,0], then those where it is N[f,1], each ascending
  std::vector<std::vector<int>> first(nc), second(nc), cols(nc);
  for (int f = 0; f < nf; ++f) {
    first[N[2 * f]].push_back(f);
    second[N[2 * f + 1]].push_back(-f - 1);
    cols[N[2 * f]].push_back(N[2 * f + 1]);
    cols[N[2 * f + 1]].push_back(N[2 * f]);
  }
  std::vector<int> adj_ptr(nc + 1, 0), adj, adj_rank, diag_rank(nc);
  h_rp_.assign(nc + 1, 0);
  for (int c = 0; c < nc; ++c) {
    auto& cl = cols[c];
    cl.push_back(c);
    std::sort(cl.begin(), cl.end());
    cl.erase(std::unique(cl.begin(), cl.end()), cl.end());
    diag_rank[c] = (int)(std::lower_bound(cl.begin(), cl.end(), c) - cl.begin());
    for (int pass = 0; pass < 2; ++pass)
      for (int code : (pass == 0 ? first[c] : second[c])) {
        const int f = code >= 0 ? code : -code - 1;
        const int nb = code >= 0 ? N[2 * f + 1] : N[2 * f];
        adj.push_back(code);
        adj_rank.push_back((int)(std::lower_bound(cl.begin(), cl.end(), nb) - cl.begin()));
      }
    adj_ptr[c + 1] = (int)adj.size();
    h_col_.insert(h_col_.end(), cl.begin(), cl.end());
    h_rp_[c + 1] = (int)h_col_.size();
  }
  h_dpos_.resize(nc);
  for (int c = 0; c < nc; ++c) h_dpos_[c] = h_rp_[c] + diag_rank[c];
  dpos_.upload(h_dpos_, s);
  N_.upload(N.empty() ? std::vector<int>{0, 0} : N, s);
  pv_.upload(h_pv_, s);
  adj_ptr_.upload(adj_ptr, s);
  adj_.upload(adj.empty() ? std::vector<int>{0} : adj, s);
  adj_rank_.upload(adj_rank.empty() ? std::vector<int>{0} : adj_rank, s);
  diag_rank_.upload(diag_rank, s);
  rp_.upload(h_rp_, s);
  col_.upload(h_col_, s);
  v_.resize(std::max(nf, 1));
  g_.resize(std::max(nf, 1));
  q_.resize(nc);
  fmax_.resize(nc);
  part_.resize(3 * tr::kEstBlocks + tr::kMaxBlocks);
  sbuf_.resize(2LL * nc);
  clock_.resize(1);
  h_clock_.resize(1);
  h_scalar_.resize(1);
  out1_.resize(1);
  w_.nc = nc;
  w_.nf = nf;
  w_.N = N_.get();
  w_.pv = pv_.get();
  w_.adj_ptr = adj_ptr_.get();
  w_.adj = adj_.get();
  w_.adj_rank = adj_rank_.get();
  w_.diag_rank = diag_rank_.get();
  w_.row_ptr = rp_.get();
  w_.v = v_.get();
  w_.g = g_.get();
  w_.q = q_.get();
  w_.fmax = fmax_.get();
  PMB_CUDA(cudaStreamSynchronize(s));
}

void Transport::set_flow(const double* d_v, const double* d_g, const double* d_q, const double* h_fluid4) {
  PMB_REQUIRE(d_q && h_fluid4 && (w_.nf == 0 || (d_v && d_g)), "transport: NULL flow arrays");
  for (int i = 0; i < 4; ++i) PMB_REQUIRE(std::isfinite(h_fluid4[i]), "transport: non-finite fluid parameter");
  PMB_REQUIRE(h_fluid4[0] > 0.0 && h_fluid4[1] > 0.0, "transport: viscosities must be positive");
  w_.fl.mu[0] = h_fluid4[0];
  w_.fl.mu[1] = h_fluid4[1];
  w_.fl.n[0] = h_fluid4[2];
  w_.fl.n[1] = h_fluid4[3];
  const int nc = w_.nc, nf = w_.nf;
  if (nf) {
    PMB_CUDA(cudaMemcpyAsync(v_.get(), d_v, sizeof(double) * nf, cudaMemcpyDeviceToDevice, s_));
    PMB_CUDA(cudaMemcpyAsync(g_.get(), d_g, sizeof(double) * nf, cudaMemcpyDeviceToDevice, s_));
  }
  PMB_CUDA(cudaMemcpyAsync(q_.get(), d_q, sizeof(double) * nc, cudaMemcpyDeviceToDevice, s_));
  tr::tr_fmax_kernel<<<(nc + 127) / 128, 128, 0, s_>>>(w_, fmax_.get());
  PMB_CHECK_LAUNCH();
  // the source part of the estimate needs max |q| over injecting and producing cells
  std::vector<double> hq(nc);
  PMB_CUDA(cudaMemcpyAsync(hq.data(), d_q, sizeof(double) * nc, cudaMemcpyDeviceToHost, s_));
  PMB_CUDA(cudaStreamSynchronize(s_));
  qpos_ = qneg_ = 0.0;
  has_pos_ = has_neg_ = 0;
  for (double q : hq) {
    if (q > 0.0) { has_pos_ = 1; qpos_ = std::max(qpos_, std::fabs(q)); }
    if (q < 0.0) { has_neg_ = 1; qneg_ = std::max(qneg_, std::fabs(q)); }
  }
  flow_set_ = true;
}

void Transport::residual(const double* s, const double* s0, double dt, double* res) {
  PMB_REQUIRE(flow_set_, "transport: set the flow first");
  tr::tr_residual_kernel<<<(w_.nc + 127) / 128, 128, 0, s_>>>(w_, s, s0, dt, res);
  PMB_CHECK_LAUNCH();
}

double Transport::absmax(int n, const double* x) {
  const int nb = std::max(1, std::min(tr::kMaxBlocks, (n + 255) / 256));
  double* part = part_.get() + 3 * tr::kEstBlocks;
  tr::tr_absmax_kernel<<<nb, 256, 0, s_>>>(n, x, part);
  PMB_CHECK_LAUNCH();
  tr::tr_absmax_final_kernel<<<1, 32, 0, s_>>>(nb, part, out1_.get());
  PMB_CHECK_LAUNCH();
  PMB_CUDA(cudaMemcpyAsync(h_scalar_.get(), out1_.get(), sizeof(double), cudaMemcpyDeviceToHost, s_));
  PMB_CUDA(cudaStreamSynchronize(s_));
  return h_scalar_[0];
}

void Transport::jacobian(const double* s, double dt, double* vals) {
  PMB_REQUIRE(flow_set_, "transport: set the flow first");
  tr::tr_jacobian_kernel<<<(w_.nc + 127) / 128, 128, 0, s_>>>(w_, s, dt, vals);
  PMB_CHECK_LAUNCH();
}

// Substeps run in chunks on the device clock; the host reads the clock once
// per chunk.
void Transport::explicit_run(double* s, double tf, double dt, double max_dt, double dt_factor, double satwarn,
                             double gwave, double* h_out4) {
  PMB_REQUIRE(flow_set_, "transport: set the flow first");
  PMB_REQUIRE(tf >= 0.0 && std::isfinite(tf), "transport: tf must be finite and non-negative");
  const int nc = w_.nc;
  tr::Clock& hc = h_clock_[0];
  std::memset(&hc, 0, sizeof(hc));
  hc.t = 0.0;
  hc.tf = tf;
  hc.fixed_dt = dt > 0.0 ? dt : 0.0;
  hc.max_dt = max_dt;
  hc.dt_factor = dt_factor;
  hc.satwarn = satwarn;
  hc.gwave = gwave;
  hc.pvmin = pvmin_;
  hc.qpos = qpos_;
  hc.qneg = qneg_;
  hc.has_pos = has_pos_;
  hc.has_neg = has_neg_;
  const int nparts = std::max(1, std::min(tr::kEstBlocks, (nc + tr::kEstThreads - 1) / tr::kEstThreads));
  hc.nparts = nparts;
  PMB_CUDA(cudaMemcpyAsync(clock_.get(), &hc, sizeof(hc), cudaMemcpyHostToDevice, s_));
  double* buf[2] = {sbuf_.get(), sbuf_.get() + nc};
  PMB_CUDA(cudaMemcpyAsync(buf[0], s, sizeof(double) * nc, cudaMemcpyDeviceToDevice, s_));
  const bool estimate = !(dt > 0.0);
  long long launched = 0;
  const long long kMaxSubsteps = 100000000LL;
  for (int chunk = 1;; chunk = std::min(chunk * 2, 256)) {
    for (int k = 0; k < chunk; ++k, ++launched) {
      const double* cur = buf[launched & 1];
      double* nxt = buf[(launched + 1) & 1];
      if (estimate) {
        tr::tr_estimate_partial_kernel<<<nparts, tr::kEstThreads, 0, s_>>>(w_, cur, clock_.get(), part_.get());
        PMB_CHECK_LAUNCH();
      }
      tr::tr_control_kernel<<<1, 32, 0, s_>>>(w_, clock_.get(), part_.get());
      PMB_CHECK_LAUNCH();
      tr::tr_explicit_kernel<<<(nc + 127) / 128, 128, 0, s_>>>(w_, cur, nxt, clock_.get());
      PMB_CHECK_LAUNCH();
    }
    PMB_CUDA(cudaMemcpyAsync(&hc, clock_.get(), sizeof(hc), cudaMemcpyDeviceToHost, s_));
    PMB_CUDA(cudaStreamSynchronize(s_));
    // done, or stopped by a flag (the next control would set done)
    if (hc.done || hc.bad || hc.nan_seen || !(hc.t < hc.tf)) break;
    PMB_REQUIRE(launched < kMaxSubsteps, "transport: more than 1e8 explicit substeps");
  }
  const int last = hc.nsub & 1;
  PMB_CUDA(cudaMemcpyAsync(s, buf[last], sizeof(double) * nc, cudaMemcpyDeviceToDevice, s_));
  PMB_CUDA(cudaStreamSynchronize(s_));
  h_out4[0] = hc.nsub;
  h_out4[1] = hc.t;
  h_out4[2] = hc.bad;
  h_out4[3] = hc.nan_seen;
}

// The flow order of the current Jacobian: cell c depends on each cell j with
// a_cj != 0 (its upwind neighbours).  Where two cells depend on each other
// (counter-current gravity flow) only the coupling stronger relative to its
// row's diagonal is kept; any longer cycle that remains is broken by
// releasing its lowest-numbered cell.  Levels by Kahn's algorithm.
void Transport::flow_order(const double* d_vals) {
  const int nc = w_.nc;
  const int64_t nnz = this->nnz();
  h_vals_.resize(nnz);
  PMB_CUDA(cudaMemcpyAsync(h_vals_.data(), d_vals, sizeof(double) * nnz, cudaMemcpyDeviceToHost, s_));
  PMB_CUDA(cudaStreamSynchronize(s_));
  const auto& rp = h_rp_;
  const auto& ci = h_col_;
  std::vector<unsigned char> keep(nnz, 0);
  auto rel = [&](int c, int k) {
    const double d = std::fabs(h_vals_[h_dpos_[c]]);
    return std::fabs(h_vals_[k]) / (d > 0.0 ? d : 1.0);
  };
  for (int c = 0; c < nc; ++c)
    for (int k = rp[c]; k < rp[c + 1]; ++k) {
      const int j = ci[k];
      if (j == c || h_vals_[k] == 0.0) continue;
      // the reverse coupling a_jc
      const int* b = ci.data() + rp[j];
      const int* e = ci.data() + rp[j + 1];
      const int* it = std::lower_bound(b, e, c);
      const int kr = (it != e && *it == c) ? (int)(it - ci.data()) : -1;
      if (kr >= 0 && h_vals_[kr] != 0.0) {
        const double mine = rel(c, k), theirs = rel(j, kr);
        if (mine < theirs || (mine == theirs && c < j)) continue;  // the other direction is kept
      }
      keep[k] = 1;
    }
  // Kahn: indegree = kept couplings of the row; dependents of j
  std::vector<int> indeg(nc, 0), dptr(nc + 1, 0), deps;
  for (int c = 0; c < nc; ++c)
    for (int k = rp[c]; k < rp[c + 1]; ++k)
      if (keep[k]) {
        ++indeg[c];
        ++dptr[ci[k] + 1];
      }
  for (int j = 0; j < nc; ++j) dptr[j + 1] += dptr[j];
  deps.resize(dptr[nc]);
  {
    std::vector<int> fill(dptr.begin(), dptr.end() - 1);
    for (int c = 0; c < nc; ++c)
      for (int k = rp[c]; k < rp[c + 1]; ++k)
        if (keep[k]) deps[fill[ci[k]]++] = c;
  }
  std::vector<int> perm, cur, next;
  std::vector<char> done(nc, 0);
  perm.reserve(nc);
  gs_level_ptr_.assign(1, 0);
  for (int c = 0; c < nc; ++c)
    if (indeg[c] == 0) cur.push_back(c);
  int released = 0, lowest = 0;
  while ((int)perm.size() < nc) {
    if (cur.empty()) {
      // a cycle: release the lowest-numbered cell not yet ordered, dropping
      // its remaining couplings (they lag one sweep)
      while (done[lowest]) ++lowest;
      for (int k = rp[lowest]; k < rp[lowest + 1]; ++k) keep[k] = 0;
      indeg[lowest] = 0;
      cur.push_back(lowest);
      ++released;
    }
    next.clear();
    for (int c : cur) {
      done[c] = 1;
      perm.push_back(c);
    }
    for (int c : cur)
      for (int q = dptr[c]; q < dptr[c + 1]; ++q) {
        const int d = deps[q];
        if (!done[d] && --indeg[d] == 0) next.push_back(d);
      }
    gs_level_ptr_.push_back((int)perm.size());
    std::sort(next.begin(), next.end());
    cur.swap(next);
  }
  gs_perm_.upload(perm, s_);
  gs_keep_.upload(keep, s_);
}

void Transport::flow_gs(const double* r, double* z) {
  const int nlev = (int)gs_level_ptr_.size() - 1;
  for (int l = 0; l < nlev; ++l) {
    const int lo = gs_level_ptr_[l], hi = gs_level_ptr_[l + 1];
    tr::tr_flow_gs_level_kernel<<<(hi - lo + 127) / 128, 128, 0, s_>>>(lo, hi, gs_perm_.get(), rp_.get(),
                                                                        col_.get(), gs_vals_, gs_keep_.get(),
                                                                        dpos_.get(), r, z);
    PMB_CHECK_LAUNCH();
  }
}

bool Transport::solve_flow(const double* d_vals, const double* b, double* x, const pmb_cpr_opts& o, double* info) {
  flow_order(d_vals);
  gs_vals_ = d_vals;
  const int nc = w_.nc;
  if (kry_.n() != nc) kry_.init(nc, std::max(1, std::min(o.restart, kMaxRestart)), s_);
  auto op = [&](const double* in, double* out) {
    tr::tr_spmv_kernel<<<(nc + 127) / 128, 128, 0, s_>>>(nc, rp_.get(), col_.get(), d_vals, in, out);
    PMB_CHECK_LAUNCH();
  };
  auto pc = [&](const double* in, double* out) { flow_gs(in, out); };
  return kry_.solve(op, pc, b, x, o.rtol, o.maxiter, info, nullptr, [] {});
}

// implicit_transport's loop (:335-402): backward Euler per substep, Newton
// with a bisection line search, the linear systems solved by FGMRES with the
// flow-ordered Gauss-Seidel sweep, and the substep control of
// newtonRaphson2ph.
void Transport::implicit_run(double* s, double tf, double nltol, int lstrials, int maxnewt, int tsref,
                             double resred, const pmb_cpr_opts& o, double* h_out6) {
  PMB_REQUIRE(flow_set_, "transport: set the flow first");
  PMB_REQUIRE(lstrials >= 1 && maxnewt >= 0 && tsref >= 0, "transport: bad Newton options");
  const int nc = w_.nc;
  if (res_.size() != (size_t)nc) {
    res_.resize(nc);
    ds_.resize(nc);
    rhs_.resize(nc);
    s0_.resize(nc);
    base_.resize(nc);
    vals_.resize(nnz());
  }
  PMB_REQUIRE(o.rtol > 0.0 && o.maxiter >= 1 && o.restart >= 1, "transport: bad linear-solver options");
  const int nb = (nc + 127) / 128;
  double* sn = sbuf_.get();  // the Newton iterate
  const double mints = tf * std::ldexp(1.0, -tsref);
  double t = 0.0, dt = tf, dtprev = -tf;
  int count = 0;
  long long newton = 0, lin_its = 0, lin_fail = 0, substeps = 0;
  while (t < tf && dt >= mints) {
    dt = std::min(dt, tf - t);
    int it = 0;
    double err = 0.0;
    while (true) {
      PMB_CUDA(cudaMemcpyAsync(s0_.get(), s, sizeof(double) * nc, cudaMemcpyDeviceToDevice, s_));
      tr::tr_start_kernel<<<nb, 128, 0, s_>>>(nc, s, sn);
      PMB_CHECK_LAUNCH();
      residual(sn, s0_.get(), dt, res_.get());
      err = absmax(nc, res_.get());
      it = 0;
      bool linfail = false;
      while (err > nltol && !linfail && it < maxnewt) {
        jacobian(sn, dt, vals_.get());
        tr::tr_neg_kernel<<<nb, 128, 0, s_>>>(nc, res_.get(), rhs_.get());
        PMB_CHECK_LAUNCH();
        double info[4] = {0.0, 0.0, 0.0, 0.0};
        const bool lin_ok = solve_flow(vals_.get(), rhs_.get(), ds_.get(), o, info);
        lin_its += (long long)info[0];
        if (!lin_ok) ++lin_fail;
        // bisection line search (_linesearch, :405-421)
        const double target = resred * err;
        PMB_CUDA(cudaMemcpyAsync(base_.get(), sn, sizeof(double) * nc, cudaMemcpyDeviceToDevice, s_));
        linfail = true;
        for (int k = 0; k < lstrials; ++k) {
          tr::tr_trial_kernel<<<nb, 128, 0, s_>>>(nc, base_.get(), ds_.get(), std::ldexp(1.0, -k), sn);
          PMB_CHECK_LAUNCH();
          residual(sn, s0_.get(), dt, res_.get());
          if (absmax(nc, res_.get()) < target) {
            linfail = false;
            break;
          }
        }
        ++it;
        ++newton;
        err = absmax(nc, res_.get());
      }
      --count;
      if (err > nltol) {
        dt = (count > 0 && dtprev > 0.0) ? dtprev : dt / 2.0;
        count = 5;
      } else {
        t += dt;
        ++substeps;
        dtprev = -dt;
        if (t < tf && it <= 5 && count < 0) {
          dtprev = dt;
          dt = std::min(1.5 * dt, tf - t);
          count = 5;
        }
        break;
      }
      if (!(dt >= mints)) break;
    }
    PMB_CUDA(cudaMemcpyAsync(s, sn, sizeof(double) * nc, cudaMemcpyDeviceToDevice, s_));
  }
  PMB_CUDA(cudaStreamSynchronize(s_));
  h_out6[0] = t;
  h_out6[1] = (double)substeps;
  h_out6[2] = (double)newton;
  h_out6[3] = (double)lin_its;
  h_out6[4] = (double)lin_fail;
  h_out6[5] = dt;
}

}  // namespace pmb

struct pmb_transport {
  std::unique_ptr<pmb::Transport> m;
};

extern "C" {

int pmb_transport_create(int32_t nc, int32_t nf, const int32_t* h_N, const double* h_pv, void* stream,
                         pmb_transport** out) {
  return pmb::guarded([&] {
    PMB_REQUIRE(out, "transport: out must not be NULL");
    auto h = std::make_unique<pmb_transport>();
    h->m = std::make_unique<pmb::Transport>(nc, nf, h_N, h_pv, (cudaStream_t)stream);
    *out = h.release();
  });
}

int pmb_transport_destroy(pmb_transport* h) {
  return pmb::guarded([&] { delete h; });
}

int pmb_transport_pattern(const pmb_transport* h, int64_t* h_nnz, int32_t* h_row_ptr, int32_t* h_col) {
  return pmb::guarded([&] {
    PMB_REQUIRE(h && h_nnz, "transport: NULL argument");
    *h_nnz = h->m->nnz();
    if (h_row_ptr) std::copy(h->m->row_ptr().begin(), h->m->row_ptr().end(), h_row_ptr);
    if (h_col) std::copy(h->m->col().begin(), h->m->col().end(), h_col);
  });
}

int pmb_transport_set_flow(pmb_transport* h, const double* d_flux, const double* d_gflux, const double* d_q,
                           const double* h_fluid4) {
  return pmb::guarded([&] {
    PMB_REQUIRE(h, "transport: NULL handle");
    h->m->set_flow(d_flux, d_gflux, d_q, h_fluid4);
  });
}

int pmb_transport_residual(pmb_transport* h, const double* d_s, const double* d_s0, double dt, double* d_res,
                           double* h_absmax) {
  return pmb::guarded([&] {
    PMB_REQUIRE(h && d_s && d_s0 && d_res, "transport: NULL argument");
    h->m->residual(d_s, d_s0, dt, d_res);
    if (h_absmax) *h_absmax = h->m->absmax(h->m->nc(), d_res);
  });
}

int pmb_transport_jacobian(pmb_transport* h, const double* d_s, double dt, double* d_vals) {
  return pmb::guarded([&] {
    PMB_REQUIRE(h && d_s && d_vals, "transport: NULL argument");
    h->m->jacobian(d_s, dt, d_vals);
  });
}

int pmb_transport_explicit(pmb_transport* h, double* d_s, double tf, double dt, double max_dt, double dt_factor,
                           double satwarn, double gravity_wave, double* h_out4) {
  return pmb::guarded([&] {
    PMB_REQUIRE(h && d_s && h_out4, "transport: NULL argument");
    h->m->explicit_run(d_s, tf, dt, max_dt, dt_factor, satwarn, gravity_wave, h_out4);
  });
}

int pmb_transport_implicit(pmb_transport* h, double* d_s, double tf, double nltol, int32_t lstrials,
                           int32_t maxnewt, int32_t tsref, double resred, const pmb_cpr_opts* opts, double* h_out6) {
  return pmb::guarded([&] {
    PMB_REQUIRE(h && d_s && opts && h_out6, "transport: NULL argument");
    h->m->implicit_run(d_s, tf, nltol, lstrials, maxnewt, tsref, resred, *opts, h_out6);
  });
}

}  // extern "C"
