// Three-phase black-oil model with dissolved gas on the device: the
// fully-implicit equations of ThreePhaseBlackOilModelAD
// (pymrst/modules/ad_blackoil/models/three_phase_black_oil_model.py:314-565)
// with the deck-table fluid of init_deck_blackoil_fluid
// (pymrst/modules/ad_props/props/init_deck_adi_fluid.py:60-200).
//
// Derivatives come from forward-mode dual numbers evaluated in the kernels
// (three per cell: p, sW and the switching variable x = rs or sG), so the
// Jacobian is exact for the piecewise-linear tables; values are formed with
// explicit roundings in the reference's order of operations.
//
// Layout.  The state is one FP64 vector [p | sW | sO | sG | rs | status |
// qWs | qOs | qGs | bhp] (nc entries per cell field, nw per well field,
// status 1 = undersaturated, 3 = free gas present).  The residual and the
// Jacobian are in the reference's variable-blocked order (equations water,
// oil, gas of all cells, then the three well-rate equations and the control
// equation of all wells; unknowns p, sW, x of all cells, then qWs, qOs, qGs,
// bhp), so the Jacobian goes straight to the CSR CPR solver (csrcpr.cu) and
// compares entry by entry with the reference's combine_equations output.
//
// Kernels: bo_props_kernel (per cell: every cell property with its three
// derivatives), bo_cell_kernel (per cell, gather over its interfaces:
// accumulation and the three phase fluxes, the cell rows of the Jacobian;
// no atomics), bo_well_kernel (per well: perforation rates with the
// well-stream mixture, the well rows, the perforated cells' well terms),
// bo_conv_* (CNV / MB / well tests and the CPR weights), bo_update_kernel
// (the Newton update with the reference's limits and the black-oil flash).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <numeric>
#include <vector>

#include "pmb_common.cuh"

namespace pmb {
namespace bo {

constexpr int kMaxPerfW = 16;               // perforations per well
constexpr int kWV = 4 + 3 * kMaxPerfW;      // well-local unknowns: qWs qOs qGs bhp, then (p, sW, x) per perforation
constexpr int kNumProps = 17;
constexpr double kEtol = 1.4901161193847656e-08;  // sqrt(double epsilon)

// Property slots of the per-cell property arrays (double4: value, d/dp, d/dsW, d/dx).
enum Prop { KR_W = 0, KR_O, KR_G, MU_W, MU_O, MU_G, B_W, B_O, B_G, RHO_W, RHO_O, RHO_G, P_W, P_O, P_G, RS, PV };

// ---- explicitly rounded arithmetic (no contraction into fma) --------------------
__device__ __forceinline__ double ad(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sb(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double ml(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dv(double a, double b) { return __ddiv_rn(a, b); }

// ---- dual numbers ---------------------------------------------------------------
template <int N>
struct Dual {
  double v;
  double d[N];
};

template <int N>
__device__ __forceinline__ Dual<N> dconst(double v) {
  Dual<N> r;
  r.v = v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = 0.0;
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> dvar(double v, int k) {
  Dual<N> r = dconst<N>(v);
  r.d[k] = 1.0;
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator+(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = ad(a.v, b.v);
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + b.d[i];
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = sb(a.v, b.v);
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - b.d[i];
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a) {
  Dual<N> r;
  r.v = -a.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = -a.d[i];
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = ml(a.v, b.v);
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = dv(a.v, b.v);
  const double ib = 1.0 / b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * ib;
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(double s, const Dual<N>& a) {
  Dual<N> r;
  r.v = ml(s, a.v);
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = s * a.d[i];
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(const Dual<N>& a, double s) {
  Dual<N> r;
  r.v = ml(a.v, s);
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * s;
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator+(const Dual<N>& a, double s) {
  Dual<N> r = a;
  r.v = ad(a.v, s);
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator+(double s, const Dual<N>& a) {
  Dual<N> r = a;
  r.v = ad(s, a.v);
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(double s, const Dual<N>& a) {
  Dual<N> r;
  r.v = sb(s, a.v);
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = -a.d[i];
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a, double s) {
  Dual<N> r = a;
  r.v = sb(a.v, s);
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, double s) {
  Dual<N> r;
  r.v = dv(a.v, s);
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] / s;
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator/(double s, const Dual<N>& b) {
  Dual<N> r;
  r.v = dv(s, b.v);
  const double ib = 1.0 / b.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = -r.v * b.d[i] * ib;
  return r;
}
// f(x) with f'(x) = slope, chained.
template <int N>
__device__ __forceinline__ Dual<N> chain(double fv, double slope, const Dual<N>& x) {
  Dual<N> r;
  r.v = fv;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = slope * x.d[i];
  return r;
}
// f(x, y) with partials fx, fy.
template <int N>
__device__ __forceinline__ Dual<N> chain2(double fv, double fx, const Dual<N>& x, double fy, const Dual<N>& y) {
  Dual<N> r;
  r.v = fv;
#pragma unroll
  for (int i = 0; i < N; ++i) r.d[i] = fx * x.d[i] + fy * y.d[i];
  return r;
}

// ---- tables -------------------------------------------------------------------------
struct Table {
  int n;
  const double* x;
  const double* f;
};

// Bracket index: clip(searchsorted(x, v, 'right') - 1, 0, n - 2).
__device__ __forceinline__ int bracket(const double* x, int n, double v) {
  int lo = 0, hi = n;  // count of x[i] <= v
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (x[mid] <= v) lo = mid + 1; else hi = mid;
  }
  int i = lo - 1;
  if (i < 0) i = 0;
  if (i > n - 2) i = n - 2;
  return i;
}

// interp_table (pymrst/utils/interp_table.py:17-30): weights form
// f0 (1 - t) + f1 t with linear extrapolation; slope (f1 - f0) / (x1 - x0).
__device__ __forceinline__ double interp_w(const double* x, const double* f, int n, double v, double* slope) {
  const int i = bracket(x, n, v);
  const double x0 = x[i], x1 = x[i + 1], f0 = f[i], f1 = f[i + 1];
  const double h = sb(x1, x0);
  *slope = dv(sb(f1, f0), h);
  const double t = dv(sb(v, x0), h);
  return ad(ml(f0, sb(1.0, t)), ml(f1, t));
}

// The slope form f0 + slope (x - x0) of the keyed PVT tables
// (pymrst/modules/ad_props/utils/interp_pvt.py:_interp1_slope).
// xoff shifts the abscissae: the table used is x[i] - xoff.
__device__ __forceinline__ double interp_s(const double* x, const double* f, int n, double v, double* slope,
                                           double xoff = 0.0, bool shifted = false) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    const double xm = shifted ? sb(x[mid], xoff) : x[mid];
    if (xm <= v) lo = mid + 1; else hi = mid;
  }
  int i = lo - 1;
  if (i < 0) i = 0;
  if (i > n - 2) i = n - 2;
  const double x0 = shifted ? sb(x[i], xoff) : x[i];
  const double x1 = shifted ? sb(x[i + 1], xoff) : x[i + 1];
  const double f0 = f[i], f1 = f[i + 1];
  *slope = dv(sb(f1, f0), sb(x1, x0));
  return ad(f0, ml(*slope, sb(v, x0)));
}

template <int N>
__device__ __forceinline__ Dual<N> interp_w(const Table& t, const Dual<N>& x) {
  double s;
  const double f = interp_w(t.x, t.f, t.n, x.v, &s);
  return chain(f, s, x);
}

// Keyed live-oil table (PVTO): one pressure branch per Rs key, the rows of
// branch k are [br_ptr[k], br_ptr[k+1]); sat_x / sat_f the first row of
// each branch (the saturated curve).
struct Pvt {
  int nk;
  const double* key;
  const int* br_ptr;
  const double* br_p;
  const double* br_f;
  const double* sat_x;
  const double* sat_f;
};

// pvt_interp with the 'parallel' strategy (interp_pvt.py:_pvt_values): the
// saturated curve where the cell is saturated (and above the first bubble
// point), else the two branches bracketing rs, each measured from its own
// bubble point, blended linearly in rs.  Returns f, df/dp, df/drs.
__device__ double pvt_eval(const Pvt& t, double p, double rs, bool sat, double* dfdp, double* dfdr) {
  if (sat && !(p < t.sat_x[0])) {
    *dfdr = 0.0;
    return interp_s(t.sat_x, t.sat_f, t.nk, p, dfdp);
  }
  // getBins: bin from the keys with -inf / +inf at the ends
  int bin = 0;
  for (int i = 1; i < t.nk - 1; ++i)
    if (t.key[i] <= rs) bin = i;
  const double kh = sb(t.key[bin + 1], t.key[bin]);
  const double w = dv(sb(rs, t.key[bin]), kh);
  const double dwdr = dv(1.0, kh);
  double dpsdr;
  const double ps = interp_s(t.key, t.sat_x, t.nk, rs, &dpsdr);
  const double dp = sb(p, ps);
  const int bl = bin + 1, br = bin;
  double df_l, df_r;
  const int ol = t.br_ptr[bl], nl = t.br_ptr[bl + 1] - ol;
  const int orr = t.br_ptr[br], nr = t.br_ptr[br + 1] - orr;
  const double f_l = interp_s(t.br_p + ol, t.br_f + ol, nl, dp, &df_l, t.br_p[ol], true);
  const double f_r = interp_s(t.br_p + orr, t.br_f + orr, nr, dp, &df_r, t.br_p[orr], true);
  const double omw = sb(1.0, w);
  const double f = ad(ml(f_l, w), ml(f_r, omw));
  *dfdp = ad(ml(df_l, w), ml(df_r, omw));
  *dfdr = sb(ml(sb(f_l, f_r), dwdr), ml(*dfdp, dpsdr));
  return f;
}

struct Fluid {
  double rhoS[3];
  double w_pref, w_bref, w_c, w_mu;
  double r_pref, r_c;
  double swcon;
  Table gas_b, gas_mu, rssat, krw, pcow, krow, krg, pcog, krog;  // pcow / pcog: n = 0 when absent
  Pvt oil_b, oil_mu;
};

// b_w(p) = (1 + x + x^2/2) / b_ref, x = c (p - p_ref) (assignPVTW).
template <int N>
__device__ __forceinline__ Dual<N> water_b(const Fluid& fl, const Dual<N>& p) {
  const Dual<N> x = fl.w_c * (p - fl.w_pref);
  return ((1.0 + x) + 0.5 * (x * x)) / fl.w_bref;
}

// pv_mult(p) = 1 + x + x^2/2, x = c (p - p_ref) (assignROCK).
template <int N>
__device__ __forceinline__ Dual<N> rock_mult(const Fluid& fl, const Dual<N>& p) {
  const Dual<N> x = fl.r_c * (p - fl.r_pref);
  return (1.0 + x) + 0.5 * (x * x);
}

__device__ __forceinline__ double water_b_val(const Fluid& fl, double p) {
  const double x = ml(fl.w_c, sb(p, fl.w_pref));
  return dv(ad(ad(1.0, x), ml(0.5, ml(x, x))), fl.w_bref);
}
__device__ __forceinline__ double rock_mult_val(const Fluid& fl, double p) {
  const double x = ml(fl.r_c, sb(p, fl.r_pref));
  return ad(ad(1.0, x), ml(0.5, ml(x, x)));
}
__device__ __forceinline__ double oil_b_val(const Fluid& fl, double p, double rs, bool sat) {
  double a, b;
  return pvt_eval(fl.oil_b, p, rs, sat, &a, &b);
}
__device__ __forceinline__ double gas_b_val(const Fluid& fl, double p) {
  double s;
  return interp_w(fl.gas_b.x, fl.gas_b.f, fl.gas_b.n, p, &s);
}
__device__ __forceinline__ double rssat_val(const Fluid& fl, double p) {
  double s;
  return interp_w(fl.rssat.x, fl.rssat.f, fl.rssat.n, p, &s);
}

template <int N>
__device__ __forceinline__ Dual<N> pvt(const Pvt& t, const Dual<N>& p, const Dual<N>& rs, bool sat) {
  double fp, fr;
  const double f = pvt_eval(t, p.v, rs.v, sat, &fp, &fr);
  return chain2(f, fp, p, fr, rs);
}

struct View {
  int nc, nf, nw, nperf;
  const int* N;          // nf x 2
  const double* T;
  const double* gdz;
  const double* pv_ref;
  const int* adj_ptr;    // nc + 1: interfaces of each cell, ascending
  const int* adj;        // f if the cell is N[f,0], -(f+1) if N[f,1]
  const int* adj_rank;   // rank of the cell across interface adj[k] in the cell's column list
  const int* deg;        // nc: columns per variable block of a cell row
  const int* diag_rank;  // nc
  const int* cell_well;  // nc: well perforating the cell, or -1
  const int* row_ptr;    // n + 1
  // wells
  const int* perf_ptr;   // nw + 1
  const int* perf_cell;
  const double* perf_WI;
  const int* pair_off;   // nw: offset into pair_rank of well k (np_k^2 entries)
  const int* pair_rank;  // rank of perforation j's cell in the column list of perforation i's cell
  const int* perf_srank; // rank of the perforation's cell among its well's sorted cells
  const int* well_type;  // 0 bhp, 1 rate (total surface rate), 2 orat
  const double* well_val;
  const double* compi;   // nw x 3
  double q_ref, tol_cnv, tol_mb, tol_well, ds_max, pv_tot;
  Fluid fl;
};

// State field offsets.
struct SV {
  int nc, nw;
  __host__ __device__ long long p() const { return 0; }
  __host__ __device__ long long sw() const { return nc; }
  __host__ __device__ long long so() const { return 2LL * nc; }
  __host__ __device__ long long sg() const { return 3LL * nc; }
  __host__ __device__ long long rs() const { return 4LL * nc; }
  __host__ __device__ long long st() const { return 5LL * nc; }
  __host__ __device__ long long q(int ph) const { return 6LL * nc + (long long)ph * nw; }
  __host__ __device__ long long bhp() const { return 6LL * nc + 3LL * nw; }
  __host__ __device__ long long size() const { return 6LL * nc + 4LL * nw; }
};

__device__ __forceinline__ double4 pack(const Dual<3>& a) { return make_double4(a.v, a.d[0], a.d[1], a.d[2]); }

// Primary variables of a cell as duals (p, sW, x), x = rs (undersaturated) or sG.
struct CellVars {
  Dual<3> p, sw, rs, sg, so;
  bool st1, st3;
};

__device__ __forceinline__ CellVars cell_vars(const View& v, const double* x, int c) {
  const SV s{v.nc, v.nw};
  CellVars cv;
  const double status = x[s.st() + c];
  cv.st1 = status == 1.0;
  cv.st3 = status == 3.0;
  const double xv = cv.st1 ? x[s.rs() + c] : x[s.sg() + c];
  cv.p = dvar<3>(x[s.p() + c], 0);
  cv.sw = dvar<3>(x[s.sw() + c], 1);
  const Dual<3> xd = dvar<3>(xv, 2);
  // rs = x st1 + rsSat(p) (1 - st1); sG = x st3 (assemble, :318-322)
  const Dual<3> rssat = interp_w(v.fl.rssat, cv.p);
  cv.rs = cv.st1 ? xd : rssat;
  cv.sg = cv.st3 ? xd : dconst<3>(0.0);
  cv.so = (1.0 - cv.sw) - cv.sg;
  return cv;
}

__global__ void __launch_bounds__(128) bo_props_kernel(View v, const double* __restrict__ x, double4* __restrict__ props) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= v.nc) return;
  const Fluid& fl = v.fl;
  const CellVars cv = cell_vars(v, x, c);
  const long long nc = v.nc;
  // relative permeabilities (SWOF / SGOF tables, flat-extended) and the
  // saturation-weighted three-phase oil curve (BlackOilFluid.kr_o)
  const Dual<3> krw = interp_w(fl.krw, cv.sw);
  const Dual<3> krg = interp_w(fl.krg, cv.sg);
  const double swcon = fmin(fl.swcon, sb(cv.sw.v, 1e-5));
  const Dual<3> dd = (cv.sg + cv.sw) - swcon;
  const Dual<3> ww = (cv.sw - swcon) / dd;
  const Dual<3> kro = (1.0 - ww) * interp_w(fl.krog, cv.so) + ww * interp_w(fl.krow, cv.so);
  // phase pressures
  const Dual<3> pcow = fl.pcow.n ? interp_w(fl.pcow, cv.sw) : dconst<3>(0.0);
  const Dual<3> pcog = fl.pcog.n ? interp_w(fl.pcog, cv.sg) : dconst<3>(0.0);
  const Dual<3> pw = cv.p - pcow;
  const Dual<3> pg = cv.p + pcog;
  // PVT
  const Dual<3> bw = water_b<3>(fl, pw);
  const Dual<3> muw = dconst<3>(fl.w_mu);
  const Dual<3> bo = pvt(fl.oil_b, cv.p, cv.rs, cv.st3);
  const Dual<3> muo = pvt(fl.oil_mu, cv.p, cv.rs, cv.st3);
  const Dual<3> bg = interp_w(fl.gas_b, pg);
  const Dual<3> mug = interp_w(fl.gas_mu, pg);
  const Dual<3> rhow = bw * fl.rhoS[0];
  const Dual<3> rhoo = bo * (cv.rs * fl.rhoS[2] + fl.rhoS[1]);
  const Dual<3> rhog = bg * ad(ml(0.0, fl.rhoS[1]), fl.rhoS[2]);
  const Dual<3> pv = v.pv_ref[c] * rock_mult<3>(fl, cv.p);
  props[KR_W * nc + c] = pack(krw);
  props[KR_O * nc + c] = pack(kro);
  props[KR_G * nc + c] = pack(krg);
  props[MU_W * nc + c] = pack(muw);
  props[MU_O * nc + c] = pack(muo);
  props[MU_G * nc + c] = pack(mug);
  props[B_W * nc + c] = pack(bw);
  props[B_O * nc + c] = pack(bo);
  props[B_G * nc + c] = pack(bg);
  props[RHO_W * nc + c] = pack(rhow);
  props[RHO_O * nc + c] = pack(rhoo);
  props[RHO_G * nc + c] = pack(rhog);
  props[P_W * nc + c] = pack(pw);
  props[P_O * nc + c] = pack(cv.p);
  props[P_G * nc + c] = pack(pg);
  props[RS * nc + c] = pack(cv.rs);
  props[PV * nc + c] = pack(pv);
}

// A cell property as a dual over (own p, sW, x, other p, sW, x): slot 0 puts
// the derivatives in 0..2, slot 1 in 3..5.
__device__ __forceinline__ Dual<6> lift(double4 a, int slot) {
  Dual<6> r = dconst<6>(a.x);
  r.d[3 * slot + 0] = a.y;
  r.d[3 * slot + 1] = a.z;
  r.d[3 * slot + 2] = a.w;
  return r;
}
__device__ __forceinline__ Dual<3> unpack(double4 a) {
  Dual<3> r;
  r.v = a.x;
  r.d[0] = a.y;
  r.d[1] = a.z;
  r.d[2] = a.w;
  return r;
}

// Cell rows: accumulation (assemble, :345-357) plus the divergence of the
// three surface-volume fluxes (:336-343, :355-357); the well terms are
// subtracted afterwards by bo_well_kernel.
__global__ void __launch_bounds__(128) bo_cell_kernel(View v, const double* __restrict__ x,
                                                      const double* __restrict__ x0, double dt,
                                                      const double4* __restrict__ props, double* __restrict__ res,
                                                      double* __restrict__ vals) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= v.nc) return;
  const Fluid& fl = v.fl;
  const long long nc = v.nc;
  const SV s{v.nc, v.nw};
  const CellVars cv = cell_vars(v, x, c);
  const Dual<3> pv = unpack(props[PV * nc + c]);
  const Dual<3> bw = unpack(props[B_W * nc + c]);
  const Dual<3> bo = unpack(props[B_O * nc + c]);
  const Dual<3> bg = unpack(props[B_G * nc + c]);
  // previous state (values)
  const double p0 = x0[s.p() + c];
  const double s0w = x0[s.sw() + c], s0o = x0[s.so() + c], s0g = x0[s.sg() + c];
  const double rs0 = x0[s.rs() + c];
  const bool st3_0 = x0[s.st() + c] == 3.0;
  const double pv0 = ml(v.pv_ref[c], rock_mult_val(fl, p0));
  const double bw0 = water_b_val(fl, p0);
  const double bo0 = oil_b_val(fl, p0, rs0, st3_0);
  const double bg0 = gas_b_val(fl, p0);
  const double idt = dv(1.0, dt);
  Dual<3> acc[3];
  acc[0] = idt * ((pv * bw) * cv.sw - ml(ml(pv0, bw0), s0w));
  acc[1] = idt * ((pv * bo) * cv.so - ml(ml(pv0, bo0), s0o));
  acc[2] = idt * (pv * (bg * cv.sg + (cv.rs * bo) * cv.so) - ml(pv0, ad(ml(bg0, s0g), ml(ml(rs0, bo0), s0o))));

  // zero this cell's three rows
  const int deg = v.deg[c];
  const bool perforated = v.cell_well[c] >= 0;
  const int rowlen = 3 * deg + (perforated ? 4 : 0);
  for (int e = 0; e < 3; ++e) {
    const long long base = v.row_ptr[e * nc + c];
    for (int k = 0; k < rowlen; ++k) vals[base + k] = 0.0;
  }
  // divergence, interface by interface in ascending order
  Dual<3> div[3];
  for (int e = 0; e < 3; ++e) div[e] = dconst<3>(0.0);
  for (int k = v.adj_ptr[c]; k < v.adj_ptr[c + 1]; ++k) {
    const int code = v.adj[k];
    const bool first = code >= 0;  // this cell is N[f,0]
    const int f = first ? code : -code - 1;
    const int a = v.N[2 * f], b = v.N[2 * f + 1];
    const int sa = first ? 0 : 1, sbb = first ? 1 : 0;  // derivative slots of N0 / N1
    const double T = v.T[f], gdz = v.gdz[f];
    Dual<6> flux[3];
    bool up_o = true;
    const int pslot[3] = {P_W, P_O, P_G}, rslot[3] = {RHO_W, RHO_O, RHO_G}, kslot[3] = {KR_W, KR_O, KR_G},
              mslot[3] = {MU_W, MU_O, MU_G}, bslot[3] = {B_W, B_O, B_G};
#pragma unroll
    for (int ph = 0; ph < 3; ++ph) {
      const Dual<6> rhof = 0.5 * lift(props[rslot[ph] * nc + a], sa) + 0.5 * lift(props[rslot[ph] * nc + b], sbb);
      const Dual<6> dp = (lift(props[pslot[ph] * nc + b], sbb) - lift(props[pslot[ph] * nc + a], sa)) - rhof * gdz;
      const bool up = dp.v <= 0.0;
      const int u = up ? a : b, su = up ? sa : sbb;
      const Dual<6> krf = lift(props[kslot[ph] * nc + u], su);
      const Dual<6> muf = lift(props[mslot[ph] * nc + u], su);
      const Dual<6> vph = ((-(krf / muf)) * T) * dp;
      flux[ph] = lift(props[bslot[ph] * nc + u], su) * vph;
      if (ph == 1) up_o = up;
    }
    {
      const int u = up_o ? a : b, su = up_o ? sa : sbb;
      flux[2] = flux[2] + lift(props[RS * nc + u], su) * flux[1];
    }
    const int nb_rank = v.adj_rank[k];
#pragma unroll
    for (int e = 0; e < 3; ++e) {
      const Dual<6>& fl6 = flux[e];
      if (first) {
        div[e].v = ad(div[e].v, fl6.v);
      } else {
        div[e].v = sb(div[e].v, fl6.v);
      }
      const double sg = first ? 1.0 : -1.0;
#pragma unroll
      for (int q = 0; q < 3; ++q) div[e].d[q] += sg * fl6.d[q];
      const long long base = v.row_ptr[e * nc + c];
#pragma unroll
      for (int q = 0; q < 3; ++q) vals[base + (long long)q * deg + nb_rank] += sg * fl6.d[3 + q];
    }
  }
  const int dr = v.diag_rank[c];
#pragma unroll
  for (int e = 0; e < 3; ++e) {
    const Dual<3> r = acc[e] + div[e];
    res[e * nc + c] = r.v;
    const long long base = v.row_ptr[e * nc + c];
#pragma unroll
    for (int q = 0; q < 3; ++q) vals[base + (long long)q * deg + dr] += r.d[q];
  }
}

// ---- wells -------------------------------------------------------------------------
// Well-local dual: value and derivatives over [qWs, qOs, qGs, bhp, (p, sW, x)
// of each perforated cell].
using WD = Dual<kWV>;

__device__ __forceinline__ WD wd_from(double4 a, int perf) {
  WD r = dconst<kWV>(a.x);
  r.d[4 + 3 * perf + 0] = a.y;
  r.d[4 + 3 * perf + 1] = a.z;
  r.d[4 + 3 * perf + 2] = a.w;
  return r;
}

// One thread per well: the single-well model with dissolved gas
// (ThreePhaseBlackOilModelAD._well, :383-437).
__global__ void bo_well_kernel(View v, const double* __restrict__ x, const double4* __restrict__ props,
                               double* __restrict__ res, double* __restrict__ vals) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= v.nw) return;
  const long long nc = v.nc;
  const int nw = v.nw;
  const SV s{v.nc, v.nw};
  const int p0 = v.perf_ptr[k], np = v.perf_ptr[k + 1] - p0;
  WD q[3];
  for (int ph = 0; ph < 3; ++ph) q[ph] = dvar<kWV>(x[s.q(ph) + k], ph);
  const WD bhp = dvar<kWV>(x[s.bhp() + k], 3);
  const double compi[3] = {v.compi[3 * k], v.compi[3 * k + 1], v.compi[3 * k + 2]};

  bool any_inj = false, any_prod = false;
  for (int i = 0; i < np; ++i) {
    const int c = v.perf_cell[p0 + i];
    const double dd = ad(-x[s.bhp() + k], x[s.p() + c]);
    if (dd < 0.0) any_inj = true; else any_prod = true;
  }
  // mixture of the well stream (producing perforations and positive rates)
  WD mix[3];
  if (any_prod) {
    WD wbq[3];
    for (int ph = 0; ph < 3; ++ph) wbq[ph] = q[ph] * (q[ph].v > 0.0 ? 1.0 : 0.0);
    WD sum[3];
    for (int ph = 0; ph < 3; ++ph) sum[ph] = dconst<kWV>(0.0);
    for (int i = 0; i < np; ++i) {
      const int c = v.perf_cell[p0 + i];
      const WD dd = (-bhp) + wd_from(props[P_O * nc + c], i);
      const double con = (dd.v < 0.0 ? 0.0 : 1.0) * v.perf_WI[p0 + i];
      const WD mw = wd_from(props[KR_W * nc + c], i) / wd_from(props[MU_W * nc + c], i);
      const WD mo = wd_from(props[KR_O * nc + c], i) / wd_from(props[MU_O * nc + c], i);
      const WD mg = wd_from(props[KR_G * nc + c], i) / wd_from(props[MU_G * nc + c], i);
      const WD cw = ((-con) * mw) * dd, co = ((-con) * mo) * dd, cg = ((-con) * mg) * dd;
      const WD bo_co = wd_from(props[B_O * nc + c], i) * co;
      sum[0] = sum[0] + wd_from(props[B_W * nc + c], i) * cw;
      sum[1] = sum[1] + bo_co;
      sum[2] = sum[2] + (wd_from(props[B_G * nc + c], i) * cg + wd_from(props[RS * nc + c], i) * bo_co);
    }
    for (int ph = 0; ph < 3; ++ph) wbq[ph] = wbq[ph] - sum[ph];
    const WD wbqt = (wbq[0] + wbq[1]) + wbq[2];
    for (int ph = 0; ph < 3; ++ph) mix[ph] = wbqt.v == 0.0 ? dconst<kWV>(compi[ph]) : wbq[ph] / wbqt;
  } else {
    for (int ph = 0; ph < 3; ++ph) mix[ph] = dconst<kWV>(compi[ph]);
  }
  WD weq[3];
  for (int ph = 0; ph < 3; ++ph) weq[ph] = dconst<kWV>(0.0);
  for (int i = 0; i < np; ++i) {
    const int c = v.perf_cell[p0 + i];
    const WD dd = (-bhp) + wd_from(props[P_O * nc + c], i);
    const bool inj = dd.v < 0.0;
    const WD mw = wd_from(props[KR_W * nc + c], i) / wd_from(props[MU_W * nc + c], i);
    const WD mo = wd_from(props[KR_O * nc + c], i) / wd_from(props[MU_O * nc + c], i);
    const WD mg = wd_from(props[KR_G * nc + c], i) / wd_from(props[MU_G * nc + c], i);
    const WD bw = wd_from(props[B_W * nc + c], i), bo = wd_from(props[B_O * nc + c], i),
             bg = wd_from(props[B_G * nc + c], i), rs = wd_from(props[RS * nc + c], i);
    const double tw = v.perf_WI[p0 + i];
    WD cq[3];
    if (any_prod) {
      const double con = (inj ? 0.0 : 1.0) * tw;
      const WD cw = ((-con) * mw) * dd, co = ((-con) * mo) * dd, cg = ((-con) * mg) * dd;
      cq[0] = bw * cw;
      cq[1] = bo * co;
      cq[2] = bg * cg + rs * (bo * co);
    }
    if (any_inj) {
      const WD mt = (mw + mo) + mg;
      const WD cqt = (-((inj ? 1.0 : 0.0) * tw)) * (mt * dd);
      const WD vol_rat = (mix[0] / bw + mix[1] / bo) + (mix[2] - rs * mix[1]) / bg;
      const WD cqts = cqt / vol_rat;
      for (int ph = 0; ph < 3; ++ph) cq[ph] = any_prod ? cq[ph] + mix[ph] * cqts : mix[ph] * cqts;
    }
    // the perforated cell's rows lose what the perforation takes
    const int deg = v.deg[c];
    for (int ph = 0; ph < 3; ++ph) {
      res[ph * nc + c] = sb(res[ph * nc + c], cq[ph].v);
      const long long base = v.row_ptr[ph * nc + c];
      for (int j = 0; j < np; ++j) {
        const int rk = v.pair_rank[v.pair_off[k] + i * np + j];
        for (int q3 = 0; q3 < 3; ++q3) vals[base + (long long)q3 * deg + rk] -= cq[ph].d[4 + 3 * j + q3];
      }
      for (int m = 0; m < 4; ++m) vals[base + 3LL * deg + m] -= cq[ph].d[m];
      weq[ph] = weq[ph] + cq[ph];
    }
  }
  // well-rate equations q_s - sum cq_s, then the control
  for (int ph = 0; ph < 3; ++ph) {
    const WD e = q[ph] - weq[ph];
    const long long row = 3LL * nc + (long long)ph * nw + k;
    res[row] = e.v;
    const long long base = v.row_ptr[row];
    for (int i = 0; i < np; ++i) {
      const int r = v.perf_srank[p0 + i];
      for (int q3 = 0; q3 < 3; ++q3) vals[base + (long long)q3 * np + r] = e.d[4 + 3 * i + q3];
    }
    for (int m = 0; m < 4; ++m) vals[base + 3LL * np + m] = e.d[m];
  }
  WD ctrl;
  const int type = v.well_type[k];
  if (type == 0) ctrl = bhp - v.well_val[k];
  else if (type == 1) ctrl = ((q[0] + q[1]) + q[2]) - v.well_val[k];
  else ctrl = q[1] - v.well_val[k];
  const long long row = 3LL * nc + 3LL * nw + k;
  res[row] = ctrl.v;
  const long long base = v.row_ptr[row];
  for (int m = 0; m < 4; ++m) vals[base + m] = ctrl.d[m];
}

// ---- convergence ----------------------------------------------------------------------
constexpr int kConvBlocks = 2 * kNumSM;
constexpr int kConvThreads = 256;
constexpr int kConvSums = 8;   // sum 1/bW, 1/bO, 1/bG, pv, rW, rO, rG, p
constexpr int kConvMax = 3;    // max |r_i / pv|

__global__ void __launch_bounds__(kConvThreads) bo_conv_partial_kernel(View v, const double* __restrict__ res,
                                                                        const double* __restrict__ x,
                                                                        double* __restrict__ part) {
  const SV s{v.nc, v.nw};
  const Fluid& fl = v.fl;
  double sum[kConvSums], mx[kConvMax];
  for (int i = 0; i < kConvSums; ++i) sum[i] = 0.0;
  for (int i = 0; i < kConvMax; ++i) mx[i] = 0.0;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < v.nc; c += gridDim.x * blockDim.x) {
    const double p = x[s.p() + c];
    const bool st3 = x[s.st() + c] == 3.0;
    const double pv = ml(v.pv_ref[c], rock_mult_val(fl, p));
    sum[0] += 1.0 / water_b_val(fl, p);
    sum[1] += 1.0 / oil_b_val(fl, p, x[s.rs() + c], st3);
    sum[2] += 1.0 / gas_b_val(fl, p);
    sum[3] += pv;
    for (int e = 0; e < 3; ++e) {
      const double r = res[(long long)e * v.nc + c];
      sum[4 + e] += r;
      const double a = fabs(r / pv);
      mx[e] = (a > mx[e] || a != a) ? a : mx[e];
    }
    sum[7] += p;
  }
  __shared__ double sh[kConvThreads / 32][kConvSums + kConvMax];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int i = 0; i < kConvSums; ++i)
    for (int o = 16; o; o >>= 1) sum[i] += __shfl_xor_sync(0xffffffffu, sum[i], o);
  for (int i = 0; i < kConvMax; ++i)
    for (int o = 16; o; o >>= 1) {
      const double b = __shfl_xor_sync(0xffffffffu, mx[i], o);
      mx[i] = (b > mx[i] || b != b) ? b : mx[i];
    }
  if (lane == 0) {
    for (int i = 0; i < kConvSums; ++i) sh[wid][i] = sum[i];
    for (int i = 0; i < kConvMax; ++i) sh[wid][kConvSums + i] = mx[i];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double out[kConvSums + kConvMax];
    for (int i = 0; i < kConvSums + kConvMax; ++i) out[i] = sh[0][i];
    for (int w = 1; w < kConvThreads / 32; ++w) {
      for (int i = 0; i < kConvSums; ++i) out[i] += sh[w][i];
      for (int i = 0; i < kConvMax; ++i) {
        const double b = sh[w][kConvSums + i];
        out[kConvSums + i] = (b > out[kConvSums + i] || b != b) ? b : out[kConvSums + i];
      }
    }
    for (int i = 0; i < kConvSums + kConvMax; ++i) part[(long long)blockIdx.x * (kConvSums + kConvMax) + i] = out[i];
  }
}

// out: cnv[3], mb[3], max well-rate residual / q_ref, max |ctrl| / scale,
// converged, CPR weights 1/b_i at the mean pressure [3], mean pressure, pv total.
constexpr int kConvOut = 14;

__global__ void bo_conv_final_kernel(View v, int nparts, const double* __restrict__ part,
                                     const double* __restrict__ res, double dt, double* __restrict__ out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double sum[kConvSums], mx[kConvMax];
  for (int i = 0; i < kConvSums; ++i) sum[i] = 0.0;
  for (int i = 0; i < kConvMax; ++i) mx[i] = 0.0;
  for (int b = 0; b < nparts; ++b) {
    const double* pp = part + (long long)b * (kConvSums + kConvMax);
    for (int i = 0; i < kConvSums; ++i) sum[i] += pp[i];
    for (int i = 0; i < kConvMax; ++i) mx[i] = (pp[kConvSums + i] > mx[i] || pp[kConvSums + i] != pp[kConvSums + i]) ? pp[kConvSums + i] : mx[i];
  }
  const double n = (double)v.nc;
  double cnv = 0.0, mb = 0.0;
  bool ok = true;
  for (int e = 0; e < 3; ++e) {
    const double bavg = sum[e] / n;
    const double c = bavg * dt * mx[e];
    const double m = bavg * dt * fabs(sum[4 + e]) / sum[3];
    out[e] = c;
    out[3 + e] = m;
    cnv = (c > cnv || c != c) ? c : cnv;
    mb = (m > mb || m != m) ? m : mb;
  }
  ok = cnv <= v.tol_cnv && mb <= v.tol_mb;
  // wells (_converged, :528-539)
  const long long nc = v.nc;
  double wmax = 0.0;
  for (int i = 0; i < 3 * v.nw; ++i) {
    const double a = fabs(res[3 * nc + i]);
    wmax = (a > wmax || a != a) ? a : wmax;
  }
  const bool well_ok = wmax <= v.tol_well * v.q_ref;
  bool ctrl_ok = true;
  double cmax = 0.0;
  for (int k = 0; k < v.nw; ++k) {
    const double scale = v.well_type[k] == 0 ? 1e5 : fabs(v.well_val[k]);
    const double a = fabs(res[3 * nc + 3LL * v.nw + k]);
    if (!(a <= v.tol_well * scale)) ctrl_ok = false;
    const double r = a / scale;
    cmax = (r > cmax || r != r) ? r : cmax;
  }
  out[6] = wmax / v.q_ref;
  out[7] = cmax;
  out[8] = (ok && well_ok && ctrl_ok) ? 1.0 : 0.0;
  // quasi-IMPES weights at the mean pressure, saturated oil (get_scaling_factors_cpr, :205-245)
  const double pm = sum[7] / n;
  const double rs = rssat_val(v.fl, pm);
  out[9] = 1.0 / water_b_val(v.fl, pm);
  out[10] = 1.0 / oil_b_val(v.fl, pm, rs, true);
  out[11] = 1.0 / gas_b_val(v.fl, pm);
  out[12] = pm;
  out[13] = sum[3];
}

// ---- Newton update and flash (update_state :439-469, _flash :471-508) ---------------
__device__ __forceinline__ double clipd(double a, double lo, double hi) { return a < lo ? lo : (a > hi ? hi : a); }
__device__ __forceinline__ double maxz(double a) { return a < 0.0 ? 0.0 : a; }          // np.maximum(a, 0)
__device__ __forceinline__ double minn(double a, double b) { return (a != a || b != b) ? (a + b) : (a < b ? a : b); }

__global__ void bo_update_kernel(View v, double* __restrict__ x, const double* __restrict__ dx) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const SV s{v.nc, v.nw};
  const long long nc = v.nc;
  if (t < v.nw) {
    for (int ph = 0; ph < 3; ++ph) x[s.q(ph) + t] = ad(x[s.q(ph) + t], dx[3 * nc + (long long)ph * v.nw + t]);
    x[s.bhp() + t] = ad(x[s.bhp() + t], dx[3 * nc + 3LL * v.nw + t]);
  }
  if (t >= v.nc) return;
  const int c = t;
  const Fluid& fl = v.fl;
  const double p_prev = x[s.p() + c], rs_prev = x[s.rs() + c], sg_prev = x[s.sg() + c];
  const bool st1 = x[s.st() + c] == 1.0, st3 = x[s.st() + c] == 3.0;
  const double dp = dx[c], dsw = dx[nc + c], dxx = dx[2 * nc + c];
  const double p = ad(p_prev, dp);
  const double dsg = st3 ? dxx : 0.0;
  double rs = maxz(ad(rs_prev, st1 ? dxx : 0.0));
  const double a = v.ds_max;
  double sw = ad(x[s.sw() + c], clipd(dsw, -a, a));
  double so = ad(x[s.so() + c], clipd(-ad(dsg, dsw), -a, a));
  double sg = ad(sg_prev, clipd(dsg, -a, a));
  // flash
  const bool wat_only = sw > 1.0 - kEtol;
  const double rs_sat = rssat_val(fl, p), rs_sat0 = rssat_val(fl, p_prev);
  bool gas = ((sg > 0.0) || (rs == 0.0)) && !st1;
  gas = gas || wat_only;
  gas = gas || ((sg < 0.0) && (sg_prev > kEtol));
  const bool ix2 = (rs > ml(rs_sat, ad(1.0, kEtol))) && st1 && (rs_prev > ml(rs_sat0, sb(1.0, kEtol)));
  if (ix2) sg = 0.0;
  gas = gas || ix2;
  if (sg < 0.0) {
    const double d = sb(1.0, sg);
    sw = dv(sw, d);
    so = dv(so, d);
    sg = 0.0;
  }
  if (so < 0.0) {
    const double d = sb(1.0, so);
    sw = dv(sw, d);
    sg = dv(sg, d);
    so = 0.0;
  }
  if (sw < 0.0) {
    const double d = sb(1.0, sw);
    so = dv(so, d);
    sg = dv(sg, d);
    sw = 0.0;
  }
  rs = gas ? rs_sat : minn(rs_sat, rs);
  rs = maxz(rs);
  const double tot = ad(ad(sw, so), sg);
  x[s.p() + c] = p;
  x[s.sw() + c] = dv(sw, tot);
  x[s.so() + c] = dv(so, tot);
  x[s.sg() + c] = dv(sg, tot);
  x[s.rs() + c] = rs;
  x[s.st() + c] = gas ? 3.0 : 1.0;
}

__global__ void bo_negate_kernel(long long n, const double* __restrict__ a, double* __restrict__ b) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    b[i] = -a[i];
}

// Fluid evaluation at points (tests and the host-side fluid check).
__global__ void bo_pvt_points_kernel(View v, int n, const double* __restrict__ p, const double* __restrict__ rs,
                                     const double* __restrict__ sat, double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Fluid& fl = v.fl;
  double a, b;
  const bool st = sat[i] != 0.0;
  out[i] = water_b_val(fl, p[i]);
  out[n + i] = pvt_eval(fl.oil_b, p[i], rs[i], st, &a, &b);
  out[2LL * n + i] = pvt_eval(fl.oil_mu, p[i], rs[i], st, &a, &b);
  out[3LL * n + i] = interp_w(fl.gas_b.x, fl.gas_b.f, fl.gas_b.n, p[i], &a);
  out[4LL * n + i] = interp_w(fl.gas_mu.x, fl.gas_mu.f, fl.gas_mu.n, p[i], &a);
  out[5LL * n + i] = rssat_val(fl, p[i]);
  out[6LL * n + i] = rock_mult_val(fl, p[i]);
}

__global__ void bo_relperm_points_kernel(View v, int n, const double* __restrict__ sw, const double* __restrict__ sg,
                                         double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Fluid& fl = v.fl;
  const Dual<3> w = dvar<3>(sw[i], 1), g = dvar<3>(sg[i], 2);
  const Dual<3> o = (1.0 - w) - g;
  const double swcon = fmin(fl.swcon, sb(w.v, 1e-5));
  const Dual<3> ww = (w - swcon) / ((g + w) - swcon);
  out[i] = interp_w(fl.krw, w).v;
  out[n + i] = ((1.0 - ww) * interp_w(fl.krog, o) + ww * interp_w(fl.krow, o)).v;
  out[2LL * n + i] = interp_w(fl.krg, g).v;
  out[3LL * n + i] = fl.pcow.n ? interp_w(fl.pcow, w).v : 0.0;
  out[4LL * n + i] = fl.pcog.n ? interp_w(fl.pcog, g).v : 0.0;
}

}  // namespace bo

// ---- host model --------------------------------------------------------------------------
class BOModel {
 public:
  BOModel(const pmb_bo_desc& d, cudaStream_t s);
  ~BOModel() {
    if (cpr_) pmb_csr_cpr_destroy(cpr_);
  }
  int64_t n() const { return 3LL * v_.nc + 4LL * v_.nw; }
  int64_t nnz() const { return h_row_ptr_.back(); }
  int64_t state_size() const { return 6LL * v_.nc + 4LL * v_.nw; }
  const std::vector<int>& row_ptr() const { return h_row_ptr_; }
  const std::vector<int>& col() const { return h_col_; }
  void assemble(const double* x, const double* x0, double dt, double* res, double* vals);
  void convergence(const double* res, const double* x, double dt, double* h_out);
  void update(double* x, const double* dx);
  void step(double* x, double dt, int maxit, const pmb_cpr_opts& o, double* stats);
  void pvt_points(int n, const double* p, const double* rs, const double* sat, double* out);
  void relperm_points(int n, const double* sw, const double* sg, double* out);

 private:
  cudaStream_t s_;
  bo::View v_{};
  std::vector<int> h_row_ptr_, h_col_;
  DArray<int> N_, adj_ptr_, adj_, adj_rank_, deg_, diag_rank_, cell_well_, row_ptr_, perf_ptr_, perf_cell_,
      pair_off_, pair_rank_, perf_srank_, well_type_, br_ptr_;
  DArray<double> T_, gdz_, pv_, perf_WI_, well_val_, compi_, tab_;
  DArray<double4> props_;
  DArray<double> part_, conv_out_, res_, vals_, rhs_, dx_, x0_;
  PinnedArray<double> h_conv_;
  pmb_csr_cpr* cpr_ = nullptr;
  pmb_cpr_opts cpr_opts_{};

 public:
  bool cell_weights_ = false;
};

namespace {
template <class T>
std::vector<T> hv(const T* p, int64_t n) {
  return std::vector<T>(p, p + n);
}
}  // namespace

BOModel::BOModel(const pmb_bo_desc& d, cudaStream_t s) : s_(s) {
  PMB_REQUIRE(d.nc > 0 && d.nf >= 0 && d.nw >= 0, "bo: sizes must be nc > 0, nf >= 0, nw >= 0");
  PMB_REQUIRE(d.h_N && d.h_T && d.h_gdz && d.h_pv, "bo: grid arrays must not be NULL");
  const int nc = d.nc, nf = d.nf, nw = d.nw;
  // ---- fluid tables into one device buffer
  std::vector<double> tab;
  auto put = [&](const double* p, int n, const char* what) -> int64_t {
    PMB_REQUIRE(n >= 2 && p != nullptr, std::string("bo: table ") + what + " needs at least two rows");
    const int64_t off = (int64_t)tab.size();
    tab.insert(tab.end(), p, p + n);
    return off;
  };
  auto incr = [&](const double* x, int n, const char* what) {
    for (int i = 1; i < n; ++i)
      PMB_REQUIRE(x[i] > x[i - 1], std::string("bo: abscissae of ") + what + " must be strictly increasing");
  };
  struct TabOff { int n; int64_t x, f; };
  auto table = [&](int n, const double* x, const double* f, const char* what) {
    incr(x, n, what);
    TabOff t{n, put(x, n, what), put(f, n, what)};
    return t;
  };
  TabOff gb = table(d.n_gas, d.h_gas_p, d.h_gas_b, "gas b"), gm = table(d.n_gas, d.h_gas_p, d.h_gas_mu, "gas mu");
  TabOff rss = table(d.n_rssat, d.h_rssat_p, d.h_rssat_rs, "rs_sat");
  TabOff tkrw = table(d.n_sw, d.h_sw, d.h_krw, "krw");
  TabOff tpcw = d.h_pcow ? table(d.n_sw, d.h_sw, d.h_pcow, "pcow") : TabOff{0, 0, 0};
  TabOff tkrow = table(d.n_sow, d.h_sow, d.h_krow, "krow");
  TabOff tkrg = table(d.n_sg, d.h_sg, d.h_krg, "krg");
  TabOff tpcg = d.h_pcog ? table(d.n_sg, d.h_sg, d.h_pcog, "pcog") : TabOff{0, 0, 0};
  TabOff tkrog = table(d.n_sog, d.h_sog, d.h_krog, "krog");
  const int nk = d.n_key;
  PMB_REQUIRE(nk >= 2 && d.h_key && d.h_branch_ptr && d.h_branch_p && d.h_branch_b && d.h_branch_mu,
              "bo: the live-oil table needs at least two Rs keys");
  incr(d.h_key, nk, "Rs keys");
  std::vector<int> bptr = hv(d.h_branch_ptr, nk + 1);
  PMB_REQUIRE(bptr[0] == 0, "bo: branch_ptr[0] must be 0");
  std::vector<double> sat_x(nk), sat_b(nk), sat_mu(nk);
  for (int k = 0; k < nk; ++k) {
    PMB_REQUIRE(bptr[k + 1] - bptr[k] >= 2, "bo: every live-oil branch needs at least two rows");
    incr(d.h_branch_p + bptr[k], bptr[k + 1] - bptr[k], "a live-oil branch");
    sat_x[k] = d.h_branch_p[bptr[k]];
    sat_b[k] = d.h_branch_b[bptr[k]];
    sat_mu[k] = d.h_branch_mu[bptr[k]];
  }
  const int nrows = bptr[nk];
  const int64_t o_key = put(d.h_key, nk, "keys");
  const int64_t o_bp = put(d.h_branch_p, nrows, "branch p");
  const int64_t o_bb = put(d.h_branch_b, nrows, "branch b");
  const int64_t o_bm = put(d.h_branch_mu, nrows, "branch mu");
  const int64_t o_sx = put(sat_x.data(), nk, "sat x");
  const int64_t o_sb = put(sat_b.data(), nk, "sat b");
  const int64_t o_sm = put(sat_mu.data(), nk, "sat mu");
  tab_.upload(tab, s);
  br_ptr_.upload(bptr, s);
  const double* tb = tab_.get();
  auto dtab = [&](const TabOff& t) { return bo::Table{t.n, tb + t.x, tb + t.f}; };
  bo::Fluid& fl = v_.fl;
  for (int i = 0; i < 3; ++i) fl.rhoS[i] = d.rhoS[i];
  fl.w_pref = d.pvtw[0];
  fl.w_bref = d.pvtw[1];
  fl.w_c = d.pvtw[2];
  fl.w_mu = d.pvtw[3];
  fl.r_pref = d.rock[0];
  fl.r_c = d.rock[1];
  fl.swcon = d.swcon;
  fl.gas_b = dtab(gb);
  fl.gas_mu = dtab(gm);
  fl.rssat = dtab(rss);
  fl.krw = dtab(tkrw);
  fl.pcow = dtab(tpcw);
  fl.krow = dtab(tkrow);
  fl.krg = dtab(tkrg);
  fl.pcog = dtab(tpcg);
  fl.krog = dtab(tkrog);
  fl.oil_b = bo::Pvt{nk, tb + o_key, br_ptr_.get(), tb + o_bp, tb + o_bb, tb + o_sx, tb + o_sb};
  fl.oil_mu = bo::Pvt{nk, tb + o_key, br_ptr_.get(), tb + o_bp, tb + o_bm, tb + o_sx, tb + o_sm};

  // ---- grid
  std::vector<int> N = hv(d.h_N, 2LL * nf);
  for (int f = 0; f < nf; ++f)
    PMB_REQUIRE(N[2 * f] >= 0 && N[2 * f] < nc && N[2 * f + 1] >= 0 && N[2 * f + 1] < nc &&
                    N[2 * f] != N[2 * f + 1],
                "bo: interface neighbours must be two distinct cells in [0, nc)");
  // wells
  std::vector<int> pptr = nw ? hv(d.h_perf_ptr, nw + 1) : std::vector<int>{0};
  PMB_REQUIRE(pptr[0] == 0, "bo: perf_ptr[0] must be 0");
  for (int k = 0; k < nw; ++k)
    PMB_REQUIRE(pptr[k + 1] - pptr[k] >= 1 && pptr[k + 1] - pptr[k] <= bo::kMaxPerfW,
                "bo: every well needs 1 to 16 perforations");
  const int nperf = pptr[nw];
  std::vector<int> pcell = nperf ? hv(d.h_perf_cell, nperf) : std::vector<int>{};
  std::vector<int> cell_well(nc, -1);
  for (int k = 0; k < nw; ++k)
    for (int i = pptr[k]; i < pptr[k + 1]; ++i) {
      PMB_REQUIRE(pcell[i] >= 0 && pcell[i] < nc, "bo: perforation cell out of range");
      PMB_REQUIRE(cell_well[pcell[i]] < 0, "bo: a cell may be perforated once, by one well");
      cell_well[pcell[i]] = k;
    }
  std::vector<int> wtype = nw ? hv(d.h_well_type, nw) : std::vector<int>{};
  for (int t : wtype) PMB_REQUIRE(t >= 0 && t <= 2, "bo: well type must be 0 (bhp), 1 (rate) or 2 (orat)");
  // cell column lists: itself, interface neighbours, cells perforated by the same well
  std::vector<std::vector<int>> cols(nc);
  std::vector<std::vector<int>> adjc(nc);
  for (int c = 0; c < nc; ++c) cols[c].push_back(c);
  for (int f = 0; f < nf; ++f) {
    const int a = N[2 * f], b = N[2 * f + 1];
    cols[a].push_back(b);
    cols[b].push_back(a);
    adjc[a].push_back(f);
    adjc[b].push_back(-f - 1);
  }
  for (int k = 0; k < nw; ++k)
    for (int i = pptr[k]; i < pptr[k + 1]; ++i)
      for (int j = pptr[k]; j < pptr[k + 1]; ++j) cols[pcell[i]].push_back(pcell[j]);
  std::vector<int> deg(nc), diag_rank(nc), adj_ptr(nc + 1, 0), adj, adj_rank;
  for (int c = 0; c < nc; ++c) {
    auto& cl = cols[c];
    std::sort(cl.begin(), cl.end());
    cl.erase(std::unique(cl.begin(), cl.end()), cl.end());
    deg[c] = (int)cl.size();
    diag_rank[c] = (int)(std::lower_bound(cl.begin(), cl.end(), c) - cl.begin());
    auto& al = adjc[c];
    std::sort(al.begin(), al.end(), [](int x, int y) {
      const int fx = x >= 0 ? x : -x - 1, fy = y >= 0 ? y : -y - 1;
      return fx < fy;
    });
    for (int code : al) {
      const int f = code >= 0 ? code : -code - 1;
      const int nb = code >= 0 ? N[2 * f + 1] : N[2 * f];
      adj.push_back(code);
      adj_rank.push_back((int)(std::lower_bound(cl.begin(), cl.end(), nb) - cl.begin()));
    }
    adj_ptr[c + 1] = (int)adj.size();
  }
  // well-local maps
  std::vector<int> pair_off(nw), pair_rank, perf_srank(nperf);
  for (int k = 0; k < nw; ++k) {
    pair_off[k] = (int)pair_rank.size();
    std::vector<int> sc(pcell.begin() + pptr[k], pcell.begin() + pptr[k + 1]);
    std::sort(sc.begin(), sc.end());
    for (int i = pptr[k]; i < pptr[k + 1]; ++i) {
      perf_srank[i] = (int)(std::lower_bound(sc.begin(), sc.end(), pcell[i]) - sc.begin());
      const auto& cl = cols[pcell[i]];
      for (int j = pptr[k]; j < pptr[k + 1]; ++j)
        pair_rank.push_back((int)(std::lower_bound(cl.begin(), cl.end(), pcell[j]) - cl.begin()));
    }
  }
  // CSR pattern in the variable-blocked order
  const int64_t n = 3LL * nc + 4LL * nw;
  h_row_ptr_.assign(n + 1, 0);
  h_col_.clear();
  for (int e = 0; e < 3; ++e)
    for (int c = 0; c < nc; ++c) {
      for (int q = 0; q < 3; ++q)
        for (int cc : cols[c]) h_col_.push_back(q * nc + cc);
      if (cell_well[c] >= 0)
        for (int m = 0; m < 4; ++m) h_col_.push_back(3 * nc + m * nw + cell_well[c]);
      h_row_ptr_[(int64_t)e * nc + c + 1] = (int)h_col_.size();
    }
  for (int e = 0; e < 4; ++e)
    for (int k = 0; k < nw; ++k) {
      if (e < 3) {
        std::vector<int> sc(pcell.begin() + pptr[k], pcell.begin() + pptr[k + 1]);
        std::sort(sc.begin(), sc.end());
        for (int q = 0; q < 3; ++q)
          for (int cc : sc) h_col_.push_back(q * nc + cc);
      }
      for (int m = 0; m < 4; ++m) h_col_.push_back(3 * nc + m * nw + k);
      h_row_ptr_[3LL * nc + (int64_t)e * nw + k + 1] = (int)h_col_.size();
    }
  PMB_REQUIRE(h_col_.size() < (size_t)INT32_MAX, "bo: Jacobian too large for 32-bit indices");

  N_.upload(N, s);
  T_.upload(d.h_T, nf, s);
  gdz_.upload(d.h_gdz, nf, s);
  pv_.upload(d.h_pv, nc, s);
  adj_ptr_.upload(adj_ptr, s);
  adj_.upload(adj, s);
  adj_rank_.upload(adj_rank, s);
  deg_.upload(deg, s);
  diag_rank_.upload(diag_rank, s);
  cell_well_.upload(cell_well, s);
  row_ptr_.upload(h_row_ptr_, s);
  perf_ptr_.upload(pptr, s);
  perf_cell_.upload(pcell, s);
  if (nperf) perf_WI_.upload(d.h_perf_WI, nperf, s);
  pair_off_.upload(pair_off, s);
  pair_rank_.upload(pair_rank, s);
  perf_srank_.upload(perf_srank, s);
  well_type_.upload(wtype, s);
  if (nw) {
    well_val_.upload(d.h_well_val, nw, s);
    compi_.upload(d.h_compi, 3LL * nw, s);
  }
  double pv_tot = 0.0;
  for (int c = 0; c < nc; ++c) pv_tot += d.h_pv[c];
  double q_ref = 0.0;
  for (int k = 0; k < nw; ++k) q_ref = std::max(q_ref, std::fabs(d.h_well_val[k]));
  v_.nc = nc;
  v_.nf = nf;
  v_.nw = nw;
  v_.nperf = nperf;
  v_.N = N_.get();
  v_.T = T_.get();
  v_.gdz = gdz_.get();
  v_.pv_ref = pv_.get();
  v_.adj_ptr = adj_ptr_.get();
  v_.adj = adj_.get();
  v_.adj_rank = adj_rank_.get();
  v_.deg = deg_.get();
  v_.diag_rank = diag_rank_.get();
  v_.cell_well = cell_well_.get();
  v_.row_ptr = row_ptr_.get();
  v_.perf_ptr = perf_ptr_.get();
  v_.perf_cell = perf_cell_.get();
  v_.perf_WI = perf_WI_.get();
  v_.pair_off = pair_off_.get();
  v_.pair_rank = pair_rank_.get();
  v_.perf_srank = perf_srank_.get();
  v_.well_type = well_type_.get();
  v_.well_val = well_val_.get();
  v_.compi = compi_.get();
  v_.q_ref = q_ref;
  v_.tol_cnv = d.tol_cnv;
  v_.tol_mb = d.tol_mb;
  v_.tol_well = d.tol_well;
  v_.ds_max = d.ds_max;
  v_.pv_tot = pv_tot;
  {
    // opt-in: per-cell true-IMPES weights (measured slower on the lattice
    // case: 86 Newton / 7153 Krylov iterations against 61 / 5234)
    const char* e = std::getenv("PMB_BO_CELL_WEIGHTS");
    cell_weights_ = e && e[0] == '1';
  }
  props_.resize((size_t)bo::kNumProps * nc);
  part_.resize((size_t)bo::kConvBlocks * (bo::kConvSums + bo::kConvMax));
  conv_out_.resize(bo::kConvOut);
  h_conv_.resize(bo::kConvOut);
  PMB_CUDA(cudaStreamSynchronize(s));
}

void BOModel::assemble(const double* x, const double* x0, double dt, double* res, double* vals) {
  PMB_REQUIRE(dt > 0.0, "bo: dt must be positive");
  const int nc = v_.nc;
  bo::bo_props_kernel<<<(nc + 127) / 128, 128, 0, s_>>>(v_, x, props_.get());
  PMB_CHECK_LAUNCH();
  bo::bo_cell_kernel<<<(nc + 127) / 128, 128, 0, s_>>>(v_, x, x0, dt, props_.get(), res, vals);
  PMB_CHECK_LAUNCH();
  if (v_.nw) {
    bo::bo_well_kernel<<<(v_.nw + 31) / 32, 32, 0, s_>>>(v_, x, props_.get(), res, vals);
    PMB_CHECK_LAUNCH();
  }
}

void BOModel::convergence(const double* res, const double* x, double dt, double* h_out) {
  const int nb = std::max(1, std::min(bo::kConvBlocks, (v_.nc + bo::kConvThreads - 1) / bo::kConvThreads));
  bo::bo_conv_partial_kernel<<<nb, bo::kConvThreads, 0, s_>>>(v_, res, x, part_.get());
  PMB_CHECK_LAUNCH();
  bo::bo_conv_final_kernel<<<1, 32, 0, s_>>>(v_, nb, part_.get(), res, dt, conv_out_.get());
  PMB_CHECK_LAUNCH();
  PMB_CUDA(cudaMemcpyAsync(h_conv_.get(), conv_out_.get(), bo::kConvOut * sizeof(double), cudaMemcpyDeviceToHost, s_));
  PMB_CUDA(cudaStreamSynchronize(s_));
  for (int i = 0; i < bo::kConvOut; ++i) h_out[i] = h_conv_[i];
}

void BOModel::update(double* x, const double* dx) {
  const int n = std::max(v_.nc, v_.nw);
  bo::bo_update_kernel<<<(n + 127) / 128, 128, 0, s_>>>(v_, x, dx);
  PMB_CHECK_LAUNCH();
}

void BOModel::step(double* x, double dt, int maxit, const pmb_cpr_opts& o, double* stats) {
  PMB_REQUIRE(maxit >= 1, "bo: max_iterations must be >= 1");
  const int64_t n = this->n(), nnz = this->nnz();
  if (res_.size() != (size_t)n) {
    res_.resize(n);
    rhs_.resize(n);
    dx_.resize(n);
    vals_.resize(nnz);
    x0_.resize(state_size());
  }
  if (!cpr_ || std::memcmp(&o, &cpr_opts_, sizeof(o)) != 0) {
    if (cpr_) pmb_csr_cpr_destroy(cpr_);
    cpr_ = nullptr;
    int rc = pmb_csr_cpr_create((int32_t)n, v_.nc, 3, h_row_ptr_.data(), h_col_.data(), 0, &o, s_, &cpr_);
    if (rc != PMB_OK) throw Error(rc, std::string("bo: CPR setup failed: ") + pmb_last_error());
    rc = pmb_csr_cpr_set_cell_weights(cpr_, cell_weights_ ? 1 : 0);
    if (rc != PMB_OK) throw Error(rc, std::string("bo: CPR setup failed: ") + pmb_last_error());
    cpr_opts_ = o;
  }
  PMB_CUDA(cudaMemcpyAsync(x0_.get(), x, state_size() * sizeof(double), cudaMemcpyDeviceToDevice, s_));
  double out[bo::kConvOut];
  double lin_its = 0.0, lin_fail = 0.0;
  for (int it = 0; it < maxit; ++it) {
    assemble(x, x0_.get(), dt, res_.get(), vals_.get());
    convergence(res_.get(), x, dt, out);
    if (out[8] != 0.0) {
      stats[0] = it;
      stats[1] = 1.0;
      stats[2] = lin_its;
      stats[3] = lin_fail;
      return;
    }
    if (!(std::isfinite(out[0]) && std::isfinite(out[1]) && std::isfinite(out[2]))) break;
    bo::bo_negate_kernel<<<std::max<int64_t>(1, std::min<int64_t>(4 * kNumSM, (n + 255) / 256)), 256, 0, s_>>>(
        n, res_.get(), rhs_.get());
    PMB_CHECK_LAUNCH();
    const double w[3] = {out[9], out[10], out[11]};
    int rc = pmb_csr_cpr_setup(cpr_, vals_.get(), w);
    if (rc != PMB_OK) throw Error(rc, std::string("bo: CPR setup failed: ") + pmb_last_error());
    double info[4];
    rc = pmb_csr_cpr_solve(cpr_, rhs_.get(), dx_.get(), info);
    if (rc != PMB_OK && rc != PMB_ERR_NOCONV) throw Error(rc, std::string("bo: linear solve failed: ") + pmb_last_error());
    lin_its += info[0];
    if (rc != PMB_OK || info[2] == 0.0) {
      // the update of a solve that stopped above its tolerance is still used
      // (the Newton test decides); a non-finite one ends the step
      lin_fail += 1.0;
      if (!std::isfinite(info[1])) break;
    }
    update(x, dx_.get());
  }
  assemble(x, x0_.get(), dt, res_.get(), vals_.get());
  convergence(res_.get(), x, dt, out);
  stats[0] = maxit;
  stats[1] = out[8];
  stats[2] = lin_its;
  stats[3] = lin_fail;
}

void BOModel::pvt_points(int n, const double* p, const double* rs, const double* sat, double* out) {
  if (n <= 0) return;
  bo::bo_pvt_points_kernel<<<(n + 127) / 128, 128, 0, s_>>>(v_, n, p, rs, sat, out);
  PMB_CHECK_LAUNCH();
}

void BOModel::relperm_points(int n, const double* sw, const double* sg, double* out) {
  if (n <= 0) return;
  bo::bo_relperm_points_kernel<<<(n + 127) / 128, 128, 0, s_>>>(v_, n, sw, sg, out);
  PMB_CHECK_LAUNCH();
}

}  // namespace pmb

struct pmb_bo {
  std::unique_ptr<pmb::BOModel> m;
};

extern "C" {

int pmb_bo_create(const pmb_bo_desc* desc, void* stream, pmb_bo** out) {
  return pmb::guarded([&] {
    PMB_REQUIRE(desc && out, "bo: desc and out must not be NULL");
    auto h = std::make_unique<pmb_bo>();
    h->m = std::make_unique<pmb::BOModel>(*desc, (cudaStream_t)stream);
    *out = h.release();
  });
}

int pmb_bo_destroy(pmb_bo* h) {
  return pmb::guarded([&] { delete h; });
}

int pmb_bo_sizes(const pmb_bo* h, int64_t* h_out3) {
  return pmb::guarded([&] {
    PMB_REQUIRE(h && h_out3, "bo: NULL argument");
    h_out3[0] = h->m->n();
    h_out3[1] = h->m->nnz();
    h_out3[2] = h->m->state_size();
  });
}

int pmb_bo_pattern(const pmb_bo* h, int32_t* h_row_ptr, int32_t* h_col) {
  return pmb::guarded([&] {
    PMB_REQUIRE(h && h_row_ptr && h_col, "bo: NULL argument");
    std::copy(h->m->row_ptr().begin(), h->m->row_ptr().end(), h_row_ptr);
    std::copy(h->m->col().begin(), h->m->col().end(), h_col);
  });
}

int pmb_bo_assemble(pmb_bo* h, const double* d_state, const double* d_state0, double dt, double* d_res,
                    double* d_vals) {
  return pmb::guarded([&] {
    PMB_REQUIRE(h && d_state && d_state0 && d_res && d_vals, "bo: NULL argument");
    h->m->assemble(d_state, d_state0, dt, d_res, d_vals);
  });
}

int pmb_bo_convergence(pmb_bo* h, const double* d_res, const double* d_state, double dt, double* h_out14) {
  return pmb::guarded([&] {
    PMB_REQUIRE(h && d_res && d_state && h_out14, "bo: NULL argument");
    h->m->convergence(d_res, d_state, dt, h_out14);
  });
}

int pmb_bo_update(pmb_bo* h, double* d_state, const double* d_dx) {
  return pmb::guarded([&] {
    PMB_REQUIRE(h && d_state && d_dx, "bo: NULL argument");
    h->m->update(d_state, d_dx);
  });
}

int pmb_bo_step(pmb_bo* h, double* d_state, double dt, int32_t max_iterations, const pmb_cpr_opts* opts,
                double* h_stats4) {
  return pmb::guarded([&] {
    PMB_REQUIRE(h && d_state && opts && h_stats4, "bo: NULL argument");
    PMB_REQUIRE(dt > 0.0, "bo: dt must be positive");
    h->m->step(d_state, dt, max_iterations, *opts, h_stats4);
  });
}

int pmb_bo_pvt_points(pmb_bo* h, int32_t n, const double* d_p, const double* d_rs, const double* d_sat,
                      double* d_out7) {
  return pmb::guarded([&] {
    PMB_REQUIRE(h && (n == 0 || (d_p && d_rs && d_sat && d_out7)), "bo: NULL argument");
    h->m->pvt_points(n, d_p, d_rs, d_sat, d_out7);
  });
}

int pmb_bo_relperm_points(pmb_bo* h, int32_t n, const double* d_sw, const double* d_sg, double* d_out5) {
  return pmb::guarded([&] {
    PMB_REQUIRE(h && (n == 0 || (d_sw && d_sg && d_out5)), "bo: NULL argument");
    h->m->relperm_points(n, d_sw, d_sg, d_out5);
  });
}

}  // extern "C"
