// Incompressible two-point pressure system on the device: the assembly of
// incomp_tpfa (pymrst/modules/incomp/incomp_tpfa.py:55-164: mobility-weighted
// one-sided and face transmissibilities, gravity / boundary / source
// right-hand side, well rows, the pressure pin), its solve (:172-184, SuperLU
// there, AMG-preconditioned CG here) and the reconstruction of face
// pressures, face fluxes and well fluxes (:186-211).
//
// Layout.  The system has n = nc + nw unknowns: cell pressures, then one bhp
// per well.  Its CSR pattern is built once per grid and well set: row c holds
// the diagonal, the other cell of each interface of c, and the bhp column of
// every rate well that perforates c; row nc + k holds the perforated cells of
// a rate well and the diagonal (a bhp well's row is its diagonal only).
// Every half-face knows the CSR slot of its off-diagonal entry and every
// perforation the slots of its two well-coupling entries, so each kernel
// writes whole rows from one thread (cells) or one warp (wells): no atomics,
// a fixed summation order, bit-identical results from run to run.
#include <algorithm>
#include <cmath>
#include <memory>

#include "pmb_common.cuh"

namespace pmb {

struct ScalarPCGHandle;  // pcg.cu
ScalarPCGHandle* make_scalar_pcg(int n, const int* h_rp, const int* h_ci, cudaStream_t s, double theta,
                                 int coarse);
void destroy_scalar_pcg(ScalarPCGHandle* p);
void scalar_pcg_setup(ScalarPCGHandle* p, const double* d_vals);
bool scalar_pcg_solve(ScalarPCGHandle* p, const double* b, double* x, double rtol, int maxiter, double* info);

constexpr int kMaxPhases = 4;

struct TpfaPhases {
  double rho[kMaxPhases];
};

struct TpfaDev {
  int nc, nf, nhf, nw, nperf, n, dim, use_trans;
  const int* face_pos;    // nc+1
  const int* hf_cell;     // nhf
  const int* hf_face;     // nhf
  const int* hf_slot;     // nhf: CSR slot of (cell, other cell) for interior interfaces, else -1
  const int* nbr;         // nf x 2
  const int* face_hf;     // nf x 2: the half-face on side 0 / side 1, -1 if none
  const double* cc;       // nc x dim cell centroids
  const double* fc;       // nf x dim face centroids
  const int* row_ptr;     // n+1
  const int* diag;        // n: CSR slot of the diagonal
  const int* perf_cell;   // nperf
  const int* perf_ptr;    // nw+1
  const int* cperf_ptr;   // nc+1: perforations of each cell, ascending
  const int* cperf_idx;
  const int* perf_cslot;  // nperf: slot (cell, nc+k) of a rate well, -1 for bhp
  const int* perf_wslot;  // nperf: slot (nc+k, cell) of a rate well, -1 for bhp
  const int* well_rate;   // nw: 1 rate, 0 bhp
};

struct TpfaWork {
  double* totmob;   // nc
  double* omega;    // nc
  double* th;       // nhf: mobility-weighted one-sided T
  double* grav;     // nhf: gravity potential of the half-face, omega (x_f - x_c).g
  double* ft;       // nf: mobility-weighted face T
  double* fg;       // nf: signed gravity sum over the interior or Dirichlet half-faces
  int* bc_type;     // nf: 0 none, 1 pressure, 2 flux
  double* bc_val;   // nf
  double* src;      // nc
  double* perf_wi;  // nperf: WI * total mobility
  double* perf_dp;  // nperf: hydrostatic drop to the perforation
  double* well_val; // nw
};

// total mobility and its density weighting per cell (_dynamic_quantities,
// incomp_tpfa.py:214-220)
__global__ void tpfa_cell_kernel(int nc, int nph, const double* __restrict__ mob, TpfaPhases ph,
                                 double* __restrict__ totmob, double* __restrict__ omega) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  double t = 0.0, w = 0.0;
  for (int i = 0; i < nph; ++i) {
    const double m = mob[(long long)c * nph + i];
    t += m;
    w += m * ph.rho[i];
  }
  totmob[c] = t;
  omega[c] = w / t;
}

// one-sided T times the cell's total mobility, and the half-face gravity
// potential omega (x_f - x_c).g (compute_pressure_rhs.py's gp)
__global__ void tpfa_halfface_kernel(TpfaDev d, const double* __restrict__ T, double g0, double g1, double g2,
                                     int grav_on, TpfaWork w) {
  const int h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= d.nhf) return;
  const int c = d.hf_cell[h], f = d.hf_face[h];
  if (!d.use_trans) w.th[h] = T[h] * w.totmob[c];
  double gp = 0.0;
  if (grav_on) {
    const double g[3] = {g0, g1, g2};
    double s = 0.0;
    for (int k = 0; k < d.dim; ++k) s += (d.fc[(long long)f * d.dim + k] - d.cc[(long long)c * d.dim + k]) * g[k];
    gp = w.omega[c] * s;
  }
  w.grav[h] = gp;
}

__device__ __forceinline__ double hf_sign(const TpfaDev& d, int h) {
  return d.nbr[2 * d.hf_face[h]] == d.hf_cell[h] ? 1.0 : -1.0;
}

// face T: harmonic sum of the one-sided T (or, with use_trans, the interface
// T times the mean total mobility of its cells, _compute_trans :223-243), and
// the signed gravity sum fg over the half-faces of interior and Dirichlet faces
__global__ void tpfa_face_kernel(TpfaDev d, const double* __restrict__ T, TpfaWork w) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= d.nf) return;
  const int h0 = d.face_hf[2 * f], h1 = d.face_hf[2 * f + 1];
  double ft;
  if (d.use_trans) {
    const int cnt = (d.nbr[2 * f] >= 0) + (d.nbr[2 * f + 1] >= 0);
    double m = 0.0;
    if (h0 >= 0) m += w.totmob[d.hf_cell[h0]];
    if (h1 >= 0) m += w.totmob[d.hf_cell[h1]];
    ft = T[f] * (m / cnt);
    if (h0 >= 0) w.th[h0] = ft * cnt;
    if (h1 >= 0) w.th[h1] = ft * cnt;
  } else {
    double inv = 0.0;
    if (h0 >= 0) inv += 1.0 / w.th[h0];
    if (h1 >= 0) inv += 1.0 / w.th[h1];
    ft = 1.0 / inv;
  }
  w.ft[f] = ft;
  const bool interior = d.nbr[2 * f] >= 0 && d.nbr[2 * f + 1] >= 0;
  double fg = 0.0;
  if (interior || w.bc_type[f] == 1) {
    if (h0 >= 0) fg += w.grav[h0] * hf_sign(d, h0);
    if (h1 >= 0) fg += w.grav[h1] * hf_sign(d, h1);
  }
  w.fg[f] = fg;
}

// Perforations and well rows, one warp per well (incomp_tpfa.py:126-148 with
// compute_incomp_well_pressure_drop): connection factors WI * totmob, the
// mixture density (an injector's from its composition, a producer's the
// WI-weighted mean of the fractional-flow-weighted densities of its cells),
// the hydrostatic drops, then the well row: a bhp well has the diagonal
// max(wi) and right-hand side max(wi) * target; a rate well couples to its
// cells with -wi, has the diagonal sum(wi) and right-hand side target -
// sum(wi * dp).
__global__ void tpfa_well_kernel(TpfaDev d, TpfaWork w, const double* __restrict__ mob, int nph,
                                 const double* __restrict__ WI, const double* __restrict__ dZ,
                                 const double* __restrict__ compi, int ncompi, const int* __restrict__ injector,
                                 TpfaPhases ph, double norm_g, double* __restrict__ vals,
                                 double* __restrict__ rhs) {
  const int k = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (k >= d.nw) return;
  const int p0 = d.perf_ptr[k], p1 = d.perf_ptr[k + 1];
  double rho_mix;
  if (injector[k]) {
    rho_mix = 0.0;
    const int m = min(nph, ncompi);
    for (int i = 0; i < m; ++i) rho_mix += ph.rho[i] * compi[k * ncompi + i];
  } else {
    double num = 0.0, den = 0.0;
    for (int p = p0 + lane; p < p1; p += 32) {
      const int c = d.perf_cell[p];
      double tm = 0.0, fr = 0.0;
      for (int i = 0; i < nph; ++i) tm += mob[(long long)c * nph + i];
      for (int i = 0; i < nph; ++i) fr += (mob[(long long)c * nph + i] / tm) * ph.rho[i];
      num += WI[p] * fr;
      den += WI[p];
    }
    rho_mix = warp_sum(num) / warp_sum(den);
  }
  double wmax = -INFINITY, wsum = 0.0, wdp = 0.0;
  for (int p = p0 + lane; p < p1; p += 32) {
    const double wi = WI[p] * w.totmob[d.perf_cell[p]];
    const double dp = norm_g * (dZ[p] * rho_mix);
    w.perf_wi[p] = wi;
    w.perf_dp[p] = dp;
    wmax = fmax(wmax, wi);
    wsum += wi;
    wdp += wi * dp;
  }
  wmax = warp_max(wmax);
  wsum = warp_sum(wsum);
  wdp = warp_sum(wdp);
  __syncwarp();
  if (lane != 0) return;
  const int row = d.nc + k;
  for (int s = d.row_ptr[row]; s < d.row_ptr[row + 1]; ++s) vals[s] = 0.0;
  if (d.well_rate[k]) {
    for (int p = p0; p < p1; ++p) vals[d.perf_wslot[p]] -= w.perf_wi[p];
    vals[d.diag[row]] = wsum;
    rhs[row] = w.well_val[k] - wdp;
  } else {
    vals[d.diag[row]] = wmax;
    rhs[row] = wmax * w.well_val[k];
  }
}

// Cell rows, one thread per cell (gather over the cell's half-faces and
// perforations): off-diagonals -ft, diagonal sum(ft) over interior
// interfaces + one-sided T of Dirichlet faces + well connection factors,
// right-hand side -ft (sgn fg + ff) + source - hh + well terms.
__global__ void tpfa_row_kernel(TpfaDev d, TpfaWork w, double* __restrict__ vals, double* __restrict__ rhs) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.nc) return;
  for (int s = d.row_ptr[c]; s < d.row_ptr[c + 1]; ++s) vals[s] = 0.0;
  double r_face = 0.0, r_flux = 0.0, d_int = 0.0, d_dir = 0.0;
  for (int h = d.face_pos[c]; h < d.face_pos[c + 1]; ++h) {
    const int f = d.hf_face[h];
    const double t = w.ft[f];
    const int bt = w.bc_type[f];
    const double ff = bt == 1 ? -w.bc_val[f] : 0.0;
    const double hh = bt == 2 ? -w.bc_val[f] : 0.0;
    r_face += -t * (hf_sign(d, h) * w.fg[f] + ff);
    r_flux += -hh;
    const int slot = d.hf_slot[h];
    if (slot >= 0) {
      vals[slot] -= t;
      d_int += t;
    }
    if (bt == 1) d_dir += w.th[h];
  }
  double r = (r_face + w.src[c]) + r_flux;
  double d_well = 0.0;
  for (int q = d.cperf_ptr[c]; q < d.cperf_ptr[c + 1]; ++q) {
    const int p = d.cperf_idx[q];
    const double wi = w.perf_wi[p];
    d_well += wi;
    const int cs = d.perf_cslot[p];
    if (cs >= 0) {
      vals[cs] -= wi;
      r += wi * w.perf_dp[p];
    } else {
      // the well of a bhp perforation: its index from perf_ptr (binary search)
      int lo = 0, hi = d.nw;
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (d.perf_ptr[mid] <= p) lo = mid; else hi = mid;
      }
      r += wi * (w.well_val[lo] + w.perf_dp[p]);
    }
  }
  vals[d.diag[c]] = (d_well + d_dir) + d_int;
  rhs[c] = r;
}

// The pin of a pressure level when nothing fixes it (no Dirichlet face, no
// bhp well): the first diagonal entry is doubled, or, when it is not
// positive, the first largest diagonal entry (incomp_tpfa.py:156-161).
__global__ void __launch_bounds__(1024) tpfa_pin_kernel(int n, const int* __restrict__ diag, double* __restrict__ vals) {
  __shared__ double sv[32];
  __shared__ int si[32];
  if (vals[diag[0]] > 0.0) {
    if (threadIdx.x == 0) vals[diag[0]] *= 2.0;
    return;
  }
  double best = -INFINITY;
  int bi = n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double v = vals[diag[i]];
    if (v > best) { best = v; bi = i; }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double ov = __shfl_xor_sync(0xffffffffu, best, o);
    const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
    if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) { sv[wid] = best; si[wid] = bi; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < (int)(blockDim.x >> 5); ++k)
      if (sv[k] > sv[0] || (sv[k] == sv[0] && si[k] < si[0])) { sv[0] = sv[k]; si[0] = si[k]; }
    if (si[0] < n) vals[diag[si[0]]] *= 2.0;
  }
}

// face pressures and face fluxes from the solved pressures (:186-201)
__global__ void tpfa_face_recon_kernel(TpfaDev d, TpfaWork w, const double* __restrict__ p,
                                       double* __restrict__ flux, double* __restrict__ fpress) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= d.nf) return;
  const int h0 = d.face_hf[2 * f], h1 = d.face_hf[2 * f + 1];
  double num = 0.0, den = 0.0, gsum = 0.0;
  if (h0 >= 0) { num += (p[d.hf_cell[h0]] + w.grav[h0]) * w.th[h0]; den += w.th[h0]; gsum += w.grav[h0]; }
  if (h1 >= 0) { num += (p[d.hf_cell[h1]] + w.grav[h1]) * w.th[h1]; den += w.th[h1]; gsum += w.grav[h1]; }
  double fp = num / den;
  const int n0 = d.nbr[2 * f], n1 = d.nbr[2 * f + 1];
  const double ft = w.ft[f];
  const int bt = w.bc_type[f];
  const bool interior = n0 >= 0 && n1 >= 0;
  if (!interior) {
    const double hh = bt == 2 ? -w.bc_val[f] : 0.0;
    fp = fp - hh / ft;
  }
  if (bt == 1) fp = w.bc_val[f];
  fpress[f] = fp;
  double q;
  if (interior) {
    q = -(ft * (p[n1] - p[n0] - w.fg[f]));
  } else {
    const int c = max(n0, n1);
    const double sgn_b = n1 < 0 ? 1.0 : -1.0;
    q = -sgn_b * ft * (fp - p[c] - gsum);
  }
  flux[f] = q;
}

// well connection fluxes WI totmob (bhp + dp - p_cell) (:205-209)
__global__ void tpfa_perf_recon_kernel(TpfaDev d, TpfaWork w, const double* __restrict__ p,
                                       double* __restrict__ perf_flux, double* __restrict__ perf_dp) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= d.nperf) return;
  int lo = 0, hi = d.nw;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (d.perf_ptr[mid] <= q) lo = mid; else hi = mid;
  }
  perf_flux[q] = w.perf_wi[q] * (p[d.nc + lo] + w.perf_dp[q] - p[d.perf_cell[q]]);
  if (perf_dp) perf_dp[q] = w.perf_dp[q];
}

class Tpfa {
 public:
  Tpfa(const pmb_tpfa_desc& desc, cudaStream_t s) : s_(s) {
    nc_ = desc.nc; nf_ = desc.nf; nhf_ = desc.nhf; nw_ = desc.nw; dim_ = desc.dim; use_trans_ = desc.use_trans;
    PMB_REQUIRE(nc_ > 0 && nf_ >= 0 && nhf_ >= 0 && nw_ >= 0, "bad sizes");
    PMB_REQUIRE(dim_ >= 1 && dim_ <= 3, "dim must be 1, 2 or 3");
    PMB_REQUIRE(desc.h_face_pos && desc.h_cell_faces && desc.h_neighbors && desc.h_cell_centroids &&
                    desc.h_face_centroids, "NULL grid array");
    PMB_REQUIRE(nw_ == 0 || (desc.h_perf_ptr && desc.h_perf_cell && desc.h_well_rate), "NULL well array");
    n_ = nc_ + nw_;
    const int* fp = desc.h_face_pos;
    PMB_REQUIRE(fp[0] == 0 && fp[nc_] == nhf_, "face_pos must run from 0 to nhf");
    std::vector<int> hf_cell(nhf_), face_hf(2 * (size_t)nf_, -1);
    std::vector<int> nbr(desc.h_neighbors, desc.h_neighbors + 2 * (size_t)nf_);
    for (int f = 0; f < nf_; ++f) {
      PMB_REQUIRE(nbr[2 * f] >= -1 && nbr[2 * f] < nc_ && nbr[2 * f + 1] >= -1 && nbr[2 * f + 1] < nc_,
                  "neighbour index out of range");
      PMB_REQUIRE(nbr[2 * f] != nbr[2 * f + 1], "a face must join two different cells (periodic faces are not supported)");
    }
    for (int c = 0; c < nc_; ++c) {
      PMB_REQUIRE(fp[c] <= fp[c + 1], "face_pos must be non-decreasing");
      for (int h = fp[c]; h < fp[c + 1]; ++h) {
        const int f = desc.h_cell_faces[h];
        PMB_REQUIRE(f >= 0 && f < nf_, "cell face index out of range");
        hf_cell[h] = c;
        const int side = nbr[2 * f] == c ? 0 : (nbr[2 * f + 1] == c ? 1 : -1);
        PMB_REQUIRE(side >= 0, "a cell lists a face that does not neighbour it");
        PMB_REQUIRE(face_hf[2 * f + side] < 0, "a face is listed twice for the same cell");
        face_hf[2 * f + side] = h;
      }
    }
    // wells
    std::vector<int> perf_ptr(nw_ + 1, 0), perf_cell, well_rate(nw_);
    if (nw_) {
      perf_ptr.assign(desc.h_perf_ptr, desc.h_perf_ptr + nw_ + 1);
      PMB_REQUIRE(perf_ptr[0] == 0, "perf_ptr must start at 0");
      for (int k = 0; k < nw_; ++k) {
        PMB_REQUIRE(perf_ptr[k] <= perf_ptr[k + 1], "perf_ptr must be non-decreasing");
        well_rate[k] = desc.h_well_rate[k] ? 1 : 0;
      }
      perf_cell.assign(desc.h_perf_cell, desc.h_perf_cell + perf_ptr[nw_]);
      for (int c : perf_cell) PMB_REQUIRE(c >= 0 && c < nc_, "perforated cell out of range");
    }
    nperf_ = perf_ptr[nw_];
    std::vector<int> perf_well(nperf_);
    for (int k = 0; k < nw_; ++k)
      for (int p = perf_ptr[k]; p < perf_ptr[k + 1]; ++p) perf_well[p] = k;
    // CSR pattern
    std::vector<std::vector<int>> cols(n_);
    for (int c = 0; c < nc_; ++c) {
      cols[c].push_back(c);
      for (int h = fp[c]; h < fp[c + 1]; ++h) {
        const int f = desc.h_cell_faces[h];
        if (nbr[2 * f] >= 0 && nbr[2 * f + 1] >= 0) cols[c].push_back(nbr[2 * f] == c ? nbr[2 * f + 1] : nbr[2 * f]);
      }
    }
    for (int p = 0; p < nperf_; ++p) {
      const int k = perf_well[p];
      if (!well_rate[k]) continue;
      cols[perf_cell[p]].push_back(nc_ + k);
      cols[nc_ + k].push_back(perf_cell[p]);
    }
    for (int k = 0; k < nw_; ++k) cols[nc_ + k].push_back(nc_ + k);
    h_rp_.assign(n_ + 1, 0);
    for (int i = 0; i < n_; ++i) {
      auto& v = cols[i];
      std::sort(v.begin(), v.end());
      v.erase(std::unique(v.begin(), v.end()), v.end());
      h_rp_[i + 1] = h_rp_[i] + (int)v.size();
    }
    h_ci_.resize(h_rp_[n_]);
    std::vector<int> diag(n_);
    for (int i = 0; i < n_; ++i) {
      std::copy(cols[i].begin(), cols[i].end(), h_ci_.begin() + h_rp_[i]);
      diag[i] = slot(i, i);
    }
    std::vector<int> hf_slot(nhf_, -1);
    for (int c = 0; c < nc_; ++c)
      for (int h = fp[c]; h < fp[c + 1]; ++h) {
        const int f = desc.h_cell_faces[h];
        if (nbr[2 * f] >= 0 && nbr[2 * f + 1] >= 0) hf_slot[h] = slot(c, nbr[2 * f] == c ? nbr[2 * f + 1] : nbr[2 * f]);
      }
    std::vector<int> cperf_ptr(nc_ + 1, 0), cperf_idx(nperf_), perf_cslot(nperf_, -1), perf_wslot(nperf_, -1);
    for (int p = 0; p < nperf_; ++p) ++cperf_ptr[perf_cell[p] + 1];
    for (int c = 0; c < nc_; ++c) cperf_ptr[c + 1] += cperf_ptr[c];
    {
      std::vector<int> fill(cperf_ptr.begin(), cperf_ptr.end() - 1);
      for (int p = 0; p < nperf_; ++p) cperf_idx[fill[perf_cell[p]]++] = p;
    }
    for (int p = 0; p < nperf_; ++p) {
      const int k = perf_well[p];
      if (!well_rate[k]) continue;
      perf_cslot[p] = slot(perf_cell[p], nc_ + k);
      perf_wslot[p] = slot(nc_ + k, perf_cell[p]);
    }
    // upload
    face_pos_.upload(fp, nc_ + 1, s);
    hf_cell_.upload(hf_cell, s);
    hf_face_.upload(desc.h_cell_faces, nhf_, s);
    hf_slot_.upload(hf_slot, s);
    nbr_.upload(nbr, s);
    face_hf_.upload(face_hf, s);
    cc_.upload(desc.h_cell_centroids, (size_t)nc_ * dim_, s);
    fc_.upload(desc.h_face_centroids, (size_t)nf_ * dim_, s);
    rp_.upload(h_rp_, s);
    diag_.upload(diag, s);
    perf_cell_.upload(perf_cell, s);
    perf_ptr_.upload(perf_ptr, s);
    cperf_ptr_.upload(cperf_ptr, s);
    cperf_idx_.upload(cperf_idx, s);
    perf_cslot_.upload(perf_cslot, s);
    perf_wslot_.upload(perf_wslot, s);
    well_rate_.upload(well_rate, s);
    h_well_rate_ = well_rate;
    totmob_.resize(nc_); omega_.resize(nc_); th_.resize(std::max(nhf_, 1)); grav_.resize(std::max(nhf_, 1));
    ft_.resize(std::max(nf_, 1)); fg_.resize(std::max(nf_, 1));
    bc_type_.resize(std::max(nf_, 1)); bc_val_.resize(std::max(nf_, 1)); src_.resize(nc_);
    perf_wi_.resize(std::max(nperf_, 1)); perf_dp_.resize(std::max(nperf_, 1)); well_val_.resize(std::max(nw_, 1));
    h_bc_type_.assign(nf_, 0);
    h_bc_val_.assign(nf_, 0.0);
    h_src_.assign(nc_, 0.0);
    PMB_CUDA(cudaStreamSynchronize(s));
  }
  ~Tpfa() { if (pcg_) destroy_scalar_pcg(pcg_); }

  int n() const { return n_; }
  int nnz() const { return h_rp_[n_]; }
  int nperf() const { return nperf_; }
  const std::vector<int>& row_ptr() const { return h_rp_; }
  const std::vector<int>& col() const { return h_ci_; }

  void assemble(const pmb_tpfa_forces& fr, double* vals, double* rhs) {
    PMB_REQUIRE(fr.d_T && fr.d_mob && vals && rhs, "NULL argument");
    PMB_REQUIRE(fr.nph >= 1 && fr.nph <= kMaxPhases, "1 to 4 phases");
    PMB_REQUIRE(nw_ == 0 || (fr.d_perf_WI && fr.d_perf_dZ && fr.h_well_val && fr.h_injector &&
                             (fr.ncompi == 0 || fr.h_compi)), "NULL well force array");
    TpfaPhases ph{};
    for (int i = 0; i < fr.nph; ++i) ph.rho[i] = fr.h_rho[i];
    // boundary conditions and sources, scattered to per-face / per-cell arrays
    std::fill(h_bc_type_.begin(), h_bc_type_.end(), 0);
    std::fill(h_bc_val_.begin(), h_bc_val_.end(), 0.0);
    std::fill(h_src_.begin(), h_src_.end(), 0.0);
    has_dirichlet_ = false;
    for (int i = 0; i < fr.nbc; ++i) {
      const int f = fr.h_bc_face[i];
      PMB_REQUIRE(f >= 0 && f < nf_, "boundary condition refers to a face outside the grid");
      PMB_REQUIRE(h_bc_type_[f] == 0, "repeated face in the boundary conditions");
      PMB_REQUIRE(fr.h_bc_type[i] == 1 || fr.h_bc_type[i] == 2, "boundary condition type must be 1 (pressure) or 2 (flux)");
      h_bc_type_[f] = fr.h_bc_type[i];
      h_bc_val_[f] = fr.h_bc_value[i];
      has_dirichlet_ |= fr.h_bc_type[i] == 1;
    }
    for (int i = 0; i < fr.nsrc; ++i) {
      const int c = fr.h_src_cell[i];
      PMB_REQUIRE(c >= 0 && c < nc_, "source refers to a cell outside the grid");
      h_src_[c] += fr.h_src_rate[i];
    }
    bool any_bhp = false;
    for (int k = 0; k < nw_; ++k) any_bhp |= !h_well_rate_[k];
    bc_type_.upload(h_bc_type_.data(), nf_, s_);
    bc_val_.upload(h_bc_val_.data(), nf_, s_);
    src_.upload(h_src_, s_);
    if (nw_) well_val_.upload(fr.h_well_val, nw_, s_);
    if (nw_) {
      injector_.upload(fr.h_injector, nw_, s_);
      if (fr.ncompi) compi_.upload(fr.h_compi, (size_t)nw_ * fr.ncompi, s_);
    }
    const TpfaDev d = dev();
    const TpfaWork w = work();
    const double* g = fr.gravity;
    const int grav_on = (g[0] != 0.0 || g[1] != 0.0 || g[2] != 0.0) ? 1 : 0;
    tpfa_cell_kernel<<<grid_for(nc_, 256), 256, 0, s_>>>(nc_, fr.nph, fr.d_mob, ph, w.totmob, w.omega);
    PMB_CHECK_LAUNCH();
    if (nhf_) {
      tpfa_halfface_kernel<<<grid_for(nhf_, 256), 256, 0, s_>>>(d, fr.d_T, g[0], g[1], g[2], grav_on, w);
      PMB_CHECK_LAUNCH();
    }
    if (nf_) {
      tpfa_face_kernel<<<grid_for(nf_, 256), 256, 0, s_>>>(d, fr.d_T, w);
      PMB_CHECK_LAUNCH();
    }
    if (nw_) {
      tpfa_well_kernel<<<grid_for((long long)nw_ * 32, 128), 128, 0, s_>>>(
          d, w, fr.d_mob, fr.nph, fr.d_perf_WI, fr.d_perf_dZ, fr.ncompi ? compi_.get() : nullptr, fr.ncompi,
          injector_.get(), ph, fr.well_gravity, vals, rhs);
      PMB_CHECK_LAUNCH();
    }
    tpfa_row_kernel<<<grid_for(nc_, 128), 128, 0, s_>>>(d, w, vals, rhs);
    PMB_CHECK_LAUNCH();
    pinned_ = !has_dirichlet_ && !any_bhp;
    if (pinned_) {
      tpfa_pin_kernel<<<1, 1024, 0, s_>>>(n_, diag_.get(), vals);
      PMB_CHECK_LAUNCH();
    }
    assembled_ = true;
  }

  bool solve(const double* vals, const double* rhs, double* p, double rtol, int maxiter, double* info) {
    PMB_REQUIRE(vals && rhs && p && info, "NULL argument");
    PMB_REQUIRE(rhs != p, "rhs and p must not alias");
    if (!pcg_) pcg_ = make_scalar_pcg(n_, h_rp_.data(), h_ci_.data(), s_, 0.25, 200);
    scalar_pcg_setup(pcg_, vals);
    return scalar_pcg_solve(pcg_, rhs, p, rtol, maxiter, info);
  }

  void reconstruct(const double* p, double* flux, double* fpress, double* perf_flux, double* perf_dp) {
    PMB_REQUIRE(assembled_, "pmb_tpfa_reconstruct needs a preceding pmb_tpfa_assemble");
    PMB_REQUIRE(p && flux && fpress && (nperf_ == 0 || perf_flux), "NULL argument");
    const TpfaDev d = dev();
    const TpfaWork w = work();
    if (nf_) {
      tpfa_face_recon_kernel<<<grid_for(nf_, 256), 256, 0, s_>>>(d, w, p, flux, fpress);
      PMB_CHECK_LAUNCH();
    }
    if (nperf_) {
      tpfa_perf_recon_kernel<<<grid_for(nperf_, 128), 128, 0, s_>>>(d, w, p, perf_flux, perf_dp);
      PMB_CHECK_LAUNCH();
    }
  }
  bool pinned() const { return pinned_; }
  int levels(int64_t* sizes, int maxl) const;
  ScalarPCGHandle* pcg() const { return pcg_; }

 private:
  int slot(int row, int col) const {
    const auto b = h_ci_.begin() + h_rp_[row], e = h_ci_.begin() + h_rp_[row + 1];
    const auto it = std::lower_bound(b, e, col);
    if (it == e || *it != col) throw Error(PMB_ERR_INTERNAL, "CSR slot missing");
    return (int)(it - h_ci_.begin());
  }
  TpfaDev dev() const {
    TpfaDev d;
    d.nc = nc_; d.nf = nf_; d.nhf = nhf_; d.nw = nw_; d.nperf = nperf_; d.n = n_; d.dim = dim_; d.use_trans = use_trans_;
    d.face_pos = face_pos_.get(); d.hf_cell = hf_cell_.get(); d.hf_face = hf_face_.get(); d.hf_slot = hf_slot_.get();
    d.nbr = nbr_.get(); d.face_hf = face_hf_.get(); d.cc = cc_.get(); d.fc = fc_.get();
    d.row_ptr = rp_.get(); d.diag = diag_.get(); d.perf_cell = perf_cell_.get(); d.perf_ptr = perf_ptr_.get();
    d.cperf_ptr = cperf_ptr_.get(); d.cperf_idx = cperf_idx_.get(); d.perf_cslot = perf_cslot_.get();
    d.perf_wslot = perf_wslot_.get(); d.well_rate = well_rate_.get();
    return d;
  }
  TpfaWork work() const {
    TpfaWork w;
    w.totmob = totmob_.get(); w.omega = omega_.get(); w.th = th_.get(); w.grav = grav_.get(); w.ft = ft_.get();
    w.fg = fg_.get(); w.bc_type = bc_type_.get(); w.bc_val = bc_val_.get(); w.src = src_.get();
    w.perf_wi = perf_wi_.get(); w.perf_dp = perf_dp_.get(); w.well_val = well_val_.get();
    return w;
  }

  cudaStream_t s_;
  int nc_, nf_, nhf_, nw_, nperf_ = 0, n_, dim_, use_trans_;
  bool has_dirichlet_ = false, pinned_ = false, assembled_ = false;
  std::vector<int> h_rp_, h_ci_, h_well_rate_, h_bc_type_;
  std::vector<double> h_bc_val_, h_src_;
  DArray<int> face_pos_, hf_cell_, hf_face_, hf_slot_, nbr_, face_hf_, rp_, diag_, perf_cell_, perf_ptr_,
      cperf_ptr_, cperf_idx_, perf_cslot_, perf_wslot_, well_rate_, bc_type_, injector_;
  DArray<double> cc_, fc_, totmob_, omega_, th_, grav_, ft_, fg_, bc_val_, src_, perf_wi_, perf_dp_, well_val_,
      compi_;
  ScalarPCGHandle* pcg_ = nullptr;
};

int scalar_pcg_levels(const ScalarPCGHandle* p, int64_t* sizes, int maxl);

int Tpfa::levels(int64_t* sizes, int maxl) const { return pcg_ ? scalar_pcg_levels(pcg_, sizes, maxl) : 0; }

}  // namespace pmb

using namespace pmb;

struct pmb_tpfa {
  std::unique_ptr<Tpfa> t;
};

extern "C" {

int pmb_tpfa_create(const pmb_tpfa_desc* desc, void* stream, pmb_tpfa** out) {
  return guarded([&] {
    PMB_REQUIRE(desc && out, "NULL argument");
    *out = nullptr;
    auto h = std::make_unique<pmb_tpfa>();
    h->t = std::make_unique<Tpfa>(*desc, (cudaStream_t)stream);
    *out = h.release();
  });
}

int pmb_tpfa_destroy(pmb_tpfa* h) {
  return guarded([&] { delete h; });
}

int pmb_tpfa_sizes(const pmb_tpfa* h, int64_t* h_out4) {
  return guarded([&] {
    PMB_REQUIRE(h && h_out4, "NULL argument");
    h_out4[0] = h->t->n();
    h_out4[1] = h->t->nnz();
    h_out4[2] = h->t->nperf();
    h_out4[3] = h->t->pinned() ? 1 : 0;
  });
}

int pmb_tpfa_pattern(const pmb_tpfa* h, int32_t* h_row_ptr, int32_t* h_col) {
  return guarded([&] {
    PMB_REQUIRE(h && h_row_ptr && h_col, "NULL argument");
    std::copy(h->t->row_ptr().begin(), h->t->row_ptr().end(), h_row_ptr);
    std::copy(h->t->col().begin(), h->t->col().end(), h_col);
  });
}

int pmb_tpfa_assemble(pmb_tpfa* h, const pmb_tpfa_forces* forces, double* d_vals, double* d_rhs) {
  return guarded([&] {
    PMB_REQUIRE(h && forces, "NULL argument");
    h->t->assemble(*forces, d_vals, d_rhs);
  });
}

int pmb_tpfa_solve(pmb_tpfa* h, const double* d_vals, const double* d_rhs, double* d_p, double rtol,
                   int32_t maxiter, double* h_info3) {
  return guarded([&] {
    PMB_REQUIRE(h, "NULL argument");
    if (!h->t->solve(d_vals, d_rhs, d_p, rtol, maxiter, h_info3))
      throw Error(PMB_ERR_NOCONV, "pressure PCG did not reach its tolerance (relres " +
                                      std::to_string(h_info3[1]) + ")");
  });
}

int pmb_tpfa_reconstruct(pmb_tpfa* h, const double* d_p, double* d_flux, double* d_face_pressure,
                         double* d_perf_flux, double* d_perf_dp) {
  return guarded([&] {
    PMB_REQUIRE(h, "NULL argument");
    h->t->reconstruct(d_p, d_flux, d_face_pressure, d_perf_flux, d_perf_dp);
  });
}

int pmb_tpfa_levels(const pmb_tpfa* h, int32_t max_levels, int64_t* h_sizes, int32_t* n_levels) {
  return guarded([&] {
    PMB_REQUIRE(h && h_sizes && n_levels, "NULL argument");
    *n_levels = h->t->levels(h_sizes, max_levels);
  });
}

}  // extern "C"
