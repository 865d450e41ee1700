// Oil-water fully-implicit residual and Jacobian on sm_100a.
//
// Restates, for the device, TwoPhaseOilWaterModelAD.assemble and its well
// model (pymrst/modules/ad_blackoil/models/two_phase_oil_water_model.py:
// 205-546), _converged (:549-567) and the update limits of step (:641-651).
//
// Layout: the cell part of the Jacobian is block-CSR with 2x2 blocks
// (row-major in the block: d water/dp, d water/dsW, d oil/dp, d oil/dsW),
// one block row per cell, columns sorted, diagonal included.  Every
// interface flux is evaluated by both of its cells from the same canonical
// (N0, N1) orientation, so the two evaluations are bitwise identical and each
// cell sums only into its own row: no atomics, bit-reproducible residuals.
#include <climits>
#include <algorithm>
#include <cmath>
#include <numeric>

#include "pmb_ow.cuh"

namespace pmb {

// ---------------------------------------------------------------------------
// fluid
// ---------------------------------------------------------------------------

struct CellProps {
  double bw, dbw, bo, dbo, mw, dmw, mo, dmo;
};

__device__ __forceinline__ void shrink(const FluidDev& f, int i, double p, double& b, double& db) {
  if (f.c[i] == 0.0) {
    b = f.b0[i];
    db = 0.0;
  } else {
    b = f.b0[i] * exp(f.c[i] * (p - f.p_ref));
    db = f.c[i] * b;
  }
}

// kr(s) = clamp((s - sl)/(su - sl), 0, 1)^n with the derivative passed where
// 0 <= u <= 1 (ad_max / ad_min keep ties), or s^n when unscaled.
__device__ __forceinline__ void relperm(const FluidDev& f, int i, double s, double& kr, double& dkr) {
  const double n = f.n[i];
  double v, d;
  if (f.plain[i]) {
    v = s;
    d = 1.0;
  } else {
    const double u = (s - f.sl[i]) * f.inv_range[i];
    const double m = fmin(u, 1.0);
    v = fmax(m, 0.0);
    d = (u <= 1.0 && m >= 0.0) ? f.inv_range[i] : 0.0;
  }
  if (n == 2.0) {
    kr = v * v;
    dkr = d == 0.0 ? 0.0 : 2.0 * v * d;
  } else if (n == 1.0) {
    kr = v;
    dkr = d;
  } else {
    kr = pow(v, n);
    dkr = d == 0.0 ? 0.0 : n * pow(v, n - 1.0) * d;
  }
}

__device__ __forceinline__ CellProps cell_props(const FluidDev& f, double p, double sw) {
  CellProps P;
  shrink(f, 0, p, P.bw, P.dbw);
  shrink(f, 1, p, P.bo, P.dbo);
  double kr, dkr;
  relperm(f, 0, sw, kr, dkr);
  P.mw = kr * f.mu_inv[0];
  P.dmw = dkr * f.mu_inv[0];
  relperm(f, 1, 1.0 - sw, kr, dkr);
  P.mo = kr * f.mu_inv[1];
  P.dmo = -(dkr * f.mu_inv[1]);
  return P;
}

// Phase flux F = b_up * (-T mob_up) * pot with pot = (pR - pL) - avg(rho) gdz,
// upstream N0 where pot <= 0 (faceUpstr), and its derivatives.
struct PhaseFlux {
  double F, dpL, dpR, dsL, dsR;
};

__device__ __forceinline__ PhaseFlux phase_flux(double rhoS, double T, double g, double dp,
                                                double bL, double dbL, double mL, double dmL,
                                                double bR, double dbR, double mR, double dmR) {
  PhaseFlux o;
  const double pot = dp - (0.5 * (rhoS * bL) + 0.5 * (rhoS * bR)) * g;
  const bool upL = pot <= 0.0;
  const double mob = upL ? mL : mR, dmob = upL ? dmL : dmR;
  const double b = upL ? bL : bR, db = upL ? dbL : dbR;
  const double tm = -T * mob;
  const double v = tm * pot;
  o.F = b * v;
  const double dpotL = -1.0 - g * 0.5 * (rhoS * dbL);
  const double dpotR = 1.0 - g * 0.5 * (rhoS * dbR);
  o.dpL = (upL ? db * v : 0.0) + b * tm * dpotL;
  o.dpR = (upL ? 0.0 : db * v) + b * tm * dpotR;
  const double ds = b * (-T * dmob * pot);
  o.dsL = upL ? ds : 0.0;
  o.dsR = upL ? 0.0 : ds;
  return o;
}

// ---------------------------------------------------------------------------
// cell + face assembly: one thread per cell, gathering over its block row
// ---------------------------------------------------------------------------

template <bool JAC>
__global__ void __launch_bounds__(256) ow_cell_kernel(OWView v, const double2* __restrict__ x,
                                                      const double2* __restrict__ x0, double idt,
                                                      double2* __restrict__ res,
                                                      double4* __restrict__ jac) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= v.nc) return;
  const FluidDev& f = v.fl;
  const double2 xs = x[c];
  const double2 xs0 = x0[c];
  const double p = xs.x, sw = xs.y;
  const CellProps P = cell_props(f, p, sw);
  double bw0, dbw0, bo0, dbo0;
  shrink(f, 0, xs0.x, bw0, dbw0);
  shrink(f, 1, xs0.x, bo0, dbo0);
  const double pv = v.pv[c];
  const double so = 1.0 - sw;
  const double acc_w = idt * (pv * P.bw * sw - pv * bw0 * xs0.y);
  const double acc_o = idt * (pv * P.bo * so - pv * bo0 * (1.0 - xs0.y));
  double d00 = idt * pv * P.dbw * sw, d01 = idt * pv * P.bw;
  double d10 = idt * pv * P.dbo * so, d11 = -idt * pv * P.bo;
  double fw = 0.0, fo = 0.0;
  const int k0 = v.row_ptr[c], k1 = v.row_ptr[c + 1];
  for (int k = k0; k < k1; ++k) {
    const int code = v.nz_face[k];
    if (code == INT_MIN) continue;
    const int nb = v.col[k];
    const bool rowL = code >= 0;
    const int fi = rowL ? code : -code - 1;
    const double T = v.T[fi], g = v.gdz[fi];
    const double2 xn = x[nb];
    const CellProps Q = cell_props(f, xn.x, xn.y);
    const CellProps& A = rowL ? P : Q;  // N0 side
    const CellProps& B = rowL ? Q : P;  // N1 side
    const double pL = rowL ? p : xn.x, pR = rowL ? xn.x : p;
    const double dp = pR - pL;
    const PhaseFlux W = phase_flux(f.rhoS[0], T, g, dp, A.bw, A.dbw, A.mw, A.dmw, B.bw, B.dbw, B.mw, B.dmw);
    const PhaseFlux O = phase_flux(f.rhoS[1], T, g, dp, A.bo, A.dbo, A.mo, A.dmo, B.bo, B.dbo, B.mo, B.dmo);
    const double sg = rowL ? 1.0 : -1.0;
    fw += sg * W.F;
    fo += sg * O.F;
    if (JAC) {
      if (rowL) {
        d00 += W.dpL; d01 += W.dsL; d10 += O.dpL; d11 += O.dsL;
        jac[k] = make_double4(W.dpR, W.dsR, O.dpR, O.dsR);
      } else {
        d00 -= W.dpR; d01 -= W.dsR; d10 -= O.dpR; d11 -= O.dsR;
        jac[k] = make_double4(-W.dpL, -W.dsL, -O.dpL, -O.dsL);
      }
    }
  }
  res[c] = make_double2(acc_w + fw, acc_o + fo);
  if (JAC) jac[v.diag_pos[c]] = make_double4(d00, d01, d10, d11);
}

// Phase fluxes of every interface, written by its N0 cell with the arithmetic
// of ow_cell_kernel: face f adds flux[f] to the residual rows (water, oil) of
// N[f,0] and subtracts it from those of N[f,1].
__global__ void __launch_bounds__(256) ow_face_flux_kernel(OWView v, const double2* __restrict__ x,
                                                           double2* __restrict__ flux) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= v.nc) return;
  const FluidDev& f = v.fl;
  const double2 xs = x[c];
  const CellProps P = cell_props(f, xs.x, xs.y);
  for (int k = v.row_ptr[c]; k < v.row_ptr[c + 1]; ++k) {
    const int code = v.nz_face[k];
    if (code == INT_MIN || code < 0) continue;  // diagonal, or this cell is N[f,1]
    const int nb = v.col[k];
    const double T = v.T[code], g = v.gdz[code];
    const double2 xn = x[nb];
    const CellProps Q = cell_props(f, xn.x, xn.y);
    const double dp = xn.x - xs.x;
    const PhaseFlux W = phase_flux(f.rhoS[0], T, g, dp, P.bw, P.dbw, P.mw, P.dmw, Q.bw, Q.dbw, Q.mw, Q.dmw);
    const PhaseFlux O = phase_flux(f.rhoS[1], T, g, dp, P.bo, P.dbo, P.mo, P.dmo, Q.bo, Q.dbo, Q.mo, Q.dmo);
    flux[code] = make_double2(W.F, O.F);
  }
}

// ---------------------------------------------------------------------------
// wells: one warp per well inside a single CTA (standard well model,
// _well_contributions_batched, two_phase_oil_water_model.py:286-491)
// ---------------------------------------------------------------------------

struct PerfProd {
  double dd, cq_psw, cq_pso, dpsw_p, dpsw_s, dpso_p, dpso_s, dpsw_b, dpso_b;
  bool inj;
  CellProps P;
};

__device__ __forceinline__ PerfProd perf_prod(const OWView& v, const double2* x, int i, double bhp,
                                              double cdp) {
  PerfProd r;
  const int c = v.perf_cell[i];
  const double t = v.perf_WI[i];
  const double2 xs = x[c];
  r.P = cell_props(v.fl, xs.x, xs.y);
  r.dd = -(bhp + cdp) + xs.x;
  r.inj = r.dd < 0.0;
  const double ce = r.inj ? 0.0 : t;
  const double cq_pw = -ce * r.P.mw * r.dd;
  const double cq_po = -ce * r.P.mo * r.dd;
  r.cq_psw = r.P.bw * cq_pw;
  r.cq_pso = r.P.bo * cq_po;
  r.dpsw_p = r.P.dbw * cq_pw + r.P.bw * (-ce * r.P.mw);
  r.dpsw_s = r.P.bw * (-ce * r.P.dmw * r.dd);
  r.dpso_p = r.P.dbo * cq_po + r.P.bo * (-ce * r.P.mo);
  r.dpso_s = r.P.bo * (-ce * r.P.dmo * r.dd);
  r.dpsw_b = r.P.bw * (ce * r.P.mw);
  r.dpso_b = r.P.bo * (ce * r.P.mo);
  return r;
}

struct WellMix {
  double mix_w, mix_o, inv_t;
  double dmix[2][3];
  bool dead;
};

// Wellbore mixture of well k from the warp-reduced producer sums.
__device__ __forceinline__ WellMix well_mix(const OWView& v, int k, double qws, double qos,
                                            double S_w, double S_o, double Sb_w, double Sb_o,
                                            bool any_prod) {
  WellMix m;
  const double pos_w = qws > 0.0 ? 1.0 : 0.0, pos_o = qos > 0.0 ? 1.0 : 0.0;
  const double wbq_w = qws * pos_w - S_w;
  const double wbq_o = qos * pos_o - S_o;
  const double wbqt = wbq_w + wbq_o;
  m.dead = (wbqt == 0.0) || !any_prod;
  for (int a = 0; a < 2; ++a)
    for (int j = 0; j < 3; ++j) m.dmix[a][j] = 0.0;
  if (m.dead) {
    m.mix_w = v.compi[2 * k];
    m.mix_o = v.compi[2 * k + 1];
    m.inv_t = 0.0;
  } else {
    m.inv_t = 1.0 / wbqt;
    m.mix_w = wbq_w * m.inv_t;
    m.mix_o = wbq_o * m.inv_t;
    const double dqw[3] = {pos_w, 0.0, -Sb_w};
    const double dqo[3] = {0.0, pos_o, -Sb_o};
    for (int j = 0; j < 3; ++j) {
      const double dqt = dqw[j] + dqo[j];
      m.dmix[0][j] = (dqw[j] - m.mix_w * dqt) * m.inv_t;
      m.dmix[1][j] = (dqo[j] - m.mix_o * dqt) * m.inv_t;
    }
  }
  return m;
}

struct PerfFull {
  double cq_sw, cq_so;
  double dloc[2][2];
  double U[2][2];
  double dcq_b[2];  // direct d cq / d bhp (without the mixture term)
  double V[2][2];
};

__device__ __forceinline__ PerfFull perf_full(const OWView& v, int i, const PerfProd& r,
                                              const WellMix& m) {
  PerfFull o;
  const CellProps& P = r.P;
  const double t = v.perf_WI[i];
  const double ci = r.inj ? t : 0.0;
  const double mt = P.mw + P.mo, dmt = P.dmw + P.dmo;
  const double cqt_i = -ci * (mt * r.dd);
  const double dcqt_p = -ci * mt, dcqt_s = -ci * (dmt * r.dd), dcqt_b = ci * mt;
  const double vol_rat = m.mix_w / P.bw + m.mix_o / P.bo;
  const double inv_vr = 1.0 / vol_rat;
  const double cqt_is = cqt_i * inv_vr;
  const double dvr_p = -m.mix_w * P.dbw / (P.bw * P.bw) - m.mix_o * P.dbo / (P.bo * P.bo);
  const double dis_p = (dcqt_p - cqt_is * dvr_p) * inv_vr;
  const double dis_s = dcqt_s * inv_vr;
  const double dis_b = dcqt_b * inv_vr;
  const double dis_mw = -cqt_is * (1.0 / P.bw) * inv_vr;
  const double dis_mo = -cqt_is * (1.0 / P.bo) * inv_vr;
  o.cq_sw = r.cq_psw + m.mix_w * cqt_is;
  o.cq_so = r.cq_pso + m.mix_o * cqt_is;
  o.dloc[0][0] = r.dpsw_p + m.mix_w * dis_p;
  o.dloc[0][1] = r.dpsw_s + m.mix_w * dis_s;
  o.dloc[1][0] = r.dpso_p + m.mix_o * dis_p;
  o.dloc[1][1] = r.dpso_s + m.mix_o * dis_s;
  o.U[0][0] = cqt_is + m.mix_w * dis_mw;
  o.U[0][1] = m.mix_w * dis_mo;
  o.U[1][0] = m.mix_o * dis_mw;
  o.U[1][1] = cqt_is + m.mix_o * dis_mo;
  o.dcq_b[0] = r.dpsw_b + m.mix_w * dis_b;
  o.dcq_b[1] = r.dpso_b + m.mix_o * dis_b;
  if (m.dead) {
    o.V[0][0] = o.V[0][1] = o.V[1][0] = o.V[1][1] = 0.0;
  } else {
    const double wt_p = -(r.dpsw_p + r.dpso_p), wt_s = -(r.dpsw_s + r.dpso_s);
    o.V[0][0] = (-r.dpsw_p - m.mix_w * wt_p) * m.inv_t;
    o.V[0][1] = (-r.dpsw_s - m.mix_w * wt_s) * m.inv_t;
    o.V[1][0] = (-r.dpso_p - m.mix_o * wt_p) * m.inv_t;
    o.V[1][1] = (-r.dpso_s - m.mix_o * wt_s) * m.inv_t;
  }
  return o;
}

template <bool JAC>
__global__ void __launch_bounds__(256) ow_well_kernel(OWView v, const double2* __restrict__ x,
                                                      const double* __restrict__ cdp,
                                                      double* __restrict__ res,
                                                      double4* __restrict__ jac,
                                                      double* __restrict__ wj,
                                                      double2* __restrict__ pf_cq,
                                                      double4* __restrict__ pf_dloc) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const double* xw = reinterpret_cast<const double*>(x) + 2LL * v.nc;
  const WellLayout& L = v.wl;
  for (int k = warp; k < v.nw; k += nwarp) {
    const int i0 = v.perf_ptr[k], i1 = v.perf_ptr[k + 1];
    const double qws = xw[3 * k], qos = xw[3 * k + 1], bhp = xw[3 * k + 2];
    double S_w = 0, S_o = 0, Sb_w = 0, Sb_o = 0;
    bool anyp = false;
    for (int i = i0 + lane; i < i1; i += 32) {
      const PerfProd r = perf_prod(v, x, i, bhp, cdp[i]);
      S_w += r.cq_psw; S_o += r.cq_pso; Sb_w += r.dpsw_b; Sb_o += r.dpso_b;
      anyp |= !r.inj;
    }
    S_w = warp_sum(S_w); S_o = warp_sum(S_o); Sb_w = warp_sum(Sb_w); Sb_o = warp_sum(Sb_o);
    anyp = __any_sync(0xffffffffu, anyp);
    const WellMix m = well_mix(v, k, qws, qos, S_w, S_o, Sb_w, Sb_o, anyp);
    double Q_w = 0, Q_o = 0, Us[2][2] = {{0, 0}, {0, 0}}, Sd[2][3] = {{0, 0, 0}, {0, 0, 0}};
    for (int i = i0 + lane; i < i1; i += 32) {
      const PerfProd r = perf_prod(v, x, i, bhp, cdp[i]);
      const PerfFull o = perf_full(v, i, r, m);
      pf_cq[i] = make_double2(o.cq_sw, o.cq_so);
      Q_w += o.cq_sw; Q_o += o.cq_so;
      if (JAC) {
        pf_dloc[i] = make_double4(o.dloc[0][0], o.dloc[0][1], o.dloc[1][0], o.dloc[1][1]);
        double* B = wj + L.B + 6LL * i;
        for (int a = 0; a < 2; ++a) {
          for (int j = 0; j < 3; ++j) {
            const double d = (j == 2 ? o.dcq_b[a] : 0.0) + o.U[a][0] * m.dmix[0][j] + o.U[a][1] * m.dmix[1][j];
            B[3 * a + j] = -d;
            Sd[a][j] += d;
          }
        }
        double* U = wj + L.U + 4LL * i;
        double* V = wj + L.V + 4LL * i;
        for (int a = 0; a < 2; ++a)
          for (int b = 0; b < 2; ++b) {
            U[2 * a + b] = m.dead ? 0.0 : -o.U[a][b];
            V[2 * a + b] = o.V[a][b];
            Us[a][b] += o.U[a][b];
          }
      }
    }
    Q_w = warp_sum(Q_w); Q_o = warp_sum(Q_o);
    if (JAC) {
      for (int a = 0; a < 2; ++a) {
        for (int b = 0; b < 2; ++b) Us[a][b] = warp_sum(Us[a][b]);
        for (int j = 0; j < 3; ++j) Sd[a][j] = warp_sum(Sd[a][j]);
      }
      for (int i = i0 + lane; i < i1; i += 32) {
        const double4 dl = pf_dloc[i];
        const double* V = wj + L.V + 4LL * i;
        double* C = wj + L.C + 4LL * i;
        const double dloc[2][2] = {{dl.x, dl.y}, {dl.z, dl.w}};
        for (int a = 0; a < 2; ++a)
          for (int b = 0; b < 2; ++b)
            C[2 * a + b] = -(dloc[a][b] + (m.dead ? 0.0 : Us[a][0] * V[b] + Us[a][1] * V[2 + b]));
      }
    }
    if (lane == 0) {
      double* rw = res + 2LL * v.nc + 3LL * k;
      rw[0] = qws - Q_w;
      rw[1] = qos - Q_o;
      const bool is_bhp = v.well_type[k] == 0;
      rw[2] = is_bhp ? bhp - v.well_val[k] : qws + qos - v.well_val[k];
      if (JAC) {
        double* D = wj + L.D + 9LL * k;
        D[0] = 1.0 - Sd[0][0]; D[1] = -Sd[0][1]; D[2] = -Sd[0][2];
        D[3] = -Sd[1][0]; D[4] = 1.0 - Sd[1][1]; D[5] = -Sd[1][2];
        D[6] = is_bhp ? 0.0 : 1.0; D[7] = is_bhp ? 0.0 : 1.0; D[8] = is_bhp ? 1.0 : 0.0;
        wj[L.M + k] = m.dead ? 0.0 : 1.0;
      }
    }
  }
  __syncthreads();
  // perforated cells: subtract the connection rates from the cell rows
  double2* rc = reinterpret_cast<double2*>(res);
  for (int q = threadIdx.x; q < v.npc; q += blockDim.x) {
    const int c = v.pcell[q];
    double2 r = rc[c];
    double4 dg = JAC ? jac[v.diag_pos[c]] : make_double4(0, 0, 0, 0);
    for (int j = v.pc_ptr[q]; j < v.pc_ptr[q + 1]; ++j) {
      const int i = v.pc_perf[j];
      const double2 cq = pf_cq[i];
      r.x -= cq.x;
      r.y -= cq.y;
      if (JAC) {
        const double4 dl = pf_dloc[i];
        dg.x -= dl.x; dg.y -= dl.y; dg.z -= dl.z; dg.w -= dl.w;
      }
    }
    rc[c] = r;
    if (JAC) jac[v.diag_pos[c]] = dg;
  }
}

// Wellbore hydrostatics once per step (_compute_cdp_per_well,
// _segment_mix_fractions, _topology_cdp; two_phase_oil_water_model.py:205-284).
__global__ void __launch_bounds__(256) ow_cdp_kernel(OWView v, const double2* __restrict__ x0,
                                                     const double* __restrict__ prev_cdp,
                                                     double2* __restrict__ pf_cq,
                                                     double* __restrict__ cdp_out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const double* xw = reinterpret_cast<const double*>(x0) + 2LL * v.nc;
  for (int k = warp; k < v.nw; k += nwarp) {
    const int i0 = v.perf_ptr[k], i1 = v.perf_ptr[k + 1];
    const double qws = xw[3 * k], qos = xw[3 * k + 1], bhp = xw[3 * k + 2];
    double S_w = 0, S_o = 0, Sb_w = 0, Sb_o = 0;
    bool anyp = false;
    for (int i = i0 + lane; i < i1; i += 32) {
      const PerfProd r = perf_prod(v, x0, i, bhp, prev_cdp[i]);
      S_w += r.cq_psw; S_o += r.cq_pso; Sb_w += r.dpsw_b; Sb_o += r.dpso_b;
      anyp |= !r.inj;
    }
    S_w = warp_sum(S_w); S_o = warp_sum(S_o); Sb_w = warp_sum(Sb_w); Sb_o = warp_sum(Sb_o);
    anyp = __any_sync(0xffffffffu, anyp);
    const WellMix m = well_mix(v, k, qws, qos, S_w, S_o, Sb_w, Sb_o, anyp);
    for (int i = i0 + lane; i < i1; i += 32) {
      const PerfProd r = perf_prod(v, x0, i, bhp, prev_cdp[i]);
      const PerfFull o = perf_full(v, i, r, m);
      pf_cq[i] = make_double2(o.cq_sw, o.cq_so);
    }
    __syncwarp();
    if (lane == 0) {
      // reverse cumulative segment rates -> per-segment mixture fractions
      // (stashed in pf_cq), then the cumulated g * rho_mix * dz
      double seg_w = 0.0, seg_o = 0.0;
      for (int i = i1 - 1; i >= i0; --i) {
        const double2 cq = pf_cq[i];
        seg_w += cq.x;
        seg_o += cq.y;
        const double seg_t = seg_w + seg_o;
        const bool dead = seg_t == 0.0;
        const double safe = dead ? 1.0 : seg_t;
        pf_cq[i] = make_double2(dead ? v.compi[2 * k] : seg_w / safe,
                                dead ? v.compi[2 * k + 1] : seg_o / safe);
      }
      double acc = 0.0, zprev = 0.0;
      for (int i = i0; i < i1; ++i) {
        const double2 mx = pf_cq[i];
        const double2 xs = x0[v.perf_cell[i]];
        double bw, dbw, bo, dbo;
        shrink(v.fl, 0, xs.x, bw, dbw);
        shrink(v.fl, 1, xs.x, bo, dbo);
        const double vol_rat = mx.x / bw + mx.y / bo;
        const double rho_mix = (mx.x * v.fl.rhoS[0] + mx.y * v.fl.rhoS[1]) / vol_rat;
        const double dz = v.perf_dZ[i] - zprev;
        zprev = v.perf_dZ[i];
        acc += v.gravity * rho_mix * dz;
        cdp_out[i] = acc;
      }
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// operator application y = J x
// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(256) bsr2_spmv_kernel(int nc, const int* __restrict__ row_ptr,
                                                        const int* __restrict__ col,
                                                        const double4* __restrict__ A,
                                                        const double2* __restrict__ x,
                                                        double2* __restrict__ y) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  double y0 = 0.0, y1 = 0.0;
  const int k1 = row_ptr[c + 1];
  for (int k = row_ptr[c]; k < k1; ++k) {
    const double4 a = A[k];
    const double2 xv = x[col[k]];
    y0 += a.x * xv.x + a.y * xv.y;
    y1 += a.z * xv.x + a.w * xv.y;
  }
  y[c] = make_double2(y0, y1);
}

// Well rows, and the well columns / mixture coupling of perforated cells.
__global__ void __launch_bounds__(256) ow_well_spmv_kernel(OWView v, const double* __restrict__ wj,
                                                           const double* __restrict__ x,
                                                           double* __restrict__ y) {
  extern __shared__ double s_mix[];  // 2 per well
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const WellLayout& L = v.wl;
  const double* xw = x + 2LL * v.nc;
  for (int k = warp; k < v.nw; k += nwarp) {
    double s0 = 0, s1 = 0, e0 = 0, e1 = 0;
    for (int i = v.perf_ptr[k] + lane; i < v.perf_ptr[k + 1]; i += 32) {
      const int c = v.perf_cell[i];
      const double xp = x[2LL * c], xs = x[2LL * c + 1];
      const double* V = wj + L.V + 4LL * i;
      const double* C = wj + L.C + 4LL * i;
      s0 += V[0] * xp + V[1] * xs;
      s1 += V[2] * xp + V[3] * xs;
      e0 += C[0] * xp + C[1] * xs;
      e1 += C[2] * xp + C[3] * xs;
    }
    s0 = warp_sum(s0); s1 = warp_sum(s1); e0 = warp_sum(e0); e1 = warp_sum(e1);
    if (lane == 0) {
      const double* D = wj + L.D + 9LL * k;
      const double a = xw[3 * k], b = xw[3 * k + 1], c = xw[3 * k + 2];
      double* yw = y + 2LL * v.nc + 3LL * k;
      yw[0] = e0 + D[0] * a + D[1] * b + D[2] * c;
      yw[1] = e1 + D[3] * a + D[4] * b + D[5] * c;
      yw[2] = D[6] * a + D[7] * b + D[8] * c;
      const bool on = wj[L.M + k] != 0.0;
      s_mix[2 * k] = on ? s0 : 0.0;
      s_mix[2 * k + 1] = on ? s1 : 0.0;
    }
  }
  __syncthreads();
  for (int q = threadIdx.x; q < v.npc; q += blockDim.x) {
    const int c = v.pcell[q];
    double y0 = y[2LL * c], y1 = y[2LL * c + 1];
    for (int j = v.pc_ptr[q]; j < v.pc_ptr[q + 1]; ++j) {
      const int i = v.pc_perf[j];
      const int k = v.perf_well[i];
      const double* B = wj + L.B + 6LL * i;
      const double* U = wj + L.U + 4LL * i;
      const double a = xw[3 * k], b = xw[3 * k + 1], cc = xw[3 * k + 2];
      y0 += B[0] * a + B[1] * b + B[2] * cc + U[0] * s_mix[2 * k] + U[1] * s_mix[2 * k + 1];
      y1 += B[3] * a + B[4] * b + B[5] * cc + U[2] * s_mix[2 * k] + U[3] * s_mix[2 * k + 1];
    }
    y[2LL * c] = y0;
    y[2LL * c + 1] = y1;
  }
}

// ---------------------------------------------------------------------------
// convergence (CNV / MB / wells) and the limited Newton update
// ---------------------------------------------------------------------------

constexpr int kConvBlocks = 2 * kNumSM;
constexpr int kConvVals = 7;

// Per-block partial maxima and sums; a non-finite residual is counted
// separately so that fmax cannot hide it.
__global__ void __launch_bounds__(256) ow_conv_partial_kernel(OWView v, const double2* __restrict__ res,
                                                              const double2* __restrict__ x,
                                                              double* __restrict__ part) {
  __shared__ double sh[32];
  double mw = 0, mo = 0, sw = 0, so = 0, iw = 0, io = 0, bad = 0;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < v.nc; c += gridDim.x * blockDim.x) {
    const double2 r = res[c];
    const double pv = v.pv[c];
    const double aw = fabs(r.x / pv), ao = fabs(r.y / pv);
    if (!(isfinite(aw) && isfinite(ao))) bad += 1.0;
    mw = fmax(mw, aw);
    mo = fmax(mo, ao);
    sw += r.x;
    so += r.y;
    double b, db;
    shrink(v.fl, 0, x[c].x, b, db);
    iw += 1.0 / b;
    shrink(v.fl, 1, x[c].x, b, db);
    io += 1.0 / b;
  }
  const double bmw = block_max(mw, sh);
  const double bmo = block_max(mo, sh);
  const double bsw = block_sum(sw, sh);
  const double bso = block_sum(so, sh);
  const double biw = block_sum(iw, sh);
  const double bio = block_sum(io, sh);
  const double bbad = block_sum(bad, sh);
  if (threadIdx.x == 0) {
    double* o = part + kConvVals * blockIdx.x;
    o[0] = bmw; o[1] = bmo; o[2] = bsw; o[3] = bso; o[4] = biw; o[5] = bio; o[6] = bbad;
  }
}

__global__ void __launch_bounds__(256) ow_conv_final_kernel(OWView v, const double* __restrict__ part,
                                                            int nparts, const double* __restrict__ res,
                                                            double dt, double pv_tot,
                                                            double* __restrict__ out) {
  __shared__ double sh[32];
  double mw = 0, mo = 0, sw = 0, so = 0, iw = 0, io = 0, bad = 0;
  for (int b = threadIdx.x; b < nparts; b += blockDim.x) {
    const double* o = part + kConvVals * b;
    mw = fmax(mw, o[0]); mo = fmax(mo, o[1]);
    sw += o[2]; so += o[3]; iw += o[4]; io += o[5]; bad += o[6];
  }
  mw = block_max(mw, sh); mo = block_max(mo, sh);
  sw = block_sum(sw, sh); so = block_sum(so, sh);
  iw = block_sum(iw, sh); io = block_sum(io, sh);
  bad = block_sum(bad, sh);
  if (threadIdx.x == 0) {
    const double bw = iw / v.nc, bo = io / v.nc;
    const double cnv = fmax(bw * dt * mw, bo * dt * mo);
    const double mb = fmax(bw * dt * fabs(sw) / pv_tot, bo * dt * fabs(so) / pv_tot);
    double ew = 0.0, eo = 0.0;
    bool ctrl_ok = true, finite = bad == 0.0 && isfinite(cnv) && isfinite(mb);
    const double* rw = res + 2LL * v.nc;
    for (int k = 0; k < v.nw; ++k) {
      const double a = fabs(rw[3 * k]), b = fabs(rw[3 * k + 1]), c = fabs(rw[3 * k + 2]);
      finite = finite && isfinite(a) && isfinite(b) && isfinite(c);
      ew = fmax(ew, a);
      eo = fmax(eo, b);
      const double scale = v.well_type[k] == 0 ? 1.0e5 : v.q_ref;
      ctrl_ok = ctrl_ok && (c <= v.tol_well * scale);
    }
    const bool well_ok = v.nw == 0 || (ew <= v.tol_well * v.q_ref && eo <= v.tol_well * v.q_ref);
    const bool conv = finite && cnv <= v.tol_cnv && mb <= v.tol_mb && well_ok && ctrl_ok;
    out[0] = cnv;
    out[1] = mb;
    out[2] = ew / v.q_ref;
    out[3] = eo / v.q_ref;
    out[4] = ctrl_ok ? 1.0 : 0.0;
    out[5] = conv ? 1.0 : 0.0;
    out[6] = finite ? 0.0 : 1.0;
    out[7] = 0.0;
  }
}

// Convergence of each member of a batch of independent models stored as one
// (block m: cells [cell_ptr[m], cell_ptr[m+1]), wells [well_ptr[m],
// well_ptr[m+1])): the values of ow_conv_final_kernel computed over the
// member alone, its pore volume and rate scale included.
__global__ void __launch_bounds__(256) ow_member_conv_kernel(OWView v, const int* __restrict__ cell_ptr,
                                                             const int* __restrict__ well_ptr,
                                                             const double* __restrict__ res,
                                                             const double* __restrict__ x, double dt,
                                                             double* __restrict__ out) {
  __shared__ double sh[32];
  const int m = blockIdx.x;
  const int c0 = cell_ptr[m], c1 = cell_ptr[m + 1];
  const double2* r2 = reinterpret_cast<const double2*>(res);
  const double2* x2 = reinterpret_cast<const double2*>(x);
  double mw = 0, mo = 0, sw = 0, so = 0, iw = 0, io = 0, bad = 0, pvs = 0;
  for (int c = c0 + threadIdx.x; c < c1; c += blockDim.x) {
    const double2 r = r2[c];
    const double pv = v.pv[c];
    const double aw = fabs(r.x / pv), ao = fabs(r.y / pv);
    if (!(isfinite(aw) && isfinite(ao))) bad += 1.0;
    mw = fmax(mw, aw);
    mo = fmax(mo, ao);
    sw += r.x;
    so += r.y;
    pvs += pv;
    double b, db;
    shrink(v.fl, 0, x2[c].x, b, db);
    iw += 1.0 / b;
    shrink(v.fl, 1, x2[c].x, b, db);
    io += 1.0 / b;
  }
  mw = block_max(mw, sh); mo = block_max(mo, sh);
  sw = block_sum(sw, sh); so = block_sum(so, sh);
  iw = block_sum(iw, sh); io = block_sum(io, sh);
  bad = block_sum(bad, sh); pvs = block_sum(pvs, sh);
  if (threadIdx.x != 0) return;
  const int nc = c1 - c0, w0 = well_ptr[m], w1 = well_ptr[m + 1];
  double qmax = 0.0;
  bool any_rate = false;
  for (int k = w0; k < w1; ++k)
    if (v.well_type[k] == 1) { any_rate = true; qmax = fmax(qmax, fabs(v.well_val[k])); }
  const double q_ref = any_rate ? fmax(qmax, 1e-12) : 1.0;
  const double bw = iw / nc, bo = io / nc;
  const double cnv = fmax(bw * dt * mw, bo * dt * mo);
  const double mb = fmax(bw * dt * fabs(sw) / pvs, bo * dt * fabs(so) / pvs);
  double ew = 0.0, eo = 0.0;
  bool ctrl_ok = true, finite = bad == 0.0 && isfinite(cnv) && isfinite(mb);
  const double* rw = res + 2LL * v.nc;
  for (int k = w0; k < w1; ++k) {
    const double a = fabs(rw[3 * k]), b = fabs(rw[3 * k + 1]), c = fabs(rw[3 * k + 2]);
    finite = finite && isfinite(a) && isfinite(b) && isfinite(c);
    ew = fmax(ew, a);
    eo = fmax(eo, b);
    const double scale = v.well_type[k] == 0 ? 1.0e5 : q_ref;
    ctrl_ok = ctrl_ok && (c <= v.tol_well * scale);
  }
  const bool well_ok = w1 == w0 || (ew <= v.tol_well * q_ref && eo <= v.tol_well * q_ref);
  const bool conv = finite && cnv <= v.tol_cnv && mb <= v.tol_mb && well_ok && ctrl_ok;
  double* o = out + 8LL * m;
  o[0] = cnv;
  o[1] = mb;
  o[2] = ew / q_ref;
  o[3] = eo / q_ref;
  o[4] = ctrl_ok ? 1.0 : 0.0;
  o[5] = conv ? 1.0 : 0.0;
  o[6] = finite ? 0.0 : 1.0;
  o[7] = 0.0;
}

// Per member m, out[2m] = ||b_m - y_m||^2 and out[2m+1] = ||b_m||^2 over its
// cells and wells (y = J dx of the shared solve); one CTA per member.
__global__ void __launch_bounds__(256) ow_member_linres_kernel(OWView v, const int* __restrict__ cell_ptr,
                                                               const int* __restrict__ well_ptr,
                                                               const double* __restrict__ b,
                                                               const double* __restrict__ y,
                                                               double* __restrict__ out) {
  __shared__ double sh[32];
  const int m = blockIdx.x;
  double rr = 0.0, bb = 0.0;
  for (long long i = 2LL * cell_ptr[m] + threadIdx.x; i < 2LL * cell_ptr[m + 1]; i += blockDim.x) {
    const double d = b[i] - y[i];
    rr += d * d;
    bb += b[i] * b[i];
  }
  for (long long i = 2LL * v.nc + 3LL * well_ptr[m] + threadIdx.x; i < 2LL * v.nc + 3LL * well_ptr[m + 1];
       i += blockDim.x) {
    const double d = b[i] - y[i];
    rr += d * d;
    bb += b[i] * b[i];
  }
  rr = block_sum(rr, sh);
  bb = block_sum(bb, sh);
  if (threadIdx.x == 0) {
    out[2 * m] = rr;
    out[2 * m + 1] = bb;
  }
}

// Zero the entries (cells and wells) of every member whose flag is 0.
__global__ void __launch_bounds__(256) ow_member_mask_kernel(OWView v, const int* __restrict__ cell_ptr,
                                                             const int* __restrict__ well_ptr,
                                                             const int* __restrict__ flag,
                                                             double* __restrict__ vec) {
  const int m = blockIdx.x;
  if (flag[m] != 0) return;
  for (int c = cell_ptr[m] + threadIdx.x; c < cell_ptr[m + 1]; c += blockDim.x)
    reinterpret_cast<double2*>(vec)[c] = make_double2(0.0, 0.0);
  for (int t = 3 * well_ptr[m] + threadIdx.x; t < 3 * well_ptr[m + 1]; t += blockDim.x) vec[2LL * v.nc + t] = 0.0;
}

__global__ void __launch_bounds__(256) ow_update_kernel(OWView v, double* __restrict__ x,
                                                        const double* __restrict__ dx, double sgn) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < v.nc) {
    const double p = x[2LL * t], sw = x[2LL * t + 1];
    double dp = sgn * dx[2LL * t], ds = sgn * dx[2LL * t + 1];
    const double cap = v.dp_max_rel * fabs(p);
    // comparisons keep a NaN update NaN (np.clip semantics)
    dp = dp < -cap ? -cap : (dp > cap ? cap : dp);
    ds = ds < -v.ds_max ? -v.ds_max : (ds > v.ds_max ? v.ds_max : ds);
    double s = sw + ds;
    s = s < 0.0 ? 0.0 : (s > 1.0 ? 1.0 : s);
    x[2LL * t] = p + dp;
    x[2LL * t + 1] = s;
  }
  if (t < 3 * v.nw) x[2LL * v.nc + t] += sgn * dx[2LL * v.nc + t];
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

OWModel::OWModel(const pmb_ow_desc& d, cudaStream_t s) : stream_(s) {
  PMB_REQUIRE(d.nc > 0, "model needs at least one cell");
  PMB_REQUIRE(d.nf >= 0 && d.nw >= 0, "negative sizes");
  PMB_REQUIRE(d.nf == 0 || (d.h_N && d.h_T && d.h_gdz), "face arrays missing");
  PMB_REQUIRE(d.h_pv, "pore volumes missing");
  const int nc = d.nc, nf = d.nf, nw = d.nw;
  PMB_REQUIRE(2LL * nf + nc < 2147483647LL, "too many connections for 32-bit indices");
  // --- block-CSR pattern from the interface list
  std::vector<int> deg(nc, 1);
  for (int f = 0; f < nf; ++f) {
    const int a = d.h_N[2 * f], b = d.h_N[2 * f + 1];
    PMB_REQUIRE(a >= 0 && a < nc && b >= 0 && b < nc, "interface cell index out of range");
    PMB_REQUIRE(a != b, "interface connects a cell to itself");
    ++deg[a];
    ++deg[b];
  }
  h_row_ptr_.assign(nc + 1, 0);
  for (int c = 0; c < nc; ++c) h_row_ptr_[c + 1] = h_row_ptr_[c] + deg[c];
  nnzb_ = h_row_ptr_[nc];
  h_col_.assign(nnzb_, 0);
  std::vector<int> code(nnzb_, 0), fill(nc, 0);
  for (int c = 0; c < nc; ++c) {
    h_col_[h_row_ptr_[c]] = c;
    code[h_row_ptr_[c]] = INT_MIN;
    fill[c] = 1;
  }
  for (int f = 0; f < nf; ++f) {
    const int a = d.h_N[2 * f], b = d.h_N[2 * f + 1];
    int k = h_row_ptr_[a] + fill[a]++;
    h_col_[k] = b;
    code[k] = f;
    k = h_row_ptr_[b] + fill[b]++;
    h_col_[k] = a;
    code[k] = -(f + 1);
  }
  std::vector<int> diag(nc, 0);
  {
    std::vector<std::pair<int, int>> tmp;
    for (int c = 0; c < nc; ++c) {
      const int k0 = h_row_ptr_[c], k1 = h_row_ptr_[c + 1];
      tmp.clear();
      for (int k = k0; k < k1; ++k) tmp.emplace_back(h_col_[k], code[k]);
      std::sort(tmp.begin(), tmp.end(), [](const std::pair<int, int>& p, const std::pair<int, int>& q) {
        return p.first < q.first;
      });
      for (int k = k0; k < k1; ++k) {
        h_col_[k] = tmp[k - k0].first;
        code[k] = tmp[k - k0].second;
        if (k > k0) PMB_REQUIRE(h_col_[k] != h_col_[k - 1], "two interfaces join the same pair of cells");
        if (h_col_[k] == c) diag[c] = k;
      }
    }
  }
  // --- greedy colouring of the cell graph (red-black on Cartesian grids)
  std::vector<int> color(nc, -1);
  ncolors_ = 0;
  {
    std::vector<int> mark;
    for (int c = 0; c < nc; ++c) {
      mark.assign(ncolors_ + 1, 0);
      for (int k = h_row_ptr_[c]; k < h_row_ptr_[c + 1]; ++k) {
        const int j = h_col_[k];
        if (j != c && color[j] >= 0) mark[color[j]] = 1;
      }
      int col = 0;
      while (col < ncolors_ && mark[col]) ++col;
      color[c] = col;
      if (col == ncolors_) ++ncolors_;
    }
  }
  h_color_ptr_.assign(ncolors_ + 1, 0);
  for (int c = 0; c < nc; ++c) ++h_color_ptr_[color[c] + 1];
  for (int q = 0; q < ncolors_; ++q) h_color_ptr_[q + 1] += h_color_ptr_[q];
  std::vector<int> ccells(nc), cfill(h_color_ptr_.begin(), h_color_ptr_.end() - 1);
  for (int c = 0; c < nc; ++c) ccells[cfill[color[c]]++] = c;

  // --- wells
  int nperf = 0;
  std::vector<int> perf_ptr(nw + 1, 0);
  if (nw) {
    PMB_REQUIRE(d.h_perf_ptr && d.h_perf_cell && d.h_perf_WI && d.h_perf_dZ && d.h_compi &&
                    d.h_well_type && d.h_well_val,
                "well arrays missing");
    for (int k = 0; k <= nw; ++k) perf_ptr[k] = d.h_perf_ptr[k];
    PMB_REQUIRE(perf_ptr[0] == 0, "perf_ptr must start at 0");
    for (int k = 0; k < nw; ++k) {
      PMB_REQUIRE(perf_ptr[k + 1] > perf_ptr[k], "every well needs a perforation");
      PMB_REQUIRE(d.h_well_type[k] == 0 || d.h_well_type[k] == 1, "unsupported well control");
    }
    nperf = perf_ptr[nw];
    for (int i = 0; i < nperf; ++i)
      PMB_REQUIRE(d.h_perf_cell[i] >= 0 && d.h_perf_cell[i] < nc, "perforation cell out of range");
  }
  std::vector<int> order(nperf);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return d.h_perf_cell[a] < d.h_perf_cell[b]; });
  std::vector<int> pcell, pc_ptr(1, 0), pc_perf;
  for (int j = 0; j < nperf; ++j) {
    const int i = order[j], c = d.h_perf_cell[i];
    if (pcell.empty() || pcell.back() != c) {
      if (!pcell.empty()) pc_ptr.push_back((int)pc_perf.size());
      pcell.push_back(c);
    }
    pc_perf.push_back(i);
  }
  if (!pcell.empty()) pc_ptr.push_back((int)pc_perf.size());
  std::vector<int> cell_pc(nc, -1);
  for (size_t q = 0; q < pcell.size(); ++q) cell_pc[pcell[q]] = (int)q;

  // --- upload
  row_ptr_.upload(h_row_ptr_, s);
  col_.upload(h_col_, s);
  nz_face_.upload(code, s);
  diag_pos_.upload(diag, s);
  color_cells_.upload(ccells, s);
  cell_pc_.upload(cell_pc, s);
  if (nf) {
    T_.upload(d.h_T, nf, s);
    gdz_.upload(d.h_gdz, nf, s);
  }
  pv_.upload(d.h_pv, nc, s);
  double pv_tot = 0.0;
  for (int c = 0; c < nc; ++c) pv_tot += d.h_pv[c];
  perf_ptr_.upload(perf_ptr, s);
  if (nw) {
    std::vector<int> perf_well(nperf);
    for (int k = 0; k < nw; ++k)
      for (int i = perf_ptr[k]; i < perf_ptr[k + 1]; ++i) perf_well[i] = k;
    perf_well_.upload(perf_well, s);
    perf_cell_.upload(d.h_perf_cell, nperf, s);
    perf_WI_.upload(d.h_perf_WI, nperf, s);
    perf_dZ_.upload(d.h_perf_dZ, nperf, s);
    compi_.upload(d.h_compi, 2 * nw, s);
    well_type_.upload(d.h_well_type, nw, s);
    well_val_.upload(d.h_well_val, nw, s);
    pcell_.upload(pcell, s);
    pc_ptr_.upload(pc_ptr, s);
    pc_perf_.upload(pc_perf, s);
  }
  pf_cq_.resize(2 * std::max(nperf, 1));
  pf_dloc_.resize(4 * std::max(nperf, 1));
  last_cdp_.resize(std::max(nperf, 1));
  cdp_.resize(std::max(nperf, 1));
  cdp_.zero(s);
  last_cdp_.zero(s);
  conv_part_.resize(kConvVals * kConvBlocks);
  conv_out_.resize(8);

  // --- view
  v_.nc = nc; v_.nf = nf; v_.nw = nw; v_.nperf = nperf;
  v_.row_ptr = row_ptr_.get(); v_.col = col_.get(); v_.nz_face = nz_face_.get();
  v_.diag_pos = diag_pos_.get(); v_.T = T_.get(); v_.gdz = gdz_.get(); v_.pv = pv_.get();
  for (int i = 0; i < 2; ++i) {
    PMB_REQUIRE(d.mu[i] > 0.0, "viscosities must be positive");
    PMB_REQUIRE(d.c[i] >= 0.0, "compressibilities must be non-negative");
    v_.fl.mu_inv[i] = 1.0 / d.mu[i];
    v_.fl.rhoS[i] = d.rhoS[i];
    v_.fl.n[i] = d.n_exp[i];
    v_.fl.c[i] = d.c[i];
    v_.fl.b0[i] = d.b0[i];
    v_.fl.sl[i] = d.sl[i];
    v_.fl.plain[i] = (d.sl[i] == 0.0 && d.su[i] == 1.0) ? 1 : 0;
    v_.fl.inv_range[i] = v_.fl.plain[i] ? 1.0 : 1.0 / (d.su[i] - d.sl[i]);
  }
  v_.fl.p_ref = d.p_ref;
  v_.perf_ptr = perf_ptr_.get(); v_.perf_cell = perf_cell_.get(); v_.perf_WI = perf_WI_.get();
  v_.well_type = well_type_.get(); v_.well_val = well_val_.get(); v_.compi = compi_.get();
  v_.perf_dZ = perf_dZ_.get();
  v_.perf_well = perf_well_.get();
  v_.npc = (int)pcell.size(); v_.pcell = pcell_.get(); v_.pc_ptr = pc_ptr_.get(); v_.pc_perf = pc_perf_.get();
  v_.cell_pc = cell_pc_.get();
  v_.wl = WellLayout::make(nperf, nw);
  v_.gravity = d.gravity;
  h_well_type_.assign(d.h_well_type, d.h_well_type + nw);
  double qmax = 0.0;
  bool any_rate = false;
  for (int k = 0; k < nw; ++k)
    if (d.h_well_type[k] == 1) { any_rate = true; qmax = std::max(qmax, std::fabs(d.h_well_val[k])); }
  v_.q_ref = any_rate ? std::max(qmax, 1e-12) : 1.0;
  v_.tol_cnv = d.tol_cnv; v_.tol_mb = d.tol_mb; v_.tol_well = d.tol_well;
  v_.ds_max = d.ds_max; v_.dp_max_rel = d.dp_max_rel;
  pv_tot_ = pv_tot;

  build_lines(d, code);
  jac_.resize(4 * nnzb_);
  well_.resize(std::max<int64_t>(v_.wl.total, 1));
  res_.resize(nvec());
  x0_.resize(nvec());
  dx_.resize(nvec());
  PMB_CUDA(cudaStreamSynchronize(s));
}

void OWModel::set_well_values(const double* h_val) {
  const int nw = v_.nw;
  for (int k = 0; k < nw; ++k) PMB_REQUIRE(std::isfinite(h_val[k]), "non-finite well target");
  if (nw) well_val_.upload(h_val, nw, stream_);
  double qmax = 0.0;
  bool any_rate = false;
  for (int k = 0; k < nw; ++k)
    if (h_well_type_[k] == 1) { any_rate = true; qmax = std::max(qmax, std::fabs(h_val[k])); }
  v_.q_ref = any_rate ? std::max(qmax, 1e-12) : 1.0;
  PMB_CUDA(cudaStreamSynchronize(stream_));
}

void OWModel::compute_cdp(const double* x0, double* cdp) {
  const int np_ = v_.nperf;
  if (np_ == 0) return;
  if (v_.gravity == 0.0) {
    PMB_CUDA(cudaMemsetAsync(cdp, 0, sizeof(double) * np_, stream_));
    return;
  }
  if (!have_last_cdp_) last_cdp_.zero(stream_);
  ow_cdp_kernel<<<1, 256, 0, stream_>>>(v_, reinterpret_cast<const double2*>(x0), last_cdp_.get(),
                                        reinterpret_cast<double2*>(pf_cq_.get()), cdp);
  PMB_CHECK_LAUNCH();
  PMB_CUDA(cudaMemcpyAsync(last_cdp_.get(), cdp, sizeof(double) * np_, cudaMemcpyDeviceToDevice, stream_));
  have_last_cdp_ = true;
}

void OWModel::fluxes(const double* x, const double* cdp, double* face_flux, double* perf_rate) {
  ow_face_flux_kernel<<<grid_for(v_.nc, 256), 256, 0, stream_>>>(v_, reinterpret_cast<const double2*>(x),
                                                                 reinterpret_cast<double2*>(face_flux));
  PMB_CHECK_LAUNCH();
  if (v_.nw) {
    // the well kernel also subtracts the rates from a residual: give it the
    // model's residual workspace
    ow_well_kernel<false><<<1, 256, 0, stream_>>>(v_, reinterpret_cast<const double2*>(x), cdp, res_.get(),
                                                  nullptr, nullptr, reinterpret_cast<double2*>(pf_cq_.get()),
                                                  reinterpret_cast<double4*>(pf_dloc_.get()));
    PMB_CHECK_LAUNCH();
    PMB_CUDA(cudaMemcpyAsync(perf_rate, pf_cq_.get(), sizeof(double) * 2 * v_.nperf, cudaMemcpyDeviceToDevice,
                             stream_));
  }
}

void OWModel::assemble(const double* x, const double* x0, double dt, const double* cdp, double* res,
                       double* jac, double* well, bool want_jac) {
  const double idt = 1.0 / dt;
  const int g = grid_for(v_.nc, 256);
  if (want_jac)
    ow_cell_kernel<true><<<g, 256, 0, stream_>>>(v_, reinterpret_cast<const double2*>(x),
                                                 reinterpret_cast<const double2*>(x0), idt,
                                                 reinterpret_cast<double2*>(res),
                                                 reinterpret_cast<double4*>(jac));
  else
    ow_cell_kernel<false><<<g, 256, 0, stream_>>>(v_, reinterpret_cast<const double2*>(x),
                                                  reinterpret_cast<const double2*>(x0), idt,
                                                  reinterpret_cast<double2*>(res), nullptr);
  PMB_CHECK_LAUNCH();
  if (v_.nw) {
    if (want_jac)
      ow_well_kernel<true><<<1, 256, 0, stream_>>>(v_, reinterpret_cast<const double2*>(x), cdp, res,
                                                   reinterpret_cast<double4*>(jac), well,
                                                   reinterpret_cast<double2*>(pf_cq_.get()),
                                                   reinterpret_cast<double4*>(pf_dloc_.get()));
    else
      ow_well_kernel<false><<<1, 256, 0, stream_>>>(v_, reinterpret_cast<const double2*>(x), cdp, res,
                                                    nullptr, nullptr,
                                                    reinterpret_cast<double2*>(pf_cq_.get()),
                                                    reinterpret_cast<double4*>(pf_dloc_.get()));
    PMB_CHECK_LAUNCH();
  }
}

void OWModel::spmv(const double* jac, const double* well, const double* x, double* y) {
  bsr2_spmv_kernel<<<grid_for(v_.nc, 256), 256, 0, stream_>>>(
      v_.nc, v_.row_ptr, v_.col, reinterpret_cast<const double4*>(jac),
      reinterpret_cast<const double2*>(x), reinterpret_cast<double2*>(y));
  PMB_CHECK_LAUNCH();
  if (v_.nw) {
    ow_well_spmv_kernel<<<1, 256, sizeof(double) * 2 * v_.nw, stream_>>>(v_, well, x, y);
    PMB_CHECK_LAUNCH();
  }
}

void OWModel::member_convergence_async(int nmem, const int* cell_ptr, const int* well_ptr, const double* res,
                                       const double* x, double dt, double* d_out) {
  ow_member_conv_kernel<<<nmem, 256, 0, stream_>>>(v_, cell_ptr, well_ptr, res, x, dt, d_out);
  PMB_CHECK_LAUNCH();
}

void OWModel::member_linear_residuals_async(int nmem, const int* cell_ptr, const int* well_ptr, const double* b,
                                            const double* dx, double* tmp, double* d_out) {
  spmv(jac(), well(), dx, tmp);
  ow_member_linres_kernel<<<nmem, 256, 0, stream_>>>(v_, cell_ptr, well_ptr, b, tmp, d_out);
  PMB_CHECK_LAUNCH();
}

void OWModel::mask_members(int nmem, const int* cell_ptr, const int* well_ptr, const int* flag, double* vec) {
  ow_member_mask_kernel<<<nmem, 256, 0, stream_>>>(v_, cell_ptr, well_ptr, flag, vec);
  PMB_CHECK_LAUNCH();
}

void OWModel::convergence_async(const double* res, const double* x, double dt, double* d_out) {
  ow_conv_partial_kernel<<<kConvBlocks, 256, 0, stream_>>>(
      v_, reinterpret_cast<const double2*>(res), reinterpret_cast<const double2*>(x), conv_part_.get());
  PMB_CHECK_LAUNCH();
  ow_conv_final_kernel<<<1, 256, 0, stream_>>>(v_, conv_part_.get(), kConvBlocks, res, dt, pv_tot_, d_out);
  PMB_CHECK_LAUNCH();
}

// Vertical lines from the flagged interfaces: each cell keeps at most one
// successor (N[f,1] of a flagged face where it is N[f,0]) and one predecessor;
// lines start at cells without a predecessor.  Cells caught in a cycle of
// flagged faces become lines of their own.
void OWModel::build_lines(const pmb_ow_desc& d, const std::vector<int>& code) {
  (void)code;
  const int nc = v_.nc, nf = v_.nf;
  if (!d.h_line_face || nf == 0) return;
  std::vector<int> next(nc, -1), prev(nc, -1);
  for (int f = 0; f < nf; ++f) {
    if (!d.h_line_face[f]) continue;
    const int a = d.h_N[2 * f], b = d.h_N[2 * f + 1];
    if (next[a] == -1 && prev[b] == -1) {
      next[a] = b;
      prev[b] = a;
    }
  }
  std::vector<int> line_ptr(1, 0), cells;
  cells.reserve(nc);
  std::vector<char> seen(nc, 0);
  for (int c = 0; c < nc; ++c) {
    if (prev[c] != -1) continue;
    for (int t = c; t != -1 && !seen[t]; t = next[t]) {
      seen[t] = 1;
      cells.push_back(t);
    }
    line_ptr.push_back((int)cells.size());
  }
  for (int c = 0; c < nc; ++c)
    if (!seen[c]) {
      seen[c] = 1;
      cells.push_back(c);
      line_ptr.push_back((int)cells.size());
    }
  const int nl = (int)line_ptr.size() - 1;
  auto find = [&](int row, int colv) {
    const int* b = h_col_.data() + h_row_ptr_[row];
    const int* e = h_col_.data() + h_row_ptr_[row + 1];
    const int* it = std::lower_bound(b, e, colv);
    return (it != e && *it == colv) ? (int)(it - h_col_.data()) : -1;
  };
  std::vector<int> lo(nc, -1), up(nc, -1), line_of(nc, 0);
  int max_len = 0;
  for (int L = 0; L < nl; ++L) {
    const int t0 = line_ptr[L], t1 = line_ptr[L + 1];
    max_len = std::max(max_len, t1 - t0);
    for (int t = t0; t < t1; ++t) {
      line_of[cells[t]] = L;
      if (t > t0) lo[t] = find(cells[t], cells[t - 1]);
      if (t + 1 < t1) up[t] = find(cells[t], cells[t + 1]);
    }
  }
  // greedy colouring of the line graph
  std::vector<int> lcolor(nl, -1), mark;
  int ncol = 0;
  for (int L = 0; L < nl; ++L) {
    mark.assign(ncol + 1, 0);
    for (int t = line_ptr[L]; t < line_ptr[L + 1]; ++t) {
      const int c = cells[t];
      for (int k = h_row_ptr_[c]; k < h_row_ptr_[c + 1]; ++k) {
        const int M = line_of[h_col_[k]];
        if (M != L && lcolor[M] >= 0) mark[lcolor[M]] = 1;
      }
    }
    int q = 0;
    while (q < ncol && mark[q]) ++q;
    lcolor[L] = q;
    if (q == ncol) ++ncol;
  }
  lines_.h_color_ptr.assign(ncol + 1, 0);
  for (int L = 0; L < nl; ++L) ++lines_.h_color_ptr[lcolor[L] + 1];
  for (int q = 0; q < ncol; ++q) lines_.h_color_ptr[q + 1] += lines_.h_color_ptr[q];
  std::vector<int> clines(nl), cf(lines_.h_color_ptr.begin(), lines_.h_color_ptr.end() - 1);
  for (int L = 0; L < nl; ++L) clines[cf[lcolor[L]]++] = L;
  lines_.nlines = nl;
  lines_.max_len = max_len;
  lines_.line_ptr.upload(line_ptr, stream_);
  lines_.line_cells.upload(cells, stream_);
  lines_.line_lo.upload(lo, stream_);
  lines_.line_up.upload(up, stream_);
  lines_.color_lines.upload(clines, stream_);
  std::vector<int2> crange(nl);
  for (int k = 0; k < nl; ++k) crange[k] = make_int2(line_ptr[clines[k]], line_ptr[clines[k] + 1] - line_ptr[clines[k]]);
  lines_.color_range.upload(crange, stream_);
}

void OWModel::update(double* x, const double* dx, double sgn) {
  const long long n = std::max<long long>(v_.nc, 3LL * v_.nw);
  ow_update_kernel<<<grid_for(n, 256), 256, 0, stream_>>>(v_, x, dx, sgn);
  PMB_CHECK_LAUNCH();
}

}  // namespace pmb
