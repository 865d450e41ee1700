// Device pieces of the adjoint gradient (compute_gradient_adjoint,
// pymrst/modules/optimization/adjoint.py:163-225): the coupling of one step
// to the previous state, the Jacobian (or its transpose) as a CSR matrix in
// the reference's variable-blocked layout built on the device from the
// model's block-CSR and well part, the permeability sensitivity contracted
// with the adjoint, and the well pressure-drop history that a recomputed
// forward segment must start from.
#include <climits>

#include "pmb_ow.cuh"

namespace pmb {

__device__ __forceinline__ void b_and_db(const FluidDev& f, int i, double p, double& b, double& db) {
  if (f.c[i] == 0.0) {
    b = f.b0[i];
    db = 0.0;
  } else {
    b = f.b0[i] * exp(f.c[i] * (p - f.p_ref));
    db = f.c[i] * b;
  }
}

// dR_{n+1}/dx_n (_jac_wrt_previous, adjoint.py:83-105): water row
// -(pv/dt) d(b_w(p0) s0), oil row -(pv/dt) d(b_o(p0) (1 - s0)), in (p0, s0);
// y = its transpose times lam, one thread per cell.
__global__ void ow_prev_tmul_kernel(OWView v, const double2* __restrict__ x_prev, double idt,
                                    const double* __restrict__ lam, double* __restrict__ y) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int nc = v.nc;
  if (c < nc) {
    const double2 xs = x_prev[c];
    double bw, dbw, bo, dbo;
    b_and_db(v.fl, 0, xs.x, bw, dbw);
    b_and_db(v.fl, 1, xs.x, bo, dbo);
    const double k = idt * v.pv[c], lw = lam[c], lo = lam[nc + c];
    y[c] = -k * dbw * xs.y * lw - k * dbo * (1.0 - xs.y) * lo;
    y[nc + c] = -k * bw * lw + k * bo * lo;
  }
  const int w = c - nc;
  if (w >= 0 && w < 3 * v.nw) y[2 * nc + w] = 0.0;
}

__global__ void ow_csr_values_kernel(int64_t n, const int64_t* __restrict__ ptr, const int64_t* __restrict__ terms,
                                     const double* __restrict__ jac, int64_t njac, const double* __restrict__ well,
                                     WellLayout wl, int nperf, const int* __restrict__ perf_well,
                                     double* __restrict__ vals) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= n) return;
  double s = 0.0;
  for (int64_t q = ptr[e]; q < ptr[e + 1]; ++q) {
    const int64_t t = terms[q];
    if (t >= 0) {
      s += t < njac ? jac[t] : well[t - njac];
    } else {
      const int64_t code = -1 - t;
      const int ab = (int)(code & 3);
      const int64_t ij = code >> 2;
      const int i = (int)(ij / nperf), j = (int)(ij % nperf);
      const int a = ab >> 1, b = ab & 1;
      if (well[wl.M + perf_well[i]] != 0.0) {
        const double* U = well + wl.U + 4LL * i;
        const double* V = well + wl.V + 4LL * j;
        s += U[2 * a] * V[b] + U[2 * a + 1] * V[2 + b];
      }
    }
  }
  vals[e] = s;
}

// One thread per cell: the interfaces of c from its block-CSR row (nz_face
// gives the interface and whether c is N[f,0]), then its perforations.
__global__ void ow_perm_contract_kernel(OWView v, const double2* __restrict__ flux, const double2* __restrict__ q,
                                        const double* __restrict__ lam, const double* __restrict__ t0,
                                        const double* __restrict__ t1, double* __restrict__ out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= v.nc) return;
  const int nc = v.nc;
  const double lwc = lam[c], loc = lam[nc + c];
  double acc = 0.0;
  for (int k = v.row_ptr[c]; k < v.row_ptr[c + 1]; ++k) {
    const int code = v.nz_face[k];
    if (code == INT_MIN) continue;
    const int o = v.col[k];
    const bool first = code >= 0;
    const int f = first ? code : -(code + 1);
    const double th = first ? t0[f] : t1[f];
    if (!(th > 0.0)) continue;
    // lam^T dR/dT_f * T_f = F . (lam[N0] - lam[N1])
    const double2 F = flux[f];
    const double dw = first ? lwc - lam[o] : lam[o] - lwc;
    const double dn = first ? loc - lam[nc + o] : lam[nc + o] - loc;
    acc += (F.x * dw + F.y * dn) * v.T[f] / th;
  }
  const int pq = v.cell_pc[c];
  if (pq >= 0) {
    const int nw = v.nw;
    for (int m = v.pc_ptr[pq]; m < v.pc_ptr[pq + 1]; ++m) {
      const int p = v.pc_perf[m];
      const int w = v.perf_well[p];
      const double2 r = q[p];
      acc += -(lwc + lam[2 * nc + w]) * r.x - (loc + lam[2 * nc + nw + w]) * r.y;
    }
  }
  out[c] += acc;
}

void OWModel::prev_jacobian_tmul(const double* x_prev, double dt, const double* lam, double* y) {
  PMB_REQUIRE(x_prev && lam && y && dt > 0.0, "bad argument");
  const long long n = std::max<long long>(v_.nc, (long long)v_.nc + 3LL * v_.nw);
  ow_prev_tmul_kernel<<<grid_for(n, 256), 256, 0, stream_>>>(v_, reinterpret_cast<const double2*>(x_prev), 1.0 / dt,
                                                             lam, y);
  PMB_CHECK_LAUNCH();
}

void OWModel::csr_values(const double* jac, const double* well, int64_t n, const int64_t* ptr,
                         const int64_t* terms, double* vals) {
  PMB_REQUIRE(jac && ptr && terms && vals && n >= 0, "bad argument");
  PMB_REQUIRE(v_.nw == 0 || well, "NULL well part");
  if (!n) return;
  const WellLayout wl = WellLayout::make(v_.nperf, v_.nw);
  ow_csr_values_kernel<<<grid_for(n, 256), 256, 0, stream_>>>(n, ptr, terms, jac, 4LL * nnzb_, well, wl,
                                                              std::max(v_.nperf, 1), v_.perf_well, vals);
  PMB_CHECK_LAUNCH();
}

void OWModel::perm_contract(const double* x, const double* lam, const double* t0, const double* t1,
                            double* face_flux, double* perf_rate, double* out) {
  PMB_REQUIRE(x && lam && t0 && t1 && face_flux && out, "NULL argument");
  PMB_REQUIRE(v_.nw == 0 || perf_rate, "NULL perforation-rate scratch");
  // the fluxes at cdp = 0, as the adjoint's Jacobians are assembled
  cdp_zero_.resize(std::max(v_.nperf, 1));
  cdp_zero_.zero(stream_);
  fluxes(x, cdp_zero_.get(), face_flux, perf_rate);
  ow_perm_contract_kernel<<<grid_for(v_.nc, 128), 128, 0, stream_>>>(
      v_, reinterpret_cast<const double2*>(face_flux), reinterpret_cast<const double2*>(perf_rate), lam, t0, t1, out);
  PMB_CHECK_LAUNCH();
}

void OWModel::get_last_cdp(double* out, int* have) {
  PMB_REQUIRE(have && (v_.nperf == 0 || out), "NULL argument");
  *have = have_last_cdp_ ? 1 : 0;
  if (have_last_cdp_ && v_.nperf)
    PMB_CUDA(cudaMemcpyAsync(out, last_cdp_.get(), sizeof(double) * v_.nperf, cudaMemcpyDeviceToDevice, stream_));
}

void OWModel::set_last_cdp(const double* in) {
  if (!in) {
    have_last_cdp_ = false;
    return;
  }
  if (v_.nperf)
    PMB_CUDA(cudaMemcpyAsync(last_cdp_.get(), in, sizeof(double) * v_.nperf, cudaMemcpyDeviceToDevice, stream_));
  have_last_cdp_ = true;
}

__global__ void csr_row_scale_kernel(int n, const int* __restrict__ rp, double* __restrict__ vals,
                                     double* __restrict__ scale) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  double m = 0.0;
  for (int k = rp[r]; k < rp[r + 1]; ++k) m = fmax(m, fabs(vals[k]));
  const double d = m > 0.0 ? 1.0 / m : 1.0;
  for (int k = rp[r]; k < rp[r + 1]; ++k) vals[k] *= d;
  scale[r] = d;
}

}  // namespace pmb

extern "C" int pmb_csr_row_scale(int32_t n, const int32_t* d_row_ptr, double* d_vals, double* d_scale,
                                 void* stream) {
  using namespace pmb;
  return guarded([&] {
    PMB_REQUIRE(n >= 0 && d_row_ptr && d_vals && d_scale, "bad argument");
    if (!n) return;
    csr_row_scale_kernel<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(n, d_row_ptr, d_vals, d_scale);
    PMB_CHECK_LAUNCH();
  });
}
