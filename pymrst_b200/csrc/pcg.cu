// AMG-preconditioned conjugate gradients for scalar CSR systems: the
// pressure solve of the incompressible TPFA path (incomp_tpfa's `solve`,
// pymrst/modules/incomp/incomp_tpfa.py:172-184, which calls SuperLU).
//
// The matrix pattern is fixed at creation; values are refreshed by setup.
// The AMG hierarchy (pairwise aggregation, Chebyshev smoothing applied
// identically before and after the coarse correction, dense coarsest solve)
// is a symmetric preconditioner, as CG needs.
#include <cmath>
#include <memory>

#include "pmb_amg.cuh"

namespace pmb {

constexpr int kPcgBlocks = 2 * kNumSM;

__global__ void __launch_bounds__(256) pcg_spmv_kernel(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                                                       const double* __restrict__ a, const double* __restrict__ x,
                                                       double* __restrict__ y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s = 0.0;
  for (int k = rp[i]; k < rp[i + 1]; ++k) s += a[k] * x[ci[k]];
  y[i] = s;
}

__global__ void __launch_bounds__(256) pcg_dot_kernel(int n, const double* __restrict__ a, const double* __restrict__ b,
                                                      double* __restrict__ part) {
  __shared__ double sh[32];
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s += a[i] * b[i];
  s = block_sum(s, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void pcg_sum_kernel(int G, const double* __restrict__ part, double* __restrict__ out) {
  if (threadIdx.x != 0) return;
  double s = 0.0;
  for (int b = 0; b < G; ++b) s += part[b];
  out[0] = s;
}

// x += alpha p; r -= alpha q with alpha = rz / pq (device scalars)
__global__ void pcg_update_xr_kernel(int n, const double* __restrict__ rz, const double* __restrict__ pq,
                                     const double* __restrict__ p, const double* __restrict__ q,
                                     double* __restrict__ x, double* __restrict__ r) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double alpha = pq[0] != 0.0 ? rz[0] / pq[0] : 0.0;
  x[i] += alpha * p[i];
  r[i] -= alpha * q[i];
}

// p = z + beta p with beta = rz_new / rz_old
__global__ void pcg_update_p_kernel(int n, const double* __restrict__ rz_new, const double* __restrict__ rz_old,
                                    const double* __restrict__ z, double* __restrict__ p) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double beta = rz_old[0] != 0.0 ? rz_new[0] / rz_old[0] : 0.0;
  p[i] = z[i] + beta * p[i];
}

__global__ void pcg_copy_kernel(int n, const double* __restrict__ a, double* __restrict__ b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = a[i];
}

class ScalarPCG {
 public:
  ScalarPCG(int n, const int* h_rp, const int* h_ci, cudaStream_t s, double theta, int coarse)
      : n_(n), s_(s), theta_(theta), coarse_(coarse) {
    PMB_REQUIRE(n > 0, "empty system");
    h_rp_.assign(h_rp, h_rp + n + 1);
    h_ci_.assign(h_ci, h_ci + h_rp[n]);
    for (int i = 0; i < n; ++i)
      for (int k = h_rp[i]; k < h_rp[i + 1]; ++k)
        PMB_REQUIRE(h_ci[k] >= 0 && h_ci[k] < n, "column index out of range");
    rp_.upload(h_rp_, s);
    ci_.upload(h_ci_, s);
    val_.resize(h_ci_.size());
    r_.resize(n); z_.resize(n); p_.resize(n); q_.resize(n);
    part_.resize(kPcgBlocks);
    sc_.resize(4);
    status_.resize(1);
    status_.zero(s);
    pin_.resize(4);
    PMB_CUDA(cudaStreamSynchronize(s));
  }
  void setup(const double* d_vals) {
    PMB_CUDA(cudaMemcpyAsync(val_.get(), d_vals, sizeof(double) * h_ci_.size(), cudaMemcpyDeviceToDevice, s_));
    if (!amg_.built()) {
      std::vector<double> hv(h_ci_.size());
      PMB_CUDA(cudaMemcpyAsync(hv.data(), d_vals, sizeof(double) * hv.size(), cudaMemcpyDeviceToHost, s_));
      PMB_CUDA(cudaStreamSynchronize(s_));
      amg_.build(n_, h_rp_, h_ci_, rp_.get(), ci_.get(), hv, theta_, coarse_, s_);
    }
    PMB_CUDA(cudaMemcpyAsync(amg_.level0_val(), d_vals, sizeof(double) * h_ci_.size(), cudaMemcpyDeviceToDevice, s_));
    amg_.refresh(s_, status_.get());
  }
  // info = [iterations, relres, ok]
  bool solve(const double* b, double* x, double rtol, int maxiter, double* info) {
    const int g = grid_for(n_, 256);
    double* rz = sc_.get();       // r.z
    double* pq = sc_.get() + 1;   // p.q
    double* rz2 = sc_.get() + 2;  // new r.z
    double* rr = sc_.get() + 3;   // r.r
    PMB_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * n_, s_));
    pcg_copy_kernel<<<g, 256, 0, s_>>>(n_, b, r_.get());
    PMB_CHECK_LAUNCH();
    const double bnorm = std::sqrt(dot(r_.get(), r_.get(), rr, true));
    info[0] = 0; info[1] = 0; info[2] = 1;
    if (!std::isfinite(bnorm)) throw Error(PMB_ERR_NONFINITE, "non-finite right-hand side");
    if (bnorm == 0.0) return true;
    amg_.apply(r_.get(), z_.get(), s_);
    pcg_copy_kernel<<<g, 256, 0, s_>>>(n_, z_.get(), p_.get());
    PMB_CHECK_LAUNCH();
    dot(r_.get(), z_.get(), rz, false);
    double res = bnorm;
    int it = 0;
    while (it < maxiter) {
      pcg_spmv_kernel<<<g, 256, 0, s_>>>(n_, rp_.get(), ci_.get(), val_.get(), p_.get(), q_.get());
      PMB_CHECK_LAUNCH();
      dot(p_.get(), q_.get(), pq, false);
      pcg_update_xr_kernel<<<g, 256, 0, s_>>>(n_, rz, pq, p_.get(), q_.get(), x, r_.get());
      PMB_CHECK_LAUNCH();
      ++it;
      res = std::sqrt(dot(r_.get(), r_.get(), rr, true));
      if (!std::isfinite(res)) throw Error(PMB_ERR_NONFINITE, "non-finite residual in PCG");
      if (res <= rtol * bnorm) break;
      amg_.apply(r_.get(), z_.get(), s_);
      dot(r_.get(), z_.get(), rz2, false);
      pcg_update_p_kernel<<<g, 256, 0, s_>>>(n_, rz2, rz, z_.get(), p_.get());
      PMB_CHECK_LAUNCH();
      PMB_CUDA(cudaMemcpyAsync(rz, rz2, sizeof(double), cudaMemcpyDeviceToDevice, s_));
    }
    info[0] = it;
    info[1] = res / bnorm;
    info[2] = res <= rtol * bnorm ? 1 : 0;
    return info[2] != 0.0;
  }
  int levels(int64_t* sizes, int maxl) const {
    const int nl = amg_.num_levels();
    for (int l = 0; l < nl && l < maxl; ++l) sizes[l] = amg_.level_size(l);
    return nl;
  }

 private:
  double dot(const double* a, const double* b, double* out, bool fetch) {
    pcg_dot_kernel<<<kPcgBlocks, 256, 0, s_>>>(n_, a, b, part_.get());
    PMB_CHECK_LAUNCH();
    pcg_sum_kernel<<<1, 32, 0, s_>>>(kPcgBlocks, part_.get(), out);
    PMB_CHECK_LAUNCH();
    if (!fetch) return 0.0;
    PMB_CUDA(cudaMemcpyAsync(pin_.get(), out, sizeof(double), cudaMemcpyDeviceToHost, s_));
    PMB_CUDA(cudaStreamSynchronize(s_));
    return pin_[0];
  }
  int n_;
  cudaStream_t s_;
  double theta_;
  int coarse_;
  std::vector<int> h_rp_, h_ci_;
  DArray<int> rp_, ci_;
  DArray<double> val_, r_, z_, p_, q_, part_, sc_;
  DArray<int> status_;
  PinnedArray<double> pin_;
  AMG<double> amg_;
};

// Handle used by the incompressible TPFA path (tpfa.cu), which owns one
// pressure solver per grid and well set.
struct ScalarPCGHandle {
  std::unique_ptr<ScalarPCG> s;
};

ScalarPCGHandle* make_scalar_pcg(int n, const int* h_rp, const int* h_ci, cudaStream_t s, double theta,
                                 int coarse) {
  auto h = std::make_unique<ScalarPCGHandle>();
  h->s = std::make_unique<ScalarPCG>(n, h_rp, h_ci, s, theta, coarse);
  return h.release();
}
void destroy_scalar_pcg(ScalarPCGHandle* p) { delete p; }
void scalar_pcg_setup(ScalarPCGHandle* p, const double* d_vals) { p->s->setup(d_vals); }
bool scalar_pcg_solve(ScalarPCGHandle* p, const double* b, double* x, double rtol, int maxiter, double* info) {
  return p->s->solve(b, x, rtol, maxiter, info);
}
int scalar_pcg_levels(const ScalarPCGHandle* p, int64_t* sizes, int maxl) { return p->s->levels(sizes, maxl); }

}  // namespace pmb

using namespace pmb;

struct pmb_pcg {
  std::unique_ptr<ScalarPCG> s;
};

extern "C" {

int pmb_pcg_create(int32_t n, const int32_t* h_row_ptr, const int32_t* h_col, double amg_theta,
                   int32_t amg_coarse_size, void* stream, pmb_pcg** out) {
  return guarded([&] {
    PMB_REQUIRE(h_row_ptr && h_col && out, "NULL argument");
    *out = nullptr;
    auto p = std::make_unique<pmb_pcg>();
    p->s = std::make_unique<ScalarPCG>(n, h_row_ptr, h_col, (cudaStream_t)stream, amg_theta,
                                       std::max(16, amg_coarse_size));
    *out = p.release();
  });
}

int pmb_pcg_destroy(pmb_pcg* p) {
  return guarded([&] { delete p; });
}

int pmb_pcg_setup(pmb_pcg* p, const double* d_vals) {
  return guarded([&] {
    PMB_REQUIRE(p && d_vals, "NULL argument");
    p->s->setup(d_vals);
  });
}

int pmb_pcg_solve(pmb_pcg* p, const double* d_b, double* d_x, double rtol, int32_t maxiter, double* h_info3) {
  return guarded([&] {
    PMB_REQUIRE(p && d_b && d_x && h_info3, "NULL argument");
    PMB_REQUIRE(d_b != d_x, "b and x must not alias");
    if (!p->s->solve(d_b, d_x, rtol, maxiter, h_info3))
      throw Error(PMB_ERR_NOCONV, "PCG did not reach its tolerance (relres " + std::to_string(h_info3[1]) + ")");
  });
}

int pmb_pcg_levels(const pmb_pcg* p, int32_t max_levels, int64_t* h_sizes, int32_t* n_levels) {
  return guarded([&] {
    PMB_REQUIRE(p && h_sizes && n_levels, "NULL argument");
    *n_levels = p->s->levels(h_sizes, max_levels);
  });
}

}  // extern "C"
