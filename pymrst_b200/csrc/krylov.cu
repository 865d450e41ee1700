// Flexible GMRES and preconditioner graph replay (pmb_krylov.cuh).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <vector>

#include "pmb_krylov.cuh"

namespace pmb {

constexpr int kRedBlocks = 4 * kNumSM;
constexpr int kDotChunk = 8;

// Chunked multi-dot: part[i * G + blk] = partial dot(V_i, w) for i < nv and,
// with with_ww, part[nv * G + blk] = partial dot(w, w).  Eight dots share one
// read of w and one block reduction; each block owns one contiguous chunk.
// VEC reads pairs of elements (16-byte loads; V's row stride even, V and w
// 16-byte aligned); an odd last element is added by the last block.
// Skipped (returns at once) when `gate` is given and *gate != run_if.
template <bool VEC>
__global__ void __launch_bounds__(256, 4) mdot8_kernel(long long n, const double* __restrict__ V, long long ld, int nv,
                                                       const double* __restrict__ w, int with_ww,
                                                       double* __restrict__ part, const int* __restrict__ gate,
                                                       int run_if) {
  if (gate && *gate != run_if) return;
  __shared__ double sh[kDotChunk][8];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const long long nu = VEC ? n / 2 : n;
  const long long chunk = (nu + gridDim.x - 1) / gridDim.x;
  const long long e0 = blockIdx.x * chunk;
  const long long e1 = min(nu, e0 + chunk);
  const bool tail = VEC && (n & 1) && blockIdx.x == gridDim.x - 1 && threadIdx.x == 0;
  const int ntot = nv + (with_ww ? 1 : 0);
  for (int i0 = 0; i0 < ntot; i0 += kDotChunk) {
    double acc[kDotChunk];
#pragma unroll
    for (int q = 0; q < kDotChunk; ++q) acc[q] = 0.0;
    for (long long e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
      if (VEC) {
        const double2 we = reinterpret_cast<const double2*>(w)[e];
#pragma unroll
        for (int q = 0; q < kDotChunk; ++q) {
          const int i = i0 + q;
          if (i < nv) {
            const double2 v = reinterpret_cast<const double2*>(V + i * ld)[e];
            acc[q] += v.x * we.x + v.y * we.y;
          } else if (i == nv && with_ww) {
            acc[q] += we.x * we.x + we.y * we.y;
          }
        }
      } else {
        const double we = w[e];
#pragma unroll
        for (int q = 0; q < kDotChunk; ++q) {
          const int i = i0 + q;
          if (i < nv) acc[q] += V[i * ld + e] * we;
          else if (i == nv && with_ww) acc[q] += we * we;
        }
      }
    }
    if (tail) {
      const long long e = n - 1;
      const double we = w[e];
#pragma unroll
      for (int q = 0; q < kDotChunk; ++q) {
        const int i = i0 + q;
        if (i < nv) acc[q] += V[i * ld + e] * we;
        else if (i == nv && with_ww) acc[q] += we * we;
      }
    }
#pragma unroll
    for (int q = 0; q < kDotChunk; ++q) {
      double s = warp_sum(acc[q]);
      if (lane == 0) sh[q][wid] = s;
    }
    __syncthreads();
    if (threadIdx.x < kDotChunk) {
      const int q = threadIdx.x;
      double s = 0.0;
      for (int ww = 0; ww < nwarp; ++ww) s += sh[q][ww];
      if (i0 + q < ntot) part[(long long)(i0 + q) * gridDim.x + blockIdx.x] = s;
    }
    __syncthreads();
  }
}

// Launches mdot8_kernel, with pair loads where the alignment allows them.
static void launch_mdot8(cudaStream_t s, long long n, const double* V, long long ld, int nv, const double* w,
                         int with_ww, double* part, const int* gate, int run_if) {
  const bool vec = ((uintptr_t)w % 16 == 0) && (nv == 0 || ((uintptr_t)V % 16 == 0 && ld % 2 == 0));
  if (vec)
    mdot8_kernel<true><<<kRedBlocks, 256, 0, s>>>(n, V, ld, nv, w, with_ww, part, gate, run_if);
  else
    mdot8_kernel<false><<<kRedBlocks, 256, 0, s>>>(n, V, ld, nv, w, with_ww, part, gate, run_if);
  PMB_CHECK_LAUNCH();
}

// hs[q] = sum_b part[q*G + b] for q < nq (fixed order: lane-strided sums, then
// a fixed warp tree); one warp per value.
__device__ void reduce_partials(int nq, int G, const double* __restrict__ part, double* hs) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  for (int q = warp; q < nq; q += nwarp) {
    double s = 0.0;
    for (int b = lane; b < G; b += 32) s += part[(long long)q * G + b];
    s = warp_sum(s);
    if (lane == 0) hs[q] = s;
  }
  __syncthreads();
}

// After the first projection: h[i] = V_i . w (i < nv); decides whether a second
// pass is needed.  With |w'|^2 = |w|^2 - |h|^2 >= 0.49 |w|^2 the projection
// lost little, *flag = 0 and h[nv] = |w'|; otherwise *flag = 1.
__global__ void __launch_bounds__(256) orth_decide_kernel(int nv, int G, const double* __restrict__ part,
                                                          double* __restrict__ h, int* __restrict__ flag) {
  __shared__ double hs[kMaxRestart + 2];
  reduce_partials(nv + 1, G, part, hs);
  const int i = threadIdx.x;
  if (i < nv) h[i] = hs[i];
  if (i == 0) {
    double proj = 0.0;
    for (int k = 0; k < nv; ++k) proj += hs[k] * hs[k];
    const double ww = hs[nv];
    const double after = ww - proj;
    if (after >= 0.49 * ww && ww > 0.0) {
      *flag = 0;
      h[nv] = sqrt(after);
    } else {
      *flag = 1;
    }
  }
}

// out[i] = sum_b part[i*G+b]; acc[i] += out[i] when given; sqrt of each
// value when do_sqrt.
__global__ void __launch_bounds__(256) mdot_final_kernel(int nv, int G, const double* __restrict__ part,
                                                         double* __restrict__ out, double* __restrict__ acc,
                                                         int do_sqrt, const int* __restrict__ gate = nullptr,
                                                         int run_if = 1) {
  if (gate && *gate != run_if) return;
  __shared__ double hs[kMaxRestart + 2];
  reduce_partials(nv, G, part, hs);
  const int i = threadIdx.x;
  if (i >= nv) return;
  double s = hs[i];
  if (do_sqrt) s = sqrt(s);
  out[i] = s;
  if (acc) acc[i] += s;
}

// w -= sum_i h[i] V_i, subtracting in the order of i.  Each thread takes a
// pair of elements (16-byte loads: V is the basis, its row stride a multiple
// of 32, and w the work vector, both allocated by Fgmres) and issues the
// loads of four vectors before their updates; the thread with global index 0
// also takes an odd last element.
__global__ void __launch_bounds__(256) vupdate_kernel(long long n, const double* __restrict__ V, long long ld,
                                                      int nv, const double* __restrict__ h,
                                                      double* __restrict__ w, const int* __restrict__ gate = nullptr,
                                                      int run_if = 1) {
  if (gate && *gate != run_if) return;
  __shared__ double hs[kMaxRestart + 2];
  for (int i = threadIdx.x; i < nv; i += blockDim.x) hs[i] = h[i];
  __syncthreads();
  const long long nu = n / 2;
  const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  for (long long e = tid; e < nu; e += (long long)gridDim.x * blockDim.x) {
    double2 s = reinterpret_cast<const double2*>(w)[e];
    int i = 0;
    for (; i + 4 <= nv; i += 4) {
      double2 v[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) v[q] = reinterpret_cast<const double2*>(V + (i + q) * ld)[e];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        s.x -= hs[i + q] * v[q].x;
        s.y -= hs[i + q] * v[q].y;
      }
    }
    for (; i < nv; ++i) {
      const double2 v = reinterpret_cast<const double2*>(V + i * ld)[e];
      s.x -= hs[i] * v.x;
      s.y -= hs[i] * v.y;
    }
    reinterpret_cast<double2*>(w)[e] = s;
  }
  if ((n & 1) && tid == 0) {
    const long long e = n - 1;
    double s = w[e];
    for (int i = 0; i < nv; ++i) s -= hs[i] * V[i * ld + e];
    w[e] = s;
  }
}

// x += sum_i y[i] Z_i
__global__ void __launch_bounds__(256) xupdate_kernel(long long n, const double* __restrict__ Z, long long ld,
                                                      int nv, const double* __restrict__ y,
                                                      double* __restrict__ x) {
  __shared__ double ys[kMaxRestart + 2];
  for (int i = threadIdx.x; i < nv; i += blockDim.x) ys[i] = y[i];
  __syncthreads();
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    double s = x[e];
    for (int i = 0; i < nv; ++i) s += ys[i] * Z[i * ld + e];
    x[e] = s;
  }
}

// out = a / s[0]
__global__ void scale_kernel(long long n, const double* __restrict__ a, const double* __restrict__ s,
                             double* __restrict__ out) {
  const double inv = 1.0 / s[0];
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x)
    out[e] = a[e] * inv;
}

// r = b - y
__global__ void sub_kernel(long long n, const double* __restrict__ b, const double* __restrict__ y,
                           double* __restrict__ r) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x)
    r[e] = b[e] - y[e];
}

// ---- Fgmres -------------------------------------------------------------------

void Fgmres::init(long long n, int restart, cudaStream_t s) {
  PMB_REQUIRE(restart >= 1 && restart <= kMaxRestart, "restart must be in 1..60");
  n_ = n;
  m_ = restart;
  s_ = s;
  // Krylov vectors are stored with a stride padded to 32 doubles so that every
  // slice V_j / Z_j stays 256-byte aligned for vector loads.
  ld_ = (n + 31) / 32 * 32;
  V_.resize((size_t)(m_ + 1) * ld_);
  Z_.resize((size_t)m_ * ld_);
  wv_.resize(n);
  r_.resize(n);
  hcol_.resize(m_ + 2);
  htmp_.resize(m_ + 2);
  y_.resize(m_ + 1);
  part_.resize((size_t)kRedBlocks * (m_ + 2));
  flag_.resize(1);
  flag_.zero(s_);
  h_pin_.resize(m_ + 8);
  st_pin_.resize(1);
  st_pin_[0] = 0;
}

double Fgmres::norm(const double* a) {
  launch_mdot8(s_, n_, a, n_, 0, a, 1, part_.get(), nullptr, 0);
  mdot_final_kernel<<<1, 256, 0, s_>>>(1, kRedBlocks, part_.get(), htmp_.get(), nullptr, 1);
  PMB_CHECK_LAUNCH();
  PMB_CUDA(cudaMemcpyAsync(h_pin_.get(), htmp_.get(), sizeof(double), cudaMemcpyDeviceToHost, s_));
  PMB_CUDA(cudaStreamSynchronize(s_));
  return h_pin_[0];
}

bool Fgmres::solve(const Apply& op, const Apply& prec, const double* b, double* x, double rtol, int maxiter,
                   double* info, const int* d_status, const std::function<void()>& on_status) {
  PMB_REQUIRE(maxiter >= 1, "maxiter must be positive");
  PMB_REQUIRE(rtol > 0.0, "rtol must be positive");
  const long long n = n_;
  const int mm = m_;
  const int gv = 4 * kNumSM;
  PMB_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * n, s_));
  const double beta0 = norm(b);
  info[0] = 0; info[1] = 0; info[2] = 1;
  if (!std::isfinite(beta0)) throw Error(PMB_ERR_NONFINITE, "non-finite right-hand side");
  if (beta0 == 0.0) return true;
  const double target = rtol * beta0;
  PMB_CUDA(cudaMemcpyAsync(r_.get(), b, sizeof(double) * n, cudaMemcpyDeviceToDevice, s_));
  double beta = beta0;
  int its = 0;
  std::vector<double> H((size_t)(mm + 1) * mm), cs(mm), sn(mm), g(mm + 1), y(mm);
  bool converged = false;
  while (its < maxiter) {
    h_pin_[0] = beta;
    PMB_CUDA(cudaMemcpyAsync(htmp_.get(), h_pin_.get(), sizeof(double), cudaMemcpyHostToDevice, s_));
    scale_kernel<<<gv, 256, 0, s_>>>(n, r_.get(), htmp_.get(), V_.get());
    PMB_CHECK_LAUNCH();
    std::fill(g.begin(), g.end(), 0.0);
    g[0] = beta;
    int j = 0;
    bool stop = false;
    for (; j < mm && !stop; ++j) {
      double* vj = V_.get() + (size_t)j * ld_;
      double* zj = Z_.get() + (size_t)j * ld_;
      prec(vj, zj);
      op(zj, wv_.get());
      // classical Gram-Schmidt; the second pass (and the separate norm) only
      // when the first projection cancelled most of w, decided on the device
      const int nv = j + 1;
      PhaseTimer pt_orth("gmres.orthogonalise", s_);
      int* flag = flag_.get();
      launch_mdot8(s_, n, V_.get(), ld_, nv, wv_.get(), 1, part_.get(), nullptr, 0);
      orth_decide_kernel<<<1, 256, 0, s_>>>(nv, kRedBlocks, part_.get(), hcol_.get(), flag);
      PMB_CHECK_LAUNCH();
      vupdate_kernel<<<gv, 256, 0, s_>>>(n, V_.get(), ld_, nv, hcol_.get(), wv_.get());
      PMB_CHECK_LAUNCH();
      launch_mdot8(s_, n, V_.get(), ld_, nv, wv_.get(), 0, part_.get(), flag, 1);
      mdot_final_kernel<<<1, 256, 0, s_>>>(nv, kRedBlocks, part_.get(), htmp_.get(), hcol_.get(), 0, flag, 1);
      PMB_CHECK_LAUNCH();
      vupdate_kernel<<<gv, 256, 0, s_>>>(n, V_.get(), ld_, nv, htmp_.get(), wv_.get(), flag, 1);
      PMB_CHECK_LAUNCH();
      launch_mdot8(s_, n, wv_.get(), n, 0, wv_.get(), 1, part_.get(), flag, 1);
      mdot_final_kernel<<<1, 256, 0, s_>>>(1, kRedBlocks, part_.get(), hcol_.get() + nv, nullptr, 1, flag, 1);
      PMB_CHECK_LAUNCH();
      scale_kernel<<<gv, 256, 0, s_>>>(n, wv_.get(), hcol_.get() + nv, V_.get() + (size_t)(j + 1) * ld_);
      PMB_CHECK_LAUNCH();
      PMB_CUDA(cudaMemcpyAsync(h_pin_.get(), hcol_.get(), sizeof(double) * (nv + 1), cudaMemcpyDeviceToHost, s_));
      if (d_status)
        PMB_CUDA(cudaMemcpyAsync(st_pin_.get(), d_status, sizeof(int), cudaMemcpyDeviceToHost, s_));
      PMB_CUDA(cudaStreamSynchronize(s_));
      if (d_status && st_pin_[0] != 0) {
        st_pin_[0] = 0;
        on_status();
      }
      for (int i = 0; i <= nv; ++i) {
        if (!std::isfinite(h_pin_[i])) throw Error(PMB_ERR_NONFINITE, "non-finite Krylov scalar in GMRES");
        H[(size_t)i * mm + j] = h_pin_[i];
      }
      for (int i = 0; i < j; ++i) {
        const double t0 = cs[i] * H[(size_t)i * mm + j] + sn[i] * H[(size_t)(i + 1) * mm + j];
        H[(size_t)(i + 1) * mm + j] = -sn[i] * H[(size_t)i * mm + j] + cs[i] * H[(size_t)(i + 1) * mm + j];
        H[(size_t)i * mm + j] = t0;
      }
      const double a = H[(size_t)j * mm + j], bb = H[(size_t)(j + 1) * mm + j];
      const double den = std::hypot(a, bb);
      cs[j] = den == 0.0 ? 1.0 : a / den;
      sn[j] = den == 0.0 ? 0.0 : bb / den;
      H[(size_t)j * mm + j] = den;
      H[(size_t)(j + 1) * mm + j] = 0.0;
      g[j + 1] = -sn[j] * g[j];
      g[j] = cs[j] * g[j];
      ++its;
      if (std::fabs(g[j + 1]) <= target || its >= maxiter || bb == 0.0) stop = true;
    }
    // y = H^{-1} g (upper triangular, j x j), x += Z y
    for (int i = j - 1; i >= 0; --i) {
      double s = g[i];
      for (int k = i + 1; k < j; ++k) s -= H[(size_t)i * mm + k] * y[k];
      const double d = H[(size_t)i * mm + i];
      y[i] = d == 0.0 ? 0.0 : s / d;
    }
    for (int i = 0; i < j; ++i) h_pin_[i] = y[i];
    PMB_CUDA(cudaMemcpyAsync(y_.get(), h_pin_.get(), sizeof(double) * j, cudaMemcpyHostToDevice, s_));
    xupdate_kernel<<<gv, 256, 0, s_>>>(n, Z_.get(), ld_, j, y_.get(), x);
    PMB_CHECK_LAUNCH();
    // true residual
    op(x, wv_.get());
    sub_kernel<<<gv, 256, 0, s_>>>(n, b, wv_.get(), r_.get());
    PMB_CHECK_LAUNCH();
    beta = norm(r_.get());
    if (!std::isfinite(beta)) throw Error(PMB_ERR_NONFINITE, "non-finite residual in GMRES");
    if (beta <= target) {
      converged = true;
      break;
    }
  }
  info[0] = its;
  info[1] = beta / beta0;
  info[2] = converged ? 1 : 0;
  return converged;
}

// ---- GraphedApply -------------------------------------------------------------

GraphedApply::~GraphedApply() {
  invalidate();
  if (cap_) cudaStreamDestroy(cap_);
}

void GraphedApply::invalidate() {
  if (exec_) cudaGraphExecDestroy(exec_);
  exec_ = nullptr;
}

void GraphedApply::run(long long n, const double* r, double* z, cudaStream_t& s,
                       const std::function<void(const double*, double*)>& body) {
  static const bool use_graph = [] {
    const char* e = std::getenv("PMB_NO_GRAPH");
    return !(e && e[0] == '1');
  }();
  if (!use_graph || !enabled || PhaseTimer::enabled()) {
    body(r, z);
    return;
  }
  if ((long long)in_.size() != n) {
    invalidate();
    in_.resize(n);
    out_.resize(n);
  }
  if (!exec_) {
    if (failures_ >= kMaxCaptureFailures) {
      body(r, z);
      return;
    }
    // capture on a private stream (the legacy default stream cannot be
    // captured); the graph is then launched on the owner's stream
    if (!cap_) PMB_CUDA(cudaStreamCreateWithFlags(&cap_, cudaStreamNonBlocking));
    PMB_CUDA(cudaStreamSynchronize(s));
    const long long before = launch_count();
    const cudaStream_t saved = s;
    s = cap_;
    PMB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
    cudaGraph_t g = nullptr;
    bool captured = true;
    try {
      body(in_.get(), out_.get());
    } catch (const Error& e) {
      // only a CUDA-level failure can come from the capture being disturbed
      // (by other threads' device work); anything else is a real error
      if (e.code != PMB_ERR_CUDA) {
        cudaStreamEndCapture(s, &g);
        if (g) cudaGraphDestroy(g);
        s = saved;
        count_launch(-(launch_count() - before));
        throw;
      }
      captured = false;
    }
    const cudaError_t ce = cudaStreamEndCapture(s, &g);
    s = saved;
    count_launch(-(launch_count() - before));  // captured (or abandoned), not launched
    if (!captured || ce != cudaSuccess || !g) {
      // the capture was invalidated: clear the non-sticky capture error and
      // run this application directly; later calls try to capture again
      if (g) cudaGraphDestroy(g);
      (void)cudaGetLastError();
      ++failures_;
      body(r, z);
      return;
    }
    nodes_ = 0;
    PMB_CUDA(cudaGraphGetNodes(g, nullptr, reinterpret_cast<size_t*>(&nodes_)));
    const cudaError_t e = cudaGraphInstantiate(&exec_, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      exec_ = nullptr;
      (void)cudaGetLastError();
      ++failures_;
      body(r, z);
      return;
    }
  }
  PMB_CUDA(cudaMemcpyAsync(in_.get(), r, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  PMB_CUDA(cudaGraphLaunch(exec_, s));
  count_launch(nodes_);
  PMB_CUDA(cudaMemcpyAsync(z, out_.get(), sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
}

}  // namespace pmb
