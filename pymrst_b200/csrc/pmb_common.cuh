// Shared infrastructure for the pymrst_b200 CUDA library: status codes,
// error capture, device buffers, deterministic reductions.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/pymrst_b200.h"

namespace pmb {

// Last error message of the calling host thread (read by pmb_last_error()).
void set_error(const std::string& msg);

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define PMB_CUDA(call)                                                                          \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess)                                                                      \
      throw ::pmb::Error(PMB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_) +   \
                                           " (" + __FILE__ + ":" + std::to_string(__LINE__) + ")"); \
  } while (0)

// Every kernel launch in this library is followed by exactly one
// PMB_CHECK_LAUNCH(), which also counts it (pmb_launch_count).
void count_launch(long long n = 1);
long long launch_count();

// Optional phase timing (environment PMB_PROFILE=1): CUDA events bracket a
// named phase on a stream; elapsed times are collected when the host next
// synchronises and reported by pmb_profile_report.
class PhaseTimer {
 public:
  PhaseTimer(const char* name, cudaStream_t s);
  ~PhaseTimer();
  static bool enabled();

 private:
  const char* name_;
  cudaStream_t s_;
  cudaEvent_t e0_ = nullptr;
};

#define PMB_CHECK_LAUNCH()          \
  do {                              \
    ::pmb::count_launch();          \
    PMB_CUDA(cudaGetLastError());   \
  } while (0)

#define PMB_REQUIRE(cond, msg)                                        \
  do {                                                                \
    if (!(cond)) throw ::pmb::Error(PMB_ERR_ARG, std::string(msg));   \
  } while (0)

// Run `body` and turn exceptions into status codes at the C-ABI boundary.
template <class F>
int guarded(F&& body) {
  try {
    body();
    return PMB_OK;
  } catch (const Error& e) {
    set_error(e.what());
    return e.code;
  } catch (const std::bad_alloc&) {
    set_error("host allocation failed");
    return PMB_ERR_ALLOC;
  } catch (const std::exception& e) {
    set_error(e.what());
    return PMB_ERR_INTERNAL;
  }
}

// Owning device array (cudaMalloc / cudaFree).
template <class T>
class DArray {
 public:
  DArray() = default;
  explicit DArray(size_t n) { resize(n); }
  DArray(const DArray&) = delete;
  DArray& operator=(const DArray&) = delete;
  DArray(DArray&& o) noexcept : p_(o.p_), n_(o.n_) { o.p_ = nullptr; o.n_ = 0; }
  DArray& operator=(DArray&& o) noexcept {
    if (this != &o) { release(); p_ = o.p_; n_ = o.n_; o.p_ = nullptr; o.n_ = 0; }
    return *this;
  }
  ~DArray() { release(); }
  void resize(size_t n) {
    release();
    if (n) {
      cudaError_t e = cudaMalloc(&p_, n * sizeof(T));
      if (e != cudaSuccess) {
        p_ = nullptr;
        throw Error(PMB_ERR_ALLOC, std::string("cudaMalloc of ") + std::to_string(n * sizeof(T)) +
                                       " bytes failed: " + cudaGetErrorString(e));
      }
    }
    n_ = n;
  }
  void upload(const T* h, size_t n, cudaStream_t s) {
    if (n != n_) resize(n);
    if (n) PMB_CUDA(cudaMemcpyAsync(p_, h, n * sizeof(T), cudaMemcpyHostToDevice, s));
  }
  void upload(const std::vector<T>& h, cudaStream_t s) { upload(h.data(), h.size(), s); }
  void zero(cudaStream_t s) { if (n_) PMB_CUDA(cudaMemsetAsync(p_, 0, n_ * sizeof(T), s)); }
  T* get() const { return p_; }
  size_t size() const { return n_; }
  size_t bytes() const { return n_ * sizeof(T); }

 private:
  void release() { if (p_) cudaFree(p_); p_ = nullptr; n_ = 0; }
  T* p_ = nullptr;
  size_t n_ = 0;
};

// Pinned host staging buffer.
template <class T>
class PinnedArray {
 public:
  PinnedArray() = default;
  explicit PinnedArray(size_t n) { resize(n); }
  PinnedArray(const PinnedArray&) = delete;
  PinnedArray& operator=(const PinnedArray&) = delete;
  ~PinnedArray() { if (p_) cudaFreeHost(p_); }
  void resize(size_t n) {
    if (p_) cudaFreeHost(p_);
    p_ = nullptr;
    if (n) PMB_CUDA(cudaMallocHost(&p_, n * sizeof(T)));
    n_ = n;
  }
  T* get() const { return p_; }
  T& operator[](size_t i) { return p_[i]; }
  size_t size() const { return n_; }

 private:
  T* p_ = nullptr;
  size_t n_ = 0;
};

constexpr int kNumSM = 148;

// Programmatic dependent launch (sm_90+).  A kernel launched by launch_pdl
// may be scheduled while its predecessor on the stream is still draining;
// pdl_enter(), its first statement, waits until the predecessor grid has
// completed and its memory is visible, then lets the successor be scheduled.
// So only the launch latency overlaps, never the data.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

bool pdl_enabled();  // false when the environment has PMB_NO_PDL=1

template <class... KArgs, class... Args>
void launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = pdl_enabled() ? 1 : 0;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  PMB_CUDA(cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...));
  count_launch();
  PMB_CUDA(cudaGetLastError());
}

inline int grid_for(long long n, int block) {
  long long g = (n + block - 1) / block;
  if (g < 1) g = 1;
  if (g > 2147483647LL) g = 2147483647LL;
  return static_cast<int>(g);
}

// ---- device helpers --------------------------------------------------------

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Block-wide sum with a fixed tree (deterministic); all threads get the
// result.  `sh` needs blockDim.x/32 slots.
template <class T>
__device__ T block_sum(T v, T* sh) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  T t = (threadIdx.x < nw) ? sh[threadIdx.x] : T(0);
  if (wid == 0) t = warp_sum(t);
  if (threadIdx.x == 0) sh[0] = t;
  __syncthreads();
  T r = sh[0];
  __syncthreads();
  return r;
}

__device__ __forceinline__ double block_max(double v, double* sh) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_max(v);
  __syncthreads();
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double t = (threadIdx.x < nw) ? sh[threadIdx.x] : 0.0;
  if (wid == 0) t = warp_max(t);
  if (threadIdx.x == 0) sh[0] = t;
  __syncthreads();
  double r = sh[0];
  __syncthreads();
  return r;
}

}  // namespace pmb
