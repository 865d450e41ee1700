// Allocation-free variant of the oil-water convergence reduction.
//
// For callers that cannot allocate device memory at the point where they
// need the check: code running inside another framework's memory pool or
// allocator hooks, a host that has reserved the device for its own
// allocator, or a real-time loop where cudaMalloc's implicit synchronisation
// is not allowed.  They pass their own inputs and output; the per-block
// partial sums live in a fixed device array compiled into this library.
#include <cstdint>
#include <mutex>

#include "pmb_common.cuh"

namespace pmb {

// Cells reduced by one block: 256 threads x 8 cells.
constexpr int kNaCellsPerBlock = 2048;
// Largest grid the static scratch holds: 8192 blocks, so up to
// 8192 * 2048 = 16,777,216 cells.
constexpr int kNaMaxBlocks = 8192;
constexpr int kNaVals = 7;
constexpr long long kNaMaxCells = (long long)kNaMaxBlocks * kNaCellsPerBlock;

// 8192 blocks x 7 doubles = 458,752 bytes, resident on every device that
// loads this library until the process exits.  Every call overwrites the
// slots it later reads, so nothing has to start at zero; calls whose kernels
// overlap on the GPU (other streams, other threads) share this array and race.
static __device__ __align__(256) double g_noalloc_partials[kNaMaxBlocks * kNaVals];

__device__ __forceinline__ double na_b(double c, double b0, double p_ref, double p) {
  return c == 0.0 ? b0 : b0 * exp(c * (p - p_ref));
}

__global__ void __launch_bounds__(256) na_partial_kernel(int nc, const double2* __restrict__ res,
                                                         const double2* __restrict__ x,
                                                         const double* __restrict__ pv, double cw, double co,
                                                         double b0w, double b0o, double p_ref,
                                                         double* __restrict__ part) {
  __shared__ double sh[32];
  double mw = 0, mo = 0, sw = 0, so = 0, iw = 0, io = 0, bad = 0;
  const long long c0 = (long long)blockIdx.x * kNaCellsPerBlock;
  const long long c1 = min((long long)nc, c0 + kNaCellsPerBlock);
  for (long long c = c0 + threadIdx.x; c < c1; c += blockDim.x) {
    const double2 r = res[c];
    const double v = pv[c];
    const double aw = fabs(r.x / v), ao = fabs(r.y / v);
    if (!(isfinite(aw) && isfinite(ao))) bad += 1.0;
    mw = fmax(mw, aw);
    mo = fmax(mo, ao);
    sw += r.x;
    so += r.y;
    const double p = x[c].x;
    iw += 1.0 / na_b(cw, b0w, p_ref, p);
    io += 1.0 / na_b(co, b0o, p_ref, p);
  }
  const double bmw = block_max(mw, sh), bmo = block_max(mo, sh);
  const double bsw = block_sum(sw, sh), bso = block_sum(so, sh);
  const double biw = block_sum(iw, sh), bio = block_sum(io, sh), bbad = block_sum(bad, sh);
  if (threadIdx.x == 0) {
    double* o = part + (long long)kNaVals * blockIdx.x;
    o[0] = bmw; o[1] = bmo; o[2] = bsw; o[3] = bso; o[4] = biw; o[5] = bio; o[6] = bbad;
  }
}

__global__ void __launch_bounds__(256) na_final_kernel(int nc, int nblocks, const double* __restrict__ part,
                                                       double dt, double pv_tot, double* __restrict__ out) {
  __shared__ double sh[32];
  double mw = 0, mo = 0, sw = 0, so = 0, iw = 0, io = 0, bad = 0;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
    const double* o = part + (long long)kNaVals * b;
    mw = fmax(mw, o[0]); mo = fmax(mo, o[1]);
    sw += o[2]; so += o[3]; iw += o[4]; io += o[5]; bad += o[6];
  }
  mw = block_max(mw, sh); mo = block_max(mo, sh);
  sw = block_sum(sw, sh); so = block_sum(so, sh);
  iw = block_sum(iw, sh); io = block_sum(io, sh); bad = block_sum(bad, sh);
  if (threadIdx.x == 0) {
    const double bw = iw / nc, bo = io / nc;
    out[0] = fmax(bw * dt * mw, bo * dt * mo);
    out[1] = fmax(bw * dt * fabs(sw) / pv_tot, bo * dt * fabs(so) / pv_tot);
    out[2] = bad;
    out[3] = 0.0;
  }
}

// Device address of the scratch array, looked up once per device (the
// array's name in host code is only a stand-in for the symbol).  The address
// is cached for the life of the process, so the entry point must not be used
// on a device after cudaDeviceReset() of that device in the same process.
static double* scratch_address(int device) {
  constexpr int kMaxDevices = 64;
  static std::mutex mu;
  static double* addr[kMaxDevices] = {};
  PMB_REQUIRE(device >= 0 && device < kMaxDevices, "device ordinal out of range");
  std::lock_guard<std::mutex> g(mu);
  if (!addr[device]) {
    void* p = nullptr;
    PMB_CUDA(cudaGetSymbolAddress(&p, g_noalloc_partials));
    addr[device] = static_cast<double*>(p);
  }
  return addr[device];
}

}  // namespace pmb

using namespace pmb;

extern "C" int pmb_ow_cnv_mb_noalloc(int32_t nc, const double* d_res, const double* d_x, const double* d_pv,
                                     double pv_total, const double* h_fluid5, double dt, double* d_out4,
                                     void* stream) {
  return guarded([&] {
    PMB_REQUIRE(nc > 0, "nc must be positive");
    PMB_REQUIRE((long long)nc <= kNaMaxCells,
                "nc = " + std::to_string(nc) + " exceeds the " + std::to_string(kNaMaxCells) +
                    " cells the allocation-free scratch holds; use pmb_ow_convergence");
    PMB_REQUIRE(d_res && d_x && d_pv && h_fluid5 && d_out4, "NULL argument");
    PMB_REQUIRE(reinterpret_cast<uintptr_t>(d_res) % 16 == 0 && reinterpret_cast<uintptr_t>(d_x) % 16 == 0,
                "res and x must be 16-byte aligned");
    PMB_REQUIRE(reinterpret_cast<uintptr_t>(d_pv) % 8 == 0 && reinterpret_cast<uintptr_t>(d_out4) % 8 == 0,
                "pv and out must be 8-byte aligned");
    PMB_REQUIRE(dt > 0.0 && pv_total > 0.0, "dt and pv_total must be positive");
    int dev = 0;
    PMB_CUDA(cudaGetDevice(&dev));
    double* part = scratch_address(dev);
    const int nblocks = (int)((nc + kNaCellsPerBlock - 1) / kNaCellsPerBlock);
    cudaStream_t s = (cudaStream_t)stream;
    na_partial_kernel<<<nblocks, 256, 0, s>>>(nc, reinterpret_cast<const double2*>(d_res),
                                              reinterpret_cast<const double2*>(d_x), d_pv, h_fluid5[0],
                                              h_fluid5[1], h_fluid5[2], h_fluid5[3], h_fluid5[4], part);
    PMB_CHECK_LAUNCH();
    na_final_kernel<<<1, 256, 0, s>>>(nc, nblocks, part, dt, pv_total, d_out4);
    PMB_CHECK_LAUNCH();
  });
}
