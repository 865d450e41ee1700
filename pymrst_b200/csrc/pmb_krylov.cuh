// Restarted flexible GMRES on device vectors, and the CUDA-graph replay of a
// preconditioner.  Shared by the oil-water CPR (block layout of the device
// model) and the CPR on a caller's CSR matrix.
#pragma once

#include <functional>

#include "pmb_common.cuh"

namespace pmb {

constexpr int kMaxRestart = 60;

// Right-preconditioned FGMRES(m) with classical Gram-Schmidt; the second
// Gram-Schmidt pass runs only when the first one cancelled most of the new
// vector, decided on the device.  Host work per iteration: one small D2H
// (the Hessenberg column) and the Givens rotations.  Follows the outer
// iteration of CPRSolver.solve (pymrst/modules/ad_core/solvers/
// linear_solvers.py:519-531): zero initial guess, stop at
// |r| <= rtol |b|, restart, maxiter counted in inner iterations.
class Fgmres {
 public:
  using Apply = std::function<void(const double* in, double* out)>;
  void init(long long n, int restart, cudaStream_t s);
  // x = solution of op(x) = b.  info = [iterations, |r|/|b|, converged].
  // d_status (may be null) is read with every Hessenberg column; a nonzero
  // value calls on_status (which throws).
  bool solve(const Apply& op, const Apply& prec, const double* b, double* x, double rtol, int maxiter,
             double* info, const int* d_status, const std::function<void()>& on_status);
  double norm(const double* v);
  long long n() const { return n_; }

 private:
  long long n_ = 0, ld_ = 0;
  int m_ = 0;
  cudaStream_t s_ = nullptr;
  DArray<double> V_, Z_, wv_, r_, hcol_, htmp_, y_, part_;
  DArray<int> flag_;
  PinnedArray<double> h_pin_;
  PinnedArray<int> st_pin_;
};

// z = body(r) replayed from one captured CUDA graph on fixed staging vectors.
// The body enqueues on the stream variable it is given (`s`), which is
// pointed at a private capture stream while the body is recorded; the graph
// then runs on the owner's stream.  PMB_NO_GRAPH=1, PMB_PROFILE=1 or
// `enabled` false run the body directly, and so does a call whose capture was
// invalidated (device work of other threads can do that); after three such
// failures the graph is no longer attempted.
class GraphedApply {
 public:
  ~GraphedApply();
  void invalidate();
  void run(long long n, const double* r, double* z, cudaStream_t& s,
           const std::function<void(const double*, double*)>& body);
  long long nodes() const { return nodes_; }
  bool enabled = true;  // false: run() always launches the body directly

 private:
  static constexpr int kMaxCaptureFailures = 3;
  cudaGraphExec_t exec_ = nullptr;
  cudaStream_t cap_ = nullptr;
  long long nodes_ = 0;
  int failures_ = 0;  // invalidated captures; after kMaxCaptureFailures the body always runs directly
  DArray<double> in_, out_;
};

}  // namespace pmb
