// CPR-preconditioned flexible GMRES on the oil-water operator.
#pragma once

#include "pmb_amg.cuh"
#include "pmb_krylov.cuh"
#include "pmb_ow.cuh"

namespace pmb {

class CPRSolver {
 public:
  CPRSolver(OWModel& m, const pmb_cpr_opts& o);
  void setup(const double* jac, const double* well, const double* x);
  // Returns true when converged; info = [iterations, relres, ok, setups].
  bool solve(const double* b, double* x, double* info);
  const pmb_cpr_opts& opts() const { return o_; }
  int num_levels() const { return f32_ ? amg32_.num_levels() : amg_.num_levels(); }
  int level_size(int l) const { return f32_ ? amg32_.level_size(l) : amg_.level_size(l); }
  long long setups() const { return setups_; }
  long long total_iterations() const { return total_its_; }
  // Mean milliseconds of one application of a preconditioner stage (0: the
  // second stage, every sweep; 1: the AMG cycle on the restricted r; 2: the
  // whole preconditioner, not replayed from a graph), by CUDA events on the
  // solver's stream, after one untimed application.
  double time_stage(int stage, const double* r, double* z, int reps);
  // One visit of AMG level l >= 1 (graph replay) and the level's stored entries.
  double time_level(int l, int reps, long long* nnz) {
    PMB_REQUIRE(o_.use_pressure_stage, "the pressure stage is switched off");
    if (f32_) {
      *nnz = amg32_.level_nnz(l);
      return amg32_.time_visit(l, reps, s_);
    }
    *nnz = amg_.level_nnz(l);
    return amg_.time_visit(l, reps, s_);
  }
  // Algorithmic bytes (every array read or written once per launch, storage
  // types): [AMG cycle, one second-stage sweep, operator product, pressure
  // restriction + prolongation of one application, one setup without
  // aggregation, FGMRES vector length, AMG refresh, 0].
  void bytes(double* out) const;

 private:
  void precond(const double* r, double* z);
  void precond_body(const double* r, double* z);
  // entered: rl / zl already hold r and z in line order (ell_ path only)
  void local_stage(const double* r, double* z, bool entered = false);
  // r (and z, or the prolonged pressure correction xp) into line order
  template <class T>
  void enter_lines(const T* xp, const double* r, double* z, bool from_z, bool pw);
  void prepare_local(const double* jac);
  void build_line_ell();
  void check_status();

  OWModel& m_;
  pmb_cpr_opts o_;
  cudaStream_t s_;
  const double* jac_ = nullptr;
  const double* well_ = nullptr;
  Fgmres kry_;
  // The preconditioner replayed as one CUDA graph; re-captured when the
  // hierarchy or the operator buffers change.
  GraphedApply graph_;
  const double* pg_jac_ = nullptr;
  const double* pg_well_ = nullptr;
  AMG<double> amg_;
  // precision 1: the preconditioner works on FP32 copies of the matrices
  // (AMG values and vectors, line-smoother blocks) inside the FP64 FGMRES
  bool f32_ = false;
  AMG<float> amg32_;
  DArray<float> jac32_, bp32_, xp32_;
  int since_build_ = 0;
  long long setups_ = 0, total_its_ = 0;
  DArray<double> w_;        // quasi-IMPES weights (2)
  DArray<double> part_;     // reduction partials
  DArray<int> status_;
  DArray<double> bp_, xp_, ap_;  // pressure system rhs / solution / values for aggregation
  DArray<double> line_y_, line_g_;  // line Gauss-Seidel scratch (per line position)
  // Line-ordered copy of the line smoother's operator (vertical lines of at
  // most 256 cells, at most 12 blocks per row): `slots` blocks per position,
  // slot-major, refreshed from the Jacobian at every setup; the lateral
  // columns as line positions; per position the cell's perforated-cell index;
  // per perforation its cell's position; r and z of the cells in line order.
  struct LineEll {
    int slots = 0;
    DArray<int> src, col, pc, perf_pos;
    DArray<double> blk64, rl, zl;  // rl, zl: r and z in line order (FP64 arithmetic)
    DArray<float> rl32, zl32;       // the same in mixed precision
    DArray<float> blk32;
  } ell_;
  bool use_ell_ = false;
  // Pressure system with one bhp unknown per well (np_ = nc + nw): CSR
  // pattern, the position of every cell block in it (bsr2ext), of each
  // perforation's (cell, well) and (well, cell) entries, and of each well's
  // diagonal; per-perforation and per-well elimination coefficients.
  int np_ = 0;
  std::vector<int> h_erp_, h_ecol_;
  DArray<int> erp_, ecol_, bsr2ext_, perf_cw_, perf_wc_, well_diag_;
  bool ext_par_ = false;  // the pressure system's well entries by a thread per perforation
  DArray<double> g_perf_, a_well_;
  void build_pressure_pattern();
  void pressure_values(double* ext);
  PinnedArray<int> st_pin_;
  std::vector<double> h_ap_;
};

}  // namespace pmb
