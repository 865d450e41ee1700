// Oil-water model: device data layout and the host class owning it.
#pragma once

#include "pmb_common.cuh"

namespace pmb {

struct FluidDev {
  double mu_inv[2], rhoS[2], n[2], c[2], b0[2], sl[2], inv_range[2], p_ref;
  int plain[2];  // kr = s^n without end-point scaling
};

// Well part of the Jacobian, one contiguous buffer of doubles:
//   Bp[nperf][2][3]  d(cell rows water, oil of the perforated cell) / d(qWs, qOs, bhp)
//   Cp[nperf][2][2]  d(eq_w, eq_o) / d(p, sW of the perforated cell)
//   Up[nperf][2][2]  cell rows of perf i  <-  mixture (mix_w, mix_o) of its well
//   Vp[nperf][2][2]  d(mix_w, mix_o) / d(p, sW of perf cell j)
//   D [nw][3][3]     well rows / well unknowns
//   M [nw]           1.0 where the mixture coupling is active (not a dead well)
// The cell-cell coupling through the mixture, d cell_i / d cell_j = Up_i Vp_j
// for perforations i, j of one well, is kept in this rank-2 form.
struct WellLayout {
  int64_t B, C, U, V, D, M, total;
  static WellLayout make(int nperf, int nw) {
    WellLayout l;
    l.B = 0;
    l.C = l.B + 6LL * nperf;
    l.U = l.C + 4LL * nperf;
    l.V = l.U + 4LL * nperf;
    l.D = l.V + 4LL * nperf;
    l.M = l.D + 9LL * nw;
    l.total = l.M + nw;
    return l;
  }
};

// Read-only view passed to kernels by value.
struct OWView {
  int nc, nf, nw, nperf;
  const int* row_ptr;    // nc+1
  const int* col;        // nnzb
  const int* nz_face;    // nnzb: f if the row cell is N[f,0], -(f+1) if N[f,1]; diagonal: INT_MIN
  const int* diag_pos;   // nc
  const double* T;       // nf
  const double* gdz;     // nf
  const double* pv;      // nc
  FluidDev fl;
  // wells
  const int* perf_ptr;   // nw+1
  const int* perf_cell;  // nperf
  const double* perf_WI;
  const int* well_type;  // 0 bhp, 1 rate
  const double* well_val;
  const double* compi;   // nw*2
  const double* perf_dZ;
  const int* perf_well;  // nperf
  // perforated cells: unique cells pcell[0..npc), perfs of pcell q are
  // pc_perf[pc_ptr[q] .. pc_ptr[q+1])
  int npc;
  const int* pcell;
  const int* pc_ptr;
  const int* pc_perf;
  const int* cell_pc;    // nc: index into pcell, or -1
  WellLayout wl;
  double gravity;
  double q_ref;
  double tol_cnv, tol_mb, tol_well, ds_max, dp_max_rel;
};

class OWModel {
 public:
  OWModel(const pmb_ow_desc& d, cudaStream_t s);
  OWView view() const { return v_; }
  cudaStream_t stream() const { return stream_; }
  int nc() const { return v_.nc; }
  int nw() const { return v_.nw; }
  int nperf() const { return v_.nperf; }
  int64_t nnzb() const { return nnzb_; }
  int64_t nvec() const { return 2LL * v_.nc + 3LL * v_.nw; }
  int ncolors() const { return ncolors_; }
  const std::vector<int>& h_row_ptr() const { return h_row_ptr_; }
  const std::vector<int>& h_col() const { return h_col_; }
  const std::vector<int>& h_color_ptr() const { return h_color_ptr_; }
  const int* color_cells() const { return color_cells_.get(); }
  // Vertical lines: cells of line L are line_cells[line_ptr[L] .. line_ptr[L+1])
  // top to bottom; line_lo / line_up give, per line position, the block-CSR
  // index of the coupling to the previous / next cell of the line (-1 at the
  // ends).  Lines are coloured so that lines of one colour never touch.
  struct Lines {
    int nlines = 0, max_len = 0;
    std::vector<int> h_color_ptr;  // per colour: range in color_lines
    DArray<int> line_ptr, line_cells, line_lo, line_up, color_lines;
    DArray<int2> color_range;  // per entry of color_lines: (line_ptr, length) of that line
  };
  const Lines& lines() const { return lines_; }
  bool has_lines() const { return lines_.nlines > 0 && lines_.max_len > 1; }

  void compute_cdp(const double* x0, double* cdp);
  void reset_cdp() { have_last_cdp_ = false; }
  // New well targets (bhp or total rate per well), and the rate scale of
  // the well convergence test that depends on them.
  void set_well_values(const double* h_val);
  // A batch of independent models stored as one (member m: cells
  // [cell_ptr[m], cell_ptr[m+1]), wells [well_ptr[m], well_ptr[m+1]), device
  // arrays): the convergence values of each member (8 per member, the layout
  // of convergence_async), and zeroing the entries of members whose flag is 0.
  void member_convergence_async(int nmem, const int* cell_ptr, const int* well_ptr, const double* res,
                                const double* x, double dt, double* d_out);
  void mask_members(int nmem, const int* cell_ptr, const int* well_ptr, const int* flag, double* vec);
  // Per member squared norms [||b - J dx||^2, ||b||^2] of a shared linear
  // solve (J the current Jacobian; tmp an nvec scratch vector).
  void member_linear_residuals_async(int nmem, const int* cell_ptr, const int* well_ptr, const double* b,
                                     const double* dx, double* tmp, double* d_out);
  // Phase fluxes of every interface (what face f adds to the rows of N[f,0]
  // and subtracts from those of N[f,1]) and every perforation's surface
  // rates (what it subtracts from its cell's rows and its well's rate rows)
  // at state x; uses the model's residual workspace.
  void fluxes(const double* x, const double* cdp, double* face_flux, double* perf_rate);
  void assemble(const double* x, const double* x0, double dt, const double* cdp, double* res,
                double* jac, double* well, bool want_jac);
  void spmv(const double* jac, const double* well, const double* x, double* y);
  // Device-side convergence values into d_out (8 doubles); no sync.
  void convergence_async(const double* res, const double* x, double dt, double* d_out);
  // x += sgn * dx with the reference update limits
  void update(double* x, const double* dx, double sgn = 1.0);

  // Adjoint support (adjoint.cu).  y = (dR_{n+1}/dx_n)^T lam for the
  // accumulation terms, the only ones that see the previous state, with
  // x_prev the state x_n (cell-major) and dt the step n+1; lam and y in the
  // variable-blocked layout [p, sW, qWs, qOs, bhp] (y's well entries 0).
  void prev_jacobian_tmul(const double* x_prev, double dt, const double* lam, double* y);
  // Values of a CSR matrix each of whose entries e is the sum, over the
  // terms ptr[e] .. ptr[e+1]-1, of one Jacobian entry (term t >= 0: jac[t]
  // for t < 4 nnzb, else well[t - 4 nnzb]) or one entry of a cross-flow
  // mixture product (t < 0: code -1 - t = ((i nperf + j) 4 + 2a + b), entry
  // (a, b) of Up_i Vp_j, counted where the well's mixture coupling is on).
  void csr_values(const double* jac, const double* well, int64_t n, const int64_t* ptr, const int64_t* terms,
                  double* vals);
  // out[c] += lam^T dR/d(log k_c) at state x (cdp = 0): through the
  // interface transmissibilities (dT_f/dlog k_c = T_f^2 / t_{c,f}, t0 / t1
  // the half-face T of N[f,0] / N[f,1]) and the well indices of the
  // perforations of c; face_flux (2 nf) and perf_rate (2 nperf) are scratch.
  void perm_contract(const double* x, const double* lam, const double* t0, const double* t1, double* face_flux,
                     double* perf_rate, double* out);
  // The previous timestep's well pressure drops, kept for the next
  // compute_cdp (nperf values; *have = 0 when there are none).
  void get_last_cdp(double* out, int* have);
  void set_last_cdp(const double* in);

  // internal buffers
  double* jac() { return jac_.get(); }
  double* well() { return well_.get(); }
  double* res() { return res_.get(); }
  double* cdp() { return cdp_.get(); }
  double* x0() { return x0_.get(); }
  double* dx() { return dx_.get(); }
  double* conv_out() { return conv_out_.get(); }

 private:
  cudaStream_t stream_;
  OWView v_{};
  int64_t nnzb_ = 0;
  int ncolors_ = 0;
  std::vector<int> h_row_ptr_, h_col_, h_color_ptr_;
  DArray<int> row_ptr_, col_, nz_face_, diag_pos_, perf_ptr_, perf_cell_, well_type_, perf_well_;
  DArray<int> pcell_, pc_ptr_, pc_perf_, color_cells_, cell_pc_;
  DArray<double> T_, gdz_, pv_, perf_WI_, perf_dZ_, well_val_, compi_;
  std::vector<int> h_well_type_;
  // scratch / state
  DArray<double> pf_cq_, pf_dloc_, last_cdp_, conv_part_, conv_out_, cdp_zero_;
  DArray<double> jac_, well_, res_, cdp_, x0_, dx_;
  bool have_last_cdp_ = false;
  double pv_tot_ = 0.0;
  Lines lines_;
  void build_lines(const pmb_ow_desc& d, const std::vector<int>& code);
};

}  // namespace pmb
