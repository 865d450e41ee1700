/*
 * pymrst_b200 — C-ABI of the B200 (sm_100a) TPFA flow hot path.
 *
 * Plain pointers and sizes only.  Pointers named d_* are device pointers
 * (e.g. torch.Tensor.data_ptr() of CUDA tensors); h_* are host pointers.
 * `stream` is a cudaStream_t passed as void* (0 = legacy default stream).
 * Every entry point returns an int status (PMB_OK == 0) and never throws;
 * pmb_last_error() gives the message of the last failure on the calling
 * thread.  A handle is bound to the stream it was created with and is not
 * thread-safe; distinct handles are independent.  The caller owns every
 * d_* / h_* buffer it passes; handles own their internal workspaces and
 * release them in the matching *_destroy.
 *
 * Vector layout of the oil-water system ("cell-major"): for cell c,
 * x[2c] = pressure, x[2c+1] = water saturation; then for well k,
 * x[2nc+3k+0] = qWs, +1 = qOs, +2 = bhp.  Residual rows use the same
 * layout: water, oil per cell, then eq_w, eq_o, ctrl per well.  The
 * reference assembles the same system in variable-blocked order
 * (pymrst/utils/adi/operators.py:204-211); the Python layer permutes.
 */
#ifndef PYMRST_B200_H
#define PYMRST_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  PMB_OK = 0,
  PMB_ERR_CUDA = 1,      /* CUDA runtime error */
  PMB_ERR_ARG = 2,       /* invalid argument / unsupported input */
  PMB_ERR_NONFINITE = 3, /* NaN or Inf in a residual, update or Krylov scalar */
  PMB_ERR_PIVOT = 4,     /* zero pivot in a block inverse or coarse solve */
  PMB_ERR_NOCONV = 5,    /* Krylov solver did not reach its tolerance */
  PMB_ERR_ALLOC = 6,     /* device or host allocation failed */
  PMB_ERR_INTERNAL = 7
};

const char* pmb_last_error(void);
int pmb_version(void);
/* Number of kernels this library has launched in the process so far. */
int pmb_launch_count(int64_t* h_out);
/* Phase timings collected when the environment has PMB_PROFILE=1, as text
 * lines "name total_ms count" (synchronises the device). */
int pmb_profile_report(char* h_buf, int32_t len, int32_t reset);

/* ------------------------------------------------------------------------
 * Grid geometry.
 * pmb_compute_geometry3d replaces compute_geometry for 3-D grids
 * (pymrst/gridprocessing/compute_geometry.py:211-325): every face is split
 * into a fan of triangles around its pivot (the mean of its nodes, or row f
 * of d_hinge where that row's x is finite; d_hinge may be NULL), giving its
 * area (the sum of the triangles' areas), normal (the sum of their area
 * vectors) and centroid (area-weighted, the pivot where the area is not
 * positive); every cell into the tetrahedra joining the mean of its face
 * centroids to its faces' triangles, oriented out of the cell, giving its
 * volume and centroid.  Topology: node_pos (nf + 1) / nodes, face_pos
 * (nc + 1) / cell_faces, neighbors (nf x 2, -1 outside), coords nn x 3;
 * outputs face_areas (nf), face_normals and face_centroids (nf x 3),
 * cell_volumes (nc), cell_centroids (nc x 3).  Synchronises the stream.
 */
int pmb_compute_geometry3d(int32_t nf, int32_t nc, const double* d_coords, const int32_t* d_node_pos,
                           const int32_t* d_nodes, const double* d_hinge, const int32_t* d_face_pos,
                           const int32_t* d_cell_faces, const int32_t* d_neighbors, double* d_face_areas,
                           double* d_face_normals, double* d_face_centroids, double* d_cell_volumes,
                           double* d_cell_centroids, void* stream);

/* ------------------------------------------------------------------------
 * Transmissibilities.
 * pmb_compute_trans replaces compute_trans (pymrst/solvers/compute_trans.py:11-53):
 * one-sided T = (c . K n) / (c . c) per half-face, c = face centroid - cell
 * centroid, n the face normal oriented out of the cell, K the full 3x3
 * tensor given row-major per cell (perm9, nc x 9), then |T| where
 * fix_negative != 0, then the net-to-gross multiplier (ntg and half_tag may
 * be NULL; half-faces with tag // 2 == 2 keep 1).
 * pmb_face_trans replaces get_face_transmissibility
 * (pymrst/solvers/get_face_transmissibility.py:12-31): T_f = 1 / sum 1/T_hf
 * over the half-faces of face f, listed CSR-style by hf_ptr/hf_idx.
 */
int pmb_compute_trans(int64_t n_half, const int32_t* d_cell_no, const int32_t* d_half_face,
                      const int32_t* d_face_first_cell, const double* d_cell_centroid,
                      const double* d_face_centroid, const double* d_face_normal,
                      const double* d_perm9, const double* d_ntg, const int32_t* d_half_tag,
                      int32_t fix_negative, double* d_t_half, void* stream);
int pmb_face_trans(int64_t nf, const int32_t* d_hf_ptr, const int32_t* d_hf_idx,
                   const double* d_t_half, double* d_t_face, void* stream);

/* ------------------------------------------------------------------------
 * Oil-water fully-implicit model (TwoPhaseOilWaterModelAD,
 * pymrst/modules/ad_blackoil/models/two_phase_oil_water_model.py:77-657).
 */
typedef struct pmb_ow pmb_ow;

typedef struct pmb_ow_desc {
  int32_t nc, nf, nw;
  const int32_t* h_N;     /* nf x 2 internal neighbour pairs (N[:,0], N[:,1]) */
  const double* h_T;      /* nf harmonic face transmissibilities */
  const double* h_gdz;    /* nf gravity * (z[N1] - z[N0]) */
  const double* h_pv;     /* nc pore volumes */
  /* fluid (init_simple_adi_fluid.py:217-239), water then oil */
  double mu[2], rhoS[2], n_exp[2], c[2], b0[2], sl[2], su[2], p_ref;
  /* wells: perforations of well k are perf_ptr[k] .. perf_ptr[k+1]-1,
   * in the well's top-to-bottom order */
  const int32_t* h_perf_ptr; /* nw+1 */
  const int32_t* h_perf_cell;
  const double* h_perf_WI;
  const double* h_perf_dZ;
  const double* h_compi;     /* nw x 2 */
  const int32_t* h_well_type; /* 0 = bhp, 1 = rate */
  const double* h_well_val;
  double gravity;
  double tol_cnv, tol_mb, tol_well, ds_max, dp_max_rel;
  /* nf flags (may be NULL): nonzero where the interface is vertical, so that
   * N[f,0] -> N[f,1] continues a vertical line of cells; the CPR second stage
   * solves along these lines */
  const int32_t* h_line_face;
} pmb_ow_desc;

int pmb_ow_create(const pmb_ow_desc* desc, void* stream, pmb_ow** out);
int pmb_ow_destroy(pmb_ow* h);
/* h_out8 = [nc, nf, nw, nperf, nnzb, nvec, well_part_len, ncolors] */
int pmb_ow_sizes(const pmb_ow* h, int64_t* h_out8);
/* Block-CSR pattern of the cell part: row_ptr (nc+1), col (nnzb), host. */
int pmb_ow_pattern(const pmb_ow* h, int32_t* h_row_ptr, int32_t* h_col);

/* Per-perforation wellbore pressure drop for a timestep starting at d_x0
 * (_compute_cdp_per_well, two_phase_oil_water_model.py:205-284).  Uses and
 * updates the handle's previous-step cdp, as the reference model does. */
int pmb_ow_compute_cdp(pmb_ow* h, const double* d_x0, double* d_cdp);
/* Forget the previous-step cdp (a fresh model). */
int pmb_ow_reset_cdp(pmb_ow* h);
/* The flux terms of assemble at state d_x (two_phase_oil_water_model.py:
 * 520-546 and the perforation rates of :286-491): d_face_flux (nf x 2,
 * water then oil) holds what interface f adds to the residual rows of
 * N[f,0] and subtracts from those of N[f,1]; d_perf_rate (nperf x 2) the
 * surface rates each perforation subtracts from its cell's rows and from its
 * well's rate equations.  Both are linear in T[f] and in the perforation's
 * well index (for wells without cross-flow), which is what the adjoint
 * gradient with respect to permeability uses.  Uses the model's residual
 * workspace (not during a step on the same handle). */
int pmb_ow_fluxes(pmb_ow* h, const double* d_x, const double* d_cdp, double* d_face_flux, double* d_perf_rate);
/* Adjoint pieces (compute_gradient_adjoint, pymrst/modules/optimization/
 * adjoint.py:163-225), all on the device and in the reference's
 * variable-blocked layout [p (nc), sW (nc), qWs, qOs, bhp (nw each)]:
 * pmb_ow_prev_jacobian_tmul: d_y = (dR_{n+1}/dx_n)^T d_lam, the coupling of
 *   step n+1 to its start state x_n (d_x_prev, cell-major) through the
 *   accumulation terms (_jac_wrt_previous, adjoint.py:83-105), dt the step
 *   n+1; the well entries of d_y are 0.
 * pmb_ow_csr_values: values of a CSR matrix (the Jacobian, or its transpose,
 *   on a pattern the caller built once) whose entry e is the sum over terms
 *   d_ptr[e] .. d_ptr[e+1]-1: t >= 0 is d_jac[t] (t < 4 nnzb) or
 *   d_well[t - 4 nnzb]; t < 0 encodes -1 - ((i nperf + j) 4 + 2a + b), entry
 *   (a, b) of the cross-flow product Up_i Vp_j of perforations i, j of one
 *   well (counted where that well's mixture coupling is on).  This is the
 *   device counterpart of combine_equations (pymrst/utils/adi/operators.py:
 *   204-211) on the model's block layout.
 * pmb_ow_perm_contract: d_out[c] += lam^T dR/d(log k_c) at d_x with the
 *   well pressure drops 0, through every interface transmissibility of c
 *   (dT_f/dlog k_c = T_f^2 / t_{c,f}; d_t0 / d_t1 the half-face T of N[f,0] /
 *   N[f,1], nf each) and the well indices of c's perforations; no reference
 *   counterpart (its adjoint has no permeability gradient).  d_face_flux
 *   (2 nf) and d_perf_rate (2 nperf) are scratch.
 * pmb_ow_get_last_cdp / pmb_ow_set_last_cdp: the previous timestep's well
 *   pressure drops that the next pmb_ow_compute_cdp starts from (nperf
 *   values; *h_have = 0 when there are none; d_in NULL forgets them): what
 *   a forward segment recomputed from a checkpoint must be given to take
 *   the same steps again. */
int pmb_ow_prev_jacobian_tmul(pmb_ow* h, const double* d_x_prev, double dt, const double* d_lam, double* d_y);
int pmb_ow_csr_values(pmb_ow* h, const double* d_jac, const double* d_well, int64_t n, const int64_t* d_ptr,
                      const int64_t* d_terms, double* d_vals);
int pmb_ow_perm_contract(pmb_ow* h, const double* d_x, const double* d_lam, const double* d_t0, const double* d_t1,
                         double* d_face_flux, double* d_perf_rate, double* d_out);
int pmb_ow_get_last_cdp(pmb_ow* h, double* d_out, int32_t* h_have);
int pmb_ow_set_last_cdp(pmb_ow* h, const double* d_in);
/* New well targets, one per well: bhp for bhp wells, total surface rate for
 * rate wells (_set_controls, pymrst/modules/optimization/adjoint.py:63-65,
 * which sets w.val between timesteps).  Also rescales the well convergence
 * test, whose rate reference is the largest rate target (_converged,
 * two_phase_oil_water_model.py:549-567). */
int pmb_ow_set_controls(pmb_ow* h, const double* h_well_val);

/* Residual and Jacobian at d_x for the step from d_x0 over dt
 * (assemble, two_phase_oil_water_model.py:493-546).  d_jac: nnzb 2x2
 * blocks, row-major within a block; d_well: the well part
 * (well_part_len doubles).  want_jac = 0 computes the residual only. */
int pmb_ow_assemble(pmb_ow* h, const double* d_x, const double* d_x0, double dt,
                    const double* d_cdp, double* d_res, double* d_jac, double* d_well,
                    int32_t want_jac);
/* y = J x with the full operator (cells, wells, mixture coupling). */
int pmb_ow_spmv(pmb_ow* h, const double* d_jac, const double* d_well, const double* d_x,
                double* d_y);
/* Convergence values (_converged, two_phase_oil_water_model.py:549-567):
 * h_out8 = [cnv, mb, max|eq_w|/q_ref, max|eq_o|/q_ref, ctrl_ok, converged,
 *           nonfinite, 0]. */
int pmb_ow_convergence(pmb_ow* h, const double* d_res, const double* d_x, double dt,
                       double* h_out8);
/* Allocation-free CNV / MB check over the cells; it has no counterpart in
 * the reference.  For callers that cannot allocate device memory where they
 * run the check (inside another framework's memory pool, or where
 * cudaMalloc's implicit synchronisation is not allowed): no handle, no
 * cudaMalloc / cudaFree; the per-block partial sums live in a static device
 * array of 458,752 bytes, so nc may be at most 16,777,216 (larger sizes are
 * rejected with PMB_ERR_ARG).  d_res and d_x hold the cell part of the
 * cell-major layout (2*nc doubles each), d_pv the pore volumes;
 * h_fluid5 = [c_w, c_o, b0_w, b0_o, p_ref]; d_out4 (device) receives
 * [cnv, mb, non-finite cell count, 0], the cnv and mb of pmb_ow_convergence.
 * The first call on a device looks up the array's device address, so make
 * it before any stream capture; the address is kept for the life of the
 * process, so do not call it on a device after cudaDeviceReset() of that
 * device.  d_res and d_x must be 16-byte aligned, d_pv and d_out4 8-byte
 * aligned.  Calls that overlap on the GPU share the array and race. */
int pmb_ow_cnv_mb_noalloc(int32_t nc, const double* d_res, const double* d_x, const double* d_pv,
                          double pv_total, const double* h_fluid5, double dt, double* d_out4,
                          void* stream);

/* Newton update with the reference's limits (step, :641-651): dp clipped to
 * dp_max_rel*|p|, ds to ds_max, sW to [0,1]; well unknowns unclipped.
 * The increment applied is sign * d_dx. */
int pmb_ow_update(pmb_ow* h, double* d_x, const double* d_dx, double sign);

/* ------------------------------------------------------------------------
 * CPR-preconditioned GMRES on the oil-water operator (replaces CPRSolver.solve,
 * pymrst/modules/ad_core/solvers/linear_solvers.py:426-545).
 */
typedef struct pmb_cpr pmb_cpr;

typedef struct pmb_cpr_opts {
  double rtol;              /* relative residual target, ||b - A x|| <= rtol ||b|| */
  int32_t maxiter;          /* total Krylov iterations */
  int32_t restart;          /* GMRES restart length */
  int32_t precision;        /* 0: FP64 throughout; 1: FP32 AMG and FP32 smoother blocks
                               inside the FP64 FGMRES */
  int32_t use_pressure_stage;
  int32_t local_sweeps;     /* second-stage sweeps: vertical-line block Gauss-Seidel where
                               the model has vertical lines, else red-black block GS */
  int32_t amg_smoother_degree; /* Chebyshev degree on each level */
  int32_t amg_cycle;        /* 0: V-cycle; k > 0: K-cycle, the coarse corrections of the
                               first k levels accelerated by two Krylov steps */
  double amg_theta;         /* strength threshold of pairwise aggregation */
  int32_t amg_coarse_size;  /* stop coarsening at this many unknowns */
  int32_t amg_rebuild_interval; /* re-aggregate after this many setups */
  double inner_rtol;        /* mixed precision: FP32 inner solve target */
  int32_t replay_graph;     /* 1: the preconditioner is captured once and replayed as a CUDA
                               graph; 0: its kernels are launched directly (for callers
                               that drive several solvers from concurrent host threads) */
  int32_t amg_coarse_degree; /* Chebyshev degree on the levels below the K-cycle levels;
                                0: amg_smoother_degree */
} pmb_cpr_opts;

/* Defaults: rtol 1e-8, maxiter 200, restart 50 (CPRSolver's,
 * linear_solvers.py:113-116); local_sweeps 4, Chebyshev degree 2, K-cycle on
 * 3 levels, theta 0.1, coarse size 200, re-aggregation every 8 setups,
 * graph replay on, coarse degree 0 (the smoother degree on every level). */
int pmb_cpr_default_opts(pmb_cpr_opts* out);
int pmb_cpr_create(pmb_ow* model, const pmb_cpr_opts* opts, pmb_cpr** out);
int pmb_cpr_destroy(pmb_cpr* s);
/* Build / refresh the preconditioner for the Jacobian (d_jac, d_well) at
 * state d_x (quasi-IMPES weights 1/b at the mean pressure). */
int pmb_cpr_setup(pmb_cpr* s, const double* d_jac, const double* d_well, const double* d_x);
/* Solve J x = b from x = 0.  h_info4 = [iterations, relres, ok, setups].
 * Returns PMB_ERR_NOCONV when the tolerance was not reached. */
int pmb_cpr_solve(pmb_cpr* s, const double* d_b, double* d_x, double* h_info4);
/* Unknowns per level of the current pressure hierarchy. */
int pmb_cpr_levels(const pmb_cpr* s, int32_t max_levels, int64_t* h_sizes, int32_t* n_levels);
/* Measurement aid, no counterpart in the reference: mean milliseconds of one
 * application of a preconditioner stage on the solver's stream (CUDA events,
 * after one untimed application).  stage 0: the second stage (all local
 * sweeps, updating d_z in place); 1: one AMG cycle on the restricted d_r;
 * 2: the whole preconditioner z = M^{-1} r, launched kernel by kernel; 3:
 * the same, replayed from its CUDA graph as the solver applies it.  Needs
 * pmb_cpr_setup first. */
/* Measurement aid, no counterpart in the reference: algorithmic bytes of the
 * solver's launches on its current hierarchy (every array read or written
 * once per launch, in its storage type), h_out8 = [one AMG cycle, one
 * second-stage sweep, one operator product, the pressure restriction and
 * prolongation of one preconditioner application, one setup without
 * aggregation, the Krylov vector length, one AMG refresh, 0].  Needs
 * pmb_cpr_setup first. */
int pmb_cpr_bytes(const pmb_cpr* s, double* h_out8);
int pmb_cpr_time_stage(pmb_cpr* s, int32_t stage, const double* d_r, double* d_z, int32_t reps,
                       double* h_ms);
/* Diagnostics: the mean time of one visit of AMG level `level` (0 .. the
 * coarsest; the cycle from that level down, on its own right-hand side,
 * zero for level 0, replayed `reps` times from a CUDA graph) and the entries
 * stored for that level (the dense inverse's n * n on the coarsest).
 * Overwrites the AMG's work vectors; needs pmb_cpr_setup first. */
int pmb_cpr_time_level(pmb_cpr* s, int32_t level, int32_t reps, double* h_ms, int64_t* h_nnz);

/* A batch of independent models (an ensemble of realisations, run_ensemble,
 * pymrst/modules/ensemble/ensemble_impl.py:49-67, which runs them one after
 * another) stored as one model whose members share no interface: member m
 * owns cells [h_cell_ptr[m], h_cell_ptr[m+1]) and wells [h_well_ptr[m],
 * h_well_ptr[m+1]).  One backward-Euler step of every member with h_state[m]
 * = 1, by one Newton loop whose kernels cover all members, with the
 * convergence test of step (two_phase_oil_water_model.py:605-657) applied
 * to each member alone: a converged member is frozen (zero right-hand side,
 * zero correction) while the others iterate.  Members with h_state[m] = 0
 * are left as they are.  On return h_state[m] = 1 converged, 0 failed (its
 * state restored to the start of the step), -1 frozen; h_its[m] its Newton
 * iterations; h_stats4 = [krylov iterations, setups, Newton iterations of
 * the batch, 0]. */
int pmb_ow_step_members(pmb_ow* h, pmb_cpr* s, double* d_x, double dt, int32_t max_iterations, int32_t nmem,
                        const int32_t* h_cell_ptr, const int32_t* h_well_ptr, int32_t* h_state, int32_t* h_its,
                        double* h_stats4);

/* ------------------------------------------------------------------------
 * CPR on a caller's CSR matrix: the device side of the drop-in for
 * CPRSolver.solve(jac, rhs, model, state)
 * (pymrst/modules/ad_core/solvers/linear_solvers.py:426-545).
 * The n x n matrix is in the reference's variable-blocked ordering: nph
 * blocks of nc cell unknowns (pressure first), then n - nph*nc facility
 * unknowns.  The second stage inverts the facility block group by group, a
 * group being a connected component of the facility block's own pattern
 * (one well's unknowns where wells do not couple), of at most 4096
 * unknowns each.  h_row_ptr / h_col: canonical CSR (columns
 * strictly increasing in a row), fixed for the handle's life; values are
 * given per setup.  opts as for pmb_cpr_create; local_sweeps counts
 * block-Jacobi sweeps of the second stage (1 = the reference's single
 * application).  h_weights (nph doubles): the decoupling weights
 * (_weighting, :155-190: 1/b_i at the mean pressure).  h_info4 =
 * [iterations, relres, ok, setups]; PMB_ERR_NOCONV when rtol was not
 * reached, PMB_ERR_PIVOT for a singular cell block.  transposed != 0: the
 * matrix given is J^T (the adjoint system of compute_gradient_adjoint,
 * pymrst/modules/optimization/adjoint.py:209) and the CPR transfer
 * operators are transposed with it (restriction to the pressure rows,
 * prolongation by the weights). */
typedef struct pmb_csr_cpr pmb_csr_cpr;
int pmb_csr_cpr_create(int32_t n, int32_t nc, int32_t nph, const int32_t* h_row_ptr, const int32_t* h_col,
                       int32_t transposed, const pmb_cpr_opts* opts, void* stream, pmb_csr_cpr** out);
int pmb_csr_cpr_destroy(pmb_csr_cpr* h);
int pmb_csr_cpr_setup(pmb_csr_cpr* h, const double* d_values, const double* h_weights);
int pmb_csr_cpr_solve(pmb_csr_cpr* h, const double* d_b, double* d_x, double* h_info4);
/* on != 0: the pressure stage uses per-cell weights, row 0 of the inverse of
 * each cell's diagonal nph x nph block (the weighted sum of the cell's rows
 * then has a unit derivative in its own pressure and none in its other
 * unknowns: true-IMPES on the full diagonal block), instead of the phase
 * weights given to setup; non-transposed systems only.  No reference
 * counterpart (its CPRSolver uses the quasi-IMPES phase weights). */
int pmb_csr_cpr_set_cell_weights(pmb_csr_cpr* h, int32_t on);
/* y = A x with the values d_values on the handle's pattern. */
int pmb_csr_spmv(pmb_csr_cpr* h, const double* d_values, const double* d_x, double* d_y);
int pmb_csr_cpr_levels(const pmb_csr_cpr* h, int32_t max_levels, int64_t* h_sizes, int32_t* n_levels);

/* Each row of the CSR matrix (device row pointers, values) divided by its
 * largest |entry|; d_scale[r] receives the factor (1 for an empty or zero
 * row).  The transposed adjoint systems need it: the rows of J^T span many
 * orders of magnitude (well-control columns of J are O(1), cell columns
 * O(1e-10)), and unit rows make the Krylov residual test uniform.  No
 * reference counterpart (the reference solves J^T directly). */
int pmb_csr_row_scale(int32_t n, const int32_t* d_row_ptr, double* d_vals, double* d_scale, void* stream);

/* d_inv = d_a^-1 for a dense row-major n x n FP64 matrix (1 <= n <= 4096),
 * the AMG coarsest-level solver: Gauss-Jordan with row pivoting.  Returns
 * PMB_ERR_PIVOT for a singular matrix.  Synchronises the stream.  An
 * internal of the device AMG, exported for testing; no reference
 * counterpart. */
int pmb_dense_inverse(int32_t n, const double* d_a, double* d_inv, void* stream);

/* ------------------------------------------------------------------------
 * One backward-Euler step solved by Newton on the device (step,
 * two_phase_oil_water_model.py:605-657): d_x holds the state at the start
 * of the step and receives the new state.  h_stats8 = [iterations,
 * converged, krylov_iterations, setups, cnv, mb, nonfinite, linear solves
 * that stopped above their tolerance but were used].  Returns PMB_OK also
 * when Newton did not converge (converged = 0).  A linear solve that stops
 * above rtol with a relative residual of at most 1e-6 still updates the
 * iterate (the Newton test decides, as with an exact solve); a worse or
 * non-finite one returns PMB_ERR_NOCONV with d_x restored to the start
 * state. */
int pmb_ow_step(pmb_ow* h, pmb_cpr* s, double* d_x, double dt, int32_t max_iterations,
                double* h_stats8);

/* ------------------------------------------------------------------------
 * AMG-preconditioned conjugate gradients for a scalar SPD CSR system: the
 * pressure solve of incomp_tpfa (pymrst/modules/incomp/incomp_tpfa.py:172-184,
 * `spsolve` or the caller's LinSolve).  The pattern (host row_ptr / col,
 * sorted, diagonal present) is fixed at creation; pmb_pcg_setup refreshes
 * the values (device, one per entry); solves start from x = 0 and stop at
 * ||b - A x|| <= rtol ||b||.  h_info3 = [iterations, relres, ok]. */
typedef struct pmb_pcg pmb_pcg;
int pmb_pcg_create(int32_t n, const int32_t* h_row_ptr, const int32_t* h_col, double amg_theta,
                   int32_t amg_coarse_size, void* stream, pmb_pcg** out);
int pmb_pcg_destroy(pmb_pcg* p);
int pmb_pcg_setup(pmb_pcg* p, const double* d_vals);
int pmb_pcg_solve(pmb_pcg* p, const double* d_b, double* d_x, double rtol, int32_t maxiter,
                  double* h_info3);
int pmb_pcg_levels(const pmb_pcg* p, int32_t max_levels, int64_t* h_sizes, int32_t* n_levels);

/* ------------------------------------------------------------------------
 * Incompressible TPFA pressure system on the device (incomp_tpfa,
 * pymrst/modules/incomp/incomp_tpfa.py:55-211).  The handle holds the grid
 * topology and the well perforations; per call the caller gives the
 * transmissibilities, phase mobilities and driving forces.
 *
 * Unknowns: nc cell pressures, then one bottom-hole pressure per well (the
 * reference's ordering, :104-106).  The matrix is CSR on a pattern fixed at
 * creation (pmb_tpfa_pattern): per cell row the diagonal, the cell across each
 * interior interface, and the bhp of each rate well perforating the cell; per
 * well row the perforated cells of a rate well and the diagonal.
 */
typedef struct pmb_tpfa pmb_tpfa;

typedef struct pmb_tpfa_desc {
  int32_t nc, nf, nhf, dim;
  const int32_t* h_face_pos;        /* nc+1: half-faces of cell c are face_pos[c] .. face_pos[c+1]-1
                                       (G.cells.facePos) */
  const int32_t* h_cell_faces;      /* nhf: the face of each half-face (G.cells.faces[:, 0]) */
  const int32_t* h_neighbors;       /* nf x 2 (G.faces.neighbors, -1 outside the grid) */
  const double* h_cell_centroids;   /* nc x dim */
  const double* h_face_centroids;   /* nf x dim */
  int32_t nw;
  const int32_t* h_perf_ptr;        /* nw+1: perforations of well k are perf_ptr[k] .. perf_ptr[k+1]-1 */
  const int32_t* h_perf_cell;       /* the perforated cells (W[k].cells) */
  const int32_t* h_well_rate;       /* nw: 1 for a rate well, 0 for a bhp well (W[k].type) */
  int32_t use_trans;                /* 1: d_T holds one T per face, not per half-face (use_trans) */
} pmb_tpfa_desc;

typedef struct pmb_tpfa_forces {
  const double* d_T;      /* nhf one-sided T (or nf face T with use_trans) */
  const double* d_mob;    /* nc x nph phase mobilities kr / mu, row-major */
  int32_t nph;            /* 1 .. 4 */
  const double* h_rho;    /* nph phase densities */
  double gravity[3];      /* gravity vector of the half-face potentials (zero: off) */
  double well_gravity;    /* |g| of the wells' hydrostatic drops */
  int32_t nbc;            /* boundary conditions (the reference's bc struct): */
  const int32_t* h_bc_face; /*   faces (no face twice) */
  const int32_t* h_bc_type; /*   1 pressure, 2 flux */
  const double* h_bc_value; /*   pressure, or flux out of the domain */
  int32_t nsrc;           /* sources (src.cell, src.rate) */
  const int32_t* h_src_cell;
  const double* h_src_rate;
  const double* h_well_val;  /* nw targets (bhp or total rate) */
  const double* d_perf_WI;   /* well indices per perforation */
  const double* d_perf_dZ;   /* depth below the well's reference depth per perforation */
  int32_t ncompi;            /* phases of the injected composition */
  const double* h_compi;     /* nw x ncompi */
  const int32_t* h_injector; /* nw: 1 where the mixture density is the injected composition's */
} pmb_tpfa_forces;

int pmb_tpfa_create(const pmb_tpfa_desc* desc, void* stream, pmb_tpfa** out);
int pmb_tpfa_destroy(pmb_tpfa* h);
/* h_out4 = [n, nnz, perforations, pinned]; pinned = 1 when the last assembly
 * doubled a diagonal entry to fix the pressure level (no pressure boundary,
 * no bhp well; incomp_tpfa.py:156-161). */
int pmb_tpfa_sizes(const pmb_tpfa* h, int64_t* h_out4);
int pmb_tpfa_pattern(const pmb_tpfa* h, int32_t* h_row_ptr, int32_t* h_col);
/* Matrix values (nnz, device) and right-hand side (n, device) of the system
 * (incomp_tpfa.py:91-161); the handle keeps the mobility-weighted
 * transmissibilities and potentials for pmb_tpfa_reconstruct. */
int pmb_tpfa_assemble(pmb_tpfa* h, const pmb_tpfa_forces* forces, double* d_vals, double* d_rhs);
/* Solve the assembled system by AMG-preconditioned CG from p = 0 to
 * ||rhs - A p|| <= rtol ||rhs|| (the reference calls SuperLU, :172-184).
 * h_info3 = [iterations, relres, ok]; PMB_ERR_NOCONV when rtol was not met. */
int pmb_tpfa_solve(pmb_tpfa* h, const double* d_vals, const double* d_rhs, double* d_p, double rtol,
                   int32_t maxiter, double* h_info3);
/* Face pressures, face fluxes (nf each) and per-perforation well fluxes and
 * hydrostatic drops (may be NULL) from the solution d_p (n) of the last
 * assembly (incomp_tpfa.py:186-211). */
int pmb_tpfa_reconstruct(pmb_tpfa* h, const double* d_p, double* d_flux, double* d_face_pressure,
                         double* d_perf_flux, double* d_perf_dp);
int pmb_tpfa_levels(const pmb_tpfa* h, int32_t max_levels, int64_t* h_sizes, int32_t* n_levels);

/* ------------------------------------------------------------------------
 * Two-phase incompressible transport (explicit_transport and
 * implicit_transport, pymrst/modules/incomp/transport/__init__.py:152-402)
 * for a Corey fluid.  The handle holds the interior interfaces (h_N, nf x 2)
 * and the pore volumes; pmb_transport_set_flow copies the frozen Darcy flux
 * and gravity flux of each interior interface (d_flux, d_gflux, nf each) and
 * the water source of each cell (d_q, nc; transport_source, :33-93) and takes
 * h_fluid4 = [mu_w, mu_o, n_w, n_o].  Saturations d_s are the water
 * saturations (nc), updated in place.
 *
 * pmb_transport_explicit: forward-Euler substeps over tf seconds, every
 *   substep dt (dt > 0) or min(max_dt, dt_factor * the reference's stable-step
 *   estimate, _estimate_dt :232-282) whose constant gravity part
 *   max |dg gflux_est drho| the caller passes as gravity_wave; the substep
 *   clock runs on the device.  Stops at the first substep that leaves
 *   [-satwarn, 1 + satwarn] or produces NaN.  h_out4 = [substeps, time
 *   reached, out-of-range flag, NaN flag].
 * pmb_transport_implicit: backward Euler with Newton, bisection line search
 *   and the substep control of newtonRaphson2ph; linear systems by FGMRES
 *   (rtol, maxiter and restart of opts) preconditioned by a Gauss-Seidel
 *   sweep in flow order: the cells ordered so that every upwind coupling
 *   points at an earlier level (exact when the upwind graph has no cycle;
 *   of two cells coupled both ways the weaker coupling lags), one launch per
 *   level.
 *   h_out6 = [time reached, substeps, Newton iterations, Krylov iterations,
 *   linear solves that missed their tolerance, last substep length]; the
 *   time reached is below tf when the minimum substep tf 2^-tsref failed.
 * pmb_transport_residual / _jacobian: r(s, s0, dt) and dr/ds on the fixed
 *   pattern of pmb_transport_pattern (each cell and its neighbours). */
typedef struct pmb_transport pmb_transport;
int pmb_transport_create(int32_t nc, int32_t nf, const int32_t* h_N, const double* h_pv, void* stream,
                         pmb_transport** out);
int pmb_transport_destroy(pmb_transport* h);
/* *h_nnz = nonzeros; h_row_ptr (nc + 1) and h_col (nnz) may be NULL. */
int pmb_transport_pattern(const pmb_transport* h, int64_t* h_nnz, int32_t* h_row_ptr, int32_t* h_col);
int pmb_transport_set_flow(pmb_transport* h, const double* d_flux, const double* d_gflux, const double* d_q,
                           const double* h_fluid4);
/* *h_absmax (may be NULL) receives max |r|; synchronises when given. */
int pmb_transport_residual(pmb_transport* h, const double* d_s, const double* d_s0, double dt, double* d_res,
                           double* h_absmax);
int pmb_transport_jacobian(pmb_transport* h, const double* d_s, double dt, double* d_vals);
int pmb_transport_explicit(pmb_transport* h, double* d_s, double tf, double dt, double max_dt, double dt_factor,
                           double satwarn, double gravity_wave, double* h_out4);
int pmb_transport_implicit(pmb_transport* h, double* d_s, double tf, double nltol, int32_t lstrials,
                           int32_t maxnewt, int32_t tsref, double resred, const pmb_cpr_opts* opts, double* h_out6);

/* ------------------------------------------------------------------------
 * Three-phase black-oil model with dissolved gas (ThreePhaseBlackOilModelAD,
 * pymrst/modules/ad_blackoil/models/three_phase_black_oil_model.py:93-565)
 * and the deck-table fluid of init_deck_blackoil_fluid
 * (pymrst/modules/ad_props/props/init_deck_adi_fluid.py:60-200).
 *
 * State (device, doubles): [p | sW | sO | sG | rs | status | qWs | qOs | qGs
 * | bhp], nc entries per cell field and nw per well field; status is 1.0
 * (undersaturated: the third unknown is rs) or 3.0 (free gas: it is sG).
 * Residual and Jacobian are in the reference's variable-blocked order:
 * equations water, oil, gas of every cell, then the water, oil and gas rate
 * equations and the control equation of every well; unknowns p, sW, x of
 * every cell, then qWs, qOs, qGs, bhp (combine_equations of assemble's
 * seven equations).  The Jacobian's CSR pattern is fixed per handle
 * (pmb_bo_pattern): every cell row holds its cell, its interface neighbours,
 * the other cells of its well, and its well's four unknowns.
 * Tables are piecewise linear with strictly increasing abscissae; interp_table
 * (weights form, linear extrapolation) for gas, Rs_sat and saturation tables,
 * the keyed 'parallel' interpolation for the live oil. */
typedef struct pmb_bo pmb_bo;

typedef struct pmb_bo_desc {
  int32_t nc, nf, nw;
  const int32_t* h_N;      /* nf x 2 interior interface neighbours */
  const double* h_T;       /* nf transmissibilities */
  const double* h_gdz;     /* nf gravity * (z[N1] - z[N0]) */
  const double* h_pv;      /* nc reference pore volumes */
  double rhoS[3];          /* surface densities water, oil, gas */
  double pvtw[4];          /* p_ref, Bw at p_ref, compressibility, viscosity (assignPVTW) */
  double rock[2];          /* p_ref, compressibility (assignROCK) */
  double swcon;            /* connate water (first SWOF row) */
  int32_t n_gas;           /* dry gas (PVDG with a p = 0 row): p, 1/Bg, mu_g */
  const double* h_gas_p;
  const double* h_gas_b;
  const double* h_gas_mu;
  int32_t n_rssat;         /* saturated Rs against pressure */
  const double* h_rssat_p;
  const double* h_rssat_rs;
  int32_t n_key;           /* live oil (PVTO): Rs keys; rows of key k are branch_ptr[k] .. branch_ptr[k+1]-1 */
  const double* h_key;
  const int32_t* h_branch_ptr;
  const double* h_branch_p;
  const double* h_branch_b;   /* 1/Bo */
  const double* h_branch_mu;
  int32_t n_sw;            /* SWOF (flat-extended): sW, krW, pcOW (may be NULL) */
  const double* h_sw;
  const double* h_krw;
  const double* h_pcow;
  int32_t n_sow;           /* oil in water: sO, krOW */
  const double* h_sow;
  const double* h_krow;
  int32_t n_sg;            /* SGOF (flat-extended): sG, krG, pcOG (may be NULL) */
  const double* h_sg;
  const double* h_krg;
  const double* h_pcog;
  int32_t n_sog;           /* oil in gas: sO, krOG */
  const double* h_sog;
  const double* h_krog;
  /* wells: perforations of well k are perf_ptr[k] .. perf_ptr[k+1]-1 (1 to
   * 16 each); a cell is perforated at most once */
  const int32_t* h_perf_ptr;
  const int32_t* h_perf_cell;
  const double* h_perf_WI;
  const int32_t* h_well_type;  /* 0 bhp, 1 rate (total surface rate), 2 orat */
  const double* h_well_val;
  const double* h_compi;       /* nw x 3 */
  double tol_cnv, tol_mb, tol_well, ds_max;
} pmb_bo_desc;

int pmb_bo_create(const pmb_bo_desc* desc, void* stream, pmb_bo** out);
int pmb_bo_destroy(pmb_bo* h);
/* h_out3 = [unknowns 3 nc + 4 nw, Jacobian nonzeros, state length 6 nc + 4 nw]. */
int pmb_bo_sizes(const pmb_bo* h, int64_t* h_out3);
int pmb_bo_pattern(const pmb_bo* h, int32_t* h_row_ptr, int32_t* h_col);
/* Residual and Jacobian values at d_state, with d_state0 the state at the
 * start of the step (assemble, three_phase_black_oil_model.py:314-381). */
int pmb_bo_assemble(pmb_bo* h, const double* d_state, const double* d_state0, double dt, double* d_res,
                    double* d_vals);
/* Convergence of an assembled residual (_converged, :528-539): h_out14 =
 * [cnv water, oil, gas, mb water, oil, gas, max well-rate residual / q_ref,
 * max |control residual| / scale, converged, CPR weights 1/bW 1/bO 1/bG at
 * the mean pressure (get_scaling_factors_cpr, :205-245), mean pressure,
 * total pore volume].  Synchronises the stream. */
int pmb_bo_convergence(pmb_bo* h, const double* d_res, const double* d_state, double dt, double* h_out14);
/* Newton update with the reference's limits and the black-oil flash
 * (update_state and _flash, :439-508); d_dx in the unknowns' order. */
int pmb_bo_update(pmb_bo* h, double* d_state, const double* d_dx);
/* One step by Newton (step, :541-565) with the CSR CPR-GMRES as the linear
 * solver; d_state holds the start state and receives the last iterate.
 * h_stats4 = [iterations, converged, Krylov iterations, linear solves that
 * missed their tolerance].  The update of a solve that missed its tolerance
 * is still used (the Newton test decides); a non-finite one ends the step
 * unconverged. */
int pmb_bo_step(pmb_bo* h, double* d_state, double dt, int32_t max_iterations, const pmb_cpr_opts* opts,
                double* h_stats4);
/* The fluid at n points (tests and the host's fluid check): d_out7 =
 * [bW(p), bO(p, rs, sat), muO(p, rs, sat), bG(p), muG(p), Rs_sat(p),
 * pore-volume multiplier(p)], n entries each. */
int pmb_bo_pvt_points(pmb_bo* h, int32_t n, const double* d_p, const double* d_rs, const double* d_sat,
                      double* d_out7);
/* d_out5 = [krW, krO, krG, pcOW, pcOG] at (sW, sG), sO = 1 - sW - sG. */
int pmb_bo_relperm_points(pmb_bo* h, int32_t n, const double* d_sw, const double* d_sg, double* d_out5);

/* Host-side aggregation of the AMG hierarchy for a CSR matrix (no device
 * needed): unknowns per level into h_sizes (up to max_levels), count in
 * *n_levels.  Exposed for testing the set-up logic. */
int pmb_amg_hierarchy_host(int32_t n, const int32_t* h_row_ptr, const int32_t* h_col,
                           const double* h_val, double theta, int32_t coarse_size,
                           int32_t max_levels, int64_t* h_sizes, int32_t* n_levels);

#ifdef __cplusplus
}
#endif

#endif /* PYMRST_B200_H */
