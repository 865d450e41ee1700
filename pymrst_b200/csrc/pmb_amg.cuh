// Aggregation AMG for the CPR pressure system.
//
// Set-up splits in two.  Aggregation (which fine unknowns form a coarse
// unknown) runs in C++ on the host from the current matrix values and is
// kept for several Newton iterations.  Every refresh then recomputes all
// coarse operators on the device from the new fine values: plain
// (unsmoothed) aggregation makes the Galerkin product P^T A P a pure sum of
// fine entries, done as a gather over precomputed index lists, so the whole
// hierarchy is exact for the current matrix without a sparse triple product.
#pragma once

#include "pmb_common.cuh"

namespace pmb {

// inv = A^-1 for a dense row-major n x n FP64 matrix on the device: in-place
// Gauss-Jordan with row pivoting in one CTA (n up to about 11,000).  A zero or
// non-finite pivot sets PMB_ERR_PIVOT in *d_status.
void dense_inverse(int n, const double* a, double* inv, int* d_status, cudaStream_t s);

struct AMGHostLevel {
  int n = 0;
  std::vector<int> row_ptr, col;      // pattern of this level's matrix
  std::vector<int> agg;               // fine unknown -> coarse unknown (next level)
  std::vector<int> cptr, cmem;        // members of each coarse unknown
  std::vector<int> gptr, gidx;        // coarse nnz <- fine nnz indices
};

// Pairwise aggregation hierarchy from a CSR matrix (host).  `passes`
// successive pairwise matchings form one level (aggregates of up to
// 2^passes); a matching whose coarsening ratio is poor at threshold `theta`
// is redone with theta = 0; levels with fewer than aggressive_below unknowns
// take one pass more.  The last entry is the coarsest level (no agg).
std::vector<AMGHostLevel> amg_build_hierarchy(int n, const int* row_ptr, const int* col,
                                              const double* val, double theta, int passes,
                                              int coarse_size, int max_levels, int aggressive_below = 0);

// The first Chebyshev step of a level from a zero start (no matrix:
// d = c2 D^-1 b, x = d), fused into the kernel that writes that level's
// right-hand side; dinv null: not fused.
template <class T>
struct ZeroStep {
  const T* dinv = nullptr;
  const double* tab = nullptr;  // the level's Chebyshev table
  T* d = nullptr;
  T* x = nullptr;
};

constexpr int kEllMaxK = 8;  // slots of an ELL level

// An ELL level as its kernels see it (by value).  Column form: col holds
// every slot's column, a row longer than K marks its last slot -1 - o (o its
// overflow row).  Diagonal form (col null): slot k of row i is column
// i + off[k], and orow[i] is the row's overflow row or -1.
template <class T>
struct EllView {
  int n = 0, K = 0;
  const int* col = nullptr;
  const T* val = nullptr;
  const int* orow = nullptr;
  const int* optr = nullptr;
  const int* ocol = nullptr;
  const T* oval = nullptr;
  int off[kEllMaxK] = {};
};

template <class T>
struct AMGLevel {
  int n = 0, nnz = 0;
  int lanes = 1;  // threads per row in the row-wise kernels (from the mean row length)
  const int* row_ptr = nullptr;  // device (level 0 borrows the operator pattern)
  const int* col = nullptr;
  DArray<int> own_row_ptr, own_col;
  DArray<T> val, dinv, x, b, r, t, u;  // u: first output of an odd smoothing count
  DArray<T> kc1, kc2, kv1, kv2, kr2;  // K-cycle vectors of this level (as a coarse level)
  DArray<double> kpart;               // K-cycle reduction partials
  DArray<int> agg, cptr, cmem, gptr, gidx;
  DArray<double> lmax;  // Chebyshev upper bound (device scalar)
  // Restriction plan: CTA b of restrict_rows_kernel takes the aggregates
  // [rblk[b], rblk[b+1]), at most one member row per lane group unless a
  // single aggregate is larger; rsmem bytes of shared memory hold the member
  // residuals of the largest CTA.
  DArray<int> rblk;
  int rblocks = 0;
  size_t rsmem = 0;
  int degree = 0;  // Chebyshev degree of this level; 0: the hierarchy's
  // Slot-major ELL copy of the matrix, on levels whose rows are short and of
  // nearly equal length (ell_k > 0): entry k of row i at [k * n + i], so that
  // one thread per row issues all its loads at once and a warp's loads of
  // one slot are contiguous.  Short rows are padded with their own column
  // and a zero value.  A row longer than ell_k keeps ell_k - 1 entries in the
  // slots; its last slot holds -1 - o (o: its overflow row) and value zero,
  // and the rest of its entries follow in the overflow CSR.
  int ell_k = 0;
  bool ell_dia = false;  // diagonal form: slot k of row i is column i + ell_off[k]
  int ell_off[kEllMaxK] = {};
  DArray<int> ell_orow;          // diagonal form: the row's overflow row or -1
  DArray<int> ell_col, ell_src;  // ell_src: CSR index of each slot's value (-1: zero)
  DArray<T> ell_val;
  DArray<int> ell_optr, ell_ocol, ell_osrc;
  DArray<T> ell_oval;
  long long ell_ovf = 0;  // overflow entries
  DArray<double> ell_rr;  // member residuals of the restriction
  // cluster tail: packed (CTA << 16 | row in its chunk) columns, aggregates
  // and member rows
  DArray<unsigned> ct_pcol, ct_pagg, ct_pmem;
};

// The cluster tail cycle (amg.cu): the levels from its first one down to
// the coarsest, resident in the shared memory of one thread-block cluster.
// One tail level: global sources (loaded at every launch: the values change
// at every refresh) and the byte offsets of its sections in shared memory
// (the same in every CTA; each section is sized for the largest chunk).
template <class T>
struct CtLevel {
  int lanes, steps;
  const T* val;                  // CSR values of the level
  const T* dinv;
  const unsigned* pcol;          // packed column of every entry
  const int* rp;                 // CSR row starts
  const unsigned* pagg;          // packed aggregate of every row (next level / coarsest)
  const int* cptr;               // member ranges of the next level's rows
  const unsigned* pmem;          // packed member rows
  const double* tab;             // Chebyshev table
  int s_rp, s_col, s_val, s_dinv, s_b, s_x, s_t, s_u, s_d, s_rr, s_agg, s_cptr, s_mem;
};

// The chunk of CTA c on a level: rows [r0, r0 + nr), entries [z0, z0 + nz),
// the next level's rows [R0, R0 + ncr) with members [m0, m0 + nm).
struct CtPart {
  int r0, nr, z0, nz, R0, ncr, m0, nm;
};

struct CtCoarse {
  int nco;
  const double* inv;     // dense inverse, row-major
  const unsigned* pco;   // packed owner of every coarsest row
  int s_inv, s_b, s_x, s_pco, s_bfull;
};

// One level as seen by the fused coarse-cycle kernel.
template <class T>
struct CoopLevel {
  int n, lanes;
  const int* rp;
  const int* ci;
  const T* val;
  const T* dinv;
  const double* lmax;
  T* x;
  T* b;
  T* d;  // Chebyshev direction
  T* t;  // ping-pong partner of x
  const int* cptr;
  const int* cmem;
  const int* agg;
};

template <class T>
class AMG {
 public:
  // Build aggregation from host values of the level-0 matrix (pattern given
  // both on host and device).
  void build(int n, const std::vector<int>& h_row_ptr, const std::vector<int>& h_col,
             const int* d_row_ptr, const int* d_col, const std::vector<double>& h_val, double theta,
             int coarse_size, cudaStream_t s);
  // Refresh all levels from level-0 values already written to level0_val().
  void refresh(cudaStream_t s, int* d_status);
  // x = M^{-1} b with one cycle: V-cycle, or (k_levels > 0) a K-cycle whose
  // coarse corrections on the first k_levels levels are accelerated by two
  // minimal-residual Krylov steps.
  void apply(const T* b, T* x, cudaStream_t s);
  int k_levels = 0;
  T* level0_val() { return levels_.empty() ? co_val_.get() : levels_[0].val.get(); }
  bool built() const { return nco_ > 0; }
  int num_levels() const { return (int)levels_.size() + (nco_ > 0 ? 1 : 0); }
  int level_size(int l) const { return l < (int)levels_.size() ? levels_[l].n : nco_; }
  int degree = 2;
  int coarse_degree = 0;  // degree below the K-cycle levels (0: degree)
  // Run the levels below the K-cycle levels, down to the dense coarsest
  // solve, as one cooperative kernel when they are small (set before build;
  // also needs PMB_FUSED_COARSE=1 in the environment).
  bool fused_coarse = true;
  int fused_first_level() const { return coop_start_; }
  // Algorithmic bytes of one apply() and of one refresh(): every array a
  // kernel reads or writes counted once per launch, values in T, indices in
  // 4 bytes, the dense coarsest inverse in 8 bytes per entry.
  double cycle_bytes() const { return num_levels() ? cycle_bytes_from(0) : 0.0; }
  double refresh_bytes() const;
  long long level_nnz(int l) const { return l < (int)levels_.size() ? levels_[l].nnz : co_nnz_; }
  // Mean time of one visit of level l (the cycle from l down, on the level's
  // own right-hand side; level 0: the whole cycle on a zero right-hand side),
  // replayed from a CUDA graph.
  double time_visit(int l, int reps, cudaStream_t s);
  // The levels from tail_first_level() down (the first level below the
  // K-cycle levels with at most PMB_AMG_TAIL_ROWS rows whose levels fit a
  // cluster's shared memory, and all coarser ones) run as one
  // thread-block-cluster launch per visit (amg_ctail_kernel), bitwise the
  // per-step path; -1 when off (the default, or no layout fits).
  int tail_first_level() const { return tail_start_; }
  int tail_cluster_size() const { return tail_cluster_; }

 private:
  int tail_start_ = -1, tail_cluster_ = 0;
  DArray<unsigned char> tail_levels_;
  DArray<CtPart> tail_parts_;
  DArray<unsigned> ct_pco_;
  CtCoarse tail_co_{};
  size_t tail_smem_ = 0;
  void build_tail(const std::vector<AMGHostLevel>& H, cudaStream_t s);
  void launch_tail(const T* b, T* x, cudaStream_t s);
  double cycle_bytes_from(int l) const;
  double coarse_bytes(int l) const;
  int coop_start_ = -1, coop_grid_ = 0;
  DArray<unsigned char> coop_levels_;
  DArray<unsigned int> coop_bar_;  // grid barrier: arrivals, generation
  int* coop_status_ = nullptr;
  void build_fused(cudaStream_t s);
  void launch_fused(const T* b, T* x, cudaStream_t s);
  // zero_done / first_done: the kernel that wrote b already took the first
  // pre-smoothing step of level l (l + 1)
  void cycle(int l, const T* b, T* x, cudaStream_t s, bool zero_done = false);
  void coarse_correction(int l, const T* rc, T* ec, cudaStream_t s, bool first_done = false);
  ZeroStep<T> zero_step_for(int m, T* x);
  // xc (non-zero start only): fold x += P xc into the first step
  void smooth(AMGLevel<T>& L, const T* b, T* x, cudaStream_t s, bool zero_start, const T* xc = nullptr,
              bool first_done = false);
  void build_ell(AMGLevel<T>& L, const AMGHostLevel& h, cudaStream_t s);
  std::vector<AMGLevel<T>> levels_;
  // coarsest level: dense inverse in FP64
  int nco_ = 0, co_nnz_ = 0;
  int gj_rows_ = 0;     // rows of the coarse inverse's working matrix held in shared memory
  size_t gj_smem_ = 0;  // its dynamic shared memory
  int gj_cluster_ = 0;  // > 0: the inverse runs on a cluster of this many CTAs
  size_t gj_csmem_ = 0;
  DArray<int> co_row_ptr_, co_col_;
  DArray<T> co_val_;
  DArray<double> co_dense_, co_inv_;
  DArray<T> co_x_, co_b_;
  DArray<unsigned long long> bits_;
};

}  // namespace pmb
