// extern "C" entry points (include/pymrst_b200.h) and the device Newton step.
#include <atomic>
#include <cstdlib>
#include <map>
#include <mutex>
#include <cmath>
#include <cstring>
#include <memory>

#include "pmb_cpr.cuh"

namespace pmb {

static thread_local std::string g_last_error;
void set_error(const std::string& msg) { g_last_error = msg; }

bool pdl_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("PMB_NO_PDL");
    return !(e && e[0] == '1');
  }();
  return on;
}

static std::atomic<long long> g_launches{0};
void count_launch(long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
long long launch_count() { return g_launches.load(); }

// ---- phase timers -----------------------------------------------------------
struct PendingPhase {
  std::string name;
  cudaEvent_t e0, e1;
};
static std::mutex g_prof_mu;
static std::vector<PendingPhase> g_pending;
static std::map<std::string, std::pair<double, long long>> g_phase;  // ms, count

static void collect_phases() {
  std::vector<PendingPhase> keep;
  for (auto& p : g_pending) {
    if (cudaEventQuery(p.e1) == cudaSuccess) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, p.e0, p.e1);
      auto& a = g_phase[p.name];
      a.first += ms;
      a.second += 1;
      cudaEventDestroy(p.e0);
      cudaEventDestroy(p.e1);
    } else {
      keep.push_back(p);
    }
  }
  g_pending.swap(keep);
}

bool PhaseTimer::enabled() {
  static const bool on = [] {
    const char* e = std::getenv("PMB_PROFILE");
    return e && e[0] == '1';
  }();
  return on;
}

PhaseTimer::PhaseTimer(const char* name, cudaStream_t s) : name_(name), s_(s) {
  if (!enabled()) return;
  cudaEventCreate(&e0_);
  cudaEventRecord(e0_, s_);
}

PhaseTimer::~PhaseTimer() {
  if (!e0_) return;
  cudaEvent_t e1;
  cudaEventCreate(&e1);
  cudaEventRecord(e1, s_);
  std::lock_guard<std::mutex> g(g_prof_mu);
  g_pending.push_back({name_, e0_, e1});
  if (g_pending.size() > 4096) {
    cudaEventSynchronize(e1);
    collect_phases();
  }
}

void compute_trans(long long nh, const int* cell_no, const int* hface, const int* first_cell, const double* cc,
                   const double* fc, const double* fn, const double* K9, const double* ntg, const int* tag,
                   int fix_negative, double* out, cudaStream_t s);
void face_trans(long long nf, const int* ptr, const int* idx, const double* th, double* tf, cudaStream_t s);

static void require_aligned(const void* p, size_t a, const char* what) {
  PMB_REQUIRE(p != nullptr, std::string(what) + " is NULL");
  PMB_REQUIRE(reinterpret_cast<uintptr_t>(p) % a == 0,
              std::string(what) + " must be " + std::to_string(a) + "-byte aligned");
}

}  // namespace pmb

using namespace pmb;

struct pmb_ow {
  std::unique_ptr<OWModel> m;
  PinnedArray<double> conv;
  // batch-of-members stepping: member ranges, flags and per-member values
  DArray<int> mem_cell, mem_well, mem_flag;
  DArray<double> mem_conv, mem_lin, mem_linres;
  PinnedArray<double> mem_conv_h, mem_linres_h;
  PinnedArray<int> mem_flag_h;
};

struct pmb_cpr {
  pmb_ow* owner = nullptr;
  std::unique_ptr<CPRSolver> s;
};

extern "C" {

const char* pmb_last_error(void) { return g_last_error.c_str(); }

int pmb_version(void) { return 1; }

int pmb_profile_report(char* buf, int32_t len, int32_t reset) {
  return guarded([&] {
    PMB_REQUIRE(buf && len > 0, "invalid buffer");
    cudaDeviceSynchronize();
    std::lock_guard<std::mutex> g(g_prof_mu);
    collect_phases();
    std::string s;
    for (auto& kv : g_phase)
      s += kv.first + " " + std::to_string(kv.second.first) + " " + std::to_string(kv.second.second) + "\n";
    std::strncpy(buf, s.c_str(), (size_t)len - 1);
    buf[len - 1] = 0;
    if (reset) g_phase.clear();
  });
}

int pmb_launch_count(int64_t* out) {
  return guarded([&] {
    PMB_REQUIRE(out, "NULL argument");
    *out = g_launches.load();
  });
}

int pmb_compute_trans(int64_t n_half, const int32_t* d_cell_no, const int32_t* d_half_face,
                      const int32_t* d_face_first_cell, const double* d_cell_centroid,
                      const double* d_face_centroid, const double* d_face_normal, const double* d_perm9,
                      const double* d_ntg, const int32_t* d_half_tag, int32_t fix_negative, double* d_t_half,
                      void* stream) {
  return guarded([&] {
    PMB_REQUIRE(n_half >= 0, "negative half-face count");
    if (n_half == 0) return;
    PMB_REQUIRE(d_cell_no && d_half_face && d_face_first_cell && d_cell_centroid && d_face_centroid &&
                    d_face_normal && d_perm9 && d_t_half,
                "NULL argument");
    compute_trans(n_half, d_cell_no, d_half_face, d_face_first_cell, d_cell_centroid, d_face_centroid,
                  d_face_normal, d_perm9, d_ntg, d_half_tag, fix_negative, d_t_half, (cudaStream_t)stream);
  });
}

int pmb_face_trans(int64_t nf, const int32_t* d_hf_ptr, const int32_t* d_hf_idx, const double* d_t_half,
                   double* d_t_face, void* stream) {
  return guarded([&] {
    PMB_REQUIRE(nf >= 0, "negative face count");
    if (nf == 0) return;
    PMB_REQUIRE(d_hf_ptr && d_hf_idx && d_t_half && d_t_face, "NULL argument");
    face_trans(nf, d_hf_ptr, d_hf_idx, d_t_half, d_t_face, (cudaStream_t)stream);
  });
}

int pmb_dense_inverse(int32_t n, const double* d_a, double* d_inv, void* stream) {
  return guarded([&] {
    PMB_REQUIRE(n >= 1 && n <= 4096, "n must be in 1..4096");
    PMB_REQUIRE(d_a && d_inv && d_a != d_inv, "NULL or aliased argument");
    const cudaStream_t s = (cudaStream_t)stream;
    DArray<int> st;
    st.resize(1);
    st.zero(s);
    dense_inverse(n, d_a, d_inv, st.get(), s);
    int h = 0;
    PMB_CUDA(cudaMemcpyAsync(&h, st.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    PMB_CUDA(cudaStreamSynchronize(s));
    if (h != 0) throw Error(h, "zero pivot: the matrix is singular");
  });
}

int pmb_ow_create(const pmb_ow_desc* desc, void* stream, pmb_ow** out) {
  return guarded([&] {
    PMB_REQUIRE(desc && out, "NULL argument");
    *out = nullptr;
    auto h = std::make_unique<pmb_ow>();
    h->m = std::make_unique<OWModel>(*desc, (cudaStream_t)stream);
    h->conv.resize(8);
    *out = h.release();
  });
}

int pmb_ow_destroy(pmb_ow* h) {
  return guarded([&] { delete h; });
}

int pmb_ow_sizes(const pmb_ow* h, int64_t* out) {
  return guarded([&] {
    PMB_REQUIRE(h && out, "NULL argument");
    const OWModel& m = *h->m;
    const OWView v = m.view();
    out[0] = v.nc; out[1] = v.nf; out[2] = v.nw; out[3] = v.nperf;
    out[4] = m.nnzb(); out[5] = m.nvec(); out[6] = v.wl.total; out[7] = m.ncolors();
  });
}

int pmb_ow_pattern(const pmb_ow* h, int32_t* row_ptr, int32_t* col) {
  return guarded([&] {
    PMB_REQUIRE(h && row_ptr && col, "NULL argument");
    const auto& rp = h->m->h_row_ptr();
    const auto& cc = h->m->h_col();
    std::memcpy(row_ptr, rp.data(), rp.size() * sizeof(int32_t));
    std::memcpy(col, cc.data(), cc.size() * sizeof(int32_t));
  });
}

int pmb_ow_compute_cdp(pmb_ow* h, const double* d_x0, double* d_cdp) {
  return guarded([&] {
    PMB_REQUIRE(h, "NULL handle");
    require_aligned(d_x0, 16, "x0");
    if (h->m->nperf() == 0) return;
    PMB_REQUIRE(d_cdp, "cdp is NULL");
    h->m->compute_cdp(d_x0, d_cdp);
  });
}

int pmb_ow_reset_cdp(pmb_ow* h) {
  return guarded([&] {
    PMB_REQUIRE(h, "NULL handle");
    h->m->reset_cdp();
  });
}

int pmb_ow_prev_jacobian_tmul(pmb_ow* h, const double* d_x_prev, double dt, const double* d_lam, double* d_y) {
  return guarded([&] {
    PMB_REQUIRE(h && d_x_prev && d_lam && d_y, "NULL argument");
    require_aligned(d_x_prev, 16, "x_prev");
    h->m->prev_jacobian_tmul(d_x_prev, dt, d_lam, d_y);
  });
}

int pmb_ow_csr_values(pmb_ow* h, const double* d_jac, const double* d_well, int64_t n, const int64_t* d_ptr,
                      const int64_t* d_terms, double* d_vals) {
  return guarded([&] {
    PMB_REQUIRE(h, "NULL argument");
    h->m->csr_values(d_jac, d_well, n, d_ptr, d_terms, d_vals);
  });
}

int pmb_ow_perm_contract(pmb_ow* h, const double* d_x, const double* d_lam, const double* d_t0, const double* d_t1,
                         double* d_face_flux, double* d_perf_rate, double* d_out) {
  return guarded([&] {
    PMB_REQUIRE(h, "NULL argument");
    require_aligned(d_x, 16, "x");
    require_aligned(d_face_flux, 16, "face_flux");
    if (h->m->nw()) require_aligned(d_perf_rate, 16, "perf_rate");
    h->m->perm_contract(d_x, d_lam, d_t0, d_t1, d_face_flux, d_perf_rate, d_out);
  });
}

int pmb_ow_get_last_cdp(pmb_ow* h, double* d_out, int32_t* h_have) {
  return guarded([&] {
    PMB_REQUIRE(h && h_have, "NULL argument");
    int have = 0;
    h->m->get_last_cdp(d_out, &have);
    *h_have = have;
  });
}

int pmb_ow_set_last_cdp(pmb_ow* h, const double* d_in) {
  return guarded([&] {
    PMB_REQUIRE(h, "NULL argument");
    h->m->set_last_cdp(d_in);
  });
}

int pmb_ow_fluxes(pmb_ow* h, const double* d_x, const double* d_cdp, double* d_face_flux, double* d_perf_rate) {
  return guarded([&] {
    PMB_REQUIRE(h && d_x && d_face_flux, "NULL argument");
    const OWView v = h->m->view();
    PMB_REQUIRE(v.nw == 0 || (d_cdp && d_perf_rate), "wells need cdp and a rate buffer");
    require_aligned(d_x, 16, "x");
    require_aligned(d_face_flux, 16, "face_flux");
    if (v.nw) require_aligned(d_perf_rate, 16, "perf_rate");
    h->m->fluxes(d_x, d_cdp, d_face_flux, d_perf_rate);
    PMB_CUDA(cudaStreamSynchronize(h->m->stream()));
  });
}

int pmb_ow_set_controls(pmb_ow* h, const double* h_well_val) {
  return guarded([&] {
    PMB_REQUIRE(h && (h_well_val || h->m->view().nw == 0), "NULL argument");
    h->m->set_well_values(h_well_val);
  });
}

int pmb_ow_assemble(pmb_ow* h, const double* d_x, const double* d_x0, double dt, const double* d_cdp,
                    double* d_res, double* d_jac, double* d_well, int32_t want_jac) {
  return guarded([&] {
    PMB_REQUIRE(h, "NULL handle");
    PMB_REQUIRE(dt > 0.0, "dt must be positive");
    require_aligned(d_x, 16, "x");
    require_aligned(d_x0, 16, "x0");
    require_aligned(d_res, 16, "res");
    if (want_jac) {
      require_aligned(d_jac, 32, "jac");
      PMB_REQUIRE(d_well, "well part is NULL");
    }
    PMB_REQUIRE(h->m->nperf() == 0 || d_cdp, "cdp is NULL");
    h->m->assemble(d_x, d_x0, dt, d_cdp, d_res, d_jac, d_well, want_jac != 0);
  });
}

int pmb_ow_spmv(pmb_ow* h, const double* d_jac, const double* d_well, const double* d_x, double* d_y) {
  return guarded([&] {
    PMB_REQUIRE(h, "NULL handle");
    require_aligned(d_jac, 32, "jac");
    require_aligned(d_x, 16, "x");
    require_aligned(d_y, 16, "y");
    PMB_REQUIRE(d_well, "well part is NULL");
    PMB_REQUIRE(d_x != d_y, "x and y must not alias");
    h->m->spmv(d_jac, d_well, d_x, d_y);
  });
}

int pmb_ow_convergence(pmb_ow* h, const double* d_res, const double* d_x, double dt, double* out8) {
  return guarded([&] {
    PMB_REQUIRE(h && out8, "NULL argument");
    require_aligned(d_res, 16, "res");
    require_aligned(d_x, 16, "x");
    OWModel& m = *h->m;
    m.convergence_async(d_res, d_x, dt, m.conv_out());
    PMB_CUDA(cudaMemcpyAsync(h->conv.get(), m.conv_out(), 8 * sizeof(double), cudaMemcpyDeviceToHost, m.stream()));
    PMB_CUDA(cudaStreamSynchronize(m.stream()));
    for (int i = 0; i < 8; ++i) out8[i] = h->conv[i];
  });
}

int pmb_ow_update(pmb_ow* h, double* d_x, const double* d_dx, double sign) {
  return guarded([&] {
    PMB_REQUIRE(h, "NULL handle");
    require_aligned(d_x, 16, "x");
    require_aligned(d_dx, 16, "dx");
    h->m->update(d_x, d_dx, sign);
  });
}

int pmb_cpr_default_opts(pmb_cpr_opts* o) {
  return guarded([&] {
    PMB_REQUIRE(o, "NULL argument");
    o->rtol = 1e-8;
    o->maxiter = 200;
    o->restart = 50;
    o->precision = 0;
    o->use_pressure_stage = 1;
    o->local_sweeps = 4;
    o->amg_smoother_degree = 2;
    o->amg_cycle = 3;
    o->amg_theta = 0.1;
    o->amg_coarse_size = 200;
    o->amg_rebuild_interval = 8;
    o->inner_rtol = 1e-4;
    o->replay_graph = 1;
    o->amg_coarse_degree = 0;
  });
}

int pmb_cpr_create(pmb_ow* model, const pmb_cpr_opts* opts, pmb_cpr** out) {
  return guarded([&] {
    PMB_REQUIRE(model && opts && out, "NULL argument");
    *out = nullptr;
    auto s = std::make_unique<pmb_cpr>();
    s->owner = model;
    s->s = std::make_unique<CPRSolver>(*model->m, *opts);
    *out = s.release();
  });
}

int pmb_cpr_destroy(pmb_cpr* s) {
  return guarded([&] { delete s; });
}

int pmb_cpr_setup(pmb_cpr* s, const double* d_jac, const double* d_well, const double* d_x) {
  return guarded([&] {
    PMB_REQUIRE(s, "NULL handle");
    require_aligned(d_jac, 32, "jac");
    require_aligned(d_x, 16, "x");
    PMB_REQUIRE(d_well, "well part is NULL");
    s->s->setup(d_jac, d_well, d_x);
  });
}

int pmb_cpr_solve(pmb_cpr* s, const double* d_b, double* d_x, double* info4) {
  int rc = guarded([&] {
    PMB_REQUIRE(s && info4, "NULL argument");
    require_aligned(d_b, 16, "b");
    require_aligned(d_x, 16, "x");
    PMB_REQUIRE(d_b != d_x, "b and x must not alias");
    if (!s->s->solve(d_b, d_x, info4))
      throw Error(PMB_ERR_NOCONV, "CPR-GMRES did not reach its tolerance (relres " +
                                      std::to_string(info4[1]) + " after " +
                                      std::to_string((long long)info4[0]) + " iterations)");
  });
  return rc;
}

int pmb_cpr_levels(const pmb_cpr* s, int32_t max_levels, int64_t* sizes, int32_t* n_levels) {
  return guarded([&] {
    PMB_REQUIRE(s && sizes && n_levels, "NULL argument");
    const int nl = s->s->num_levels();
    *n_levels = nl;
    for (int l = 0; l < nl && l < max_levels; ++l) sizes[l] = s->s->level_size(l);
  });
}

int pmb_cpr_bytes(const pmb_cpr* s, double* h_out8) {
  return guarded([&] {
    PMB_REQUIRE(s && h_out8, "NULL argument");
    s->s->bytes(h_out8);
  });
}

int pmb_cpr_time_level(pmb_cpr* s, int32_t level, int32_t reps, double* h_ms, int64_t* h_nnz) {
  return guarded([&] {
    PMB_REQUIRE(s && h_ms && h_nnz, "NULL argument");
    long long nnz = 0;
    *h_ms = s->s->time_level(level, reps, &nnz);
    *h_nnz = nnz;
  });
}

int pmb_cpr_time_stage(pmb_cpr* s, int32_t stage, const double* d_r, double* d_z, int32_t reps,
                       double* h_ms) {
  return guarded([&] {
    PMB_REQUIRE(s && d_r && d_z && h_ms, "NULL argument");
    PMB_REQUIRE(stage >= 0 && stage <= 3, "stage must be 0, 1, 2 or 3");
    PMB_REQUIRE(reps >= 1, "reps must be positive");
    require_aligned(d_r, 16, "r");
    require_aligned(d_z, 16, "z");
    *h_ms = s->s->time_stage(stage, d_r, d_z, reps);
  });
}

int pmb_ow_step(pmb_ow* h, pmb_cpr* s, double* d_x, double dt, int32_t max_iterations, double* stats) {
  return guarded([&] {
    PMB_REQUIRE(h && s && stats, "NULL argument");
    PMB_REQUIRE(s->owner == h, "solver belongs to another model");
    PMB_REQUIRE(dt > 0.0, "dt must be positive");
    PMB_REQUIRE(max_iterations >= 0, "negative iteration limit");
    require_aligned(d_x, 16, "x");
    OWModel& m = *h->m;
    CPRSolver& cpr = *s->s;
    cudaStream_t st = m.stream();
    const long long n = m.nvec();
    for (int i = 0; i < 8; ++i) stats[i] = 0.0;
    PMB_CUDA(cudaMemcpyAsync(m.x0(), d_x, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    m.compute_cdp(m.x0(), m.cdp());
    double krylov = 0.0, soft = 0.0;
    // a solve that stopped above rtol but this close to exact still makes a
    // Newton update
    constexpr double kUsableRelres = 1e-6;
    auto evaluate = [&](bool want_jac) {
      {
        PhaseTimer pt("newton.assemble", st);
        m.assemble(d_x, m.x0(), dt, m.cdp(), m.res(), m.jac(), m.well(), want_jac);
      }
      PhaseTimer pt("newton.convergence", st);
      m.convergence_async(m.res(), d_x, dt, m.conv_out());
      PMB_CUDA(cudaMemcpyAsync(h->conv.get(), m.conv_out(), 8 * sizeof(double), cudaMemcpyDeviceToHost, st));
      PMB_CUDA(cudaStreamSynchronize(st));
    };
    for (int it = 0; it < max_iterations; ++it) {
      evaluate(true);
      stats[4] = h->conv[0];
      stats[5] = h->conv[1];
      stats[6] = h->conv[6];
      if (h->conv[5] != 0.0) {
        stats[0] = it;
        stats[1] = 1.0;
        stats[2] = krylov;
        stats[3] = (double)cpr.setups();
        stats[7] = soft;
        return;
      }
      if (h->conv[6] != 0.0) break;  // non-finite residual: the step fails
      {
        PhaseTimer pt("newton.cpr_setup", st);
        cpr.setup(m.jac(), m.well(), d_x);
      }
      double info[4];
      bool ok;
      {
        PhaseTimer pt("newton.cpr_solve", st);
        ok = cpr.solve(m.res(), m.dx(), info);
      }
      static const bool trace = [] {
        const char* e = std::getenv("PMB_NEWTON_TRACE");
        return e && e[0] == '1';
      }();
      if (trace)
        std::fprintf(stderr, "# newton it=%d cnv=%.3e mb=%.3e well_w=%.3e well_o=%.3e ctrl_ok=%g krylov=%g relres=%.2e\n",
                     it, h->conv[0], h->conv[1], h->conv[2], h->conv[3], h->conv[4], info[0], info[1]);
      krylov += info[0];
      if (!ok && std::isfinite(info[1]) && info[1] <= kUsableRelres) {
        ok = true;  // close enough to an exact solve: let the Newton test decide
        soft += 1.0;
      }
      if (!ok) {
        PMB_CUDA(cudaMemcpyAsync(d_x, m.x0(), sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
        PMB_CUDA(cudaStreamSynchronize(st));
        stats[0] = it;
        stats[2] = krylov;
        stats[3] = (double)cpr.setups();
        throw Error(PMB_ERR_NOCONV, "CPR-GMRES did not converge in Newton iteration " + std::to_string(it) +
                                        " (relres " + std::to_string(info[1]) + ")");
      }
      m.update(d_x, m.dx(), -1.0);
    }
    if (h->conv[6] == 0.0) evaluate(false);
    stats[0] = max_iterations;
    stats[1] = h->conv[5] != 0.0 ? 1.0 : 0.0;
    stats[2] = krylov;
    stats[3] = (double)cpr.setups();
    stats[4] = h->conv[0];
    stats[5] = h->conv[1];
    stats[6] = h->conv[6];
    stats[7] = soft;
  });
}

int pmb_ow_step_members(pmb_ow* h, pmb_cpr* s, double* d_x, double dt, int32_t max_iterations, int32_t nmem,
                        const int32_t* h_cell_ptr, const int32_t* h_well_ptr, int32_t* h_state, int32_t* h_its,
                        double* h_stats4) {
  return guarded([&] {
    PMB_REQUIRE(h && s && h_cell_ptr && h_well_ptr && h_state && h_its && h_stats4, "NULL argument");
    PMB_REQUIRE(s->owner == h, "solver belongs to another model");
    PMB_REQUIRE(dt > 0.0, "dt must be positive");
    PMB_REQUIRE(max_iterations >= 0, "negative iteration limit");
    PMB_REQUIRE(nmem >= 1, "need at least one member");
    require_aligned(d_x, 16, "x");
    OWModel& m = *h->m;
    const OWView v = m.view();
    PMB_REQUIRE(h_cell_ptr[0] == 0 && h_cell_ptr[nmem] == v.nc, "member cell ranges must cover the cells");
    PMB_REQUIRE(h_well_ptr[0] == 0 && h_well_ptr[nmem] == v.nw, "member well ranges must cover the wells");
    for (int k = 0; k < nmem; ++k) {
      PMB_REQUIRE(h_cell_ptr[k + 1] > h_cell_ptr[k], "every member needs cells");
      PMB_REQUIRE(h_well_ptr[k + 1] >= h_well_ptr[k], "member well ranges must be non-decreasing");
    }
    CPRSolver& cpr = *s->s;
    cudaStream_t st = m.stream();
    const long long n = m.nvec();
    if ((int)h->mem_flag.size() != nmem) {
      h->mem_cell.resize(nmem + 1);
      h->mem_well.resize(nmem + 1);
      h->mem_flag.resize(nmem);
      h->mem_conv.resize(8LL * nmem);
      h->mem_conv_h.resize(8LL * nmem);
      h->mem_flag_h.resize(nmem);
    }
    PMB_CUDA(cudaMemcpyAsync(h->mem_cell.get(), h_cell_ptr, sizeof(int) * (nmem + 1), cudaMemcpyHostToDevice, st));
    PMB_CUDA(cudaMemcpyAsync(h->mem_well.get(), h_well_ptr, sizeof(int) * (nmem + 1), cudaMemcpyHostToDevice, st));
    // h_state in: 1 take the step, 0 frozen.  Working state: 1 active,
    // 2 converged, 3 failed, 0 frozen.
    std::vector<int> state(nmem);
    for (int k = 0; k < nmem; ++k) {
      state[k] = h_state[k] != 0 ? 1 : 0;
      h_its[k] = 0;
    }
    for (int i = 0; i < 4; ++i) h_stats4[i] = 0.0;
    PMB_CUDA(cudaMemcpyAsync(m.x0(), d_x, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    m.compute_cdp(m.x0(), m.cdp());
    double krylov = 0.0;
    auto evaluate = [&](bool want_jac) {
      m.assemble(d_x, m.x0(), dt, m.cdp(), m.res(), m.jac(), m.well(), want_jac);
      m.member_convergence_async(nmem, h->mem_cell.get(), h->mem_well.get(), m.res(), d_x, dt, h->mem_conv.get());
      PMB_CUDA(cudaMemcpyAsync(h->mem_conv_h.get(), h->mem_conv.get(), sizeof(double) * 8 * nmem,
                               cudaMemcpyDeviceToHost, st));
      PMB_CUDA(cudaStreamSynchronize(st));
    };
    auto classify = [&](int it) {  // returns the number of members still active
      int active = 0;
      for (int k = 0; k < nmem; ++k) {
        if (state[k] != 1) continue;
        const double* c = h->mem_conv_h.get() + 8LL * k;
        if (c[5] != 0.0) {
          state[k] = 2;
          h_its[k] = it;
        } else if (c[6] != 0.0) {
          state[k] = 3;  // non-finite residual: the member's step fails
          h_its[k] = it;
        } else {
          ++active;
        }
      }
      return active;
    };
    int it = 0;
    int active = 0;
    for (; it < max_iterations; ++it) {
      evaluate(true);
      active = classify(it);
      if (active == 0) break;
      for (int k = 0; k < nmem; ++k) h->mem_flag_h[k] = state[k] == 1 ? 1 : 0;
      PMB_CUDA(cudaMemcpyAsync(h->mem_flag.get(), h->mem_flag_h.get(), sizeof(int) * nmem, cudaMemcpyHostToDevice,
                               st));
      // members that are not active get a zero right-hand side, hence a zero
      // correction: the preconditioner never couples members
      m.mask_members(nmem, h->mem_cell.get(), h->mem_well.get(), h->mem_flag.get(), m.res());
      cpr.setup(m.jac(), m.well(), d_x);
      double info[4];
      const bool ok = cpr.solve(m.res(), m.dx(), info);
      krylov += info[0];
      static const bool trace = [] {
        const char* e = std::getenv("PMB_NEWTON_TRACE");
        return e && e[0] == '1';
      }();
      if (trace) std::fprintf(stderr, "# members it=%d active=%d krylov=%g relres=%.2e ok=%d\n", it, active, info[0],
                              info[1], (int)ok);
      if (!ok) {
        // The shared solve missed its tolerance.  A member whose own block of
        // the linear residual meets it has the update a solve of its system
        // alone would accept: it goes on; the others fail this step.
        if (h->mem_lin.size() != (size_t)m.nvec()) h->mem_lin.resize(m.nvec());
        if (h->mem_linres.size() != 2 * (size_t)nmem) {
          h->mem_linres.resize(2LL * nmem);
          h->mem_linres_h.resize(2LL * nmem);
        }
        m.member_linear_residuals_async(nmem, h->mem_cell.get(), h->mem_well.get(), m.res(), m.dx(),
                                        h->mem_lin.get(), h->mem_linres.get());
        PMB_CUDA(cudaMemcpyAsync(h->mem_linres_h.get(), h->mem_linres.get(), sizeof(double) * 2 * nmem,
                                 cudaMemcpyDeviceToHost, st));
        PMB_CUDA(cudaStreamSynchronize(st));
        const double tol2 = cpr.opts().rtol * cpr.opts().rtol;
        int kept = 0;
        for (int k = 0; k < nmem; ++k) {
          if (state[k] != 1) continue;
          const double rr = h->mem_linres_h[2 * k], bb = h->mem_linres_h[2 * k + 1];
          if (std::isfinite(rr) && rr <= tol2 * bb) {
            ++kept;
          } else {
            state[k] = 3;
            h_its[k] = it;
          }
        }
        if (trace) std::fprintf(stderr, "# members it=%d kept %d of %d after the shared solve failed\n", it, kept,
                                active);
        active = kept;
        if (kept == 0) break;
        for (int k = 0; k < nmem; ++k) h->mem_flag_h[k] = state[k] == 1 ? 1 : 0;
        PMB_CUDA(cudaMemcpyAsync(h->mem_flag.get(), h->mem_flag_h.get(), sizeof(int) * nmem,
                                 cudaMemcpyHostToDevice, st));
      }
      m.mask_members(nmem, h->mem_cell.get(), h->mem_well.get(), h->mem_flag.get(), m.dx());
      m.update(d_x, m.dx(), -1.0);
    }
    if (active > 0) {  // iteration limit: one more check, as the reference's step makes
      evaluate(false);
      for (int k = 0; k < nmem; ++k)
        if (state[k] == 1) {
          const double* c = h->mem_conv_h.get() + 8LL * k;
          state[k] = c[5] != 0.0 ? 2 : 3;
          h_its[k] = max_iterations;
        }
    }
    // failed members go back to the start of the step
    for (int k = 0; k < nmem; ++k) {
      if (state[k] != 3) continue;
      const long long c0 = h_cell_ptr[k], c1 = h_cell_ptr[k + 1];
      PMB_CUDA(cudaMemcpyAsync(d_x + 2 * c0, m.x0() + 2 * c0, sizeof(double) * 2 * (c1 - c0),
                               cudaMemcpyDeviceToDevice, st));
      const long long w0 = h_well_ptr[k], w1 = h_well_ptr[k + 1];
      if (w1 > w0)
        PMB_CUDA(cudaMemcpyAsync(d_x + 2LL * v.nc + 3 * w0, m.x0() + 2LL * v.nc + 3 * w0,
                                 sizeof(double) * 3 * (w1 - w0), cudaMemcpyDeviceToDevice, st));
    }
    PMB_CUDA(cudaStreamSynchronize(st));
    for (int k = 0; k < nmem; ++k) h_state[k] = state[k] == 2 ? 1 : (state[k] == 3 ? 0 : -1);
    h_stats4[0] = krylov;
    h_stats4[1] = (double)cpr.setups();
    h_stats4[2] = it;
    h_stats4[3] = 0.0;
  });
}

int pmb_amg_hierarchy_host(int32_t n, const int32_t* row_ptr, const int32_t* col, const double* val,
                           double theta, int32_t coarse_size, int32_t max_levels, int64_t* sizes,
                           int32_t* n_levels) {
  return guarded([&] {
    PMB_REQUIRE(n > 0 && row_ptr && col && val && sizes && n_levels, "invalid argument");
    auto H = amg_build_hierarchy(n, row_ptr, col, val, theta, 2, coarse_size, 40);
    *n_levels = (int)H.size();
    for (int l = 0; l < (int)H.size() && l < max_levels; ++l) sizes[l] = H[l].n;
    // consistency of every level's aggregation and Galerkin map
    for (size_t l = 0; l + 1 < H.size(); ++l) {
      const AMGHostLevel& L = H[l];
      const int nc = H[l + 1].n;
      for (int a : L.agg) PMB_REQUIRE(a >= 0 && a < nc, "aggregate index out of range");
      PMB_REQUIRE((int)L.cmem.size() == L.n, "aggregates do not partition the unknowns");
      PMB_REQUIRE((int)L.gidx.size() == (int)L.col.size(), "Galerkin map does not cover every entry");
    }
  });
}

}  // extern "C"
