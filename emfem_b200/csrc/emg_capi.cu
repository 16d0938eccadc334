// C ABI of emfem_b200 (include/emfem_b200.h).  Each entry point validates its
// arguments, runs the host/device work on the context's stream and converts
// exceptions into status codes with a thread-local message.

#include <nvtx3/nvToolsExt.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <sstream>
#include <string>
#include <array>
#include <atomic>
#include <chrono>

#include "emg_api.h"
#include "emg_internal.h"
#include "emg_kernels.cuh"
#include "emg_linalg.h"
#include "emg_locate.h"
#include "emg_io.h"
#include "emg_solver.h"

namespace emg {

static thread_local std::string g_last_error;

void set_last_error(const char *msg) { g_last_error = msg ? msg : ""; }

void fail(int code, const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  throw Error(code, buf);
}

static std::atomic<long> g_launches{0};
long launch_count() { return g_launches.load(); }
void add_launches(long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

void launch_check(const char *file, int line) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  check_cuda(cudaGetLastError(), "kernel launch", file, line);
}

KernelProfiler &profiler() {
  static KernelProfiler p;
  return p;
}

// every profiled bin is also an NVTX range of its name, so that a profiler
// can select the launches of one bin (ncu --nvtx --nvtx-include "bin/")
void KernelProfiler::begin(const std::string &bin, cudaStream_t s, double algo_bytes, cudaEvent_t *start_out) {
  nvtxRangePushA(bin.c_str());
  cudaEvent_t a, b;
  EMG_CUDA(cudaEventCreate(&a));
  EMG_CUDA(cudaEventCreate(&b));
  EMG_CUDA(cudaEventRecord(a, s));
  open[bin].push_back(Rec{a, b, algo_bytes});
  *start_out = a;
}

void KernelProfiler::end(const std::string &bin, cudaStream_t s, cudaEvent_t start) {
  auto &v = open[bin];
  if (v.empty() || v.back().a != start) fail(EMG_ERR_STATE, "profiler: unbalanced records");
  EMG_CUDA(cudaEventRecord(v.back().b, s));
  nvtxRangePop();
}

void KernelProfiler::collect() {
  for (auto &kv : open) {
    for (auto &r : kv.second) {
      EMG_CUDA(cudaEventSynchronize(r.b));
      float t = 0;
      EMG_CUDA(cudaEventElapsedTime(&t, r.a, r.b));
      ms[kv.first] += t;
      bytes[kv.first] += r.bytes;
      count[kv.first] += 1;
      cudaEventDestroy(r.a);
      cudaEventDestroy(r.b);
    }
    kv.second.clear();
  }
}

void KernelProfiler::reset() {
  collect();
  ms.clear();
  bytes.clear();
  count.clear();
}

void check_cuda(cudaError_t e, const char *what, const char *file, int line) {
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    fail(e == cudaErrorMemoryAllocation ? EMG_ERR_NOMEM : EMG_ERR_CUDA, "%s failed at %s:%d: %s", what, file, line,
         cudaGetErrorString(e));
  }
}

// launchers defined in emg_estimate.cu
void launch_estimate(Context &c, double omega, int nsol, const double *const *sol_dev, double *eta_dev,
                     double *err_dev, double *scratch_vol, double *scratch_fe);
void launch_rhs_mt(Context &c, int k, const double *omega_dev, const double *bv_dev, const int *brank_dev,
                   double *s_dev);

struct Workspace {
  Fcg<double> fcg64;
  Fcg<float> fcg32;
  Fgmres gm;
  DBuf<double> vec_a, vec_b;       // host<->device staging of complex block vectors
  DBuf<float> f_in, f_out;         // FP32 inner vectors
  DBuf<double> est_vol, est_fe, est_eta, est_err;
  DBuf<double> bvals, omega_k, omega_cols;
  DBuf<double> blk_rhs, blk_x;     // one padded block of a wider or ragged solve
  // plain path: hierarchy of B(w) for the assembled frequency (create_pc)
  Ams<double> pams64;
  // batched path: two-part hierarchy valid for every frequency of a block
  bool block_ready64 = false, block_ready32 = false;
  Ams<double> bams64;
  Ams<float> bams32;
  // divergence correction of the batched path
  Fcg<double> fcg_div;
  DBuf<double> div_d, div_dis, div_ds;          // nv: l1 scale, its -1/2 and 1/2 powers (0 on the boundary)
  DBuf<double> div_rhs, div_y, div_t, div_u;    // nv x K2
  DBuf<double> div_e, div_me;                   // ne x K2
  DBuf<float> div_tf, div_uf;                   // nv x K2, the FP32 hierarchy's operands
};

Context::Context() : ws(new Workspace()) {}
Context::~Context() {
  ws.reset();
  if (stream) cudaStreamDestroy(stream);
}

// ---------------------------------------------------------------------------
// options (process_options, src/em_ctx.cc:100-175)
// ---------------------------------------------------------------------------
static bool is_number(const std::string &s) {
  if (s.empty()) return false;
  char *end = nullptr;
  std::strtod(s.c_str(), &end);
  return end && *end == '\0';
}

static void parse_options(Options &o, const std::string &text, std::vector<std::string> &ignored) {
  std::vector<std::string> tok;
  std::istringstream ls(text);
  std::string line;
  while (std::getline(ls, line)) {
    size_t h = line.find('#');
    if (h != std::string::npos) line.erase(h);
    std::istringstream ws(line);
    std::string t;
    while (ws >> t) tok.push_back(t);
  }
  auto geti = [](const std::string &k, const std::string &v) {
    if (!is_number(v)) fail(EMG_ERR_OPTION, "option %s expects a number, got '%s'", k.c_str(), v.c_str());
    return (int)std::lround(std::strtod(v.c_str(), nullptr));
  };
  auto getr = [](const std::string &k, const std::string &v) {
    if (!is_number(v)) fail(EMG_ERR_OPTION, "option %s expects a number, got '%s'", k.c_str(), v.c_str());
    return std::strtod(v.c_str(), nullptr);
  };
  auto elist = [](const std::string &k, const std::string &v, std::initializer_list<const char *> names) {
    int i = 0;
    for (const char *n : names) {
      if (v == n) return i;
      ++i;
    }
    fail(EMG_ERR_OPTION, "option %s: unknown value '%s'", k.c_str(), v.c_str());
  };
  auto getb = [](const std::string &v) { return !(v == "0" || v == "false" || v == "FALSE" || v == "no"); };
  for (size_t i = 0; i < tok.size(); ++i) {
    const std::string &k = tok[i];
    if (k.size() < 2 || k[0] != '-' || is_number(k)) fail(EMG_ERR_OPTION, "unexpected token '%s'", k.c_str());
    std::string v;
    if (i + 1 < tok.size() && (tok[i + 1][0] != '-' || is_number(tok[i + 1]))) v = tok[++i];
    std::string key = k.substr(1);
    if (key == "iprefix") o.iprefix = v;
    else if (key == "oprefix") o.oprefix = v;
    else if (key == "n_groups") o.n_groups = geti(k, v);
    else if (key == "max_tx_edge_length") o.max_tx_edge_length = getr(k, v);
    else if (key == "max_rx_edge_length") o.max_rx_edge_length = getr(k, v);
    else if (key == "mesh_format") o.mesh_format = elist(k, v, {"mdl", "mesh"});
    else if (key == "inner_pc_type") o.inner_pc_type = elist(k, v, {"mixed", "ams", "direct"});
    else if (key == "pc_threshold") o.pc_threshold = geti(k, v);
    else if (key == "direct_solver_type") o.direct_solver_type = elist(k, v, {"mumps", "superlu_dist"});
    else if (key == "K_max_it") o.K_max_it = geti(k, v);
    else if (key == "e_rtol") o.e_rtol = getr(k, v);
    else if (key == "dual_rtol") o.dual_rtol = getr(k, v);
    else if (key == "max_adaptive_refinements") o.max_adaptive_refinements = geti(k, v);
    else if (key == "n_uniform_refinements") o.n_uniform_refinements = geti(k, v);
    else if (key == "max_dofs") o.max_dofs = geti(k, v);
    else if (key == "refine_fraction") o.refine_fraction = getr(k, v);
    else if (key == "refine_strategy") o.refine_strategy = elist(k, v, {"fixed_number", "fixed_fraction"});
    else if (key == "save_mesh") o.save_mesh = v.empty() ? 1 : getb(v);
    else if (key == "n_tx_divisions") o.n_tx_divisions = geti(k, v);
    else if (key == "options_file") ;
    // A_ (outer) and B_ (inner) prefixes: the subset the GPU solver implements
    else if (key == "A_ksp_gmres_restart") o.gmres_restart = geti(k, v);
    else if (key == "B_ksp_rtol") o.inner_rtol = getr(k, v);
    else if (key == "B_ksp_max_it") o.inner_max_it = geti(k, v);
    else if (key == "B_ksp_fcg_mmax") o.fcg_mmax = geti(k, v);
    else if (key == "B_pc_hypre_ams_cycle_type") {
      int ct = geti(k, v);
      // hypre's multiplicative AMS cycles: 0 edge smoothing, 1 gradient
      // space, 2 vector Pi space, 3/4/5 its x/y/z components
      if (ct == 1) o.ams_cycle = "01210";
      else if (ct == 3) o.ams_cycle = "02120";
      else if (ct == 5) o.ams_cycle = "0102010";
      else if (ct == 7) o.ams_cycle = "0201020";
      else if (ct == 11) o.ams_cycle = "013454310";
      else if (ct == 13) o.ams_cycle = "034515430";
      else fail(EMG_ERR_OPTION, "AMS cycle type %d is not implemented (1, 3, 5, 7, 11 and 13 are)", ct);
    } else if (key == "B_pc_hypre_ams_relax_times") o.ams_relax_times = geti(k, v);
    else if (key == "B_pc_hypre_ams_relax_weight") o.ams_relax_weight = getr(k, v);
    else if (key == "B_pc_hypre_ams_amg_alpha_theta" || key == "B_pc_hypre_ams_amg_beta_theta") o.amg_theta = getr(k, v);
    // emg_* keys of this implementation
    else if (key == "emg_inner_precision") o.inner_fp32 = elist(k, v, {"fp64", "fp32"});
    else if (key == "emg_amg_max_coarse") o.amg_max_coarse = geti(k, v);
    else if (key == "emg_amg_max_levels") o.amg_max_levels = geti(k, v);
    else if (key == "emg_amg_relax_times") o.amg_relax_times = geti(k, v);
    else if (key == "emg_amg_pmax") o.amg_pmax = geti(k, v);
    else if (key == "emg_smoother") o.smoother_cheb = elist(k, v, {"l1jacobi", "chebyshev"});
    else if (key == "emg_fp32_cycle") o.fp32_cycle = v;
    else if (key == "emg_graphs") o.graphs = v.empty() ? 1 : getb(v);
    else if (key == "emg_fused_vcycle") o.ams_fused = v.empty() ? 1 : getb(v);
    else if (key == "emg_fused_blocks_per_sm") o.fused_bps = geti(k, v);
    else if (key == "emg_fused_rows") o.fused_rows = geti(k, v);
    else if (key == "emg_gpu_amg") o.gpu_amg = v.empty() ? 1 : getb(v);
    else if (key == "emg_block_fp64_fallback") o.block_fp64_fallback = v.empty() ? 1 : getb(v);
    else if (key == "emg_block_fp32_rtol_factor") o.block_fp32_rtol_factor = getr(k, v);
    else if (key == "emg_block_fp64_below") o.block_fp64_below_hz = getr(k, v);
    else if (key == "emg_div_correction") o.div_correction = v.empty() ? 1 : getb(v);
    else if (key == "emg_div_rtol") o.div_rtol = getr(k, v);
    else if (key == "emg_div_max_it") o.div_max_it = geti(k, v);
    else if (key == "emg_fused_wait_ms") o.fused_wait_ms = getr(k, v);
    else if (key == "emg_fused_test_withhold") o.fused_test_withhold = geti(k, v);
    else if (key == "emg_pi_coupled") o.pi_coupled = v.empty() ? 1 : getb(v);
    else if (key == "emg_block_inner_rtol") o.block_inner_rtol = getr(k, v);
    else if (key == "emg_block_inner_max_it") o.block_inner_max_it = geti(k, v);
    else if (key == "emg_block_fcg_mmax") o.block_fcg_mmax = geti(k, v);
    else if (key == "emg_block_fcg_check_every") o.block_fcg_check_every = geti(k, v);
    else if (key == "emg_block_relax_times") o.block_relax_times = geti(k, v);
    else if (key == "emg_cheb_degree") o.cheb_degree = geti(k, v);
    else if (key == "emg_block_cheb_degree") o.block_cheb_degree = geti(k, v);
    else if (key == "emg_amg_cheb_degree") o.amg_cheb_degree = geti(k, v);
    else if (key == "emg_restrict_smooth") o.restrict_j0 = v.empty() ? 1 : getb(v);
    else if (key == "emg_block_floor_stop") o.block_floor_stop = v.empty() ? 1 : getb(v);
    else if (key == "emg_amg_pre_smooth") o.amg_pre_smooth = v.empty() ? 1 : getb(v);
    else if (key == "emg_spmm_tiled") o.spmm_tiled = v.empty() ? 1 : getb(v);
    else if (key == "emg_tiled_smem_kb") o.tiled_smem_kb = geti(k, v);
    else if (key == "emg_verbose") o.verbose = v.empty() ? 1 : geti(k, v);
    else if (key.rfind("A_", 0) == 0 || key.rfind("B_", 0) == 0) ignored.push_back(k);
    else fail(EMG_ERR_OPTION, "unknown option %s", k.c_str());
  }
  if (o.gmres_restart < 1 || o.gmres_restart > 128) fail(EMG_ERR_OPTION, "A_ksp_gmres_restart must be in [1, 128]");
  if (o.block_fcg_check_every < 1) fail(EMG_ERR_OPTION, "-emg_block_fcg_check_every must be >= 1");
  if (o.div_max_it < 1 || !(o.div_rtol > 0)) fail(EMG_ERR_OPTION, "-emg_div_max_it must be >= 1, -emg_div_rtol > 0");
  if (!(o.block_fp32_rtol_factor > 0 && o.block_fp32_rtol_factor <= 1))
    fail(EMG_ERR_OPTION, "-emg_block_fp32_rtol_factor must be in (0, 1]");
  if (o.fcg_mmax < 1 || o.fcg_mmax > 30 || o.block_fcg_mmax < 1 || o.block_fcg_mmax > 30)
    fail(EMG_ERR_OPTION, "FCG truncation lengths must be in [1, 30]");
  if (o.cheb_degree < 2 || o.cheb_degree > 6 || o.block_cheb_degree < 2 || o.block_cheb_degree > 6 ||
      o.amg_cheb_degree < 2 || o.amg_cheb_degree > 6)
    fail(EMG_ERR_OPTION, "Chebyshev degrees (-emg_cheb_degree, -emg_block_cheb_degree, -emg_amg_cheb_degree) must be "
                         "in [2, 6]");
  if (o.ams_relax_times < 1 || o.amg_relax_times < 1 || o.block_relax_times < 1)
    fail(EMG_ERR_OPTION, "relax times must be >= 1");
  if (o.inner_max_it < 1 || o.block_inner_max_it < 1) fail(EMG_ERR_OPTION, "inner iteration caps must be >= 1");
  if (!(o.inner_rtol > 0) || !(o.block_inner_rtol > 0)) fail(EMG_ERR_OPTION, "inner tolerances must be > 0");
  if (o.tiled_smem_kb < 4 || o.tiled_smem_kb > 227) fail(EMG_ERR_OPTION, "emg_tiled_smem_kb must be in [4, 227]");
}

// ---------------------------------------------------------------------------
// host FE helpers for the sparse RHS pieces (dipoles, receivers, boundary
// values): gradients of the barycentric coordinates of one tet
// ---------------------------------------------------------------------------
struct HostTet {
  double x[4][3], gr[4][3], vol;
  int v[4];
};

static void host_tet(const Context &c, int t, HostTet &h) {
  for (int i = 0; i < 4; ++i) {
    h.v[i] = c.h_tets[4 * (size_t)t + i];
    for (int d = 0; d < 3; ++d) h.x[i][d] = c.h_pts[3 * (size_t)h.v[i] + d];
  }
  double e1[3], e2[3], e3[3];
  for (int d = 0; d < 3; ++d) {
    e1[d] = h.x[1][d] - h.x[0][d];
    e2[d] = h.x[2][d] - h.x[0][d];
    e3[d] = h.x[3][d] - h.x[0][d];
  }
  double c23[3] = {e2[1] * e3[2] - e2[2] * e3[1], e2[2] * e3[0] - e2[0] * e3[2], e2[0] * e3[1] - e2[1] * e3[0]};
  double c31[3] = {e3[1] * e1[2] - e3[2] * e1[1], e3[2] * e1[0] - e3[0] * e1[2], e3[0] * e1[1] - e3[1] * e1[0]};
  double c12[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
  double det = e1[0] * c23[0] + e1[1] * c23[1] + e1[2] * c23[2];
  for (int d = 0; d < 3; ++d) {
    h.gr[1][d] = c23[d] / det;
    h.gr[2][d] = c31[d] / det;
    h.gr[3][d] = c12[d] / det;
    h.gr[0][d] = -(h.gr[1][d] + h.gr[2][d] + h.gr[3][d]);
  }
  h.vol = det / 6.0;
}

static double host_lambda(const HostTet &h, int p, const double *y) {
  return 1.0 + h.gr[p][0] * (y[0] - h.x[p][0]) + h.gr[p][1] * (y[1] - h.x[p][1]) + h.gr[p][2] * (y[2] - h.x[p][2]);
}

// local edge i of tet t: value of phi_i at y (global orientation lower->higher id)
static void host_phi(const Context &c, const HostTet &h, int t, int i, const double *y, double out[3], int *ge) {
  int e = c.h_t2e[6 * (size_t)t + i];
  int a = c.h_edges[2 * (size_t)e], b = c.h_edges[2 * (size_t)e + 1];
  int la = -1, lb = -1;
  for (int q = 0; q < 4; ++q) {
    if (h.v[q] == a) la = q;
    if (h.v[q] == b) lb = q;
  }
  if (la < 0 || lb < 0) fail(EMG_ERR_USER, "tet %d does not contain its edge %d", t, e);
  double l0 = host_lambda(h, la, y), l1 = host_lambda(h, lb, y);
  for (int d = 0; d < 3; ++d) out[d] = l0 * h.gr[lb][d] - l1 * h.gr[la][d];
  *ge = e;
}

// 1-D layered plane wave (src/em_pw.h:6-139)
struct PlaneWave1D {
  typedef std::complex<double> zc;
  int nlay = 0;
  double omega = 0;
  std::vector<double> ztop, lsig;
  std::vector<zc> a, b, cc, d;
  void init(const double *zt, const double *ls, int n, double freq) {
    const zc I(0, 1);
    nlay = n;
    ztop.assign(zt, zt + n);
    lsig.assign(ls, ls + n);
    omega = 2 * PI * freq;
    std::vector<zc> kk(n + 1), Rp(n + 1, 0.0), ex(n + 1, 0.0);
    for (int i = 1; i <= n; ++i) kk[i] = std::sqrt(-I * omega * MU * lsig[i - 1]);
    kk[0] = std::sqrt(-I * omega * MU * lsig[0]);
    for (int i = 1; i <= n - 1; ++i) ex[i] = std::exp(-kk[i] * (ztop[i] - ztop[i - 1]));
    for (int i = n - 1; i >= 1; --i) {
      zc gm = (-I * omega * MU * (lsig[i - 1] - lsig[i])) / ((kk[i] + kk[i + 1]) * (kk[i] + kk[i + 1]));
      zc rj = Rp[i + 1] * ex[i + 1];
      Rp[i] = (gm + rj) / (1.0 + gm * rj) * ex[i];
    }
    a.assign(n + 1, 0.0);
    b.assign(n + 1, 0.0);
    cc.assign(n + 1, 0.0);
    d.assign(n + 1, 0.0);
    a[0] = 1.0;
    cc[0] = 1.0;
    for (int i = 1; i <= n; ++i) {
      zc At = a[i - 1] + b[i - 1] * ex[i - 1];
      b[i] = At / (1.0 + Rp[i] * ex[i]);
      a[i] = b[i] * Rp[i];
      At = cc[i - 1] + d[i - 1] * ex[i - 1];
      d[i] = At / (1.0 - Rp[i] * ex[i]);
      cc[i] = -d[i] * Rp[i];
    }
  }
  void field(double z, zc eh[4]) const {
    const zc I(0, 1);
    int il = 0;
    for (int i = nlay - 1; i >= 0; --i)
      if (z >= ztop[i]) { il = i; break; }
    zc kk = std::sqrt(-I * omega * MU * lsig[il]);
    zc ep = 0.0, epd = 0.0;
    zc em = std::exp(-kk * (z - ztop[il]));
    zc emd = -kk * em;
    if (il != nlay - 1) {
      ep = std::exp(kk * (z - ztop[il + 1]));
      epd = kk * ep;
    }
    eh[0] = a[il + 1] * ep + b[il + 1] * em;
    eh[1] = (a[il + 1] * epd + b[il + 1] * emd) / (I * MU * omega);
    eh[2] = (cc[il + 1] * epd + d[il + 1] * emd) / lsig[il];
    eh[3] = cc[il + 1] * ep + d[il + 1] * em;
    for (int i = 0; i < 4; ++i)
      if (std::abs(eh[i]) < 1E-80) eh[i] = 0.0;
  }
};

// calculate_boundary_values (src/em_fwd.cc:402-486): Dirichlet value of every
// boundary edge (first encounter in ascending tet order wins)
const TiledPattern *tiled_pattern(Context &c, const int *rp_dev, const std::vector<int> &h_rp,
                                  const std::vector<int> &h_ci, int row_bytes) {
  if (!c.opt.spmm_tiled || h_rp.size() < 2) return nullptr;
  const auto key = std::make_pair(rp_dev, row_bytes);
  auto it = c.tiles.find(key);
  if (it != c.tiles.end()) return it->second.get();
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  EMG_CUDA(cudaStreamIsCapturing(c.stream, &cs));
  if (cs != cudaStreamCaptureStatusNone) fail(EMG_ERR_STATE, "tiled pattern first needed inside a capture");
  auto tp = std::make_unique<TiledPattern>();
  const int umax = (int)((long)c.opt.tiled_smem_kb * 1024 / row_bytes);
  const bool ok = build_tiled((int)h_rp.size() - 1, h_rp, h_ci, umax, 128, *tp, c.stream);
  const TiledPattern *res = ok ? tp.get() : nullptr;
  c.tiles[key] = ok ? std::move(tp) : nullptr;
  return res;
}

// Geometry of the MT boundary values (assemble_rhs_mt, src/em_fwd.cc:488-580)
// that does not depend on frequency or polarisation: per boundary edge its
// midpoint depth, the blend weights of the four corner soundings and the
// tangential components.  Each edge is evaluated in the lowest-numbered
// boundary tet that holds it, as the reference's tet loop does.
struct MtBoundary {
  std::vector<int> edge, zslot;
  std::vector<double> co, ed, den;  // 4, 2 and 1 per edge
  std::vector<double> zs;           // distinct midpoint depths
};

static void mt_boundary_geometry(Context &c, const std::vector<unsigned char> &bdr_cell, MtBoundary &g) {
  need(!c.bg_nlay.empty(), EMG_ERR_STATE, "MT right-hand side needs emg_set_background first");
  const double *tc = c.bg_corners.data();
  auto T = [&](int q, int d) { return tc[3 * q + d]; };
  std::vector<char> have(c.ne, 0);
  std::vector<int> tet, loc;
  g.edge.clear();
  for (int t = 0; t < c.nt; ++t) {
    if (!bdr_cell[t]) continue;
    for (int i = 0; i < 6; ++i) {
      int e = c.h_t2e[6 * (size_t)t + i];
      if (!c.h_ebdr[e] || have[e]) continue;
      have[e] = 1;
      g.edge.push_back(e);
      tet.push_back(t);
      loc.push_back(i);
    }
  }
  const int nb = (int)g.edge.size();
  std::vector<double> z(nb);
  g.co.assign(4 * (size_t)nb, 0.0);
  g.ed.assign(2 * (size_t)nb, 0.0);
  g.den.assign(nb, 0.0);
#pragma omp parallel for schedule(static)
  for (int b = 0; b < nb; ++b) {
    const int e = g.edge[b], t = tet[b], i = loc[b];
    HostTet h;
    host_tet(c, t, h);
    const double *p0 = &c.h_pts[3 * (size_t)c.h_edges[2 * (size_t)e]];
    const double *p1 = &c.h_pts[3 * (size_t)c.h_edges[2 * (size_t)e + 1]];
    double ec[3], ed[3];
    for (int d = 0; d < 3; ++d) {
      ec[d] = (p0[d] + p1[d]) / 2.0;
      ed[d] = p1[d] - p0[d];
    }
    double *co = &g.co[4 * (size_t)b];
    if (std::fabs(ec[0] - T(0, 0)) < EPS) {
      double w = (1.0 - std::cos(PI * (ec[1] - T(0, 1)) / (T(2, 1) - T(0, 1)))) / 2.0;
      co[0] = 1.0 - w; co[1] = 0.0; co[2] = 0.0; co[3] = w;
    } else if (std::fabs(ec[1] - T(0, 1)) < EPS) {
      double w = (1.0 - std::cos(PI * (ec[0] - T(0, 0)) / (T(2, 0) - T(0, 0)))) / 2.0;
      co[0] = 1.0 - w; co[1] = w; co[2] = 0.0; co[3] = 0.0;
    } else if (std::fabs(ec[0] - T(2, 0)) < EPS) {
      double w = (1.0 - std::cos(PI * (ec[1] - T(0, 1)) / (T(2, 1) - T(0, 1)))) / 2.0;
      co[0] = 0.0; co[1] = 1.0 - w; co[2] = w; co[3] = 0.0;
    } else if (std::fabs(ec[1] - T(2, 1)) < EPS) {
      double w = (1.0 - std::cos(PI * (ec[0] - T(0, 0)) / (T(2, 0) - T(0, 0)))) / 2.0;
      co[0] = 0.0; co[1] = 0.0; co[2] = w; co[3] = 1.0 - w;
    } else {
      double area = (T(2, 0) - T(0, 0)) * (T(2, 1) - T(0, 1));
      co[0] = ((T(2, 0) - ec[0]) * (T(2, 1) - ec[1])) / area;
      co[1] = ((ec[0] - T(3, 0)) * (T(3, 1) - ec[1])) / area;
      co[2] = ((ec[0] - T(0, 0)) * (ec[1] - T(0, 1))) / area;
      co[3] = ((T(1, 0) - ec[0]) * (ec[1] - T(1, 1))) / area;
    }
    double phi[3];
    int ge;
    host_phi(c, h, t, i, ec, phi, &ge);
    g.ed[2 * (size_t)b] = ed[0];
    g.ed[2 * (size_t)b + 1] = ed[1];
    g.den[b] = ed[0] * phi[0] + ed[1] * phi[1] + ed[2] * phi[2];
    z[b] = ec[2];
  }
  g.zs = z;
  std::sort(g.zs.begin(), g.zs.end());
  g.zs.erase(std::unique(g.zs.begin(), g.zs.end()), g.zs.end());
  g.zslot.resize(nb);
  for (int b = 0; b < nb; ++b) g.zslot[b] = (int)(std::lower_bound(g.zs.begin(), g.zs.end(), z[b]) - g.zs.begin());
}

// boundary DOF values of one (frequency, polarisation): the 1-D plane-wave
// field of the four corner soundings at each distinct depth, blended per edge
static void boundary_values(Context &c, const MtBoundary &g, double freq, int mode,
                            std::vector<std::complex<double>> &bv) {  // bv[b]: value of edge g.edge[b]
  typedef std::complex<double> zc;
  PlaneWave1D pw[4];
  for (int q = 0; q < 4; ++q) pw[q].init(&c.bg_ztop[q * c.bg_maxl], &c.bg_lsig[q * c.bg_maxl], c.bg_nlay[q], freq);
  const int nz = (int)g.zs.size(), nb = (int)g.edge.size();
  // polarisation XY drives E_x (field component 0), YX drives E_y (component 2)
  const int comp = mode == EMG_SOL_MT_XY ? 0 : 2;
  std::vector<zc> f(4 * (size_t)nz);
#pragma omp parallel for schedule(static)
  for (int iz = 0; iz < nz; ++iz)
    for (int q = 0; q < 4; ++q) {
      zc eh[4];
      pw[q].field(g.zs[iz], eh);
      f[4 * (size_t)iz + q] = std::conj(eh[comp]);
    }
  bv.assign(nb, zc(0));
#pragma omp parallel for schedule(static)
  for (int b = 0; b < nb; ++b) {
    const double *co = &g.co[4 * (size_t)b];
    const zc *fz = &f[4 * (size_t)g.zslot[b]];
    zc ep[3] = {0.0, 0.0, 0.0};
    for (int q = 0; q < 4; ++q) ep[comp == 0 ? 0 : 1] += co[q] * fz[q];
    const double ed0 = g.ed[2 * (size_t)b], ed1 = g.ed[2 * (size_t)b + 1];
    zc num = ed0 * ep[0] + ed1 * ep[1];
    zc dof = num / g.den[b];
    bv[b] = std::abs(dof) > 1E-13 ? dof : zc(0.0);
  }
}

static DBuf<double> &slot_buf(Context &c, int target) {
  need(target == EMG_SOL_MT_XY || target == EMG_SOL_MT_YX || target == EMG_SOL_CSEM || target == EMG_SOL_DUAL,
       EMG_ERR_ARG, "unknown solution slot");
  DBuf<double> &b = c.sol[target];
  if (b.n != (size_t)c.ne * 2) {
    b.alloc((size_t)c.ne * 2);
    b.zero(c.stream);
  }
  return b;
}

static std::vector<double> interleave(const double *re, const double *im, int n) {
  std::vector<double> v((size_t)n * 2);
  for (int i = 0; i < n; ++i) {
    v[2 * (size_t)i] = re ? re[i] : 0.0;
    v[2 * (size_t)i + 1] = im ? im[i] : 0.0;
  }
  return v;
}

}  // namespace emg

using namespace emg;

// Eigen::VectorXd::sum() (the total of refine_fixed_fraction,
// src/em_fwd.cc:1192) in the order Eigen evaluates it when the reference is
// built for x86-64 without -march flags, where Eigen vectorises with SSE2
// packets of two doubles: two packet accumulators advance over pairs of
// packets, then they are added, a leftover whole packet is added, the two
// lanes are summed, and an odd last element comes last.  The threshold, and
// so the flag set, can move by one ulp of the total with another order.
static double eigen_sse2_sum(const double *x, int n) {
  if (n < 2) return n == 1 ? x[0] : 0.0;
  const int n1 = n / 2 * 2;  // elements in whole packets
  const int n2 = n / 4 * 4;  // elements in whole packet pairs
  double a0 = x[0], a1 = x[1];
  if (n1 > 2) {
    double b0 = x[2], b1 = x[3];
    for (int i = 4; i < n2; i += 4) {
      a0 += x[i];
      a1 += x[i + 1];
      b0 += x[i + 2];
      b1 += x[i + 3];
    }
    a0 += b0;
    a1 += b1;
    if (n1 > n2) {
      a0 += x[n2];
      a1 += x[n2 + 1];
    }
  }
  double r = a0 + a1;
  for (int i = n1; i < n; ++i) r += x[i];
  return r;
}

extern "C" {

const char *emg_last_error(void) { return emg::g_last_error.c_str(); }
const char *emg_version(void) { return "emfem_b200 0.1 (sm_100a)"; }

int emg_create_context(emg_context **ctx, int device) {
  EMG_API_BEGIN
  need(ctx != nullptr, EMG_ERR_ARG, "null context pointer");
  if (device < 0) {  // host-only context: options and host-side helpers, no GPU work
    emg_context *c = new emg_context();
    c->device = -1;
    *ctx = c;
    return EMG_OK;
  }
  int ndev = 0;
  EMG_CUDA(cudaGetDeviceCount(&ndev));
  need(device >= 0 && device < ndev, EMG_ERR_ARG, "no such CUDA device");
  EMG_CUDA(cudaSetDevice(device));
  emg_context *c = new emg_context();
  c->device = device;
  cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete c;
    check_cuda(e, "cudaStreamCreate", __FILE__, __LINE__);
  }
  try {
    // the allocation-free estimator's scratch address, looked up now so that
    // its module is loaded and the address cached before any run
    (void)noalloc_scratch_address(device);
  } catch (...) {
    delete c;
    throw;
  }
  *ctx = c;
  EMG_API_END
}

int emg_destroy_context(emg_context *ctx) {
  EMG_API_BEGIN
  if (!ctx) return EMG_OK;
  if (ctx->device >= 0) {
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
  }
  delete ctx;
  EMG_API_END
}

int emg_process_options(emg_context *ctx, const char *text) {
  EMG_API_BEGIN
  need(ctx && text, EMG_ERR_ARG, "null argument");
  Options o = ctx->opt;
  std::vector<std::string> ignored;
  parse_options(o, text, ignored);
  ctx->opt = o;
  for (auto &k : ignored)
    if (o.verbose) fprintf(stderr, "emfem_b200: option %s is not used by the GPU solver\n", k.c_str());
  EMG_API_END
}

int emg_get_option(emg_context *ctx, const char *key, double *value) {
  EMG_API_BEGIN
  need(ctx && key && value, EMG_ERR_ARG, "null argument");
  std::string k = key[0] == '-' ? key + 1 : key;
  const Options &o = ctx->opt;
  if (k == "K_max_it") *value = o.K_max_it;
  else if (k == "e_rtol") *value = o.e_rtol;
  else if (k == "dual_rtol") *value = o.dual_rtol;
  else if (k == "inner_pc_type") *value = o.inner_pc_type;
  else if (k == "pc_threshold") *value = o.pc_threshold;
  else if (k == "n_tx_divisions") *value = o.n_tx_divisions;
  else if (k == "refine_fraction") *value = o.refine_fraction;
  else if (k == "refine_strategy") *value = o.refine_strategy;
  else if (k == "max_adaptive_refinements") *value = o.max_adaptive_refinements;
  else if (k == "n_uniform_refinements") *value = o.n_uniform_refinements;
  else if (k == "max_dofs") *value = o.max_dofs;
  else if (k == "save_mesh") *value = o.save_mesh;
  else if (k == "n_groups") *value = o.n_groups;
  else if (k == "A_ksp_gmres_restart") *value = o.gmres_restart;
  else if (k == "B_ksp_rtol") *value = o.inner_rtol;
  else if (k == "B_ksp_max_it") *value = o.inner_max_it;
  else if (k == "B_ksp_fcg_mmax") *value = o.fcg_mmax;
  else if (k == "emg_inner_precision") *value = o.inner_fp32;
  else if (k == "emg_graphs") *value = o.graphs;
  else if (k == "emg_fused_vcycle") *value = o.ams_fused;
  else if (k == "emg_fused_blocks_per_sm") *value = o.fused_bps;
  else if (k == "emg_fused_rows") *value = o.fused_rows;
  else if (k == "emg_gpu_amg") *value = o.gpu_amg;
  else if (k == "emg_block_fp64_fallback") *value = o.block_fp64_fallback;
  else if (k == "emg_block_fp32_rtol_factor") *value = o.block_fp32_rtol_factor;
  else if (k == "emg_block_fp64_below") *value = o.block_fp64_below_hz;
  else if (k == "emg_div_correction") *value = o.div_correction;
  else if (k == "emg_div_rtol") *value = o.div_rtol;
  else if (k == "emg_div_max_it") *value = o.div_max_it;
  else if (k == "emg_fused_wait_ms") *value = o.fused_wait_ms;
  else if (k == "emg_fused_test_withhold") *value = o.fused_test_withhold;
  else if (k == "emg_pi_coupled") *value = o.pi_coupled;
  else if (k == "emg_block_inner_rtol") *value = o.block_inner_rtol;
  else if (k == "emg_block_inner_max_it") *value = o.block_inner_max_it;
  else if (k == "emg_block_fcg_mmax") *value = o.block_fcg_mmax;
  else if (k == "emg_block_fcg_check_every") *value = o.block_fcg_check_every;
  else if (k == "emg_block_relax_times") *value = o.block_relax_times;
  else if (k == "emg_cheb_degree") *value = o.cheb_degree;
  else if (k == "emg_block_cheb_degree") *value = o.block_cheb_degree;
  else if (k == "emg_amg_cheb_degree") *value = o.amg_cheb_degree;
  else if (k == "emg_restrict_smooth") *value = o.restrict_j0;
  else if (k == "emg_block_floor_stop") *value = o.block_floor_stop;
  else if (k == "emg_amg_pre_smooth") *value = o.amg_pre_smooth;
  else if (k == "emg_spmm_tiled") *value = o.spmm_tiled;
  else if (k == "emg_tiled_smem_kb") *value = o.tiled_smem_kb;
  else fail(EMG_ERR_OPTION, "unknown option %s", key);
  EMG_API_END
}

int emg_set_mesh(emg_context *c, int nv, const double *pts, int nt, const int *tets, const int *attr, int ne,
                 const int *edges, const int *t2e, const int *nbr, const int *non, const unsigned char *ebdr) {
  EMG_API_BEGIN
  need(c && pts && tets && attr && edges && t2e && nbr && non && ebdr, EMG_ERR_ARG, "null mesh array");
  need(nv > 0 && nt > 0 && ne > 0, EMG_ERR_ARG, "empty mesh");
  if (c->device >= 0) EMG_CUDA(cudaSetDevice(c->device));
  for (long i = 0; i < 4L * nt; ++i)
    need(tets[i] >= 0 && tets[i] < nv, EMG_ERR_ARG, "tetrahedronlist index out of range");
  for (long i = 0; i < 6L * nt; ++i) need(t2e[i] >= 0 && t2e[i] < ne, EMG_ERR_ARG, "tet2edgelist index out of range");
  for (long i = 0; i < 2L * ne; ++i) need(edges[i] >= 0 && edges[i] < nv, EMG_ERR_ARG, "edgelist index out of range");
  for (long i = 0; i < ne; ++i) need(edges[2 * i] < edges[2 * i + 1], EMG_ERR_ARG, "edgelist endpoints must be sorted ascending");
  for (long i = 0; i < 4L * nt; ++i) {
    need(nbr[i] >= -1 && nbr[i] < nt, EMG_ERR_ARG, "neighborlist index out of range");
    need(nbr[i] < 0 || (non[i] >= 0 && non[i] < 4), EMG_ERR_ARG, "tet_non index out of range");
  }
  c->nv = nv;
  c->nt = nt;
  c->ne = ne;
  c->h_pts.assign(pts, pts + 3L * nv);
  c->h_tets.assign(tets, tets + 4L * nt);
  c->h_attr.assign(attr, attr + nt);
  c->h_edges.assign(edges, edges + 2L * ne);
  c->h_t2e.assign(t2e, t2e + 6L * nt);
  c->h_nbr.assign(nbr, nbr + 4L * nt);
  c->h_non.assign(non, non + 4L * nt);
  c->h_ebdr.assign(ebdr, ebdr + ne);
  c->bnd_rank.release();
  c->tiles.clear();
  c->locator.reset();
  c->have_ls = false;
  c->assembled = false;
  c->have_pc = false;
  c->ws->block_ready64 = c->ws->block_ready32 = false;
  c->sol.clear();
  if (c->device < 0) return EMG_OK;  // host-only context: host-side entry points only
  c->pts.upload(c->h_pts, c->stream);
  c->tets.upload(c->h_tets, c->stream);
  c->attr.upload(c->h_attr, c->stream);
  c->edges.upload(c->h_edges, c->stream);
  c->t2e.upload(c->h_t2e, c->stream);
  c->nbr.upload(c->h_nbr, c->stream);
  c->non.upload(c->h_non, c->stream);
  c->ebdr.upload(c->h_ebdr, c->stream);
  canonicalize(*c);
  EMG_CUDA(cudaStreamSynchronize(c->stream));
  EMG_API_END
}

int emg_set_model(emg_context *c, int aniso_form, int n_rho, int ncol, const double *rho) {
  EMG_API_BEGIN
  need(c && rho && n_rho > 0, EMG_ERR_ARG, "bad model");
  static const int need_cols[4] = {1, 2, 3, 6};
  if (aniso_form < 0 || aniso_form > 3) fail(EMG_ERR_USER, "Unsupported anisotropy form %d.", aniso_form);
  need(ncol >= need_cols[aniso_form], EMG_ERR_ARG, "too few resistivity columns for the anisotropy form");
  if (c->nt) {
    for (int a : c->h_attr) need(a >= 0 && a < n_rho, EMG_ERR_ARG, "tet attribute beyond the resistivity table");
  }
  c->aniso_form = aniso_form;
  c->nrho = n_rho;
  c->ncol = ncol;
  c->rho.assign(rho, rho + (size_t)n_rho * ncol);
  sigma_table(aniso_form, n_rho, ncol, rho, c->h_sigma_tab);
  if (c->device >= 0) c->sigma_tab.upload(c->h_sigma_tab, c->stream);
  c->assembled = false;
  c->ws->block_ready64 = c->ws->block_ready32 = false;
  if (c->device >= 0) EMG_CUDA(cudaStreamSynchronize(c->stream));
  EMG_API_END
}

int emg_set_frequencies(emg_context *c, int n, const double *f) {
  EMG_API_BEGIN
  need(c && (n == 0 || f), EMG_ERR_ARG, "bad frequencies");
  c->freqs.assign(f, f + n);
  EMG_API_END
}

// makes the context's GPU current; a host-only context (device -1) refuses
static void use_device(const Context &c) {
  need(c.device >= 0, EMG_ERR_STATE, "host-only context has no device");
  EMG_CUDA(cudaSetDevice(c.device));
}

int emg_create_linear_system(emg_context *c, int tidx) {
  EMG_API_BEGIN
  need(c && c->nt > 0, EMG_ERR_STATE, "create_linear_system before emg_set_mesh");
  use_device(*c);
  c->tidx = tidx;
  c->tiles.clear();
  build_sparsity(*c);
  build_vertex_pattern(*c);
  build_slot_maps(*c);
  c->gslot.release();
  build_gtb_pattern(*c);
  c->have_ls = true;
  c->assembled = false;
  c->have_pc = false;
  c->ws->block_ready64 = c->ws->block_ready32 = false;
  // named solution vectors (src/em_fwd.cc:267-280)
  c->sol.clear();
  slot_buf(*c, EMG_SOL_DUAL);
  if (tidx < 0) {
    slot_buf(*c, EMG_SOL_MT_XY);
    slot_buf(*c, EMG_SOL_MT_YX);
  } else {
    slot_buf(*c, EMG_SOL_CSEM);
  }
  EMG_CUDA(cudaStreamSynchronize(c->stream));
  EMG_API_END
}

int emg_destroy_linear_system(emg_context *c) {
  EMG_API_BEGIN
  need(c != nullptr, EMG_ERR_ARG, "null context");
  c->Cv.release();
  c->Msv.release();
  c->slot.release();
  c->vslot.release();
  c->rp.release();
  c->ci.release();
  c->sol.clear();
  c->have_ls = c->assembled = c->have_pc = false;
  c->ws->block_ready64 = c->ws->block_ready32 = false;
  EMG_API_END
}

int emg_get_sparsity(emg_context *c, long *nnz, int *rptr, int *cidx) {
  EMG_API_BEGIN
  need(c && nnz, EMG_ERR_ARG, "null argument");
  need(c->have_ls, EMG_ERR_STATE, "no linear system");
  *nnz = c->nnz;
  if (rptr) std::copy(c->h_rp.begin(), c->h_rp.end(), rptr);
  if (cidx) std::copy(c->h_ci.begin(), c->h_ci.end(), cidx);
  EMG_API_END
}

int emg_assemble_matrix(emg_context *c, int fidx) {
  EMG_API_BEGIN
  need(c && c->have_ls, EMG_ERR_STATE, "assemble_matrix before create_linear_system");
  need(c->nrho > 0, EMG_ERR_STATE, "assemble_matrix before emg_set_model");
  need(fidx >= 0 && fidx < (int)c->freqs.size(), EMG_ERR_ARG, "frequency index out of range");
  use_device(*c);
  c->omega = 2 * PI * c->freqs[fidx];
  cudaEvent_t e0, e1;
  EMG_CUDA(cudaEventCreate(&e0));
  EMG_CUDA(cudaEventCreate(&e1));
  EMG_CUDA(cudaEventRecord(e0, c->stream));
  assemble_edge(*c);
  EMG_CUDA(cudaEventRecord(e1, c->stream));
  EMG_CUDA(cudaEventSynchronize(e1));
  float ms = 0;
  EMG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  c->kernel_ms["assemble"] = ms;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  c->assembled = true;
  c->have_pc = false;
  c->ws->block_ready64 = c->ws->block_ready32 = false;
  EMG_API_END
}

__global__ static void scale_copy_kernel(long n, const double *a, double w, double *b) {
  long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < n) b[i] = w * a[i];
}

int emg_get_matrices(emg_context *c, double *C, double *M, unsigned char *bdr) {
  EMG_API_BEGIN
  need(c && c->assembled, EMG_ERR_STATE, "matrices not assembled");
  use_device(*c);
  if (C) c->Cv.download(C, c->nnz, c->stream);
  if (M) {
    DBuf<double> tmp(c->nnz);
    scale_copy_kernel<<<(unsigned)((c->nnz + 255) / 256), 256, 0, c->stream>>>(c->nnz, c->Msv.p, c->omega, tmp.p);
    EMG_LAUNCH_CHECK();
    tmp.download(M, c->nnz, c->stream);
    EMG_CUDA(cudaStreamSynchronize(c->stream));
  }
  if (bdr) c->bdr_cell.download(bdr, c->nt, c->stream);
  EMG_CUDA(cudaStreamSynchronize(c->stream));
  EMG_API_END
}

int emg_create_pc(emg_context *c) {
  EMG_API_BEGIN
  need(c && c->assembled, EMG_ERR_STATE, "create_pc before assemble_matrix");
  use_device(*c);
  cudaEvent_t e0, e1;
  EMG_CUDA(cudaEventCreate(&e0));
  EMG_CUDA(cudaEventCreate(&e1));
  EMG_CUDA(cudaEventRecord(e0, c->stream));
  ams_setup<double>(*c, c->ws->pams64, true, c->omega, c->omega);
  c->ws->pams64.set_columns({c->omega, c->omega}, c->stream);
  EMG_CUDA(cudaEventRecord(e1, c->stream));
  EMG_CUDA(cudaEventSynchronize(e1));
  float ms = 0;
  EMG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  c->kernel_ms["create_pc"] = ms;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  c->pc_omega = c->omega;
  c->have_pc = true;
  EMG_API_END
}

int emg_destroy_pc(emg_context *c) {
  EMG_API_BEGIN
  need(c != nullptr, EMG_ERR_ARG, "null context");
  c->ws->pams64 = Ams<double>();
  c->have_pc = false;
  EMG_API_END
}

int emg_matshell_mult_a(emg_context *c, const double *x, double *y) {
  EMG_API_BEGIN
  need(c && x && y, EMG_ERR_ARG, "null argument");
  need(c->assembled, EMG_ERR_STATE, "operator not assembled");
  use_device(*c);
  const int n = c->ne;
  std::vector<double> xi = interleave(x, x + n, n);
  Workspace &w = *c->ws;
  w.vec_a.upload(xi, c->stream);
  w.vec_b.alloc((size_t)n * 2);
  w.omega_k.upload(&c->omega, 1, c->stream);
  spmm_complex(n, 1, c->rp.p, c->ci.p, c->Cv.p, c->Msv.p, w.omega_k.p, w.vec_a.p, nullptr, w.vec_b.p, false, true,
               c->stream);
  std::vector<double> yo((size_t)n * 2);
  w.vec_b.download(yo.data(), yo.size(), c->stream);
  EMG_CUDA(cudaStreamSynchronize(c->stream));
  for (int i = 0; i < n; ++i) {
    y[i] = yo[2 * (size_t)i];
    y[n + i] = yo[2 * (size_t)i + 1];
  }
  EMG_API_END
}

int emg_pc_apply_b(emg_context *c, const double *b, double *x) {
  EMG_API_BEGIN
  need(c && b && x, EMG_ERR_ARG, "null argument");
  need(c->have_pc, EMG_ERR_STATE, "pc_apply_b before create_pc");
  use_device(*c);
  const int n = c->ne;
  Workspace &w = *c->ws;
  std::vector<double> bi = interleave(b, b + n, n);
  w.vec_a.upload(bi, c->stream);
  w.vec_b.alloc((size_t)n * 2);
  w.fcg64.mmax = c->opt.fcg_mmax;
  w.fcg64.check_every = 1;
  w.fcg64.solve(w.pams64, w.vec_a.p, w.vec_b.p, c->opt.inner_rtol, c->opt.inner_max_it, c->stream);
  std::vector<double> xo((size_t)n * 2);
  w.vec_b.download(xo.data(), xo.size(), c->stream);
  EMG_CUDA(cudaStreamSynchronize(c->stream));
  w.pams64.check_fused(c->stream);
  for (int i = 0; i < n; ++i) {
    x[i] = xo[2 * (size_t)i];
    x[n + i] = xo[2 * (size_t)i + 1];
  }
  EMG_API_END
}

static void fill_info(emg_solve_info *info, const SolveStats &st, long inner, int col) {
  if (!info) return;
  info->outer_its = col >= 0 && col < (int)st.col_its.size() ? st.col_its[col] : st.outer_its;
  info->inner_its = (int)inner;
  info->true_rel_res = col >= 0 && col < (int)st.true_res.size() ? st.true_res[col] : 0.0;
  info->reason = 0;
  if (col >= 0 && col < (int)st.converged.size() && !st.converged[col])
    info->reason = col < (int)st.at_floor.size() && st.at_floor[col] ? EMG_STOPPED_AT_FLOOR : EMG_DIVERGED_ITS;
  info->seconds = st.seconds;
}

int emg_solve_linear_system(emg_context *c, int target, const double *s_re, const double *s_im, int max_it,
                            double rtol, emg_solve_info *info) {
  EMG_API_BEGIN
  need(c && s_re && s_im, EMG_ERR_ARG, "null argument");
  need(c->have_pc, EMG_ERR_STATE, "solve_linear_system before create_pc");
  need(max_it > 0 && rtol > 0, EMG_ERR_ARG, "bad tolerances");
  use_device(*c);
  const int n = c->ne;
  Workspace &w = *c->ws;
  DBuf<double> &x = slot_buf(*c, target);
  std::vector<double> bi = interleave(s_re, s_im, n);
  w.vec_a.upload(bi, c->stream);
  w.gm.k = 1;
  w.gm.restart = c->opt.gmres_restart;
  w.gm.stall_factor = 0.0;  // the reference's FGMRES runs to rtol or max_it
  w.gm.omega.upload(&c->omega, 1, c->stream);
  w.fcg64.mmax = c->opt.fcg_mmax;
  w.fcg64.check_every = 1;
  w.fcg64.total_its = 0;
  SolveStats st;
  auto pc = [&](const double *v, double *z) {
    w.fcg64.solve(w.pams64, v, z, c->opt.inner_rtol, c->opt.inner_max_it, c->stream);
  };
  w.gm.solve(*c, w.vec_a.p, x.p, false, rtol, max_it, true, pc, st);
  EMG_CUDA(cudaStreamSynchronize(c->stream));
  w.pams64.check_fused(c->stream);
  fill_info(info, st, w.fcg64.total_its, 0);
  c->kernel_ms["solve"] = st.seconds * 1e3;
  if (!st.converged[0]) fail(EMG_DIVERGED_ITS, "FGMRES reached %d iterations at relative residual %.3e", max_it,
                             st.true_res[0]);
  EMG_API_END
}

int emg_get_solution(emg_context *c, int target, double *e_re, double *e_im) {
  EMG_API_BEGIN
  need(c && (e_re || e_im), EMG_ERR_ARG, "null argument");
  need(c->have_ls, EMG_ERR_STATE, "no linear system");
  use_device(*c);
  DBuf<double> &x = slot_buf(*c, target);
  std::vector<double> v((size_t)c->ne * 2);
  x.download(v.data(), v.size(), c->stream);
  EMG_CUDA(cudaStreamSynchronize(c->stream));
  for (int i = 0; i < c->ne; ++i) {
    if (e_re) e_re[i] = v[2 * (size_t)i];
    if (e_im) e_im[i] = v[2 * (size_t)i + 1];
  }
  EMG_API_END
}

int emg_set_solution(emg_context *c, int target, const double *e_re, const double *e_im) {
  EMG_API_BEGIN
  need(c && e_re && e_im, EMG_ERR_ARG, "null argument");
  need(c->have_ls, EMG_ERR_STATE, "no linear system");
  use_device(*c);
  DBuf<double> &x = slot_buf(*c, target);
  std::vector<double> v = interleave(e_re, e_im, c->ne);
  x.upload(v, c->stream);
  EMG_CUDA(cudaStreamSynchronize(c->stream));
  EMG_API_END
}

int emg_set_background(emg_context *c, const double *corners, const int *nlay, const double *ztop,
                       const double *lsig, int maxl) {
  EMG_API_BEGIN
  need(c && corners && nlay && ztop && lsig && maxl > 0, EMG_ERR_ARG, "bad background model");
  for (int q = 0; q < 4; ++q) need(nlay[q] >= 1 && nlay[q] <= maxl, EMG_ERR_ARG, "bad layer count");
  c->bg_corners.assign(corners, corners + 12);
  c->bg_nlay.assign(nlay, nlay + 4);
  c->bg_ztop.assign(ztop, ztop + 4 * maxl);
  c->bg_lsig.assign(lsig, lsig + 4 * maxl);
  c->bg_maxl = maxl;
  EMG_API_END
}

// MT right-hand side for k (frequency, polarisation) columns on the device:
// boundary values on the host (plane waves), lifting by the GPU kernel.
static void rhs_mt_block(Context &c, int k, const double *freqs, const int *modes, double *s_dev) {
  Workspace &w = *c.ws;
  std::vector<unsigned char> bdr(c.nt);
  c.bdr_cell.download(bdr.data(), c.nt, c.stream);
  EMG_CUDA(cudaStreamSynchronize(c.stream));
  // boundary values travel compact: row r = rank of the edge among the
  // boundary edges (edge_bdr_marker order), k complex columns per row
  if (c.bnd_rank.n != (size_t)c.ne) {
    std::vector<int> rank(c.ne, -1);
    int r = 0;
    for (int e = 0; e < c.ne; ++e)
      if (c.h_ebdr[e]) rank[e] = r++;
    c.n_bnd = r;
    c.h_bnd_rank = rank;
    c.bnd_rank.upload(rank, c.stream);
  }
  MtBoundary g;
  mt_boundary_geometry(c, bdr, g);
  std::vector<double> bv((size_t)std::max(c.n_bnd, 1) * k * 2, 0.0), om(k);
  for (int j = 0; j < k; ++j) {
    std::vector<std::complex<double>> v;
    boundary_values(c, g, freqs[j], modes[j], v);
#pragma omp parallel for schedule(static)
    for (int b = 0; b < (int)g.edge.size(); ++b) {
      const size_t r = (size_t)c.h_bnd_rank[g.edge[b]];
      bv[2 * (r * k + j)] = v[b].real();
      bv[2 * (r * k + j) + 1] = v[b].imag();
    }
    om[j] = 2 * PI * freqs[j];
  }
  w.bvals.upload(bv, c.stream);
  w.omega_k.upload(om, c.stream);
  launch_rhs_mt(c, k, w.omega_k.p, w.bvals.p, c.bnd_rank.p, s_dev);
  EMG_CUDA(cudaStreamSynchronize(c.stream));
}

int emg_assemble_rhs_mt(emg_context *c, int fidx, int mode, double *s_re, double *s_im) {
  EMG_API_BEGIN
  need(c && s_re && s_im, EMG_ERR_ARG, "null argument");
  need(c->assembled, EMG_ERR_STATE, "assemble_rhs_mt before assemble_matrix");
  need(fidx >= 0 && fidx < (int)c->freqs.size(), EMG_ERR_ARG, "frequency index out of range");
  need(mode == EMG_SOL_MT_XY || mode == EMG_SOL_MT_YX, EMG_ERR_ARG, "mode must be XY_POLAR or YX_POLAR");
  use_device(*c);
  DBuf<double> s((size_t)c->ne * 2);
  double f = c->freqs[fidx];
  rhs_mt_block(*c, 1, &f, &mode, s.p);
  std::vector<double> v((size_t)c->ne * 2);
  s.download(v.data(), v.size(), c->stream);
  EMG_CUDA(cudaStreamSynchronize(c->stream));
  for (int i = 0; i < c->ne; ++i) {
    s_re[i] = v[2 * (size_t)i];
    s_im[i] = v[2 * (size_t)i + 1];
  }
  EMG_API_END
}

// divide_line_source + assemble_rhs_csem (src/em_fwd.cc:582-671); the cell of
// every dipole comes from the host mesh's point location.
int emg_assemble_rhs_csem(emg_context *c, int fidx, const double *tx, const int *dtets, double *s_re,
                          double *s_im) {
  EMG_API_BEGIN
  need(c && tx && dtets && s_re && s_im, EMG_ERR_ARG, "null argument");
  need(fidx >= 0 && fidx < (int)c->freqs.size(), EMG_ERR_ARG, "frequency index out of range");
  const double omega = 2 * PI * c->freqs[fidx];
  double dir[3] = {std::cos(tx[3] * DTOR) * std::cos(tx[4] * DTOR), std::sin(tx[3] * DTOR) * std::cos(tx[4] * DTOR),
                   std::sin(tx[4] * DTOR)};
  double current = tx[5], length = tx[6];
  std::vector<std::array<double, 3>> pts;
  std::vector<double> wts;
  if (std::fabs(length) <= 0.1) {
    pts.push_back({tx[0], tx[1], tx[2]});
    wts.push_back(1.0);
  } else {
    int nd = c->opt.n_tx_divisions;
    double A[3] = {tx[0] - dir[0] * length / 2, tx[1] - dir[1] * length / 2, tx[2] - dir[2] * length / 2};
    for (int i = 0; i < nd; ++i) {
      double Bp[3] = {A[0] + dir[0] * length / nd, A[1] + dir[1] * length / nd, A[2] + dir[2] * length / nd};
      pts.push_back({(A[0] + Bp[0]) / 2, (A[1] + Bp[1]) / 2, (A[2] + Bp[2]) / 2});
      wts.push_back(1.0 / nd);
      for (int d = 0; d < 3; ++d) A[d] = Bp[d];
    }
  }
  std::fill(s_re, s_re + c->ne, 0.0);
  std::fill(s_im, s_im + c->ne, 0.0);
  for (size_t j = 0; j < pts.size(); ++j) {
    int t = dtets[j];
    if (t < 0 || t >= c->nt) fail(EMG_ERR_USER, "Transmitter %d is not found in mesh.", (int)j);
    HostTet h;
    host_tet(*c, t, h);
    for (int i = 0; i < 6; ++i) {
      double phi[3];
      int ge;
      host_phi(*c, h, t, i, pts[j].data(), phi, &ge);
      s_im[ge] += omega * current * (phi[0] * dir[0] + phi[1] * dir[1] + phi[2] * dir[2]) * wts[j];
    }
  }
  EMG_API_END
}

// assemble_rhs_dual (src/em_fwd.cc:673-717)
int emg_assemble_rhs_dual(emg_context *c, int nrx, const double *rx, const int *rtets, double *s_re, double *s_im) {
  EMG_API_BEGIN
  need(c && rx && rtets && s_re && s_im, EMG_ERR_ARG, "null argument");
  std::fill(s_re, s_re + c->ne, 0.0);
  std::fill(s_im, s_im + c->ne, 0.0);
  for (int r = 0; r < nrx; ++r) {
    int t = rtets[r];
    if (t < 0 || t >= c->nt) fail(EMG_ERR_USER, "Receiver %d is not found in mesh.", r);
    HostTet h;
    host_tet(*c, t, h);
    for (int j = 0; j < 6; ++j) {
      double phi[3];
      int ge;
      host_phi(*c, h, t, j, rx + 3 * r, phi, &ge);
      double v = phi[0] + phi[1] + phi[2];
      s_re[ge] += v;
      s_im[ge] += v;
    }
  }
  EMG_API_END
}

int emg_estimate_error(emg_context *c, int fidx, int tidx, double *err, double *eta_raw) {
  EMG_API_BEGIN
  need(c && (err || eta_raw), EMG_ERR_ARG, "null argument");
  need(c->have_ls && c->nrho > 0, EMG_ERR_STATE, "estimate_error before create_linear_system");
  need(fidx >= 0 && fidx < (int)c->freqs.size(), EMG_ERR_ARG, "frequency index out of range");
  use_device(*c);
  Workspace &w = *c->ws;
  std::vector<int> slots = tidx < 0 ? std::vector<int>{EMG_SOL_MT_XY, EMG_SOL_MT_YX, EMG_SOL_DUAL}
                                    : std::vector<int>{EMG_SOL_CSEM, EMG_SOL_DUAL};
  int nsol = (int)slots.size();
  const double *sp[3];
  for (int s = 0; s < nsol; ++s) sp[s] = slot_buf(*c, slots[s]).p;
  w.est_vol.alloc((size_t)nsol * c->nt);
  w.est_fe.alloc((size_t)nsol * c->nt * 4);
  w.est_eta.alloc((size_t)nsol * c->nt);
  w.est_err.alloc((size_t)(nsol - 1) * c->nt);
  cudaEvent_t e0, e1;
  EMG_CUDA(cudaEventCreate(&e0));
  EMG_CUDA(cudaEventCreate(&e1));
  EMG_CUDA(cudaEventRecord(e0, c->stream));
  launch_estimate(*c, 2 * PI * c->freqs[fidx], nsol, sp, w.est_eta.p, w.est_err.p, w.est_vol.p, w.est_fe.p);
  EMG_CUDA(cudaEventRecord(e1, c->stream));
  if (err) w.est_err.download(err, (size_t)(nsol - 1) * c->nt, c->stream);
  if (eta_raw) w.est_eta.download(eta_raw, (size_t)nsol * c->nt, c->stream);
  EMG_CUDA(cudaEventSynchronize(e1));
  float ms = 0;
  EMG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  c->kernel_ms["estimate"] = ms;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  EMG_CUDA(cudaStreamSynchronize(c->stream));
  EMG_API_END
}

// refine_fixed_fraction (src/em_fwd.cc:1182-1215)
int emg_refine_fixed_fraction(int n, const double *err, double fraction, unsigned char *flag) {
  EMG_API_BEGIN
  need(n >= 0 && (n == 0 || (err && flag)), EMG_ERR_ARG, "null argument");
  const double total = eigen_sse2_sum(err, n);
  std::vector<double> s(err, err + n);
  std::sort(s.begin(), s.end(), std::greater<double>());
  double sum = 0, thr = 0;
  for (int i = 0; i < n; ++i) {
    if (sum < fraction * total) sum += s[i];
    else { thr = s[i]; break; }
  }
  for (int i = 0; i < n; ++i)
    if (err[i] > thr) flag[i] = 1;
  EMG_API_END
}

// refine_fixed_number (src/em_fwd.cc:1217-1240)
int emg_refine_fixed_number(int n, const double *err, double fraction, unsigned char *flag) {
  EMG_API_BEGIN
  need(n > 0 && err && flag, EMG_ERR_ARG, "null argument");
  int k = (int)(n * fraction);
  need(k >= 0 && k < n, EMG_ERR_ARG, "refine fraction out of range");
  std::vector<double> s(err, err + n);
  std::nth_element(s.begin(), s.begin() + k, s.end(), std::greater<double>());
  double thr = s[k];
  for (int i = 0; i < n; ++i)
    if (err[i] > thr) flag[i] = 1;
  EMG_API_END
}

// interpolate_fields (src/em_fwd.cc:719-744)
// E and H at n points in known cells from an edge solution v (complex,
// interleaved re/im per edge): interpolate_fields (src/em_fwd.cc:719-744)
static void interpolate_host(const Context &c, double freq, int n, const double *pts, const int *tets,
                             const double *v, double *eh) {
  typedef std::complex<double> zc;
  const zc hfac = -1.0 / (zc(0, 1) * 2.0 * PI * freq * MU);
  for (int r = 0; r < n; ++r) {
    int t = tets[r];
    if (t < 0 || t >= c.nt) fail(EMG_ERR_USER, "Receiver %d is not found in mesh.", r);
    HostTet h;
    host_tet(c, t, h);
    zc E[3] = {0.0, 0.0, 0.0}, H[3] = {0.0, 0.0, 0.0};
    for (int i = 0; i < 6; ++i) {
      double phi[3];
      int ge;
      host_phi(c, h, t, i, pts + 3 * r, phi, &ge);
      int e = ge, a = c.h_edges[2 * (size_t)e], b = c.h_edges[2 * (size_t)e + 1];
      int la = 0, lb = 0;
      for (int q = 0; q < 4; ++q) {
        if (h.v[q] == a) la = q;
        if (h.v[q] == b) lb = q;
      }
      double cu[3] = {2.0 * (h.gr[la][1] * h.gr[lb][2] - h.gr[la][2] * h.gr[lb][1]),
                      2.0 * (h.gr[la][2] * h.gr[lb][0] - h.gr[la][0] * h.gr[lb][2]),
                      2.0 * (h.gr[la][0] * h.gr[lb][1] - h.gr[la][1] * h.gr[lb][0])};
      zc u(v[2 * (size_t)e], v[2 * (size_t)e + 1]);
      for (int d = 0; d < 3; ++d) {
        E[d] += u * phi[d];
        H[d] += hfac * u * cu[d];
      }
    }
    for (int d = 0; d < 3; ++d) {
      eh[12 * r + 2 * d] = E[d].real();
      eh[12 * r + 2 * d + 1] = E[d].imag();
      eh[12 * r + 6 + 2 * d] = H[d].real();
      eh[12 * r + 6 + 2 * d + 1] = H[d].imag();
    }
  }
}

int emg_interpolate_fields(emg_context *c, int target, int fidx, int n, const double *pts, const int *tets,
                           double *eh) {
  EMG_API_BEGIN
  need(c && pts && tets && eh, EMG_ERR_ARG, "null argument");
  need(fidx >= 0 && fidx < (int)c->freqs.size(), EMG_ERR_ARG, "frequency index out of range");
  use_device(*c);
  DBuf<double> &x = slot_buf(*c, target);
  // the slot is an n x 1 complex block: the receiver kernel reads only the
  // edges of the receivers' cells
  const double f = c->freqs[fidx];
  int rc = emg_interpolate_fields_block_dev(c, 1, &f, x.p, n, pts, tets, eh);
  if (rc != EMG_OK) fail(rc, "%s", emg_last_error());
  EMG_API_END
}

int emg_interpolate_fields_host(emg_context *c, int fidx, int n, const double *pts, const int *tets,
                                const double *e_re, const double *e_im, double *eh) {
  EMG_API_BEGIN
  need(c && pts && tets && e_re && e_im && eh, EMG_ERR_ARG, "null argument");
  need(c->nt > 0, EMG_ERR_STATE, "interpolate_fields before emg_set_mesh");
  need(fidx >= 0 && fidx < (int)c->freqs.size(), EMG_ERR_ARG, "frequency index out of range");
  std::vector<double> v((size_t)c->ne * 2);
  for (int e = 0; e < c->ne; ++e) {
    v[2 * (size_t)e] = e_re[e];
    v[2 * (size_t)e + 1] = e_im[e];
  }
  interpolate_host(*c, c->freqs[fidx], n, pts, tets, v.data(), eh);
  EMG_API_END
}

__global__ static void conj_copy_kernel(long n, const double2 *a, double2 *b) {
  long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < n) {
    double2 v = a[i];
    b[i] = make_double2(v.x, -v.y);
  }
}

// ---------------------------------------------------------------------------
// divergence correction of a block solution
//
// The FP32 AMS leaves rounding noise in the near-null space of A = C + i w Ms:
// gradients in the air, where C G = 0 and w sigma_air is tiny, so the
// residual hardly sees it while the receiver E fields do.  The exact solution
// satisfies G^T (b - A x) = 0 at every interior vertex (the weak divergence
// condition, div(sigma E) = source).  With r = b - A x, the vertex potential
// phi (zero at boundary vertices, so the Dirichlet edges keep their values and
// C G phi = 0) solving
//     i w (G^T Ms G) phi = G^T r
// restores it: x <- x + G phi removes the divergence error without touching
// the curl part.  G^T Ms G is solved by FCG in FP64 on the symmetrically
// scaled system D^-1/2 N D^-1/2 (D: the l1 scale of each vertex row, so that
// air and earth rows converge alike), preconditioned by the gradient space's
// nodal V-cycle of the block's AMS.
// ---------------------------------------------------------------------------
__global__ void div_scale_edges_kernel(int ne, const int *__restrict__ rp, const int *__restrict__ ci,
                                       const double *__restrict__ ms, const int *__restrict__ edges,
                                       const unsigned char *__restrict__ ebdr, double *__restrict__ d,
                                       double *__restrict__ bnd) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  double m = 0;
  for (int k = rp[e]; k < rp[e + 1]; ++k)
    if (ci[k] == e) {
      m = fabs(ms[k]);
      break;
    }
  const int v0 = edges[2 * (long)e], v1 = edges[2 * (long)e + 1];
  atomicAdd(d + v0, m);
  atomicAdd(d + v1, m);
  if (ebdr[e]) {
    bnd[v0] = 1.0;
    bnd[v1] = 1.0;
  }
}

__global__ void div_scale_vertices_kernel(int nv, const double *__restrict__ d, const double *__restrict__ bnd,
                                          double *__restrict__ dis, double *__restrict__ ds) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  const bool in = bnd[v] == 0.0 && d[v] > 0.0;
  dis[v] = in ? 1.0 / sqrt(d[v]) : 0.0;
  ds[v] = in ? sqrt(d[v]) : 0.0;
}

// out = dis * (G^T r) / (i w_j) for nv x k complex entries
__global__ void div_rhs_kernel(long total, int k, const double *__restrict__ omega, const double *__restrict__ dis,
                               const double2 *__restrict__ gtr, double2 *__restrict__ out) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= total) return;
  const long v = i / k;
  const int j = (int)(i - v * k);
  const double f = dis[v] / omega[j];
  const double2 a = gtr[i];
  out[i] = make_double2(a.y * f, -a.x * f);
}

extern "C++" {
template <typename TI, typename TO>
__global__ void vrow_scale_kernel(long total, int K, const double *__restrict__ sv, const TI *__restrict__ in,
                                  TO *__restrict__ out) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= total) return;
  out[i] = (TO)(sv[i / K] * (double)in[i]);
}

template <typename TI, typename TO>
static void vrow_scale(long rows, int K, const double *sv, const TI *in, TO *out, cudaStream_t s) {
  const long total = rows * K;
  vrow_scale_kernel<TI, TO><<<(unsigned)((total + 255) / 256), 256, 0, s>>>(total, K, sv, in, out);
  EMG_LAUNCH_CHECK();
}
}  // extern "C++"

// x (ne x k complex, device) <- x + G phi; b is the right-hand side the block
// solved (conjugated form), omega the k column frequencies (device); returns
// the inner FCG iterations
static long div_correct(Context &c, int k, bool fp32, const double *b, double *x, const double *omega) {
  Workspace &w = *c.ws;
  cudaStream_t s = c.stream;
  const int ne = c.ne, nv = c.nv, K2 = 2 * k;
  const size_t NV = (size_t)nv * K2, NE = (size_t)ne * K2;
  w.div_d.alloc(nv);
  w.div_dis.alloc(nv);
  w.div_ds.alloc(nv);
  w.div_rhs.alloc(NV);
  w.div_y.alloc(NV);
  w.div_t.alloc(NV);
  w.div_u.alloc(NV);
  w.div_e.alloc(NE);
  w.div_me.alloc(NE);
  // vertex scale and boundary mask (div_rhs holds the mask for a moment)
  w.div_d.zero(s);
  EMG_CUDA(cudaMemsetAsync(w.div_rhs.p, 0, sizeof(double) * nv, s));
  div_scale_edges_kernel<<<(unsigned)((ne + 255) / 256), 256, 0, s>>>(ne, c.rp.p, c.ci.p, c.Msv.p, c.edges.p,
                                                                      c.ebdr.p, w.div_d.p, w.div_rhs.p);
  EMG_LAUNCH_CHECK();
  div_scale_vertices_kernel<<<(unsigned)((nv + 255) / 256), 256, 0, s>>>(nv, w.div_d.p, w.div_rhs.p, w.div_dis.p,
                                                                         w.div_ds.p);
  EMG_LAUNCH_CHECK();
  // right-hand side: D^-1/2 G^T (b - A x) / (i w)
  spmm_complex(ne, k, c.rp.p, c.ci.p, c.Cv.p, c.Msv.p, omega, x, b, w.div_e.p, true, false, s);
  ams_restrict<double>(nv, K2, 0, c.vinc_rp.p, c.vinc.p, nullptr, w.div_e.p, w.div_t.p, s);
  {
    const long total = (long)nv * k;
    div_rhs_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(total, k, omega, w.div_dis.p,
                                                                   (const double2 *)w.div_t.p,
                                                                   (double2 *)w.div_rhs.p);
    EMG_LAUNCH_CHECK();
  }
  // scaled operator: D^-1/2 G^T Ms G D^-1/2
  auto op = [&](const double *p_, double *s_) {
    vrow_scale<double, double>(nv, K2, w.div_dis.p, p_, w.div_t.p, s);
    w.div_e.zero(s);
    ams_prolong_add<double>(ne, K2, 0, c.edges.p, nullptr, w.div_t.p, w.div_e.p, s);
    SpmmArgs a;
    std::memset(&a, 0, sizeof(a));
    a.n = ne;
    a.rp = c.rp.p;
    a.ci = c.ci.p;
    a.vc = c.Msv.p;
    a.vm = nullptr;
    a.omega = omega;
    a.x = w.div_e.p;
    a.y = w.div_me.p;
    a.relax_w = 1.0;
    a.mode = SPMM_AX;
    spmm_nnz<double>(K2, a, c.nnz, s);
    ams_restrict<double>(nv, K2, 0, c.vinc_rp.p, c.vinc.p, nullptr, w.div_me.p, w.div_u.p, s);
    vrow_scale<double, double>(nv, K2, w.div_dis.p, w.div_u.p, s_, s);
  };
  // scaled preconditioner: D^1/2 V D^1/2 with V the gradient space's V-cycle
  auto pc = [&](const double *r_, double *z_) {
    if (fp32) {
      w.div_tf.alloc(NV);
      w.div_uf.alloc(NV);
      vrow_scale<double, float>(nv, K2, w.div_ds.p, r_, w.div_tf.p, s);
      w.bams32.grad_vcycle(w.div_tf.p, w.div_uf.p, s);
      vrow_scale<float, double>(nv, K2, w.div_ds.p, w.div_uf.p, z_, s);
    } else {
      vrow_scale<double, double>(nv, K2, w.div_ds.p, r_, w.div_t.p, s);
      w.bams64.grad_vcycle(w.div_t.p, w.div_u.p, s);
      vrow_scale<double, double>(nv, K2, w.div_ds.p, w.div_u.p, z_, s);
    }
  };
  w.fcg_div.mmax = 2;
  w.fcg_div.check_every = c.opt.block_fcg_check_every;
  w.fcg_div.verbose = c.opt.verbose > 1;
  w.fcg_div.total_its = 0;
  w.fcg_div.solve_with(nv, K2, pc, op, w.div_rhs.p, w.div_y.p, c.opt.div_rtol, c.opt.div_max_it, s);
  // x += G D^-1/2 y
  vrow_scale<double, double>(nv, K2, w.div_dis.p, w.div_y.p, w.div_t.p, s);
  ams_prolong_add<double>(ne, K2, 0, c.edges.p, nullptr, w.div_t.p, x, s);
  return w.fcg_div.total_its;
}

// batched fast path on device vectors, one block of k (a power of two <= 32)
// columns
static void solve_block_pow2(Context &c, int k, const double *freqs, const double *rhs_dev, double *x_dev,
                             const emg_block_opts &o, emg_solve_info *infos) {
  need(c.assembled, EMG_ERR_STATE, "solve_block before assemble_matrix");
  need(k >= 1 && (k & (k - 1)) == 0 && k <= 32, EMG_ERR_ARG, "block width k must be a power of two <= 32");
  Workspace &w = *c.ws;
  const int n = c.ne;
  std::vector<double> om(k), col(2 * k);
  double lg = 0;
  for (int j = 0; j < k; ++j) {
    need(freqs[j] > 0, EMG_ERR_ARG, "frequencies must be positive");
    om[j] = 2 * PI * freqs[j];
    col[2 * j] = col[2 * j + 1] = om[j];
    lg += std::log(om[j]);
  }
  const double wref = std::exp(lg / k);
  const bool fp32 = o.inner_fp32 < 0 ? c.opt.inner_fp32 != 0 : o.inner_fp32 != 0;
  auto t0 = std::chrono::steady_clock::now();
  if (fp32 && !w.block_ready32) {
    ams_setup<float>(c, w.bams32, false, 0.0, wref);
    w.block_ready32 = true;
  }
  if (!fp32 && !w.block_ready64) {
    ams_setup<double>(c, w.bams64, false, 0.0, wref);
    w.block_ready64 = true;
  }
  c.kernel_ms["block_setup"] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  auto tc = std::chrono::steady_clock::now();
  if (fp32) w.bams32.set_columns(col, c.stream);
  else w.bams64.set_columns(col, c.stream);
  c.kernel_ms["setup_columns"] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tc).count();
  // b = conj(s): the real-form system equals (C + i w Ms) z = conj(s)
  w.vec_a.alloc((size_t)n * k * 2);
  conj_copy_kernel<<<(unsigned)(((long)n * k + 255) / 256), 256, 0, c.stream>>>((long)n * k, (const double2 *)rhs_dev,
                                                                               (double2 *)w.vec_a.p);
  EMG_LAUNCH_CHECK();
  w.gm.k = k;
  w.gm.restart = o.restart > 0 ? o.restart : c.opt.gmres_restart;
  // with the FP64 fallback behind it, an FP32 column that stops making
  // progress (less than 2x over a restart cycle) is handed over early
  w.gm.stall_factor = (fp32 && c.opt.block_fp64_fallback) ? 0.5 : 0.0;
  w.gm.floor_stop = c.opt.block_floor_stop != 0;
  w.gm.omega.upload(om, c.stream);
  w.fcg64.mmax = w.fcg32.mmax = c.opt.block_fcg_mmax;
  w.fcg64.check_every = w.fcg32.check_every = c.opt.block_fcg_check_every;
  w.fcg64.verbose = w.fcg32.verbose = c.opt.verbose > 1;
  w.fcg64.total_its = w.fcg32.total_its = 0;
  if (fp32) {
    w.f_in.alloc((size_t)n * k * 2);
    w.f_out.alloc((size_t)n * k * 2);
  }
  // mixed precision: the AMS preconditioner (smoothers, transfers, nodal
  // V-cycles) runs in FP32; the FCG recurrences and its operator B = C + w Ms
  // stay in FP64, because B p loses the gradient subspace of the air in FP32
  // (w sigma_air mu h^2 ~ 1e-10 sits far below FP32 resolution).
  const int K2 = 2 * k;
  if (fp32) w.omega_cols.upload(col, c.stream);
  auto opB64 = [&](const double *p_, double *s_) {
    SpmmArgs a;
    std::memset(&a, 0, sizeof(a));
    a.n = n;
    a.rp = c.rp.p;
    a.ci = c.ci.p;
    a.vc = c.Cv.p;
    a.vm = c.Msv.p;
    a.l1c = a.l1m = nullptr;
    a.omega = w.omega_cols.p;
    a.x = p_;
    a.b = nullptr;
    a.y = s_;
    a.relax_w = 1.0;
    a.mode = SPMM_AX;
    KernelProfiler &pf = profiler();
    cudaEvent_t ev = nullptr, ph = nullptr;
    if (pf.enabled)
      pf.begin("spmm_edge_fp64", c.stream, spmm_algo_bytes(n, c.nnz, K2, 8, true, SPMM_AX), &ev);
    if (pf.phases) pf.begin("phase_opB", c.stream, 0, &ph);
    const TiledPattern *tp = tiled_pattern(c, c.rp.p, c.h_rp, c.h_ci, K2 * 8);
    if (tp) spmm_tiled<double>(K2, a, *tp, c.stream);
    else spmm_nnz<double>(K2, a, c.nnz, c.stream);
    if (pf.enabled) pf.end("spmm_edge_fp64", c.stream, ev);
    if (pf.phases) pf.end("phase_opB", c.stream, ph);
  };
  auto pc32 = [&](const double *r_, double *z_) {
    KernelProfiler &pf = profiler();
    cudaEvent_t ph = nullptr;
    if (pf.phases) pf.begin("phase_ams", c.stream, 0, &ph);
    (void)r_;  // w.f_in holds (float) r_: the FCG update writes it
    (void)z_;  // z = f_out + G gphi is formed inside the FCG's passes
    w.bams32.apply(w.f_in.p, w.f_out.p, c.stream);
    if (pf.phases) pf.end("phase_ams", c.stream, ph);
  };
  Fcg<double>::ZSplit zsplit{c.edges.p, nullptr, nullptr};
  auto pc = [&](const double *v, double *z) {
    KernelProfiler &pf = profiler();
    cudaEvent_t ph = nullptr;
    if (pf.phases) pf.begin("phase_fcg", c.stream, 0, &ph);
    if (fp32) {
      if (w.fcg64.mmax > 4) fail(EMG_ERR_OPTION, "-emg_block_fcg_mmax above 4 with the FP32 preconditioner");
      zsplit.x = w.f_out.p;
      zsplit.phi = w.bams32.gphi();
      w.fcg64.solve_with(n, K2, pc32, opB64, v, z, c.opt.block_inner_rtol, c.opt.block_inner_max_it, c.stream,
                         w.f_in.p, &zsplit);
    }
    else w.fcg64.solve(w.bams64, v, z, c.opt.block_inner_rtol, c.opt.block_inner_max_it, c.stream);
    if (pf.phases) pf.end("phase_fcg", c.stream, ph);
  };
  SolveStats st;
  {
    KernelProfiler &pf = profiler();
    cudaEvent_t ph = nullptr;
    if (pf.phases) pf.begin("phase_fgmres", c.stream, 0, &ph);
    // FP32-preconditioned columns iterate further (rounding noise of the
    // FP32 AMS in the gradient space of the air is invisible to the residual)
    const double rtol = (o.rtol > 0 ? o.rtol : c.opt.e_rtol) * (fp32 ? c.opt.block_fp32_rtol_factor : 1.0);
    try {
      w.gm.solve(c, w.vec_a.p, x_dev, o.use_guess != 0, rtol, o.max_it > 0 ? o.max_it : c.opt.K_max_it, false, pc,
                 st);
    } catch (...) {
      // a fused V-cycle whose barrier wait gave up leaves garbage that the
      // Krylov checks report first: name the root cause instead
      (void)cudaStreamSynchronize(c.stream);
      if (fp32) w.bams32.check_fused(c.stream);
      else w.bams64.check_fused(c.stream);
      throw;
    }
    if (pf.phases) pf.end("phase_fgmres", c.stream, ph);
  }
  EMG_CUDA(cudaStreamSynchronize(c.stream));
  if (fp32) w.bams32.check_fused(c.stream);
  else w.bams64.check_fused(c.stream);
  long inner = w.fcg64.total_its;
  c.kernel_ms["div_correction"] = 0;
  c.kernel_ms["div_its"] = 0;
  if (c.opt.div_correction) {
    auto td = std::chrono::steady_clock::now();
    const long dits = div_correct(c, k, fp32, w.vec_a.p, x_dev, w.gm.omega.p);
    // the true residual of the corrected solution
    std::vector<double> rn(k), bn(k);
    spmm_complex(n, k, c.rp.p, c.ci.p, c.Cv.p, c.Msv.p, w.gm.omega.p, x_dev, w.vec_a.p, w.gm.r.p, true, false,
                 c.stream);
    w.gm.nrm.zero(c.stream);
    cnorm2(n, k, w.gm.r.p, w.gm.nrm.p, c.stream);
    w.gm.nrm.download(rn.data(), k, c.stream);
    w.gm.nrm.zero(c.stream);
    cnorm2(n, k, w.vec_a.p, w.gm.nrm.p, c.stream);
    w.gm.nrm.download(bn.data(), k, c.stream);
    EMG_CUDA(cudaStreamSynchronize(c.stream));
    const double rtol_c = (o.rtol > 0 ? o.rtol : c.opt.e_rtol) * (fp32 ? c.opt.block_fp32_rtol_factor : 1.0);
    for (int j = 0; j < k; ++j) {
      st.true_res[j] = bn[j] > 0 ? std::sqrt(rn[j] / bn[j]) : 0.0;
      st.converged[j] = st.true_res[j] <= rtol_c * 1.0000001 || bn[j] == 0 ? 1 : 0;
      if (j < (int)st.at_floor.size())
        st.at_floor[j] = !st.converged[j] && w.gm.floor_stop && st.true_res[j] <= 2.0 * st.floor_res[j] ? 1 : 0;
    }
    const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - td).count();
    st.seconds += ms * 1e-3;
    c.kernel_ms["div_correction"] = ms;
    c.kernel_ms["div_its"] = (double)dits;
    // the correction is an oblique projection of the residual (its metric is
    // the sigma-weighted mass), so a column's residual norm can rise past
    // rtol; such columns continue from the corrected solution
    bool all_ok = true;
    for (int j = 0; j < k; ++j) all_ok = all_ok && st.settled(j);
    if (!all_ok) {
      SolveStats st2;
      w.gm.solve(c, w.vec_a.p, x_dev, true, rtol_c, o.max_it > 0 ? o.max_it : c.opt.K_max_it, false, pc, st2);
      st.outer_its += st2.outer_its;
      st.seconds += st2.seconds;
      for (int j = 0; j < k; ++j) {
        st.col_its[j] += st2.col_its[j];
        st.true_res[j] = st2.true_res[j];
        st.converged[j] = st2.converged[j];
        st.floor_res[j] = st2.floor_res[j];
        st.at_floor[j] = st2.at_floor[j];
      }
      inner = w.fcg64.total_its;
    }
  }
  if (infos)
    for (int j = 0; j < k; ++j) fill_info(&infos[j], st, inner, j);
  c.kernel_ms["solve_block"] = st.seconds * 1e3;
  c.block_initial_res = st.initial_res;
  c.block_floor_res = st.floor_res;
  // a column the FP32 preconditioner could not carry to rtol within max_it
  // (stagnation at low frequency) is finished with the FP64 preconditioner,
  // starting from where it stopped; converged columns pass through at the
  // cost of one residual
  bool all_conv = true;
  for (int j = 0; j < k; ++j) all_conv = all_conv && st.settled(j);
  if (fp32 && !all_conv && c.opt.block_fp64_fallback) {
    emg_block_opts o2 = o;
    o2.inner_fp32 = 0;
    o2.use_guess = 1;
    std::vector<emg_solve_info> inf2(k);
    std::vector<double> r0 = st.initial_res;
    const double s1 = st.seconds;
    solve_block_pow2(c, k, freqs, rhs_dev, x_dev, o2, inf2.data());
    // block_floor_res now holds the FP64 pass's floors
    if (infos)
      for (int j = 0; j < k; ++j) {
        infos[j].outer_its += inf2[j].outer_its;
        infos[j].inner_its += inf2[j].inner_its;
        infos[j].reason = inf2[j].reason;
        infos[j].true_rel_res = inf2[j].true_rel_res;
        infos[j].seconds += inf2[j].seconds;
      }
    c.kernel_ms["solve_block"] += s1 * 1e3;
    c.block_initial_res = r0;
  }
}

// columns src[0..m) of an n x k complex block into an n x kb block (zero
// columns beyond m), and back
struct ColMap {
  int m;
  int src[32];
};

__global__ void gather_cols_kernel(long n, int k, int kb, ColMap cm, const double2 *__restrict__ in,
                                   double2 *__restrict__ out) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= n * kb) return;
  const long i = t / kb;
  const int j = (int)(t - i * kb);
  out[t] = j < cm.m ? in[i * k + cm.src[j]] : make_double2(0.0, 0.0);
}

__global__ void scatter_cols_kernel(long n, int k, int kb, ColMap cm, const double2 *__restrict__ in,
                                    double2 *__restrict__ out) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= n * cm.m) return;
  const long i = t / cm.m;
  const int j = (int)(t - i * cm.m);
  out[i * k + cm.src[j]] = in[i * kb + j];
}

// The columns idx of an n x k block, in blocks of at most kMaxBlock columns
// solved one after another; a block whose width is not a power of two is
// padded with zero right-hand sides (they converge at once and stay inactive
// in the inner solves) at its last column's frequency.
static void solve_block_subset(Context &c, const std::vector<int> &idx, int k, const double *freqs,
                               const double *rhs_dev, double *x_dev, const emg_block_opts &o,
                               emg_solve_info *infos, double &total_s, std::vector<double> &r0,
                               std::vector<double> &fl) {
  constexpr int kMaxBlock = 32;
  const int m = (int)idx.size();
  int kp = 1;
  while (kp < m) kp <<= 1;
  if (m == k && kp == k && k <= kMaxBlock) {  // the whole block as it lies
    solve_block_pow2(c, k, freqs, rhs_dev, x_dev, o, infos);
    total_s += c.kernel_ms["solve_block"] * 1e-3;
    for (int j = 0; j < k && j < (int)c.block_initial_res.size(); ++j) r0[j] = c.block_initial_res[j];
    for (int j = 0; j < k && j < (int)c.block_floor_res.size(); ++j) fl[j] = c.block_floor_res[j];
    return;
  }
  Workspace &w = *c.ws;
  const long n = c.ne;
  for (int j0 = 0; j0 < m; j0 += kMaxBlock) {
    ColMap cm;
    cm.m = std::min(kMaxBlock, m - j0);
    int kb = 1;
    while (kb < cm.m) kb <<= 1;
    std::vector<double> f(kb, freqs[idx[j0 + cm.m - 1]]);
    for (int j = 0; j < cm.m; ++j) {
      cm.src[j] = idx[j0 + j];
      f[j] = freqs[cm.src[j]];
    }
    w.blk_rhs.alloc((size_t)n * kb * 2);
    w.blk_x.alloc((size_t)n * kb * 2);
    const unsigned gb = (unsigned)((n * kb + 255) / 256), gs = (unsigned)((n * cm.m + 255) / 256);
    gather_cols_kernel<<<gb, 256, 0, c.stream>>>(n, k, kb, cm, (const double2 *)rhs_dev, (double2 *)w.blk_rhs.p);
    EMG_LAUNCH_CHECK();
    if (o.use_guess) {
      gather_cols_kernel<<<gb, 256, 0, c.stream>>>(n, k, kb, cm, (const double2 *)x_dev, (double2 *)w.blk_x.p);
      EMG_LAUNCH_CHECK();
    }
    std::vector<emg_solve_info> inf(kb);
    solve_block_pow2(c, kb, f.data(), w.blk_rhs.p, w.blk_x.p, o, inf.data());
    scatter_cols_kernel<<<gs, 256, 0, c.stream>>>(n, k, kb, cm, (const double2 *)w.blk_x.p, (double2 *)x_dev);
    EMG_LAUNCH_CHECK();
    total_s += c.kernel_ms["solve_block"] * 1e-3;
    for (int j = 0; j < cm.m; ++j) {
      if (infos) infos[cm.src[j]] = inf[j];
      if (j < (int)c.block_initial_res.size()) r0[cm.src[j]] = c.block_initial_res[j];
      if (j < (int)c.block_floor_res.size()) fl[cm.src[j]] = c.block_floor_res[j];
    }
  }
}

// Any number of columns.  With the FP32 preconditioner, columns below
// -emg_block_fp64_below Hz are solved as their own block with the FP64 one:
// there the FP32 rounding noise left in the gradient space of the air reaches
// the receiver fields at the 1e-3 level whatever the residual.
static void solve_block_dev(Context &c, int k, const double *freqs, const double *rhs_dev, double *x_dev,
                            const emg_block_opts &o, emg_solve_info *infos) {
  need(k >= 1, EMG_ERR_ARG, "block width k must be positive");
  const bool fp32 = o.inner_fp32 < 0 ? c.opt.inner_fp32 != 0 : o.inner_fp32 != 0;
  std::vector<int> lo, hi;
  for (int j = 0; j < k; ++j) (fp32 && freqs[j] < c.opt.block_fp64_below_hz ? lo : hi).push_back(j);
  double total_s = 0;
  std::vector<double> r0(k, 1.0), fl(k, 0.0);
  if (!lo.empty()) {
    emg_block_opts o64 = o;
    o64.inner_fp32 = 0;
    solve_block_subset(c, lo, k, freqs, rhs_dev, x_dev, o64, infos, total_s, r0, fl);
  }
  if (!hi.empty()) solve_block_subset(c, hi, k, freqs, rhs_dev, x_dev, o, infos, total_s, r0, fl);
  EMG_CUDA(cudaStreamSynchronize(c.stream));
  c.kernel_ms["solve_block"] = total_s * 1e3;
  c.block_initial_res = r0;
  c.block_floor_res = fl;
}

int emg_solve_block_dev(emg_context *c, int k, const double *freqs, const double *rhs_dev, double *x_dev,
                        const emg_block_opts *opts, emg_solve_info *infos) {
  EMG_API_BEGIN
  need(c && freqs && rhs_dev && x_dev && opts, EMG_ERR_ARG, "null argument");
  use_device(*c);
  solve_block_dev(*c, k, freqs, rhs_dev, x_dev, *opts, infos);
  EMG_API_END
}

int emg_divergence_correct_dev(emg_context *c, int k, const double *freqs, const double *rhs_dev, double *x_dev,
                               int fp32, long *its) {
  EMG_API_BEGIN
  need(c && freqs && rhs_dev && x_dev, EMG_ERR_ARG, "null argument");
  need(k >= 1 && (k & (k - 1)) == 0 && k <= 32, EMG_ERR_ARG, "block width k must be a power of two <= 32");
  need(c->assembled, EMG_ERR_STATE, "divergence correction before assemble_matrix");
  use_device(*c);
  Workspace &w = *c->ws;
  need(fp32 ? w.block_ready32 : w.block_ready64, EMG_ERR_STATE,
       "divergence correction before a block solve of that precision");
  std::vector<double> om(k), col(2 * k);
  for (int j = 0; j < k; ++j) {
    need(freqs[j] > 0, EMG_ERR_ARG, "frequencies must be positive");
    om[j] = 2 * PI * freqs[j];
    col[2 * j] = col[2 * j + 1] = om[j];
  }
  if (fp32) w.bams32.set_columns(col, c->stream);
  else w.bams64.set_columns(col, c->stream);
  const long n = c->ne;
  w.vec_a.alloc((size_t)n * k * 2);
  conj_copy_kernel<<<(unsigned)((n * k + 255) / 256), 256, 0, c->stream>>>(n * k, (const double2 *)rhs_dev,
                                                                          (double2 *)w.vec_a.p);
  EMG_LAUNCH_CHECK();
  w.gm.omega.upload(om, c->stream);
  const long dits = div_correct(*c, k, fp32 != 0, w.vec_a.p, x_dev, w.gm.omega.p);
  EMG_CUDA(cudaStreamSynchronize(c->stream));
  if (its) *its = dits;
  EMG_API_END
}

int emg_solve_block(emg_context *c, int k, const double *freqs, const double *rhs, double *x,
                    const emg_block_opts *opts, emg_solve_info *infos) {
  EMG_API_BEGIN
  need(c && freqs && rhs && x && opts, EMG_ERR_ARG, "null argument");
  use_device(*c);
  const size_t N = (size_t)c->ne * k * 2;
  DBuf<double> b(N), xd(N);
  b.upload(rhs, N, c->stream);
  if (opts->use_guess) xd.upload(x, N, c->stream);
  solve_block_dev(*c, k, freqs, b.p, xd.p, *opts, infos);
  xd.download(x, N, c->stream);
  EMG_CUDA(cudaStreamSynchronize(c->stream));
  EMG_API_END
}

int emg_spmv_complex_dev(emg_context *c, int k, const double *omegas, const double *x_dev, double *y_dev,
                         int conj_out) {
  EMG_API_BEGIN
  need(c && omegas && x_dev && y_dev, EMG_ERR_ARG, "null argument");
  need(c->assembled, EMG_ERR_STATE, "operator not assembled");
  use_device(*c);
  c->ws->omega_k.upload(omegas, k, c->stream);
  spmm_complex(c->ne, k, c->rp.p, c->ci.p, c->Cv.p, c->Msv.p, c->ws->omega_k.p, x_dev, nullptr, y_dev, false,
               conj_out != 0, c->stream);
  EMG_API_END
}

int emg_spmm_layout_dev(emg_context *c, int fp32, int K, int v, int variant, const double *omegas,
                        const void *x_dev, const void *b_dev, void *y_dev) {
  EMG_API_BEGIN
  need(c && omegas && x_dev && b_dev && y_dev, EMG_ERR_ARG, "null argument");
  need(c->assembled, EMG_ERR_STATE, "operator not assembled");
  need(K >= 1 && K <= 64, EMG_ERR_ARG, "block width K out of range");
  use_device(*c);
  cudaStream_t s = c->stream;
  c->ws->omega_k.upload(omegas, K, s);
  SpmmArgs a;
  std::memset(&a, 0, sizeof(a));
  a.n = c->ne;
  a.rp = c->rp.p;
  a.ci = c->ci.p;
  a.omega = c->ws->omega_k.p;
  a.x = x_dev;
  a.b = b_dev;
  a.y = y_dev;
  a.relax_w = 1.0;
  a.mode = SPMM_RES;
  bool ok;
  if (fp32) {
    // the operator in FP32 (and as packed records) for this call only
    DBuf<float> vc(c->nnz), vm(c->nnz);
    DBuf<int4> pk(c->nnz);
    cvt_d2f(c->nnz, c->Cv.p, vc.p, s);
    cvt_d2f(c->nnz, c->Msv.p, vm.p, s);
    pack_records(c->nnz, c->ci.p, vc.p, vm.p, pk.p, s);
    std::vector<int> crp;
    const long nch = chunk_row_pointer(c->h_rp, crp);
    DBuf<int> dcrp;
    dcrp.upload(crp, s);
    DBuf<int4> ch((size_t)std::max(3 * nch, 3L));
    chunk_records(c->ne, c->rp.p, c->ci.p, vc.p, vm.p, dcrp.p, ch.p, s);
    a.vc = vc.p;
    a.vm = vm.p;
    a.pk = pk.p;
    a.ch = ch.p;
    a.crp = dcrp.p;
    ok = spmm_layout<float>(K, v, variant, a, s);
    EMG_CUDA(cudaStreamSynchronize(s));  // the temporaries are freed next
  } else {
    a.vc = c->Cv.p;
    a.vm = c->Msv.p;
    ok = spmm_layout<double>(K, v, variant, a, s);
  }
  if (!ok) fail(EMG_ERR_ARG, "lane layout V=%d variant %d is not available for K=%d", v, variant, K);
  EMG_API_END
}

int emg_last_residual_floors(emg_context *c, int k, double *rel) {
  EMG_API_BEGIN
  need(c && rel && k >= 0, EMG_ERR_ARG, "null argument");
  need((size_t)k <= c->block_floor_res.size(), EMG_ERR_STATE, "no block solve of that width yet");
  std::copy(c->block_floor_res.begin(), c->block_floor_res.begin() + k, rel);
  EMG_API_END
}

int emg_last_initial_residuals(emg_context *c, int k, double *rel) {
  EMG_API_BEGIN
  need(c && rel && k >= 0, EMG_ERR_ARG, "null argument");
  need((size_t)k <= c->block_initial_res.size(), EMG_ERR_STATE, "no block solve of that width yet");
  std::copy(c->block_initial_res.begin(), c->block_initial_res.begin() + k, rel);
  EMG_API_END
}

int emg_amg_levels(emg_context *c, int sp, int gpu, double w_ref, int max_rows, int *nlev, double *out) {
  EMG_API_BEGIN
  need(c && nlev && out, EMG_ERR_ARG, "null argument");
  need(c->assembled, EMG_ERR_STATE, "AMG levels before assemble_matrix");
  need(sp >= 0 && sp < NSUB, EMG_ERR_ARG, "subspace index out of range");
  use_device(*c);
  std::vector<double> v;
  amg_levels_report(*c, sp, gpu != 0, w_ref, v);
  const int nl = (int)(v.size() / 5);
  need(nl <= max_rows, EMG_ERR_ARG, "output holds too few levels");
  *nlev = nl;
  std::copy(v.begin(), v.end(), out);
  EMG_API_END
}

int emg_last_kernel_ms(emg_context *c, const char *name, double *ms) {
  EMG_API_BEGIN
  need(c && name && ms, EMG_ERR_ARG, "null argument");
  auto it = c->kernel_ms.find(name);
  need(it != c->kernel_ms.end(), EMG_ERR_ARG, "no timing recorded under that name");
  *ms = it->second;
  EMG_API_END
}

int emg_stream_synchronize(emg_context *c) {
  EMG_API_BEGIN
  need(c != nullptr, EMG_ERR_ARG, "null context");
  EMG_CUDA(cudaStreamSynchronize(c->stream));
  EMG_API_END
}

int emg_launch_count(long *n) {
  EMG_API_BEGIN
  need(n != nullptr, EMG_ERR_ARG, "null argument");
  *n = launch_count();
  EMG_API_END
}

int emg_profile_enable(int on) {
  EMG_API_BEGIN
  KernelProfiler &p = profiler();
  p.reset();
  p.enabled = on == 1;
  p.phases = on == 2;
  EMG_API_END
}

int emg_spmm_layouts(char *buf, long len) {
  EMG_API_BEGIN
  need(buf && len > 0, EMG_ERR_ARG, "null argument");
  const std::string r = tuner().report();
  const size_t m = std::min((size_t)len - 1, r.size());
  std::memcpy(buf, r.data(), m);
  buf[m] = '\0';
  EMG_API_END
}

int emg_profile_get(const char *bin, long *count, double *ms, double *bytes) {
  EMG_API_BEGIN
  need(bin && count && ms && bytes, EMG_ERR_ARG, "null argument");
  KernelProfiler &p = profiler();
  p.collect();
  *count = p.count.count(bin) ? p.count[bin] : 0;
  *ms = p.ms.count(bin) ? p.ms[bin] : 0.0;
  *bytes = p.bytes.count(bin) ? p.bytes[bin] : 0.0;
  EMG_API_END
}

// batched MT right-hand sides on the device: column j is polarisation
// modes[j] at frequency freqs[j]; out: n x k complex interleaved
int emg_assemble_rhs_mt_block_dev(emg_context *c, int k, const double *freqs, const int *modes, double *s_dev) {
  EMG_API_BEGIN
  need(c && freqs && modes && s_dev && k > 0, EMG_ERR_ARG, "null argument");
  need(c->assembled, EMG_ERR_STATE, "assemble_rhs_mt before assemble_matrix");
  for (int j = 0; j < k; ++j)
    need(modes[j] == EMG_SOL_MT_XY || modes[j] == EMG_SOL_MT_YX, EMG_ERR_ARG, "mode must be XY_POLAR or YX_POLAR");
  use_device(*c);
  rhs_mt_block(*c, k, freqs, modes, s_dev);
  EMG_API_END
}

int emg_assemble_rhs_mt_block(emg_context *c, int k, const double *freqs, const int *modes, double *s) {
  EMG_API_BEGIN
  need(c && freqs && modes && s && k > 0, EMG_ERR_ARG, "null argument");
  need(c->assembled, EMG_ERR_STATE, "assemble_rhs_mt before assemble_matrix");
  use_device(*c);
  DBuf<double> d((size_t)c->ne * k * 2);
  rhs_mt_block(*c, k, freqs, modes, d.p);
  d.download(s, (size_t)c->ne * k * 2, c->stream);
  EMG_CUDA(cudaStreamSynchronize(c->stream));
  EMG_API_END
}

}  // extern "C"
