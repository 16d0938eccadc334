// Internal declarations of the emfem_b200 library (host C++ + sm_100a CUDA).
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdint>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/emfem_b200.h"

namespace emg {

constexpr double PI = 3.14159265358979323846;  // em_defs.h:16
constexpr double MU = 4 * PI * 1E-7;           // em_defs.h:17
constexpr double DTOR = PI / 180.0;            // em_defs.h:21
constexpr double EPS = 1.0E-6;                 // em_defs.h:23

// ---------------------------------------------------------------------------
// errors: every C-ABI call catches Error and returns its code
// ---------------------------------------------------------------------------
struct Error : public std::runtime_error {
  int code;
  Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] void fail(int code, const char *fmt, ...);
void check_cuda(cudaError_t e, const char *what, const char *file, int line);
#define EMG_CUDA(x) ::emg::check_cuda((x), #x, __FILE__, __LINE__)
// every kernel launch is followed by this check, which also counts launches
void launch_check(const char *file, int line);
#define EMG_LAUNCH_CHECK() ::emg::launch_check(__FILE__, __LINE__)

// Event-based per-kernel profiler: bins named by kernel role; each record is a
// start/stop event pair on the launching stream plus the launch's
// algorithmic bytes.  Disabled unless enabled through the C ABI.
struct KernelProfiler {
  bool enabled = false;  // every kernel launch timed (AMS runs eagerly)
  bool phases = false;   // solver phases timed (graphs and fused launches kept)
  struct Rec {
    cudaEvent_t a, b;
    double bytes;
  };
  std::map<std::string, std::vector<Rec>> open;
  std::map<std::string, double> ms, bytes;
  std::map<std::string, long> count;
  void begin(const std::string &bin, cudaStream_t s, double algo_bytes, cudaEvent_t *start_out);
  void end(const std::string &bin, cudaStream_t s, cudaEvent_t start);
  void collect();  // synchronizes on the recorded events and folds them in
  void reset();
};
KernelProfiler &profiler();
long launch_count();
// a replayed CUDA graph runs the kernels captured into it: count them
void add_launches(long n);

// ---------------------------------------------------------------------------
// device buffer (cudaMalloc-backed, move-only)
// ---------------------------------------------------------------------------
template <typename T>
struct DBuf {
  T *p = nullptr;
  size_t n = 0;
  DBuf() = default;
  explicit DBuf(size_t count) { alloc(count); }
  DBuf(const DBuf &) = delete;
  DBuf &operator=(const DBuf &) = delete;
  DBuf(DBuf &&o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
  DBuf &operator=(DBuf &&o) noexcept {
    if (this != &o) { release(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
    return *this;
  }
  ~DBuf() { release(); }
  void alloc(size_t count) {
    if (count == n && p) return;
    release();
    if (count == 0) return;
    cudaError_t e = cudaMalloc((void **)&p, count * sizeof(T));
    if (e != cudaSuccess) {
      p = nullptr;
      (void)cudaGetLastError();
      fail(EMG_ERR_NOMEM, "device allocation of %zu bytes failed: %s", count * sizeof(T), cudaGetErrorString(e));
    }
    n = count;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  // grows the buffer when needed (never shrinks it) and copies count elements
  void upload(const T *h, size_t count, cudaStream_t s) {
    if (!p || count > n) alloc(count);
    if (count) EMG_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
  }
  void upload(const std::vector<T> &h, cudaStream_t s) { upload(h.data(), h.size(), s); }
  void download(T *h, size_t count, cudaStream_t s) const {
    if (count) EMG_CUDA(cudaMemcpyAsync(h, p, count * sizeof(T), cudaMemcpyDeviceToHost, s));
  }
  // count elements starting at element offset
  void download_at(T *h, size_t offset, size_t count, cudaStream_t s) const {
    if (offset + count > n) fail(EMG_ERR_ARG, "download past the end of a device buffer");
    if (count) EMG_CUDA(cudaMemcpyAsync(h, p + offset, count * sizeof(T), cudaMemcpyDeviceToHost, s));
  }
  void zero(cudaStream_t s) {
    if (n) EMG_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), s));
  }
  size_t bytes() const { return n * sizeof(T); }
};

// host CSR
struct HCsr {
  int n = 0, m = 0;
  std::vector<int> rp, ci;
  std::vector<double> vc, vm;  // two value parts (vm may be empty)
  long nnz() const { return rp.empty() ? 0 : rp[n]; }
};

// device CSR with one or two value parts in precision T
template <typename T>
struct DCsr {
  int n = 0, m = 0;
  long nnz = 0;
  DBuf<int> rp, ci;
  DBuf<T> vc, vm;
  DBuf<T> l1c, l1m;  // l1 row sums of |vc| and |vm| (smoother diagonals)
};

// Row tiles of a CSR pattern with per-tile column lists (spmm_tiled): tile t
// covers rows [t R, t R + R), its distinct columns are ucol[urp[t] ..
// urp[t+1]), and lci[k] is nonzero k's index in that list.
struct TiledPattern {
  int n = 0, R = 0, ntiles = 0, umax = 0;
  DBuf<int> urp, ucol;
  DBuf<unsigned short> lci;
};

// ---------------------------------------------------------------------------
// options (process_options, em_ctx.cc:100-175) + A_/B_ subset + emg keys
// ---------------------------------------------------------------------------
struct Options {
  int K_max_it = 100;
  double e_rtol = 1e-8, dual_rtol = 1e-6;
  int inner_pc_type = 0;  // mixed=0 ams=1 direct=2
  int pc_threshold = 500000;
  int n_tx_divisions = 20;
  double refine_fraction = 0.1;
  int refine_strategy = 1;
  int max_adaptive_refinements = 0, n_uniform_refinements = 0, max_dofs = 1000000;
  int n_groups = 1, mesh_format = 0, direct_solver_type = 0, save_mesh = 1;
  double max_tx_edge_length = -1, max_rx_edge_length = -1;
  std::string iprefix, oprefix;
  // A_ / B_ prefixes honoured by the GPU solver
  int gmres_restart = 30;
  double inner_rtol = 1e-2;
  int inner_max_it = 100;
  int fcg_mmax = 1;
  std::string ams_cycle = "034515430";  // cycle type 13
  std::string fp32_cycle = "0201";      // cycle of the FP32 AMS (gradient last)
  int ams_relax_times = 1;
  double ams_relax_weight = 1.0;
  double amg_theta = 0.25;
  int amg_pmax = 4;
  int amg_max_coarse = 200;
  int amg_max_levels = 25;
  int amg_relax_times = 1;
  int smoother_cheb = 1;  // Chebyshev (1) or l1-Jacobi (0) in AMS and AMG
  int cheb_degree = 2;        // Chebyshev degree of the edge smoother (reference-facing path)
  // the same in the batched path's AMS: one degree-4 sweep per smoothing
  // step (measured on the MT topography block of 16 columns at 1.8M edges:
  // 8.8 s per solve against 9.6 s for two degree-2 sweeps, 11.5 s for one)
  int block_cheb_degree = 4;
  int amg_cheb_degree = 2;    // the same on the nodal AMG levels
  int restrict_j0 = 1;        // nodal restrictions take the fed level's first smoothing step
  int amg_pre_smooth = 1;     // nodal levels smooth before the coarse correction (V(m, m)) or not (V(0, m))
  int block_floor_stop = 1;   // block FGMRES columns stop at the rounding floor of their residual
  int gpu_amg = 1;        // nodal AMG setup on the device (1) or on the host (0)
  int block_fp64_fallback = 1;  // batched path: columns the FP32 AMS leaves unconverged finish in FP64
  // batched path accuracy policy: FP32-preconditioned columns iterate to rtol
  // times this factor, and columns below block_fp64_below_hz are solved with
  // the FP64 AMS (0: none).  At one relative residual the receiver fields of
  // different preconditioners differ: on the MT topography block (1.8M
  // edges, rtol 1e-8) the per-RHS FP64 method's worst receiver H error was
  // 1.3e-4, the block path's 2.2e-4 at rtol x 0.1 and 4.6e-5 at rtol x 0.01
  double block_fp32_rtol_factor = 0.01;
  double block_fp64_below_hz = 0;
  // divergence correction after every block solve: x += G phi with phi the
  // vertex potential that makes G^T (b - A x) vanish at interior vertices
  int div_correction = 1;
  double div_rtol = 1e-9;
  int div_max_it = 100;
  // emg_*
  int inner_fp32 = 0;
  int graphs = 1;
  int ams_fused = 0;          // small nodal levels as one cooperative launch per V-cycle
  int fused_bps = 0;          // its resident blocks per SM cap (0: occupancy limit)
  int fused_rows = 1 << 30;   // levels below this many rows run fused
  double fused_wait_ms = 2000;   // bound of a fused V-cycle's grid-barrier wait
  int fused_test_withhold = 0;   // tests only: withhold the first barrier's release
  int pi_coupled = 0;         // vector Pi space with (1) or without (0) its x/y/z couplings
  // inner FCG of the batched path (emg_solve_block): a capped iteration count
  // per outer step; the flexible outer Krylov absorbs the inexactness
  double block_inner_rtol = 1e-2;
  int block_inner_max_it = 30;
  int block_fcg_mmax = 2;
  int block_fcg_check_every = 5;  // inner iterations between host looks at the column status
  int block_relax_times = 1;      // edge smoothing sweeps per '0' of the batched path's AMS cycle
  int spmm_tiled = 0;         // edge-column SpMMs gather through per-tile shared memory
  int tiled_smem_kb = 64;     // shared memory budget of one tile
  int verbose = 0;
};

struct Workspace;

// ---------------------------------------------------------------------------
// context (mirrors EMContext, em_ctx.h:15-64)
// ---------------------------------------------------------------------------
struct Context {
  int device = 0;
  cudaStream_t stream = nullptr;
  Options opt;
  // mesh
  int nv = 0, nt = 0, ne = 0;
  std::vector<double> h_pts;
  std::vector<int> h_tets, h_attr, h_edges, h_t2e, h_nbr, h_non;
  std::vector<unsigned char> h_ebdr;
  DBuf<double> pts;
  DBuf<int> tets, attr, edges, t2e, nbr, non;
  DBuf<unsigned char> ebdr;
  DBuf<int> ctet, cedge;           // canonical tets: sorted vertices, canonical edges
  DBuf<signed char> cpar;          // parity of the vertex sort
  // model
  int aniso_form = 0;
  std::vector<double> rho;
  int nrho = 0, ncol = 0;
  DBuf<double> sigma_tab;  // nrho x 9
  std::vector<double> h_sigma_tab;
  std::vector<double> freqs;
  // background (MT boundary data)
  std::vector<double> bg_corners, bg_ztop, bg_lsig;
  std::vector<int> bg_nlay;
  int bg_maxl = 0;
  // linear system
  bool have_ls = false;
  int tidx = -3;
  std::vector<int> h_rp, h_ci;
  long nnz = 0;
  DBuf<int> rp, ci, slot;          // slot: 36 per tet
  DBuf<double> Cv, Msv;            // C and Ms (omega-free mass) on the pattern
  DBuf<unsigned char> bdr_cell;
  bool assembled = false;
  double omega = 0;                // omega of the last assemble_matrix
  // vertex adjacency pattern for the nodal subspace operators
  std::vector<int> h_vrp, h_vci;
  DBuf<int> vrp, vci, vslot;       // vslot: 16 per tet
  DBuf<int> vinc_rp, vinc;         // vertex -> incident edge (e*2+endpoint)
  // vertex x edge pattern of G^T B (row v: edges of the tets around v)
  std::vector<int> h_grp, h_gci;
  DBuf<int> grp, gci, gslot;       // gslot: 24 per tet (4 vertices x 6 edges)
  // AMS (the preconditioner objects live in the workspace)
  bool have_pc = false;
  double pc_omega = 0;             // omega the hierarchy was built for (plain path)
  // solutions: named slots, interleaved complex n
  std::map<int, DBuf<double>> sol;
  // timing
  std::map<std::string, double> kernel_ms;
  // per column of the last block solve: ||b - A x0|| / ||b|| of its start
  std::vector<double> block_initial_res;
  std::vector<double> block_floor_res;  // per column of the last block solve: FP64 rounding floor of its residual
  // rank of each boundary edge among the boundary edges (-1 elsewhere)
  std::vector<int> h_bnd_rank;
  DBuf<int> bnd_rank;
  int n_bnd = 0;
  // point location index over the host mesh (built on first use)
  std::shared_ptr<struct PointIndex> locator;
  // tiled copies of the fixed patterns, keyed by (row pointer, bytes per x row)
  std::map<std::pair<const int *, int>, std::unique_ptr<TiledPattern>> tiles;
  std::unique_ptr<Workspace> ws;
  // learned warm start (network, optimiser state, per-edge features), built on first use
  std::shared_ptr<struct WarmStartNet> warm;
  Context();
  ~Context();
};

// the tiled copy of a fixed pattern of the context for x rows of row_bytes
// bytes (built on first use, before any capture); nullptr when tiling is off
// or no tile size fits the shared-memory budget
const TiledPattern *tiled_pattern(Context &c, const int *rp_dev, const std::vector<int> &h_rp,
                                  const std::vector<int> &h_ci, int row_bytes);

// device address of the fixed scratch of emg_estimate_error_noalloc on a
// device (looked up once per device, with it current; emg_estimate.cu)
double *noalloc_scratch_address(int device);

// records the message returned by emg_last_error() on this thread
void set_last_error(const char *msg);

// helpers implemented in the .cu/.cpp files
void sigma_table(int aniso_form, int nrho, int ncol, const double *rho, std::vector<double> &out);
void build_sparsity(Context &c);          // host: CSR pattern (make_sparsity_patterns)
void build_vertex_pattern(Context &c);    // host: vertex adjacency + incidence
void canonicalize(Context &c);            // device: sorted tets + canonical edges
void build_slot_maps(Context &c);         // device: tet -> CSR slots
void assemble_edge(Context &c);           // device: C, Ms, bdr cells
void assemble_nodal(Context &c, HCsr out[4]);  // device + download (G, Pi_x, Pi_y, Pi_z)
// the same on the device only: buf holds 8 vertex-pattern arrays, part p of
// operator sp (G, Pi_x, Pi_y, Pi_z) at (2 sp + p) x nnz(vertex pattern)
void assemble_nodal_device(Context &c, DBuf<double> &buf);
// Pi^T K Pi, 3 nv rows, row 3 v + d; coupled = false keeps only the x/y/z
// diagonal blocks (the three component spaces side by side, corrected at once)
void assemble_pi_vector(Context &c, HCsr &out, bool coupled);
void build_gtb_pattern(Context &c);       // host pattern + device slot map of G^T B
void assemble_gtb(Context &c, DBuf<double> &gc, DBuf<double> &gm);  // G^T C (boundary part), G^T Ms
void create_pc(Context &c, bool per_frequency_hierarchy, const std::vector<double> &omegas);
void destroy_pc(Context &c);

}  // namespace emg

// the opaque handle of the C ABI is the context itself
struct emg_context : public emg::Context {};
