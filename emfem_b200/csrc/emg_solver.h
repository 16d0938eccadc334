// Solver engine: AMS preconditioner, batched FCG, batched FGMRES.
#pragma once

#include <algorithm>
#include <functional>
#include <map>
#include <utility>
#include <string>
#include <vector>

#include "emg_amg.h"
#include "emg_internal.h"
#include "emg_linalg.h"

namespace emg {

// Cache of instantiated CUDA graphs keyed by an argument pair; owns the execs.
struct GraphCache {
  std::map<std::pair<const void *, void *>, cudaGraphExec_t> exec;
  std::map<std::pair<const void *, void *>, int> seen;
  std::map<std::pair<const void *, void *>, long> kernels;  // kernel nodes per graph
  GraphCache() = default;
  GraphCache(const GraphCache &) = delete;
  GraphCache &operator=(const GraphCache &) = delete;
  GraphCache(GraphCache &&o) noexcept
      : exec(std::move(o.exec)), seen(std::move(o.seen)), kernels(std::move(o.kernels)), epoch(o.epoch + 1) {
    o.exec.clear();
  }
  GraphCache &operator=(GraphCache &&o) noexcept {
    if (this != &o) {
      clear();
      exec = std::move(o.exec);
      seen = std::move(o.seen);
      kernels = std::move(o.kernels);
      epoch = std::max(epoch, o.epoch) + 1;
      o.exec.clear();
    }
    return *this;
  }
  ~GraphCache() { clear(); }
  long epoch = 0;  // bumped by every clear(): device addresses may have moved
  void clear() {
    ++epoch;
    for (auto &kv : exec) cudaGraphExecDestroy(kv.second);
    exec.clear();
    seen.clear();
    kernels.clear();
  }
};

// one pinned host word (move-only)
struct PinnedWord {
  int *p = nullptr;
  PinnedWord() = default;
  PinnedWord(const PinnedWord &) = delete;
  PinnedWord &operator=(const PinnedWord &) = delete;
  PinnedWord(PinnedWord &&o) noexcept : p(o.p) { o.p = nullptr; }
  PinnedWord &operator=(PinnedWord &&o) noexcept {
    if (this != &o) {
      release();
      p = o.p;
      o.p = nullptr;
    }
    return *this;
  }
  ~PinnedWord() { release(); }
  void release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
  }
};

// AMS subspaces: 0 = gradient G (cycle character '1'), 1..3 = Pi_x, Pi_y,
// Pi_z as separate scalar spaces ('3', '4', '5'), 4 = the vector space Pi
// with its coupled operator Pi^T B Pi ('2')
constexpr int NSUB = 5;
constexpr int SUB_PIVEC = 4;
inline int ams_subspace(char ch) {
  switch (ch) {
  case '1': return 0;
  case '2': return SUB_PIVEC;
  case '3': return 1;
  case '4': return 2;
  case '5': return 3;
  }
  return -1;
}

// AMS (Hiptmair-Xu auxiliary space preconditioner, as hypre's AMS applies it)
// for B(w) = C + w Ms on K real columns with per-column w.
template <typename T>
struct Ams {
  struct Level {
    DCsr<T> A, P, R;
    long nnzA = 0, nnzP = 0, nnzR = 0;
  };
  struct Sub {
    std::vector<Level> lv;       // operator levels (last has no P/R)
    HCsr coarse;                 // coarsest operator (host, two parts)
    int nc = 0;
    DBuf<double> cinv;           // n_distinct_omega x nc x nc
    std::vector<double> cinv_w;  // omegas the inverses were built for
  };
  Context *ctx = nullptr;          // owner of the fixed patterns (tiled copies)
  DCsr<T> B;                       // values only: pattern is the context's
  DBuf<int4> Bpk;                  // FP32 two-part B as packed records (column, vc, vm, 0); empty otherwise
  DBuf<int4> Bch;                  // the same in chunks of 4 nonzeros per row (SpmmArgs::ch); empty otherwise
  DBuf<int> Bcrp;                  // chunk row pointer of Bch
  const int *brp = nullptr, *bci = nullptr;
  long nnzB = 0;
  bool two = true;  // two value parts (batched) or combined (one frequency)
  Sub sub[NSUB];
  DBuf<T> tangent;
  // G^T B (vertex x edge): curl part (boundary elements only) and mass part
  const int *grp = nullptr, *gci = nullptr;
  long nnzG = 0;
  DBuf<T> gvc, gvm;
  DBuf<T> gtmp;                    // G^T b (nv x K)
  int ne = 0, nv = 0;
  const int *edges = nullptr, *inc_rp = nullptr, *inc = nullptr;
  std::string cycle = "034515430";
  int relax_times = 1;
  double relax_w = 1.0;
  int amg_relax_times = 1;
  int cheb = 1;                    // 1: Chebyshev smoothing, 0: l1-Jacobi
  int cheb_degree = 2;             // operator applications per edge smoothing sweep
  int amg_cheb_degree = 2;         // the same on the nodal levels
  bool restrict_j0 = true;         // restrictions take the fed level's first smoothing step
  bool amg_pre_smooth = true;      // nodal V(m, m) cycles; false: V(0, m)
  bool use_graphs = true;          // replay each application as one CUDA graph
  bool split_gradient = false;     // last '1' of the cycle returned as potential gphi()
  // each nodal V-cycle as one cooperative launch (emg_fused.cu) instead of
  // its 40-70 step launches; the step lists are recorded from vcycle()
  bool fused = false;
  int fused_bps = 0;               // resident blocks per SM cap (0: occupancy limit)
  int fused_rows = 1 << 30;        // levels with fewer rows run fused
  unsigned long long fused_wait_ns = 2000000000ull;  // bound of every grid-barrier wait
  int fused_withhold = 0;          // tests: the first barrier is never released
  int fused_from[NSUB] = {0, 0, 0, 0, 0};
  GraphCache graphs;
  std::vector<FusedOp> *rec = nullptr;  // set while vcycle() records instead of launching
  DBuf<FusedOp> fops[NSUB];
  int fops_n[NSUB] = {0, 0, 0, 0, 0};
  double fops_bytes[NSUB] = {0, 0, 0, 0, 0};
  long fused_epoch = -1;           // graphs.epoch the step lists were recorded at
  DBuf<unsigned> fbar;             // grid barrier words
  DBuf<int> ferr;                  // barrier timeout flag (device)
  PinnedWord h_ferr;               // pinned copy, refreshed after every application
  // per-call state
  int K = 0;
  DBuf<double> omega;              // K
  DBuf<int> cslot;                 // K, coarse-inverse index per column
  std::vector<double> h_omega;
  // workspace
  DBuf<T> er, ex2, ed, ed2;        // ed2, wd2: second direction buffers (degree > 2)
  std::vector<DBuf<T>> wb[NSUB], wx[NSUB], wr[NSUB], wx2[NSUB], wd[NSUB], wd2[NSUB];

  void set_columns(const std::vector<double> &col_omega, cudaStream_t s);
  void apply(const T *b, T *x, cudaStream_t s);
  void apply_eager(const T *b, T *x, cudaStream_t s);
  const T *gphi() const { return wx[0][0].p; }  // gradient potential (split form)
  // one V-cycle of the gradient space's nodal hierarchy on K vertex columns
  // (b, x: nv x K, device); the divergence correction's preconditioner
  void grad_vcycle(const T *b, T *x, cudaStream_t s);
  void spmm_B(int mode, const T *x, const T *b, T *y, cudaStream_t s);
  size_t device_bytes() const;

  // started: the restriction that fed level l already took its first
  // zero-guess smoothing step (SPMM_AXJ0)
  void vcycle(int sp, int l, cudaStream_t s, bool started = false);
  // runs subspace sp's V-cycle: the levels with at least fused_rows rows
  // step by step, the rest as one fused launch
  void run_vcycle(int sp, cudaStream_t s);
  void launch_fused(int sp, cudaStream_t s);
  // records the fused step lists for the current workspace (not while capturing)
  void prepare_fused(cudaStream_t s);
  // fails (and resets the barrier) when a fused launch reported a timeout
  void check_fused(cudaStream_t s);
  // step emitters: launch now, or append to *rec
  void emit_spmm(const SpmmArgs &a, long nnz, const char *bin, cudaStream_t s, const TiledPattern *tp = nullptr);
  // tiled copies of the edge pattern and of G^T B for this precision and K
  const TiledPattern *edge_tiles();
  const TiledPattern *gtb_tiles();
  void emit_jac0(int n, const T *b, const T *l1c, const T *l1m, double w, T *y, T *d, cudaStream_t s);
  void emit_coarse(int sp, const T *b, T *x, cudaStream_t s);
  // one smoothing application on operator A (edge B when A == nullptr);
  // returns the buffer holding the result (cur, or oth after a swap)
  T *smooth(const DCsr<T> *A, long nnz, int n, T *cur, T *oth, const T *b, T *rbuf, T *dbuf, T *dbuf2,
            bool zero_guess, const char *bin, cudaStream_t s, bool started = false);
  void ensure_workspace(cudaStream_t s);
  int ws_K = 0;
};

// Builds the AMS data for the context's mesh and operators.
//   per_frequency = true: the reference's flow -- B = C + w Ms combined for
//   one w, hierarchies from B(w) (create_pc per frequency);
//   per_frequency = false: two-part operators, hierarchies from w_ref, valid
//   for every frequency of a block.
template <typename T>
void ams_setup(Context &c, Ams<T> &ams, bool per_frequency, double w, double w_ref);

// tests: rows, nonzeros and absolute sums per level of a nodal hierarchy
// built on the device (gpu) or on the host
void amg_levels_report(Context &c, int sp, bool gpu, double w_ref, std::vector<double> &out);

// batched FCG on B(w_c) with AMS, K real columns; returns per-column iteration
// counts; x starts at zero.  Columns converge independently to
// ||r_c|| <= rtol ||b_c|| (unpreconditioned norm, src/em_la.cc:120).
template <typename T>
struct Fcg {
  int K = 0;
  int mmax = 1;
  DBuf<T> r, z, p;
  std::vector<DBuf<T>> P, S;  // previous directions and B-products (ring)
  DBuf<double> dots, eta, eord, alpha, beta, rn, bn;
  DBuf<T *> ptrs;          // ring orderings of the previous directions, per (head, nprev)
  int ptab_mmax = 0;
  DBuf<int> act, itsd, status;  // per-column activity and iteration counts; active count, NaN flag
  PinnedWord h_status;          // two words (see fcg_status_kernel)
  std::vector<int> its;
  long total_its = 0;
  int verbose = 0;
  int check_every = 1;     // iterations between host looks at the column status
  int solve(Ams<T> &ams, const T *b, T *x, double rtol, int maxit, cudaStream_t s);
  // generic form: pc(r, z) applies the preconditioner, opB(p, s) the operator;
  // n rows, K columns
  // r32: when given, kept equal to (float) r for an FP32 preconditioner
  // zs: the preconditioner leaves z split as x + G phi in FP32 (zs->x, zs->phi
  // over the edges zs->edges) instead of writing z; the dot products and the
  // direction then form z on the fly
  struct ZSplit {
    const int *edges;
    const float *x, *phi;
  };
  int solve_with(int n, int Kc, const std::function<void(const T *, T *)> &pc,
                 const std::function<void(const T *, T *)> &opB, const T *b, T *x, double rtol, int maxit,
                 cudaStream_t s, float *r32 = nullptr, const ZSplit *zs = nullptr);
};

struct SolveStats {
  int outer_its = 0;
  long inner_its = 0;
  std::vector<double> true_res;  // per column
  std::vector<int> col_its;
  std::vector<int> converged;
  std::vector<double> initial_res;  // per column: ||b - A x0|| / ||b|| of the start used
  std::vector<double> floor_res;    // per column: the FP64 rounding floor of the relative residual at exit
  std::vector<int> at_floor;        // per column: stopped at that floor above rtol
  double seconds = 0;
  bool settled(int c) const { return converged[c] || (c < (int)at_floor.size() && at_floor[c]); }
};

// Batched FGMRES(restart) on k complex columns (FP64):
//   real_form = true: the reference's real 2n system [[C,-M],[-M,-C]] with
//   real inner products (matshell_mult_a, src/em_la.cc:65-87);
//   real_form = false: (C + i w Ms) z = conj(s) with complex inner products.
// precond(v, z): z = P v on n x k complex (interleaved) device vectors.
struct Fgmres {
  int n = 0, k = 0, restart = 30;
  DBuf<double> V, Z, w, r, h, hn, scale, y, omega, nrm;
  DBuf<double> bnd, Hd, csd, snd, gd;  // per-column norms, Hessenberg, rotations, rotated rhs (device)
  DBuf<int> ints;                      // done, jc, its, conv per column; two status words
  PinnedWord h_status;
  DBuf<double> prevb;                  // residual norm at the previous restart, per column
  double stall_factor = 0;             // > 0: stop a column whose residual fell less than this over a cycle
  // complex form only: a column also stops once its residual reaches the
  // rounding floor of its own computation, u || |b| + |A| |x| || (recomputed
  // at every restart), when that lies above rtol ||b||
  bool floor_stop = false;
  DBuf<double> tol, bound2;            // per column: absolute stopping tolerance, the floor's squared scale
  int solve(Context &c, const double *b, double *x, bool use_guess, double rtol, int maxit, bool real_form,
            const std::function<void(const double *, double *)> &precond, SolveStats &st);
};

}  // namespace emg
