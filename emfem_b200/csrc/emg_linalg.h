// Host interface of the batched linear-algebra kernels (emg_linalg.cu).
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <string>
#include <tuple>

#include "emg_internal.h"
#include "emg_linalg.cuh"
#include "emg_tiles.h"

namespace emg {

// SpMM launcher with an autotuned lane layout per (precision, K, row-length
// class).  Tuning runs on the first large non-accumulating call it sees and
// times every legal (V, NL) candidate with CUDA events.
struct SpmmTuner {
  // (sizeof T, K, nonzeros-per-row class, row-count class) -> (V, NL)
  std::map<std::tuple<int, int, int, int>, std::pair<int, int>> best;
  bool allow_tuning = true;
  int tuned_count = 0;
  std::string report() const;
};

SpmmTuner &tuner();

// algorithmic bytes of one SpMM launch: every stored array read or written
// once (pattern, value parts, x, y, and b / x-row / l1 sums as the mode needs)
double spmm_algo_bytes(long n, long nnz, int K, int elem, bool two_parts, int mode);

// nnz of the operator selects the row-length class of the tuning table
template <typename T>
void spmm_nnz(int K, const SpmmArgs &a, long nnz, cudaStream_t s);

// one SpMM with a given lane layout (v, nl as in the tuning table: nl > 0 the
// row-split kernel, -B the row-group kernel, 100 + NL packed records,
// 200 + U / 300 + U the software-pipelined kernel on arrays / packed
// records, 400 + NL / 500 + NL the register-capped row-split kernel on packed
// records / arrays); false when the layout is not legal for (T, K)
template <typename T>
bool spmm_layout(int K, int v, int nl, const SpmmArgs &a, cudaStream_t s);
// FP32 two-part operator as one 16-byte record per nonzero (column, vc, vm, 0)
void pack_records(long nnz, const int *ci, const float *vc, const float *vm, int4 *out, cudaStream_t s);
// the same in chunks of 4 nonzeros per row (SpmmArgs::ch, spmm_chunk_kernel):
// chunk row pointer from a host CSR row pointer (returns the chunk count),
// then the chunks (3 int4 each) on the device
long chunk_row_pointer(const std::vector<int> &rp, std::vector<int> &crp);
void chunk_records(int n, const int *rp, const int *ci, const float *vc, const float *vm, const int *crp, int4 *ch,
                   cudaStream_t s);

// Tiles rows of a host CSR pattern for spmm_tiled: the largest R (a power of
// two <= r_max, >= 8) whose busiest tile has at most umax_limit distinct
// columns.  Returns false (tp untouched) when no such R exists.
bool build_tiled(int n, const std::vector<int> &rp, const std::vector<int> &ci, int umax_limit, int r_max,
                 TiledPattern &tp, cudaStream_t s);
// SpMM through a tiled pattern (a.rp is the pattern's row pointer; a.ci unused)
template <typename T>
void spmm_tiled(int K, const SpmmArgs &a, const TiledPattern &tp, cudaStream_t s);

// out[c] (+)= sum_i a[i*K+c] * b[i*K+c]   (FP64 accumulation); out must be zeroed
template <typename T>
void coldot(int n, int K, const T *a, const T *b, double *out, cudaStream_t s);
// three dot products in one pass: out[0..K) = (a1,b1), out[K..2K) = (a2,b2), out[2K..3K) = (a3,b3)
template <typename T>
void coldot3(int n, int K, const T *a1, const T *b1, const T *a2, const T *b2, const T *a3, const T *b3,
             double *out, cudaStream_t s);
// x += alpha_c p ; r -= alpha_c s ; rn[c] += ||r_c||^2 ; r32 = (float) r when given
template <typename T>
void fcg_update(int n, int K, const double *alpha, const T *p, const T *sv, T *x, T *r, double *rn, cudaStream_t s,
                float *r32 = nullptr);
// p = z - sum_j beta[j*K+c] * P_j  (nprev directions, pointers in a device array)
template <typename T>
void fcg_direction(int n, int K, const T *z, int nprev, T *const *Pj, const double *beta, T *p, cudaStream_t st);
// y = w * b / d   (first l1-Jacobi sweep from a zero guess)
template <typename T>
void jacobi0(int n, int K, const T *b, const T *l1c, const T *l1m, const double *omega, double w, T *y,
             cudaStream_t s);
// y = d = w * b / D  (first smoothing step from a zero guess, two outputs)
template <typename T>
void jacobi0_2(int n, int K, const T *b, const T *l1c, const T *l1m, const double *omega, double w, T *y, T *d,
               cudaStream_t s);
// precision conversion of block vectors
void cvt_d2f(long count, const double *a, float *b, cudaStream_t s);
void cvt_f2d(long count, const float *a, double *b, cudaStream_t s);
// z = x + G phi in FP64 (edge e: phi[v1] - phi[v0]) for K columns
void add_gradient_f2d(int ne, int K, const int *edges, const float *x, const float *phi, double *z, cudaStream_t s);
template <typename T>
void fill_zero(long count, T *a, cudaStream_t s);
// FCG steps with z = x + G phi formed on the fly (FP32 AMS output x, FP32
// gradient potential phi): out[j*K+c] += (z_c, S_j,c) for j < nprev (<= 4),
// and p = z - sum_j beta[j*K+c] P_j
struct DevPtrs4 {
  const double *p[4];
};
void zsplit_dots(int n, int K, const int *edges, const float *x, const float *phi, int nprev, const DevPtrs4 &S,
                 double *out, cudaStream_t s);
void zsplit_direction(int n, int K, const int *edges, const float *x, const float *phi, int nprev,
                      double *const *Pj, const double *beta, double *p, cudaStream_t s);

// AMS transfers between edges and vertices for K columns.
//   sp == 0: gradient G (row e: -1 at edges[e][0], +1 at edges[e][1])
//   sp == 1..3: Pi_d, d = sp-1 (row e: 0.5 t_e[d] at both endpoints)
//   sp == 4: Pi = [Pi_x Pi_y Pi_z], vertex vectors stored as rows 3 v + d
template <typename T>
void ams_restrict(int nv, int K, int sp, const int *inc_rp, const int *inc, const T *tangent, const T *r_edge,
                  T *r_vert, cudaStream_t s);
template <typename T>
void ams_prolong_add(int ne, int K, int sp, const int *edges, const T *tangent, const T *e_vert, T *x_edge,
                     cudaStream_t s);
// x[i,c] = sum_j inv[slot(c)][i][j] b[j,c]  (FP64 generalized inverse of the coarsest operator)
template <typename T>
void coarse_apply(int nc, int K, const double *inv, const int *col_slot, const T *b, T *x, cudaStream_t s);

// One nodal V-cycle as a single cooperative launch (emg_fused.cu): runs the
// recorded steps in order with a grid barrier between them.  bar: two words,
// zero before the first launch (every launch leaves them consistent); err:
// set nonzero when a barrier wait gave up, which ends the launch early.
// max_bps caps the resident blocks per SM (0: the occupancy limit).
// wait_ns bounds every barrier wait; withhold != 0 (tests only) makes the
// last block to arrive at the first barrier skip the release, so that the
// others' waits run out
template <typename T>
void vcycle_fused(int K, const FusedOp *ops, int nops, unsigned *bar, int *err, int max_bps, cudaStream_t s,
                  unsigned long long wait_ns = 2000000000ull, int withhold = 0);

// ---- complex (FP64) kernels of the outer FGMRES ------------------------------
// y = b - A(w_c) x  or  y = A(w_c) x, complex n x K; conj_out conjugates the
// product (the real-form operator of matshell_mult_a).
void spmm_complex(int n, int K, const int *rp, const int *ci, const double *Cv, const double *Mv,
                  const double *omega, const double *x, const double *b, double *y, bool residual, bool conj_out,
                  cudaStream_t s);
// h[j*K+c] = sum_i conj(V_j[i,c]) w[i,c]  for j < J (complex), V_j = V + j*stride
void cmultidot(int n, int K, int J, const double *V, long stride, const double *w, double *h, double *partial,
               int partial_blocks, cudaStream_t s);
// w -= sum_j h[j*K+c] V_j ; hn[c] = ||w_c||^2
void cgs_update(int n, int K, int J, const double *V, long stride, const double *h, double *w, double *hn,
                cudaStream_t s);
// v = w / scale[c]  (scale real)
void cscale(int n, int K, const double *w, const double *scale, double *v, cudaStream_t s);
// x += sum_j y[j*K+c] Z_j   (complex coefficients)
void cupdate(int n, int K, int J, const double *Z, long stride, const double *y, double *x, cudaStream_t s);
// out[c] += ||x_c||^2 over complex columns
void cnorm2(int n, int K, const double *x, double *out, cudaStream_t s);
// out[c] += || |b_c| + (|C| + w_c |Ms|) |x_c| ||^2 for K complex columns (K
// divides 32): u times its root bounds the rounding error of a computed
// residual b - (C + i w Ms) x, the floor below which no iteration can push it
void abs_bound2(int n, int K, const int *rp, const int *ci, const double *Cv, const double *Mv, const double *omega,
                const double *x, const double *b, double *out, cudaStream_t s);

}  // namespace emg
