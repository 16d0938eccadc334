// Batched sparse kernels over block vectors.
//
// Block vectors are n x K row-major (the K columns of a row are contiguous),
// so one pass over a matrix row serves every column.  Operators are stored as
// one CSR pattern with one or two value parts: A(w_c) = Ac + w_c * Am, where
// w_c is the angular frequency of column c.  This is the form of every
// operator of the path: B = C + w Ms on edges (src/em_la.cc:122-128) and the
// Galerkin operators of the nodal AMS subspaces, which are affine in w once
// their interpolation is fixed.
//
// Lane layout of spmm_kernel<T, K, V, NL>: a row is served by NL*CL lanes,
// CL = K/V lanes over column blocks of V contiguous columns (vector loads of
// V*sizeof(T) bytes) and NL lanes splitting the row's nonzeros (reduced with
// warp shuffles); 32/(NL*CL) rows per warp.  (V, NL) per (T, K) is picked by
// the autotuner in emg_linalg.cu.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace emg {

enum SpmmMode : int {
  SPMM_AX = 0,    // y = A x
  SPMM_RES = 1,   // y = b - A x
  SPMM_JAC = 2,   // y = x + w (b - A x) / d,  d = l1c + w_c l1m
  SPMM_ADD = 3,   // y = y + A x   (prolongation)
  // degree-2 Chebyshev smoothing on D^-1 A (D = l1 row sums, spectrum in
  // (0, 1]), fused into the two operator applications it needs:
  SPMM_CHEB1 = 4, // r = b - A x ; d = inv_theta D^-1 r ; y = x + d   (stores r, d)
  SPMM_CHEB2 = 5, // y += c1 d + c2 D^-1 (r - A d)      (x = d gathered, y in place)
  // a middle step of a Chebyshev smoother of degree > 2 (three-term
  // recurrence): r' = r - A d ; d' = c1 d + c2 D^-1 r' ; y += d'
  // (x = d gathered, b = r in, r = r' out (may alias b), d = d' out (not x))
  SPMM_CHEBK = 6,
  // restriction that also takes the first smoothing step of the level it
  // feeds from a zero guess: y = A x (that level's right-hand side b'), and
  // r = d = c1 b' / D' with D' = l1c + w_c l1m the fed level's l1 diagonal
  // (l1c/l1m of the args; d may be null), c1 = 1/theta (Chebyshev) or the
  // l1-Jacobi weight
  SPMM_AXJ0 = 7,
};

template <typename T, int V>
struct VecT;
template <> struct VecT<float, 1> { typedef float type; };
template <> struct VecT<float, 2> { typedef float2 type; };
template <> struct VecT<float, 4> { typedef float4 type; };
template <> struct VecT<double, 1> { typedef double type; };
template <> struct VecT<double, 2> { typedef double2 type; };

template <typename T, int V>
__device__ __forceinline__ void ldv(const T *__restrict__ p, T (&v)[V]) {
  typedef typename VecT<T, V>::type VT;
  VT t = __ldg(reinterpret_cast<const VT *>(p));
  const T *s = reinterpret_cast<const T *>(&t);
#pragma unroll
  for (int i = 0; i < V; ++i) v[i] = s[i];
}

template <typename T, int V>
__device__ __forceinline__ void ldv_plain(const T *p, T (&v)[V]) {
  typedef typename VecT<T, V>::type VT;
  VT t = *reinterpret_cast<const VT *>(p);
  const T *s = reinterpret_cast<const T *>(&t);
#pragma unroll
  for (int i = 0; i < V; ++i) v[i] = s[i];
}

template <typename T, int V>
__device__ __forceinline__ void stv(T *p, const T (&v)[V]) {
  typedef typename VecT<T, V>::type VT;
  VT t;
  T *s = reinterpret_cast<T *>(&t);
#pragma unroll
  for (int i = 0; i < V; ++i) s[i] = v[i];
  *reinterpret_cast<VT *>(p) = t;
}

struct SpmmArgs {
  int n;
  const int *rp, *ci;
  const void *vc, *vm;     // value parts (vm may be null)
  const void *l1c, *l1m;   // l1 row sums for SPMM_JAC
  const double *omega;     // K per-column shifts (device), may be null if vm null
  const void *x, *b;
  void *y;
  double relax_w;
  int mode;
  void *r, *d;             // Chebyshev work vectors (n x K)
  double c1, c2;           // Chebyshev coefficients (inv_theta in c1 for CHEB1)
  // FP32 two-part operators may also come as one 16-byte record per nonzero
  // (column, vc bits, vm bits, 0): one load per nonzero instead of three
  const int4 *pk;
  // ... or in chunks of 4 nonzeros, rows padded to whole chunks: chunk q is
  // three int4 at ch[3q]: columns, vc bits, vm bits (padding: column = the
  // row, values 0); row r owns chunks crp[r] .. crp[r+1]
  const int *crp;
  const int4 *ch;
};

// One step of a fused nodal V-cycle (vcycle_fused_kernel): the operations a
// V-cycle launches one by one, recorded with their arguments and replayed in
// order inside one cooperative launch with a grid barrier between steps.
enum FusedKind : int {
  FOP_SPMM = 0,    // SpMM in any mode (a: all fields)
  FOP_JAC0 = 1,    // y = w b / d                 (a: n, b, l1c, l1m, omega, relax_w, y)
  FOP_JAC0_2 = 2,  // y = d = w b / d             (a: n, b, l1c, l1m, omega, relax_w, y, d)
  FOP_COARSE = 3,  // x = inv(slot(c)) b, dense   (a: n = nc, b, y = x, vc = FP64 inverses, ci = column slots)
};

struct FusedOp {
  int kind;
  long nnz;        // nonzeros of an SpMM (algorithmic bytes)
  SpmmArgs a;
};

// Row epilogue shared by the SpMM kernels, in two halves: epi_load reads
// the row vectors the mode needs (b, x, r, y and the l1 sums; none of them
// depends on the row product, so the kernels issue these loads before the
// gathers and they overlap), epi_store combines them with the row product
// acc (columns cb*V .. cb*V+V-1 of row `row`) and stores the results.
template <typename T, int V>
struct EpiIn {
  T b[V], x[V], r[V], y[V];
  T dc, dm;
};

template <typename T, int K, int V>
__device__ __forceinline__ void epi_load(const SpmmArgs &a, int row, int cb, bool two, EpiIn<T, V> &e) {
  const long o = (long)row * K + cb * V;
  const T *__restrict__ x = static_cast<const T *>(a.x);
  T *y = static_cast<T *>(a.y);
  const int mode = a.mode;
  const bool cheb = mode == SPMM_CHEB1 || mode == SPMM_CHEB2 || mode == SPMM_CHEBK;
  // b of SPMM_CHEBK is r, which the same row overwrites: plain load
  if (mode == SPMM_RES || mode == SPMM_JAC || mode == SPMM_CHEB1) ldv<T, V>(static_cast<const T *>(a.b) + o, e.b);
  if (mode == SPMM_CHEBK) ldv_plain<T, V>(static_cast<const T *>(a.b) + o, e.b);
  if (mode == SPMM_JAC || cheb) ldv<T, V>(x + o, e.x);
  if (mode == SPMM_CHEB2) ldv<T, V>(static_cast<const T *>(a.r) + o, e.r);
  if (mode == SPMM_ADD || mode == SPMM_CHEB2 || mode == SPMM_CHEBK) ldv_plain<T, V>(y + o, e.y);
  if (mode == SPMM_JAC || cheb) {
    e.dc = __ldg(static_cast<const T *>(a.l1c) + row);
    e.dm = two ? __ldg(static_cast<const T *>(a.l1m) + row) : T(0);
  }
  if (mode == SPMM_AXJ0) {  // the fed level's diagonal; A itself has one part
    e.dc = __ldg(static_cast<const T *>(a.l1c) + row);
    e.dm = a.l1m ? __ldg(static_cast<const T *>(a.l1m) + row) : T(0);
  }
}

template <typename T, int K, int V>
__device__ __forceinline__ void epi_store(const SpmmArgs &a, int row, int cb, const T (&acc)[V], const T (&w)[V],
                                          bool two, const EpiIn<T, V> &e) {
  const long o = (long)row * K + cb * V;
  T *y = static_cast<T *>(a.y);
  T out[V];
  switch (a.mode) {
  case SPMM_AX:
#pragma unroll
    for (int i = 0; i < V; ++i) out[i] = acc[i];
    break;
  case SPMM_RES:
#pragma unroll
    for (int i = 0; i < V; ++i) out[i] = e.b[i] - acc[i];
    break;
  case SPMM_JAC:
#pragma unroll
    for (int i = 0; i < V; ++i) {
      T d = two ? e.dc + w[i] * e.dm : e.dc;
      out[i] = e.x[i] + (T)a.relax_w * (e.b[i] - acc[i]) / d;
    }
    break;
  case SPMM_ADD:
#pragma unroll
    for (int i = 0; i < V; ++i) out[i] = e.y[i] + acc[i];
    break;
  case SPMM_CHEB1: {
    T rr[V], dd[V];
#pragma unroll
    for (int i = 0; i < V; ++i) {
      T dg = two ? e.dc + w[i] * e.dm : e.dc;
      rr[i] = e.b[i] - acc[i];
      dd[i] = (T)a.c1 * rr[i] / dg;
      out[i] = e.x[i] + dd[i];
    }
    stv<T, V>(static_cast<T *>(a.r) + o, rr);
    stv<T, V>(static_cast<T *>(a.d) + o, dd);
    break;
  }
  case SPMM_AXJ0: {
    T dd[V];
#pragma unroll
    for (int i = 0; i < V; ++i) {
      const T dg = a.l1m ? e.dc + (T)__ldg(a.omega + cb * V + i) * e.dm : e.dc;
      out[i] = acc[i];
      dd[i] = (T)a.c1 * acc[i] / dg;
    }
    stv<T, V>(static_cast<T *>(a.r) + o, dd);
    if (a.d) stv<T, V>(static_cast<T *>(a.d) + o, dd);
    break;
  }
  case SPMM_CHEBK: {
    T rr[V], dd[V];
#pragma unroll
    for (int i = 0; i < V; ++i) {
      T dg = two ? e.dc + w[i] * e.dm : e.dc;
      rr[i] = e.b[i] - acc[i];
      dd[i] = (T)a.c1 * e.x[i] + (T)a.c2 * rr[i] / dg;
      out[i] = e.y[i] + dd[i];
    }
    stv<T, V>(static_cast<T *>(a.r) + o, rr);
    stv<T, V>(static_cast<T *>(a.d) + o, dd);
    break;
  }
  default:  // SPMM_CHEB2: x is d (gathered), r holds the residual
#pragma unroll
    for (int i = 0; i < V; ++i) {
      T dg = two ? e.dc + w[i] * e.dm : e.dc;
      out[i] = e.y[i] + (T)a.c1 * e.x[i] + (T)a.c2 * (e.r[i] - acc[i]) / dg;
    }
  }
  stv<T, V>(y + o, out);
}

template <typename T, int K, int V>
__device__ __forceinline__ void spmm_epilogue(const SpmmArgs &a, int row, int cb, const T (&acc)[V], const T (&w)[V],
                                              bool two) {
  EpiIn<T, V> e;
  epi_load<T, K, V>(a, row, cb, two, e);
  epi_store<T, K, V>(a, row, cb, acc, w, two, e);
}

// MINB > 1 caps the registers so that MINB blocks of 256 threads fit on an SM
// (more warps in flight for the load-latency-bound gathers, a few spills)
template <typename T, int K, int V, int NL, bool PK = false, int MINB = 1>
__global__ void __launch_bounds__(256, MINB) spmm_kernel(SpmmArgs a) {
  constexpr int CL = K / V;
  constexpr int G = NL * CL;
  static_assert(G <= 32 && (32 % G) == 0, "bad lane layout");
  const int lane = threadIdx.x & 31;
  const int gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int row = gwarp * (32 / G) + lane / G;
  const int sub = lane % G;
  const int cb = sub % CL;      // column block
  const int sl = sub / CL;      // nonzero slice
  const T *__restrict__ vc = static_cast<const T *>(a.vc);
  const T *__restrict__ vm = static_cast<const T *>(a.vm);
  const T *__restrict__ x = static_cast<const T *>(a.x);
  T acc[V];
#pragma unroll
  for (int i = 0; i < V; ++i) acc[i] = T(0);
  T w[V];
  const bool two = vm != nullptr;
#pragma unroll
  for (int i = 0; i < V; ++i) w[i] = two ? (T)__ldg(a.omega + cb * V + i) : T(0);
  const bool valid = row < a.n;
  EpiIn<T, V> epi;
  if (valid && sl == 0) epi_load<T, K, V>(a, row, cb, two, epi);
  if (valid) {
    const int kb = __ldg(a.rp + row), ke = __ldg(a.rp + row + 1);
    // U nonzeros per lane per round: all index/value loads of the round are
    // issued before the dependent x gathers, so U gathers are in flight at
    // once (rows are short, ~16 nonzeros, and split NL ways)
    constexpr int U = 4;
    for (int k0 = kb + sl; k0 < ke; k0 += NL * U) {
      int j[U];
      T c[U], m[U];
      bool ok[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int k = k0 + u * NL;
        ok[u] = k < ke;
        if constexpr (PK) {
          const int4 rec = ok[u] ? __ldg(a.pk + k) : make_int4(0, 0, 0, 0);
          j[u] = rec.x;
          c[u] = (T)__int_as_float(rec.y);
          m[u] = (T)__int_as_float(rec.z);
        } else {
          j[u] = ok[u] ? __ldg(a.ci + k) : 0;
          c[u] = ok[u] ? __ldg(vc + k) : T(0);
          m[u] = (ok[u] && two) ? __ldg(vm + k) : T(0);
        }
      }
      T xv[U][V];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (ok[u]) ldv<T, V>(x + (long)j[u] * K + cb * V, xv[u]);
        else {
#pragma unroll
          for (int i = 0; i < V; ++i) xv[u][i] = T(0);
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u)
#pragma unroll
        for (int i = 0; i < V; ++i) acc[i] = fma(two ? c[u] + w[i] * m[u] : c[u], xv[u][i], acc[i]);
    }
  }
#pragma unroll
  for (int off = CL; off < G; off <<= 1)
#pragma unroll
    for (int i = 0; i < V; ++i) acc[i] += __shfl_xor_sync(0xffffffffu, acc[i], off);
  if (!valid || sl != 0) return;
  epi_store<T, K, V>(a, row, cb, acc, w, two, epi);
}

// Software-pipelined row SpMM: CL = K / V lanes serve one row (lane j owns
// column block j), 32 / CL rows per warp.  A row's nonzeros go in chunks of
// U; the index and value loads of chunk i + 1 are issued right after the x
// gathers of chunk i, before its FMAs, so the two dependent latencies of a
// chunk (index load, then gather) overlap with those of its neighbours
// instead of adding up chunk after chunk.  No warp shuffles: a lane whose row
// is past the end leaves at once.  Measured on the MT topography edge matrix
// (1.8M rows, 32 columns) it was never faster than spmm_kernel with packed
// records over the solver's mix of modes, so the autotuner does not try it;
// emg_spmm_layout_dev runs it (tests, experiments).
template <typename T, int K, int V, int U, bool PK>
__global__ void __launch_bounds__(256) spmm_pipe_kernel(SpmmArgs a) {
  constexpr int CL = K / V;
  static_assert(CL <= 32 && (32 % CL) == 0, "bad lane layout");
  const int lane = threadIdx.x & 31;
  const int gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int row = gwarp * (32 / CL) + lane / CL;
  const int cb = lane % CL;
  if (row >= a.n) return;
  const T *__restrict__ vc = static_cast<const T *>(a.vc);
  const T *__restrict__ vm = static_cast<const T *>(a.vm);
  const T *__restrict__ x = static_cast<const T *>(a.x);
  const bool two = vm != nullptr;
  T w[V], acc[V];
#pragma unroll
  for (int i = 0; i < V; ++i) {
    w[i] = two ? (T)__ldg(a.omega + cb * V + i) : T(0);
    acc[i] = T(0);
  }
  EpiIn<T, V> epi;
  epi_load<T, K, V>(a, row, cb, two, epi);
  const int kb = __ldg(a.rp + row), ke = __ldg(a.rp + row + 1);
  int j[U];
  T c[U], m[U];
  auto load_chunk = [&](int k0) {
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int k = k0 + u;
      const bool ok = k < ke;
      if constexpr (PK) {
        const int4 rec = ok ? __ldg(a.pk + k) : make_int4(0, 0, 0, 0);
        j[u] = rec.x;
        c[u] = (T)__int_as_float(rec.y);
        m[u] = (T)__int_as_float(rec.z);
      } else {
        j[u] = ok ? __ldg(a.ci + k) : 0;
        c[u] = ok ? __ldg(vc + k) : T(0);
        m[u] = (ok && two) ? __ldg(vm + k) : T(0);
      }
    }
  };
  load_chunk(kb);
  for (int k0 = kb; k0 < ke; k0 += U) {
    T xv[U][V];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (k0 + u < ke) ldv<T, V>(x + (long)j[u] * K + cb * V, xv[u]);
      else {
#pragma unroll
        for (int i = 0; i < V; ++i) xv[u][i] = T(0);
      }
    }
    T cc[U], mm[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      cc[u] = c[u];
      mm[u] = m[u];
    }
    if (k0 + U < ke) load_chunk(k0 + U);
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
      for (int i = 0; i < V; ++i) acc[i] = fma(two ? cc[u] + w[i] * mm[u] : cc[u], xv[u][i], acc[i]);
  }
  epi_store<T, K, V>(a, row, cb, acc, w, two, epi);
}

// Chunked SpMM for FP32 two-part operators (SpmmArgs::ch): CL = K / V lanes
// per row as spmm_kernel with NL = 1, but a row's nonzeros come in whole
// chunks of 4 (three 16-byte loads per chunk, no bounds predicates, no zero
// fills), and where the lane's V columns come in pairs with one frequency
// (the real and imaginary parts of a complex column) each pair shares one
// coefficient c + w m.
template <bool PAIRS, int K, int V>
__device__ __forceinline__ void chunk_rows(const SpmmArgs &a, int q0, int q1, int cb, const float (&w)[V],
                                           float (&acc)[V]) {
  const float *__restrict__ xb = static_cast<const float *>(a.x) + cb * V;
  for (int q = q0; q < q1; ++q) {
    const int4 jj = __ldg(a.ch + 3 * q);
    const int4 cr = __ldg(a.ch + 3 * q + 1);
    const int4 mr = __ldg(a.ch + 3 * q + 2);
    const int j[4] = {jj.x, jj.y, jj.z, jj.w};
    const float c[4] = {__int_as_float(cr.x), __int_as_float(cr.y), __int_as_float(cr.z), __int_as_float(cr.w)};
    const float m[4] = {__int_as_float(mr.x), __int_as_float(mr.y), __int_as_float(mr.z), __int_as_float(mr.w)};
    float xv[4][V];
#pragma unroll
    for (int u = 0; u < 4; ++u) ldv<float, V>(xb + (long)j[u] * K, xv[u]);
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      if constexpr (PAIRS) {
#pragma unroll
        for (int i = 0; i < V; i += 2) {
          const float co = fmaf(w[i], m[u], c[u]);
          acc[i] = fmaf(co, xv[u][i], acc[i]);
          acc[i + 1] = fmaf(co, xv[u][i + 1], acc[i + 1]);
        }
      } else {
#pragma unroll
        for (int i = 0; i < V; ++i) acc[i] = fmaf(fmaf(w[i], m[u], c[u]), xv[u][i], acc[i]);
      }
    }
  }
}

template <int K, int V, int MINB>
__global__ void __launch_bounds__(256, MINB) spmm_chunk_kernel(SpmmArgs a) {
  constexpr int CL = K / V;
  static_assert(CL <= 32 && (32 % CL) == 0, "bad lane layout");
  const int lane = threadIdx.x & 31;
  const int gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int row = gwarp * (32 / CL) + lane / CL;
  const int cb = lane % CL;
  if (row >= a.n) return;  // no shuffles: a lane past the end leaves at once
  float w[V], acc[V];
  bool pairs = (V % 2) == 0;
#pragma unroll
  for (int i = 0; i < V; ++i) {
    w[i] = (float)__ldg(a.omega + cb * V + i);
    acc[i] = 0.f;
  }
#pragma unroll
  for (int i = 0; i + 1 < V; i += 2) pairs = pairs && w[i] == w[i + 1];
  EpiIn<float, V> epi;
  epi_load<float, K, V>(a, row, cb, true, epi);
  const int q0 = __ldg(a.crp + row), q1 = __ldg(a.crp + row + 1);
  if (pairs) chunk_rows<true, K, V>(a, q0, q1, cb, w, acc);
  else chunk_rows<false, K, V>(a, q0, q1, cb, w, acc);
  epi_store<float, K, V>(a, row, cb, acc, w, true, epi);
}

// Row-group SpMM: G = K / V lanes serve one row (lane j owns column block j),
// 32 / G rows per warp.  A row's nonzeros are loaded cooperatively, G at a
// time (lane j loads nonzero j of the chunk: index and both value parts in
// coalesced loads, no dependent rounds), then broadcast with warp shuffles,
// so that B gathers of x rows per lane are in flight at once.  Trip counts are
// uniform across the warp (the longest row of the warp sets them); entries
// past a row's end have zero coefficients and issue no gather.
template <typename T, int K, int V, int B>
__global__ void __launch_bounds__(256) spmm_rows_kernel(SpmmArgs a) {
  constexpr int G = K / V;
  constexpr int RPW = 32 / G;
  static_assert(G <= 32 && (32 % G) == 0 && (G % B) == 0, "bad row-group layout");
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int grp = lane / G, j = lane % G;
  const int row = gw * RPW + grp;
  const bool valid = row < a.n;
  const T *__restrict__ vc = static_cast<const T *>(a.vc);
  const T *__restrict__ vm = static_cast<const T *>(a.vm);
  const T *__restrict__ x = static_cast<const T *>(a.x);
  const bool two = vm != nullptr;
  T w[V], acc[V];
#pragma unroll
  for (int i = 0; i < V; ++i) {
    w[i] = two ? (T)__ldg(a.omega + j * V + i) : T(0);
    acc[i] = T(0);
  }
  const int kb = valid ? __ldg(a.rp + row) : 0;
  const int len = valid ? __ldg(a.rp + row + 1) - kb : 0;
  EpiIn<T, V> epi;
  if (valid) epi_load<T, K, V>(a, row, j, two, epi);
  int maxlen = len;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) maxlen = max(maxlen, __shfl_xor_sync(0xffffffffu, maxlen, off));
  for (int c0 = 0; c0 < maxlen; c0 += G) {
    // the index and value streams are read once: streaming loads keep them
    // out of L1, which the x gathers reuse
    const bool ok = c0 + j < len;
    const int cj = ok ? __ldcs(a.ci + kb + c0 + j) : 0;
    const T cc = ok ? __ldcs(vc + kb + c0 + j) : T(0);
    const T cm = (ok && two) ? __ldcs(vm + kb + c0 + j) : T(0);
#pragma unroll
    for (int t0 = 0; t0 < G; t0 += B) {
      T xv[B][V], ct[B], mt[B];
#pragma unroll
      for (int t = 0; t < B; ++t) {
        const int src = grp * G + t0 + t;
        const int jj = __shfl_sync(0xffffffffu, cj, src);
        ct[t] = __shfl_sync(0xffffffffu, cc, src);
        mt[t] = __shfl_sync(0xffffffffu, cm, src);
        if (c0 + t0 + t < len) ldv<T, V>(x + (long)jj * K + j * V, xv[t]);
        else {
#pragma unroll
          for (int i = 0; i < V; ++i) xv[t][i] = T(0);
        }
      }
#pragma unroll
      for (int t = 0; t < B; ++t)
#pragma unroll
        for (int i = 0; i < V; ++i) acc[i] = fma(two ? ct[t] + w[i] * mt[t] : ct[t], xv[t][i], acc[i]);
    }
  }
  if (!valid) return;
  epi_store<T, K, V>(a, row, j, acc, w, two, epi);
}

// Row tiles with their own column lists: tile t covers rows [t R, t R + R);
// its distinct columns are ucol[urp[t] .. urp[t+1]) (ascending), and lci[k]
// is nonzero k's position in that list.  One CTA stages the x rows of its
// tile's columns in shared memory once, then every row gathers from there:
// the L2 traffic of the gathers drops from nnz x K to (distinct columns) x K
// values per tile.
struct TiledArgs {
  int R;
  const int *urp, *ucol;
  const unsigned short *lci;
};

template <typename T, int K, int V>
__global__ void __launch_bounds__(256) spmm_tiled_kernel(SpmmArgs a, TiledArgs t) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *xs = reinterpret_cast<T *>(smem_raw);
  typedef typename VecT<T, V>::type VT;
  constexpr int CL = K / V;     // lanes over the columns of one row
  constexpr int RPW = 32 / CL;  // rows per warp
  static_assert(CL <= 32 && (32 % CL) == 0, "bad tiled lane layout");
  const int tile = blockIdx.x;
  const int u0 = __ldg(t.urp + tile), nu = __ldg(t.urp + tile + 1) - u0;
  const T *__restrict__ x = static_cast<const T *>(a.x);
  for (int idx = threadIdx.x; idx < nu * CL; idx += blockDim.x) {
    const int u = idx / CL, cb = idx - u * CL;
    const long g = __ldg(t.ucol + u0 + u);
    *reinterpret_cast<VT *>(xs + u * K + cb * V) = __ldg(reinterpret_cast<const VT *>(x + g * K + cb * V));
  }
  __syncthreads();
  const T *__restrict__ vc = static_cast<const T *>(a.vc);
  const T *__restrict__ vm = static_cast<const T *>(a.vm);
  const bool two = vm != nullptr;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int cb = lane % CL, sub = lane / CL;
  T w[V];
#pragma unroll
  for (int i = 0; i < V; ++i) w[i] = two ? (T)__ldg(a.omega + cb * V + i) : T(0);
  const int r0 = tile * t.R;
  const int r1 = min(a.n, r0 + t.R);
  const int nwarps = blockDim.x >> 5;
  for (int row = r0 + warp * RPW + sub; row < r1; row += nwarps * RPW) {
    T acc[V];
#pragma unroll
    for (int i = 0; i < V; ++i) acc[i] = T(0);
    const int kb = __ldg(a.rp + row), ke = __ldg(a.rp + row + 1);
    constexpr int U = 4;
    for (int k0 = kb; k0 < ke; k0 += U) {
      int j[U];
      T c[U], m[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int k = k0 + u;
        const bool ok = k < ke;
        j[u] = ok ? (int)__ldg(t.lci + k) : 0;
        c[u] = ok ? __ldg(vc + k) : T(0);
        m[u] = (ok && two) ? __ldg(vm + k) : T(0);
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (k0 + u >= ke) break;
        const VT xv = *reinterpret_cast<const VT *>(xs + j[u] * K + cb * V);
        const T *xe = reinterpret_cast<const T *>(&xv);
#pragma unroll
        for (int i = 0; i < V; ++i) acc[i] = fma(two ? c[u] + w[i] * m[u] : c[u], xe[i], acc[i]);
      }
    }
    spmm_epilogue<T, K, V>(a, row, cb, acc, w, two);
  }
}

}  // namespace emg
