// Fused nodal V-cycle: one cooperative launch per AMS subspace correction.
//
// A nodal AMG V-cycle of the AMS preconditioner is some 40-70 dependent
// operations (Chebyshev smoothing, residual, restriction, prolongation on
// each level, the dense coarsest solve), most of them on levels of a few
// hundred to a few thousand rows whose launch and ramp time exceed their
// work by 5-20x.  vcycle_fused_kernel runs the whole recorded sequence
// (FusedOp list, built on the host from the same code path that launches the
// steps one by one) in one launch: every block walks the list, executes its
// share of each step grid-stride, and meets the others at a grid barrier
// before the next step.  The blocks are co-resident (cooperative launch), so
// the barrier cannot deadlock; every wait is also bounded in time and sets
// an error word the host checks, so a fault in the barrier logic cannot hang
// the GPU.
//
// Within the kernel, block vectors written by one step are read by other
// SMs in the next: those loads go through L2 (ld.global.cg), never through
// the non-coherent L1 / read-only paths.  Matrices, l1 sums, omegas and the
// coarse inverses are read-only for the launch and use __ldg.

#include <cuda_runtime.h>

#include <map>
#include <utility>

#include "emg_linalg.h"

namespace emg {

namespace {

template <typename T, int K>
struct FusedLayout {
  static constexpr int V0 = (int)(16 / sizeof(T));
  static constexpr int V1 = K < V0 ? K : V0;
  static constexpr int V = (K / V1 > 32) ? K / 32 : V1;  // columns per lane
  static constexpr int CL = K / V;                        // lanes per column set
  static constexpr int NL = 32 / CL;                      // lanes splitting the nonzeros
  static_assert(CL * NL == 32 && CL * V == K, "bad fused layout");
};

template <typename T, int V>
__device__ __forceinline__ void ldv_cg(const T *p, T (&v)[V]) {
  typedef typename VecT<T, V>::type VT;
  VT t = __ldcg(reinterpret_cast<const VT *>(p));
  const T *s = reinterpret_cast<const T *>(&t);
#pragma unroll
  for (int i = 0; i < V; ++i) v[i] = s[i];
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_release(unsigned *p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Sense-free grid barrier: bar[0] counts arrivals, bar[1] is the generation.
// The last block to arrive resets the count and publishes the next
// generation; the others wait for it, at most ~2 s or 4M polls, after which
// the waiter records EMG_FUSED_TIMEOUT in *err.  A set error word releases
// every waiter.  Returns false when the launch must stop.
constexpr int EMG_FUSED_TIMEOUT = 1;

// withhold: the last block to arrive does not publish the next generation
// (a test of the bounded wait: the others wait for a flag that nothing sets)
__device__ __forceinline__ bool grid_barrier(unsigned *bar, int *err, unsigned long long wait_ns, bool withhold) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    const unsigned g = ld_acquire(bar + 1);
    __threadfence();
    const unsigned arrived = atomicAdd(bar, 1u);
    if (arrived == gridDim.x - 1 && !withhold) {
      atomicExch(bar, 0u);
      __threadfence();
      st_release(bar + 1, g + 1);
    } else if (arrived == gridDim.x - 1) {
      // the withheld release: this block goes on; its next barrier waits
    } else {
      const unsigned long long t0 = global_ns();
      for (unsigned it = 0;; ++it) {
        if (ld_acquire(bar + 1) != g) break;
        if (*(volatile int *)err != 0) {
          ok = 0;
          break;
        }
        if (it > (1u << 22) || global_ns() - t0 > wait_ns) {
          atomicCAS(err, 0, EMG_FUSED_TIMEOUT);
          ok = 0;
          break;
        }
        __nanosleep(32);
      }
    }
    if (*(volatile int *)err != 0) ok = 0;
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// SpMM step: one row per warp, the K columns over CL lanes (V contiguous
// columns each), the row's nonzeros split over NL lanes and reduced with
// shuffles.  Modes and arithmetic as spmm_kernel.
template <typename T, int K>
__device__ __forceinline__ void fused_spmm(const SpmmArgs &a) {
  typedef FusedLayout<T, K> L;
  constexpr int V = L::V, CL = L::CL, NL = L::NL;
  constexpr int U = 4;
  const int lane = threadIdx.x & 31;
  const int cb = lane % CL, sl = lane / CL;
  const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int nw = (int)((gridDim.x * blockDim.x) >> 5);
  const int n = a.n, mode = a.mode;
  const int *__restrict__ rp = a.rp;
  const int *__restrict__ ci = a.ci;
  const T *__restrict__ vc = static_cast<const T *>(a.vc);
  const T *__restrict__ vm = static_cast<const T *>(a.vm);
  const T *x = static_cast<const T *>(a.x);
  const bool two = vm != nullptr;
  T w[V];
#pragma unroll
  for (int i = 0; i < V; ++i) w[i] = two ? (T)__ldg(a.omega + cb * V + i) : T(0);
  for (int row = gw; row < n; row += nw) {  // warp-uniform
    T acc[V];
#pragma unroll
    for (int i = 0; i < V; ++i) acc[i] = T(0);
    const int kb = __ldg(rp + row), ke = __ldg(rp + row + 1);
    for (int k0 = kb + sl; k0 < ke; k0 += NL * U) {
      int j[U];
      T c[U], m[U];
      bool ok[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int k = k0 + u * NL;
        ok[u] = k < ke;
        j[u] = ok[u] ? __ldg(ci + k) : 0;
        c[u] = ok[u] ? __ldg(vc + k) : T(0);
        m[u] = (ok[u] && two) ? __ldg(vm + k) : T(0);
      }
      T xv[U][V];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (ok[u]) ldv_cg<T, V>(x + (long)j[u] * K + cb * V, xv[u]);
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
#pragma unroll
    for (int off = CL; off < 32; off <<= 1)
#pragma unroll
      for (int i = 0; i < V; ++i) acc[i] += __shfl_xor_sync(0xffffffffu, acc[i], off);
    if (sl != 0) continue;
    const long o = (long)row * K + cb * V;
    T *y = static_cast<T *>(a.y);
    T out[V];
    if (mode == SPMM_AX) {
#pragma unroll
      for (int i = 0; i < V; ++i) out[i] = acc[i];
    } else if (mode == SPMM_RES) {
      T bv[V];
      ldv_cg<T, V>(static_cast<const T *>(a.b) + o, bv);
#pragma unroll
      for (int i = 0; i < V; ++i) out[i] = bv[i] - acc[i];
    } else if (mode == SPMM_AXJ0) {
      const T dc = __ldg(static_cast<const T *>(a.l1c) + row);
      const T dm = a.l1m ? __ldg(static_cast<const T *>(a.l1m) + row) : T(0);
      T dd[V];
#pragma unroll
      for (int i = 0; i < V; ++i) {
        const T dg = a.l1m ? dc + (T)__ldg(a.omega + cb * V + i) * dm : dc;
        out[i] = acc[i];
        dd[i] = (T)a.c1 * acc[i] / dg;
      }
      stv<T, V>(static_cast<T *>(a.r) + o, dd);
      if (a.d) stv<T, V>(static_cast<T *>(a.d) + o, dd);
    } else if (mode == SPMM_ADD) {
      T yo[V];
      ldv_cg<T, V>(y + o, yo);
#pragma unroll
      for (int i = 0; i < V; ++i) out[i] = yo[i] + acc[i];
    } else {
      const T dc = __ldg(static_cast<const T *>(a.l1c) + row);
      const T dm = two ? __ldg(static_cast<const T *>(a.l1m) + row) : T(0);
      if (mode == SPMM_JAC) {
        T bv[V], xo[V];
        ldv_cg<T, V>(static_cast<const T *>(a.b) + o, bv);
        ldv_cg<T, V>(x + o, xo);
#pragma unroll
        for (int i = 0; i < V; ++i) {
          T d = two ? dc + w[i] * dm : dc;
          out[i] = xo[i] + (T)a.relax_w * (bv[i] - acc[i]) / d;
        }
      } else if (mode == SPMM_CHEB1) {
        T bv[V], xo[V], rr[V], dd[V];
        ldv_cg<T, V>(static_cast<const T *>(a.b) + o, bv);
        ldv_cg<T, V>(x + o, xo);
#pragma unroll
        for (int i = 0; i < V; ++i) {
          T dg = two ? dc + w[i] * dm : dc;
          rr[i] = bv[i] - acc[i];
          dd[i] = (T)a.c1 * rr[i] / dg;
          out[i] = xo[i] + dd[i];
        }
        stv<T, V>(static_cast<T *>(a.r) + o, rr);
        stv<T, V>(static_cast<T *>(a.d) + o, dd);
      } else if (mode == SPMM_CHEBK) {
        T rr[V], dd[V], xo[V], yo[V];
        ldv_cg<T, V>(static_cast<const T *>(a.b) + o, rr);
        ldv_cg<T, V>(x + o, xo);
        ldv_cg<T, V>(y + o, yo);
#pragma unroll
        for (int i = 0; i < V; ++i) {
          T dg = two ? dc + w[i] * dm : dc;
          rr[i] = rr[i] - acc[i];
          dd[i] = (T)a.c1 * xo[i] + (T)a.c2 * rr[i] / dg;
          out[i] = yo[i] + dd[i];
        }
        stv<T, V>(static_cast<T *>(a.r) + o, rr);
        stv<T, V>(static_cast<T *>(a.d) + o, dd);
      } else {  // SPMM_CHEB2
        T rr[V], dd[V], yo[V];
        ldv_cg<T, V>(static_cast<const T *>(a.r) + o, rr);
        ldv_cg<T, V>(x + o, dd);
        ldv_cg<T, V>(y + o, yo);
#pragma unroll
        for (int i = 0; i < V; ++i) {
          T dg = two ? dc + w[i] * dm : dc;
          out[i] = yo[i] + (T)a.c1 * dd[i] + (T)a.c2 * (rr[i] - acc[i]) / dg;
        }
      }
    }
    stv<T, V>(y + o, out);
  }
}

// first smoothing step from a zero guess: y (= d) = w b / (l1c + w_c l1m)
template <typename T, int K>
__device__ __forceinline__ void fused_jac0(const SpmmArgs &a, bool two_out) {
  const long total = (long)a.n * K;
  const long stride = (long)gridDim.x * blockDim.x;
  const T *b = static_cast<const T *>(a.b);
  const T *__restrict__ l1c = static_cast<const T *>(a.l1c);
  const T *__restrict__ l1m = static_cast<const T *>(a.l1m);
  T *y = static_cast<T *>(a.y);
  T *d = static_cast<T *>(a.d);
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += stride) {
    const long row = i / K;
    const int c = (int)(i % K);
    T dg = __ldg(l1c + row);
    if (l1m) dg += (T)__ldg(a.omega + c) * __ldg(l1m + row);
    const T v = (T)a.relax_w * __ldcg(b + i) / dg;
    y[i] = v;
    if (two_out) d[i] = v;
  }
}

// coarsest level: x[r, c] = sum_j inv[slot(c)][r][j] b[j, c] in FP64; a warp
// serves one row and CW columns, its 32/CW lane groups split j
template <typename T, int K>
__device__ __forceinline__ void fused_coarse(const SpmmArgs &a) {
  constexpr int CW = K < 8 ? K : 8;
  constexpr int JP = 32 / CW;
  constexpr int GROUPS = K / CW;
  const int nc = a.n;
  const double *__restrict__ inv = static_cast<const double *>(a.vc);
  const int *__restrict__ slot = a.ci;
  const T *b = static_cast<const T *>(a.b);
  T *x = static_cast<T *>(a.y);
  const int lane = threadIdx.x & 31;
  const int cs = lane % CW, jp = lane / CW;
  const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int nw = (int)((gridDim.x * blockDim.x) >> 5);
  for (int t = gw; t < nc * GROUPS; t += nw) {  // warp-uniform
    const int r = t / GROUPS, c = (t % GROUPS) * CW + cs;
    const double *row = inv + ((long)__ldg(slot + c) * nc + r) * nc;
    double acc = 0;
    for (int j = jp; j < nc; j += JP) acc += __ldg(row + j) * (double)__ldcg(b + (long)j * K + c);
#pragma unroll
    for (int off = CW; off < 32; off <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if (jp == 0) x[(long)r * K + c] = (T)acc;
  }
}

template <typename T, int K>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 4 : 3) vcycle_fused_kernel(const FusedOp *__restrict__ ops, int nops,
                                                              unsigned *bar, int *err, unsigned long long wait_ns,
                                                              int withhold_first) {
  __shared__ FusedOp sop;
  for (int i = 0; i < nops; ++i) {
    if (threadIdx.x == 0) sop = ops[i];
    __syncthreads();
    switch (sop.kind) {
    case FOP_SPMM: fused_spmm<T, K>(sop.a); break;
    case FOP_JAC0: fused_jac0<T, K>(sop.a, false); break;
    case FOP_JAC0_2: fused_jac0<T, K>(sop.a, true); break;
    default: fused_coarse<T, K>(sop.a); break;
    }
    if (i + 1 < nops && !grid_barrier(bar, err, wait_ns, withhold_first && i == 0)) return;
  }
}

template <typename T, int K>
void fused_launch_k(const FusedOp *ops, int nops, unsigned *bar, int *err, int max_bps, cudaStream_t s,
                    unsigned long long wait_ns, int withhold) {
  // co-resident grid: the occupancy limit of the kernel on every SM
  static std::map<std::pair<int, int>, int> blocks_for;  // (device, max_bps) -> blocks
  int dev = 0;
  EMG_CUDA(cudaGetDevice(&dev));
  auto key = std::make_pair(dev, max_bps);
  auto it = blocks_for.find(key);
  int blocks;
  if (it == blocks_for.end()) {
    int per_sm = 0, sms = 0;
    EMG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, vcycle_fused_kernel<T, K>, 256, 0));
    EMG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    if (max_bps > 0 && per_sm > max_bps) per_sm = max_bps;
    if (per_sm < 1) fail(EMG_ERR_CUDA, "fused V-cycle kernel cannot be resident on an SM");
    blocks = per_sm * sms;
    blocks_for[key] = blocks;
  } else {
    blocks = it->second;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)blocks);
  cfg.blockDim = dim3(256);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  EMG_CUDA(cudaLaunchKernelEx(&cfg, vcycle_fused_kernel<T, K>, ops, nops, bar, err, wait_ns, withhold));
  EMG_LAUNCH_CHECK();
}

}  // namespace

template <typename T>
void vcycle_fused(int K, const FusedOp *ops, int nops, unsigned *bar, int *err, int max_bps, cudaStream_t s,
                  unsigned long long wait_ns, int withhold) {
  if (nops <= 0) return;
  switch (K) {
  case 1: fused_launch_k<T, 1>(ops, nops, bar, err, max_bps, s, wait_ns, withhold); break;
  case 2: fused_launch_k<T, 2>(ops, nops, bar, err, max_bps, s, wait_ns, withhold); break;
  case 4: fused_launch_k<T, 4>(ops, nops, bar, err, max_bps, s, wait_ns, withhold); break;
  case 8: fused_launch_k<T, 8>(ops, nops, bar, err, max_bps, s, wait_ns, withhold); break;
  case 16: fused_launch_k<T, 16>(ops, nops, bar, err, max_bps, s, wait_ns, withhold); break;
  case 32: fused_launch_k<T, 32>(ops, nops, bar, err, max_bps, s, wait_ns, withhold); break;
  case 64: fused_launch_k<T, 64>(ops, nops, bar, err, max_bps, s, wait_ns, withhold); break;
  default: fail(EMG_ERR_ARG, "unsupported block width K=%d", K);
  }
}

template void vcycle_fused<float>(int, const FusedOp *, int, unsigned *, int *, int, cudaStream_t, unsigned long long,
                                  int);
template void vcycle_fused<double>(int, const FusedOp *, int, unsigned *, int *, int, cudaStream_t, unsigned long long,
                                   int);

}  // namespace emg
