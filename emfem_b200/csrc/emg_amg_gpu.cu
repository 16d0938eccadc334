// Nodal AMG hierarchy setup on the device: the BoomerAMG setup hypre's AMS
// runs inside PCSetUp (src/em_la.cc:156-157), restated from the published
// algorithms exactly as the host build in emg_amg.cpp does it -- classical
// strength (theta), PMIS coarsening with the same hashed measure, direct
// interpolation with separate negative/positive scaling truncated to Pmax
// with row-sum preservation, R = P^T, Galerkin R A P for both value parts --
// so that the two builds give the same hierarchy (the coarse-point choices
// are identical level by level as long as the level operators agree in
// their comparisons; the Galerkin sums differ only in rounding order).
//
// Every step is a kernel: row-parallel strength and interpolation, a
// three-kernel PMIS sweep repeated until no point is undecided, counting
// transposes, and a warp-per-coarse-row Galerkin product that accumulates
// the row in a shared-memory hash table, then writes it in column order.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <vector>

#include "emg_amg.h"
#include "emg_amg_gpu.h"

namespace emg {

namespace {

constexpr unsigned FULL = 0xffffffffu;

// ---------------------------------------------------------------------------
// exclusive scan of n+1 ints (a[n] receives the total)
// ---------------------------------------------------------------------------
__global__ void scan_block_kernel(int *__restrict__ a, long n, int *__restrict__ bsum) {
  __shared__ int ws[32];
  const long i = blockIdx.x * 1024L + threadIdx.x;
  const int v = i < n ? a[i] : 0;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(FULL, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) ws[w] = x;
  __syncthreads();
  if (w == 0) {
    int t = ws[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(FULL, t, o);
      if (lane >= o) t += y;
    }
    ws[lane] = t;
  }
  __syncthreads();
  const int incl = x + (w > 0 ? ws[w - 1] : 0);
  if (i < n) a[i] = incl - v;
  if (threadIdx.x == 1023) bsum[blockIdx.x] = incl;
}

__global__ void scan_add_kernel(int *__restrict__ a, long n, const int *__restrict__ boff) {
  const long i = blockIdx.x * 1024L + threadIdx.x;
  if (i < n) a[i] += boff[blockIdx.x];
}

void scan_rec(int *a, long n, cudaStream_t s) {
  const long nb = (n + 1023) / 1024;
  DBuf<int> bs((size_t)nb);
  scan_block_kernel<<<(unsigned)nb, 1024, 0, s>>>(a, n, bs.p);
  EMG_LAUNCH_CHECK();
  if (nb > 1) {
    scan_rec(bs.p, nb, s);
    scan_add_kernel<<<(unsigned)nb, 1024, 0, s>>>(a, n, bs.p);
    EMG_LAUNCH_CHECK();
  }
  EMG_CUDA(cudaStreamSynchronize(s));  // bs goes out of scope
}

// a: n + 1 entries, a[0..n) the counts; returns the total (a[n])
int scan_excl(int *a, long n, cudaStream_t s) {
  EMG_CUDA(cudaMemsetAsync(a + n, 0, sizeof(int), s));
  scan_rec(a, n + 1, s);
  int tot = 0;
  EMG_CUDA(cudaMemcpyAsync(&tot, a + n, sizeof(int), cudaMemcpyDeviceToHost, s));
  EMG_CUDA(cudaStreamSynchronize(s));
  if (tot < 0) fail(EMG_ERR_USER, "AMG setup: a prefix sum overflowed (%d)", tot);
  return tot;
}

__device__ __forceinline__ double combined(const double *vc, const double *vm, long k, double w) {
  return vm ? vc[k] + w * vm[k] : vc[k];
}
__device__ __forceinline__ bool same_fn(const int *fn, int i, int j) { return !fn || fn[i] == fn[j]; }

// ---------------------------------------------------------------------------
// strength of connection: j strongly influences i <=>
//   -a_ij >= theta * max_{k != i, same function} (-a_ik),  max > 0
// ---------------------------------------------------------------------------
__global__ void strength_kernel(int n, const int *__restrict__ rp, const int *__restrict__ ci,
                                const double *__restrict__ vc, const double *__restrict__ vm, double w, double theta,
                                const int *__restrict__ fn, const int *__restrict__ srp, int *__restrict__ cnt,
                                int *__restrict__ sci) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double m = 0;
  for (int k = rp[i]; k < rp[i + 1]; ++k)
    if (ci[k] != i && same_fn(fn, i, ci[k])) m = fmax(m, -combined(vc, vm, k, w));
  int c = 0, p = srp ? srp[i] : 0;
  if (m > 0)
    for (int k = rp[i]; k < rp[i + 1]; ++k)
      if (ci[k] != i && same_fn(fn, i, ci[k]) && -combined(vc, vm, k, w) >= theta * m) {
        if (sci) sci[p++] = ci[k];
        ++c;
      }
  if (cnt) cnt[i] = c;
}

// counting transpose of a pattern (order inside a row unspecified)
__global__ void count_cols_kernel(long nnz, const int *__restrict__ ci, int *__restrict__ cnt) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k < nnz) atomicAdd(cnt + ci[k], 1);
}

__global__ void scatter_transpose_kernel(int n, const int *__restrict__ rp, const int *__restrict__ ci,
                                         const double *__restrict__ v, int *__restrict__ pos, int *__restrict__ tci,
                                         double *__restrict__ tv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int k = rp[i]; k < rp[i + 1]; ++k) {
    const int p = atomicAdd(pos + ci[k], 1);
    tci[p] = i;
    if (v) tv[p] = v[k];
  }
}

// rows of a transpose in increasing column order (insertion sort per row,
// rows are short)
__global__ void sort_rows_kernel(int n, const int *__restrict__ rp, int *__restrict__ ci, double *__restrict__ v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int a = rp[i], b = rp[i + 1];
  for (int k = a + 1; k < b; ++k) {
    const int c = ci[k];
    const double x = v ? v[k] : 0.0;
    int q = k - 1;
    while (q >= a && ci[q] > c) {
      ci[q + 1] = ci[q];
      if (v) v[q + 1] = v[q];
      --q;
    }
    ci[q + 1] = c;
    if (v) v[q + 1] = x;
  }
}

// ---------------------------------------------------------------------------
// PMIS (De Sterck, Yang & Heys 2006), the host build's sweep order
// ---------------------------------------------------------------------------
__device__ __forceinline__ double hash_unit(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  x ^= x >> 31;
  return (double)(x >> 11) * (1.0 / 9007199254740992.0);
}

__global__ void pmis_init_kernel(int n, const int *__restrict__ trp, uint64_t seed, double *__restrict__ lam,
                                 int *__restrict__ cf) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int infl = trp[i + 1] - trp[i];
  lam[i] = infl + hash_unit(seed * 1000003ull + (uint64_t)i);
  cf[i] = infl == 0 ? -1 : 0;
}

__global__ void pmis_select_kernel(int n, const int *__restrict__ srp, const int *__restrict__ sci,
                                   const int *__restrict__ trp, const int *__restrict__ tci,
                                   const double *__restrict__ lam, const int *__restrict__ cf,
                                   unsigned char *__restrict__ newc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  bool best = cf[i] == 0;
  const double li = lam[i];
  for (int k = srp[i]; k < srp[i + 1] && best; ++k)
    if (cf[sci[k]] == 0 && lam[sci[k]] > li) best = false;
  for (int k = trp[i]; k < trp[i + 1] && best; ++k)
    if (cf[tci[k]] == 0 && lam[tci[k]] > li) best = false;
  newc[i] = best;
}

__global__ void pmis_setc_kernel(int n, const unsigned char *__restrict__ newc, int *__restrict__ cf) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && newc[i]) cf[i] = 1;
}

// points that strongly depend on a new C point become F; counts the
// undecided points left (before this kernel's F assignments are all seen,
// the host recounts below)
__global__ void pmis_setf_kernel(int n, const unsigned char *__restrict__ newc, const int *__restrict__ trp,
                                 const int *__restrict__ tci, int *cf) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !newc[i]) return;
  for (int k = trp[i]; k < trp[i + 1]; ++k) {
    const int j = tci[k];
    if (((volatile int *)cf)[j] == 0) cf[j] = -1;
  }
}

__global__ void count_undecided_kernel(int n, const int *__restrict__ cf, int *__restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int u = (i < n && cf[i] == 0) ? 1 : 0;
  const int s = __syncthreads_count(u);
  if (threadIdx.x == 0 && s) atomicAdd(out, s);
}

__global__ void undecided_to_c_kernel(int n, int *__restrict__ cf) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && cf[i] == 0) cf[i] = 1;
}

__global__ void cmark_kernel(int n, const int *__restrict__ cf, int *__restrict__ m) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) m[i] = cf[i] == 1;
}

// ---------------------------------------------------------------------------
// direct interpolation, truncated to pmax entries with row-sum preservation
// ---------------------------------------------------------------------------
struct InterpArgs {
  int n, pmax;
  const int *rp, *ci;
  const double *vc, *vm;
  double w;
  const int *fn, *srp, *sci, *cf, *cidx;
  const int *prp;  // fill pass: row pointer of P
  int *cnt;        // count pass
  int *pci;
  double *pv;
};

__device__ __forceinline__ bool in_strong(const InterpArgs &a, int i, int j) {
  for (int k = a.srp[i]; k < a.srp[i + 1]; ++k)
    if (a.sci[k] == j) return true;
  return false;
}

__global__ void interp_kernel(InterpArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  if (a.cf[i] == 1) {
    if (a.cnt) a.cnt[i] = 1;
    else {
      a.pci[a.prp[i]] = a.cidx[i];
      a.pv[a.prp[i]] = 1.0;
    }
    return;
  }
  double diag = 0, sn = 0, sp = 0, cn = 0, cp = 0;
  int ncand = 0;
  for (int k = a.rp[i]; k < a.rp[i + 1]; ++k) {
    const int j = a.ci[k];
    const double v = combined(a.vc, a.vm, k, a.w);
    if (j == i) {
      diag = v;
      continue;
    }
    if (!same_fn(a.fn, i, j)) continue;
    if (v < 0) sn += v;
    else sp += v;
    if (a.cf[j] == 1 && in_strong(a, i, j)) {
      if (v < 0) cn += v;
      else cp += v;
    }
  }
  const double alpha = cn != 0 ? sn / cn : 0.0;
  const double beta = cp != 0 ? sp / cp : 0.0;
  if (cp == 0) diag += sp;
  // candidate entries: strong C neighbours in row order
  auto weight = [&](int k) {
    const double v = combined(a.vc, a.vm, k, a.w);
    return -(v < 0 ? alpha : beta) * v / diag;
  };
  auto cand = [&](int k) {
    const int j = a.ci[k];
    return j != i && a.cf[j] == 1 && in_strong(a, i, j);
  };
  if (diag != 0)
    for (int k = a.rp[i]; k < a.rp[i + 1]; ++k)
      if (cand(k)) ++ncand;
  const int keep = ncand > a.pmax ? a.pmax : ncand;
  if (a.cnt) {
    a.cnt[i] = keep;
    return;
  }
  if (keep == 0) return;
  int sel[8];
  double selw[8];
  if (ncand <= a.pmax) {
    int q = 0;
    for (int k = a.rp[i]; k < a.rp[i + 1]; ++k)
      if (cand(k)) {
        sel[q] = a.cidx[a.ci[k]];
        selw[q] = weight(k);
        ++q;
      }
  } else {
    // the pmax largest |w| (ties: earlier in the row first), rescaled so that
    // the row sum is kept
    double tot = 0, kept = 0;
    for (int k = a.rp[i]; k < a.rp[i + 1]; ++k)
      if (cand(k)) tot += weight(k);
    int taken[8];
    for (int q = 0; q < keep; ++q) {
      int bk = -1;
      double bw = -1.0;
      for (int k = a.rp[i]; k < a.rp[i + 1]; ++k) {
        if (!cand(k)) continue;
        bool used = false;
        for (int u = 0; u < q; ++u) used |= taken[u] == k;
        if (used) continue;
        const double aw = fabs(weight(k));
        if (aw > bw) {
          bw = aw;
          bk = k;
        }
      }
      taken[q] = bk;
      sel[q] = a.cidx[a.ci[bk]];
      selw[q] = weight(bk);
      kept += selw[q];
    }
    if (kept != 0)
      for (int q = 0; q < keep; ++q) selw[q] *= tot / kept;
  }
  // column order
  for (int q = 1; q < keep; ++q) {
    const int c = sel[q];
    const double x = selw[q];
    int r = q - 1;
    while (r >= 0 && sel[r] > c) {
      sel[r + 1] = sel[r];
      selw[r + 1] = selw[r];
      --r;
    }
    sel[r + 1] = c;
    selw[r + 1] = x;
  }
  const int p0 = a.prp[i];
  for (int q = 0; q < keep; ++q) {
    a.pci[p0 + q] = sel[q];
    a.pv[p0 + q] = selw[q];
  }
}

__global__ void coarse_fn_kernel(int n, const int *__restrict__ cf, const int *__restrict__ cidx,
                                 const int *__restrict__ fn, int *__restrict__ fc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && cf[i] == 1) fc[cidx[i]] = fn[i];
}

// ---------------------------------------------------------------------------
// Galerkin C = R A P, one warp per coarse row, shared-memory hash table of
// CAP slots per warp.  count pass: distinct columns per row (rows with more
// than CAP * 3 / 4 are listed as overflow); fill pass: values summed, written
// in column order (each entry's rank among the row's columns).
// ---------------------------------------------------------------------------
struct RapArgs {
  int nc;
  const int *rrp, *rci;
  const double *rv;
  const int *arp, *aci;
  const double *avc, *avm;
  const int *prp, *pci;
  const double *pv;
  const int *rows;  // optional row list (overflow rows); nullptr: row = warp index
  int nrows;
  int *cnt;          // count pass
  int *ovf, *novf;   // count pass: overflow rows
  const int *crp;    // fill pass
  int *cci;
  double *cvc, *cvm;
};

template <int CAP>
__global__ void __launch_bounds__(CAP >= 4096 ? 32 : 192) rap_kernel(RapArgs a, int fill) {
  extern __shared__ __align__(16) unsigned char sm[];
  const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wpb = blockDim.x >> 5;
  double *vc = reinterpret_cast<double *>(sm) + (size_t)wib * CAP * 2;
  double *vm = vc + CAP;
  int *keys = reinterpret_cast<int *>(sm + (size_t)wpb * CAP * 2 * sizeof(double)) + (size_t)wib * CAP * 2;
  int *slot = keys + CAP;  // occupied slots, compacted
  const long wid = blockIdx.x * (long)wpb + wib;
  if (wid >= a.nrows) return;
  const int I = a.rows ? a.rows[wid] : (int)wid;
  for (int t = lane; t < CAP; t += 32) {
    keys[t] = -1;
    vc[t] = 0.0;
    vm[t] = 0.0;
  }
  __syncwarp();
  const bool two = a.avm != nullptr;
  int distinct = 0;
  bool overflow = false;
  // products r_Ii a_ik p_kJ: lanes split the (R entry, A entry) pairs
  for (int kr = a.rrp[I]; kr < a.rrp[I + 1]; ++kr) {
    const int i = a.rci[kr];
    const double r = a.rv[kr];
    for (int ka = a.arp[i] + lane; ka < a.arp[i + 1]; ka += 32) {
      const int k = a.aci[ka];
      const double rc = r * a.avc[ka], rm = two ? r * a.avm[ka] : 0.0;
      for (int kp = a.prp[k]; kp < a.prp[k + 1]; ++kp) {
        const int J = a.pci[kp];
        unsigned h = ((unsigned)J * 2654435761u) & (CAP - 1);
        for (int probe = 0; probe < CAP; ++probe) {
          const int cur = atomicCAS(keys + h, -1, J);
          if (cur == -1 || cur == J) {
            if (cur == -1) ++distinct;
            if (fill) {
              atomicAdd(vc + h, rc * a.pv[kp]);
              if (two) atomicAdd(vm + h, rm * a.pv[kp]);
            }
            break;
          }
          h = (h + 1) & (CAP - 1);
          if (probe == CAP - 1) overflow = true;
        }
      }
    }
  }
  __syncwarp();
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) distinct += __shfl_xor_sync(FULL, distinct, o);
  overflow = __any_sync(FULL, overflow) || distinct > CAP * 3 / 4;
  if (!fill) {
    if (lane == 0) {
      if (overflow && a.ovf) a.ovf[atomicAdd(a.novf, 1)] = I;
      a.cnt[I] = overflow ? 0 : distinct;
    }
    return;
  }
  // fill: compact the occupied slots, then each entry's rank among the row's
  // columns gives its position
  int L = 0;
  for (int b0 = 0; b0 < CAP; b0 += 32) {
    const bool occ = keys[b0 + lane] >= 0;
    const unsigned m = __ballot_sync(FULL, occ);
    if (occ) slot[L + __popc(m & ((1u << lane) - 1u))] = b0 + lane;
    L += __popc(m);
  }
  __syncwarp();
  const int base = a.crp[I];
  for (int q = lane; q < L; q += 32) {
    const int t = slot[q];
    const int J = keys[t];
    int rank = 0;
    for (int u = 0; u < L; ++u) rank += keys[slot[u]] < J;
    a.cci[base + rank] = J;
    a.cvc[base + rank] = vc[t];
    if (two) a.cvm[base + rank] = vm[t];
  }
}

template <int CAP, int WPB>
void rap_launch(const RapArgs &a, int fill, cudaStream_t s) {
  if (a.nrows <= 0) return;
  const size_t smem = (size_t)WPB * CAP * (2 * sizeof(int) + 2 * sizeof(double));
  EMG_CUDA(cudaFuncSetAttribute(rap_kernel<CAP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const unsigned grid = (unsigned)((a.nrows + WPB - 1) / WPB);
  rap_kernel<CAP><<<grid, WPB * 32, smem, s>>>(a, fill);
  EMG_LAUNCH_CHECK();
}

inline unsigned nblk(long n, int b = 256) { return (unsigned)((n + b - 1) / b); }

}  // namespace

void gcsr_transpose(const GCsr &A, GCsr &T, cudaStream_t s) {
  T.n = A.m;
  T.m = A.n;
  T.nnz = A.nnz;
  T.rp.alloc((size_t)T.n + 1);
  T.rp.zero(s);
  T.ci.alloc(std::max<size_t>(A.nnz, 1));
  const bool vals = A.vc.p != nullptr;
  if (vals) T.vc.alloc(std::max<size_t>(A.nnz, 1));
  T.vm.release();
  count_cols_kernel<<<nblk(A.nnz), 256, 0, s>>>(A.nnz, A.ci.p, T.rp.p);
  EMG_LAUNCH_CHECK();
  scan_excl(T.rp.p, T.n, s);
  DBuf<int> pos((size_t)T.n + 1);
  EMG_CUDA(cudaMemcpyAsync(pos.p, T.rp.p, sizeof(int) * ((size_t)T.n + 1), cudaMemcpyDeviceToDevice, s));
  scatter_transpose_kernel<<<nblk(A.n), 256, 0, s>>>(A.n, A.rp.p, A.ci.p, vals ? A.vc.p : nullptr, pos.p, T.ci.p,
                                                     vals ? T.vc.p : nullptr);
  EMG_LAUNCH_CHECK();
  sort_rows_kernel<<<nblk(T.n), 256, 0, s>>>(T.n, T.rp.p, T.ci.p, vals ? T.vc.p : nullptr);
  EMG_LAUNCH_CHECK();
  EMG_CUDA(cudaStreamSynchronize(s));
}

void gcsr_galerkin(const GCsr &R, const GCsr &A, const GCsr &P, GCsr &C, cudaStream_t s) {
  C.n = R.n;
  C.m = P.m;
  C.rp.alloc((size_t)C.n + 1);
  C.rp.zero(s);
  RapArgs a{};
  a.nc = C.n;
  a.rrp = R.rp.p;
  a.rci = R.ci.p;
  a.rv = R.vc.p;
  a.arp = A.rp.p;
  a.aci = A.ci.p;
  a.avc = A.vc.p;
  a.avm = A.vm.p;
  a.prp = P.rp.p;
  a.pci = P.ci.p;
  a.pv = P.vc.p;
  a.nrows = C.n;
  DBuf<int> ovf((size_t)C.n + 1), novf(1);
  novf.zero(s);
  a.cnt = C.rp.p;
  a.ovf = ovf.p;
  a.novf = novf.p;
  rap_launch<1024, 6>(a, 0, s);
  int nov = 0;
  novf.download(&nov, 1, s);
  EMG_CUDA(cudaStreamSynchronize(s));
  RapArgs big = a;
  if (nov > 0) {  // dense coarse rows: one warp per block with 8192 slots
    big.rows = ovf.p;
    big.nrows = nov;
    big.ovf = nullptr;
    rap_launch<8192, 1>(big, 0, s);
    std::vector<int> h(nov), cnt(nov);
    ovf.download(h.data(), nov, s);
    EMG_CUDA(cudaStreamSynchronize(s));
    for (int q = 0; q < nov; ++q) C.rp.download_at(&cnt[q], h[q], 1, s);
    EMG_CUDA(cudaStreamSynchronize(s));
    for (int q = 0; q < nov; ++q)
      if (cnt[q] == 0) fail(EMG_ERR_USER, "AMG setup: a coarse operator row has more than 6144 columns");
  }
  C.nnz = scan_excl(C.rp.p, C.n, s);
  C.ci.alloc(std::max<size_t>(C.nnz, 1));
  C.vc.alloc(std::max<size_t>(C.nnz, 1));
  if (A.vm.p) C.vm.alloc(std::max<size_t>(C.nnz, 1));
  else C.vm.release();
  a.cnt = nullptr;
  a.ovf = nullptr;
  a.crp = C.rp.p;
  a.cci = C.ci.p;
  a.cvc = C.vc.p;
  a.cvm = C.vm.p;
  if (nov > 0) {
    // the small table skips the overflow rows (their count pass gave 0 and
    // their fill pass cannot hold them): mark them and fill them with the big one
    DBuf<int> isovf((size_t)C.n);
    isovf.zero(s);
    std::vector<int> h(nov);
    ovf.download(h.data(), nov, s);
    EMG_CUDA(cudaStreamSynchronize(s));
    // fill every row with the small table except the listed ones
    std::vector<int> keep;
    keep.reserve((size_t)C.n - nov);
    std::vector<char> mark((size_t)C.n, 0);
    for (int q = 0; q < nov; ++q) mark[h[q]] = 1;
    for (int I = 0; I < C.n; ++I)
      if (!mark[I]) keep.push_back(I);
    DBuf<int> rows;
    rows.upload(keep, s);
    RapArgs small = a;
    small.rows = rows.p;
    small.nrows = (int)keep.size();
    rap_launch<1024, 6>(small, 1, s);
    big = a;
    big.rows = ovf.p;
    big.nrows = nov;
    rap_launch<8192, 1>(big, 1, s);
    EMG_CUDA(cudaStreamSynchronize(s));
  } else {
    rap_launch<1024, 6>(a, 1, s);
    EMG_CUDA(cudaStreamSynchronize(s));
  }
}

void amg_build_gpu(GCsr A, double w_ref, const AmgParams &prm, std::vector<GpuLevel> &lv, GCsr &coarse,
                   cudaStream_t s) {
  lv.clear();
  DBuf<int> fn;
  if (prm.num_functions > 1) {
    std::vector<int> h(A.n);
    for (int i = 0; i < A.n; ++i) h[i] = i % prm.num_functions;
    fn.upload(h, s);
  }
  for (int l = 0;; ++l) {
    if (A.n <= prm.max_coarse || l + 1 >= prm.max_levels) break;
    const int n = A.n;
    // strength
    DBuf<int> srp((size_t)n + 1);
    strength_kernel<<<nblk(n), 256, 0, s>>>(n, A.rp.p, A.ci.p, A.vc.p, A.vm.p, w_ref, prm.theta, fn.p, nullptr,
                                            srp.p, nullptr);
    EMG_LAUNCH_CHECK();
    const int ns = scan_excl(srp.p, n, s);
    DBuf<int> sci(std::max(ns, 1));
    strength_kernel<<<nblk(n), 256, 0, s>>>(n, A.rp.p, A.ci.p, A.vc.p, A.vm.p, w_ref, prm.theta, fn.p, srp.p,
                                            nullptr, sci.p);
    EMG_LAUNCH_CHECK();
    // S^T and PMIS
    GCsr S, ST;
    S.n = S.m = n;
    S.nnz = ns;
    S.rp = std::move(srp);
    S.ci = std::move(sci);
    gcsr_transpose(S, ST, s);
    DBuf<double> lam(n);
    DBuf<int> cf(n), und(1);
    DBuf<unsigned char> newc(n);
    pmis_init_kernel<<<nblk(n), 256, 0, s>>>(n, ST.rp.p, prm.seed + (uint64_t)l, lam.p, cf.p);
    EMG_LAUNCH_CHECK();
    int left = -1;
    for (int sweep = 0; sweep < 1000; ++sweep) {
      und.zero(s);
      count_undecided_kernel<<<nblk(n), 256, 0, s>>>(n, cf.p, und.p);
      EMG_LAUNCH_CHECK();
      int u = 0;
      und.download(&u, 1, s);
      EMG_CUDA(cudaStreamSynchronize(s));
      if (u == 0) break;
      if (u == left) {  // cannot happen with distinct measures; the host build's guard
        undecided_to_c_kernel<<<nblk(n), 256, 0, s>>>(n, cf.p);
        EMG_LAUNCH_CHECK();
        break;
      }
      left = u;
      pmis_select_kernel<<<nblk(n), 256, 0, s>>>(n, S.rp.p, S.ci.p, ST.rp.p, ST.ci.p, lam.p, cf.p, newc.p);
      pmis_setc_kernel<<<nblk(n), 256, 0, s>>>(n, newc.p, cf.p);
      pmis_setf_kernel<<<nblk(n), 256, 0, s>>>(n, newc.p, ST.rp.p, ST.ci.p, cf.p);
      EMG_LAUNCH_CHECK();
    }
    // coarse numbering and interpolation
    DBuf<int> cidx((size_t)n + 1);
    cmark_kernel<<<nblk(n), 256, 0, s>>>(n, cf.p, cidx.p);
    EMG_LAUNCH_CHECK();
    const int nc = scan_excl(cidx.p, n, s);
    if (nc == 0 || nc > 0.95 * n) break;
    GCsr P;
    P.n = n;
    P.m = nc;
    P.rp.alloc((size_t)n + 1);
    P.rp.zero(s);
    InterpArgs ia{};
    ia.n = n;
    ia.pmax = std::min(prm.pmax, 8);
    ia.rp = A.rp.p;
    ia.ci = A.ci.p;
    ia.vc = A.vc.p;
    ia.vm = A.vm.p;
    ia.w = w_ref;
    ia.fn = fn.p;
    ia.srp = S.rp.p;
    ia.sci = S.ci.p;
    ia.cf = cf.p;
    ia.cidx = cidx.p;
    ia.cnt = P.rp.p;
    interp_kernel<<<nblk(n, 128), 128, 0, s>>>(ia);
    EMG_LAUNCH_CHECK();
    P.nnz = scan_excl(P.rp.p, n, s);
    P.ci.alloc(std::max<size_t>(P.nnz, 1));
    P.vc.alloc(std::max<size_t>(P.nnz, 1));
    ia.cnt = nullptr;
    ia.prp = P.rp.p;
    ia.pci = P.ci.p;
    ia.pv = P.vc.p;
    interp_kernel<<<nblk(n, 128), 128, 0, s>>>(ia);
    EMG_LAUNCH_CHECK();
    DBuf<int> fc;
    if (fn.p) {
      fc.alloc(nc);
      coarse_fn_kernel<<<nblk(n), 256, 0, s>>>(n, cf.p, cidx.p, fn.p, fc.p);
      EMG_LAUNCH_CHECK();
    }
    GCsr R, RAP;
    gcsr_transpose(P, R, s);
    gcsr_galerkin(R, A, P, RAP, s);
    if (fn.p) fn = std::move(fc);
    GpuLevel L;
    L.A = std::move(A);
    L.P = std::move(P);
    L.R = std::move(R);
    lv.push_back(std::move(L));
    A = std::move(RAP);
  }
  coarse = std::move(A);
}

namespace {
// row 3 v + d of the vector operator = row v of component d, columns 3 u + d
__global__ void interleave_rp_kernel(int nv, const int *__restrict__ vrp, int *__restrict__ rp) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > 3 * nv) return;
  if (i == 3 * nv) {
    rp[i] = 3 * vrp[nv];
    return;
  }
  const int v = i / 3, d = i % 3;
  rp[i] = 3 * vrp[v] + d * (vrp[v + 1] - vrp[v]);
}

__global__ void interleave_fill_kernel(int nv, long vnnz, const int *__restrict__ vrp, const int *__restrict__ vci,
                                       const double *__restrict__ parts, const int *__restrict__ rp,
                                       int *__restrict__ ci, double *__restrict__ vc, double *__restrict__ vm) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 3 * nv) return;
  const int v = i / 3, d = i % 3;
  // component d = Pi_d: parts 2 (1 + d) and 2 (1 + d) + 1 of the nodal buffer
  const double *pc = parts + (size_t)(2 * (1 + d)) * vnnz, *pm = parts + (size_t)(2 * (1 + d) + 1) * vnnz;
  int p = rp[i];
  for (int k = vrp[v]; k < vrp[v + 1]; ++k, ++p) {
    ci[p] = 3 * vci[k] + d;
    vc[p] = pc[k];
    vm[p] = pm[k];
  }
}

__global__ void fold_kernel(long n, double *__restrict__ vc, const double *__restrict__ vm, double w) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < n) vc[i] += w * vm[i];
}
}  // namespace

void nodal_operator_gpu(Context &c, const DBuf<double> &parts, int sp, GCsr &out, double fold_w) {
  cudaStream_t s = c.stream;
  const long vnnz = c.h_vrp[c.nv];
  if (sp < 4) {
    out.n = out.m = c.nv;
    out.nnz = vnnz;
    out.rp.alloc((size_t)c.nv + 1);
    out.ci.alloc(vnnz);
    out.vc.alloc(vnnz);
    out.vm.alloc(vnnz);
    EMG_CUDA(cudaMemcpyAsync(out.rp.p, c.vrp.p, sizeof(int) * ((size_t)c.nv + 1), cudaMemcpyDeviceToDevice, s));
    EMG_CUDA(cudaMemcpyAsync(out.ci.p, c.vci.p, sizeof(int) * vnnz, cudaMemcpyDeviceToDevice, s));
    EMG_CUDA(cudaMemcpyAsync(out.vc.p, parts.p + (size_t)(2 * sp) * vnnz, sizeof(double) * vnnz,
                             cudaMemcpyDeviceToDevice, s));
    EMG_CUDA(cudaMemcpyAsync(out.vm.p, parts.p + (size_t)(2 * sp + 1) * vnnz, sizeof(double) * vnnz,
                             cudaMemcpyDeviceToDevice, s));
  } else {
    const int n = 3 * c.nv;
    out.n = out.m = n;
    out.nnz = 3 * vnnz;
    out.rp.alloc((size_t)n + 1);
    out.ci.alloc(out.nnz);
    out.vc.alloc(out.nnz);
    out.vm.alloc(out.nnz);
    interleave_rp_kernel<<<nblk(n + 1), 256, 0, s>>>(c.nv, c.vrp.p, out.rp.p);
    interleave_fill_kernel<<<nblk(n), 256, 0, s>>>(c.nv, vnnz, c.vrp.p, c.vci.p, parts.p, out.rp.p, out.ci.p,
                                                   out.vc.p, out.vm.p);
    EMG_LAUNCH_CHECK();
  }
  if (fold_w >= 0) {  // one frequency: A = Ac + w Am as a single part
    fold_kernel<<<nblk(out.nnz), 256, 0, s>>>(out.nnz, out.vc.p, out.vm.p, fold_w);
    EMG_LAUNCH_CHECK();
    EMG_CUDA(cudaStreamSynchronize(s));
    out.vm.release();
  }
  EMG_CUDA(cudaStreamSynchronize(s));
}

void gcsr_to_host(const GCsr &d, HCsr &h, cudaStream_t s) {
  h.n = d.n;
  h.m = d.m;
  h.rp.resize((size_t)d.n + 1);
  h.ci.resize(d.nnz);
  h.vc.resize(d.nnz);
  h.vm.resize(d.vm.p ? d.nnz : 0);
  d.rp.download(h.rp.data(), (size_t)d.n + 1, s);
  d.ci.download(h.ci.data(), d.nnz, s);
  d.vc.download(h.vc.data(), d.nnz, s);
  if (d.vm.p) d.vm.download(h.vm.data(), d.nnz, s);
  EMG_CUDA(cudaStreamSynchronize(s));
}

void gcsr_from_host(const HCsr &h, GCsr &d, cudaStream_t s) {
  d.n = h.n;
  d.m = h.m;
  d.nnz = h.nnz();
  d.rp.upload(h.rp, s);
  d.ci.upload(h.ci, s);
  d.vc.upload(h.vc, s);
  if (!h.vm.empty()) d.vm.upload(h.vm, s);
  else d.vm.release();
  EMG_CUDA(cudaStreamSynchronize(s));
}

}  // namespace emg
