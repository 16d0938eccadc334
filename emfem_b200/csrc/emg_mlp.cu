// Learned warm start: a per-edge MLP (16 -> 64 -> 64 -> 64 -> 16, GELU; 13 of
// the inputs and 2 of the outputs are used) that predicts the solution of a
// (frequency, source) column from the solutions of the two nearest solved
// frequencies of the same source.  No counterpart in the reference, which
// always starts FGMRES from zero (src/em_la.cc:49); the Krylov residual judges
// the guess and zero stays the fallback.
//
// Inputs of sample (edge e, target column): the two neighbour values of edge e
// divided by s_e = max(|e_a|, |e_b|) (4), log10 of the horizontal and vertical
// resistivity around the edge (2), log10 edge length (1), direction cosines
// (3), log10 distance to the source (1), log10 f (1) and tau, the position of
// f between the two neighbour frequencies in log f (1).  Output: the
// curvature in log f; q times it (q = (log10 f - log10 f_a)(log10 f -
// log10 f_b)) is the correction added to the log-f interpolation
// e_a + tau (e_b - e_a) (in units of s_e); zero-initialised last layer, so the
// untrained network is that interpolation.
//
// One persistent CTA per SM runs 128-sample tiles through the whole network on
// the 5th-generation tensor cores: BF16 operands in shared memory (no-swizzle
// K-major core-matrix layout, 8 rows x 16 bytes per 128-byte core matrix),
// FP32 accumulators in tensor memory, one thread issues tcgen05.mma and
// tcgen05.commit signals an mbarrier; the 128 threads (one per sample = one
// TMEM lane) read the accumulators back with tcgen05.ld for the bias, GELU and
// loss epilogues.  Training adds the backward pass in the same tile loop:
//   dH_l = dZ_{l+1} W_{l+1}                       (M=128, N=64)
//   [dW1; db; dW4] += [X^T; 1; H3^T] [dZ1 dZ4 dZ2 dZ3]    (M=128, N=208, K=samples)
//   [dW2; dW3]     += [H1^T; H2^T]   [dZ2 dZ3]            (M=128, N=128, K=samples)
// The weight-gradient products accumulate in tensor memory over the CTA's
// tiles (stacking the layers' operands keeps every product at M=128); the
// row of ones gives every bias gradient from the same product.

#include <cuda_runtime.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "emg_api.h"
#include "emg_internal.h"
#include "emg_mlp.h"

namespace emg {
namespace wsnet {

// ---------------------------------------------------------------------------
// shared-memory image (bytes); every operand in the canonical layout
// ---------------------------------------------------------------------------
constexpr int T = 128;  // samples per tile = threads = TMEM lanes
constexpr int OFF_W1 = 0;                      // [64 x 16]  W1 (out x in)
constexpr int OFF_W2 = OFF_W1 + 64 * 16 * 2;   // [64 x 64]
constexpr int OFF_W3 = OFF_W2 + 64 * 64 * 2;   // [64 x 64]
constexpr int OFF_W4 = OFF_W3 + 64 * 64 * 2;   // [16 x 64]
constexpr int OFF_W2T = OFF_W4 + 16 * 64 * 2;  // [64 x 64]  W2^T (in x out)
constexpr int OFF_W3T = OFF_W2T + 64 * 64 * 2; // [64 x 64]
constexpr int OFF_W4T = OFF_W3T + 64 * 64 * 2; // [64 x 16]
constexpr int IMG_BYTES = OFF_W4T + 64 * 16 * 2;  // 38912: the packed weight image in global memory
constexpr int OFF_IN = IMG_BYTES;              // [128 x 16]  X, later dZ4
constexpr int OFF_ACT = OFF_IN + T * 16 * 2;   // [128 x 64]  H1/H2/H3, later dZ3/dZ2
constexpr int OFF_AA = OFF_ACT + T * 64 * 2;   // [128 x 128] rows: X^T 0-15, ones 16, H3^T 64-127
constexpr int OFF_AB = OFF_AA + 128 * T * 2;   // [128 x 128] rows: H1^T 0-63, H2^T 64-127
constexpr int OFF_BA = OFF_AB + 128 * T * 2;   // [208 x 128] rows: dZ1^T 0-63, dZ4^T 64-79, dZ2^T 80-143, dZ3^T 144-207
constexpr int OFF_G = OFF_BA + 208 * T * 2;    // 3 x [64][128] bf16 GELU'(Z_l), [feature][sample]
constexpr int OFF_BIAS = OFF_G + 3 * 64 * T * 2;  // 4 x 64 floats
constexpr int OFF_MBAR = OFF_BIAS + 4 * 64 * 4;   // 8 bytes
constexpr int OFF_TMEM = OFF_MBAR + 8;            // 4 bytes
constexpr int SMEM_TRAIN = OFF_TMEM + 8;
static_assert(SMEM_TRAIN <= 232448, "shared memory of the training kernel exceeds 227 KB");

// tensor-memory columns (512 allocated: one CTA per SM)
constexpr uint32_t TM_DA = 0;     // 208 columns: [dW1 | db | dW4] product
constexpr uint32_t TM_DB = 256;   // 128 columns: [dW2 | dW3] product
constexpr uint32_t TM_S = 384;    // 64 columns: Z1, Z2, Z3, dH3, dH2, dH1 in turn
constexpr uint32_t TM_Z4 = 448;   // 16 columns
constexpr uint32_t TM_COLS = 512;

// byte offset of element (r, k) in an R x K operand (K a multiple of 8):
// core matrix (r/8, k/8) at ((r/8) (K/8) + k/8) x 128, row r%8 at 16 (r%8)
__host__ __device__ constexpr int cm_off(int r, int k, int K) {
  return (((r >> 3) * (K >> 3) + (k >> 3)) << 7) + ((r & 7) << 4) + ((k & 7) << 1);
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// tcgen05 shared-memory matrix descriptor: start, leading-dimension byte
// offset (between core matrices adjacent in K), stride-dimension byte offset
// (between 8-row groups), descriptor version 1, no swizzle
__device__ __forceinline__ uint64_t mdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}

// instruction descriptor, kind::f16: FP32 accumulator, BF16 A and B, both K-major
__device__ __forceinline__ uint32_t idesc(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma(uint32_t d, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(id), "r"(acc));
}

__device__ __forceinline__ void commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// bounded wait for the mbarrier phase (1 s of %globaltimer or 2^22 polls);
// false when it gave up
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  const unsigned long long t0 = global_ns();
  for (int i = 0; i < (1 << 22); ++i) {
    if ((i & 255) == 255 && global_ns() - t0 > 1000000000ull) return false;
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

// 16 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_d(float z) {
  return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

__device__ __forceinline__ unsigned short bf16_bits(float x) {
  __nv_bfloat16 h = __float2bfloat16_rn(x);
  return *reinterpret_cast<unsigned short *>(&h);
}

// 8 consecutive values of row r (k0 .. k0+7, k0 a multiple of 8) as one
// 16-byte store into a K-column operand
__device__ __forceinline__ void st_row8(unsigned char *base, int r, int k0, int K, const float *v) {
  uint4 q;
  q.x = (uint32_t)bf16_bits(v[0]) | ((uint32_t)bf16_bits(v[1]) << 16);
  q.y = (uint32_t)bf16_bits(v[2]) | ((uint32_t)bf16_bits(v[3]) << 16);
  q.z = (uint32_t)bf16_bits(v[4]) | ((uint32_t)bf16_bits(v[5]) << 16);
  q.w = (uint32_t)bf16_bits(v[6]) | ((uint32_t)bf16_bits(v[7]) << 16);
  *reinterpret_cast<uint4 *>(base + cm_off(r, k0, K)) = q;
}

__device__ __forceinline__ void st_elem(unsigned char *base, int r, int k, int K, float v) {
  *reinterpret_cast<unsigned short *>(base + cm_off(r, k, K)) = bf16_bits(v);
}

__device__ __forceinline__ uint32_t mix32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

constexpr float kTargetClamp = 4.0f;
constexpr float kMinQ = 1e-4f;  // |q| below this: the target column is a neighbour, nothing to learn

struct KArgs {
  const unsigned char *img;  // packed BF16 weight image (IMG_BYTES)
  const float *bias;         // 4 x 64 (b1, b2, b3, b4 padded)
  const float4 *stat;        // 3 per edge: (lrh, lrv, llen, cx), (cy, cz, 0, 0), (mx, my, mz, 0)
  const Spec *spec;
  int nspec, ne;
  const double2 *xs;  // source block, ne x ks complex
  int ks;
  double2 *out;  // predict: guess block ne x kt
  int kt;
  long nsamples;
  int mode;           // 0 interpolation only, 1 network, 2 training
  uint32_t seed;
  float inv_batch;
  float *grad;        // training: 208 x 128 + 128 x 128 floats, the two products summed over CTAs
  double *loss;       // training: summed 0.5 |out - target|^2 / batch
  double *loss0;      // training: summed 0.5 |target|^2 / batch (a zero correction: the interpolation)
  int *err;
};

// features, base and scale of one sample (zeros for an invalid one)
__device__ __forceinline__ void sample_features(const KArgs &a, long s, bool valid, float (&f)[16], float &b0,
                                                float &b1, float &q, double &scale, float &t0, float &t1, int &e,
                                                int &tcol) {
#pragma unroll
  for (int i = 0; i < 16; ++i) f[i] = 0.f;
  b0 = b1 = t0 = t1 = q = 0.f;
  scale = 0.0;
  e = 0;
  tcol = 0;
  if (!valid) return;
  int sp;
  if (a.mode == 2) {
    sp = (int)(s % a.nspec);
    e = (int)(mix32((uint32_t)s * 0x9E3779B9u + a.seed) % (uint32_t)a.ne);
  } else {
    sp = (int)(s / a.ne);
    e = (int)(s % a.ne);
  }
  const Spec p = a.spec[sp];
  tcol = p.tcol;
  const double2 ea = a.xs[(long)e * a.ks + p.a];
  const double2 eb = a.xs[(long)e * a.ks + p.b];
  const double sc = fmax(sqrt(ea.x * ea.x + ea.y * ea.y), sqrt(eb.x * eb.x + eb.y * eb.y));
  if (!(sc > 1e-300)) return;  // zero field (homogeneous Dirichlet edge): the guess is zero there
  scale = sc;
  const double inv = 1.0 / sc;
  f[0] = (float)(ea.x * inv);
  f[1] = (float)(ea.y * inv);
  f[2] = (float)(eb.x * inv);
  f[3] = (float)(eb.y * inv);
  const float4 s0 = a.stat[3 * (long)e], s1 = a.stat[3 * (long)e + 1], s2 = a.stat[3 * (long)e + 2];
  f[4] = s0.x;
  f[5] = s0.y;
  f[6] = s0.z;
  f[7] = s0.w;
  f[8] = s1.x;
  f[9] = s1.y;
  float dist;
  if (p.src_kind == 0) {
    dist = s2.z;  // plane-wave source: depth below the top of the earth
  } else {
    const float dx = s2.x - p.src[0], dy = s2.y - p.src[1], dz = s2.z - p.src[2];
    dist = sqrtf(dx * dx + dy * dy + dz * dz);
  }
  f[10] = copysignf(log10f(1.0f + fabsf(dist) * 0.01f), dist) * 0.5f;
  f[11] = p.logf;
  f[12] = p.tau;
  b0 = (1.f - p.tau) * f[0] + p.tau * f[2];
  b1 = (1.f - p.tau) * f[1] + p.tau * f[3];
  q = p.q;
  if (a.mode == 2 && fabsf(q) >= kMinQ) {
    // the target is the curvature (correction / q); values beyond a few
    // neighbour magnitudes are outliers (edges where both neighbours nearly
    // vanish): clamped, so that a few of them do not dominate the squared loss
    const double2 et = a.xs[(long)e * a.ks + p.tcol];
    const float iq = 1.f / q;
    t0 = fminf(fmaxf(((float)(et.x * inv) - b0) * iq, -kTargetClamp), kTargetClamp);
    t1 = fminf(fmaxf(((float)(et.y * inv) - b1) * iq, -kTargetClamp), kTargetClamp);
  }
}

template <int MODE>
__global__ void __launch_bounds__(128, 1) mlp_kernel(KArgs a) {
  extern __shared__ __align__(128) unsigned char sm[];
  const int tid = threadIdx.x, warp = tid >> 5;
  const uint32_t sbase = smem_u32(sm);
  float *sbias = reinterpret_cast<float *>(sm + OFF_BIAS);
  const uint32_t mbar = sbase + OFF_MBAR;
  uint32_t *tm_holder = reinterpret_cast<uint32_t *>(sm + OFF_TMEM);
  constexpr bool NET = MODE >= 1, TRAIN = MODE == 2;
  const long ntiles = (a.nsamples + T - 1) / T;

  // weights and biases into shared memory; training operands cleared
  if (NET) {
    const uint4 *src = reinterpret_cast<const uint4 *>(a.img);
    for (int i = tid; i < IMG_BYTES / 16; i += T) reinterpret_cast<uint4 *>(sm)[i] = src[i];
    for (int i = tid; i < 4 * 64; i += T) sbias[i] = a.bias[i];
  }
  if (TRAIN) {
    for (int i = tid; i < (OFF_G - OFF_AA) / 16; i += T) reinterpret_cast<uint4 *>(sm + OFF_AA)[i] = make_uint4(0, 0, 0, 0);
    __syncthreads();
    // the row of ones (row 16 of A_a) gives the bias gradients
    for (int s = tid; s < T; s += T) st_elem(sm + OFF_AA, 16, s, T, 1.0f);
  }
  uint32_t tbase = 0;
  if (NET) {
    if (tid == 0) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
      asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tm_holder)),
                   "r"(TM_COLS)
                   : "memory");
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_before();
    __syncthreads();
    fence_after();
    tbase = *tm_holder;
  }
  __syncthreads();
  const uint32_t lane_addr = tbase + ((uint32_t)(warp * 32) << 16);
  uint32_t phase = 0;
  bool ok = true;
  bool first = true;
  float loss_acc = 0.f, loss0_acc = 0.f;

  // one MMA group: operands written by every thread are made visible to the
  // tensor core, thread 0 issues, everyone waits for the commit
  auto group = [&](auto issue) {
    fence_async_smem();
    fence_before();
    __syncthreads();
    if (tid == 0) {
      fence_after();
      issue();
      commit(mbar);
    }
    const bool done = mbar_wait(mbar, phase);
    ok = __syncthreads_and(ok && done) != 0;
    if (ok) phase ^= 1u;  // after a failed wait the pending phase stays the one to wait for
    fence_after();
  };
  auto gemm = [&](uint32_t d, uint32_t a_off, int a_K, uint32_t b_off, int b_K, int K, int N, uint32_t acc0) {
    // A: 128 x a_K operand, B: N x b_K operand; K columns from both starting at 0
    const uint32_t id = idesc(128, N);
    for (int kk = 0; kk < K / 16; ++kk) {
      const uint64_t da = mdesc(sbase + a_off + kk * 256, 128, a_K * 16);
      const uint64_t db = mdesc(sbase + b_off + kk * 256, 128, b_K * 16);
      mma(d, da, db, id, (kk > 0 || acc0) ? 1u : 0u);
    }
  };

  for (long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const long s = tile * T + tid;
    const bool valid = s < a.nsamples;
    float f[16], b0, b1, q, t0, t1;
    double scale;
    int e, tcol;
    sample_features(a, s, valid, f, b0, b1, q, scale, t0, t1, e, tcol);
    float o0 = 0.f, o1 = 0.f;
    if (NET) {
      st_row8(sm + OFF_IN, tid, 0, 16, f);
      st_row8(sm + OFF_IN, tid, 8, 16, f + 8);
      if (TRAIN)
#pragma unroll
        for (int i = 0; i < 16; ++i) st_elem(sm + OFF_AA, i, tid, T, f[i]);
      // forward: three hidden layers
      for (int l = 0; l < 3 && ok; ++l) {
        if (l == 0) group([&] { gemm(tbase + TM_S, OFF_IN, 16, OFF_W1, 16, 16, 64, 0); });
        else group([&] { gemm(tbase + TM_S, OFF_ACT, 64, l == 1 ? OFF_W2 : OFF_W3, 64, 64, 64, 0); });
        if (!ok) break;
#pragma unroll 1
        for (int c = 0; c < 4; ++c) {
          float z[16], h[16];
          tmem_ld16(lane_addr + TM_S + 16 * c, z);
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            const float zz = z[i] + sbias[64 * l + 16 * c + i];
            h[i] = gelu(zz);
            if (TRAIN)
              *reinterpret_cast<unsigned short *>(sm + OFF_G + ((l * 64 + 16 * c + i) * T + tid) * 2) =
                  bf16_bits(gelu_d(zz));
          }
          st_row8(sm + OFF_ACT, tid, 16 * c, 64, h);
          st_row8(sm + OFF_ACT, tid, 16 * c + 8, 64, h + 8);
          if (TRAIN) {
            // H1^T, H2^T -> A_b rows 0-63 / 64-127; H3^T -> A_a rows 64-127
            unsigned char *dst = l < 2 ? sm + OFF_AB : sm + OFF_AA;
            const int r0 = l == 0 ? 0 : 64;
#pragma unroll
            for (int i = 0; i < 16; ++i) st_elem(dst, r0 + 16 * c + i, tid, T, h[i]);
          }
        }
      }
      if (!ok) break;
      // output layer
      group([&] { gemm(tbase + TM_Z4, OFF_ACT, 64, OFF_W4, 64, 64, 16, 0); });
      if (!ok) break;
      float z4[16];
      tmem_ld16(lane_addr + TM_Z4, z4);
      o0 = z4[0] + sbias[192];
      o1 = z4[1] + sbias[193];
    }
    if (!TRAIN) {
      if (valid) {
        const double p0 = (double)(b0 + q * o0) * scale, p1 = (double)(b1 + q * o1) * scale;
        a.out[(long)e * a.kt + tcol] = make_double2(p0, p1);
      }
      continue;
    }
    // ---- training: loss and backward ----
    const float d0 = valid ? (o0 - t0) : 0.f, d1 = valid ? (o1 - t1) : 0.f;
    loss_acc += 0.5f * (d0 * d0 + d1 * d1) * a.inv_batch;
    loss0_acc += 0.5f * (t0 * t0 + t1 * t1) * a.inv_batch;
    {
      float g[16];
#pragma unroll
      for (int i = 0; i < 16; ++i) g[i] = 0.f;
      g[0] = d0 * a.inv_batch;
      g[1] = d1 * a.inv_batch;
      st_row8(sm + OFF_IN, tid, 0, 16, g);
      st_row8(sm + OFF_IN, tid, 8, 16, g + 8);
      st_elem(sm + OFF_BA, 64, tid, T, g[0]);
      st_elem(sm + OFF_BA, 65, tid, T, g[1]);
    }
    // dH3 = dZ4 W4, dZ3; dH2 = dZ3 W3, dZ2; dH1 = dZ2 W2, dZ1
    for (int l = 2; l >= 0 && ok; --l) {
      if (l == 2) group([&] { gemm(tbase + TM_S, OFF_IN, 16, OFF_W4T, 16, 16, 64, 0); });
      else group([&] { gemm(tbase + TM_S, OFF_ACT, 64, l == 1 ? OFF_W3T : OFF_W2T, 64, 64, 64, 0); });
      if (!ok) break;
      // B_a rows of dZ_l^T: dZ1 0-63, dZ2 80-143, dZ3 144-207
      const int r0 = l == 0 ? 0 : (l == 1 ? 80 : 144);
#pragma unroll 1
      for (int c = 0; c < 4; ++c) {
        float dh[16], dz[16];
        tmem_ld16(lane_addr + TM_S + 16 * c, dh);
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const unsigned short gb =
              *reinterpret_cast<const unsigned short *>(sm + OFF_G + ((l * 64 + 16 * c + i) * T + tid) * 2);
          const float gd = __uint_as_float((uint32_t)gb << 16);
          dz[i] = dh[i] * gd;
          st_elem(sm + OFF_BA, r0 + 16 * c + i, tid, T, dz[i]);
        }
        if (l > 0) {
          st_row8(sm + OFF_ACT, tid, 16 * c, 64, dz);
          st_row8(sm + OFF_ACT, tid, 16 * c + 8, 64, dz + 8);
        }
      }
    }
    if (!ok) break;
    // weight and bias gradient products, accumulated over this CTA's tiles
    const uint32_t acc = first ? 0u : 1u;
    group([&] {
      gemm(tbase + TM_DA, OFF_AA, T, OFF_BA, T, T, 208, acc);
      gemm(tbase + TM_DB, OFF_AB, T, OFF_BA + 10 * (T * 16), T, T, 128, acc);
    });
    first = false;
  }
  // ---- epilogue: gradients and loss out, tensor memory released ----
  if (TRAIN && ok && !first) {
    // lane (row) tid of the two products
    float *ga = a.grad;            // 128 x 208
    float *gb = a.grad + 128 * 208;  // 128 x 128
#pragma unroll 1
    for (int c = 0; c < 13; ++c) {
      float v[16];
      tmem_ld16(lane_addr + TM_DA + 16 * c, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) atomicAdd(ga + tid * 208 + 16 * c + i, v[i]);
    }
#pragma unroll 1
    for (int c = 0; c < 8; ++c) {
      float v[16];
      tmem_ld16(lane_addr + TM_DB + 16 * c, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) atomicAdd(gb + tid * 128 + 16 * c + i, v[i]);
    }
  }
  if (TRAIN) {
    float l = loss_acc, l0 = loss0_acc;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      l += __shfl_xor_sync(0xffffffffu, l, off);
      l0 += __shfl_xor_sync(0xffffffffu, l0, off);
    }
    if ((tid & 31) == 0) {
      atomicAdd(a.loss, (double)l);
      atomicAdd(a.loss0, (double)l0);
    }
  }
  if (!ok && tid == 0) atomicExch(a.err, 1);
  // a wait that gave up: wait once more (bounded) for the tensor-core work
  // in flight before the tensor memory is released
  if (NET && !ok) (void)mbar_wait(mbar, phase);
  if (NET) {
    fence_before();
    __syncthreads();
    if (warp == 0) {
      fence_after();
      asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(TM_COLS) : "memory");
    }
  }
}

// ---------------------------------------------------------------------------
// per-edge static features
// ---------------------------------------------------------------------------
__global__ void edge_rho_kernel(int nt, const int *__restrict__ t2e, const int *__restrict__ attr,
                                const float2 *__restrict__ lrho, float *__restrict__ acc) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  const float2 r = lrho[attr[t]];
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    const int e = t2e[6 * (long)t + i];
    atomicAdd(acc + 3 * (long)e, r.x);
    atomicAdd(acc + 3 * (long)e + 1, r.y);
    atomicAdd(acc + 3 * (long)e + 2, 1.0f);
  }
}

__global__ void edge_static_kernel(int ne, const int *__restrict__ edges, const double *__restrict__ pts,
                                   const float *__restrict__ acc, float4 *__restrict__ stat) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  const int a = edges[2 * e], b = edges[2 * e + 1];
  double d[3], m[3];
  for (int i = 0; i < 3; ++i) {
    d[i] = pts[3 * (long)b + i] - pts[3 * (long)a + i];
    m[i] = 0.5 * (pts[3 * (long)b + i] + pts[3 * (long)a + i]);
  }
  const double len = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  const float n = fmaxf(acc[3 * (long)e + 2], 1.0f);
  stat[3 * (long)e] = make_float4((acc[3 * (long)e] / n - 2.0f) / 3.0f, (acc[3 * (long)e + 1] / n - 2.0f) / 3.0f,
                                  (float)log10(fmax(len, 1e-3)) - 2.5f, (float)(d[0] / len));
  stat[3 * (long)e + 1] = make_float4((float)(d[1] / len), (float)(d[2] / len), 0.f, 0.f);
  stat[3 * (long)e + 2] = make_float4((float)m[0], (float)m[1], (float)m[2], 0.f);
}

// ---------------------------------------------------------------------------
// Adam on the FP32 master parameters; writes the BF16 weight image (W and
// W^T in the operand layout) and the bias vector
// ---------------------------------------------------------------------------
struct AdamArgs {
  float *w;        // master parameters: W1 64x16, W2 64x64, W3 64x64, W4 2x64 (rows 0-1 of 16), b1..b3 64, b4 2
  float *m, *v;
  const float *grad;  // the two products
  int step;
  float lr, b1, b2, eps;
  unsigned char *img;
  float *bias;        // 4 x 64
};

constexpr int NP_W1 = 64 * 16, NP_W2 = 64 * 64, NP_W3 = 64 * 64, NP_W4 = 2 * 64;
constexpr int P_W1 = 0, P_W2 = P_W1 + NP_W1, P_W3 = P_W2 + NP_W2, P_W4 = P_W3 + NP_W3;
constexpr int P_B1 = P_W4 + NP_W4, P_B2 = P_B1 + 64, P_B3 = P_B2 + 64, P_B4 = P_B3 + 64;
constexpr int NPARAM = P_B4 + 2;

// gradient of parameter p from the two accumulated products:
//   Da[i][o]            (i < 16, o < 64)  = dW1[o][i]
//   Da[16][o]           (o < 64)          = db1[o];  Da[16][64+o] (o<2) = db4[o]
//   Da[16][80+o]/[144+o]                  = db2[o] / db3[o]
//   Da[64+i][64+o]      (i < 64, o < 16)  = dW4[o][i]
//   Db[i][o], Db[64+i][64+o]              = dW2[o][i], dW3[o][i]
__device__ __forceinline__ float param_grad(const float *g, int p) {
  const float *ga = g, *gb = g + 128 * 208;
  if (p < P_W2) { const int o = p / 16, i = p % 16; return ga[i * 208 + o]; }
  if (p < P_W3) { const int q = p - P_W2, o = q / 64, i = q % 64; return gb[i * 128 + o]; }
  if (p < P_W4) { const int q = p - P_W3, o = q / 64, i = q % 64; return gb[(64 + i) * 128 + 64 + o]; }
  if (p < P_B1) { const int q = p - P_W4, o = q / 64, i = q % 64; return ga[(64 + i) * 208 + 64 + o]; }
  if (p < P_B2) return ga[16 * 208 + (p - P_B1)];
  if (p < P_B3) return ga[16 * 208 + 80 + (p - P_B2)];
  if (p < P_B4) return ga[16 * 208 + 144 + (p - P_B3)];
  return ga[16 * 208 + 64 + (p - P_B4)];
}

__global__ void adam_kernel(AdamArgs a) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= NPARAM) return;
  const float g = param_grad(a.grad, p);
  const float m = a.b1 * a.m[p] + (1.f - a.b1) * g;
  const float v = a.b2 * a.v[p] + (1.f - a.b2) * g * g;
  a.m[p] = m;
  a.v[p] = v;
  const float mh = m / (1.f - powf(a.b1, (float)a.step)), vh = v / (1.f - powf(a.b2, (float)a.step));
  const float w = a.w[p] - a.lr * mh / (sqrtf(vh) + a.eps);
  a.w[p] = w;
}

// BF16 image and bias vector from the master parameters
__global__ void pack_kernel(const float *__restrict__ w, unsigned char *__restrict__ img, float *__restrict__ bias) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= NPARAM) return;
  const unsigned short h = bf16_bits(w[p]);
  auto put = [&](int off, int r, int k, int K) { *reinterpret_cast<unsigned short *>(img + off + cm_off(r, k, K)) = h; };
  if (p < P_W2) {
    put(OFF_W1, p / 16, p % 16, 16);
  } else if (p < P_W3) {
    const int q = p - P_W2;
    put(OFF_W2, q / 64, q % 64, 64);
    put(OFF_W2T, q % 64, q / 64, 64);
  } else if (p < P_W4) {
    const int q = p - P_W3;
    put(OFF_W3, q / 64, q % 64, 64);
    put(OFF_W3T, q % 64, q / 64, 64);
  } else if (p < P_B1) {
    const int q = p - P_W4;
    put(OFF_W4, q / 64, q % 64, 64);
    put(OFF_W4T, q % 64, q / 64, 16);
  } else if (p < P_B2) {
    bias[p - P_B1] = w[p];
  } else if (p < P_B3) {
    bias[64 + p - P_B2] = w[p];
  } else if (p < P_B4) {
    bias[128 + p - P_B3] = w[p];
  } else {
    bias[192 + p - P_B4] = w[p];
  }
}

__global__ void param_grads_kernel(const float *__restrict__ g, float *__restrict__ out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < NPARAM) out[p] = param_grad(g, p);
}

}  // namespace wsnet

using namespace wsnet;

void warm_start_param_grads(const float *grad_products, float *out, cudaStream_t s) {
  param_grads_kernel<<<(NPARAM + 255) / 256, 256, 0, s>>>(grad_products, out);
  EMG_LAUNCH_CHECK();
}

void WarmStartNet::init(uint64_t seed, cudaStream_t s) {
  std::vector<float> w(NPARAM, 0.f);
  uint64_t st = seed * 6364136223846793005ull + 1442695040888963407ull;
  auto unif = [&]() {
    st = st * 6364136223846793005ull + 1442695040888963407ull;
    return ((st >> 11) * (1.0 / 9007199254740992.0)) * 2.0 - 1.0;  // [-1, 1)
  };
  // uniform with variance 2/fan_in (He initialisation); the output layer starts at zero
  for (int p = P_W1; p < P_W2; ++p) w[p] = (float)(unif() * std::sqrt(6.0 / 13.0));
  for (int p = P_W2; p < P_W4; ++p) w[p] = (float)(unif() * std::sqrt(6.0 / 64.0));
  params.upload(w, s);
  std::vector<float> z(NPARAM, 0.f);
  m.upload(z, s);
  v.upload(z, s);
  img.alloc(IMG_BYTES);
  img.zero(s);
  bias.alloc(4 * 64);
  bias.zero(s);
  grad.alloc(128 * 208 + 128 * 128);
  loss.alloc(1);
  loss0.alloc(1);
  err.alloc(1);
  err.zero(s);
  pack_kernel<<<(NPARAM + 255) / 256, 256, 0, s>>>(params.p, img.p, bias.p);
  EMG_LAUNCH_CHECK();
  step = 0;
  ready = true;
}

void WarmStartNet::set_params(const float *host, cudaStream_t s) {
  params.upload(host, NPARAM, s);
  pack_kernel<<<(NPARAM + 255) / 256, 256, 0, s>>>(params.p, img.p, bias.p);
  EMG_LAUNCH_CHECK();
}

int WarmStartNet::nparam() { return NPARAM; }
int WarmStartNet::image_bytes() { return IMG_BYTES; }

void WarmStartNet::statics(Context &c) {
  cudaStream_t s = c.stream;
  // log10 of the horizontal and vertical resistivity per attribute
  std::vector<float> lr(2 * (size_t)c.nrho);
  for (int i = 0; i < c.nrho; ++i) {
    const double *r = &c.rho[(size_t)i * c.ncol];
    double rh = r[0], rv = r[0];
    if (c.aniso_form == EMG_VERTICAL) rv = r[1];
    else if (c.aniso_form == EMG_TRIAXIAL || c.aniso_form == EMG_ARBITRARY) {
      rh = std::sqrt(r[0] * r[1]);
      rv = r[2];
    }
    lr[2 * i] = (float)std::log10(rh);
    lr[2 * i + 1] = (float)std::log10(rv);
  }
  DBuf<float> dlr, acc((size_t)c.ne * 3);
  dlr.upload(lr, s);
  acc.zero(s);
  stat.alloc((size_t)c.ne * 3);
  edge_rho_kernel<<<(c.nt + 255) / 256, 256, 0, s>>>(c.nt, c.t2e.p, c.attr.p, (const float2 *)dlr.p, acc.p);
  EMG_LAUNCH_CHECK();
  edge_static_kernel<<<(c.ne + 255) / 256, 256, 0, s>>>(c.ne, c.edges.p, c.pts.p, acc.p, stat.p);
  EMG_LAUNCH_CHECK();
  EMG_CUDA(cudaStreamSynchronize(s));  // temporaries go out of scope
  stat_ne = c.ne;
}

static void launch_mlp(int mode, const KArgs &a, int grid, cudaStream_t s) {
  // the network modes keep one CTA per SM (all 512 tensor-memory columns);
  // inference reads its bias and barrier words at the training offsets
  const int smem_need = SMEM_TRAIN;
  switch (mode) {
  case 0:
    mlp_kernel<0><<<grid, T, 0, s>>>(a);
    break;
  case 1:
    EMG_CUDA(cudaFuncSetAttribute(mlp_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_need));
    mlp_kernel<1><<<grid, T, smem_need, s>>>(a);
    break;
  default:
    EMG_CUDA(cudaFuncSetAttribute(mlp_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_need));
    mlp_kernel<2><<<grid, T, smem_need, s>>>(a);
  }
  EMG_LAUNCH_CHECK();
}

static int sm_count(int device) {
  int n = 0;
  EMG_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, device));
  return n;
}

double WarmStartNet::train_step(Context &c, const double *xs, int ks, const std::vector<Spec> &specs, long batch,
                                float lr, bool accumulate_only) {
  cudaStream_t s = c.stream;
  specs_dev.upload(specs, s);
  grad.zero(s);
  loss.zero(s);
  loss0.zero(s);
  KArgs a;
  std::memset(&a, 0, sizeof(a));
  a.img = img.p;
  a.bias = bias.p;
  a.stat = stat.p;
  a.spec = specs_dev.p;
  a.nspec = (int)specs.size();
  a.ne = c.ne;
  a.xs = (const double2 *)xs;
  a.ks = ks;
  a.nsamples = batch;
  a.mode = 2;
  a.seed = (uint32_t)(0x51ED2705u + 7919u * (uint32_t)step);
  a.inv_batch = 1.0f / (float)batch;
  a.grad = grad.p;
  a.loss = loss.p;
  a.loss0 = loss0.p;
  a.err = err.p;
  const long tiles = (batch + T - 1) / T;
  launch_mlp(2, a, (int)std::min<long>(tiles, sm_count(c.device)), s);
  if (!accumulate_only) {
    ++step;
    AdamArgs ad{params.p, m.p, v.p, grad.p, step, lr, 0.9f, 0.999f, 1e-8f, img.p, bias.p};
    adam_kernel<<<(NPARAM + 255) / 256, 256, 0, s>>>(ad);
    EMG_LAUNCH_CHECK();
    pack_kernel<<<(NPARAM + 255) / 256, 256, 0, s>>>(params.p, img.p, bias.p);
    EMG_LAUNCH_CHECK();
  }
  return 0.0;
}

void WarmStartNet::predict(Context &c, const double *xs, int ks, const std::vector<Spec> &specs, double *out,
                           int kt, bool network) {
  cudaStream_t s = c.stream;
  specs_dev.upload(specs, s);
  KArgs a;
  std::memset(&a, 0, sizeof(a));
  a.img = img.p;
  a.bias = bias.p;
  a.stat = stat.p;
  a.spec = specs_dev.p;
  a.nspec = (int)specs.size();
  a.ne = c.ne;
  a.xs = (const double2 *)xs;
  a.ks = ks;
  a.out = (double2 *)out;
  a.kt = kt;
  a.nsamples = (long)c.ne * (long)specs.size();
  a.mode = network ? 1 : 0;
  a.err = err.p;
  const long tiles = (a.nsamples + T - 1) / T;
  const int grid = network ? (int)std::min<long>(tiles, sm_count(c.device)) : (int)std::min<long>(tiles, 1L << 20);
  launch_mlp(a.mode, a, grid, s);
}

void WarmStartNet::check(cudaStream_t s) {
  int h = 0;
  err.download(&h, 1, s);
  EMG_CUDA(cudaStreamSynchronize(s));
  if (h) {
    err.zero(s);
    fail(EMG_ERR_CUDA, "warm-start network: a tensor-core completion wait timed out");
  }
}

}  // namespace emg
