// AMS preconditioner, batched FCG and batched FGMRES on the device.
//
// Restates the solver stack of solve_linear_system / pc_apply_b / create_pc
// (src/em_la.cc:35-228): FGMRES right-preconditioned by two FCG solves on
// B = C + M to rtol 1e-2, each preconditioned by AMS.  The PETSc/hypre
// internals are re-derived from the published methods: FGMRES (Saad 1993)
// with classical Gram-Schmidt, flexible CG with truncation (Notay 2000), AMS
// (Hiptmair & Xu 2007; Kolev & Vassilevski 2009) with cycle string
// "034515430" (hypre cycle type 13) and l1-Jacobi smoothing (Baker,
// Falgout, Kolev & Yang 2011) on edges and on every nodal AMG level.

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstring>
#include <numeric>
#include <cstdio>

#include "emg_amg_gpu.h"
#include "emg_solver.h"

namespace emg {

// ---------------------------------------------------------------------------
// small kernels
// ---------------------------------------------------------------------------
template <typename T>
__global__ void combine_kernel(long n, const double *__restrict__ a, const double *__restrict__ b, double w,
                               T *__restrict__ out) {
  long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < n) out[i] = (T)(a[i] + (b ? w * b[i] : 0.0));
}

template <typename T>
__global__ void l1_rowsum_kernel(int n, const int *__restrict__ rp, const double *__restrict__ a,
                                 const double *__restrict__ b, double w, T *__restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s = 0;
  for (int k = rp[i]; k < rp[i + 1]; ++k) s += fabs(a[k] + (b ? w * b[k] : 0.0));
  out[i] = (T)s;
}

__global__ void fcg_beta_kernel(int K, int nprev, const double *__restrict__ dots, const double *__restrict__ eta,
                                const int *__restrict__ active, double *__restrict__ beta) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= K * nprev) return;
  int c = i % K;
  double e = eta[i];
  beta[i] = (active[c] && e != 0.0) ? dots[i] / e : 0.0;
}

__global__ void fcg_alpha_kernel(int K, const double *__restrict__ dots, double *__restrict__ eta_slot,
                                 const int *__restrict__ active, double *__restrict__ alpha) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= K) return;
  double ps = dots[c], pr = dots[K + c];
  eta_slot[c] = ps;
  alpha[c] = (active[c] && ps != 0.0) ? pr / ps : 0.0;
}

template <typename T>
static void convert(const std::vector<double> &a, std::vector<T> &b) {
  b.resize(a.size());
  const long n = (long)a.size();
#pragma omp parallel for schedule(static)
  for (long k = 0; k < n; ++k) b[k] = (T)a[k];
}

template <typename T>
static void upload_csr(const HCsr &h, DCsr<T> &d, bool with_l1, cudaStream_t s) {
  d.n = h.n;
  d.m = h.m;
  d.nnz = h.nnz();
  d.rp.upload(h.rp, s);
  d.ci.upload(h.ci, s);
  std::vector<T> tmp;
  convert(h.vc, tmp);
  d.vc.upload(tmp, s);
  std::vector<T> tm;
  if (!h.vm.empty()) {
    convert(h.vm, tm);
    d.vm.upload(tm, s);
  } else {
    d.vm.release();
  }
  std::vector<T> lc, lm;
  if (with_l1) {
    lc.resize(h.n);
    lm.resize(h.vm.empty() ? 0 : h.n);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < h.n; ++i) {
      double a = 0, b = 0;
      for (int k = h.rp[i]; k < h.rp[i + 1]; ++k) {
        a += std::fabs(h.vc[k]);
        if (!h.vm.empty()) b += std::fabs(h.vm[k]);
      }
      lc[i] = (T)a;
      if (!h.vm.empty()) lm[i] = (T)b;
    }
    d.l1c.upload(lc, s);
    if (!h.vm.empty()) d.l1m.upload(lm, s);
    else d.l1m.release();
  }
  EMG_CUDA(cudaStreamSynchronize(s));  // host temporaries go out of scope
}

// a device AMG level operator into the solver's precision, with l1 row sums
template <typename T>
static void to_level(GCsr &g, DCsr<T> &d, bool with_l1, cudaStream_t s) {
  d.n = g.n;
  d.m = g.m;
  d.nnz = g.nnz;
  const unsigned gn = (unsigned)((g.nnz + 255) / 256), gr = (unsigned)((g.n + 255) / 256);
  d.vc.alloc(std::max<long>(g.nnz, 1));
  combine_kernel<T><<<gn, 256, 0, s>>>(g.nnz, g.vc.p, nullptr, 0.0, d.vc.p);
  if (g.vm.p) {
    d.vm.alloc(std::max<long>(g.nnz, 1));
    combine_kernel<T><<<gn, 256, 0, s>>>(g.nnz, g.vm.p, nullptr, 0.0, d.vm.p);
  } else {
    d.vm.release();
  }
  if (with_l1) {
    d.l1c.alloc(g.n);
    l1_rowsum_kernel<T><<<gr, 256, 0, s>>>(g.n, g.rp.p, g.vc.p, nullptr, 0.0, d.l1c.p);
    if (g.vm.p) {
      d.l1m.alloc(g.n);
      l1_rowsum_kernel<T><<<gr, 256, 0, s>>>(g.n, g.rp.p, g.vm.p, nullptr, 0.0, d.l1m.p);
    } else {
      d.l1m.release();
    }
  }
  EMG_LAUNCH_CHECK();
  EMG_CUDA(cudaStreamSynchronize(s));  // g's values go out of scope with the level
  d.rp = std::move(g.rp);
  d.ci = std::move(g.ci);
}

// ---------------------------------------------------------------------------
// AMS setup
// ---------------------------------------------------------------------------
// Vector nodal operator without couplings: row 3 v + d of out is row v of
// comp[d] with columns 3 u + d (comp[0..2] share one vertex pattern).
static void interleave_components(const HCsr *comp, HCsr &out) {
  const int nv = comp[0].n;
  const bool two = !comp[0].vm.empty();
  out.n = out.m = 3 * nv;
  out.rp.assign(3 * (size_t)nv + 1, 0);
  for (int v = 0; v < nv; ++v)
    for (int d = 0; d < 3; ++d) out.rp[3 * v + d + 1] = comp[d].rp[v + 1] - comp[d].rp[v];
  for (int i = 0; i < 3 * nv; ++i) out.rp[i + 1] += out.rp[i];
  out.ci.resize(out.rp[3 * nv]);
  out.vc.resize(out.rp[3 * nv]);
  out.vm.resize(two ? out.rp[3 * nv] : 0);
#pragma omp parallel for schedule(static)
  for (int v = 0; v < nv; ++v)
    for (int d = 0; d < 3; ++d) {
      long p = out.rp[3 * v + d];
      for (int k = comp[d].rp[v]; k < comp[d].rp[v + 1]; ++k, ++p) {
        out.ci[p] = 3 * comp[d].ci[k] + d;
        out.vc[p] = comp[d].vc[k];
        if (two) out.vm[p] = comp[d].vm[k];
      }
    }
}
// host wall time of a setup stage, kept in the context's timing table
struct StageClock {
  Context &c;
  std::chrono::steady_clock::time_point t = std::chrono::steady_clock::now();
  explicit StageClock(Context &cc) : c(cc) {}
  void lap(const char *name) {
    auto now = std::chrono::steady_clock::now();
    c.kernel_ms[name] = std::chrono::duration<double, std::milli>(now - t).count();
    t = now;
  }
};

template <typename T>
void ams_setup(Context &c, Ams<T> &ams, bool per_frequency, double w, double w_ref) {
  cudaStream_t s = c.stream;
  StageClock clk(c);
  ams.ctx = &c;
  ams.ne = c.ne;
  ams.nv = c.nv;
  ams.edges = c.edges.p;
  ams.inc_rp = c.vinc_rp.p;
  ams.inc = c.vinc.p;
  ams.cycle = c.opt.ams_cycle;
  // the batched path's own sweep count: with its capped inner solves, two
  // edge sweeps per smoothing step cut the AMS applications by a quarter
  ams.relax_times = per_frequency ? c.opt.ams_relax_times : c.opt.block_relax_times;
  ams.relax_w = c.opt.ams_relax_weight;
  ams.amg_relax_times = c.opt.amg_relax_times;
  ams.cheb = c.opt.smoother_cheb;
  ams.cheb_degree = per_frequency ? c.opt.cheb_degree : c.opt.block_cheb_degree;
  ams.amg_cheb_degree = c.opt.amg_cheb_degree;
  ams.restrict_j0 = c.opt.restrict_j0 != 0;
  ams.amg_pre_smooth = c.opt.amg_pre_smooth != 0;
  ams.two = !per_frequency;
  ams.use_graphs = c.opt.graphs != 0;
  ams.fused = c.opt.ams_fused != 0;
  ams.fused_bps = c.opt.fused_bps;
  ams.fused_rows = c.opt.fused_rows;
  ams.fused_wait_ns = (unsigned long long)(c.opt.fused_wait_ms * 1e6);
  ams.fused_withhold = c.opt.fused_test_withhold;
  ams.fused_epoch = -1;
  // FP32 applications close with the gradient correction and hand it back
  // as a potential: after it, no FP32 product touches the (air) gradient
  // component, which can exceed the rest of the iterate by 1e10 at low
  // frequency, far beyond what FP32 rounding of C x tolerates
  ams.split_gradient = sizeof(T) == 4;
  if (ams.split_gradient) {
    ams.cycle = c.opt.fp32_cycle;
    if (ams.cycle.empty() || ams.cycle.back() != '1')
      fail(EMG_ERR_OPTION, "the FP32 AMS cycle must end with the gradient correction '1'");
  }
  ams.graphs.clear();
  ams.K = 0;
  // edge operator B = C + w Ms (src/em_la.cc:122-128)
  ams.B.n = ams.B.m = c.ne;
  ams.B.nnz = c.nnz;
  ams.brp = c.rp.p;
  ams.bci = c.ci.p;
  ams.nnzB = c.nnz;
  unsigned g = (unsigned)((c.nnz + 255) / 256), gr = (unsigned)((c.ne + 255) / 256);
  ams.B.vc.alloc(c.nnz);
  ams.B.l1c.alloc(c.ne);
  if (per_frequency) {
    combine_kernel<T><<<g, 256, 0, s>>>(c.nnz, c.Cv.p, c.Msv.p, w, ams.B.vc.p);
    l1_rowsum_kernel<T><<<gr, 256, 0, s>>>(c.ne, c.rp.p, c.Cv.p, c.Msv.p, w, ams.B.l1c.p);
    ams.B.vm.release();
    ams.B.l1m.release();
  } else {
    ams.B.vm.alloc(c.nnz);
    ams.B.l1m.alloc(c.ne);
    combine_kernel<T><<<g, 256, 0, s>>>(c.nnz, c.Cv.p, nullptr, 0.0, ams.B.vc.p);
    combine_kernel<T><<<g, 256, 0, s>>>(c.nnz, c.Msv.p, nullptr, 0.0, ams.B.vm.p);
    l1_rowsum_kernel<T><<<gr, 256, 0, s>>>(c.ne, c.rp.p, c.Cv.p, nullptr, 0.0, ams.B.l1c.p);
    l1_rowsum_kernel<T><<<gr, 256, 0, s>>>(c.ne, c.rp.p, c.Msv.p, nullptr, 0.0, ams.B.l1m.p);
  }
  EMG_LAUNCH_CHECK();
  // FP32 two-part B also as one 16-byte record per nonzero for the SpMM's
  // packed variant (the autotuner decides whether it is used)
  if (sizeof(T) == 4 && !per_frequency) {
    ams.Bpk.alloc(c.nnz);
    pack_records(c.nnz, c.ci.p, (const float *)ams.B.vc.p, (const float *)ams.B.vm.p, ams.Bpk.p, s);
    std::vector<int> crp;
    const long nch = chunk_row_pointer(c.h_rp, crp);
    ams.Bcrp.upload(crp, s);
    ams.Bch.alloc((size_t)std::max(3 * nch, 3L));
    chunk_records(c.ne, c.rp.p, c.ci.p, (const float *)ams.B.vc.p, (const float *)ams.B.vm.p, ams.Bcrp.p,
                  ams.Bch.p, s);
    EMG_CUDA(cudaStreamSynchronize(s));  // the host row pointer goes out of scope
  } else {
    ams.Bpk.release();
    ams.Bch.release();
    ams.Bcrp.release();
  }
  // edge tangents x(v1) - x(v0)
  {
    std::vector<T> tg((size_t)c.ne * 3);
    for (int e = 0; e < c.ne; ++e)
      for (int d = 0; d < 3; ++d)
        tg[3 * (size_t)e + d] = (T)(c.h_pts[3 * (size_t)c.h_edges[2 * e + 1] + d] - c.h_pts[3 * (size_t)c.h_edges[2 * e] + d]);
    ams.tangent.upload(tg, s);
    EMG_CUDA(cudaStreamSynchronize(s));
  }
  EMG_CUDA(cudaStreamSynchronize(s));
  clk.lap("setup_edge");
  // G^T B for the gradient-space residual
  {
    DBuf<double> gc, gm;
    assemble_gtb(c, gc, gm);
    ams.grp = c.grp.p;
    ams.gci = c.gci.p;
    ams.nnzG = c.h_grp[c.nv];
    unsigned gg = (unsigned)((ams.nnzG + 255) / 256);
    ams.gvc.alloc(ams.nnzG);
    if (per_frequency) {
      combine_kernel<T><<<gg, 256, 0, s>>>(ams.nnzG, gc.p, gm.p, w, ams.gvc.p);
      ams.gvm.release();
    } else {
      ams.gvm.alloc(ams.nnzG);
      combine_kernel<T><<<gg, 256, 0, s>>>(ams.nnzG, gc.p, nullptr, 0.0, ams.gvc.p);
      combine_kernel<T><<<gg, 256, 0, s>>>(ams.nnzG, gm.p, nullptr, 0.0, ams.gvm.p);
    }
    EMG_LAUNCH_CHECK();
    EMG_CUDA(cudaStreamSynchronize(s));
  }
  // nodal subspace operators (only those the cycle visits) and their
  // hierarchies; each hierarchy's build is parallel inside
  bool want[NSUB] = {false, false, false, false, false};
  for (char ch : ams.cycle) {
    const int sp = ams_subspace(ch);
    if (sp >= 0) want[sp] = true;
  }
  clk.lap("setup_gtb");
  HCsr nod[NSUB];
  const bool pi_coupled = c.opt.pi_coupled != 0;
  AmgParams prm;
  prm.theta = c.opt.amg_theta;
  prm.pmax = c.opt.amg_pmax;
  prm.max_coarse = c.opt.amg_max_coarse;
  prm.max_levels = c.opt.amg_max_levels;
  if (c.opt.gpu_amg && !pi_coupled) {
    // nodal operators and their hierarchies built on the device
    DBuf<double> parts;
    assemble_nodal_device(c, parts);
    EMG_CUDA(cudaStreamSynchronize(s));
    clk.lap("setup_nodal");
    double amg_ms = 0, conv_ms = 0;
    for (int sp = 0; sp < NSUB; ++sp) {
      auto &S = ams.sub[sp];
      S.lv.clear();
      S.coarse = HCsr();
      S.nc = 0;
      S.cinv.release();
      S.cinv_w.clear();
      if (!want[sp]) continue;
      auto ta = std::chrono::steady_clock::now();
      GCsr A0;
      nodal_operator_gpu(c, parts, sp, A0, per_frequency ? w : -1.0);
      AmgParams p2 = prm;
      p2.seed = prm.seed + 7919ull * (uint64_t)sp;
      p2.num_functions = sp == SUB_PIVEC ? 3 : 1;
      std::vector<GpuLevel> glv;
      GCsr gco;
      amg_build_gpu(std::move(A0), w_ref, p2, glv, gco, s);
      auto tb = std::chrono::steady_clock::now();
      amg_ms += std::chrono::duration<double, std::milli>(tb - ta).count();
      S.lv.resize(glv.size());
      for (size_t l = 0; l < glv.size(); ++l) {
        S.lv[l].nnzA = glv[l].A.nnz;
        S.lv[l].nnzP = glv[l].P.nnz;
        S.lv[l].nnzR = glv[l].R.nnz;
        to_level<T>(glv[l].A, S.lv[l].A, true, s);
        to_level<T>(glv[l].P, S.lv[l].P, false, s);
        to_level<T>(glv[l].R, S.lv[l].R, false, s);
      }
      gcsr_to_host(gco, S.coarse, s);
      S.nc = S.coarse.n;
      conv_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tb).count();
    }
    c.kernel_ms["setup_amg"] = amg_ms;
    c.kernel_ms["setup_upload"] = conv_ms;
    for (int sp = 0; sp < NSUB; ++sp) {
      ams.wb[sp].clear();
      ams.wx[sp].clear();
      ams.wr[sp].clear();
      ams.wx2[sp].clear();
      ams.wd[sp].clear();
    }
    ams.ws_K = 0;
    return;
  }
  if (want[0] || want[1] || want[2] || want[3] || (want[SUB_PIVEC] && !pi_coupled)) assemble_nodal(c, nod);
  if (want[SUB_PIVEC]) {
    if (pi_coupled) assemble_pi_vector(c, nod[SUB_PIVEC], true);
    else interleave_components(nod + 1, nod[SUB_PIVEC]);  // the x/y/z operators side by side
  }
  clk.lap("setup_nodal");
  double amg_ms = 0, upload_ms = 0;
  for (int sp = 0; sp < NSUB; ++sp) {
    auto &S = ams.sub[sp];
    S.lv.clear();
    S.coarse = HCsr();
    S.nc = 0;
    S.cinv.release();
    S.cinv_w.clear();
    if (!want[sp]) continue;
    if (per_frequency) {
      for (size_t k = 0; k < nod[sp].vc.size(); ++k) nod[sp].vc[k] += w * nod[sp].vm[k];
      nod[sp].vm.clear();
    }
    HostAmg hamg;
    AmgParams p2 = prm;
    p2.seed = prm.seed + 7919ull * (uint64_t)sp;
    p2.num_functions = sp == SUB_PIVEC ? 3 : 1;
    auto ta = std::chrono::steady_clock::now();
    amg_build(std::move(nod[sp]), w_ref, p2, hamg);
    auto tb = std::chrono::steady_clock::now();
    amg_ms += std::chrono::duration<double, std::milli>(tb - ta).count();
    S.lv.resize(hamg.lv.size());
    for (size_t l = 0; l < hamg.lv.size(); ++l) {
      upload_csr(hamg.lv[l].A, S.lv[l].A, true, s);
      upload_csr(hamg.lv[l].P, S.lv[l].P, false, s);
      upload_csr(hamg.lv[l].R, S.lv[l].R, false, s);
      S.lv[l].nnzA = hamg.lv[l].A.nnz();
      S.lv[l].nnzP = hamg.lv[l].P.nnz();
      S.lv[l].nnzR = hamg.lv[l].R.nnz();
    }
    S.coarse = std::move(hamg.coarse);
    S.nc = S.coarse.n;
    upload_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tb).count();
  }
  c.kernel_ms["setup_amg"] = amg_ms;
  c.kernel_ms["setup_upload"] = upload_ms;
  for (int sp = 0; sp < NSUB; ++sp) {
    ams.wb[sp].clear();
    ams.wx[sp].clear();
    ams.wr[sp].clear();
    ams.wx2[sp].clear();
    ams.wd[sp].clear();
  }
  ams.ws_K = 0;
}

template <typename T>
void Ams<T>::set_columns(const std::vector<double> &col_omega, cudaStream_t s) {
  if ((int)col_omega.size() != K) graphs.clear();
  K = (int)col_omega.size();
  h_omega = col_omega;
  const double *om_before = omega.p;
  omega.upload(col_omega, s);
  if (omega.p != om_before) graphs.clear();
  std::vector<double> distinct;
  if (two) {
    distinct = col_omega;
    std::sort(distinct.begin(), distinct.end());
    distinct.erase(std::unique(distinct.begin(), distinct.end()), distinct.end());
  } else {
    distinct.push_back(0.0);
  }
  std::vector<int> slot(K, 0);
  for (int c = 0; c < K; ++c)
    slot[c] = two ? (int)(std::lower_bound(distinct.begin(), distinct.end(), col_omega[c]) - distinct.begin()) : 0;
  const int *cs_before = cslot.p;
  cslot.upload(slot, s);
  if (cslot.p != cs_before) graphs.clear();
  for (int sp = 0; sp < NSUB; ++sp) {
    Sub &S = sub[sp];
    if (S.nc == 0 || (S.cinv_w == distinct && S.cinv.p)) continue;
    size_t nc2 = (size_t)S.nc * S.nc;
    std::vector<double> all(nc2 * distinct.size());
#pragma omp parallel for schedule(dynamic, 1)
    for (int d = 0; d < (int)distinct.size(); ++d) {
      std::vector<double> X;
      coarse_inverse(S.coarse, distinct[d], X);
      std::copy(X.begin(), X.end(), all.begin() + nc2 * d);
    }
    const double *before = S.cinv.p;
    S.cinv.upload(all, s);
    if (S.cinv.p != before) graphs.clear();  // captured graphs hold the old address
    S.cinv_w = distinct;
  }
  EMG_CUDA(cudaStreamSynchronize(s));
  ensure_workspace(s);
  prepare_fused(s);
}

template <typename T>
void Ams<T>::ensure_workspace(cudaStream_t s) {
  (void)s;
  if (ws_K == K) return;
  graphs.clear();
  er.alloc((size_t)ne * K);
  ex2.alloc((size_t)ne * K);
  ed.alloc((size_t)ne * K);
  if (cheb && cheb_degree > 2) ed2.alloc((size_t)ne * K);
  else ed2.release();
  gtmp.alloc((size_t)nv * K);
  for (int sp = 0; sp < NSUB; ++sp) {
    Sub &S = sub[sp];
    size_t L = S.lv.size();
    wb[sp].clear();
    wx[sp].clear();
    wr[sp].clear();
    wx2[sp].clear();
    wd[sp].clear();
    wd2[sp].clear();
    wd[sp].resize(L + 1);
    wd2[sp].resize(L + 1);
    wb[sp].resize(L + 1);
    wx[sp].resize(L + 1);
    wr[sp].resize(L + 1);
    wx2[sp].resize(L + 1);
    for (size_t l = 0; l <= L; ++l) {
      size_t n = (l < L ? (size_t)S.lv[l].A.n : (size_t)S.nc) * K;
      wb[sp][l].alloc(std::max<size_t>(n, 1));
      wx[sp][l].alloc(std::max<size_t>(n, 1));
      if (l < L) {
        wr[sp][l].alloc(n);
        wx2[sp][l].alloc(n);
        wd[sp][l].alloc(n);
        if (cheb && amg_cheb_degree > 2) wd2[sp][l].alloc(n);
      }
    }
  }
  ws_K = K;
}

template <typename T>
void Ams<T>::spmm_B(int mode, const T *x, const T *b, T *y, cudaStream_t s) {
  SpmmArgs a;
  std::memset(&a, 0, sizeof(a));
  a.pk = Bpk.p;
  a.ch = Bch.p;
  a.crp = Bcrp.p;
  a.n = ne;
  a.rp = brp;
  a.ci = bci;
  a.vc = B.vc.p;
  a.vm = two ? (const void *)B.vm.p : nullptr;
  a.l1c = B.l1c.p;
  a.l1m = two ? (const void *)B.l1m.p : nullptr;
  a.omega = omega.p;
  a.x = x;
  a.b = b;
  a.y = y;
  a.relax_w = relax_w;
  a.mode = mode;
  KernelProfiler &pf = profiler();
  cudaEvent_t ev = nullptr;
  const char *bin = sizeof(T) == 4 ? "spmm_edge_fp32" : "spmm_edge_fp64";
  if (pf.enabled) pf.begin(bin, s, spmm_algo_bytes(ne, nnzB, K, sizeof(T), two, mode), &ev);
  const TiledPattern *tp = edge_tiles();
  if (tp) spmm_tiled<T>(K, a, *tp, s);
  else spmm_nnz<T>(K, a, nnzB, s);
  if (pf.enabled) pf.end(bin, s, ev);
}

template <typename T>
const TiledPattern *Ams<T>::edge_tiles() {
  return ctx ? tiled_pattern(*ctx, brp, ctx->h_rp, ctx->h_ci, K * (int)sizeof(T)) : nullptr;
}

template <typename T>
const TiledPattern *Ams<T>::gtb_tiles() {
  return ctx ? tiled_pattern(*ctx, grp, ctx->h_grp, ctx->h_gci, K * (int)sizeof(T)) : nullptr;
}

template <typename T>
void Ams<T>::emit_spmm(const SpmmArgs &a, long nnz, const char *bin, cudaStream_t s, const TiledPattern *tp) {
  if (rec) {
    FusedOp op;
    std::memset(&op, 0, sizeof(op));
    op.kind = FOP_SPMM;
    op.nnz = nnz;
    op.a = a;
    rec->push_back(op);
    return;
  }
  KernelProfiler &pf = profiler();
  cudaEvent_t ev = nullptr;
  if (pf.enabled) pf.begin(bin, s, spmm_algo_bytes(a.n, nnz, K, sizeof(T), a.vm != nullptr, a.mode), &ev);
  if (tp) spmm_tiled<T>(K, a, *tp, s);
  else spmm_nnz<T>(K, a, nnz, s);
  if (pf.enabled) pf.end(bin, s, ev);
}

template <typename T>
void Ams<T>::emit_jac0(int n, const T *b, const T *l1c, const T *l1m, double w, T *y, T *d, cudaStream_t s) {
  if (rec) {
    FusedOp op;
    std::memset(&op, 0, sizeof(op));
    op.kind = d ? FOP_JAC0_2 : FOP_JAC0;
    op.a.n = n;
    op.a.b = b;
    op.a.l1c = l1c;
    op.a.l1m = l1m;
    op.a.omega = omega.p;
    op.a.relax_w = w;
    op.a.y = y;
    op.a.d = d;
    rec->push_back(op);
    return;
  }
  if (d) jacobi0_2<T>(n, K, b, l1c, l1m, omega.p, w, y, d, s);
  else jacobi0<T>(n, K, b, l1c, l1m, omega.p, w, y, s);
}

template <typename T>
void Ams<T>::emit_coarse(int sp, const T *b, T *x, cudaStream_t s) {
  Sub &S = sub[sp];
  if (rec) {
    if (S.nc == 0) return;
    FusedOp op;
    std::memset(&op, 0, sizeof(op));
    op.kind = FOP_COARSE;
    op.a.n = S.nc;
    op.a.vc = S.cinv.p;
    op.a.ci = cslot.p;
    op.a.b = b;
    op.a.y = x;
    rec->push_back(op);
    return;
  }
  coarse_apply<T>(S.nc, K, S.cinv.p, cslot.p, b, x, s);
}

template <typename T>
static SpmmArgs level_args(const DCsr<T> &A, int mode, const double *omega, double w, const T *x, const T *b,
                           T *y) {
  SpmmArgs a;
  std::memset(&a, 0, sizeof(a));
  a.n = A.n;
  a.rp = A.rp.p;
  a.ci = A.ci.p;
  a.vc = A.vc.p;
  a.vm = A.vm.p;
  a.l1c = A.l1c.p;
  a.l1m = A.l1m.p;
  a.omega = omega;
  a.x = x;
  a.b = b;
  a.y = y;
  a.relax_w = w;
  a.mode = mode;
  return a;
}

// Chebyshev smoothing of degree m on D^-1 A with D the l1 row sums: the
// spectrum lies in (0, 1], the smoothed interval is [1/30, 1].  Three-term
// recurrence (Saad, Iterative Methods for Sparse Linear Systems, 2nd ed.,
// Alg. 12.1): theta, delta the interval's centre and half-width, sigma =
// theta / delta, rho_0 = 1 / sigma, rho_k = 1 / (2 sigma - rho_{k-1});
// d_0 = D^-1 r_0 / theta, then r_k = r_{k-1} - A d_{k-1},
// d_k = rho_k rho_{k-1} d_{k-1} + (2 rho_k / delta) D^-1 r_k, x += d_k.
struct ChebCoef {
  double inv_theta;
  double c1[8], c2[8];  // step k = 1 .. m-1
  explicit ChebCoef(int m) {
    const double lmax = 1.0, lmin = lmax / 30.0;
    const double th = 0.5 * (lmax + lmin), de = 0.5 * (lmax - lmin), sg = th / de;
    inv_theta = 1.0 / th;
    double rho = 1.0 / sg;
    for (int k = 1; k < m && k < 8; ++k) {
      const double rn = 1.0 / (2.0 * sg - rho);
      c1[k] = rn * rho;
      c2[k] = 2.0 * rn / de;
      rho = rn;
    }
  }
};

static const ChebCoef &cheb_coef(int m) {
  static const ChebCoef tab[7] = {ChebCoef(2), ChebCoef(2), ChebCoef(2), ChebCoef(3),
                                  ChebCoef(4), ChebCoef(5), ChebCoef(6)};
  return tab[std::min(std::max(m, 2), 6)];
}

template <typename T>
T *Ams<T>::smooth(const DCsr<T> *A, long nnz, int n, T *cur, T *oth, const T *b, T *rbuf, T *dbuf, T *dbuf2,
                  bool zero_guess, const char *bin, cudaStream_t s, bool started) {
  const bool edge = A == nullptr;
  const T *l1c = edge ? B.l1c.p : A->l1c.p;
  const T *l1m = edge ? (two ? B.l1m.p : nullptr) : A->l1m.p;
  auto run = [&](int mode, const T *x, const T *bb, T *y, T *r, T *d, double c1, double c2) {
    SpmmArgs a;
    std::memset(&a, 0, sizeof(a));
    a.pk = edge ? Bpk.p : nullptr;
    a.ch = edge ? Bch.p : nullptr;
    a.crp = edge ? Bcrp.p : nullptr;
    a.n = n;
    a.rp = edge ? brp : A->rp.p;
    a.ci = edge ? bci : A->ci.p;
    a.vc = edge ? (const void *)B.vc.p : (const void *)A->vc.p;
    a.vm = edge ? (two ? (const void *)B.vm.p : nullptr) : (const void *)A->vm.p;
    a.l1c = l1c;
    a.l1m = l1m;
    a.omega = omega.p;
    a.x = x;
    a.b = bb;
    a.y = y;
    a.relax_w = relax_w;
    a.mode = mode;
    a.r = r;
    a.d = d;
    a.c1 = c1;
    a.c2 = c2;
    emit_spmm(a, nnz, bin, s, edge ? edge_tiles() : nullptr);
  };
  if (!cheb) {
    if (zero_guess) {
      if (!started) emit_jac0(n, b, l1c, l1m, relax_w, cur, nullptr, s);
      return cur;
    }
    run(SPMM_JAC, cur, b, oth, nullptr, nullptr, 0, 0);
    return oth;
  }
  const int m = std::min(std::max(edge ? cheb_degree : amg_cheb_degree, 2), 6);
  if (m > 2 && !dbuf2) fail(EMG_ERR_STATE, "Chebyshev degree %d without its second direction buffer", m);
  const ChebCoef &ch = cheb_coef(m);
  T *y = zero_guess ? cur : oth;
  const T *rprev;  // r_{k-1}: b itself after a zero start, else rbuf
  if (zero_guess) {
    if (!started) emit_jac0(n, b, l1c, l1m, ch.inv_theta, cur, dbuf, s);
    rprev = b;
  } else {
    run(SPMM_CHEB1, cur, b, oth, rbuf, dbuf, ch.inv_theta, 0);
    rprev = rbuf;
  }
  T *dA = dbuf, *dB = dbuf2;
  for (int k = 1; k < m; ++k) {
    if (k + 1 == m) {
      run(SPMM_CHEB2, dA, nullptr, y, const_cast<T *>(rprev), nullptr, ch.c1[k], ch.c2[k]);
    } else {
      run(SPMM_CHEBK, dA, rprev, y, rbuf, dB, ch.c1[k], ch.c2[k]);
      rprev = rbuf;
      std::swap(dA, dB);
    }
  }
  return y;
}

template <typename T>
void Ams<T>::vcycle(int sp, int l, cudaStream_t s, bool started) {
  Sub &S = sub[sp];
  const int L = (int)S.lv.size();
  if (fused && !rec && l == fused_from[sp] && l < L) {
    launch_fused(sp, s);
    return;
  }
  if (l == L) {
    emit_coarse(sp, wb[sp][l].p, wx[sp][l].p, s);
    return;
  }
  Level &lv = S.lv[l];
  const int n = lv.A.n;
  const char *bin = sizeof(T) == 4 ? "spmm_nodal_fp32" : "spmm_nodal_fp64";
  // out-of-place smoothing applications after the zero-guess one:
  // (amg_relax_times - 1) pre + amg_relax_times post (without pre-smoothing:
  // the amg_relax_times post ones); start in the buffer that makes the last
  // one land in wx
  const int swaps = amg_pre_smooth ? 2 * amg_relax_times - 1 : amg_relax_times;
  T *cur = (swaps & 1) ? wx2[sp][l].p : wx[sp][l].p;
  T *oth = (swaps & 1) ? wx[sp][l].p : wx2[sp][l].p;
  const T *b = wb[sp][l].p;
  T *r = wr[sp][l].p, *d = wd[sp][l].p, *d2 = wd2[sp][l].p;
  if (!amg_pre_smooth) {
    // V(0, m): zero start, so the residual is b itself; the coarse
    // correction P e is the first iterate
    emit_spmm(level_args<T>(lv.R, SPMM_AX, nullptr, 1.0, b, nullptr, wb[sp][l + 1].p), lv.nnzR, bin, s);
    vcycle(sp, l + 1, s, false);
    emit_spmm(level_args<T>(lv.P, SPMM_AX, nullptr, 1.0, wx[sp][l + 1].p, nullptr, cur), lv.nnzP, bin, s);
    for (int it = 0; it < amg_relax_times; ++it) {
      T *res = smooth(&lv.A, lv.nnzA, n, cur, oth, b, r, d, d2, false, bin, s);
      if (res != cur) std::swap(cur, oth);
    }
    return;
  }
  for (int it = 0; it < amg_relax_times; ++it) {
    T *res = smooth(&lv.A, lv.nnzA, n, cur, oth, b, r, d, d2, it == 0, bin, s, started && it == 0);
    if (res != cur) std::swap(cur, oth);
  }
  emit_spmm(level_args<T>(lv.A, SPMM_RES, omega.p, relax_w, cur, b, r), lv.nnzA, bin, s);
  // the restriction to a level (not the coarsest) also takes that level's
  // first zero-guess smoothing step, into the buffer vcycle(l + 1) starts in
  SpmmArgs ra = level_args<T>(lv.R, SPMM_AX, nullptr, 1.0, r, nullptr, wb[sp][l + 1].p);
  const bool j0 = restrict_j0 && l + 1 < L;
  if (j0) {
    const DCsr<T> &An = S.lv[l + 1].A;
    ra.mode = SPMM_AXJ0;
    ra.omega = omega.p;
    ra.l1c = An.l1c.p;
    ra.l1m = An.l1m.p;
    ra.r = (swaps & 1) ? wx2[sp][l + 1].p : wx[sp][l + 1].p;
    ra.d = cheb ? wd[sp][l + 1].p : nullptr;
    ra.c1 = cheb ? cheb_coef(amg_cheb_degree).inv_theta : relax_w;
  }
  emit_spmm(ra, lv.nnzR, bin, s);
  vcycle(sp, l + 1, s, j0);
  emit_spmm(level_args<T>(lv.P, SPMM_ADD, nullptr, 1.0, wx[sp][l + 1].p, nullptr, cur), lv.nnzP, bin, s);
  for (int it = 0; it < amg_relax_times; ++it) {
    T *res = smooth(&lv.A, lv.nnzA, n, cur, oth, b, r, d, d2, false, bin, s);
    if (res != cur) std::swap(cur, oth);
  }
}

template <typename T>
void Ams<T>::prepare_fused(cudaStream_t s) {
  if (!fused || (fused_epoch == graphs.epoch && ws_K == K)) return;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  EMG_CUDA(cudaStreamIsCapturing(s, &cs));
  if (cs != cudaStreamCaptureStatusNone) fail(EMG_ERR_STATE, "fused V-cycle steps not recorded before capture");
  ensure_workspace(s);
  bool moved = false;
  std::vector<FusedOp> lists[NSUB];  // alive until the uploads have completed
  for (int sp = 0; sp < NSUB; ++sp) {
    std::vector<FusedOp> &ops = lists[sp];
    // levels below fused_rows rows run fused; the larger ones step by step
    const int L = (int)sub[sp].lv.size();
    int l0 = 0;
    while (l0 < L && sub[sp].lv[l0].A.n >= fused_rows) ++l0;
    fused_from[sp] = l0;
    if (l0 >= L) {
      fops_n[sp] = 0;
      fops_bytes[sp] = 0;
      continue;
    }
    rec = &ops;
    try {
      vcycle(sp, l0, s);
    } catch (...) {
      rec = nullptr;
      throw;
    }
    rec = nullptr;
    double bytes = 0;
    for (const FusedOp &op : ops)
      if (op.kind == FOP_SPMM) bytes += spmm_algo_bytes(op.a.n, op.nnz, K, sizeof(T), op.a.vm != nullptr, op.a.mode);
    const FusedOp *before = fops[sp].p;
    fops[sp].upload(ops, s);
    moved |= fops[sp].p != before;
    fops_n[sp] = (int)ops.size();
    fops_bytes[sp] = bytes;
  }
  if (!fbar.p) {
    fbar.alloc(2);
    ferr.alloc(1);
    moved = true;
  }
  fbar.zero(s);
  ferr.zero(s);
  if (!h_ferr.p) EMG_CUDA(cudaMallocHost((void **)&h_ferr.p, sizeof(int)));
  *h_ferr.p = 0;
  EMG_CUDA(cudaStreamSynchronize(s));  // host step lists go out of scope
  if (moved) graphs.clear();           // captured graphs hold the old addresses
  fused_epoch = graphs.epoch;
}

template <typename T>
void Ams<T>::check_fused(cudaStream_t s) {
  if (!h_ferr.p || *(volatile int *)h_ferr.p == 0) return;
  fbar.zero(s);
  ferr.zero(s);
  EMG_CUDA(cudaStreamSynchronize(s));
  *h_ferr.p = 0;
  fail(EMG_ERR_CUDA, "fused nodal V-cycle: a grid barrier wait timed out");
}

template <typename T>
void Ams<T>::run_vcycle(int sp, cudaStream_t s) {
  if (fused && (fused_epoch != graphs.epoch || ws_K != K)) prepare_fused(s);
  vcycle(sp, 0, s);
}

template <typename T>
void Ams<T>::launch_fused(int sp, cudaStream_t s) {
  KernelProfiler &pf = profiler();
  cudaEvent_t ev = nullptr;
  const char *bin = sizeof(T) == 4 ? "vcycle_fused_fp32" : "vcycle_fused_fp64";
  if (pf.enabled) pf.begin(bin, s, fops_bytes[sp], &ev);
  vcycle_fused<T>(K, fops[sp].p, fops_n[sp], fbar.p, ferr.p, fused_bps, s, fused_wait_ns, fused_withhold);
  if (pf.enabled) pf.end(bin, s, ev);
}

// One AMS application.  With graphs enabled the first call for a (b, x) pair
// runs eagerly (it also lets the SpMM autotuner pick lane layouts); the
// second is captured into a CUDA graph that every later call replays, so the
// few hundred small launches of the nodal V-cycles cost one graph launch.
template <typename T>
void Ams<T>::apply(const T *b, T *x, cudaStream_t s) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  EMG_CUDA(cudaStreamIsCapturing(s, &cs));
  if (fused && cs == cudaStreamCaptureStatusNone) {
    check_fused(s);
    prepare_fused(s);
  }
  if (!use_graphs || cs != cudaStreamCaptureStatusNone || profiler().enabled) {
    apply_eager(b, x, s);
    return;
  }
  auto key = std::make_pair((const void *)b, (void *)x);
  auto it = graphs.exec.find(key);
  if (it != graphs.exec.end()) {
    EMG_CUDA(cudaGraphLaunch(it->second, s));
    add_launches(graphs.kernels[key]);
    return;
  }
  if (graphs.seen[key]++ == 0) {
    apply_eager(b, x, s);
    return;
  }
  cudaGraph_t g;
  const long l0 = launch_count();
  EMG_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  try {
    apply_eager(b, x, s);
  } catch (...) {
    cudaStreamEndCapture(s, &g);
    if (g) cudaGraphDestroy(g);
    throw;
  }
  EMG_CUDA(cudaStreamEndCapture(s, &g));
  cudaGraphExec_t ex;
  cudaError_t e = cudaGraphInstantiate(&ex, g, 0);
  cudaGraphDestroy(g);
  EMG_CUDA(e);
  graphs.exec[key] = ex;
  graphs.kernels[key] = launch_count() - l0;  // counted at capture; the launch below runs them
  EMG_CUDA(cudaGraphLaunch(ex, s));
}

template <typename T>
void Ams<T>::grad_vcycle(const T *b, T *x, cudaStream_t s) {
  if (fused) prepare_fused(s);
  ensure_workspace(s);
  const size_t bytes = sizeof(T) * (size_t)nv * K;
  EMG_CUDA(cudaMemcpyAsync(wb[0][0].p, b, bytes, cudaMemcpyDeviceToDevice, s));
  run_vcycle(0, s);
  EMG_CUDA(cudaMemcpyAsync(x, wx[0][0].p, bytes, cudaMemcpyDeviceToDevice, s));
}

template <typename T>
void Ams<T>::apply_eager(const T *b, T *x, cudaStream_t s) {
  // count out-of-place edge smoothing applications to choose the start buffer
  int zeros = 0;
  for (char ch : cycle)
    if (ch == '0') ++zeros;
  const bool starts_with_smoother = !cycle.empty() && cycle[0] == '0';
  const int sweeps = zeros * relax_times - (starts_with_smoother ? 1 : 0);
  T *cur = (sweeps & 1) ? ex2.p : x;
  T *oth = (sweeps & 1) ? x : ex2.p;
  const char *bin = sizeof(T) == 4 ? "spmm_edge_fp32" : "spmm_edge_fp64";
  bool zero = true;
  for (size_t ci = 0; ci < cycle.size(); ++ci) {
    const char ch = cycle[ci];
    if (ch == '0') {
      for (int it = 0; it < relax_times; ++it) {
        T *res = smooth(nullptr, nnzB, ne, cur, oth, b, er.p, ed.p, ed2.p, zero, bin, s);
        if (res != cur) std::swap(cur, oth);
        zero = false;
      }
      continue;
    }
    const int sp = ams_subspace(ch);
    if (sp < 0) fail(EMG_ERR_OPTION, "bad AMS cycle character '%c'", ch);
    const T *tg = sp == 0 ? nullptr : tangent.p;
    if (sp == 0) {
      // gradient space: G^T (b - B x) = G^T b - (G^T B) x
      if (zero) {
        fill_zero<T>((long)ne * K, cur, s);
        ams_restrict<T>(nv, K, 0, inc_rp, inc, nullptr, b, wb[0][0].p, s);
        zero = false;
      } else {
        ams_restrict<T>(nv, K, 0, inc_rp, inc, nullptr, b, gtmp.p, s);
        SpmmArgs a;
        std::memset(&a, 0, sizeof(a));
        a.n = nv;
        a.rp = grp;
        a.ci = gci;
        a.vc = gvc.p;
        a.vm = two ? (const void *)gvm.p : nullptr;
        a.l1c = a.l1m = nullptr;
        a.omega = omega.p;
        a.x = cur;
        a.b = gtmp.p;
        a.y = wb[0][0].p;
        a.relax_w = 1.0;
        a.mode = SPMM_RES;
        a.r = a.d = nullptr;
        a.c1 = a.c2 = 0;
        const TiledPattern *tp = gtb_tiles();
        if (tp) spmm_tiled<T>(K, a, *tp, s);
        else spmm_nnz<T>(K, a, nnzG, s);
      }
    } else {
      if (zero) {
        fill_zero<T>((long)ne * K, cur, s);
        EMG_CUDA(cudaMemcpyAsync(er.p, b, sizeof(T) * (size_t)ne * K, cudaMemcpyDeviceToDevice, s));
        zero = false;
      } else {
        spmm_B(SPMM_RES, cur, b, er.p, s);
      }
      ams_restrict<T>(nv, K, sp, inc_rp, inc, tg, er.p, wb[sp][0].p, s);
    }
    run_vcycle(sp, s);
    // split form: the closing gradient correction stays a vertex potential
    // (wx[0][0]); the caller adds G phi in higher precision
    if (split_gradient && sp == 0 && ci + 1 == cycle.size()) continue;
    ams_prolong_add<T>(ne, K, sp, edges, tg, wx[sp][0].p, cur, s);
  }
  if (cur != x) EMG_CUDA(cudaMemcpyAsync(x, cur, sizeof(T) * (size_t)ne * K, cudaMemcpyDeviceToDevice, s));
  if (fused && h_ferr.p) EMG_CUDA(cudaMemcpyAsync(h_ferr.p, ferr.p, sizeof(int), cudaMemcpyDeviceToHost, s));
}

template <typename T>
size_t Ams<T>::device_bytes() const {
  size_t b = B.vc.bytes() + B.vm.bytes() + B.l1c.bytes() + B.l1m.bytes() + tangent.bytes();
  for (int sp = 0; sp < NSUB; ++sp)
    for (auto &l : sub[sp].lv)
      b += l.A.rp.bytes() + l.A.ci.bytes() + l.A.vc.bytes() + l.A.vm.bytes() + l.P.rp.bytes() + l.P.ci.bytes() +
           l.P.vc.bytes() + l.R.rp.bytes() + l.R.ci.bytes() + l.R.vc.bytes();
  return b;
}

// ---------------------------------------------------------------------------
// batched FCG
// ---------------------------------------------------------------------------
template <typename T>
int Fcg<T>::solve(Ams<T> &ams, const T *b, T *x, double rtol, int maxit, cudaStream_t s) {
  return solve_with(
      ams.ne, ams.K, [&](const T *r_, T *z_) { ams.apply(r_, z_, s); },
      [&](const T *p_, T *s_) { ams.spmm_B(SPMM_AX, p_, nullptr, s_, s); }, b, x, rtol, maxit, s);
}

// device-side column bookkeeping of the batched FCG: no host round trip per
// iteration
__global__ void fcg_init_kernel(int K, const double *__restrict__ bn, int *__restrict__ act, int *__restrict__ its,
                                int *__restrict__ status) {
  const int c = threadIdx.x;
  if (c < K) {
    act[c] = bn[c] > 0.0;
    its[c] = 0;
  }
  if (c == 0) status[0] = status[1] = 0;
}

// after an update: count the iteration of every active column, retire the
// converged ones (||r_c||^2 <= rtol^2 ||b_c||^2), flag NaN/Inf; status[0] =
// active columns left, status[1] = 1 + the first non-finite column (0: none)
__global__ void fcg_status_kernel(int K, const double *__restrict__ rn, const double *__restrict__ bn, double rtol2,
                                  int *__restrict__ act, int *__restrict__ its, int *__restrict__ status) {
  const int c = threadIdx.x;
  int a = 0;
  if (c < K && act[c]) {
    its[c]++;
    const double v = rn[c];
    if (!isfinite(v)) {
      atomicCAS(status + 1, 0, c + 1);
      act[c] = 0;
    } else if (v <= rtol2 * bn[c]) {
      act[c] = 0;
    } else {
      a = 1;
    }
  }
  const int n = __syncthreads_count(a);
  if (c == 0) status[0] = n;
}

template <typename T>
int Fcg<T>::solve_with(int n, int Kc, const std::function<void(const T *, T *)> &pc,
                       const std::function<void(const T *, T *)> &opB, const T *b, T *x, double rtol, int maxit,
                       cudaStream_t s, float *r32, const ZSplit *zs) {
  K = Kc;
  if (zs && (sizeof(T) != 8 || mmax > 4)) fail(EMG_ERR_STATE, "split z needs FP64 recurrences and at most 4 directions");
  const size_t N = (size_t)n * K;
  if (mmax < 1) mmax = 1;
  if (K > 1024) fail(EMG_ERR_ARG, "batched FCG supports at most 1024 columns");
  r.alloc(N);
  z.alloc(N);
  bool new_ring = false;
  if ((int)P.size() != mmax || P.empty() || P[0].n != N) {
    P.clear();
    S.clear();
    P.resize(mmax);
    S.resize(mmax);
    for (int j = 0; j < mmax; ++j) {
      P[j].alloc(N);
      S[j].alloc(N);
    }
    new_ring = true;
  }
  dots.alloc((size_t)(mmax + 3) * K);
  eta.alloc((size_t)mmax * K);
  eord.alloc((size_t)mmax * K);
  alpha.alloc(K);
  beta.alloc((size_t)mmax * K);
  rn.alloc(K);
  bn.alloc(K);
  act.alloc(K);
  itsd.alloc(K);
  status.alloc(2);
  if (!h_status.p) EMG_CUDA(cudaMallocHost((void **)&h_status.p, 2 * sizeof(int)));
  // ring orderings: for (head, nprev) the previous directions oldest first
  if (new_ring || ptab_mmax != mmax || ptrs.n != (size_t)mmax * (mmax + 1) * mmax) {
    std::vector<T *> tab((size_t)mmax * (mmax + 1) * mmax, nullptr);
    for (int h = 0; h < mmax; ++h)
      for (int np = 1; np <= mmax; ++np)
        for (int j = 0; j < np; ++j) tab[((size_t)h * (mmax + 1) + np) * mmax + j] = P[(h - np + j + mmax) % mmax].p;
    ptrs.upload(tab, s);
    EMG_CUDA(cudaStreamSynchronize(s));
    ptab_mmax = mmax;
  }
  its.assign(K, 0);
  fill_zero<T>((long)N, x, s);
  EMG_CUDA(cudaMemcpyAsync(r.p, b, sizeof(T) * N, cudaMemcpyDeviceToDevice, s));
  if (r32) {
    if (sizeof(T) != 8) fail(EMG_ERR_STATE, "FP32 residual copy needs FP64 recurrences");
    cvt_d2f((long)N, reinterpret_cast<const double *>(b), r32, s);
  }
  bn.zero(s);
  coldot<T>(n, K, b, b, bn.p, s);
  fcg_init_kernel<<<1, 1024, 0, s>>>(K, bn.p, act.p, itsd.p, status.p);
  EMG_LAUNCH_CHECK();
  const int every = std::max(1, check_every);
  int nprev = 0, head = 0, it = 0;
  for (it = 0; it < maxit; ++it) {
    pc(r.p, z.p);
    if (zs) {
      // z = x + G phi only inside these two passes
      if (nprev > 0) {
        EMG_CUDA(cudaMemsetAsync(dots.p, 0, sizeof(double) * nprev * K, s));
        DevPtrs4 Sj{{nullptr, nullptr, nullptr, nullptr}};
        for (int j = 0; j < nprev; ++j) {
          const int sl = (head - nprev + j + mmax) % mmax;
          Sj.p[j] = reinterpret_cast<const double *>(S[sl].p);
          EMG_CUDA(cudaMemcpyAsync(eord.p + (size_t)j * K, eta.p + (size_t)sl * K, sizeof(double) * K,
                                   cudaMemcpyDeviceToDevice, s));
        }
        zsplit_dots(n, K, zs->edges, zs->x, zs->phi, nprev, Sj, dots.p, s);
        fcg_beta_kernel<<<(nprev * K + 127) / 128, 128, 0, s>>>(K, nprev, dots.p, eord.p, act.p, beta.p);
        EMG_LAUNCH_CHECK();
      }
      zsplit_direction(n, K, zs->edges, zs->x, zs->phi, nprev,
                       reinterpret_cast<double *const *>(ptrs.p + ((size_t)head * (mmax + 1) + nprev) * mmax),
                       beta.p, reinterpret_cast<double *>(P[head].p), s);
    } else if (nprev > 0) {
      EMG_CUDA(cudaMemsetAsync(dots.p, 0, sizeof(double) * nprev * K, s));
      for (int j = 0; j < nprev; ++j) {
        const int sl = (head - nprev + j + mmax) % mmax;
        coldot<T>(n, K, z.p, S[sl].p, dots.p + (size_t)j * K, s);
        // eta of the ring slots in the same order
        EMG_CUDA(cudaMemcpyAsync(eord.p + (size_t)j * K, eta.p + (size_t)sl * K, sizeof(double) * K,
                                 cudaMemcpyDeviceToDevice, s));
      }
      fcg_beta_kernel<<<(nprev * K + 127) / 128, 128, 0, s>>>(K, nprev, dots.p, eord.p, act.p, beta.p);
      EMG_LAUNCH_CHECK();
      fcg_direction<T>(n, K, z.p, nprev, ptrs.p + ((size_t)head * (mmax + 1) + nprev) * mmax, beta.p, P[head].p,
                       s);
    } else {
      EMG_CUDA(cudaMemcpyAsync(P[head].p, z.p, sizeof(T) * N, cudaMemcpyDeviceToDevice, s));
    }
    T *p = P[head].p;
    T *sv = S[head].p;
    opB(p, sv);
    EMG_CUDA(cudaMemsetAsync(dots.p, 0, sizeof(double) * 2 * K, s));
    coldot3<T>(n, K, p, sv, p, r.p, nullptr, nullptr, dots.p, s);
    fcg_alpha_kernel<<<(K + 63) / 64, 64, 0, s>>>(K, dots.p, eta.p + (size_t)head * K, act.p, alpha.p);
    EMG_LAUNCH_CHECK();
    rn.zero(s);
    fcg_update<T>(n, K, alpha.p, p, sv, x, r.p, rn.p, s, r32);
    fcg_status_kernel<<<1, 1024, 0, s>>>(K, rn.p, bn.p, rtol * rtol, act.p, itsd.p, status.p);
    EMG_LAUNCH_CHECK();
    head = (head + 1) % mmax;
    nprev = std::min(nprev + 1, mmax);
    // the host looks at the column status only every `every` iterations (and
    // at the cap); columns that converged in between stay frozen (alpha = beta
    // = 0 keeps x and r)
    if (verbose || (it + 1) % every == 0 || it + 1 == maxit) {
      EMG_CUDA(cudaMemcpyAsync(h_status.p, status.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
      EMG_CUDA(cudaStreamSynchronize(s));
      if (verbose) {
        std::vector<double> ha(K), hrn(K), hbn(K);
        alpha.download(ha.data(), K, s);
        rn.download(hrn.data(), K, s);
        bn.download(hbn.data(), K, s);
        EMG_CUDA(cudaStreamSynchronize(s));
        fprintf(stderr, "fcg it %d:", it);
        for (int c = 0; c < K; ++c)
          fprintf(stderr, " [%d a=%.3e r=%.3e]", c, ha[c], std::sqrt(hrn[c] / std::max(hbn[c], 1e-300)));
        fprintf(stderr, "\n");
      }
      if (h_status.p[1]) fail(EMG_DIVERGED_NANORINF, "inner FCG: NaN or Inf in the residual of column %d",
                              h_status.p[1] - 1);
      if (h_status.p[0] == 0) {
        ++it;
        break;
      }
    }
  }
  itsd.download(its.data(), K, s);
  EMG_CUDA(cudaStreamSynchronize(s));
  long tot = 0;
  for (int c = 0; c < K; ++c) tot += its[c];
  total_its += tot;
  return it;
}

// ---------------------------------------------------------------------------
// batched FGMRES (FP64)
// ---------------------------------------------------------------------------
typedef std::complex<double> zc;

// x[:, c] *= keep[c] on an n x K complex block
__global__ void column_mask_kernel(long n, int K, const double *__restrict__ keep, double2 *__restrict__ x) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n * K) return;
  const double m = keep[i % K];
  if (m != 1.0) {
    double2 v = x[i];
    x[i] = make_double2(v.x * m, v.y * m);
  }
}

// Per-column Arnoldi bookkeeping of the block FGMRES on the device (one
// thread per column): the Hessenberg columns, Givens rotations and the
// rotated right-hand side g stay in device memory; the host reads two status
// words per step (columns still iterating, NaN flag).
struct GmDev {
  double2 *H;      // K x (J+1) x J
  double2 *cs, *sn;  // K x J
  double2 *g;      // K x (J+1)
  int *done, *jc, *colits, *conv;
  const double *bnorm;
  double *scale;   // K: divisor of the next basis vector (0: column finished)
  int *status;     // [0] columns still iterating, [1] 1 + first column with NaN/Inf
  const double *tol;  // K: absolute stopping tolerance of the residual norm
};

// per column: tol = max(rtol ||b||, u || |b| + |A| |x| ||), u the FP64 unit
// roundoff; below the second term the computed residual is rounding noise
__global__ void gm_tol_kernel(int K, double rtol, const double *__restrict__ bnorm,
                              const double *__restrict__ bound2, double *__restrict__ tol) {
  const int c = threadIdx.x;
  if (c < K) tol[c] = fmax(rtol * bnorm[c], 0x1p-53 * sqrt(bound2[c]));
}

__device__ __forceinline__ double2 zmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 zconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double zabs(double2 a) { return hypot(a.x, a.y); }

// start of a restart cycle: nrm2[c] = ||b - A x||^2.  stall > 0: a column
// whose residual fell by less than that factor over the last cycle stops
// iterating (it leaves unconverged, for a caller with a stronger
// preconditioner to finish)
__global__ void gm_start_kernel(int K, int J, const double *__restrict__ nrm2, double rtol, double stall,
                                double *__restrict__ prev, GmDev st) {
  const int c = threadIdx.x;
  int act = 0;
  if (c < K) {
    const double beta = sqrt(nrm2[c]);
    if (!isfinite(beta)) atomicCAS(st.status + 1, 0, c + 1);
    if (beta <= st.tol[c]) st.conv[c] = 1;
    if (stall > 0 && prev[c] > 0 && beta > stall * prev[c]) st.conv[c] = 1;
    prev[c] = beta;
    const bool cv = st.conv[c] != 0 || !isfinite(beta);
    for (int i = 0; i <= J; ++i) st.g[(long)c * (J + 1) + i] = make_double2(0, 0);
    st.g[(long)c * (J + 1)] = make_double2(cv ? 0.0 : beta, 0.0);
    st.done[c] = cv;
    st.jc[c] = 0;
    st.scale[c] = cv ? 0.0 : beta;
    act = !cv;
  }
  const int n = __syncthreads_count(act);
  if (c == 0) st.status[0] = n;
}

__global__ void zero_imag_kernel(int n, double *__restrict__ h) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) h[2 * i + 1] = 0.0;
}

// step j: h[i*K + c] (i <= j) = V_i^H w, hn[c] = ||w - sum h_i V_i||^2
__global__ void gm_givens_kernel(int K, int J, int j, const double2 *__restrict__ h, const double *__restrict__ hn,
                                 double rtol, GmDev st) {
  const int c = threadIdx.x;
  int act = 0;
  if (c < K) {
    const double hnext = sqrt(fmax(0.0, hn[c]));
    if (!isfinite(hnext)) atomicCAS(st.status + 1, 0, c + 1);
    st.scale[c] = isfinite(hnext) ? hnext : 0.0;
    if (!st.done[c]) {
      double2 *Hc = st.H + (long)c * (J + 1) * J;
      double2 *cs = st.cs + (long)c * J, *sn = st.sn + (long)c * J, *g = st.g + (long)c * (J + 1);
      for (int i = 0; i <= j; ++i) Hc[i * J + j] = h[i * K + c];
      Hc[(j + 1) * J + j] = make_double2(hnext, 0.0);
      for (int i = 0; i < j; ++i) {
        const double2 a = Hc[i * J + j], b = Hc[(i + 1) * J + j];
        const double2 t0 = zmul(cs[i], a), t1 = zmul(sn[i], b);
        const double2 u0 = zmul(zconj(sn[i]), a), u1 = zmul(cs[i], b);
        Hc[i * J + j] = make_double2(t0.x + t1.x, t0.y + t1.y);
        Hc[(i + 1) * J + j] = make_double2(u1.x - u0.x, u1.y - u0.y);
      }
      const double2 a = Hc[j * J + j], b = Hc[(j + 1) * J + j];
      const double aa = zabs(a);
      const double rho = sqrt(a.x * a.x + a.y * a.y + b.x * b.x + b.y * b.y);
      if (aa == 0.0) {
        cs[j] = make_double2(0, 0);
        sn[j] = make_double2(1, 0);
      } else {
        cs[j] = make_double2(aa / rho, 0);
        const double2 ph = make_double2(a.x / aa, a.y / aa);
        const double2 t = zmul(ph, zconj(b));
        sn[j] = make_double2(t.x / rho, t.y / rho);
      }
      const double2 t0 = zmul(cs[j], a), t1 = zmul(sn[j], b);
      Hc[j * J + j] = make_double2(t0.x + t1.x, t0.y + t1.y);
      Hc[(j + 1) * J + j] = make_double2(0, 0);
      const double2 gj = g[j];
      const double2 gn = zmul(zconj(sn[j]), gj);
      g[j + 1] = make_double2(-gn.x, -gn.y);
      g[j] = zmul(cs[j], gj);
      st.jc[c] = j + 1;
      st.colits[c]++;
      if (zabs(g[j + 1]) <= st.tol[c] || hnext == 0.0 || !isfinite(hnext)) st.done[c] = 1;
      act = !st.done[c];
    }
  }
  const int n = __syncthreads_count(act);
  if (c == 0) st.status[0] = n;
}

// least-squares solutions of the cycle: y[i*K + c] (complex), zero past jc[c]
__global__ void gm_lsq_kernel(int K, int J, int m, int real_form, GmDev st, double2 *__restrict__ y) {
  const int c = threadIdx.x;
  if (c >= K) return;
  const double2 *Hc = st.H + (long)c * (J + 1) * J;
  const double2 *g = st.g + (long)c * (J + 1);
  const int mc = st.jc[c];
  for (int i = m - 1; i >= 0; --i) {
    if (i >= mc) {
      y[i * K + c] = make_double2(0, 0);
      continue;
    }
    double2 v = g[i];
    for (int q = i + 1; q < mc; ++q) {
      const double2 t = zmul(Hc[i * J + q], y[q * K + c]);
      v.x -= t.x;
      v.y -= t.y;
    }
    const double2 d = Hc[i * J + i];
    const double dd = d.x * d.x + d.y * d.y;
    double2 r = make_double2((v.x * d.x + v.y * d.y) / dd, (v.y * d.x - v.x * d.y) / dd);
    if (real_form) r.y = 0.0;
    y[i * K + c] = r;
  }
}

// Dirichlet rows of A are diagonal (their off-diagonal C and all of Ms are
// zeroed at assembly), so the exact solution's boundary values are
// b_e / C_ee: a guess takes them from the right-hand side
__global__ void guess_boundary_kernel(int ne, int k, const int *__restrict__ rp, const int *__restrict__ ci,
                                      const double *__restrict__ cv, const unsigned char *__restrict__ ebdr,
                                      const double2 *__restrict__ b, double2 *__restrict__ x) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne || !ebdr[e]) return;
  double d = 0;
  for (int q = rp[e]; q < rp[e + 1]; ++q)
    if (ci[q] == e) {
      d = cv[q];
      break;
    }
  if (d == 0) return;
  for (int j = 0; j < k; ++j) {
    const double2 v = b[(long)e * k + j];
    x[(long)e * k + j] = make_double2(v.x / d, v.y / d);
  }
}

int Fgmres::solve(Context &c, const double *b, double *x, bool use_guess, double rtol, int maxit, bool real_form,
                  const std::function<void(const double *, double *)> &precond, SolveStats &st) {
  cudaStream_t s = c.stream;
  n = c.ne;
  const int J = restart;
  if (J < 1 || J > 128) fail(EMG_ERR_ARG, "FGMRES restart must be in 1..128");
  if (k > 1024) fail(EMG_ERR_ARG, "block FGMRES supports at most 1024 columns");
  const size_t N2 = (size_t)n * k * 2;  // doubles per block vector
  V.alloc(N2 * (J + 1));
  Z.alloc(N2 * J);
  w.alloc(N2);
  r.alloc(N2);
  h.alloc((size_t)(J + 1) * k * 2);
  hn.alloc(k);
  scale.alloc(k);
  y.alloc((size_t)J * k * 2);
  nrm.alloc(k);
  bnd.alloc(k);
  Hd.alloc((size_t)k * (J + 1) * J * 2);
  csd.alloc((size_t)k * J * 2);
  snd.alloc((size_t)k * J * 2);
  gd.alloc((size_t)k * (J + 1) * 2);
  ints.alloc((size_t)4 * k + 2);
  tol.alloc(k);
  bound2.alloc(k);
  const bool use_floor = floor_stop && !real_form;
  if (!h_status.p) EMG_CUDA(cudaMallocHost((void **)&h_status.p, 2 * sizeof(int)));
  GmDev gs;
  gs.H = (double2 *)Hd.p;
  gs.cs = (double2 *)csd.p;
  gs.sn = (double2 *)snd.p;
  gs.g = (double2 *)gd.p;
  gs.done = ints.p;
  gs.jc = ints.p + k;
  gs.colits = ints.p + 2 * k;
  gs.conv = ints.p + 3 * k;
  gs.status = ints.p + 4 * k;
  gs.bnorm = bnd.p;
  gs.scale = scale.p;
  gs.tol = tol.p;
  ints.zero(s);
  prevb.alloc(k);
  prevb.zero(s);
  if (!use_guess) fill_zero<double>((long)N2, x, s);
  cudaEvent_t e0, e1;
  EMG_CUDA(cudaEventCreate(&e0));
  EMG_CUDA(cudaEventCreate(&e1));
  EMG_CUDA(cudaEventRecord(e0, s));
  std::vector<double> hb(k);
  nrm.zero(s);
  cnorm2(n, k, b, nrm.p, s);
  nrm.download(hb.data(), k, s);
  EMG_CUDA(cudaStreamSynchronize(s));
  std::vector<double> bnorm(k);
  std::vector<int> conv0(k, 0);
  for (int col = 0; col < k; ++col) {
    bnorm[col] = std::sqrt(hb[col]);
    if (bnorm[col] == 0) conv0[col] = 1;
  }
  bnd.upload(bnorm, s);
  {
    std::vector<double> t0(k);
    for (int col = 0; col < k; ++col) t0[col] = rtol * bnorm[col];
    tol.upload(t0, s);
  }
  EMG_CUDA(cudaMemcpyAsync(gs.conv, conv0.data(), sizeof(int) * k, cudaMemcpyHostToDevice, s));
  st.initial_res.assign(k, 1.0);
  if (use_guess) {
    if (!real_form) {
      guess_boundary_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, k, c.rp.p, c.ci.p, c.Cv.p, c.ebdr.p,
                                                                        (const double2 *)b, (double2 *)x);
      EMG_LAUNCH_CHECK();
    }
    // the residual judges the guess: a column whose guess leaves a larger
    // residual than zero starts from zero instead
    spmm_complex(n, k, c.rp.p, c.ci.p, c.Cv.p, c.Msv.p, omega.p, x, b, r.p, true, real_form, s);
    nrm.zero(s);
    cnorm2(n, k, r.p, nrm.p, s);
    std::vector<double> r0(k);
    nrm.download(r0.data(), k, s);
    EMG_CUDA(cudaStreamSynchronize(s));
    std::vector<double> keep(k, 1.0);
    bool drop = false;
    for (int col = 0; col < k; ++col) {
      const double rel = bnorm[col] > 0 ? std::sqrt(r0[col]) / bnorm[col] : 0.0;
      st.initial_res[col] = rel;
      if (!(rel <= 1.0)) {
        keep[col] = 0.0;
        st.initial_res[col] = 1.0;
        drop = true;
      }
    }
    if (drop) {
      scale.upload(keep, s);
      column_mask_kernel<<<(unsigned)(((long)n * k + 255) / 256), 256, 0, s>>>((long)n, k, scale.p, (double2 *)x);
      EMG_LAUNCH_CHECK();
    }
  }
  int total = 0;
  auto read_status = [&]() {
    EMG_CUDA(cudaMemcpyAsync(h_status.p, gs.status, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
    EMG_CUDA(cudaStreamSynchronize(s));
    if (h_status.p[1]) fail(EMG_DIVERGED_NANORINF, "FGMRES: NaN or Inf in the residual of column %d", h_status.p[1] - 1);
    return h_status.p[0];
  };
  auto floor_scale = [&]() {
    bound2.zero(s);
    abs_bound2(n, k, c.rp.p, c.ci.p, c.Cv.p, c.Msv.p, omega.p, x, b, bound2.p, s);
  };
  while (total < maxit) {
    spmm_complex(n, k, c.rp.p, c.ci.p, c.Cv.p, c.Msv.p, omega.p, x, b, r.p, true, real_form, s);
    nrm.zero(s);
    cnorm2(n, k, r.p, nrm.p, s);
    if (use_floor) {
      floor_scale();
      gm_tol_kernel<<<1, 1024, 0, s>>>(k, rtol, bnd.p, bound2.p, tol.p);
      EMG_LAUNCH_CHECK();
    }
    gm_start_kernel<<<1, 1024, 0, s>>>(k, J, nrm.p, rtol, stall_factor, prevb.p, gs);
    EMG_LAUNCH_CHECK();
    if (read_status() == 0) break;
    cscale(n, k, r.p, scale.p, V.p, s);
    int j;
    for (j = 0; j < J && total < maxit; ++j) {
      double *Vj = V.p + N2 * j;
      double *Zj = Z.p + N2 * j;
      precond(Vj, Zj);
      spmm_complex(n, k, c.rp.p, c.ci.p, c.Cv.p, c.Msv.p, omega.p, Zj, nullptr, w.p, false, real_form, s);
      cmultidot(n, k, j + 1, V.p, (long)N2, w.p, h.p, nullptr, 0, s);
      if (real_form) {
        zero_imag_kernel<<<((j + 1) * k + 255) / 256, 256, 0, s>>>((j + 1) * k, h.p);
        EMG_LAUNCH_CHECK();
      }
      cgs_update(n, k, j + 1, V.p, (long)N2, h.p, w.p, hn.p, s);
      gm_givens_kernel<<<1, 1024, 0, s>>>(k, J, j, (const double2 *)h.p, hn.p, rtol, gs);
      EMG_LAUNCH_CHECK();
      cscale(n, k, w.p, scale.p, V.p + N2 * (j + 1), s);
      ++total;
      // one status read per step: a further step would cost a whole inner
      // solve, far more than waiting for two words
      if (read_status() == 0) {
        ++j;
        break;
      }
    }
    if (j > 0) {
      gm_lsq_kernel<<<1, 1024, 0, s>>>(k, J, j, real_form ? 1 : 0, gs, (double2 *)y.p);
      EMG_LAUNCH_CHECK();
      cupdate(n, k, j, Z.p, (long)N2, y.p, x, s);
    }
  }
  // true residual in FP64
  spmm_complex(n, k, c.rp.p, c.ci.p, c.Cv.p, c.Msv.p, omega.p, x, b, r.p, true, real_form, s);
  nrm.zero(s);
  cnorm2(n, k, r.p, nrm.p, s);
  std::vector<double> tr(k), fb(k, 0.0);
  nrm.download(tr.data(), k, s);
  if (use_floor) {
    floor_scale();
    bound2.download(fb.data(), k, s);
  }
  st.col_its.assign(k, 0);
  EMG_CUDA(cudaMemcpyAsync(st.col_its.data(), gs.colits, sizeof(int) * k, cudaMemcpyDeviceToHost, s));
  EMG_CUDA(cudaEventRecord(e1, s));
  EMG_CUDA(cudaEventSynchronize(e1));
  float ms = 0;
  EMG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  EMG_CUDA(cudaEventDestroy(e0));
  EMG_CUDA(cudaEventDestroy(e1));
  st.seconds = ms * 1e-3;
  st.true_res.assign(k, 0.0);
  st.converged.assign(k, 0);
  st.floor_res.assign(k, 0.0);
  st.at_floor.assign(k, 0);
  for (int col = 0; col < k; ++col) {
    st.true_res[col] = bnorm[col] > 0 ? std::sqrt(tr[col]) / bnorm[col] : 0.0;
    st.converged[col] = st.true_res[col] <= rtol * 1.0000001 || bnorm[col] == 0 ? 1 : 0;
    st.floor_res[col] = bnorm[col] > 0 ? 0x1p-53 * std::sqrt(fb[col]) / bnorm[col] : 0.0;
    // above rtol but within twice the rounding floor: no iteration can do better
    st.at_floor[col] = !st.converged[col] && use_floor && st.true_res[col] <= 2.0 * st.floor_res[col] ? 1 : 0;
  }
  st.outer_its = total;
  return total;
}

// per level of subspace sp's nodal hierarchy (built on the device or on the
// host from the context's assembled operators): rows, nonzeros of A and P,
// sums of |A| (both parts) and |P|; the coarsest operator adds a last row
void amg_levels_report(Context &c, int sp, bool gpu, double w_ref, std::vector<double> &out) {
  cudaStream_t s = c.stream;
  AmgParams prm;
  prm.theta = c.opt.amg_theta;
  prm.pmax = c.opt.amg_pmax;
  prm.max_coarse = c.opt.amg_max_coarse;
  prm.max_levels = c.opt.amg_max_levels;
  prm.seed = prm.seed + 7919ull * (uint64_t)sp;
  prm.num_functions = sp == SUB_PIVEC ? 3 : 1;
  std::vector<HCsr> As, Ps;
  if (gpu) {
    DBuf<double> parts;
    assemble_nodal_device(c, parts);
    GCsr A0;
    nodal_operator_gpu(c, parts, sp, A0, -1.0);
    std::vector<GpuLevel> glv;
    GCsr gco;
    amg_build_gpu(std::move(A0), w_ref, prm, glv, gco, s);
    for (auto &L : glv) {
      As.emplace_back();
      Ps.emplace_back();
      gcsr_to_host(L.A, As.back(), s);
      gcsr_to_host(L.P, Ps.back(), s);
    }
    As.emplace_back();
    gcsr_to_host(gco, As.back(), s);
  } else {
    HCsr nod[NSUB];
    assemble_nodal(c, nod);
    if (sp == SUB_PIVEC) interleave_components(nod + 1, nod[SUB_PIVEC]);
    HostAmg h;
    amg_build(std::move(nod[sp]), w_ref, prm, h);
    for (auto &L : h.lv) {
      As.push_back(std::move(L.A));
      Ps.push_back(std::move(L.P));
    }
    As.push_back(std::move(h.coarse));
  }
  out.clear();
  for (size_t l = 0; l < As.size(); ++l) {
    const HCsr &A = As[l];
    double sa = 0, sp_ = 0;
    for (long k = 0; k < A.nnz(); ++k) sa += std::fabs(A.vc[k]) + (A.vm.empty() ? 0.0 : std::fabs(A.vm[k]));
    long np = 0;
    if (l < Ps.size()) {
      np = Ps[l].nnz();
      for (long k = 0; k < np; ++k) sp_ += std::fabs(Ps[l].vc[k]);
    }
    out.insert(out.end(), {(double)A.n, (double)A.nnz(), (double)np, sa, sp_});
  }
}

template void ams_setup<float>(Context &, Ams<float> &, bool, double, double);
template void ams_setup<double>(Context &, Ams<double> &, bool, double, double);
template struct Ams<float>;
template struct Ams<double>;
template struct Fcg<float>;
template struct Fcg<double>;

}  // namespace emg
