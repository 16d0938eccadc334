// Goal-oriented error indicator and RHS lifting kernels.
//
// estimate_error (src/em_fwd.cc:1102-1180): per tet the volume residual
//   sum_q |i w sigma e(q)|^2 jxw * R_t^2          (integrate_over_cell, :1005-1043)
// plus, per interior face, the normal-current and tangential-curl jumps
//   (sum_q |((sigma e) - (sigma_n e_n)).n|^2 jxw + |(curl e - curl e_n) x n|^2 jxw) R_f / 2
// (integrate_over_face, :1045-1100), credited in full to both tets.  A face is
// evaluated once, by the tet with the lower index and from its side, exactly
// as the reference's face_errors(t, f) >= 0 test arranges in its ascending tet
// loop; boundary faces contribute 0.  R_t, R_f are circumradii
// (src/em_mesh.h:232-274); the face rule is the reference's 3-point rule whose
// weights sum to 6x the face area (em_fe.cc:46-80).  Solutions are complex
// interleaved per edge.

#include <cuda_runtime.h>

#include <map>
#include <mutex>

#include "emg_internal.h"
#include "emg_kernels.cuh"

namespace emg {

struct EstIn {
  const double *pts;
  const int *ctet, *cedge, *attr, *tets, *nbr, *non;
  const signed char *cpar;
  const double *sig;
  int nsol;
  const double2 *sol[3];
  double omega;
};

__device__ __forceinline__ void load_coef(const EstIn &in, const TetGeom &g, int s, double ur[6], double ui[6]) {
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    double2 v = __ldg(in.sol[s] + g.ge[k]);
    ur[k] = v.x;
    ui[k] = v.y;
  }
}

// e(x) at barycentric coordinates lam (sorted-vertex order)
__device__ __forceinline__ void field_at(const TetGeom &g, const double lam[4], const double ur[6],
                                         const double ui[6], double er[3], double ei[3]) {
#pragma unroll
  for (int d = 0; d < 3; ++d) { er[d] = 0; ei[d] = 0; }
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const int p = kEdgeP(k), q = kEdgeQ(k);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      double phi = lam[p] * g.gr[q][d] - lam[q] * g.gr[p][d];
      er[d] = fma(ur[k], phi, er[d]);
      ei[d] = fma(ui[k], phi, ei[d]);
    }
  }
}

__device__ __forceinline__ void curl_of(const TetGeom &g, const double ur[6], const double ui[6], double cr[3],
                                        double ci[3]) {
#pragma unroll
  for (int d = 0; d < 3; ++d) { cr[d] = 0; ci[d] = 0; }
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const int a = kEdgeP(k), b = kEdgeQ(k);
    double cu[3] = {2.0 * (g.gr[a][1] * g.gr[b][2] - g.gr[a][2] * g.gr[b][1]),
                    2.0 * (g.gr[a][2] * g.gr[b][0] - g.gr[a][0] * g.gr[b][2]),
                    2.0 * (g.gr[a][0] * g.gr[b][1] - g.gr[a][1] * g.gr[b][0])};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      cr[d] = fma(ur[k], cu[d], cr[d]);
      ci[d] = fma(ui[k], cu[d], ci[d]);
    }
  }
}

__device__ __forceinline__ void load_sigma(const EstIn &in, int t, double s[9]) {
  const double *sg = in.sig + 9 * (long)__ldg(in.attr + t);
#pragma unroll
  for (int k = 0; k < 9; ++k) s[k] = __ldg(sg + k);
}

__device__ __forceinline__ double dist3(const double *a, const double *b) {
  double dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
  return sqrt(dx * dx + dy * dy + dz * dz);
}

__device__ __forceinline__ double sel4(int p, double a0, double a1, double a2, double a3) {
  return p == 0 ? a0 : (p == 1 ? a1 : (p == 2 ? a2 : a3));
}

// vol[s*T + t] = volume term of tet t (integrate_over_cell)
__global__ void __launch_bounds__(128) estimate_cell_kernel(EstIn in, int nt, double *__restrict__ vol) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  TetGeom g;
  load_tet_geom(in.pts, in.ctet, in.cedge, in.cpar, t, g);
  double sg[9];
  load_sigma(in, t, sg);
  // circumradius of the tet (src/em_mesh.h:232-254)
  double diam;
  {
    double a = dist3(g.x[1], g.x[2]), b = dist3(g.x[0], g.x[2]), c = dist3(g.x[0], g.x[1]);
    double aa = dist3(g.x[0], g.x[3]), bb = dist3(g.x[1], g.x[3]), cc = dist3(g.x[2], g.x[3]);
    double la = a * aa, lb = b * bb, lc = c * cc;
    double sh = 0.5 * (la + lb + lc);
    diam = sqrt(sh * (sh - la) * (sh - lb) * (sh - lc)) / (6.0 * g.vol);
  }
  const double A = 0.585410196624969, B = 0.138196601125011;
  const double jxw_c = g.vol * 6.0 / 24.0;  // det(J) * 1/24
  const double w2 = in.omega * in.omega;
#pragma unroll 1
  for (int s = 0; s < in.nsol; ++s) {
    double ur[6], ui[6];
    load_coef(in, g, s, ur, ui);
    double res = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      double lam[4];
#pragma unroll
      for (int p = 0; p < 4; ++p) lam[p] = (p == q) ? A : B;
      double er[3], ei[3];
      field_at(g, lam, ur, ui, er, ei);
      double sq = 0;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        double yr = sg[3 * d] * er[0] + sg[3 * d + 1] * er[1] + sg[3 * d + 2] * er[2];
        double yi = sg[3 * d] * ei[0] + sg[3 * d + 1] * ei[1] + sg[3 * d + 2] * ei[2];
        sq += w2 * (yr * yr + yi * yi);
      }
      res += sq * jxw_c;
    }
    vol[(long)s * nt + t] = res * diam * diam;
  }
}

// fe[(s*T + t)*4 + f]: face f (input index) of tet t, evaluated by the lower
// of the two tets (integrate_over_face)
__global__ void __launch_bounds__(128) estimate_face_kernel(EstIn in, int nt, double *__restrict__ fe) {
  const long id = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (id >= (long)nt * 4) return;
  const int t = (int)(id >> 2), f = (int)(id & 3);
  const int n = __ldg(in.nbr + id);
  if (n < 0) {
    for (int s = 0; s < in.nsol; ++s) fe[((long)s * nt + t) * 4 + f] = 0.0;
    return;
  }
  if (n < t) return;  // the neighbour evaluates this face
  const int non = __ldg(in.non + id);
  TetGeom g;
  load_tet_geom(in.pts, in.ctet, in.cedge, in.cpar, t, g);
  // sorted position of the vertex opposite face f
  const int vf = __ldg(in.tets + 4 * (long)t + f);
  const int p = vf == g.v[0] ? 0 : (vf == g.v[1] ? 1 : (vf == g.v[2] ? 2 : 3));
  double sg[9];
  load_sigma(in, t, sg);
  // outward normal -grad(l_p)/|grad(l_p)| and the reference's face weight
  const double gx = sel4(p, g.gr[0][0], g.gr[1][0], g.gr[2][0], g.gr[3][0]);
  const double gy = sel4(p, g.gr[0][1], g.gr[1][1], g.gr[2][1], g.gr[3][1]);
  const double gz = sel4(p, g.gr[0][2], g.gr[1][2], g.gr[2][2], g.gr[3][2]);
  const double gl = sqrt(gx * gx + gy * gy + gz * gz);
  const double nrm[3] = {-gx / gl, -gy / gl, -gz / gl};
  const double jxw_f = gl * fabs(6.0 * g.vol) * 6.0 / 6.0;
  // face circumradius (src/em_mesh.h:256-274): edge lengths of the face
  double fd;
  {
    double d01 = dist3(g.x[0], g.x[1]), d02 = dist3(g.x[0], g.x[2]), d03 = dist3(g.x[0], g.x[3]);
    double d12 = dist3(g.x[1], g.x[2]), d13 = dist3(g.x[1], g.x[3]), d23 = dist3(g.x[2], g.x[3]);
    double a = sel4(p, d23, d23, d13, d12), b = sel4(p, d13, d03, d03, d02), c = sel4(p, d12, d02, d01, d01);
    double area = 0.25 * sqrt((a + b + c) * (b + c - a) * (c + a - b) * (a + b - c));
    fd = a * b * c / (4.0 * area);
  }
  TetGeom gn;
  load_tet_geom(in.pts, in.ctet, in.cedge, in.cpar, n, gn);
  double sgn[9];
  load_sigma(in, n, sgn);
#pragma unroll 1
  for (int s = 0; s < in.nsol; ++s) {
    double ur[6], ui[6], urn[6], uin[6];
    load_coef(in, g, s, ur, ui);
    load_coef(in, gn, s, urn, uin);
    double cr[3], ci[3], crn[3], cin[3];
    curl_of(g, ur, ui, cr, ci);
    curl_of(gn, urn, uin, crn, cin);
    double dr[3] = {cr[0] - crn[0], cr[1] - crn[1], cr[2] - crn[2]};
    double di[3] = {ci[0] - cin[0], ci[1] - cin[1], ci[2] - cin[2]};
    double xr0 = dr[1] * nrm[2] - dr[2] * nrm[1], xr1 = dr[2] * nrm[0] - dr[0] * nrm[2],
           xr2 = dr[0] * nrm[1] - dr[1] * nrm[0];
    double xi0 = di[1] * nrm[2] - di[2] * nrm[1], xi1 = di[2] * nrm[0] - di[0] * nrm[2],
           xi2 = di[0] * nrm[1] - di[1] * nrm[0];
    const double cross2 = xr0 * xr0 + xr1 * xr1 + xr2 * xr2 + xi0 * xi0 + xi1 * xi1 + xi2 * xi2;
    double dotj = 0, crossh = 0;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      // face vertices (p+1, p+2, p+3) mod 4 get 2/3 (rotated by q) or 1/6
      const int hot = (p + 1 + q) & 3;
      double lam[4], y[3];
#pragma unroll
      for (int i = 0; i < 4; ++i) lam[i] = (i == p) ? 0.0 : ((i == hot) ? 2.0 / 3.0 : 1.0 / 6.0);
#pragma unroll
      for (int d = 0; d < 3; ++d)
        y[d] = lam[0] * g.x[0][d] + lam[1] * g.x[1][d] + lam[2] * g.x[2][d] + lam[3] * g.x[3][d];
      double lamn[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) lamn[i] = lambda_at(gn, i, y);
      double er[3], ei[3], ern[3], ein[3];
      field_at(g, lam, ur, ui, er, ei);
      field_at(gn, lamn, urn, uin, ern, ein);
      double jr = 0, ji = 0;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        double sr = sg[3 * d] * er[0] + sg[3 * d + 1] * er[1] + sg[3 * d + 2] * er[2];
        double si = sg[3 * d] * ei[0] + sg[3 * d + 1] * ei[1] + sg[3 * d + 2] * ei[2];
        double snr = sgn[3 * d] * ern[0] + sgn[3 * d + 1] * ern[1] + sgn[3 * d + 2] * ern[2];
        double sni = sgn[3 * d] * ein[0] + sgn[3 * d + 1] * ein[1] + sgn[3 * d + 2] * ein[2];
        jr += (sr - snr) * nrm[d];
        ji += (si - sni) * nrm[d];
      }
      dotj += (jr * jr + ji * ji) * jxw_f;
      crossh += cross2 * jxw_f;
    }
    double v = (dotj + crossh) * fd / 2.0;
    fe[((long)s * nt + t) * 4 + f] = v;
    fe[((long)s * nt + n) * 4 + non] = v;
  }
}

// eta[s][t] = vol + fe[0] + fe[1] + fe[2] + fe[3] (the reference's order), then
// the primal x dual combination sqrt(eta_p * eta_d) (src/em_fwd.cc:1172-1177).
__global__ void estimate_sum_kernel(int nt, int nsol, const double *__restrict__ vol, const double *__restrict__ fe,
                                    double *__restrict__ eta) {
  long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= (long)nt * nsol) return;
  double v = vol[i];
#pragma unroll
  for (int f = 0; f < 4; ++f) v += fe[i * 4 + f];
  eta[i] = v;
}

__global__ void combine_err_kernel(int nt, int nsol, const double *__restrict__ eta, double *__restrict__ err) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  const double *dual = eta + (long)(nsol - 1) * nt;
  for (int s = 0; s < nsol - 1; ++s) err[(long)s * nt + t] = sqrt(eta[(long)s * nt + t] * dual[t]);
}

void launch_estimate(Context &c, double omega, int nsol, const double *const *sol_dev, double *eta_dev,
                     double *err_dev, double *scratch_vol, double *scratch_fe) {
  EstIn in;
  in.pts = c.pts.p;
  in.ctet = c.ctet.p;
  in.cedge = c.cedge.p;
  in.attr = c.attr.p;
  in.tets = c.tets.p;
  in.nbr = c.nbr.p;
  in.non = c.non.p;
  in.cpar = c.cpar.p;
  in.sig = c.sigma_tab.p;
  in.nsol = nsol;
  for (int s = 0; s < 3; ++s) in.sol[s] = s < nsol ? (const double2 *)sol_dev[s] : nullptr;
  in.omega = omega;
  estimate_cell_kernel<<<(unsigned)((c.nt + 127) / 128), 128, 0, c.stream>>>(in, c.nt, scratch_vol);
  EMG_LAUNCH_CHECK();
  estimate_face_kernel<<<(unsigned)(((long)c.nt * 4 + 127) / 128), 128, 0, c.stream>>>(in, c.nt, scratch_fe);
  EMG_LAUNCH_CHECK();
  long n = (long)c.nt * nsol;
  estimate_sum_kernel<<<(unsigned)((n + 255) / 256), 256, 0, c.stream>>>(c.nt, nsol, scratch_vol, scratch_fe, eta_dev);
  EMG_LAUNCH_CHECK();
  if (err_dev) {
    combine_err_kernel<<<(unsigned)((c.nt + 255) / 256), 256, 0, c.stream>>>(c.nt, nsol, eta_dev, err_dev);
    EMG_LAUNCH_CHECK();
  }
}

// ---------------------------------------------------------------------------
// MT boundary lifting (assemble_rhs_mt, src/em_fwd.cc:516-572) for k boundary
// value sets at once: bv[e*k + j] (complex) holds the Dirichlet value of
// boundary edge e for column j; out s (complex interleaved, n x k).
// ---------------------------------------------------------------------------
struct LiftIn {
  const double *pts;
  const int *ctet, *cedge, *attr;
  const signed char *cpar;
  const unsigned char *ebdr, *bdr_cell;
  const double *sig;
};

__global__ void __launch_bounds__(128) rhs_mt_kernel(LiftIn in, int nt, int k, const double *__restrict__ omega,
                                                     const double2 *__restrict__ bv, const int *__restrict__ brank,
                                                     double *__restrict__ s) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt || !__ldg(in.bdr_cell + t)) return;
  TetGeom g;
  load_tet_geom(in.pts, in.ctet, in.cedge, in.cpar, t, g);
  const double *sgp = in.sig + 9 * (long)__ldg(in.attr + t);
  double sg[9];
#pragma unroll
  for (int q = 0; q < 9; ++q) sg[q] = __ldg(sgp + q);
  double S[10];
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = p; q < 4; ++q) {
      double a0 = sg[0] * g.gr[q][0] + sg[1] * g.gr[q][1] + sg[2] * g.gr[q][2];
      double a1 = sg[3] * g.gr[q][0] + sg[4] * g.gr[q][1] + sg[5] * g.gr[q][2];
      double a2 = sg[6] * g.gr[q][0] + sg[7] * g.gr[q][1] + sg[8] * g.gr[q][2];
      S[sym_idx(p, q)] = g.gr[p][0] * a0 + g.gr[p][1] * a1 + g.gr[p][2] * a2;
    }
  double cu[6][3];
#pragma unroll
  for (int e = 0; e < 6; ++e) {
    const int a = kEdgeP(e), b = kEdgeQ(e);
    cu[e][0] = 2.0 * (g.gr[a][1] * g.gr[b][2] - g.gr[a][2] * g.gr[b][1]);
    cu[e][1] = 2.0 * (g.gr[a][2] * g.gr[b][0] - g.gr[a][0] * g.gr[b][2]);
    cu[e][2] = 2.0 * (g.gr[a][0] * g.gr[b][1] - g.gr[a][1] * g.gr[b][0]);
  }
  bool bd[6];
#pragma unroll
  for (int e = 0; e < 6; ++e) bd[e] = __ldg(in.ebdr + g.ge[e]) != 0;
  const double vc = g.vol / MU, vm = g.vol / 20.0;
  for (int j = 0; j < k; ++j) {
    const double w = __ldg(omega + j);
    double br[6] = {0, 0, 0, 0, 0, 0}, bi[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      if (!bd[i]) continue;
      double2 v = __ldg(bv + (long)__ldg(brank + g.ge[i]) * k + j);
      double cii = vc * (cu[i][0] * cu[i][0] + cu[i][1] * cu[i][1] + cu[i][2] * cu[i][2]);
      br[i] += v.x * cii;
      bi[i] += -v.y * cii;
#pragma unroll
      for (int l = 0; l < 6; ++l) {
        if (bd[l]) continue;
        const int p = kEdgeP(l), q = kEdgeQ(l), r = kEdgeP(i), u = kEdgeQ(i);
        double cli = vc * (cu[l][0] * cu[i][0] + cu[l][1] * cu[i][1] + cu[l][2] * cu[i][2]);
        double mli = w * vm *
                     ((1.0 + (p == r)) * S[sym_idx(q, u)] - (1.0 + (p == u)) * S[sym_idx(q, r)] -
                      (1.0 + (q == r)) * S[sym_idx(p, u)] + (1.0 + (q == u)) * S[sym_idx(p, r)]);
        br[l] -= cli * v.x;
        bi[l] += mli * v.x;
        br[l] += mli * v.y;
        bi[l] += cli * v.y;
      }
    }
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      atomicAdd(s + 2 * ((long)g.ge[i] * k + j), br[i]);
      atomicAdd(s + 2 * ((long)g.ge[i] * k + j) + 1, bi[i]);
    }
  }
}

void launch_rhs_mt(Context &c, int k, const double *omega_dev, const double *bv_dev, const int *brank_dev,
                   double *s_dev) {
  LiftIn in{c.pts.p, c.ctet.p, c.cedge.p, c.attr.p, c.cpar.p, c.ebdr.p, c.bdr_cell.p, c.sigma_tab.p};
  EMG_CUDA(cudaMemsetAsync(s_dev, 0, sizeof(double) * 2 * (size_t)c.ne * k, c.stream));
  rhs_mt_kernel<<<(unsigned)((c.nt + 127) / 128), 128, 0, c.stream>>>(in, c.nt, k, omega_dev, (const double2 *)bv_dev,
                                                                      brank_dev, s_dev);
  EMG_LAUNCH_CHECK();
}

}  // namespace emg

// ---------------------------------------------------------------------------
// Error estimate without any device allocation.
//
// emg_estimate_error obtains its per-tet and per-face scratch from the
// context's workspace, which the library allocates with cudaMalloc on first
// use.  Some callers cannot allow an allocation at that point -- a host
// application whose memory manager owns all device memory and forbids
// allocations once a run has started, or a caller that must not synchronise
// the device the way cudaMalloc/cudaFree can.  For them this variant keeps
// the scratch in a fixed file-scope device array and writes its results into
// device buffers the caller owns.
// ---------------------------------------------------------------------------
namespace {

constexpr int kNoAllocMaxTets = 131072;  // largest mesh the fixed scratch serves
constexpr int kNoAllocMaxSol = 3;        // MT: XY, YX and the dual solution

// volume terms (n_sol x T) followed by face terms (n_sol x T x 4): 15.7 MB,
// held on every GPU that loads the library until the process exits
__device__ __align__(256) double g_estimate_scratch[kNoAllocMaxSol * kNoAllocMaxTets * 5];

}  // namespace

namespace emg {
// In host code g_estimate_scratch only names a host-side stand-in; the device
// address is looked up once per device, with that device current.  Device
// contexts call this when they are created, which also loads this file's
// module on that device, so emg_estimate_error_noalloc itself never loads a
// module or allocates.
double *noalloc_scratch_address(int device) {
  static std::mutex mu;
  static std::map<int, double *> addr;
  std::lock_guard<std::mutex> lock(mu);
  auto it = addr.find(device);
  if (it != addr.end()) return it->second;
  double *p = nullptr;
  emg::check_cuda(cudaGetSymbolAddress((void **)&p, g_estimate_scratch), "cudaGetSymbolAddress(g_estimate_scratch)",
                  __FILE__, __LINE__);
  addr[device] = p;
  return p;
}
}  // namespace emg

extern "C" int emg_estimate_error_noalloc(emg_context *ctx, int fidx, int tidx, double *err_dev, double *eta_dev) {
  using namespace emg;
  try {
    if (!ctx || !err_dev || !eta_dev) fail(EMG_ERR_ARG, "null argument");
    Context &c = *ctx;
    if (c.device < 0) fail(EMG_ERR_STATE, "host-only context has no device");
    if (!c.have_ls || c.nrho <= 0) fail(EMG_ERR_STATE, "estimate_error before create_linear_system");
    if (fidx < 0 || fidx >= (int)c.freqs.size()) fail(EMG_ERR_ARG, "frequency index out of range");
    if (c.nt > kNoAllocMaxTets)
      fail(EMG_ERR_ARG, "emg_estimate_error_noalloc serves meshes of at most %d tets (this one has %d); "
           "use emg_estimate_error", kNoAllocMaxTets, c.nt);
    const int slots3[3] = {EMG_SOL_MT_XY, EMG_SOL_MT_YX, EMG_SOL_DUAL};
    const int slots2[2] = {EMG_SOL_CSEM, EMG_SOL_DUAL};
    const int nsol = tidx < 0 ? 3 : 2;
    const double *sp[3];
    for (int s = 0; s < nsol; ++s) {
      auto it = c.sol.find(tidx < 0 ? slots3[s] : slots2[s]);
      if (it == c.sol.end() || it->second.n != (size_t)c.ne * 2) fail(EMG_ERR_STATE, "solution slot not created");
      sp[s] = it->second.p;
    }
    check_cuda(cudaSetDevice(c.device), "cudaSetDevice", __FILE__, __LINE__);
    double *scratch = noalloc_scratch_address(c.device);
    // every volume and face entry is written before it is read, so nothing
    // left in the array by an earlier call needs clearing
    launch_estimate(c, 2 * PI * c.freqs[fidx], nsol, sp, eta_dev, err_dev, scratch, scratch + (size_t)nsol * c.nt);
    check_cuda(cudaStreamSynchronize(c.stream), "cudaStreamSynchronize", __FILE__, __LINE__);
  } catch (const Error &e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return EMG_ERR_USER;
  }
  return EMG_OK;
}
