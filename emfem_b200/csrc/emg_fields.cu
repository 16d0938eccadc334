// Receiver fields and point-source right-hand sides for block columns on the
// device.
//
// interpolate_fields (src/em_fwd.cc:719-744) evaluates E = sum_i e_i phi_i and
// H = -curl E / (i w mu) at the receivers from the edge solution; the reference
// reads the 6 edge values of each receiver's cell one scalar at a time
// (access_vec, src/em_la.cc:7-33).  Here one thread serves one (receiver,
// column) pair of an n x k block that stays on the device: only the k x 12
// values per receiver come back to the host.
//
// assemble_rhs_csem (src/em_fwd.cc:616-671, dipoles from divide_line_source,
// :582-614) and assemble_rhs_dual (src/em_fwd.cc:673-717) add
// c * (phi_i(y) . d) into the 6 edges of the cell around a point y: one thread
// per (point, column) entry, atomics into the zeroed block.  The host divides
// line sources and locates the points (host mesh work, as in the reference).

#include <cuda_runtime.h>

#include <array>
#include <cmath>
#include <complex>
#include <vector>

#include "emg_api.h"
#include "emg_internal.h"
#include "emg_kernels.cuh"

namespace emg {

namespace {

struct FieldArgs {
  const double *pts;
  const int *ctet, *cedge;
  const signed char *cpar;
  const double *rx;      // n x 3
  const int *rx_tet;     // n
  const double *omega;   // k
  const double2 *x;      // ne x k complex
  double *eh;            // n x k x 12
  int n, k;
};

__global__ void __launch_bounds__(128) fields_block_kernel(FieldArgs a) {
  const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (idx >= (long)a.n * a.k) return;
  const int r = (int)(idx / a.k), j = (int)(idx % a.k);
  const int t = __ldg(a.rx_tet + r);
  TetGeom g;
  load_tet_geom(a.pts, a.ctet, a.cedge, a.cpar, t, g);
  const double y[3] = {__ldg(a.rx + 3 * r), __ldg(a.rx + 3 * r + 1), __ldg(a.rx + 3 * r + 2)};
  double lam[4];
#pragma unroll
  for (int p = 0; p < 4; ++p) lam[p] = lambda_at(g, p, y);
  double er[3] = {0, 0, 0}, ei[3] = {0, 0, 0}, cr[3] = {0, 0, 0}, ci[3] = {0, 0, 0};
#pragma unroll
  for (int e = 0; e < 6; ++e) {
    const int p = kEdgeP(e), q = kEdgeQ(e);
    const double2 u = __ldg(a.x + (long)g.ge[e] * a.k + j);
    double phi[3], cu[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) phi[d] = lam[p] * g.gr[q][d] - lam[q] * g.gr[p][d];
    cu[0] = 2.0 * (g.gr[p][1] * g.gr[q][2] - g.gr[p][2] * g.gr[q][1]);
    cu[1] = 2.0 * (g.gr[p][2] * g.gr[q][0] - g.gr[p][0] * g.gr[q][2]);
    cu[2] = 2.0 * (g.gr[p][0] * g.gr[q][1] - g.gr[p][1] * g.gr[q][0]);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      er[d] += u.x * phi[d];
      ei[d] += u.y * phi[d];
      cr[d] += u.x * cu[d];
      ci[d] += u.y * cu[d];
    }
  }
  // H = -curl E / (i w mu) = (i / (w mu)) curl E
  const double s = 1.0 / (__ldg(a.omega + j) * MU);
  double *o = a.eh + 12 * idx;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    o[2 * d] = er[d];
    o[2 * d + 1] = ei[d];
    o[6 + 2 * d] = -s * ci[d];
    o[6 + 2 * d + 1] = s * cr[d];
  }
}

// one point-source entry: s[ge_i, col] += coef * (phi_i(y) . dir) for the six
// edges of tet t
struct PointSource {
  double y[3], dir[3];
  double cre, cim;
  int tet, col;
};

__global__ void __launch_bounds__(128) point_source_kernel(const double *pts, const int *ctet, const int *cedge,
                                                           const signed char *cpar, const PointSource *src, int ns,
                                                           int k, double *s) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ns) return;
  const PointSource ps = src[i];
  TetGeom g;
  load_tet_geom(pts, ctet, cedge, cpar, ps.tet, g);
  double lam[4];
#pragma unroll
  for (int p = 0; p < 4; ++p) lam[p] = lambda_at(g, p, ps.y);
#pragma unroll
  for (int e = 0; e < 6; ++e) {
    const int p = kEdgeP(e), q = kEdgeQ(e);
    double v = 0;
#pragma unroll
    for (int d = 0; d < 3; ++d) v += (lam[p] * g.gr[q][d] - lam[q] * g.gr[p][d]) * ps.dir[d];
    double *o = s + 2 * ((long)g.ge[e] * k + ps.col);
    atomicAdd(o, ps.cre * v);
    atomicAdd(o + 1, ps.cim * v);
  }
}

void device_only(const Context &c) {
  need(c.device >= 0, EMG_ERR_STATE, "this entry point needs a device context (device >= 0)");
  EMG_CUDA(cudaSetDevice(c.device));
}

void launch_point_sources(Context &c, const std::vector<PointSource> &src, int k, double *s_dev) {
  EMG_CUDA(cudaMemsetAsync(s_dev, 0, sizeof(double) * 2 * (size_t)c.ne * k, c.stream));
  if (src.empty()) return;
  DBuf<PointSource> d(src.size());
  d.upload(src, c.stream);
  point_source_kernel<<<(unsigned)((src.size() + 127) / 128), 128, 0, c.stream>>>(
      c.pts.p, c.ctet.p, c.cedge.p, c.cpar.p, d.p, (int)src.size(), k, s_dev);
  EMG_LAUNCH_CHECK();
  EMG_CUDA(cudaStreamSynchronize(c.stream));  // d goes out of scope
}

}  // namespace

}  // namespace emg

using namespace emg;

extern "C" {

int emg_interpolate_fields_block_dev(emg_context *c, int k, const double *freqs, const double *x_dev, int n,
                                     const double *pts, const int *tets, double *eh) {
  EMG_API_BEGIN
  need(c && freqs && x_dev && (n == 0 || (pts && tets && eh)), EMG_ERR_ARG, "null argument");
  need(k >= 1 && n >= 0, EMG_ERR_ARG, "bad block width or receiver count");
  need(c->have_ls, EMG_ERR_STATE, "interpolate_fields before create_linear_system");
  device_only(*c);
  if (n == 0) return EMG_OK;
  for (int r = 0; r < n; ++r)
    if (tets[r] < 0 || tets[r] >= c->nt) fail(EMG_ERR_USER, "Receiver %d is not found in mesh.", r);
  std::vector<double> om(k);
  for (int j = 0; j < k; ++j) {
    need(freqs[j] > 0, EMG_ERR_ARG, "frequencies must be positive");
    om[j] = 2 * PI * freqs[j];
  }
  DBuf<double> drx, dom, deh((size_t)n * k * 12);
  DBuf<int> dt;
  drx.upload(pts, (size_t)n * 3, c->stream);
  dt.upload(tets, (size_t)n, c->stream);
  dom.upload(om, c->stream);
  FieldArgs a{c->pts.p, c->ctet.p, c->cedge.p, c->cpar.p, drx.p, dt.p, dom.p, (const double2 *)x_dev, deh.p, n, k};
  const long m = (long)n * k;
  fields_block_kernel<<<(unsigned)((m + 127) / 128), 128, 0, c->stream>>>(a);
  EMG_LAUNCH_CHECK();
  deh.download(eh, (size_t)n * k * 12, c->stream);
  EMG_CUDA(cudaStreamSynchronize(c->stream));
  EMG_API_END
}

int emg_assemble_rhs_csem_block_dev(emg_context *c, int k, const double *freqs, const double *tx, double *s_dev) {
  EMG_API_BEGIN
  need(c && freqs && tx && s_dev, EMG_ERR_ARG, "null argument");
  need(k >= 1, EMG_ERR_ARG, "bad block width");
  need(c->have_ls, EMG_ERR_STATE, "assemble_rhs_csem before create_linear_system");
  device_only(*c);
  std::vector<PointSource> src;
  std::vector<double> P;
  std::vector<int> owner;
  std::vector<PointSource> proto;
  for (int j = 0; j < k; ++j) {
    const double *t = tx + 7 * (size_t)j;
    const double omega = 2 * PI * freqs[j];
    // divide_line_source (src/em_fwd.cc:582-614)
    const double dir[3] = {std::cos(t[3] * DTOR) * std::cos(t[4] * DTOR),
                           std::sin(t[3] * DTOR) * std::cos(t[4] * DTOR), std::sin(t[4] * DTOR)};
    const double current = t[5], length = t[6];
    auto add = [&](const double y[3], double weight) {
      PointSource ps;
      for (int d = 0; d < 3; ++d) {
        ps.y[d] = y[d];
        ps.dir[d] = dir[d];
      }
      ps.cre = 0.0;
      ps.cim = omega * current * weight;
      ps.tet = -1;
      ps.col = j;
      proto.push_back(ps);
      P.insert(P.end(), y, y + 3);
    };
    if (std::fabs(length) <= 0.1) {
      add(t, 1.0);
    } else {
      const int nd = c->opt.n_tx_divisions;
      double A[3] = {t[0] - dir[0] * length / 2, t[1] - dir[1] * length / 2, t[2] - dir[2] * length / 2};
      for (int i = 0; i < nd; ++i) {
        double B[3] = {A[0] + dir[0] * length / nd, A[1] + dir[1] * length / nd, A[2] + dir[2] * length / nd};
        double M[3] = {(A[0] + B[0]) / 2, (A[1] + B[1]) / 2, (A[2] + B[2]) / 2};
        add(M, 1.0 / nd);
        for (int d = 0; d < 3; ++d) A[d] = B[d];
      }
    }
  }
  std::vector<int> cell(proto.size());
  int rc = emg_find_cell_around_point(c, (int)proto.size(), P.data(), cell.data());
  if (rc != EMG_OK) fail(rc, "%s", emg_last_error());
  for (size_t i = 0; i < proto.size(); ++i) {
    if (cell[i] < 0) fail(EMG_ERR_USER, "Transmitter %d-%d is not found in mesh.", proto[i].col, (int)i);
    proto[i].tet = cell[i];
  }
  launch_point_sources(*c, proto, k, s_dev);
  EMG_API_END
}

int emg_assemble_rhs_dual_block_dev(emg_context *c, int k, int n_rx, const double *rx, double *s_dev) {
  EMG_API_BEGIN
  need(c && (n_rx == 0 || rx) && s_dev, EMG_ERR_ARG, "null argument");
  need(k >= 1 && n_rx >= 0, EMG_ERR_ARG, "bad block width or receiver count");
  need(c->have_ls, EMG_ERR_STATE, "assemble_rhs_dual before create_linear_system");
  device_only(*c);
  std::vector<int> cell(n_rx);
  if (n_rx) {
    int rc = emg_find_cell_around_point(c, n_rx, rx, cell.data());
    if (rc != EMG_OK) fail(rc, "%s", emg_last_error());
  }
  std::vector<PointSource> src;
  src.reserve((size_t)n_rx * k);
  for (int i = 0; i < n_rx; ++i) {
    if (cell[i] < 0) fail(EMG_ERR_USER, "Receiver %d is not found in mesh.", i);
    // b_re = b_im = sum of the components of phi_j(rx) (src/em_fwd.cc:702-705)
    for (int j = 0; j < k; ++j) {
      PointSource ps;
      for (int d = 0; d < 3; ++d) {
        ps.y[d] = rx[3 * (size_t)i + d];
        ps.dir[d] = 1.0;
      }
      ps.cre = ps.cim = 1.0;
      ps.tet = cell[i];
      ps.col = j;
      src.push_back(ps);
    }
  }
  launch_point_sources(*c, src, k, s_dev);
  EMG_API_END
}

}  // extern "C"
