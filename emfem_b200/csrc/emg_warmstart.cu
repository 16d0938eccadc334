// Warm start of block solves from already solved (frequency, source) columns:
// the C-ABI entry points that train the per-edge network (emg_mlp.cu) on a
// solved block and predict initial guesses for new columns.  No counterpart in
// the reference (FGMRES always starts from zero there, src/em_la.cc:49).

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <memory>
#include <vector>

#include "emg_api.h"
#include "emg_internal.h"
#include "emg_mlp.h"

namespace emg {

namespace {

WarmStartNet &net_of(Context &c) {
  if (!c.warm) c.warm = std::make_shared<WarmStartNet>();
  return *c.warm;
}

struct Column {
  double f;
  int src;
  double pos[3];
  bool point;
};

std::vector<Column> columns(int k, const double *freqs, const int *src, const double *pos) {
  std::vector<Column> c(k);
  for (int j = 0; j < k; ++j) {
    need(freqs[j] > 0, EMG_ERR_ARG, "frequencies must be positive");
    c[j].f = freqs[j];
    c[j].src = src ? src[j] : 0;
    c[j].point = pos != nullptr;
    for (int d = 0; d < 3; ++d) c[j].pos[d] = pos ? pos[3 * j + d] : 0.0;
  }
  return c;
}

// the two solved columns of the same source nearest to frequency f in log f
// (skip: a column index to leave out); false when there is none
bool neighbours(const std::vector<Column> &solved, const Column &t, int skip, Spec &sp) {
  std::vector<std::pair<double, int>> cand;
  for (int j = 0; j < (int)solved.size(); ++j)
    if (j != skip && solved[j].src == t.src) cand.push_back({std::fabs(std::log(solved[j].f / t.f)), j});
  if (cand.empty()) return false;
  std::sort(cand.begin(), cand.end());
  sp.a = cand[0].second;
  sp.b = cand.size() > 1 ? cand[1].second : cand[0].second;
  const double fa = solved[sp.a].f, fb = solved[sp.b].f;
  sp.tau = (fa == fb) ? 0.0f : (float)(std::log(t.f / fa) / std::log(fb / fa));
  sp.logf = (float)(0.5 * std::log10(t.f));
  sp.src_kind = t.point ? 1 : 0;
  for (int d = 0; d < 3; ++d) sp.src[d] = (float)t.pos[d];
  sp.q = (float)((std::log10(t.f) - std::log10(fa)) * (std::log10(t.f) - std::log10(fb)));
  return true;
}

// three-point Lagrange interpolation in log f: the three solved columns of
// the same source nearest to the target, used only when the target lies
// inside their frequency range (no extrapolation); false otherwise
struct Quad {
  int tcol, c[3];
  double w[3];
};

bool quad_neighbours(const std::vector<Column> &solved, const Column &t, Quad &q) {
  std::vector<std::pair<double, int>> cand;
  for (int j = 0; j < (int)solved.size(); ++j)
    if (solved[j].src == t.src) cand.push_back({std::fabs(std::log(solved[j].f / t.f)), j});
  if (cand.size() < 3) return false;
  std::sort(cand.begin(), cand.end());
  double u[3], lo = 1e300, hi = -1e300;
  for (int i = 0; i < 3; ++i) {
    q.c[i] = cand[i].second;
    u[i] = std::log(solved[q.c[i]].f);
    lo = std::min(lo, u[i]);
    hi = std::max(hi, u[i]);
  }
  const double ut = std::log(t.f);
  if (u[0] == u[1] || u[0] == u[2] || u[1] == u[2] || ut < lo || ut > hi) return false;
  for (int i = 0; i < 3; ++i) {
    const int i1 = (i + 1) % 3, i2 = (i + 2) % 3;
    q.w[i] = (ut - u[i1]) * (ut - u[i2]) / ((u[i] - u[i1]) * (u[i] - u[i2]));
  }
  return true;
}

// out[:, tcol] = sum_i w_i xs[:, c_i] for every target (complex columns)
__global__ void lagrange3_kernel(long ne, int ks, int kt, int nq, const Quad *__restrict__ q,
                                 const double2 *__restrict__ xs, double2 *__restrict__ out) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= ne * nq) return;
  const long e = t / nq;
  const Quad qq = q[t - e * nq];
  double2 v = make_double2(0.0, 0.0);
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const double2 x = xs[e * ks + qq.c[i]];
    v.x += qq.w[i] * x.x;
    v.y += qq.w[i] * x.y;
  }
  out[e * kt + qq.tcol] = v;
}

std::vector<Spec> training_specs(const std::vector<Column> &cols) {
  std::vector<Spec> specs;
  for (int j = 0; j < (int)cols.size(); ++j) {
    Spec sp;
    if (!neighbours(cols, cols[j], j, sp)) continue;
    sp.tcol = j;
    specs.push_back(sp);
  }
  return specs;
}

void prepare(Context &c, WarmStartNet &net, unsigned seed) {
  need(c.device >= 0, EMG_ERR_STATE, "the warm start needs a device context");
  need(c.have_ls && c.nrho > 0, EMG_ERR_STATE, "warm start before create_linear_system and emg_set_model");
  EMG_CUDA(cudaSetDevice(c.device));
  if (!net.ready) net.init(seed, c.stream);
  if (net.stat_ne != c.ne || !net.stat.p) net.statics(c);
}

}  // namespace

}  // namespace emg

using namespace emg;

extern "C" {

int emg_warm_start_train(emg_context *c, int k, const double *freqs, const int *src, const double *src_pos,
                         const double *x_dev, const emg_warm_opts *o, double *final_loss) {
  EMG_API_BEGIN
  need(c && freqs && x_dev && o, EMG_ERR_ARG, "null argument");
  need(k >= 2, EMG_ERR_ARG, "training needs at least two solved columns");
  need(o->steps >= 0 && o->batch >= 128 && o->lr > 0, EMG_ERR_ARG, "bad training options");
  WarmStartNet &net = net_of(*c);
  prepare(*c, net, o->seed);
  std::vector<Column> cols = columns(k, freqs, src, src_pos);
  std::vector<Spec> specs = training_specs(cols);
  need(!specs.empty(), EMG_ERR_ARG, "no solved column has a solved neighbour of the same source");
  double loss = 0.0;
  for (int it = 0; it < o->steps; ++it) {
    // constant rate, then a linear decay over the last 30 % of the steps
    const double t = (double)it / std::max(1, o->steps);
    const float lr = (float)(o->lr * (t < 0.7 ? 1.0 : std::max(0.05, (1.0 - t) / 0.3)));
    net.train_step(*c, x_dev, k, specs, o->batch, lr, false);
  }
  if (o->steps > 0) {
    double l0 = 0.0;
    net.loss.download(&loss, 1, c->stream);
    net.loss0.download(&l0, 1, c->stream);
    EMG_CUDA(cudaStreamSynchronize(c->stream));
    net.check(c->stream);
    net.last_loss = loss;
    net.last_loss0 = l0;
  }
  if (final_loss) *final_loss = loss;
  EMG_API_END
}

int emg_warm_start_predict(emg_context *c, int k, const double *freqs, const int *src, const double *src_pos,
                           const double *x_dev, int kt, const double *tfreqs, const int *tsrc,
                           const double *tsrc_pos, int network, double *guess_dev) {
  EMG_API_BEGIN
  need(c && freqs && x_dev && tfreqs && guess_dev, EMG_ERR_ARG, "null argument");
  need(k >= 1 && kt >= 1, EMG_ERR_ARG, "bad block widths");
  WarmStartNet &net = net_of(*c);
  prepare(*c, net, 1u);
  std::vector<Column> cols = columns(k, freqs, src, src_pos);
  std::vector<Column> tg = columns(kt, tfreqs, tsrc, tsrc_pos);
  std::vector<Spec> specs;
  EMG_CUDA(cudaMemsetAsync(guess_dev, 0, sizeof(double) * 2 * (size_t)c->ne * kt, c->stream));
  for (int j = 0; j < kt; ++j) {
    Spec sp;
    if (!neighbours(cols, tg[j], -1, sp)) continue;  // no solved neighbour: zero guess
    sp.tcol = j;
    specs.push_back(sp);
  }
  need(network >= 0 && network <= 3, EMG_ERR_ARG, "network must be 0, 1, 2 or 3");
  // 2: the network only where training showed it halves the interpolation's
  // curvature error (a quarter of its squared loss on the same samples)
  const bool use_net = network == 1 || (network == 2 && net.last_loss >= 0 && net.last_loss0 > 0 &&
                                        net.last_loss <= 0.25 * net.last_loss0);
  if (network == 3 || (network == 2 && !use_net)) {
    // quadratic in log f where three solved columns bracket the target; the
    // linear interpolation for the rest (mode 2 without the network: on the
    // 384-column CSEM sweep this guess left a median initial residual of
    // 0.005 against 0.020 for the linear one and 0.037 for the network's)
    std::vector<Quad> quads;
    std::vector<Spec> lin;
    for (const Spec &sp : specs) {
      Quad q;
      q.tcol = sp.tcol;
      if (quad_neighbours(cols, tg[sp.tcol], q)) quads.push_back(q);
      else lin.push_back(sp);
    }
    if (!lin.empty()) net.predict(*c, x_dev, k, lin, guess_dev, kt, false);
    if (!quads.empty()) {
      DBuf<Quad> qd;
      qd.upload(quads, c->stream);
      const long total = (long)c->ne * (long)quads.size();
      lagrange3_kernel<<<(unsigned)((total + 255) / 256), 256, 0, c->stream>>>(
          c->ne, k, kt, (int)quads.size(), qd.p, (const double2 *)x_dev, (double2 *)guess_dev);
      EMG_LAUNCH_CHECK();
      EMG_CUDA(cudaStreamSynchronize(c->stream));  // qd is freed next
    }
  } else if (!specs.empty()) {
    net.predict(*c, x_dev, k, specs, guess_dev, kt, use_net);
  }
  EMG_CUDA(cudaStreamSynchronize(c->stream));
  net.check(c->stream);
  EMG_API_END
}

int emg_warm_start_losses(emg_context *c, double *loss, double *loss_interp) {
  EMG_API_BEGIN
  need(c && loss && loss_interp, EMG_ERR_ARG, "null argument");
  WarmStartNet &net = net_of(*c);
  *loss = net.last_loss;
  *loss_interp = net.last_loss0;
  EMG_API_END
}

int emg_warm_start_params(emg_context *c, float *get, const float *set, int *nparam) {
  EMG_API_BEGIN
  need(c != nullptr, EMG_ERR_ARG, "null context");
  if (nparam) *nparam = WarmStartNet::nparam();
  if (!get && !set) return EMG_OK;
  WarmStartNet &net = net_of(*c);
  prepare(*c, net, 1u);
  if (set) net.set_params(set, c->stream);
  if (get) net.params.download(get, WarmStartNet::nparam(), c->stream);
  EMG_CUDA(cudaStreamSynchronize(c->stream));
  EMG_API_END
}

int emg_warm_start_gradients(emg_context *c, int k, const double *freqs, const int *src, const double *src_pos,
                             const double *x_dev, long batch, int step, float *grads, double *loss) {
  EMG_API_BEGIN
  need(c && freqs && x_dev && grads, EMG_ERR_ARG, "null argument");
  need(batch >= 1 && step >= 0, EMG_ERR_ARG, "bad batch or step");
  WarmStartNet &net = net_of(*c);
  prepare(*c, net, 1u);
  std::vector<Column> cols = columns(k, freqs, src, src_pos);
  std::vector<Spec> specs = training_specs(cols);
  need(!specs.empty(), EMG_ERR_ARG, "no solved column has a solved neighbour of the same source");
  const int saved = net.step;
  net.step = step;
  net.train_step(*c, x_dev, k, specs, batch, 0.f, true);
  net.step = saved;
  DBuf<float> g(WarmStartNet::nparam());
  warm_start_param_grads(net.grad.p, g.p, c->stream);
  g.download(grads, WarmStartNet::nparam(), c->stream);
  double l = 0;
  net.loss.download(&l, 1, c->stream);
  EMG_CUDA(cudaStreamSynchronize(c->stream));
  net.check(c->stream);
  if (loss) *loss = l;
  EMG_API_END
}

int emg_warm_start_reset(emg_context *c) {
  EMG_API_BEGIN
  need(c != nullptr, EMG_ERR_ARG, "null context");
  if (c->device >= 0) EMG_CUDA(cudaSetDevice(c->device));
  c->warm.reset();
  EMG_API_END
}

}  // extern "C"
