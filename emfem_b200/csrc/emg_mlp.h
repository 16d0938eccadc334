// Learned warm start: the per-edge network (emg_mlp.cu) and its training and
// prediction drivers (emg_warmstart.cu).
#pragma once

#include <cstdint>
#include <vector>

#include "emg_internal.h"

namespace emg {

// one target column of a prediction (or of a training pass): the source
// block's columns a and b hold the two nearest solved frequencies of the same
// source, tau = log(f / f_a) / log(f_b / f_a), logf = log10(f) / 2; tcol is
// the column written (prediction) or the solved column learned (training).
// src_kind 0: plane wave (distance = depth), 1: point source at src.
// q = (log10 f - log10 f_a)(log10 f - log10 f_b): the error of the linear
// interpolation in log f is half the second derivative times q, so the
// network learns that curvature and the correction it adds is q times its
// output -- which carries over between neighbour spacings (training pairs
// are twice as far apart as the prediction pairs of a sweep).
struct Spec {
  int a, b, tcol, src_kind;
  float tau, logf;
  float src[3];
  float q;
};

struct WarmStartNet {
  bool ready = false;
  int step = 0;
  DBuf<float> params, m, v;      // FP32 master parameters and Adam moments
  DBuf<unsigned char> img;       // BF16 weight operands in the tensor-core layout
  DBuf<float> bias;              // 4 x 64
  DBuf<float> grad;              // the two accumulated gradient products
  DBuf<double> loss, loss0;
  // losses of the last training step: the network's, and that of a zero
  // correction (the interpolation) on the same samples; -1 before training
  double last_loss = -1, last_loss0 = -1;
  DBuf<int> err;
  DBuf<float4> stat;             // 3 per edge
  int stat_ne = 0;
  DBuf<Spec> specs_dev;
  void init(uint64_t seed, cudaStream_t s);
  void set_params(const float *host, cudaStream_t s);
  void statics(Context &c);
  // one minibatch: forward, backward, gradient products; then (unless
  // accumulate_only) an Adam step and the new BF16 image
  double train_step(Context &c, const double *xs, int ks, const std::vector<Spec> &specs, long batch, float lr,
                    bool accumulate_only);
  // guess[e, tcol] for every edge and spec; network = false: the log-f
  // interpolation alone
  void predict(Context &c, const double *xs, int ks, const std::vector<Spec> &specs, double *out, int kt,
               bool network);
  void check(cudaStream_t s);
  static int nparam();
  static int image_bytes();
};

// per-parameter gradients (the FP32 parameter layout) from the two
// accumulated products of a training pass
void warm_start_param_grads(const float *grad_products, float *out, cudaStream_t s);

}  // namespace emg
