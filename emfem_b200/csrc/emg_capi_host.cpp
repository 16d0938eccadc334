// Host-side entry points of the C ABI (no GPU involved): point location,
// survey files, VTK output, receiver responses.  They work on host-only
// contexts as on GPU contexts.

#include <algorithm>
#include <cmath>
#include <complex>
#include <memory>
#include <string>
#include <vector>

#include "emg_api.h"
#include "emg_internal.h"
#include "emg_io.h"
#include "emg_locate.h"

using namespace emg;

extern "C" {

struct emg_point_index {
  emg::PointIndex index;
  emg_point_index(int nv, const double *pts, int nt, const int *tets, const int *nbr)
      : index(nv, pts, nt, tets, nbr) {}
};

static void locate_all(const PointIndex &ix, int n, const double *pts, int *out) {
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < n; ++i) out[i] = ix.find(pts + 3 * (size_t)i);
}

emg_point_index *emg_point_index_create(int nv, const double *pts, int nt, const int *tets, const int *nbr) {
  try {
    need(nv > 0 && nt > 0 && pts && tets && nbr, EMG_ERR_ARG, "empty or null mesh");
    for (long i = 0; i < 4L * nt; ++i) {
      need(tets[i] >= 0 && tets[i] < nv, EMG_ERR_ARG, "tetrahedronlist index out of range");
      need(nbr[i] >= -1 && nbr[i] < nt, EMG_ERR_ARG, "neighborlist index out of range");
    }
    return new emg_point_index(nv, pts, nt, tets, nbr);
  } catch (const emg::Error &e) {
    emg::set_last_error(e.what());
  } catch (const std::exception &e) {
    emg::set_last_error(e.what());
  }
  return nullptr;
}

int emg_point_index_find(const emg_point_index *idx, int n, const double *pts, int *tets_out) {
  EMG_API_BEGIN
  need(idx && n >= 0 && (n == 0 || (pts && tets_out)), EMG_ERR_ARG, "null argument");
  locate_all(idx->index, n, pts, tets_out);
  EMG_API_END
}

void emg_point_index_destroy(emg_point_index *idx) { delete idx; }

int emg_find_cell_around_point(emg_context *c, int n, const double *pts, int *tets_out) {
  EMG_API_BEGIN
  need(c && n >= 0 && (n == 0 || (pts && tets_out)), EMG_ERR_ARG, "null argument");
  need(c->nt > 0, EMG_ERR_STATE, "find_cell_around_point before emg_set_mesh");
  if (!c->locator)
    c->locator = std::make_shared<PointIndex>(c->nv, c->h_pts.data(), c->nt, c->h_tets.data(), c->h_nbr.data());
  locate_all(*c->locator, n, pts, tets_out);
  EMG_API_END
}

struct emg_survey {
  emg::Survey s;
};

emg_survey *emg_survey_read_emd(const char *path) {
  if (!path) {
    emg::set_last_error("null argument");
    return nullptr;
  }
  try {
    std::unique_ptr<emg_survey> h(new emg_survey);
    std::string err;
    if (!emg::read_emd(path, h->s, err)) {
      emg::set_last_error(err.c_str());
      return nullptr;
    }
    return h.release();
  } catch (const std::exception &e) {
    emg::set_last_error(e.what());
  }
  return nullptr;
}

int emg_survey_sizes(const emg_survey *h, int *n_freqs, int *n_tx, int *n_rx, int *n_obs) {
  EMG_API_BEGIN
  need(h, EMG_ERR_ARG, "null survey");
  if (n_freqs) *n_freqs = (int)h->s.freqs.size();
  if (n_tx) *n_tx = (int)h->s.tx.size() / kTxSize;
  if (n_rx) *n_rx = (int)h->s.rx.size() / 3;
  if (n_obs) *n_obs = (int)h->s.obs.size();
  EMG_API_END
}

int emg_survey_get(const emg_survey *h, double *freqs, double *tx, double *rx, int *otype, int *fidx, int *tidx,
                   int *ridx, double *obs, double *obserr) {
  EMG_API_BEGIN
  need(h, EMG_ERR_ARG, "null survey");
  const Survey &s = h->s;
  if (freqs) std::copy(s.freqs.begin(), s.freqs.end(), freqs);
  if (tx) std::copy(s.tx.begin(), s.tx.end(), tx);
  if (rx) std::copy(s.rx.begin(), s.rx.end(), rx);
  if (otype) std::copy(s.otype.begin(), s.otype.end(), otype);
  if (fidx) std::copy(s.fidx.begin(), s.fidx.end(), fidx);
  if (tidx) std::copy(s.tidx.begin(), s.tidx.end(), tidx);
  if (ridx) std::copy(s.ridx.begin(), s.ridx.end(), ridx);
  for (size_t i = 0; i < s.obs.size(); ++i) {
    if (obs) {
      obs[2 * i] = s.obs[i].real();
      obs[2 * i + 1] = s.obs[i].imag();
    }
    if (obserr) {
      obserr[2 * i] = s.obserr[i].real();
      obserr[2 * i + 1] = s.obserr[i].imag();
    }
  }
  EMG_API_END
}

int emg_survey_write_rsp(const emg_survey *h, const char *path, const double *rsp) {
  EMG_API_BEGIN
  need(h && path && (rsp || h->s.obs.empty()), EMG_ERR_ARG, "null argument");
  std::string err;
  if (!emg::write_rsp(path, h->s, reinterpret_cast<const std::complex<double> *>(rsp), err))
    fail(EMG_ERR_USER, "%s", err.c_str());
  EMG_API_END
}

void emg_survey_destroy(emg_survey *h) { delete h; }

int emg_save_vtk(emg_context *c, const char *path, int n_arrays, const char *const *names,
                 const double *const *data) {
  EMG_API_BEGIN
  need(c && path && n_arrays >= 0 && (n_arrays == 0 || (names && data)), EMG_ERR_ARG, "null argument");
  need(c->nt > 0, EMG_ERR_STATE, "save_vtk before emg_set_mesh");
  std::vector<std::pair<std::string, const double *>> arrays;
  for (int k = 0; k < n_arrays; ++k) {
    need(names[k] && data[k], EMG_ERR_ARG, "null array");
    const std::string nm = names[k];
    need(!nm.empty() && nm.find_first_of(" \t\n") == std::string::npos, EMG_ERR_ARG,
         "array names must be non-empty single words");
    arrays.push_back({nm, data[k]});
  }
  std::string err;
  if (!emg::write_vtk(path, c->nv, c->h_pts.data(), c->nt, c->h_tets.data(), c->h_attr.data(), arrays, err))
    fail(EMG_ERR_USER, "%s", err.c_str());
  EMG_API_END
}

// calculate_response_mt (em_fwd.cc:747-800): the reference's tensor
// impedance and tipper formulas per observation, plus apparent resistivity
// and phase from Z_XY / Z_YX.
int emg_calculate_response_mt(double freq, int nrx, const double *fields, int nobs, const int *otype,
                              const int *ridx, double *rsp) {
  EMG_API_BEGIN
  typedef std::complex<double> zc;
  need(nobs >= 0 && nrx >= 0, EMG_ERR_ARG, "negative count");
  need(nobs == 0 || (fields && otype && ridx && rsp), EMG_ERR_ARG, "null argument");
  need(freq > 0, EMG_ERR_ARG, "frequency must be positive");
  for (int o = 0; o < nobs; ++o) {
    need(ridx[o] >= 0 && ridx[o] < nrx, EMG_ERR_ARG, "receiver index out of range");
    const double *f = fields + 24 * (size_t)ridx[o];
    auto at = [&](int block, int k) { return zc(f[6 * block + 2 * k], f[6 * block + 2 * k + 1]); };
    const zc exy[3] = {at(0, 0), at(0, 1), at(0, 2)}, hxy[3] = {at(1, 0), at(1, 1), at(1, 2)};
    const zc eyx[3] = {at(2, 0), at(2, 1), at(2, 2)}, hyx[3] = {at(3, 0), at(3, 1), at(3, 2)};
    const zc den = hxy[0] * hyx[1] - hyx[0] * hxy[1];
    zc v;
    switch (otype[o]) {
    case EMG_OBS_Z_XX_RI: v = (exy[0] * hyx[1] - eyx[0] * hxy[1]) / den; break;
    case EMG_OBS_Z_XY_RI: v = (eyx[0] * hxy[0] - exy[0] * hyx[0]) / den; break;
    case EMG_OBS_Z_YX_RI: v = (exy[1] * hyx[1] - eyx[1] * hxy[1]) / den; break;
    case EMG_OBS_Z_YY_RI: v = (eyx[1] * hxy[0] - exy[1] * hyx[0]) / den; break;
    case EMG_OBS_T_ZX_RI: v = (hxy[2] * hyx[1] - hyx[2] * hxy[1]) / den; break;
    case EMG_OBS_T_ZY_RI: v = (hyx[2] * hxy[0] - hxy[2] * hyx[0]) / den; break;
    case EMG_OBS_R_XY_AP:
    case EMG_OBS_R_YX_AP: {
      const zc z = otype[o] == EMG_OBS_R_XY_AP ? (eyx[0] * hxy[0] - exy[0] * hyx[0]) / den
                                                : (exy[1] * hyx[1] - eyx[1] * hxy[1]) / den;
      // the reference's AP pair: log amplitude and phase in radians (as
      // read_emd stores the observation and save_rsp writes it back)
      v = zc(std::log(std::norm(z) / (2.0 * PI * freq * MU)), std::arg(std::conj(z)));
      break;
    }
    default: fail(EMG_ERR_USER, "Data type %d not implemented.", otype[o]);
    }
    rsp[2 * (size_t)o] = v.real();
    rsp[2 * (size_t)o + 1] = v.imag();
  }
  EMG_API_END
}

// calculate_response_csem (em_fwd.cc:802-871)
int emg_calculate_response_csem(int nrx, const double *fields, int nobs, const int *otype, const int *ridx,
                                double *rsp) {
  EMG_API_BEGIN
  typedef std::complex<double> zc;
  need(nobs >= 0 && nrx >= 0, EMG_ERR_ARG, "negative count");
  need(nobs == 0 || (fields && otype && ridx && rsp), EMG_ERR_ARG, "null argument");
  for (int o = 0; o < nobs; ++o) {
    need(ridx[o] >= 0 && ridx[o] < nrx, EMG_ERR_ARG, "receiver index out of range");
    const double *f = fields + 12 * (size_t)ridx[o];
    auto comp = [&](int k) { return zc(f[2 * k], f[2 * k + 1]); };
    zc v;
    switch (otype[o]) {
    case EMG_OBS_F_EX_RI: v = comp(0); break;
    case EMG_OBS_F_EY_RI: v = comp(1); break;
    case EMG_OBS_F_EZ_RI: v = comp(2); break;
    case EMG_OBS_F_HX_RI: v = comp(3); break;
    case EMG_OBS_F_HY_RI: v = comp(4); break;
    case EMG_OBS_F_HZ_RI: v = comp(5); break;
    case EMG_OBS_F_EX_AP: v = std::log(comp(0)); break;
    case EMG_OBS_F_EY_AP: v = std::log(comp(1)); break;
    case EMG_OBS_F_EZ_AP: v = std::log(comp(2)); break;
    case EMG_OBS_F_HX_AP: v = std::log(comp(3)); break;
    case EMG_OBS_F_HY_AP: v = std::log(comp(4)); break;
    case EMG_OBS_F_HZ_AP: v = std::log(comp(5)); break;
    default: fail(EMG_ERR_USER, "Data type %d not implemented.", otype[o]);
    }
    rsp[2 * (size_t)o] = v.real();
    rsp[2 * (size_t)o + 1] = v.imag();
  }
  EMG_API_END
}

int emg_orient3d_sign(const double *a, const double *b, const double *c, const double *d, int *sign) {
  EMG_API_BEGIN
  need(a && b && c && d && sign, EMG_ERR_ARG, "null argument");
  *sign = emg::orient3d_sign(a, b, c, d);
  EMG_API_END
}

}  // extern "C"
