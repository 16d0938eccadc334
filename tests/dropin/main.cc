/*
 * Runs the drop-in bodies (em_dropin.cc) the way the reference's forward_csem
 * (src/em_fwd.cc:1382-1439) calls them, on a mesh written by the test into a
 * directory of raw arrays.  device < 0: a host-only context -- the right-hand
 * sides and marking run, the device entry points must fail through SETERRQ.
 * device >= 0: the whole CSEM sequence (system, assembly, preconditioner,
 * primal and dual solves, operator and preconditioner applications, error
 * estimate, marking).  Results go to <dir>/out_*.  Test infrastructure.
 */
#include <cmath>
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>

#include "em_dropin.h"

template <typename T>
static std::vector<T> load(const std::string &path, size_t n) {
  std::vector<T> v(n);
  std::ifstream f(path, std::ios::binary);
  f.read(reinterpret_cast<char *>(v.data()), (std::streamsize)(n * sizeof(T)));
  if (!f) {
    std::fprintf(stderr, "cannot read %s\n", path.c_str());
    std::exit(2);
  }
  return v;
}

template <typename T>
static void save(const std::string &path, const T *p, size_t n) {
  std::ofstream f(path, std::ios::binary);
  f.write(reinterpret_cast<const char *>(p), (std::streamsize)(n * sizeof(T)));
}

static void save_vec(const std::string &path, Vec re, Vec im) {
  std::vector<double> v(re->a);
  v.insert(v.end(), im->a.begin(), im->a.end());
  save(path, v.data(), v.size());
}

#define CHECK(x)                                                   \
  do {                                                             \
    PetscErrorCode e__ = (x);                                      \
    if (e__) {                                                     \
      std::fprintf(stderr, "%s failed with %d\n", #x, (int)e__);   \
      return 1;                                                    \
    }                                                              \
  } while (0)

int main(int argc, char **argv) {
  if (argc < 3) return 2;
  const std::string dir = argv[1];
  const int device = std::atoi(argv[2]);
  int nv, nt, ne, nrho, ncol, aniso, nf, nrx;
  {
    std::ifstream m(dir + "/meta.txt");
    m >> nv >> nt >> ne >> nrho >> ncol >> aniso >> nf >> nrx;
    if (!m) return 2;
  }
  auto pts = load<double>(dir + "/pts", 3 * (size_t)nv);
  auto tets = load<int>(dir + "/tets", 4 * (size_t)nt);
  auto attr = load<int>(dir + "/attr", nt);
  auto edges = load<int>(dir + "/edges", 2 * (size_t)ne);
  auto t2e = load<int>(dir + "/t2e", 6 * (size_t)nt);
  auto nbr = load<int>(dir + "/nbr", 4 * (size_t)nt);
  auto non = load<int>(dir + "/non", 4 * (size_t)nt);
  auto ebdr = load<unsigned char>(dir + "/ebdr", ne);
  auto rho = load<double>(dir + "/rho", (size_t)nrho * ncol);

  EMContext ctx;
  ctx.freqs = load<double>(dir + "/freqs", nf);
  ctx.tx = load<double>(dir + "/tx", 7);
  ctx.rx = load<double>(dir + "/rx", 3 * (size_t)nrx);
  ctx.n_edges = ne;
  ctx.n_tets = nt;
  // create_context / Mesh / read_rho / read_emd side (src/em_ctx.cc:7-98)
  if (emg_create_context(&ctx.emg, device) != EMG_OK) return 3;
  if (emg_set_mesh(ctx.emg, nv, pts.data(), nt, tets.data(), attr.data(), ne, edges.data(), t2e.data(), nbr.data(),
                   non.data(), ebdr.data()) != EMG_OK ||
      emg_set_model(ctx.emg, aniso, nrho, ncol, rho.data()) != EMG_OK ||
      emg_set_frequencies(ctx.emg, nf, ctx.freqs.data()) != EMG_OK) {
    std::fprintf(stderr, "setup: %s\n", emg_last_error());
    return 3;
  }
  for (Vec *v : {&ctx.s.re, &ctx.s.im, &ctx.csem_e.re, &ctx.csem_e.im, &ctx.dual_e.re, &ctx.dual_e.im})
    VecCreateSeq(PETSC_COMM_SELF, ne, v);

  // host side: right-hand sides and marking
  CHECK(assemble_rhs_dual(&ctx));
  save_vec(dir + "/out_dual_rhs", ctx.s.re, ctx.s.im);
  CHECK(assemble_rhs_csem(&ctx, 0, 0));
  save_vec(dir + "/out_csem_rhs", ctx.s.re, ctx.s.im);
  {
    Eigen::VectorXd err;
    err.resize(nt);
    for (int t = 0; t < nt; ++t) err[t] = std::fabs(std::sin(0.37 * t)) + 1e-3 * (t % 7);
    std::vector<bool> f1(nt, false), f2(nt, false);
    CHECK(refine_fixed_fraction(err, f1, 0.2));
    CHECK(refine_fixed_number(err, f2, 0.2));
    std::vector<unsigned char> out(2 * (size_t)nt);
    for (int t = 0; t < nt; ++t) {
      out[t] = f1[t];
      out[nt + t] = f2[t];
    }
    save(dir + "/out_flags", out.data(), out.size());
  }

  if (device < 0) {
    // every device entry point reports through SETERRQ(EM_ERR_USER)
    const PetscErrorCode e1 = create_linear_system(&ctx, 0), e2 = assemble_matrix(&ctx, 0), e3 = create_pc(&ctx);
    std::printf("host-only: %d %d %d\n", (int)e1, (int)e2, (int)e3);
    emg_destroy_context(ctx.emg);
    return (e1 == EM_ERR_USER && e2 == EM_ERR_USER && e3 == EM_ERR_USER) ? 0 : 4;
  }

  // forward_csem (src/em_fwd.cc:1404-1419): system, operators, both solves, estimate
  CHECK(create_linear_system(&ctx, 0));
  CHECK(assemble_matrix(&ctx, 0));
  CHECK(create_pc(&ctx));
  CHECK(assemble_rhs_csem(&ctx, 0, 0));
  Vec s_copy_re, s_copy_im;
  VecCreateSeq(PETSC_COMM_SELF, ne, &s_copy_re);
  VecCreateSeq(PETSC_COMM_SELF, ne, &s_copy_im);
  s_copy_re->a = ctx.s.re->a;
  s_copy_im->a = ctx.s.im->a;
  CHECK(solve_linear_system(&ctx, ctx.s, ctx.csem_e, ctx.K_max_it, ctx.e_rtol));
  save_vec(dir + "/out_csem_e", ctx.csem_e.re, ctx.csem_e.im);
  CHECK(assemble_rhs_dual(&ctx));
  CHECK(solve_linear_system(&ctx, ctx.s, ctx.dual_e, ctx.K_max_it, ctx.dual_rtol));
  CHECK(estimate_error(&ctx, 0, 0));
  save(dir + "/out_csem_error", ctx.csem_error.data(), (size_t)nt);
  // the MatShell and PCShell callbacks on VecNest blocks: A e and B^-1 s
  _p_Mat shell;
  shell.ctx = &ctx;
  _p_PC pcs;
  pcs.ctx = &ctx;
  Vec xb[2] = {ctx.csem_e.re, ctx.csem_e.im}, x, y, yb[2], sb[2] = {s_copy_re, s_copy_im}, sn, z, zb[2];
  VecCreateSeq(PETSC_COMM_SELF, ne, &yb[0]);
  VecCreateSeq(PETSC_COMM_SELF, ne, &yb[1]);
  VecCreateSeq(PETSC_COMM_SELF, ne, &zb[0]);
  VecCreateSeq(PETSC_COMM_SELF, ne, &zb[1]);
  VecCreateNest(PETSC_COMM_SELF, 2, nullptr, xb, &x);
  VecCreateNest(PETSC_COMM_SELF, 2, nullptr, yb, &y);
  VecCreateNest(PETSC_COMM_SELF, 2, nullptr, sb, &sn);
  VecCreateNest(PETSC_COMM_SELF, 2, nullptr, zb, &z);
  CHECK(matshell_mult_a(&shell, x, y));
  save_vec(dir + "/out_Ae", yb[0], yb[1]);
  CHECK(pc_apply_b(&pcs, sn, z));
  save_vec(dir + "/out_pc_s", zb[0], zb[1]);
  CHECK(destroy_pc(&ctx));
  CHECK(destroy_linear_system(&ctx));
  emg_destroy_context(ctx.emg);
  std::printf("device run ok\n");
  return 0;
}
