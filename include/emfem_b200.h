/*
 * emfem_b200 -- C ABI of the B200-native EMFEM forward-solve path.
 *
 * One opaque context mirrors the reference's EMContext (src/em_ctx.h:15-64):
 * it owns the mesh arrays, the assembled operators, the AMS preconditioner and
 * the named solution vectors, all resident in the device memory of one GPU.
 * Every entry point returns 0 on success or a negative status; the message
 * of the last failure on the calling thread is available from
 * emg_last_error().  Vectors cross the boundary as plain host pointers (the
 * *_dev variants take device pointers); nothing in this header uses torch
 * or PETSc types.  Single-threaded per context, like the reference.
 */
#ifndef EMFEM_B200_H
#define EMFEM_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define EMG_OK 0
#define EMG_ERR_USER (-1)          /* EM_ERR_USER, src/em_defs.h:76            */
#define EMG_ERR_ARG (-2)           /* bad argument (null pointer, size)       */
#define EMG_ERR_STATE (-3)         /* call out of order (e.g. solve before pc) */
#define EMG_ERR_CUDA (-4)          /* CUDA runtime error                       */
#define EMG_ERR_NOMEM (-5)         /* device allocation failed                 */
#define EMG_DIVERGED_ITS (-6)      /* Krylov hit max_it before rtol            */
#define EMG_DIVERGED_NANORINF (-7) /* NaN or Inf in a residual                 */
#define EMG_ERR_OPTION (-8)        /* unknown or malformed option              */
/* a block-solve column whose residual reached the FP64 rounding floor of its
 * own computation, u || |b| + |A||x| || (u = 2^-53), above rtol ||b||: no
 * iteration can lower it further (emg_last_residual_floors gives the floor;
 * no counterpart in the reference, whose KSP runs on to max_it there) */
#define EMG_STOPPED_AT_FLOOR 1

/* anisotropy forms, src/em_defs.h:37 */
#define EMG_ISOTROPIC 0
#define EMG_VERTICAL 1
#define EMG_TRIAXIAL 2
#define EMG_ARBITRARY 3

/* named solution slots: ctx->mt_e[XY_POLAR], mt_e[YX_POLAR], csem_e, dual_e
 * (src/em_ctx.h:44-45, src/em_defs.h:39) */
#define EMG_SOL_MT_XY (-1)
#define EMG_SOL_MT_YX (-2)
#define EMG_SOL_CSEM 0
#define EMG_SOL_DUAL 1

typedef struct emg_context emg_context;

typedef struct emg_solve_info {
  int outer_its;        /* FGMRES iterations                                 */
  int inner_its;        /* total FCG iterations (both real blocks)           */
  int reason;           /* 0 converged, EMG_STOPPED_AT_FLOOR, EMG_DIVERGED_* */
  double true_rel_res;  /* ||b - A x|| / ||b|| recomputed in FP64 at exit    */
  double seconds;       /* device time of the solve                          */
} emg_solve_info;

const char *emg_last_error(void);
const char *emg_version(void);

/* create_context / destroy_context (src/em_ctx.cc:7-98). device: CUDA ordinal,
 * or -1 for a host-only context: it takes options, mesh, model, frequencies
 * and background, and serves the host-side entry points (CSEM and dual
 * right-hand sides, point location, marking, responses); every entry point
 * that needs a GPU returns EMG_ERR_STATE. */
int emg_create_context(emg_context **ctx, int device);
int emg_destroy_context(emg_context *ctx);

/* process_options (src/em_ctx.cc:100-175): PETSc options-file text ("-key
 * value" tokens, '#' comments).  Honours -K_max_it -e_rtol -dual_rtol
 * -inner_pc_type -pc_threshold -n_tx_divisions -refine_fraction
 * -refine_strategy -max_adaptive_refinements -n_uniform_refinements
 * -max_dofs -save_mesh -iprefix -oprefix -n_groups -max_tx_edge_length
 * -max_rx_edge_length -mesh_format -direct_solver_type, the A_/B_ subset the
 * GPU solver implements (A_ksp_gmres_restart, B_ksp_rtol, B_ksp_max_it,
 * B_pc_hypre_ams_cycle_type, B_pc_hypre_ams_relax_times, ...) and the
 * -emg_* keys of this implementation.  Unknown keys: EMG_ERR_OPTION. */
int emg_process_options(emg_context *ctx, const char *options_text);
int emg_get_option(emg_context *ctx, const char *key, double *value);

/* Mesh arrays as the host Mesh keeps them (src/em_mesh.h:81-96, one rank:
 * identity numbering).  Copied to the device; edge numbering is never
 * changed.  edge_bdr: edge_bdr_marker_ (src/em_mesh.cc:483-502). */
int emg_set_mesh(emg_context *ctx, int n_vertices, const double *pointlist, int n_tets,
                 const int *tetrahedronlist, const int *attributes, int n_edges, const int *edgelist,
                 const int *tet2edgelist, const int *neighborlist, const int *tet_non,
                 const unsigned char *edge_bdr_marker);

/* read_rho (src/em_io.cc:9-86): n_rho rows of ncol resistivities (and
 * Euler angles in degrees for the Arbitrary form). */
int emg_set_model(emg_context *ctx, int aniso_form, int n_rho, int ncol, const double *rho);

/* ctx->freqs (src/em_ctx.h:21) */
int emg_set_frequencies(emg_context *ctx, int n, const double *freqs);

/* create_linear_system / destroy_linear_system (src/em_fwd.cc:248-316).
 * tidx < 0: MT (two primal slots), tidx >= 0: CSEM. */
int emg_create_linear_system(emg_context *ctx, int tidx);
int emg_destroy_linear_system(emg_context *ctx);

/* make_sparsity_patterns (src/em_fwd.cc:191-246): *nnz always set; rptr
 * (n_edges+1) and cidx (nnz) filled when non-null. */
int emg_get_sparsity(emg_context *ctx, long *nnz, int *rptr, int *cidx);

/* assemble_matrix (src/em_fwd.cc:318-400) for frequency ctx->freqs[fidx]:
 * C (curl-curl/mu) and M (omega * mass) on the shared pattern, boundary
 * rows/columns zeroed as the reference does.  Values stay on the device;
 * emg_get_matrices copies them out (either pointer may be null), bdr_cells
 * (n_tets flags) is the reference's ctx->bdr_cells set. */
int emg_assemble_matrix(emg_context *ctx, int fidx);
int emg_get_matrices(emg_context *ctx, double *C, double *M, unsigned char *bdr_cells);

/* create_pc / destroy_pc (src/em_la.cc:113-206) incl. setup_ams
 * (src/em_la.cc:230-295): B = C + M and the AMS hierarchy. */
int emg_create_pc(emg_context *ctx);
int emg_destroy_pc(emg_context *ctx);

/* matshell_mult_a (src/em_la.cc:65-87) on host vectors of length 2n
 * ([re block; im block], the VecNest layout): y = [C xr - M xi; -M xr - C xi]. */
int emg_matshell_mult_a(emg_context *ctx, const double *x, double *y);

/* pc_apply_b (src/em_la.cc:208-228): x = [B^-1 br; B^-1 bi], each an FCG(AMS)
 * solve to the inner tolerance. */
int emg_pc_apply_b(emg_context *ctx, const double *b, double *x);

/* solve_linear_system (src/em_la.cc:35-63): real-form FGMRES right-
 * preconditioned by pc_apply_b, zero initial guess, into named slot
 * `target` (EMG_SOL_*).  Returns EMG_DIVERGED_ITS if max_it is hit (the
 * reference is silent there) -- the slot still holds the last iterate. */
int emg_solve_linear_system(emg_context *ctx, int target, const double *s_re, const double *s_im,
                            int max_it, double rtol, emg_solve_info *info);

/* access_vec / VecGetArray on a named slot (src/em_la.cc:7-33). */
int emg_get_solution(emg_context *ctx, int target, double *e_re, double *e_im);
int emg_set_solution(emg_context *ctx, int target, const double *e_re, const double *e_im);

/* RHS assembly (src/em_fwd.cc:402-717) into host vectors s_re/s_im.
 * MT: needs the layered background columns under the four top corners
 * (update_background_model, src/em_fwd.cc:135-159): corners 4x3, nlay[4],
 * ztop/lsig laid out 4 x maxl. */
int emg_set_background(emg_context *ctx, const double *corners, const int *nlay, const double *ztop,
                       const double *lsig, int maxl);
int emg_assemble_rhs_mt(emg_context *ctx, int fidx, int mode, double *s_re, double *s_im);
int emg_assemble_rhs_csem(emg_context *ctx, int fidx, const double *tx7, const int *dipole_tets,
                          double *s_re, double *s_im);
int emg_assemble_rhs_dual(emg_context *ctx, int n_rx, const double *rx, const int *rx_tets, double *s_re,
                          double *s_im);

/* estimate_error (src/em_fwd.cc:1102-1180) on the named slots: MT (tidx<0)
 * uses XY, YX and DUAL and writes err[0..T) = sqrt(eta_xy*eta_dual),
 * err[T..2T) = sqrt(eta_yx*eta_dual); CSEM writes err[0..T).  eta_raw
 * (optional, n_sol x T) receives the per-solution indicators. */
int emg_estimate_error(emg_context *ctx, int fidx, int tidx, double *err, double *eta_raw);

/* Same indicators as emg_estimate_error, for callers that cannot let the
 * library allocate device memory during a run (an application whose memory
 * manager owns the device, or code that must not be stalled by
 * cudaMalloc/cudaFree).  No counterpart in the reference.  The scratch lives
 * in a fixed 15.7 MB device array of the library (held on every GPU that
 * loads it), so meshes above 131072 tets are rejected with EMG_ERR_ARG.
 * err_dev (n_err x T) and eta_dev (n_sol x T) are caller-owned device
 * buffers laid out as in emg_estimate_error.  The array's device address is
 * looked up when a device context is created (emg_create_context), so this
 * call loads no module and allocates nothing.  It runs on the context's own
 * stream, which is not ordered after the caller's streams: any pending work
 * of the caller that writes or reads err_dev/eta_dev must be complete before
 * the call (synchronise that stream first).  Every call shares the array:
 * calls that overlap on the GPU (two contexts or threads at once) race.
 * Returns after the context's stream completes, so the outputs are ready. */
int emg_estimate_error_noalloc(emg_context *ctx, int fidx, int tidx, double *err_dev, double *eta_dev);

/* refine_fixed_fraction / refine_fixed_number (src/em_fwd.cc:1182-1240):
 * ORs flags into flag[n] exactly as the reference. Host-side. */
int emg_refine_fixed_fraction(int n, const double *err, double fraction, unsigned char *flag);
int emg_refine_fixed_number(int n, const double *err, double fraction, unsigned char *flag);

/* interpolate_fields (src/em_fwd.cc:719-744) for n points with known
 * cells: E and H (6 complex, interleaved re/im) per point from slot target. */
int emg_interpolate_fields(emg_context *ctx, int target, int fidx, int n, const double *pts,
                           const int *tets, double *eh);
/* the same from a solution the caller holds on the host (e_re, e_im: one
 * value per edge, the reference's PETScBlockVector parts); works on a
 * host-only context */
int emg_interpolate_fields_host(emg_context *ctx, int fidx, int n, const double *pts, const int *tets,
                                const double *e_re, const double *e_im, double *eh);

/* find_cell_around_point (src/em_mesh.cc:527-566) for many points: the
 * reference's walk (from the last tet of the closest vertex, breadth-first
 * over neighbours, first tet whose four orientations are >= 0), with the
 * closest vertex from a uniform grid and no per-query O(T) clearing.  The
 * index copies the arrays (tetgenio layout: pointlist, tetrahedronlist,
 * neighborlist with -1 on the boundary).  tets_out[i] = -1 where no tet
 * contains the point (the reference asserts).  Host only. */
typedef struct emg_point_index emg_point_index;
emg_point_index *emg_point_index_create(int nv, const double *pts, int nt, const int *tets, const int *nbr);
int emg_point_index_find(const emg_point_index *idx, int n, const double *pts, int *tets_out);
/* *sign = the exact sign (-1, 0, 1) of orient3d(a, b, c, d) = det[a-d; b-d;
 * c-d] for 3-vectors a..d: the predicate behind TetAccessor::contains_point
 * (src/em_mesh.h:208-230), whose robust orient3d has an exact sign */
int emg_orient3d_sign(const double *a, const double *b, const double *c, const double *d, int *sign);
void emg_point_index_destroy(emg_point_index *idx);
/* the same on the context's mesh (index built on first use, dropped by the
 * next emg_set_mesh) */
int emg_find_cell_around_point(emg_context *ctx, int n, const double *pts, int *tets_out);

/* Observation types (ObsType, src/em_defs.h:50-73). */
#define EMG_OBS_F_EX_RI 111
#define EMG_OBS_F_EY_RI 121
#define EMG_OBS_F_EZ_RI 131
#define EMG_OBS_F_HX_RI 141
#define EMG_OBS_F_HY_RI 151
#define EMG_OBS_F_HZ_RI 161
#define EMG_OBS_F_EX_AP 112
#define EMG_OBS_F_EY_AP 122
#define EMG_OBS_F_EZ_AP 132
#define EMG_OBS_F_HX_AP 142
#define EMG_OBS_F_HY_AP 152
#define EMG_OBS_F_HZ_AP 162
#define EMG_OBS_R_XY_AP 212
#define EMG_OBS_R_YX_AP 222
#define EMG_OBS_Z_XX_RI 311
#define EMG_OBS_Z_XY_RI 321
#define EMG_OBS_Z_YX_RI 331
#define EMG_OBS_Z_YY_RI 341
#define EMG_OBS_T_ZX_RI 351
#define EMG_OBS_T_ZY_RI 361

/* calculate_response_mt (src/em_fwd.cc:747-800) from the fields at the
 * receivers.  fields: per receiver 12 complex values, interleaved re/im:
 * E and H of the XY polarisation, then E and H of the YX polarisation (what
 * emg_interpolate_fields returns for EMG_SOL_MT_XY and EMG_SOL_MT_YX).  For
 * observation o: type otype[o], receiver ridx[o] -> rsp[2o], rsp[2o+1].
 * Z_XX/XY/YX/YY_RI and T_ZX/ZY_RI as the reference.  R_XY_AP / R_YX_AP,
 * which the reference declares but refuses, give the reference's AP pair
 * (read_emd / save_rsp, src/em_io.cc:248-262, 360-372): the log of the
 * apparent resistivity |Z|^2 / (w mu) (real part) and the phase of conj(Z)
 * in radians (imaginary part: the e^{-iwt} phase of the reference's e^{+iwt}
 * fields; a halfspace gives pi/4 and -3pi/4).  Other types: EMG_ERR_USER, as
 * the reference.  Host only; needs no context. */
int emg_calculate_response_mt(double freq, int nrx, const double *fields, int nobs, const int *otype,
                              const int *ridx, double *rsp);

/* calculate_response_csem (src/em_fwd.cc:802-871): fields per receiver are 6
 * complex values (E, H); F_*_RI give the component, F_*_AP its complex
 * logarithm.  Host only. */
int emg_calculate_response_csem(int nrx, const double *fields, int nobs, const int *otype, const int *ridx,
                                double *rsp);

/* Survey files in the reference's layout: read_emd (src/em_io.cc:202-287)
 * and save_rsp (src/em_io.cc:316-399).  emg_survey_read_emd returns NULL on
 * error (emg_last_error() says why).  Observations come back as the
 * reference stores them: AP types as (log amplitude, phase in radians) with
 * errors ((err_amp/100)^2, (err_phase in radians)^2), the others as
 * (re, im) with squared errors.  emg_survey_write_rsp writes the file with
 * the responses rsp (one complex value per observation, interleaved, in the
 * same convention: what emg_calculate_response_mt/csem return).  Host only. */
typedef struct emg_survey emg_survey;
emg_survey *emg_survey_read_emd(const char *path);
int emg_survey_sizes(const emg_survey *s, int *n_freqs, int *n_tx, int *n_rx, int *n_obs);
/* any output pointer may be NULL; tx holds 7 values per transmitter (TX_SIZE) */
int emg_survey_get(const emg_survey *s, double *freqs, double *tx, double *rx, int *otype, int *fidx, int *tidx,
                   int *ridx, double *obs, double *obserr);
int emg_survey_write_rsp(const emg_survey *s, const char *path, const double *rsp);
void emg_survey_destroy(emg_survey *s);

/* Mesh::save_vtk (src/em_mesh.cc:183-248): the context's mesh as a legacy
 * ASCII VTK unstructured grid with cell data "subdomain" (0: one process),
 * "tet_attr" and n_arrays per-tet arrays (names[k], data[k][nt]) written in
 * name order; a repeated name keeps its first array.  Host only. */
int emg_save_vtk(emg_context *ctx, const char *path, int n_arrays, const char *const *names,
                 const double *const *data);

/* ---- batched fast path (no reference counterpart: replaces the per-task
 * loop of forward_mt/forward_csem, src/em_fwd.cc:1320-1439) -------------
 * Solves k right-hand sides with individual frequencies as blocks of at most
 * 32 columns, one after another (a block whose width is not a power of two is
 * padded with zero columns):
 * complex FGMRES (FP64 outer, true residual in FP64) around an AMS-
 * preconditioned FCG whose precision is set by -emg_inner_precision
 * (fp32|fp64).  One AMS hierarchy serves every frequency.
 * rhs/x: n x k complex, row-major with interleaved re/im (x[(i*k+c)*2+0/1]).
 * The system solved per column c is the reference's: (C + i w_c Ms) z = conj(s).
 * x holds the initial guess on entry when use_guess != 0. */
typedef struct emg_block_opts {
  double rtol;           /* outer relative residual target (1e-8)           */
  int max_it;            /* outer iteration cap per column                   */
  int use_guess;         /* 1: x is the initial guess                        */
  int inner_fp32;        /* 1: FP32 AMS, 0: FP64, -1: -emg_inner_precision */
  int restart;           /* FGMRES restart (30)                              */
} emg_block_opts;

int emg_solve_block(emg_context *ctx, int k, const double *freqs, const double *rhs, double *x,
                    const emg_block_opts *opts, emg_solve_info *infos);
int emg_solve_block_dev(emg_context *ctx, int k, const double *freqs, const double *rhs_dev, double *x_dev,
                        const emg_block_opts *opts, emg_solve_info *infos);
/* Divergence correction of a block solution x (device, n x k complex, the
 * right-hand sides rhs_dev as emg_solve_block_dev takes them): x += G phi with
 * phi the vertex potential, zero on the Dirichlet boundary, that makes
 * G^T (b - A x) vanish at every interior vertex (b = conj(rhs), A = C + i w Ms),
 * solved by FCG with the block AMS's gradient-space V-cycle (fp32 selects
 * the FP32 or the FP64 hierarchy; the block solves run it after every solve
 * unless -emg_div_correction 0).  k: a power of two <= 32, after an
 * emg_solve_block(_dev) that set up the hierarchy of that precision.
 * its: total FCG iterations over the columns (may be NULL). */
int emg_divergence_correct_dev(emg_context *ctx, int k, const double *freqs, const double *rhs_dev, double *x_dev,
                               int fp32, long *its);

/* interpolate_fields (src/em_fwd.cc:719-744) for a device block x_dev (n_edges
 * x k complex, interleaved, as emg_solve_block_dev returns it) at n receivers
 * with known cells: eh[(r*k + j)*12 ...] holds E then H of column j at
 * receiver r (complex, interleaved re/im), H = -curl E / (i w_j mu).  One
 * device thread per (receiver, column); only the n x k x 12 values are
 * copied to the host.  emg_interpolate_fields uses it on a named slot. */
int emg_interpolate_fields_block_dev(emg_context *ctx, int k, const double *freqs, const double *x_dev, int n,
                                     const double *pts, const int *tets, double *eh);

/* assemble_rhs_csem (src/em_fwd.cc:582-671) for k columns at once: column j
 * is transmitter tx[7j .. 7j+7) (TX_SIZE values, line sources divided into
 * -n_tx_divisions dipoles) at frequency freqs[j].  The host divides the
 * sources and locates their cells (the reference's walk); the basis values
 * are evaluated and scattered into the zeroed device block s_dev (n_edges x k
 * complex) by a kernel.  A dipole outside the mesh: EMG_ERR_USER. */
int emg_assemble_rhs_csem_block_dev(emg_context *ctx, int k, const double *freqs, const double *tx,
                                    double *s_dev);
/* assemble_rhs_dual (src/em_fwd.cc:673-717) into every one of k columns of
 * s_dev (the dual right-hand side does not depend on the frequency). */
int emg_assemble_rhs_dual_block_dev(emg_context *ctx, int k, int n_rx, const double *rx, double *s_dev);

/* Batched MT right-hand sides (assemble_rhs_mt, src/em_fwd.cc:488-580, for k
 * columns at once): column j is polarisation modes[j] (EMG_SOL_MT_XY/YX) at
 * frequency freqs[j]; boundary values from the layered plane waves, lifting
 * on the device.  s: n x k complex, interleaved (host or device pointer). */
int emg_assemble_rhs_mt_block(emg_context *ctx, int k, const double *freqs, const int *modes, double *s);
int emg_assemble_rhs_mt_block_dev(emg_context *ctx, int k, const double *freqs, const int *modes, double *s_dev);

/* ---- learned warm start (no reference counterpart: the reference starts
 * every FGMRES from zero, src/em_la.cc:49) ------------------------------
 * A per-edge network (13 inputs: the two neighbour-frequency values of the
 * edge scaled by their larger magnitude, log resistivities, log length,
 * direction cosines, log distance to the source, log f and the position tau
 * of f between the neighbours in log f; three hidden layers of 64 with GELU;
 * BF16 weights, FP32 accumulation on the tensor cores) predicts a correction
 * to the log-f interpolation of the two nearest solved frequencies of the
 * same source.  Columns are (freqs[j], src[j]): src groups the columns of one
 * source (MT polarisation or transmitter); src_pos (k x 3) gives point-source
 * positions, NULL for plane waves (the distance feature is then the depth).
 * The guess only moves iteration counts: emg_solve_block with use_guess
 * falls back to zero for any column whose guess has a larger residual than
 * zero, and every column is still solved to rtol. */
typedef struct emg_warm_opts {
  int steps;        /* Adam steps (minibatches)                              */
  long batch;       /* samples (edge, column) per minibatch                  */
  float lr;         /* Adam learning rate (decays over the last 30 %)        */
  unsigned seed;    /* initialisation seed (first use of the network)        */
} emg_warm_opts;

/* trains on a solved block x_dev (n_edges x k complex): every column with a
 * solved neighbour of the same source is a target; *final_loss: mean squared
 * correction error of the last minibatch */
int emg_warm_start_train(emg_context *ctx, int k, const double *freqs, const int *src, const double *src_pos,
                         const double *x_dev, const emg_warm_opts *opts, double *final_loss);
/* guesses for kt target columns into guess_dev (n_edges x kt complex);
 * network 0: the log-f interpolation alone, 1: interpolation plus the
 * network's correction, 2: the network only if the last training step's loss
 * was at most a quarter of the interpolation's on the same samples, else as
 * 3; 3: three-point Lagrange interpolation in log f from the three nearest
 * solved columns of the source where they bracket the target, the log-f
 * interpolation elsewhere (no network); a target without a solved column of
 * its source gets zero */
int emg_warm_start_predict(emg_context *ctx, int k, const double *freqs, const int *src, const double *src_pos,
                           const double *x_dev, int kt, const double *tfreqs, const int *tsrc,
                           const double *tsrc_pos, int network, double *guess_dev);
/* the FP32 master parameters: W1 (64x16, out x in), W2, W3 (64x64), W4 (2x64),
 * b1, b2, b3 (64), b4 (2); *nparam their count; get/set may be NULL */
int emg_warm_start_params(emg_context *ctx, float *get, const float *set, int *nparam);
/* gradients of one training minibatch (sample s: target s mod n_targets,
 * a hashed edge of step `step`) without an update; tests */
int emg_warm_start_gradients(emg_context *ctx, int k, const double *freqs, const int *src, const double *src_pos,
                             const double *x_dev, long batch, int step, float *grads, double *loss);
/* drops the network (the next use re-initialises it) */
int emg_warm_start_reset(emg_context *ctx);
/* losses of the last training step: the network's and that of the
 * interpolation alone (a zero correction) on the same samples; -1 before
 * any training */
int emg_warm_start_losses(emg_context *ctx, double *loss, double *loss_interp);

/* ---- kernel-level entry points on device pointers (tests, benchmarks) -- */
/* y = (C + i w Ms) x  (conj_out=0)  or its conjugate (conj_out=1, the
 * real-form operator of matshell_mult_a) for k complex columns. */
int emg_spmv_complex_dev(emg_context *ctx, int k, const double *omegas_host, const double *x_dev,
                         double *y_dev, int conj_out);
/* y = b - (C + w_c Ms) x on K real columns (row-major n_edges x K, x, b
 * and y float when fp32 != 0, else double; omegas_host holds the K column
 * shifts w_c) with the SpMM lane layout (v, variant) forced instead of the
 * autotuner's choice: v columns per vector load; variant > 0 and < 100 the
 * row-split kernel with that many lanes per row, -B the row-group kernel,
 * 100 + NL / 300 + U packed 16-byte records (fp32 only), 200 + U the
 * software-pipelined kernel with chunks of U nonzeros, 400 + NL / 500 + NL
 * the row-split kernel capped at 64 registers (4 blocks per SM; packed
 * records / arrays, fp32, K >= 16), 601 / 604 the chunked kernel (rows in
 * whole chunks of 4 nonzeros; fp32, K >= 8; 604 register-capped).
 * EMG_ERR_ARG for a layout not built for K.  Tests every kernel the
 * autotuner can pick. */
int emg_spmm_layout_dev(emg_context *ctx, int fp32, int K, int v, int variant, const double *omegas_host,
                        const void *x_dev, const void *b_dev, void *y_dev);
/* the nodal AMG hierarchy of AMS subspace sp (0 gradient, 1-3 Pi_x/y/z, 4 the
 * vector space) of the assembled operators, built on the device (gpu != 0)
 * or by the host build, for reference frequency w_ref: per level 5 values
 * (rows, nonzeros of A, of P, sum |A| over both parts, sum |P|), the
 * coarsest operator last; *nlev levels (at most max_rows).  Tests. */
int emg_amg_levels(emg_context *ctx, int sp, int gpu, double w_ref, int max_rows, int *nlev, double *out);
/* per column of the last emg_solve_block(_dev): the relative residual
 * ||b - A x0|| / ||b|| of the start it used (1 for a zero start, also where
 * a guess was worse than zero and was dropped) */
int emg_last_initial_residuals(emg_context *ctx, int k, double *rel);
/* per column of the last emg_solve_block(_dev): u || |b| + |A||x| || / ||b||,
 * the relative residual below which the computed FP64 residual is rounding
 * noise (u = 2^-53, |.| entrywise); 0 with -emg_block_floor_stop 0 */
int emg_last_residual_floors(emg_context *ctx, int k, double *rel);
/* per-kernel device timing of the last call of each kind (ms) */
int emg_last_kernel_ms(emg_context *ctx, const char *name, double *ms);
int emg_stream_synchronize(emg_context *ctx);
/* number of kernels this library has launched in the process */
int emg_launch_count(long *n);
/* per-kernel event profiler (bins "spmm_edge_fp32", "spmm_edge_fp64",
 * "spmm_nodal_fp32", "spmm_nodal_fp64"): launches, device ms and algorithmic
 * bytes accumulated since emg_profile_enable(1) */
int emg_profile_enable(int on);
int emg_profile_get(const char *bin, long *count, double *ms, double *bytes);
/* the SpMM lane layouts the autotuner chose so far, one entry per (precision,
 * block width, nonzeros-per-row class, row-count class), as text into
 * buf[0..len) (NUL-terminated, truncated to fit) */
int emg_spmm_layouts(char *buf, long len);

#ifdef __cplusplus
}
#endif
#endif
