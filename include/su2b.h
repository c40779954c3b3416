/* su2b.h -- C ABI of libsu2b, the B200 (sm_100a) device path for the Monte-Carlo hot path
 * of the su2 lattice gauge theory code.
 *
 * The su2 host driver (YAML input, gaugeconfig I/O, observables) keeps running on the CPU
 * and calls these entry points instead of the OpenMP loops named beside each declaration
 * (file:line in the su2 sources).  The gauge field lives on the device between calls; the
 * host copy in gaugeconfig<G> is refreshed only where the driver needs it (save points,
 * host-side observables) with su2b_download_gauge.
 *
 * Conventions
 *   - Every call returns an int status (SU2B_OK == 0) and never aborts; the message of the
 *     last error of a context is available from su2b_last_error().
 *   - Host buffers belong to the caller and use the reference's host layout:
 *       links   : gaugeconfig.hh:211-222, index ((((t*Lx+x)*Ly+y)*Lz+z)*ndims + mu);
 *                 SU(2): 4 doubles {Re a, Im a, Re b, Im b} per link (su2.hh:11-70, the
 *                 N_c member of _su2 is not part of the buffer); U(1): 1 double (angle).
 *       adjoint : 3 doubles {a, b, c} (SU(2), adjointfield.hh:12-51) or 1 double (U(1))
 *                 per link, same link order.
 *       spinor  : 2 doubles {Re, Im} per site, site = ((t*Lx+x)*Ly+y)*Lz+z
 *                 (staggered.hpp:52-69).
 *   - A context owns its device memory and one CUDA stream; calls on one context are not
 *     re-entrant, distinct contexts may be used from distinct host threads.
 *   - All active extents must be even (even/odd device layout, checkerboard updates).
 */
#ifndef SU2B_H
#define SU2B_H

#include <stddef.h>
#include <stdint.h>

#if defined(SU2B_BUILD) && defined(__GNUC__)
#define SU2B_API __attribute__((visibility("default")))
#else
#define SU2B_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------- */
enum {
  SU2B_OK = 0,
  SU2B_ERR_INVALID = 1,         /* bad argument (NULL pointer, size, id) */
  SU2B_ERR_CUDA = 2,            /* a CUDA runtime call or kernel launch failed */
  SU2B_ERR_NOT_CONVERGED = 3,   /* Krylov solver hit max_iter or produced a NaN residual */
  SU2B_ERR_UNSUPPORTED = 4,     /* valid request the reference also rejects (e.g. SU(2)
                                   staggered fermions, staggered.hpp:343-350) */
  SU2B_ERR_NOMEM = 5,           /* device allocation failed */
  SU2B_ERR_TIMEOUT = 6          /* a bounded device-side wait gave up */
};

enum { SU2B_GROUP_SU2 = 0, SU2B_GROUP_U1 = 1 };

/* SU2B_PREC_FP64: links, momenta, forces in FP64 (the plain path).
 * SU2B_PREC_MIXED: SU(2) links, momenta and forces stored and computed in FP32; every
 *   global reduction (plaquette, action, kinetic energy, Delta H), the accept/reject and
 *   link reunitarisation in FP64.  For U(1) the links stay FP64 and MIXED selects FP32
 *   inner iterations with FP64 reliable updates in the CG. */
enum { SU2B_PREC_FP64 = 0, SU2B_PREC_MIXED = 1 };

/* integrator ids as the reference enum (integrator.hh:15) */
enum {
  SU2B_LEAPFROG = 0,
  SU2B_LP_LEAPFROG = 1, /* leapfrog with rounding (integrator.hh:53-80) */
  SU2B_OMF4 = 2,
  SU2B_LP_OMF4 = 3,     /* omf4 with rounding (integrator.hh:158-199) */
  SU2B_EULER = 4,
  SU2B_RUTH = 5,
  SU2B_OMF2 = 6
};

typedef struct su2b_ctx su2b_ctx;

/* ---- context ------------------------------------------------------------------------- */

/* Creates a device-resident lattice.  Extents and ndims follow gaugeconfig(Lx, Ly, Lz, Lt,
 * ndims, beta) (gaugeconfig.hh:49-63); for ndims < 4 pass Lz = 1 (and Ly = 1 for ndims = 2)
 * as parse_input_file.cc:57-67 does.  xi != 1 selects the anisotropic action
 * (flat-gaugemonomial.hh:196-202).  device = CUDA ordinal. */
SU2B_API int su2b_ctx_create(int group, int Lx, int Ly, int Lz, int Lt, int ndims, double beta,
                    double xi, int precision, int device, su2b_ctx **out);
SU2B_API int su2b_ctx_destroy(su2b_ctx *ctx);
SU2B_API const char *su2b_last_error(const su2b_ctx *ctx);
/* the context's CUDA stream (a cudaStream_t), for callers that order their own work */
SU2B_API int su2b_ctx_stream(su2b_ctx *ctx, void **stream);
SU2B_API int su2b_set_beta(su2b_ctx *ctx, double beta);
/* blocks until all work queued on the context's stream has finished */
SU2B_API int su2b_synchronize(su2b_ctx *ctx);

/* ---- gauge field transfer (gaugeconfig<G> <-> device) ------------------------------- */
SU2B_API int su2b_upload_gauge(su2b_ctx *ctx, const double *U_host);
SU2B_API int su2b_download_gauge(su2b_ctx *ctx, double *U_host);

/* ---- reductions ---------------------------------------------------------------------- */

/* flat_spacetime::gauge_energy(U, spatial_only) (flat-gauge_energy.hpp:109-137):
 * sum_x sum_{mu<nu} ReTr P_{mu nu}(x). */
SU2B_API int su2b_gauge_energy(su2b_ctx *ctx, int spatial_only, double *out);
/* flat_spacetime::retr_sum_Wplaquettes(U, xi, anisotropic, spatial_only)
 * (flat-gauge_energy.hpp:31-94), with the context's xi. */
SU2B_API int su2b_retr_sum_plaquettes(su2b_ctx *ctx, int spatial_only, double *out);
/* flat_spacetime::get_S_G_hmc (flat-gaugemonomial.hh:46-54): -beta/Nc * retr sum */
SU2B_API int su2b_gauge_action(su2b_ctx *ctx, double *out);
/* flat_spacetime::energy_density(U, E, Q, cloverdef, ss) (flat-energy_density.hh:57-164) */
SU2B_API int su2b_energy_density(su2b_ctx *ctx, int cloverdef, int ss, double *E, double *Q);

/* ---- gauge force and updates --------------------------------------------------------- */

/* gaugemonomial::derivative(deriv, h, fac) (flat-gaugemonomial.hh:105-131) into a zeroed
 * field: deriv(x,mu) = fac*beta/Nc * get_deriv(U(x,mu) * staples(x,mu)). */
SU2B_API int su2b_gauge_force(su2b_ctx *ctx, double fac, double *deriv_host);
/* gaugeconfig::restoreSU (gaugeconfig.hh:115-120) */
SU2B_API int su2b_restore_su(su2b_ctx *ctx);
/* update_gauge(h, dtau) (update_gauge.hh:8-16) with momenta given on the host */
SU2B_API int su2b_update_gauge(su2b_ctx *ctx, const double *P_host, double dtau);

/* ---- HMC trajectory (md_update, md_update.hh:18-81) ------------------------------------ */
typedef struct {
  int integrator;   /* SU2B_LEAPFROG, SU2B_OMF2, ... */
  int n_steps;      /* md_params nsteps */
  double tau;       /* md_params tau */
  uint64_t seed;    /* key of the device random streams */
  uint32_t traj;    /* trajectory index (counter of the device random streams) */
  int revtest;      /* reversibility test (md_update.hh:62-74): fills ddH */
  int accept_reject;/* 0: always accept (md_params acceptreject) */
  /* optional host inputs for replaying a host random stream (all NULL/negative = device
   * Philox streams): momenta in the adjoint host layout, and the accept uniform. */
  const double *momenta_host;
  double uniform_host;  /* used when >= 0 */
  /* U(1) only: staggered det(D Ddag) monomial (detDDdag_monomial.hh).  Enabled when
   * fermion_mass > 0. */
  double fermion_mass;
  double cg_tol;          /* absolute residual tolerance of the inner CG (CG.hpp:50) */
  int cg_max_iter;
  const double *pf_source_host; /* optional R (spinor host layout); NULL = Philox R */
  int pf_complex;         /* 0: real R as the reference (staggered.hpp:188-191) */
  int cg_start;           /* SU2B_CG_START_*: start vector of every inner CG */
  long pf_seed;           /* seed of the reference's sigma=10 Gaussian CG start */
  /* SU2B_LP_LEAPFROG / SU2B_LP_OMF4 only (FP64 links: a context with FP32 SU(2) links
   * returns SU2B_ERR_UNSUPPORTED for them), 0..19: before each momentum step the summed
   * derivative, and before each gauge step every link, is rounded componentwise to
   * round(x * 10^e) / 10^e (update_momenta.hh:36-58, update_gauge.hh:20-26; a U(1) link
   * angle a becomes round(a) * 10^e / 10^e as u1.hh:31-33 writes it).  The reference's
   * command-line default is 0. */
  int round_exponent;
} su2b_hmc_params;

typedef struct {
  int accepted;
  double dH;            /* Delta H summed over the monomials */
  double ddH;           /* reversibility violation (revtest only) */
  double H_old[3];      /* kinetic, gauge, fermion */
  double H_new[3];
  double plaquette;     /* gauge_energy after the accept/reject */
  long cg_iterations;   /* total inner CG iterations (fermions only) */
} su2b_traj_result;

SU2B_API int su2b_hmc_trajectory(su2b_ctx *ctx, const su2b_hmc_params *prm, su2b_traj_result *res);

/* ---- Metropolis (flat_spacetime::sweep, flat-sweep.hh:64-164) -------------------------- */
/* Device order: site-parity checkerboard, one pass per (mu, parity); proposal and accept
 * rule as the reference; random numbers from Philox(seed, {link, hit, sweep}).
 * rates[0] = accepted/(N_hit*links), rates[1] = temporal ones/(N_hit*volume). */
SU2B_API int su2b_metropolis_sweep(su2b_ctx *ctx, double delta, int N_hit, uint64_t seed,
                          uint32_t sweep, double *rates);

/* ---- Wilson flow (flat-gradient_flow.hh) --------------------------------------------- */
/* One Lüscher RK3 step of runge_kutta (flat-gradient_flow.hh:17-50) on the context's
 * links (in place). */
SU2B_API int su2b_flow_step(su2b_ctx *ctx, double eps);
/* gradient_flow (flat-gradient_flow.hh:70-197) on a copy of the links: rows of 9 doubles
 * {t, xi_R, P, P_ss, Ep, Ep_ss, Ec, Ec_ss, Q}, recorded at the middle of every pair of
 * steps as the reference prints them.  *n_rows receives the number of records. */
SU2B_API int su2b_gradient_flow(su2b_ctx *ctx, double tmax, double eps, double tstart, double *rows,
                       int max_rows, int *n_rows);

/* ---- staggered fermions, U(1) only (staggered.hpp) ------------------------------------- */
enum { SU2B_OP_D = 0, SU2B_OP_DDAG = 1, SU2B_OP_DDDAG = 2 };
/* apply_D / apply_Ddag / D*Ddag (staggered.hpp:290-389) */
SU2B_API int su2b_staggered_apply(su2b_ctx *ctx, int op, double mass, const double *psi_host,
                         double *out_host);

/* start vector of the CG inside the fermion monomial: the reference's real Gaussian with
 * sigma = 10 drawn from std::mt19937(seed) (staggered.hpp:267-268), or zero */
enum { SU2B_CG_START_REFERENCE = 0, SU2B_CG_START_ZERO = 1 };

enum { SU2B_SOLVER_CG = 0, SU2B_SOLVER_BICGSTAB = 1, SU2B_SOLVER_CG_MIXED = 2 };
enum { SU2B_TOL_ABS = 0, SU2B_TOL_REL = 1 };
typedef struct {
  int solver;     /* CG on D Ddag (CG.hpp), BiCGStab on D (BiCGStab.hpp), mixed CG */
  int op;         /* SU2B_OP_DDDAG for CG, SU2B_OP_D for BiCGStab */
  double mass;
  double tol;     /* residual norm bound */
  int tol_mode;   /* SU2B_TOL_ABS (the reference, CG.hpp:50) or SU2B_TOL_REL (tol*|b|) */
  int max_iter;
  double delta;   /* mixed CG: reliable-update threshold (0 = default 0.1) */
} su2b_solve_params;
typedef struct {
  long iterations;
  long restarts;          /* true-residual restarts (CG.hpp:78-84) / reliable updates */
  double residual;        /* final iterated residual norm */
  double true_residual;   /* |b - A x| recomputed in FP64 */
} su2b_solve_stats;
/* LinearCG::solve / LinearBiCGStab::solve; x0_host NULL = zero start */
SU2B_API int su2b_solve(su2b_ctx *ctx, const su2b_solve_params *prm, const double *b_host,
               const double *x0_host, double *x_host, su2b_solve_stats *stats);
/* detDDdag_monomial::derivative (detDDdag_monomial.hh:112-167): CG from x0 (NULL = the
 * reference's sigma=10 Gaussian start of DDdag_matrix_lat::inv drawn with `seed`), then the
 * per-link contraction; deriv_host receives the force (not accumulated). */
SU2B_API int su2b_fermion_force(su2b_ctx *ctx, double mass, const double *phi_host, double tol,
                       int max_iter, const double *x0_host, long seed, double *deriv_host,
                       long *cg_iterations);
/* detDDdag_monomial::accept (detDDdag_monomial.hh:93-103): Re phi^+ (D Ddag)^-1 phi */
SU2B_API int su2b_fermion_action(su2b_ctx *ctx, double mass, const double *phi_host, double tol,
                        int max_iter, const double *x0_host, long seed, double *out);

/* staggered::C_pion (propagator.hpp:25-65): pion correlator at rest, C[t] = sum_x |D^-1(x|0)|^2
 * / Vs over the time slice t, with D^-1 = D^+ (D D^+)^-1 from one CG solve (tolerance as the
 * reference's absolute |r| bound, start gaussian_spinor(0, 10, seed)); C[0] = 0 as the
 * reference skips the contact term.  C_host receives Lt values.  U(1) only. */
SU2B_API int su2b_pion_correlator(su2b_ctx *ctx, double mass, double tol, int max_iter,
                                  long seed, double *C_host, long *cg_iterations);

/* ---- batched ensembles of independent SU(2) chains ------------------------------------------ */
/* Chains of different geometry (d = 3 or 4, even extents), coupling and seed advanced together:
 * every stage of a trajectory is one persistent launch over all chains, a trajectory is one
 * CUDA graph, and each chain keeps its own accept/reject (md_update.hh:18-81).  A chain's
 * trajectory equals the one of a single-lattice context with the same seed and traj. */
typedef struct {
  int Lx, Ly, Lz, Lt, ndims;
  double beta;
  uint64_t seed;
} su2b_chain_desc;
typedef struct su2b_batch su2b_batch;
SU2B_API int su2b_batch_create(int n_chains, const su2b_chain_desc *chains, int precision,
                               int device, su2b_batch **out);
SU2B_API int su2b_batch_destroy(su2b_batch *b);
SU2B_API const char *su2b_batch_last_error(const su2b_batch *b);
SU2B_API int su2b_batch_stream(su2b_batch *b, void **stream);
SU2B_API int su2b_batch_kernel_launches(su2b_batch *b, long *count);
SU2B_API int su2b_batch_upload(su2b_batch *b, int chain, const double *U_host);
SU2B_API int su2b_batch_download(su2b_batch *b, int chain, double *U_host);
/* one trajectory (SU2B_LEAPFROG or SU2B_OMF2) of every chain; results[n_chains] */
SU2B_API int su2b_batch_hmc(su2b_batch *b, int integrator, int n_steps, double tau, uint32_t traj,
                            su2b_traj_result *results);
/* Launch shapes of the batched kernels (threads per block 64/128/128/256, the tile of a block
 * being half that many sites of each parity of one chain; force-kernel register caps from
 * 8/4/6/3 resident blocks per SM).  su2b_batch_autotune times the batched force step of each
 * shape on the ensemble's current fields (without changing them), keeps the fastest and
 * writes the microseconds per launch to times_us (SU2B_BATCH_VARIANTS entries, may be NULL). */
#define SU2B_BATCH_VARIANTS 4
SU2B_API int su2b_batch_autotune(su2b_batch *b, double *times_us);
SU2B_API int su2b_batch_tune_get(su2b_batch *b, int *variant);
SU2B_API int su2b_batch_tune_set(su2b_batch *b, int variant);

/* ---- one lattice over time slabs ------------------------------------------------------------ */
/* The t-slab decomposition of one SU(2) lattice: the lattice is cut into nslabs slabs of
 * Lt / nslabs time slices (an even number).  A slab holds its slices and one ghost slice of
 * links on each side.  A trajectory runs every force step on each slab's own sites, then
 * refreshes the ghost slices from the neighbouring slabs; the plaquette and kinetic sums add
 * over the slabs before the accept/reject.  The momenta are the Philox streams of the whole
 * lattice, so a trajectory equals the one of a single-lattice context (su2b_hmc_trajectory)
 * with the same seed and traj: the same links and accept decisions, the energies to rounding
 * (the sums add in another order).  The reference splits the same site loops over OpenMP
 * threads along t (flat-gaugemonomial.hh:105-131, flat-sweep.hh:83,128).
 * A handle holds the slabs first .. first + count - 1.  With count == nslabs every slab lives
 * on one device and the ghost slices are device copies.  With one slab per process
 * (count == 1, one GPU each) the handles exchange ghost slices and sums through NCCL
 * (su2b_slabs_connect; NCCL is loaded at run time from libnccl.so.2).
 * Trajectories: leapfrog, omf2 and omf4 with Philox momenta (momenta_host, revtest and
 * fermions return SU2B_ERR_UNSUPPORTED).  Lt % nslabs != 0 or an odd Lt / nslabs return
 * SU2B_ERR_INVALID. */
typedef struct su2b_slabs su2b_slabs;
SU2B_API int su2b_slabs_create(int Lx, int Ly, int Lz, int Lt, int ndims, double beta,
                               double xi, int precision, int nslabs, int first, int count,
                               int device, su2b_slabs **out);
SU2B_API int su2b_slabs_destroy(su2b_slabs *h);
SU2B_API const char *su2b_slabs_last_error(const su2b_slabs *h);
SU2B_API int su2b_slabs_info(const su2b_slabs *h, int *nslabs, int *first, int *count,
                             int *slices);
/* ncclGetUniqueId into id (128 bytes), for one process to pass to the others */
SU2B_API int su2b_slabs_nccl_id(void *id);
/* joins the NCCL communicator of nranks = nslabs processes; rank = the handle's slab */
SU2B_API int su2b_slabs_connect(su2b_slabs *h, const void *id, int nranks, int rank);
/* U_host: the whole lattice's field in the reference host layout; upload takes each slab's
 * slices and ghost slices from it, download writes the handle's slabs' slices into it */
SU2B_API int su2b_slabs_upload(su2b_slabs *h, const double *U_host);
SU2B_API int su2b_slabs_download(su2b_slabs *h, double *U_host);
SU2B_API int su2b_slabs_hmc_trajectory(su2b_slabs *h, const su2b_hmc_params *prm,
                                       su2b_traj_result *res);
/* flat_spacetime::sweep over the slabs (as su2b_metropolis_sweep: the same links, the same
 * acceptance rates of the whole lattice) */
SU2B_API int su2b_slabs_metropolis_sweep(su2b_slabs *h, double delta, int N_hit, uint64_t seed,
                                         uint32_t sweep, double *rates);
/* the Wilson flow over the slabs: runge_kutta on the current field (as su2b_flow_step),
 * energy_density and gradient_flow of the whole lattice (as su2b_energy_density and
 * su2b_gradient_flow, the same rows); each RK3 stage exchanges the ghost slices it wrote */
SU2B_API int su2b_slabs_flow_step(su2b_slabs *h, double eps);
SU2B_API int su2b_slabs_energy_density(su2b_slabs *h, int cloverdef, int ss, double *E,
                                       double *Q);
SU2B_API int su2b_slabs_gradient_flow(su2b_slabs *h, double tmax, double eps, double tstart,
                                      double *rows, int max_rows, int *n_rows);
/* gauge_energy of the whole lattice (as su2b_gauge_energy) */
SU2B_API int su2b_slabs_gauge_energy(su2b_slabs *h, int spatial_only, double *out);
/* su2b_autotune on the first slab of the handle; every slab takes its choice.  Slabs in
 * separate processes (a collective call: every rank calls it) reduce each shape's time to its
 * maximum over the ranks and choose from those, so every rank runs the same shape; times_us
 * (SU2B_FORCE_VARIANTS entries, may be NULL) receives the times the choice was made from. */
SU2B_API int su2b_slabs_autotune(su2b_slabs *h, double *times_us);
SU2B_API int su2b_slabs_tune_get(su2b_slabs *h, int *variant);
SU2B_API int su2b_slabs_tune_set(su2b_slabs *h, int variant);
/* Overlap (on by default after su2b_slabs_connect, off for slabs on one device): each force
 * step updates the two boundary slices of every slab first, exchanges their faces on a second
 * stream of the highest priority while the interior slices are updated, and the next step
 * waits for the exchange.  Slabs of fewer than four slices run without it.  The results are
 * the same either way; the split launches pay off against NCCL's latency, not against a
 * device copy. */
SU2B_API int su2b_slabs_set_overlap(su2b_slabs *h, int on);
SU2B_API int su2b_slabs_get_overlap(const su2b_slabs *h, int *on);
SU2B_API int su2b_slabs_kernel_launches(su2b_slabs *h, long *count);
SU2B_API int su2b_slabs_stream(su2b_slabs *h, void **stream);

/* ---- gauge configurations on disk ------------------------------------------------------- */
/* gaugeconfig<G>::save / load (gaugeconfig.hh:225-252): the reference's raw binary format, one
 * in-memory _su2 (40 bytes: size_t N_c = 2, then Re a, Im a, Re b, Im b) or _u1 (16 bytes:
 * size_t N_c = 1, then the angle) object per link in the host link order.  Records are built
 * and parsed on the device; load checks every N_c against the group and fails on a file
 * shorter than the lattice.  FP32 contexts store FP32 links widened to double. */
SU2B_API int su2b_save_gauge(su2b_ctx *ctx, const char *path);
SU2B_API int su2b_load_gauge(su2b_ctx *ctx, const char *path);
/* io::update_nconf_counter (io.hh:294-305): writes conf_dir + "nconf_counter.txt" as the
 * header line "heat i path_conf" and the line "<heat> <i> <path_conf>" (heat printed as 0 or
 * 1, no trailing newline).  conf_dir is prefixed as given, as in the reference.  Host only:
 * needs no context and no GPU. */
SU2B_API int su2b_update_nconf_counter(const char *conf_dir, int heat, long i,
                                       const char *path_conf);
/* io::read_nconf_counter (io.hh:267-285): reads the second line of conf_dir +
 * "nconf_counter.txt" and splits it at spaces into heat (0 or 1), i and path_conf (copied
 * into path_buf, at most path_cap bytes with the terminating NUL).  Fails with
 * SU2B_ERR_INVALID where the reference aborts (a missing file) or would throw (a malformed
 * line).  Host only. */
SU2B_API int su2b_read_nconf_counter(const char *conf_dir, int *heat, long *i, char *path_buf,
                                     size_t path_cap);
/* the restart of base_program.hpp:284-296: read the counter in conf_dir and load the
 * configuration it names into the context; heat and i as the counter holds them */
SU2B_API int su2b_restart(su2b_ctx *ctx, const char *conf_dir, int *heat, long *i);

/* ---- observables between trajectories ---------------------------------------------------- */
/* polyakov_loop_spatial_average (polyakov_loop.hh:48-63): sum over spatial points of ReTr of
 * the product of the temporal links, divided by the full volume as the reference does. */
SU2B_API int su2b_polyakov_loop(su2b_ctx *ctx, double *out);
/* wilsonloop(U, r, t) (wilsonloop.hh:147-157): r x t planar loops in the (mu, 0) planes,
 * mu >= 1, summed over sites, divided by V Nc ndims. */
SU2B_API int su2b_wilson_loop(su2b_ctx *ctx, int r, int t, double *out);
/* APEsmearing(U, alpha, spatial) (smearape.hh:97-131) of the context's links, in place. */
SU2B_API int su2b_ape_smear(su2b_ctx *ctx, double alpha, int spatial);

/* ---- derivatives (SU(2)) ------------------------------------------------------------------ */
/* Left Lie-algebra derivatives, the convention of gaugemonomial::derivative
 * (flat-gaugemonomial.hh:105-131): grad(x,mu)_k = d/dw O(exp(w e_k) U_mu(x)) at w = 0 with
 * exp of exp_gauge.cc:8-18.  Results use the adjoint host layout. */
/* Wilson action S = get_S_G_hmc (flat-gaugemonomial.hh:46-54) into *S (may be NULL) and
 * grad_out * dS/dU into dS_host (may be NULL); dS/dU is the gauge force with fac = 1. */
SU2B_API int su2b_action_backward(su2b_ctx *ctx, double grad_out, double *S, double *dS_host);
/* Vector-Jacobian product of the force field g(U)(x,mu) = get_deriv(U_mu(x) K_mu(x)):
 * out = (dg/dU)^T mu, i.e. the left derivative of sum mu.g (a Hessian-vector product of the
 * Wilson action up to beta/Nc). */
SU2B_API int su2b_force_vjp(su2b_ctx *ctx, const double *mu_host, double *out_host);
/* O = t^2 E_p(t) after n_steps Wilson-flow RK3 steps (runge_kutta, flat-gradient_flow.hh:
 * 17-50) of size eps from the context's links, t = n_steps*eps, E_p = d(d-1)/2 - P/(V Nc)
 * the plaquette energy of gradient_flow (flat-gradient_flow.hh:151); *objective receives O
 * and grad_host (NULL: objective only) its derivative with respect to the starting links,
 * by the adjoint of the RK3 steps with checkpoints every checkpoint_every steps
 * (0 = sqrt(n_steps)).  The links are not modified. */
SU2B_API int su2b_flow_adjoint(su2b_ctx *ctx, double eps, int n_steps, int checkpoint_every,
                               double *objective, double *grad_host);

/* ---- launch-shape autotuning ------------------------------------------------------------ */
/* The SU(2) force kernel has SU2B_FORCE_VARIANTS launch shapes (threads per block x register
 * cap).  su2b_autotune times them all on the context's field (CUDA events over launches
 * chained by programmatic dependent launch as in a trajectory, the same memory traffic as a
 * trajectory step, into scratch buffers) and keeps the fastest for this context
 * (the first shape in index order within 1 % of the fastest: shapes that tie round
 * differently, and this keeps the choice, and so the chain, the same from run to run);
 * with cache_path it first looks the choice up in that text file (unless retune) and writes
 * new measurements to it.  times_us (optional, SU2B_FORCE_VARIANTS entries) receives the
 * average launch time of each shape (-1 when not measured). */
#define SU2B_FORCE_VARIANTS 12
/* SU2B_TUNE_TRAJECTORY selects how su2b_hmc_trajectory runs an SU(2) trajectory without
 * fermions, reversibility test or rounding:
 *   SU2B_TRAJ_FUSED_GRAPH (default): each momentum step fused with the gauge step after it,
 *     three link buffers (no copy of the start field), the whole trajectory one CUDA graph;
 *   SU2B_TRAJ_PLAIN: the plain form, as md_update is written -- the start field copied, the
 *     integrator's momentum steps (staples, force and momentum update in one kernel) and
 *     gauge steps launched one by one, restoreSU, the plaquette sums, the accept launch.  It
 *     keeps the context's force launch shape (an untuned context has the default one).
 * Both give the same trajectory up to rounding. */
enum { SU2B_TUNE_FORCE = 0, SU2B_TUNE_TRAJECTORY = 1 };
enum { SU2B_TRAJ_FUSED_GRAPH = 0, SU2B_TRAJ_PLAIN = 1 };
SU2B_API int su2b_autotune(su2b_ctx *ctx, const char *cache_path, int retune, double *times_us);
SU2B_API int su2b_tune_get(su2b_ctx *ctx, int kernel, int *variant);
SU2B_API int su2b_tune_set(su2b_ctx *ctx, int kernel, int variant);

/* ---- plaquette sums without allocation ------------------------------------------------ */
/* No counterpart in the reference.  For callers that cannot allocate device memory (a host
 * framework that owns the GPU's memory through its own pool and forbids cudaMalloc in
 * plug-ins, or code running during CUDA graph capture): gauge_energy(U) and
 * gauge_energy(U, spatial_only) of a field the caller already holds on the device in the
 * reference host layout (FP64, see "links" above), written to out_dev[0] and out_dev[1] (a
 * device buffer of the caller) on `stream` (a cudaStream_t, NULL = default stream).  No
 * context is created and nothing is allocated: the only scratch is a fixed array of
 * 16384 partial-sum pairs inside the library, so the lattice may have at most 4,194,304
 * sites (larger sizes return SU2B_ERR_INVALID).  All calls share that array: calls that
 * overlap on the GPU race and must be ordered by the caller.  Each call outside a stream
 * capture looks up the array's device address in the current context; a call during a
 * capture reuses the address found by the last call outside one, so the first call on a
 * device should come before any stream capture.  Returns without waiting for the kernels;
 * errors are reported only through the status code. */
SU2B_API int su2b_gauge_energy_noalloc(int group, int Lx, int Ly, int Lz, int Lt, int ndims,
                                       const double *U_dev, double *out_dev, void *stream);

/* ---- device timers -------------------------------------------------------------------- */
/* Kernel classes.  With profiling on, every launch of a class is bracketed by CUDA events on
 * the context's stream and its device time accumulated (the events add a few microseconds
 * per launch; leave profiling off for headline timings). */
enum {
  SU2B_K_FORCE = 0,      /* fused staple / force / momentum update */
  SU2B_K_UPDATE = 1,     /* U <- exp(dt P) U */
  SU2B_K_PLAQUETTE = 2,  /* plaquette / action partial sums */
  SU2B_K_MOMENTA = 3,    /* Philox momenta + kinetic partial sums */
  SU2B_K_RESTORE = 4,    /* reunitarisation */
  SU2B_K_METROPOLIS = 5, /* checkerboard Metropolis pass */
  SU2B_K_CLOVER = 6,     /* clover energy density / charge */
  SU2B_K_STAGGERED = 7,  /* staggered D / Ddag and fermion force */
  SU2B_K_OTHER = 8,      /* reductions, solver vector updates, layout conversion */
  SU2B_K_COUNT = 9
};
/* enable (1) or disable (0) the timers; enabling clears the accumulated values */
SU2B_API int su2b_profile(su2b_ctx *ctx, int enable);
/* launches and total device milliseconds of one class since profiling was enabled
 * (synchronises the context's stream) */
SU2B_API int su2b_profile_read(su2b_ctx *ctx, int kclass, long *launches, double *total_ms);
/* number of kernels this context has launched since it was created */
SU2B_API int su2b_kernel_launches(su2b_ctx *ctx, long *count);

#ifdef __cplusplus
}
#endif
#endif
