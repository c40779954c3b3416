/* su2_oracle.h -- C restatement of the su2 reference hot path (TEST INFRASTRUCTURE ONLY).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs use this library,
 * as the checker.  The product library (su2_b200/libsu2b.so) never links or calls it.
 *
 * Host layout follows the reference (gaugeconfig.hh:211-222):
 *   link index  = ((((t*Lx+x)*Ly+y)*Lz+z)*nd + mu), coordinates c = {t, x, y, z}
 *   SU(2) link  = 4 doubles {Re a, Im a, Re b, Im b}, U = [[a, b], [-b*, a*]] (su2.hh:11-70)
 *   U(1)  link  = 1 double angle                                             (u1.hh:11-59)
 *   adjoint     = 3 doubles (SU(2)) / 1 double (U(1))                (adjointfield.hh:12-81)
 *   spinor      = 2 doubles per site, site = ((t*Lx+x)*Ly+y)*Lz+z     (staggered.hpp:52-69)
 * group: 0 = SU(2), 1 = U(1).
 */
#ifndef SU2_ORACLE_H
#define SU2_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- random numbers -------------------------------------------------------------- */
typedef struct {
  uint32_t mt[624];
  int idx;
} orc_mt19937;
void orc_mt_seed(orc_mt19937 *g, uint32_t seed);
uint32_t orc_mt_next(orc_mt19937 *g);
double orc_canonical(orc_mt19937 *g);
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* ---- gauge fields ---------------------------------------------------------------- */
void orc_hotstart(int group, int Lx, int Ly, int Lz, int Lt, int nd, int seed, double delta,
                  int trafo_seed, double *out);
void orc_random_gauge_trafo(int group, int Lx, int Ly, int Lz, int Lt, int nd, int seed,
                            double *U);
double orc_retr_sum_plaquettes(int group, int Lx, int Ly, int Lz, int Lt, int nd,
                               const double *U, double xi, int aniso, int spatial_only);
double orc_gauge_energy(int group, int Lx, int Ly, int Lz, int Lt, int nd, const double *U,
                        int spatial_only);
double orc_S_G_hmc(int group, int Lx, int Ly, int Lz, int Lt, int nd, double beta,
                   const double *U, double xi, int aniso);
void orc_gauge_derivative(int group, int Lx, int Ly, int Lz, int Lt, int nd, double beta,
                          double xi, const double *U, double fac, double *deriv);
void orc_restore_su(int group, int Lx, int Ly, int Lz, int Lt, int nd, double *U);
void orc_update_gauge(int group, int Lx, int Ly, int Lz, int Lt, int nd, double *U,
                      const double *P, double dtau);
void orc_exp_su2(const double x[3], double out[4]);

/* integrators: ids as the reference enum (integrator.hh:15):
 * 0 leapfrog, 2 omf4, 4 euler, 5 ruth, 6 omf2 */
void orc_integrate(int group, int Lx, int Ly, int Lz, int Lt, int nd, double beta, double xi,
                   int integ, int nsteps, double tau, double *U, double *P);
double orc_md_injected(int group, int Lx, int Ly, int Lz, int Lt, int nd, double beta,
                       double xi, int integ, int nsteps, double tau, double *U, double *P,
                       double *H);
double orc_md_injected_lp(int group, int Lx, int Ly, int Lz, int Lt, int nd, double beta,
                          double xi, int integ, int nsteps, double tau, double *U, double *P,
                          double *H, int exponent);
double orc_initnormal(int group, int Lx, int Ly, int Lz, int Lt, int nd, long seed, double *P);
void orc_hmc_run(int group, int Lx, int Ly, int Lz, int Lt, int nd, double beta, double xi,
                 int integ, int nsteps, double tau, long seed, int i0, int ntraj, double *U,
                 int *acc, double *dH, double *plaq);

/* ---- observables, flow ----------------------------------------------------------- */
void orc_energy_density(int group, int Lx, int Ly, int Lz, int Lt, int nd, const double *U,
                        int cloverdef, int ss, double *E, double *Q);
void orc_runge_kutta(int group, int Lx, int Ly, int Lz, int Lt, int nd, double beta,
                     double xi, double eps, double *U);
/* rows of 9 doubles {t, xi_R, P, P_ss, Ep, Ep_ss, Ec, Ec_ss, Q}; returns the row count */
int orc_gradient_flow(int group, int Lx, int Ly, int Lz, int Lt, int nd, double beta,
                      double xi, const double *U, double tmax, double eps, double tstart,
                      double *rows, int max_rows);

/* ---- staggered fermions (U(1)) ----------------------------------------------------- */
double orc_eta(int t, int x, int y, int z, int mu);
void orc_staggered_apply(int Lx, int Ly, int Lz, int Lt, int nd, const double *U, double m,
                         int op, const double *in, double *out);
long orc_cg_ddag(int Lx, int Ly, int Lz, int Lt, int nd, const double *U, double m,
                 const double *b, const double *x0, double tol, double *x);
long orc_bicgstab_d(int Lx, int Ly, int Lz, int Lt, int nd, const double *U, double m,
                    const double *b, const double *x0, double tol, double *x);
void orc_gaussian_spinor(int Lx, int Ly, int Lz, int Lt, double avr, double sigma, long seed,
                         double *out);
void orc_ddag_inv(int Lx, int Ly, int Lz, int Lt, int nd, const double *U, double m,
                  const double *psi, double tol, long seed, double *x);
double orc_fermion_heatbath(int Lx, int Ly, int Lz, int Lt, int nd, const double *U, double m,
                            long seed_pf, double *phi);
double orc_fermion_accept(int Lx, int Ly, int Lz, int Lt, int nd, const double *U, double m,
                          const double *phi, double tol, long seed);
void orc_fermion_derivative(int Lx, int Ly, int Lz, int Lt, int nd, const double *U, double m,
                            const double *phi, double tol, long seed, double *deriv);
void orc_fermion_force_from_chi(int Lx, int Ly, int Lz, int Lt, int nd, const double *U,
                                double m, const double *chi, double *deriv);
double orc_md_injected_fermion(int Lx, int Ly, int Lz, int Lt, int nd, double beta, double m,
                               double tol, long seed, int integ, int nsteps, double tau,
                               double *U, double *P, const double *R, double *H);
double orc_md_injected_fermion_lp(int Lx, int Ly, int Lz, int Lt, int nd, double beta,
                                  double m, double tol, long seed, int integ, int nsteps,
                                  double tau, double *U, double *P, const double *R, double *H,
                                  int exponent);
/* number of solve() passes of the last Krylov solve (1 + restarts, CG.hpp:78-84) */
long orc_last_solve_calls(void);
/* dense complex n x n (row-major interleaved) solvers for the reference's 3x3 tests */
long orc_cg_dense(int n, const double *A, const double *b, const double *x0, double tol,
                  double *x);
long orc_bicgstab_dense(int n, const double *A, const double *b, const double *x0, double tol,
                        double *x);

/* ---- the device algorithms' own random streams (Philox4x32-10) --------------------- */
void orc_philox_momenta(int group, int Lx, int Ly, int Lz, int Lt, int nd, uint64_t seed,
                        uint32_t traj, double *P);
double orc_philox_accept_uniform(uint64_t seed, uint32_t traj);
void orc_philox_pf_source(int Lx, int Ly, int Lz, int Lt, uint64_t seed, uint32_t traj,
                          int complex_source, double *R);
void orc_metropolis_checkerboard(int group, int Lx, int Ly, int Lz, int Lt, int nd,
                                 double beta, double xi, double delta, int N_hit, uint64_t seed,
                                 uint32_t sweep, double *U, double *rates);

#ifdef __cplusplus
}
#endif
double orc_polyakov_loop(int group, int Lx, int Ly, int Lz, int Lt, int nd, const double *U);
double orc_wilson_loop(int group, int Lx, int Ly, int Lz, int Lt, int nd, const double *U,
                       int r, int t);
void orc_ape_smear(int group, int Lx, int Ly, int Lz, int Lt, int nd, double alpha,
                   int spatial, double *U);
void orc_pion_correlator(int Lx, int Ly, int Lz, int Lt, int nd, const double *U, double m,
                         double tol, long seed, double *C);
#endif
