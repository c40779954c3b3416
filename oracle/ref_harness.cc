// ref_harness.cc -- C-ABI wrapper around the UNMODIFIED su2 reference headers.
//
// TEST INFRASTRUCTURE ONLY.  This file is compiled (by oracle/Makefile) against the
// reference's own headers and exp_gauge.cc, where they lie in the reference checkout, into
// oracle/_ref/libsu2ref.so.  It is used to pin the C restatement (oracle/su2_oracle.c),
// to generate golden fixtures (tests/golden/make_golden.py) and as the timed CPU
// baseline (bench.py --impl reference).  No product code links it.
//
// Every entry point takes plain arrays in the reference's host layout
// (gaugeconfig.hh:211-222: idx = ((((t*Lx+x)*Ly+y)*Lz+z)*ndims+mu)):
//   SU(2) link  = 4 doubles [Re a, Im a, Re b, Im b]      (su2.hh:11-70)
//   U(1)  link  = 1 double  (angle)                         (u1.hh:11-59)
//   SU(2) adjoint = 3 doubles [a, b, c]                     (adjointfield.hh:12-51)
//   U(1)  adjoint = 1 double                                (adjointfield.hh:58-77)
//   spinor      = 2 doubles per site [Re, Im], site order t-major (staggered.hpp:52-69)
#include "adjointfield.hh"
#include "detDDdag_monomial.hh"
#include "flat-energy_density.hh"
#include "flat-gauge_energy.hpp"
#include "flat-gaugemonomial.hh"
#include "flat-gradient_flow.hh"
#include "flat-sweep.hh"
#include "gaugeconfig.hh"
#include "integrator.hh"
#include "md_params.hh"
#include "md_update.hh"
#include "monomial.hh"
#include "random_gauge_trafo.hh"
#include "staggered.hpp"
#include "polyakov_loop.hh"
#include "propagator.hpp"
#include "smearape.hh"
#include "wilsonloop.hh"

#ifdef _USE_OMP_
#include <omp.h>
#endif

#include <cstring>
#include <list>
#include <random>
#include <string>

namespace {

  template <class G> struct io;
  template <> struct io<_su2> {
    static void put(gaugeconfig<_su2> &U, const double *d) {
      for (size_t i = 0; i < U.getSize(); i++)
        U[i] = _su2(Complex(d[4 * i], d[4 * i + 1]), Complex(d[4 * i + 2], d[4 * i + 3]));
    }
    static void get(const gaugeconfig<_su2> &U, double *d) {
      for (size_t i = 0; i < U.getSize(); i++) {
        const _su2 u = U[i];
        d[4 * i] = u.geta().real();
        d[4 * i + 1] = u.geta().imag();
        d[4 * i + 2] = u.getb().real();
        d[4 * i + 3] = u.getb().imag();
      }
    }
    static void putP(adjointfield<double, _su2> &P, const double *d) {
      for (size_t i = 0; i < P.getSize(); i++)
        P[i] = adjointsu2<double>(d[3 * i], d[3 * i + 1], d[3 * i + 2]);
    }
    static void getP(const adjointfield<double, _su2> &P, double *d) {
      for (size_t i = 0; i < P.getSize(); i++) {
        d[3 * i] = P[i].geta();
        d[3 * i + 1] = P[i].getb();
        d[3 * i + 2] = P[i].getc();
      }
    }
  };
  template <> struct io<_u1> {
    static void put(gaugeconfig<_u1> &U, const double *d) {
      for (size_t i = 0; i < U.getSize(); i++) U[i] = _u1(d[i]);
    }
    static void get(const gaugeconfig<_u1> &U, double *d) {
      for (size_t i = 0; i < U.getSize(); i++) d[i] = U[i].geta();
    }
    static void putP(adjointfield<double, _u1> &P, const double *d) {
      for (size_t i = 0; i < P.getSize(); i++) P[i] = adjointu1<double>(d[i]);
    }
    static void getP(const adjointfield<double, _u1> &P, double *d) {
      for (size_t i = 0; i < P.getSize(); i++) d[i] = P[i].geta();
    }
  };

  using spinor = staggered::spinor_lat<double, Complex>;

  spinor make_spinor(const gaugeconfig<_u1> &U, const double *d) {
    spinor s({U.getLt(), U.getLx(), U.getLy(), U.getLz()});
    for (size_t i = 0; i < s.size(); i++) s[i] = Complex(d[2 * i], d[2 * i + 1]);
    return s;
  }
  void put_spinor(const spinor &s, double *d) {
    for (size_t i = 0; i < s.size(); i++) {
      d[2 * i] = s[i].real();
      d[2 * i + 1] = s[i].imag();
    }
  }

  // D alone as an LAmatrix for BiCGStab (staggered.hpp has no such wrapper; the
  // reference's solver selection never reaches BiCGStab, staggered.hpp:258-263).
  struct D_matrix {
    gaugeconfig<_u1> U;
    double m;
    size_t rows() const { return U.getVolume(); }
    size_t cols() const { return U.getVolume(); }
    void operator=(const D_matrix &o) {
      U = o.U;
      m = o.m;
    }
  };
  spinor operator*(const D_matrix &M, const spinor &psi) {
    return staggered::apply_D<double, Complex>(M.U, M.m, psi);
  }

  // exposes the number of stored iterates (one per iteration plus one per solve() call)
  template <class S> struct counted : public S {
    using S::S;
    size_t n_iterates() const { return this->curve_x.size(); }
  };

  template <class G> std::list<monomial<double, G> *> gauge_monomials(
    kineticmonomial<double, G> &km, flat_spacetime::gaugemonomial<double, G> &gm) {
    std::list<monomial<double, G> *> l;
    km.setmdpassive();
    l.push_back(&km);
    l.push_back(&gm);
    return l;
  }

  // the exponent matters to the low-precision integrators (ids 1, 3) only
  template <class G> integrator<double, G> *make_integrator(int id, int exponent = 16) {
    return set_integrator<double, G>(static_cast<size_t>(id), static_cast<size_t>(exponent));
  }

} // namespace

#define DISPATCH(group, ...)                                                               \
  do {                                                                                     \
    if ((group) == 0) {                                                                    \
      typedef _su2 G;                                                                      \
      __VA_ARGS__;                                                                         \
    } else {                                                                               \
      typedef _u1 G;                                                                       \
      __VA_ARGS__;                                                                         \
    }                                                                                      \
  } while (0)

extern "C" {

int ref_omp_threads() {
#ifdef _USE_OMP_
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// hotstart(U, seed, delta) (gaugeconfig.hh:277-289), then optionally
// random_gauge_trafo(U, trafo_seed) (random_gauge_trafo.hh:10-33) as in
// base_program.hpp:296-314.
void ref_hotstart(int group, int Lx, int Ly, int Lz, int Lt, int nd, int seed, double delta,
                  int trafo_seed, double *out) {
  DISPATCH(group, {
    gaugeconfig<G> U(Lx, Ly, Lz, Lt, nd, 0.);
    hotstart(U, seed, delta);
    if (trafo_seed >= 0) random_gauge_trafo(U, trafo_seed);
    io<G>::get(U, out);
  });
}

void ref_random_gauge_trafo(int group, int Lx, int Ly, int Lz, int Lt, int nd, int seed,
                            double *inout) {
  DISPATCH(group, {
    gaugeconfig<G> U(Lx, Ly, Lz, Lt, nd, 0.);
    io<G>::put(U, inout);
    random_gauge_trafo(U, seed);
    io<G>::get(U, inout);
  });
}

double ref_retr_sum_plaquettes(int group, int Lx, int Ly, int Lz, int Lt, int nd,
                               const double *in, double xi, int aniso, int spatial_only) {
  double r = 0.;
  DISPATCH(group, {
    gaugeconfig<G> U(Lx, Ly, Lz, Lt, nd, 0.);
    io<G>::put(U, in);
    r = flat_spacetime::retr_sum_Wplaquettes(U, xi, bool(aniso), bool(spatial_only));
  });
  return r;
}

double ref_gauge_energy(int group, int Lx, int Ly, int Lz, int Lt, int nd, const double *in,
                        int spatial_only) {
  double r = 0.;
  DISPATCH(group, {
    gaugeconfig<G> U(Lx, Ly, Lz, Lt, nd, 0.);
    io<G>::put(U, in);
    r = flat_spacetime::gauge_energy(U, bool(spatial_only));
  });
  return r;
}

double ref_S_G_hmc(int group, int Lx, int Ly, int Lz, int Lt, int nd, double beta,
                   const double *in, double xi, int aniso) {
  double r = 0.;
  DISPATCH(group, {
    gaugeconfig<G> U(Lx, Ly, Lz, Lt, nd, beta);
    io<G>::put(U, in);
    r = flat_spacetime::get_S_G_hmc<double, G>(U, xi, bool(aniso));
  });
  return r;
}

// gaugemonomial::derivative (flat-gaugemonomial.hh:105-131) into a zeroed field.
void ref_gauge_derivative(int group, int Lx, int Ly, int Lz, int Lt, int nd, double beta,
                          double xi, const double *in, double fac, double *deriv_out) {
  DISPATCH(group, {
    gaugeconfig<G> U(Lx, Ly, Lz, Lt, nd, beta);
    io<G>::put(U, in);
    adjointfield<double, G> deriv(Lx, Ly, Lz, Lt, nd);
    adjointfield<double, G> mom(Lx, Ly, Lz, Lt, nd);
    zeroadjointfield(deriv);
    hamiltonian_field<double, G> h(mom, U);
    flat_spacetime::gaugemonomial<double, G> gm(0, xi);
    gm.derivative(deriv, h, fac);
    io<G>::getP(deriv, deriv_out);
  });
}

// md_update (md_update.hh:18-81) with the momentum draw replaced by injected momenta and
// no accept/reject: heatbath -> integrate -> accept.  U, P updated in place.
// H[0..3] = {kinetic Hold, gauge Hold, kinetic Hnew, gauge Hnew}; returns delta H.
double ref_md_injected_lp(int group, int Lx, int Ly, int Lz, int Lt, int nd, double beta,
                          double xi, int integ, int nsteps, double tau, double *U_io,
                          double *P_io, double *H, int exponent) {
  double dH = 0.;
  DISPATCH(group, {
    gaugeconfig<G> U(Lx, Ly, Lz, Lt, nd, beta);
    io<G>::put(U, U_io);
    adjointfield<double, G> P(Lx, Ly, Lz, Lt, nd);
    io<G>::putP(P, P_io);
    kineticmonomial<double, G> km(0);
    flat_spacetime::gaugemonomial<double, G> gm(0, xi);
    auto ml = gauge_monomials(km, gm);
    hamiltonian_field<double, G> h(P, U);
    for (auto m : ml) m->heatbath(h);
    integrator<double, G> *it = make_integrator<G>(integ, exponent);
    md_params p(nsteps, tau);
    it->integrate(ml, h, p);
    for (auto m : ml) {
      m->accept(h);
      dH += m->getDeltaH();
    }
    H[0] = km.Hold;
    H[1] = gm.Hold;
    H[2] = km.Hnew;
    H[3] = gm.Hnew;
    delete it;
    io<G>::get(U, U_io);
    io<G>::getP(P, P_io);
  });
  return dH;
}
double ref_md_injected(int group, int Lx, int Ly, int Lz, int Lt, int nd, double beta,
                       double xi, int integ, int nsteps, double tau, double *U_io,
                       double *P_io, double *H) {
  return ref_md_injected_lp(group, Lx, Ly, Lz, Lt, nd, beta, xi, integ, nsteps, tau, U_io, P_io,
                            H, 16);
}

// The reference HMC chain: for i in [i0, i0+ntraj): std::mt19937 engine(seed+i);
// md_update(...) (hmc.hpp:86-101), recording accept, delta H and gauge_energy.
void ref_hmc_run(int group, int Lx, int Ly, int Lz, int Lt, int nd, double beta, double xi,
                 int integ, int nsteps, double tau, long seed, int i0, int ntraj,
                 double *U_io, int *acc, double *dH, double *plaq) {
  DISPATCH(group, {
    gaugeconfig<G> U(Lx, Ly, Lz, Lt, nd, beta);
    io<G>::put(U, U_io);
    kineticmonomial<double, G> km(0);
    flat_spacetime::gaugemonomial<double, G> gm(0, xi);
    auto ml = gauge_monomials(km, gm);
    integrator<double, G> *it = make_integrator<G>(integ);
    md_params p(nsteps, tau);
    for (int k = 0; k < ntraj; k++) {
      const size_t i = size_t(i0 + k);
      std::mt19937 engine(seed + i);
      md_update(U, engine, p, ml, *it);
      acc[k] = p.getaccept() ? 1 : 0;
      dH[k] = p.getdeltaH();
      plaq[k] = flat_spacetime::gauge_energy(U);
    }
    delete it;
    io<G>::get(U, U_io);
  });
}

// One Metropolis sweep exactly as metropolis_algo::do_sweep seeds it (metropolis.hpp:96-105).
void ref_sweep(int group, int Lx, int Ly, int Lz, int Lt, int nd, double beta, double xi,
               int aniso, double delta, int N_hit, long seed, long i, double *U_io,
               double *rates) {
  DISPATCH(group, {
    gaugeconfig<G> U(Lx, Ly, Lz, Lt, nd, beta);
    io<G>::put(U, U_io);
    const int threads = ref_omp_threads();
    std::vector<std::mt19937> engines(threads);
    for (int e = 0; e < threads; e++) engines[e].seed(seed + i + e);
    std::vector<double> r =
      flat_spacetime::sweep(U, engines, delta, size_t(N_hit), beta, xi, bool(aniso));
    rates[0] = r[0];
    rates[1] = r[1];
    io<G>::get(U, U_io);
  });
}

void ref_energy_density(int group, int Lx, int Ly, int Lz, int Lt, int nd, const double *in,
                        int cloverdef, int ss, double *E, double *Q) {
  DISPATCH(group, {
    gaugeconfig<G> U(Lx, Ly, Lz, Lt, nd, 0.);
    io<G>::put(U, in);
    double e = 0., q = 0.;
    flat_spacetime::energy_density(U, e, q, bool(cloverdef), bool(ss));
    *E = e;
    *Q = q;
  });
}

// One Wilson-flow RK3 step: runge_kutta (flat-gradient_flow.hh:17-50).
void ref_runge_kutta(int group, int Lx, int Ly, int Lz, int Lt, int nd, double beta,
                     double xi, double eps, double *U_io) {
  DISPATCH(group, {
    gaugeconfig<G> U(Lx, Ly, Lz, Lt, nd, beta);
    io<G>::put(U, U_io);
    adjointfield<double, G> deriv(Lx, Ly, Lz, Lt, nd);
    hamiltonian_field<double, G> h(deriv, U);
    flat_spacetime::gaugemonomial<double, G> SW(0, xi);
    runge_kutta(h, SW, eps);
    io<G>::get(U, U_io);
  });
}

// gradient_flow (flat-gradient_flow.hh:70-197); records go to the text file `path`.
void ref_gradient_flow(int group, int Lx, int Ly, int Lz, int Lt, int nd, double beta,
                       double xi, const double *in, double tmax, double eps, double tstart,
                       const char *path) {
  DISPATCH(group, {
    gaugeconfig<G> U(Lx, Ly, Lz, Lt, nd, beta);
    io<G>::put(U, in);
    flat_spacetime::gradient_flow(U, std::string(path), tmax, eps, xi, tstart, false);
  });
}

// ---- staggered fermions (U(1) only: staggered.hpp:343-350 aborts for SU(2)) ----

// op: 0 = D (staggered.hpp:305-341), 1 = Ddag (:353-389), 2 = D Ddag (:290-302)
void ref_staggered_apply(int Lx, int Ly, int Lz, int Lt, int nd, const double *Uin, double m,
                         int op, const double *psi_in, double *psi_out) {
  gaugeconfig<_u1> U(Lx, Ly, Lz, Lt, nd, 0.);
  io<_u1>::put(U, Uin);
  const spinor psi = make_spinor(U, psi_in);
  spinor out;
  if (op == 0)
    out = staggered::apply_D<double, Complex>(U, m, psi);
  else if (op == 1)
    out = staggered::apply_Ddag<double, Complex>(U, m, psi);
  else {
    const staggered::DDdag_matrix_lat<double, Complex, _u1> M(U, m);
    out = M * psi;
  }
  put_spinor(out, psi_out);
}

// LinearCG::solve (CG.hpp:36-94) on D Ddag from x0, absolute tolerance on |r|.
// Returns the number of stored iterates minus one (= iterations when no restart occurs).
long ref_cg_ddag(int Lx, int Ly, int Lz, int Lt, int nd, const double *Uin, double m,
                 const double *b, const double *x0, double tol, double *x_out) {
  gaugeconfig<_u1> U(Lx, Ly, Lz, Lt, nd, 0.);
  io<_u1>::put(U, Uin);
  typedef staggered::DDdag_matrix_lat<double, Complex, _u1> M_t;
  const M_t M(U, m);
  counted<CG::LinearCG<double, Complex, M_t, spinor>> cg(M, make_spinor(U, b));
  cg.solve(make_spinor(U, x0), tol, 0);
  put_spinor(cg.get_solution(), x_out);
  return long(cg.n_iterates()) - 1;
}

// DDdag_matrix_lat::inv (staggered.hpp:249-276): CG from a sigma=10 real Gaussian start.
void ref_ddag_inv(int Lx, int Ly, int Lz, int Lt, int nd, const double *Uin, double m,
                  const double *psi, double tol, long seed, double *x_out) {
  gaugeconfig<_u1> U(Lx, Ly, Lz, Lt, nd, 0.);
  io<_u1>::put(U, Uin);
  const staggered::DDdag_matrix_lat<double, Complex, _u1> M(U, m);
  put_spinor(M.inv(make_spinor(U, psi), "CG", tol, 0, size_t(seed)), x_out);
}

// LinearBiCGStab::solve (BiCGStab.hpp:36-106) on D alone.
long ref_bicgstab_d(int Lx, int Ly, int Lz, int Lt, int nd, const double *Uin, double m,
                    const double *b, const double *x0, double tol, double *x_out) {
  D_matrix M;
  M.U = gaugeconfig<_u1>(Lx, Ly, Lz, Lt, nd, 0.);
  io<_u1>::put(M.U, Uin);
  M.m = m;
  counted<BiCGStab::LinearBiCGStab<double, Complex, D_matrix, spinor>> s(
    M, make_spinor(M.U, b));
  s.solve(make_spinor(M.U, x0), tol, 0);
  put_spinor(s.get_solution(), x_out);
  return long(s.n_iterates()) - 1;
}

// detDDdag_monomial (detDDdag_monomial.hh:64-167).
// heatbath: phi = D R, R real Gaussian sigma=1/sqrt(2) from seed_pf (+ n_traj = 0).
double ref_fermion_heatbath(int Lx, int Ly, int Lz, int Lt, int nd, const double *Uin,
                            double m, long seed_pf, double *phi_out) {
  gaugeconfig<_u1> U(Lx, Ly, Lz, Lt, nd, 0.);
  io<_u1>::put(U, Uin);
  adjointfield<double, _u1> P(Lx, Ly, Lz, Lt, nd);
  hamiltonian_field<double, _u1> h(P, U);
  staggered::detDDdag_monomial<double, _u1> f(0, m, "CG", 1e-10, size_t(seed_pf), 0);
  f.heatbath(h);
  put_spinor(f.phi, phi_out);
  return f.Hold;
}

double ref_fermion_accept(int Lx, int Ly, int Lz, int Lt, int nd, const double *Uin,
                          double m, const double *phi, double tol, long seed) {
  gaugeconfig<_u1> U(Lx, Ly, Lz, Lt, nd, 0.);
  io<_u1>::put(U, Uin);
  adjointfield<double, _u1> P(Lx, Ly, Lz, Lt, nd);
  hamiltonian_field<double, _u1> h(P, U);
  staggered::detDDdag_monomial<double, _u1> f(0, m, "CG", tol, size_t(seed), 0);
  f.phi = make_spinor(U, phi);
  f.accept(h);
  return f.Hnew;
}

void ref_fermion_derivative(int Lx, int Ly, int Lz, int Lt, int nd, const double *Uin,
                            double m, const double *phi, double tol, long seed,
                            double *deriv_out) {
  gaugeconfig<_u1> U(Lx, Ly, Lz, Lt, nd, 0.);
  io<_u1>::put(U, Uin);
  adjointfield<double, _u1> P(Lx, Ly, Lz, Lt, nd);
  adjointfield<double, _u1> deriv(Lx, Ly, Lz, Lt, nd);
  zeroadjointfield(deriv);
  hamiltonian_field<double, _u1> h(P, U);
  staggered::detDDdag_monomial<double, _u1> f(0, m, "CG", tol, size_t(seed), 0);
  f.phi = make_spinor(U, phi);
  f.derivative(deriv, h, 1.);
  io<_u1>::getP(deriv, deriv_out);
}

// U(1) md_update with gauge + detDDdag monomials, injected momenta and injected R
// (phi = D R, Hold = |R|^2 exactly as heatbath sets them, detDDdag_monomial.hh:64-83).
// exponent: the rounding exponent of the low-precision integrators (ids 1, 3); the
// round_and_update_momenta of those integrators rounds the summed gauge + fermion derivative.
double ref_md_injected_fermion_lp(int Lx, int Ly, int Lz, int Lt, int nd, double beta,
                                  double m, double tol, long seed, int integ, int nsteps,
                                  double tau, double *U_io, double *P_io, const double *R,
                                  double *H, int exponent) {
  gaugeconfig<_u1> U(Lx, Ly, Lz, Lt, nd, beta);
  io<_u1>::put(U, U_io);
  adjointfield<double, _u1> P(Lx, Ly, Lz, Lt, nd);
  io<_u1>::putP(P, P_io);
  kineticmonomial<double, _u1> km(0);
  flat_spacetime::gaugemonomial<double, _u1> gm(0, 1.0);
  staggered::detDDdag_monomial<double, _u1> f(0, m, "CG", tol, size_t(seed), 0);
  std::list<monomial<double, _u1> *> ml = gauge_monomials(km, gm);
  ml.push_back(&f);
  hamiltonian_field<double, _u1> h(P, U);
  km.heatbath(h);
  gm.heatbath(h);
  const spinor Rs = make_spinor(U, R);
  f.phi = staggered::apply_D<double, Complex>(U, m, Rs);
  f.Hold = Rs.norm_squared();
  integrator<double, _u1> *it = make_integrator<_u1>(integ, exponent);
  md_params p(nsteps, tau);
  it->integrate(ml, h, p);
  double dH = 0.;
  for (auto mo : ml) {
    mo->accept(h);
    dH += mo->getDeltaH();
  }
  H[0] = km.Hold;
  H[1] = gm.Hold;
  H[2] = f.Hold;
  H[3] = km.Hnew;
  H[4] = gm.Hnew;
  H[5] = f.Hnew;
  delete it;
  io<_u1>::get(U, U_io);
  io<_u1>::getP(P, P_io);
  return dH;
}

double ref_md_injected_fermion(int Lx, int Ly, int Lz, int Lt, int nd, double beta,
                               double m, double tol, long seed, int integ, int nsteps,
                               double tau, double *U_io, double *P_io, const double *R,
                               double *H) {
  return ref_md_injected_fermion_lp(Lx, Ly, Lz, Lt, nd, beta, m, tol, seed, integ, nsteps, tau,
                                    U_io, P_io, R, H, 16);
}

// staggered::eta (staggered.hpp:41-48)
double ref_eta(int t, int x, int y, int z, int mu) {
  return staggered::eta({t, x, y, z}, size_t(mu));
}

// initnormal (adjointfield.hh:240-258) from std::mt19937(seed), the momentum draw of
// md_update (md_update.hh:24-27); also returns the next uniform(engine) draw.
double ref_initnormal(int group, int Lx, int Ly, int Lz, int Lt, int nd, long seed,
                      double *P_out) {
  double u = 0.;
  DISPATCH(group, {
    adjointfield<double, G> P(Lx, Ly, Lz, Lt, nd);
    std::mt19937 engine(seed);
    initnormal(engine, P);
    std::uniform_real_distribution<double> uniform(0., 1.);
    u = uniform(engine);
    io<G>::getP(P, P_out);
  });
  return u;
}

// gaussian_spinor (staggered.hpp:175-193)
void ref_gaussian_spinor(int Lx, int Ly, int Lz, int Lt, double avr, double sigma, long seed,
                         double *out) {
  const staggered::nd_max_arr<size_t> dims = {size_t(Lt), size_t(Lx), size_t(Ly),
                                              size_t(Lz)};
  put_spinor(staggered::gaussian_spinor<double, Complex>(dims, avr, sigma, size_t(seed)),
             out);
}


// ---- observables between trajectories -------------------------------------------------
// polyakov_loop_spatial_average (polyakov_loop.hh:48-63)
double ref_polyakov_loop(int group, int Lx, int Ly, int Lz, int Lt, int nd, const double *in) {
  double r = 0.;
  DISPATCH(group, {
    gaugeconfig<G> U(Lx, Ly, Lz, Lt, nd, 0.);
    io<G>::put(U, in);
    r = polyakov_loop_spatial_average(U);
  });
  return r;
}

// wilsonloop(U, r, t) (wilsonloop.hh:147-157): planar r x t loops in the (mu, 0) planes
double ref_wilson_loop(int group, int Lx, int Ly, int Lz, int Lt, int nd, const double *in,
                       int r, int t) {
  double w = 0.;
  DISPATCH(group, {
    gaugeconfig<G> U(Lx, Ly, Lz, Lt, nd, 0.);
    io<G>::put(U, in);
    w = wilsonloop(U, (size_t)r, (size_t)t);
  });
  return w;
}

// APEsmearing<double>(U, alpha, spatial) (smearape.hh:97-131), in place
void ref_ape_smear(int group, int Lx, int Ly, int Lz, int Lt, int nd, double alpha, int spatial,
                   double *inout) {
  DISPATCH(group, {
    gaugeconfig<G> U(Lx, Ly, Lz, Lt, nd, 0.);
    io<G>::put(U, inout);
    APEsmearing<double, G>(U, alpha, bool(spatial));
    io<G>::get(U, inout);
  });
}

// gaugeconfig<G>::save / load (gaugeconfig.hh:225-252), the reference's binary format
void ref_save_gauge(int group, int Lx, int Ly, int Lz, int Lt, int nd, const double *in,
                    const char *path) {
  DISPATCH(group, {
    gaugeconfig<G> U(Lx, Ly, Lz, Lt, nd, 0.);
    io<G>::put(U, in);
    U.save(path);
  });
}
int ref_load_gauge(int group, int Lx, int Ly, int Lz, int Lt, int nd, const char *path,
                   double *out) {
  int rc = 1;
  DISPATCH(group, {
    gaugeconfig<G> U(Lx, Ly, Lz, Lt, nd, 0.);
    rc = U.load(path);
    io<G>::get(U, out);
  });
  return rc;
}

// staggered::C_pion<_u1>(U, m, "CG", tol, 0, seed) (propagator.hpp:25-65)
void ref_pion_correlator(int Lx, int Ly, int Lz, int Lt, int nd, const double *Uin, double m,
                         double tol, long seed, double *C) {
  gaugeconfig<_u1> U(Lx, Ly, Lz, Lt, nd, 0.);
  io<_u1>::put(U, Uin);
  const std::vector<double> c = staggered::C_pion<_u1>(U, m, "CG", tol, 0, (size_t)seed);
  for (int t = 0; t < Lt; t++) C[t] = c[t];
}
} // extern "C"
