/* su2b_device.hpp -- the su2 driver's side of the boundary: a C++ shim over su2b.h.
 *
 * The su2 code has no FFI; its drivers call template functions on gaugeconfig<G> directly.
 * This header is what those drivers include to route the hot-path calls to libsu2b.  It
 * needs the su2 headers on the include path (gaugeconfig.hh, adjointfield.hh, md_params.hh,
 * geometry.hh) and links against su2_b200/libsu2b.so.
 *
 *   su2b_device::pack / unpack          gaugeconfig<G> / adjointfield<double, G> <-> the flat
 *                                       host layout of su2b.h (gaugeconfig.hh:211-222 order)
 *   su2b_device::device_lattice<G>      a device-resident copy of one gaugeconfig, with the
 *                                       calls that replace
 *     md_update(...)                      md_update (md_update.hh:18-81) as hmc.hpp:86-101
 *                                         calls it: device Philox streams keyed by (seed, i),
 *                                         or the driver's own std::mt19937 replayed
 *     gauge_energy / energy_density       flat-gauge_energy.hpp:109-137,
 *                                         flat-energy_density.hh:57-164
 *     sweep                               flat_spacetime::sweep (flat-sweep.hh:64-164)
 *     derivative                          gaugemonomial::derivative (flat-gaugemonomial.hh:
 *                                         105-131)
 *     gradient_flow                       flat_spacetime::gradient_flow's records
 *                                         (flat-gradient_flow.hh:70-197)
 *
 * A non-zero status of libsu2b ends in the reference's own error path,
 * spacetime_lattice::fatal_error (geometry.hh:43-48), as a failure inside the reference's
 * loops would.  One host thread per device_lattice.
 */
#pragma once

#include <cmath>
#include <random>
#include <string>
#include <type_traits>
#include <vector>

#include "adjointfield.hh"
#include "gaugeconfig.hh"
#include "geometry.hh"
#include "md_params.hh"
#include "su2b.h"

namespace su2b_device {

inline void check(int rc, const su2b_ctx *c, const char *where) {
  if (rc != SU2B_OK)
    spacetime_lattice::fatal_error(std::string("libsu2b: ") + su2b_last_error(c), where);
}

template <class G> constexpr bool is_u1() { return std::is_same<G, _u1>::value; }
/* reals per link in the host layout: SU(2) {Re a, Im a, Re b, Im b}, U(1) the angle */
template <class G> constexpr size_t link_reals() { return is_u1<G>() ? 1 : 4; }
/* reals per adjoint element: SU(2) {a, b, c} (adjointfield.hh:12-51), U(1) one */
template <class G> constexpr size_t adj_reals() { return is_u1<G>() ? 1 : 3; }

/* gaugeconfig<G> -> flat host buffer in the link order of gaugeconfig.hh:211-222 (the N_c
 * member of each link object is not part of the buffer) */
inline void pack_link(const _su2 &u, double *d) {
  d[0] = u.geta().real();
  d[1] = u.geta().imag();
  d[2] = u.getb().real();
  d[3] = u.getb().imag();
}
inline void pack_link(const _u1 &u, double *d) { d[0] = u.geta(); }
inline _su2 unpack_link(const double *d, const _su2 *) {
  return _su2(Complex(d[0], d[1]), Complex(d[2], d[3]));
}
inline _u1 unpack_link(const double *d, const _u1 *) { return _u1(d[0]); }

template <class G> std::vector<double> pack(const gaugeconfig<G> &U) {
  std::vector<double> h(U.getSize() * link_reals<G>());
  for (size_t i = 0; i < U.getSize(); i++) pack_link(U[i], h.data() + link_reals<G>() * i);
  return h;
}
template <class G> void unpack(const std::vector<double> &h, gaugeconfig<G> &U) {
  if (h.size() != U.getSize() * link_reals<G>())
    spacetime_lattice::fatal_error("host buffer does not match the lattice", __func__);
  for (size_t i = 0; i < U.getSize(); i++)
    U[i] = unpack_link(h.data() + link_reals<G>() * i, static_cast<const G *>(nullptr));
}

/* adjointfield<double, G> <-> flat host buffer, same link order */
inline void pack_adj(const adjointsu2<double> &a, double *d) {
  d[0] = a.geta();
  d[1] = a.getb();
  d[2] = a.getc();
}
inline void pack_adj(const adjointu1<double> &a, double *d) { d[0] = a.geta(); }
inline void unpack_adj(const double *d, adjointsu2<double> &a) {
  a.seta(d[0]);
  a.setb(d[1]);
  a.setc(d[2]);
}
inline void unpack_adj(const double *d, adjointu1<double> &a) { a.seta(d[0]); }

template <class G> std::vector<double> pack(const adjointfield<double, G> &P) {
  std::vector<double> h(P.getSize() * adj_reals<G>());
  for (size_t i = 0; i < P.getSize(); i++) pack_adj(P[i], h.data() + adj_reals<G>() * i);
  return h;
}
template <class G> void unpack(const std::vector<double> &h, adjointfield<double, G> &P) {
  if (h.size() != P.getSize() * adj_reals<G>())
    spacetime_lattice::fatal_error("host buffer does not match the field", __func__);
  for (size_t i = 0; i < P.getSize(); i++) unpack_adj(h.data() + adj_reals<G>() * i, P[i]);
}

/* One gaugeconfig held on the device.  The host copy is refreshed only where the driver
 * needs host links (save points, host-side observables) with download(). */
template <class G> class device_lattice {
public:
  device_lattice(const gaugeconfig<G> &U, double xi = 1.0, bool mixed = false,
                 int device = 0)
    : Lx(U.getLx()), Ly(U.getLy()), Lz(U.getLz()), Lt(U.getLt()), nd(U.getndims()) {
    check(su2b_ctx_create(is_u1<G>() ? SU2B_GROUP_U1 : SU2B_GROUP_SU2, (int)Lx, (int)Ly,
                          (int)Lz, (int)Lt, (int)nd, U.getBeta(), xi,
                          mixed ? SU2B_PREC_MIXED : SU2B_PREC_FP64, device, &ctx),
          ctx, __func__);
  }
  ~device_lattice() { su2b_ctx_destroy(ctx); }
  device_lattice(const device_lattice &) = delete;
  device_lattice &operator=(const device_lattice &) = delete;

  su2b_ctx *handle() { return ctx; }

  void upload(const gaugeconfig<G> &U) {
    const std::vector<double> h = pack(U);
    check(su2b_upload_gauge(ctx, h.data()), ctx, __func__);
  }
  void download(gaugeconfig<G> &U) {
    std::vector<double> h(U.getSize() * link_reals<G>());
    check(su2b_download_gauge(ctx, h.data()), ctx, __func__);
    unpack(h, U);
  }
  /* times the force kernel's launch shapes on this field once and keeps the fastest;
   * cache_path (may be empty) remembers the choice per GPU model, precision and lattice */
  void autotune(const std::string &cache_path = "") {
    check(su2b_autotune(ctx, cache_path.empty() ? nullptr : cache_path.c_str(), 0, nullptr),
          ctx, __func__);
  }

  /* md_update as hmc.hpp:94-97 calls it for trajectory i, with the gauge monomial (and the
   * kinetic one): momenta and accept uniform from the device's Philox streams keyed by
   * (seed, i).  Sets accept, deltaH and (revtest) deltadeltaH in params like md_update;
   * returns the plaquette sum of the resulting field. */
  double md_update(md_params &params, int integrator, uint64_t seed, uint32_t i) {
    su2b_hmc_params p = base_params(params, integrator);
    p.seed = seed;
    p.traj = i;
    return run(params, p);
  }
  /* The same trajectory driven by the driver's own engine (std::mt19937(seed + i) in
   * hmc.hpp:94): the momenta are drawn on the host by the reference's initnormal
   * (adjointfield.hh:240-258) and the accept uniform by the draw md_update makes after them
   * (md_update.hh:29,55-59), so the device takes the reference's accept decisions. */
  template <class URNG>
  double md_update(md_params &params, int integrator, URNG &engine) {
    adjointfield<double, G> momenta(Lx, Ly, Lz, Lt, nd);
    initnormal(engine, momenta);
    std::uniform_real_distribution<double> uniform(0., 1.);
    const double u = uniform(engine);
    const std::vector<double> P = pack(momenta);
    su2b_hmc_params p = base_params(params, integrator);
    p.momenta_host = P.data();
    p.uniform_host = u;
    return run(params, p);
  }

  /* flat_spacetime::gauge_energy(U, spatial_only) */
  double gauge_energy(bool spatial_only = false) {
    double e = 0.;
    check(su2b_gauge_energy(ctx, spatial_only ? 1 : 0, &e), ctx, __func__);
    return e;
  }
  /* flat_spacetime::energy_density(U, E, Q, cloverdef, ss) */
  void energy_density(double &E, double &Q, bool cloverdef = true, bool ss = false) {
    check(su2b_energy_density(ctx, cloverdef ? 1 : 0, ss ? 1 : 0, &E, &Q), ctx, __func__);
  }
  /* flat_spacetime::sweep with the device's checkerboard order and Philox streams keyed by
   * (seed, i); returns the overall acceptance rate, rates[1] the temporal one */
  double sweep(double delta, size_t N_hit, uint64_t seed, uint32_t i, double *rates = nullptr) {
    double r[2] = {0., 0.};
    check(su2b_metropolis_sweep(ctx, delta, (int)N_hit, seed, i, r), ctx, __func__);
    if (rates) {
      rates[0] = r[0];
      rates[1] = r[1];
    }
    return r[0];
  }
  /* gaugemonomial::derivative(deriv, h, fac) into deriv (overwritten) */
  void derivative(adjointfield<double, G> &deriv, double fac = 1.0) {
    std::vector<double> h(deriv.getSize() * adj_reals<G>());
    check(su2b_gauge_force(ctx, fac, h.data()), ctx, __func__);
    unpack(h, deriv);
  }
  /* gradient_flow's records {t, xi_R, P, P_ss, Ep, Ep_ss, Ec, Ec_ss, Q} on a copy of the
   * device links, one row per record */
  std::vector<std::vector<double>> gradient_flow(double tmax, double eps, double tstart = 0.) {
    const int max_rows = (int)std::ceil((tmax - tstart) / eps) + 4;
    std::vector<double> flat(9 * (size_t)max_rows);
    int n = 0;
    check(su2b_gradient_flow(ctx, tmax, eps, tstart, flat.data(), max_rows, &n), ctx,
          __func__);
    std::vector<std::vector<double>> rows((size_t)n);
    for (int k = 0; k < n; k++) rows[k].assign(flat.begin() + 9 * k, flat.begin() + 9 * k + 9);
    return rows;
  }

private:
  su2b_ctx *ctx = nullptr;
  size_t Lx, Ly, Lz, Lt, nd;

  static su2b_hmc_params base_params(const md_params &params, int integrator) {
    su2b_hmc_params p{};
    p.integrator = integrator;
    p.n_steps = (int)params.getnsteps();
    p.tau = params.gettau();
    p.revtest = params.getrevtest() ? 1 : 0;
    p.accept_reject = 1;
    p.momenta_host = nullptr;
    p.uniform_host = -1.0;
    p.fermion_mass = 0.0;
    p.pf_source_host = nullptr;
    p.cg_start = SU2B_CG_START_REFERENCE;
    p.round_exponent = (int)params.getexponent();
    return p;
  }
  double run(md_params &params, const su2b_hmc_params &p) {
    su2b_traj_result r{};
    check(su2b_hmc_trajectory(ctx, &p, &r), ctx, __func__);
    params.setdeltaH(r.dH);
    params.setaccept(r.accepted != 0);
    if (p.revtest) params.setdeltadeltaH(r.ddH);
    return r.plaquette;
  }
};

}  // namespace su2b_device
