// shim_check.cc -- the su2 driver's hot path run twice in one program: once through the
// UNMODIFIED su2 headers, once through include/su2b_device.hpp and libsu2b.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles it against the reference's headers
// where they lie in the reference checkout, together with the shim header, and links
// su2_b200/libsu2b.so; the binary lands in oracle/_ref/.  tests/test_gpu_shim.py runs it on a
// GPU and reads the one JSON line it prints.
//
// What it re-enacts, per group (SU(2) d=4 8^4 beta 2.3; U(1) d=2 16x16 beta 4.0):
//   base_program.hpp:276-317   hotstart(U, seed, true) and random_gauge_trafo(U, 654321)
//   hmc.hpp:58-84              monomials: kinetic (md-passive) and the flat gauge monomial
//   hmc.hpp:86-101             per trajectory i: std::mt19937 engine(seed + i),
//                              md_update(U, engine, mdparams, monomials, omf2), then
//                              gauge_energy(U) and energy_density(U, E, Q)
// The device side drives the same trajectories through device_lattice::md_update with the
// driver's engine, so both take the same momenta and accept uniforms.  Compared: the accept
// decisions, Delta H, the plaquette and clover energies after each trajectory, the final
// links, the gauge derivative (flat-gaugemonomial.hh:105-131) and one Philox trajectory
// through the device streams.
#include <cmath>
#include <cstdio>
#include <list>
#include <random>

#include "flat-energy_density.hh"
#include "flat-gauge_energy.hpp"
#include "flat-gaugemonomial.hh"
#include "integrator.hh"
#include "md_update.hh"
#include "monomial.hh"
#include "random_gauge_trafo.hh"
#include "su2b_device.hpp"

namespace {

struct result {
  int accept_mismatch = 0;
  double dH_err = 0., plaq_err = 0., E_err = 0., U_err = 0., deriv_err = 0., ddH = 0.;
  double dH_first = 0.;
  int ntraj = 0, accepted = 0;
  bool philox_ok = false;
};

template <class G>
result run(size_t L0, size_t L1, size_t L2, size_t L3, size_t nd, double beta, int ntraj) {
  result out;
  const int seed = 13526463;
  gaugeconfig<G> U(L0, L1, L2, L3, nd, beta);
  hotstart(U, seed, true);
  random_gauge_trafo(U, 654321);

  kineticmonomial<double, G> km(0);
  km.setmdpassive();
  flat_spacetime::gaugemonomial<double, G> gm(0, 1.0);
  std::list<monomial<double, G> *> ml = {&km, &gm};
  integrator<double, G> *integ = set_integrator<double, G>(SU2B_OMF2, 16);

  su2b_device::device_lattice<G> dev(U);
  dev.upload(U);
  gaugeconfig<G> Uref(U);
  for (int i = 0; i < ntraj; i++) {
    md_params p_ref(10, 1.0), p_dev(10, 1.0);
    std::mt19937 e_ref(seed + i), e_dev(seed + i);
    md_update(Uref, e_ref, p_ref, ml, *integ);
    dev.md_update(p_dev, SU2B_OMF2, e_dev);
    out.accept_mismatch += p_ref.getaccept() != p_dev.getaccept();
    out.accepted += p_ref.getaccept();
    if (i == 0) out.dH_first = p_ref.getdeltaH();
    out.dH_err = std::fmax(out.dH_err, std::fabs(p_ref.getdeltaH() - p_dev.getdeltaH()));
    const double e_r = flat_spacetime::gauge_energy(Uref);
    const double e_d = dev.gauge_energy();
    out.plaq_err = std::fmax(out.plaq_err, std::fabs(e_r - e_d) / std::fabs(e_r));
    double E_r = 0., Q_r = 0., E_d = 0., Q_d = 0.;
    flat_spacetime::energy_density(Uref, E_r, Q_r);
    dev.energy_density(E_d, Q_d);
    out.E_err = std::fmax(out.E_err, std::fabs(E_r - E_d) / std::fabs(E_r));
  }
  out.ntraj = ntraj;
  gaugeconfig<G> Udev(U);
  dev.download(Udev);
  const std::vector<double> a = su2b_device::pack(Uref), b = su2b_device::pack(Udev);
  for (size_t k = 0; k < a.size(); k++) out.U_err = std::fmax(out.U_err, std::fabs(a[k] - b[k]));

  // gaugemonomial::derivative on the final field, through the shim and the reference
  adjointfield<double, G> d_ref(L0, L1, L2, L3, nd), d_dev(L0, L1, L2, L3, nd);
  zeroadjointfield(d_ref);
  hamiltonian_field<double, G> h(d_ref, Uref);
  gm.derivative(d_ref, h, 1.0);
  dev.derivative(d_dev, 1.0);
  const std::vector<double> fa = su2b_device::pack(d_ref), fb = su2b_device::pack(d_dev);
  double num = 0., den = 0.;
  for (size_t k = 0; k < fa.size(); k++) {
    num += (fa[k] - fb[k]) * (fa[k] - fb[k]);
    den += fa[k] * fa[k];
  }
  out.deriv_err = std::sqrt(num / den);

  // the device's own streams, keyed by (seed, i), with the reversibility test of
  // md_update.hh:62-74
  md_params p(10, 1.0);
  p.enablerevtest();
  dev.md_update(p, SU2B_OMF2, (uint64_t)seed, (uint32_t)ntraj);
  out.ddH = p.getdeltadeltaH();
  out.philox_ok = std::isfinite(p.getdeltaH()) && std::fabs(out.ddH) < 1e-8;
  delete integ;
  return out;
}

void print(const char *name, const result &r, bool last) {
  std::printf("\"%s\": {\"ntraj\": %d, \"accepted\": %d, \"accept_mismatch\": %d, "
              "\"dH_first\": %.10g, \"dH_err\": %.3e, \"plaq_rel_err\": %.3e, "
              "\"E_rel_err\": %.3e, \"U_max_err\": %.3e, \"deriv_rel_err\": %.3e, "
              "\"philox_ddH\": %.3e, \"philox_ok\": %s}%s",
              name, r.ntraj, r.accepted, r.accept_mismatch, r.dH_first, r.dH_err, r.plaq_err,
              r.E_err, r.U_err, r.deriv_err, r.ddH, r.philox_ok ? "true" : "false",
              last ? "" : ", ");
}

}  // namespace

int main() {
  const result s = run<_su2>(8, 8, 8, 8, 4, 2.3, 6);
  const result u = run<_u1>(16, 1, 1, 16, 2, 4.0, 6);
  std::printf("{");
  print("su2", s, false);
  print("u1", u, true);
  std::printf("}\n");
  return 0;
}
