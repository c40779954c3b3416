// su2b_internal.h -- host-side launchers of the libsu2b kernels (not part of the C ABI).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "su2b_common.cuh"

namespace su2b {

// ---- layout conversion (reference host AoS <-> even/odd SoA) ----
template <class T>
cudaError_t links_from_host(const Geom &g, const double *aos, void *U, int group,
                            cudaStream_t s);
template <class T>
cudaError_t links_to_host(const Geom &g, const void *U, double *aos, int group, cudaStream_t s);
template <class T>
cudaError_t adj_from_host(const Geom &g, const double *aos, T *P, int group, cudaStream_t s);
template <class T>
cudaError_t adj_to_host(const Geom &g, const T *P, double *aos, int group, cudaStream_t s);
cudaError_t spinor_from_host(const Geom &g, const double *aos, double2 *psi, cudaStream_t s);
cudaError_t spinor_to_host(const Geom &g, const double2 *psi, double *aos, cudaStream_t s);

// ---- reductions ----
// plaquette partial sums, 3 per block {full, spatial-only, xi-weighted}; returns #blocks
template <class T>
cudaError_t plaq_partials(const Geom &g, const void *U, int group, double xi, double *part,
                          int *nblocks, cudaStream_t s);
// out[k] = sum_b part[b*ncomp + k] in a fixed order, k < ncomp
cudaError_t reduce_final(const double *part, int nblocks, int ncomp, double *out,
                         cudaStream_t s);

// ---- gauge force / momenta ----
enum ForceMode : int {
  FM_HAS_IN = 1,     // P_out = P_in + scale*(f*g) (else P_out = scale*(f*g))
  FM_KINETIC = 2,    // also write per-block partials of sum P_out^2
  FM_EXTRA = 4,      // add extra[] (another monomial's derivative) to f*g before scaling
  FM_UPDATE = 8,     // SU(2): also write Uout = exp(dt_upd * P_out) U (the next gauge step)
  FM_RESTORE = 16    // SU(2): also write Uout = restoreSU(U) (the end of the trajectory)
};
// launch shapes of the SU(2) force kernel (threads per block, minimum resident blocks per
// SM, which caps registers): one thread per site 0 (256,4) 1 (128,8) 2 (128,4) 3 (128,6)
// 4 (256,2) 5 (256,3) 7 (64,16); two threads per site 6 split, 8 xsplit, both (128,8), and
// 10 split (128,5) (96 registers: FP64 links); 9 one thread per link; 11 site pairs in packed
// FP32 (FP32 links, d = 4, T a multiple of 4: the fused trajectory runs force_pair on a paired
// copy of the field; every other caller, and FP64 links, run the one-thread-per-link kernel,
// whose arithmetic force_pair reproduces lane for lane)
constexpr int FORCE_VARIANTS = 12;
constexpr int FORCE_PAIR = 11;
constexpr int PAIR_MINB = 8;  // resident blocks of 128 threads per SM of force_pair
// site pairs (pairs.cu): whether a geometry takes them (d = 4, T % 4 == 0, the whole
// lattice); the standard layout of U copied into the paired layout Upl; the fused force step
// of FP32 links on paired buffers (Uout paired for FM_UPDATE, standard for FM_RESTORE)
bool pairs_apply(const Geom &g);
cudaError_t to_pairs(const Geom &g, const void *U, void *Upl, cudaStream_t s);
cudaError_t force_pair(const Geom &g, const void *Upl, float *P, double f, double scale, int mode,
                       double *kin_part, int *nblocks, void *Uout, double dt_upd, cudaStream_t s,
                       bool pdl);
template <class T>
cudaError_t force_update(const Geom &g, const void *U, int group, T *P, const T *extra, double f,
                         double scale, double xi, int mode, double *kin_part, int *nblocks,
                         void *Uout, double dt_upd, cudaStream_t s, int variant = 1,
                         bool pdl = false);

// U = exp(dt P) U (update_gauge.hh:8-16); with round_dn > 0 the links are rounded first,
// U = exp(dt P) round(U) (round_and_update_gauge, update_gauge.hh:20-26)
template <class T>
cudaError_t link_update(const Geom &g, void *U, int group, const T *P, double dt,
                        cudaStream_t s, double round_dn = 0.0);
// P -= dt * round(D) componentwise, round(x) = round(x dn) / dn in FP64
// (round_and_update_momenta, update_momenta.hh:36-58); D, P of na components per link
template <class T>
cudaError_t adj_round_axpy(const Geom &g, T *P, const T *D, int group, double dt, double dn,
                           cudaStream_t s);
template <class T> cudaError_t restore_links(const Geom &g, void *U, int group, cudaStream_t s);
// per-trajectory parameters read by the kernels from device memory, so that a captured
// trajectory graph can be replayed with a new seed and trajectory index
struct TrajParams {
  double beta, Nc;
  double u_host;  // < 0: Philox uniform
  uint64_t seed;
  uint32_t traj;
  int accept_reject;
};
template <class T>
cudaError_t momenta_philox(const Geom &g, T *P, int group, const TrajParams *tp,
                           double *kin_part, int *nblocks, cudaStream_t s);
// SU(2): the Philox momenta of every link and the plaquette sums of the field in one pass;
// partials {|P|^2, plaquettes, spatial, weighted} per block (4 per block); with plaq false the
// plaquette components are zero (the start plaquettes are carried over from the previous
// trajectory)
template <class T>
cudaError_t momenta_plaq(const Geom &g, const void *U, T *P, const TrajParams *tp, double xi,
                         double *part, int *nblocks, cudaStream_t s, bool plaq = true);
template <class T>
cudaError_t kinetic_partials(const Geom &g, const T *P, int group, double *part, int *nblocks,
                             cudaStream_t s);
template <class T>
cudaError_t negate_adj(const Geom &g, T *P, int group, cudaStream_t s);

// ---- accept / reject ----
// reduced values read by the accept step:
//   red[0] sum P^2 before, red[1..3] plaquette sums before {full, spatial, xi-weighted},
//   red[4] sum P^2 after,  red[5..7] plaquette sums after, red[8] / red[9] fermion action
//   before / after.
struct TrajDev {
  double H_old[3], H_new[3];
  double dH, u;
  int accepted;
  int pad;
};
cudaError_t accept_step(const double *red, const TrajParams *tp, TrajDev *out, cudaStream_t s);
cudaError_t reduce_accept(const double *ps, int ns, const double *pk, int nk, const double *pp,
                          int np, double *red, const TrajParams *tp, TrajDev *out,
                          bool cached_start, cudaStream_t s);
template <class T>
cudaError_t cond_restore(const Geom &g, void *U, const void *U_old, int group,
                         const TrajDev *flag, cudaStream_t s);

// ---- Metropolis ----
template <class T>
cudaError_t metropolis_pass(const Geom &g, void *U, int group, int mu, int parity, double beta,
                            double xi, double delta, int N_hit, uint64_t seed, uint32_t sweep,
                            unsigned long long *counts, cudaStream_t s);

// ---- clover energy density / charge ----
// per-block partials {E, E_ss, Q, Q_ss}
template <class T>
cudaError_t clover_partials(const Geom &g, const void *U, int group, int cloverdef,
                            double *part, int *nblocks, cudaStream_t s);

// ---- staggered fermions ----
cudaError_t u1_phases(const Geom &g, const double *theta, double2 *ph, cudaStream_t s);
cudaError_t u1_phases_f32(const Geom &g, const double *theta, float2 *ph, cudaStream_t s);
// out = D psi (dag=0) or Ddag psi (dag=1), staggered.hpp:305-389
cudaError_t staggered_D(const Geom &g, const double2 *ph, double m, int dag, const double2 *in,
                        double2 *out, cudaStream_t s);
cudaError_t staggered_D(const Geom &g, const float2 *ph, float m, int dag, const float2 *in,
                        float2 *out, cudaStream_t s);
cudaError_t fermion_force(const Geom &g, const double2 *ph, const double2 *chi,
                          const double2 *chi1, double *deriv, cudaStream_t s);
cudaError_t pf_source(const Geom &g, uint64_t seed, uint32_t traj, int complex_source,
                      double2 *R, cudaStream_t s);

}  // namespace su2b
