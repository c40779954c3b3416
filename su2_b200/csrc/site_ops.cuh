// site_ops.cuh -- per-site bodies of the gauge kernels, shared by the single-lattice
// kernels (gauge.cu) and the batched multi-chain kernels (batch.cu), so both paths perform
// identical arithmetic.
#pragma once
#include "su2b_internal.h"

namespace su2b {

template <class T> using LinkT = typename LinkOf<T>::type;

// Prefetch into L1 of the momentum components of link l (SoA, NL apart): the force step
// reads them only at its end, where every thread then waits on them; requested at the start
// the lines arrive while the staples are summed (about 4 % of the launch at 32^4)
template <class T>
__device__ __forceinline__ void prefetch_momenta(const T *P, size_t l, size_t NL) {
#pragma unroll
  for (int k = 0; k < 3; k++) asm volatile("prefetch.global.L1 [%0];" ::"l"(P + k * NL + l));
}

// Fused gauge force + momentum update for all ND links of a site
// (flat-gaugemonomial.hh:105-131 + update_momenta.hh:10-33):
//   K_mu = sum_{nu != mu} U_nu(x+mu) U_mu(x+nu)^+ U_nu(x)^+ + U_nu(x+mu-nu)^+ U_mu(x-nu)^+ U_nu(x-nu)
//   d_mu = f * get_deriv(U_mu(x) K_mu) (+ extra),  P_mu = P_mu + scale * d_mu  (scale = -dtau)
// One thread per site.  The two forward staples of a plane share the product
// A = U_nu(x+mu) U_mu(x+nu)^+:  forward(mu; nu) = A U_nu(x)^+,  forward(nu; mu) = A^+ U_mu(x)^+.
// Per site 4 + ND(ND-1) + ND^2 + ND(ND-1) = 44 (d = 4) distinct link loads.  The kernels
// that call this give each block one band of sites of both parities (warps alternate), so
// the blocks resident at any time cover one narrow band of the lattice and the links stream
// from HBM about once per launch.  Returns the sum of the updated P^2 of the site.
// The per-link tail of the fused force step for link l with staple sum k:
//   d = f get_deriv(U K) (+ extra),  P = P + scale d,  then (FM_UPDATE) the following gauge
//   step U' = exp(dt P) U (update_gauge.hh:8-16) or (FM_RESTORE) U' = restoreSU(U) into Uout.
// Returns the link's |P|^2 in FP64.
template <class T>
__device__ __forceinline__ double finish_link(const Su2<T> &u, const Su2<T> &k, size_t l,
                                              size_t NL, T *__restrict__ P,
                                              const T *__restrict__ extra, T f, T scale_,
                                              int mode, LinkT<T> *__restrict__ Uout, T dt_upd) {
  // get_deriv(U K) = (2 Im b, 2 Re b, 2 Im a) (adjointfield.hh:53-56)
  const T sbi = fm(u.ar, k.bi, fm(u.ai, k.br, fm(u.bi, k.ar, -u.br * k.ai)));
  const T sbr = fm(u.ar, k.br, fm(-u.ai, k.bi, fm(u.br, k.ar, u.bi * k.ai)));
  const T sai = fm(u.ar, k.ai, fm(u.ai, k.ar, fm(-u.bi, k.br, u.br * k.bi)));
  const T f2 = T(2) * f;
  T d0 = f2 * sbi, d1 = f2 * sbr, d2 = f2 * sai;
  if (mode & FM_EXTRA) {
    d0 += extra[l];
    d1 += extra[NL + l];
    d2 += extra[2 * NL + l];
  }
  T p0 = 0, p1 = 0, p2 = 0;
  if (mode & FM_HAS_IN) {
    p0 = P[l];
    p1 = P[NL + l];
    p2 = P[2 * NL + l];
  }
  p0 = fm(scale_, d0, p0);
  p1 = fm(scale_, d1, p1);
  p2 = fm(scale_, d2, p2);
  P[l] = p0;
  P[NL + l] = p1;
  P[2 * NL + l] = p2;
  if (mode & FM_UPDATE)
    st_link(Uout + l, mul(exp_alg(dt_upd * p0, dt_upd * p1, dt_upd * p2), u));
  else if (mode & FM_RESTORE)
    st_link(Uout + l, from64<T>(restore_su(to64(u))));
  // |P|^2 in FP64 only where the launch sums it (a uniform branch)
  if (!(mode & FM_KINETIC)) return 0.;
  return (double)p0 * p0 + (double)p1 * p1 + (double)p2 * p2;
}

template <class T, int ND, bool ANISO>
__device__ __forceinline__ double force_site_impl(const Geom &g, const LinkT<T> *__restrict__ U,
                                                  T *__restrict__ P,
                                                  const T *__restrict__ extra, T f, T scale_,
                                                  int mode, T wt, T ws,
                                                  LinkT<T> *__restrict__ Uout, T dt_upd, int p,
                                                  int cb) {
  const int q = 1 - p;
  double k2 = 0.;
  const Site s = site_from_eo(g, p, cb);
  const size_t V = (size_t)g.V, NL = V * ND;
  const size_t self = (size_t)p * g.Vh + cb;
  int lf[ND], lb[ND];
#pragma unroll
  for (int mu = 0; mu < ND; mu++) {
    lf[mu] = s.lex + fwd(g, s, mu);
    lb[mu] = bwd(g, s, mu);
  }
  Su2<T> ux[ND], K[ND];
  if (mode & FM_HAS_IN) {
#pragma unroll
    for (int mu = 0; mu < ND; mu++) prefetch_momenta(P, mu * V + self, NL);
  }
#pragma unroll
  for (int mu = 0; mu < ND; mu++) {
    ux[mu] = ld_link(U + mu * V + self);
    K[mu] = zero_su2<T>();
  }
  // backward staples U_nu(x+mu-nu)^+ U_mu(x-nu)^+ U_nu(x-nu), before the forward ones and
  // each with its diagonal link loaded first: the loads that wait longest (the diagonal
  // neighbours are the least often in L1) are issued earliest.  At 32^4 this order runs the
  // launch about 10 % faster than the forward staples first (FP32 76 -> 68 us per launch,
  // FP64 134 -> 119 us)
#pragma unroll
  for (int nu = 0; nu < ND; nu++) {
    const int lmn = s.lex + lb[nu];
    const Su2<T> c = ld_link(U + nu * V + eo_of(g, lmn, q));  // U_nu(x-nu)
#pragma unroll
    for (int mu = 0; mu < ND; mu++) {
      if (mu == nu) continue;
      const Su2<T> e = ld_link(U + nu * V + eo_of(g, lf[mu] + lb[nu], p));  // U_nu(x+mu-nu)
      const Su2<T> h = ld_link(U + mu * V + eo_of(g, lmn, q));          // U_mu(x-nu)
      Su2<T> eh = mul(dag(e), dag(h));
      if (ANISO) eh = scale((nu == 0 || mu == 0) ? wt : ws, eh);
      K[mu] = mul_acc(K[mu], eh, c);
    }
  }
  // forward staples, one plane (mu < nu) at a time; the plane weight of the anisotropic
  // action multiplies the shared product A
#pragma unroll
  for (int mu = 0; mu < ND - 1; mu++)
#pragma unroll
    for (int nu = mu + 1; nu < ND; nu++) {
      const Su2<T> a = ld_link(U + nu * V + eo_of(g, lf[mu], q));  // U_nu(x+mu)
      const Su2<T> b = ld_link(U + mu * V + eo_of(g, lf[nu], q));  // U_mu(x+nu)
      Su2<T> A = mul(a, dag(b));
      if (ANISO) A = scale(mu == 0 ? wt : ws, A);
      K[mu] = mul_acc(K[mu], A, dag(ux[nu]));
      K[nu] = mul_acc(K[nu], dag(A), dag(ux[mu]));
    }
#pragma unroll
  for (int mu = 0; mu < ND; mu++)
    k2 += finish_link<T>(ux[mu], K[mu], mu * V + self, NL, P, extra, f, scale_, mode, Uout,
                         dt_upd);
  return k2;
}

// The same fused force step for half of a d = 4 site: links mu = 2 HALF and 2 HALF + 1.  Two
// threads share a site, so each holds two staple sums instead of four and needs about half
// the registers; the forward product A of the plane inside the half serves both of its links,
// the four planes that cross the halves compute A in both threads (64 FMAs more per site).
// The backward staples come first, and both loops run over the direction nu outside the two
// links, so U_nu(x-nu) and U_nu(x) are each loaded once for both: in FP32 this order runs
// about 3 % faster than the links outside with the forward staples first (the loads the
// diagonal backward staples wait on longest are issued earliest).
template <class T, int HALF, bool ANISO>
__device__ __forceinline__ double force_half_impl(const Geom &g, const LinkT<T> *__restrict__ U,
                                                  T *__restrict__ P,
                                                  const T *__restrict__ extra, T f, T scale_,
                                                  int mode, T wt, T ws,
                                                  LinkT<T> *__restrict__ Uout, T dt_upd, int p,
                                                  int cb) {
  const Site s = site_from_eo(g, p, cb);
  const size_t V = (size_t)g.V, NL = 4 * V;
  int fo[4], bo[4];
#pragma unroll
  for (int d = 0; d < 4; d++) {
    fo[d] = fwd(g, s, d);
    bo[d] = bwd(g, s, d);
  }
  // link U_mu at the site displaced by o (components in {-1, 0, 1}, at most two nonzero)
  auto L = [&](int mu, int o0, int o1, int o2, int o3) -> Su2<T> {
    const int o[4] = {o0, o1, o2, o3};
    int lex = s.lex, odd = 0;
#pragma unroll
    for (int d = 0; d < 4; d++) {
      if (o[d] > 0) lex += fo[d];
      if (o[d] < 0) lex += bo[d];
      odd ^= (o[d] != 0);
    }
    // a 32-bit link offset: 4 V < 2^31 for every volume a context accepts (V <= 2^29)
    return ld_link(U + ((uint32_t)mu * (uint32_t)g.V + (uint32_t)eo_of(g, lex, p ^ odd)));
  };
  auto E = [](int d, int k) { return d == k ? 1 : 0; };
  constexpr int m0 = 2 * HALF, m1 = 2 * HALF + 1;
  const size_t self = (size_t)p * g.Vh + cb;
  if (mode & FM_HAS_IN) {
    prefetch_momenta(P, m0 * V + self, NL);
    prefetch_momenta(P, m1 * V + self, NL);
  }
  Su2<T> K[2] = {zero_su2<T>(), zero_su2<T>()};
#pragma unroll
  for (int nu = 0; nu < 4; nu++) {
    const Su2<T> c = L(nu, -E(nu, 0), -E(nu, 1), -E(nu, 2), -E(nu, 3));  // U_nu(x-nu)
#pragma unroll
    for (int j = 0; j < 2; j++) {
      const int mu = m0 + j;
      if (nu == mu) continue;
      const Su2<T> e = L(nu, E(mu, 0) - E(nu, 0), E(mu, 1) - E(nu, 1), E(mu, 2) - E(nu, 2),
                         E(mu, 3) - E(nu, 3));                           // U_nu(x+mu-nu)
      const Su2<T> h = L(mu, -E(nu, 0), -E(nu, 1), -E(nu, 2), -E(nu, 3));  // U_mu(x-nu)
      Su2<T> eh = mul(dag(e), dag(h));
      if (ANISO) eh = scale((mu == 0 || nu == 0) ? wt : ws, eh);
      K[j] = mul_acc(K[j], eh, c);
    }
  }
#pragma unroll
  for (int nu = 0; nu < 4; nu++) {
    const Su2<T> cn = L(nu, 0, 0, 0, 0);  // U_nu(x)
#pragma unroll
    for (int j = 0; j < 2; j++) {
      const int mu = m0 + j;
      if (nu == mu) continue;
      const bool both = (nu == m0 || nu == m1);
      if (both && nu < mu) continue;
      const Su2<T> a = L(nu, E(mu, 0), E(mu, 1), E(mu, 2), E(mu, 3));  // U_nu(x+mu)
      const Su2<T> b = L(mu, E(nu, 0), E(nu, 1), E(nu, 2), E(nu, 3));  // U_mu(x+nu)
      Su2<T> A = mul(a, dag(b));
      if (ANISO) A = scale((mu == 0 || nu == 0) ? wt : ws, A);
      K[j] = mul_acc(K[j], A, dag(cn));
      if (both) K[nu - m0] = mul_acc(K[nu - m0], dag(A), dag(L(mu, 0, 0, 0, 0)));
    }
  }
  double k2 = 0.;
#pragma unroll
  for (int j = 0; j < 2; j++)
    k2 += finish_link<T>(L(m0 + j, 0, 0, 0, 0), K[j], (m0 + j) * V + self, NL, P, extra, f,
                         scale_, mode, Uout, dt_upd);
  return k2;
}



// The fused force step for one link U_mu(x), one thread per link: its 2(d-1) staples,
//   K = sum_{nu != mu} U_nu(x+mu) U_mu(x+nu)^+ U_nu(x)^+ + U_nu(x+mu-nu)^+ U_mu(x-nu)^+ U_nu(x-nu),
// then finish_link.  6(d-1)+1 link loads and no product shared with another link: more work
// per link than the site bodies, but d times the threads, for lattices too small to fill the
// GPU with one thread per site.  Isotropic action.
template <class T, int ND, int mu>
__device__ __forceinline__ double force_link_impl(const Geom &g, const LinkT<T> *__restrict__ U,
                                                  T *__restrict__ P,
                                                  const T *__restrict__ extra, T f, T scale_,
                                                  int mode, LinkT<T> *__restrict__ Uout,
                                                  T dt_upd, int p, int cb) {
  const int q = 1 - p;
  const Site s = site_from_eo(g, p, cb);
  const size_t V = (size_t)g.V, NL = V * ND;
  const size_t self = (size_t)p * g.Vh + cb;
  const int lpm = s.lex + fwd(g, s, mu);
  Su2<T> K = zero_su2<T>();
#pragma unroll
  for (int nu = 0; nu < ND; nu++) {
    if (nu == mu) continue;
    const int lpn = s.lex + fwd(g, s, nu), bn = bwd(g, s, nu);
    const Su2<T> a = ld_link(U + nu * V + eo_of(g, lpm, q));         // U_nu(x+mu)
    const Su2<T> b = ld_link(U + mu * V + eo_of(g, lpn, q));         // U_mu(x+nu)
    const Su2<T> c = ld_link(U + nu * V + self);                     // U_nu(x)
    const Su2<T> e = ld_link(U + nu * V + eo_of(g, lpm + bn, p));    // U_nu(x+mu-nu)
    const Su2<T> h = ld_link(U + mu * V + eo_of(g, s.lex + bn, q));  // U_mu(x-nu)
    const Su2<T> d = ld_link(U + nu * V + eo_of(g, s.lex + bn, q));  // U_nu(x-nu)
    K = mul_acc(K, mul(a, dag(b)), dag(c));
    K = mul_acc(K, mul(dag(e), dag(h)), d);
  }
  return finish_link<T>(ld_link(U + mu * V + self), K, mu * V + self, NL, P, extra, f, scale_,
                        mode, Uout, dt_upd);
}

// SU(2) elements through shared memory as the aligned storage type (one 128-bit access per
// FP32 element), laid out [2][threads] so that a warp's accesses are consecutive
__device__ __forceinline__ Link32 as_link(const Su2<float> &u) {
  return make_float4(u.ar, u.ai, u.br, u.bi);
}
__device__ __forceinline__ Link64 as_link(const Su2<double> &u) {
  return Link64{u.ar, u.ai, u.br, u.bi};
}
__device__ __forceinline__ Su2<float> from_link(const Link32 &v) {
  return Su2<float>{v.x, v.y, v.z, v.w};
}
__device__ __forceinline__ Su2<double> from_link(const Link64 &v) {
  return Su2<double>{v.ar, v.ai, v.br, v.bi};
}
template <class T> using XchgT = LinkT<T> (*)[128];

// The split force step with each of the four planes that cross the halves formed once per
// site instead of once per half.  With A_{mu,nu} = U_nu(x+mu) U_mu(x+nu)^+ the forward staples
// of a plane are K_mu += A_{mu,nu} U_nu(x)^+ and K_nu += A_{mu,nu}^+ U_mu(x)^+.  The two
// threads of a site (the same lane of a pair of warps) each form two cross products and swap
// them through shared memory:
//   HALF 0 forms A_{0,2}, A_{0,3};  HALF 1 forms A_{2,1} = A_{1,2}^+, A_{3,1} = A_{1,3}^+.
// Each thread loads 26 links instead of 30 and forms two products fewer.  xs is the block's
// exchange array (two products per thread); bar_id names the hardware barrier of the warp
// pair, which every thread of both warps reaches exactly once.  Threads past the end of the
// lattice (valid false) compute a clamped site and write nothing.  Isotropic action only.
__device__ __forceinline__ void warp_pair_sync(int bar_id) {
  // immediate barrier numbers: a register operand makes the compiler reserve all 16
  if (bar_id == 1)
    asm volatile("bar.sync 1, 64;" ::: "memory");
  else
    asm volatile("bar.sync 2, 64;" ::: "memory");
}
template <class T, int HALF>
__device__ __forceinline__ double force_half_x(const Geom &g, const LinkT<T> *__restrict__ U,
                                               T *__restrict__ P, const T *__restrict__ extra,
                                               T f, T scale_, int mode,
                                               LinkT<T> *__restrict__ Uout, T dt_upd, int p,
                                               int cb, bool valid, XchgT<T> xs,
                                               int bar_id) {
  const Site s = site_from_eo(g, p, cb);
  const size_t V = (size_t)g.V, NL = 4 * V;
  int fo[4], bo[4];
#pragma unroll
  for (int d = 0; d < 4; d++) {
    fo[d] = fwd(g, s, d);
    bo[d] = bwd(g, s, d);
  }
  auto L = [&](int mu, int o0, int o1, int o2, int o3) -> Su2<T> {
    const int o[4] = {o0, o1, o2, o3};
    int lex = s.lex, odd = 0;
#pragma unroll
    for (int d = 0; d < 4; d++) {
      if (o[d] > 0) lex += fo[d];
      if (o[d] < 0) lex += bo[d];
      odd ^= (o[d] != 0);
    }
    // a 32-bit link offset: 4 V < 2^31 for every volume a context accepts (V <= 2^29)
    return ld_link(U + ((uint32_t)mu * (uint32_t)g.V + (uint32_t)eo_of(g, lex, p ^ odd)));
  };
  auto E = [](int d, int k) { return d == k ? 1 : 0; };
  constexpr int m0 = 2 * HALF, m1 = 2 * HALF + 1;
  // the two cross products of this thread, published first so the partner can proceed
  Su2<T> X0, X1;
  if (HALF == 0) {
    X0 = mul(L(2, 1, 0, 0, 0), dag(L(0, 0, 0, 1, 0)));  // A_{0,2}
    X1 = mul(L(3, 1, 0, 0, 0), dag(L(0, 0, 0, 0, 1)));  // A_{0,3}
  } else {
    X0 = mul(L(1, 0, 0, 1, 0), dag(L(2, 0, 1, 0, 0)));  // A_{2,1}
    X1 = mul(L(1, 0, 0, 0, 1), dag(L(3, 0, 1, 0, 0)));  // A_{3,1}
  }
  const int t = threadIdx.x;
  xs[0][t] = as_link(X0);
  xs[1][t] = as_link(X1);
  // the plane inside the half
  Su2<T> K[2];
  {
    const Su2<T> A = mul(L(m1, E(m0, 0), E(m0, 1), E(m0, 2), E(m0, 3)),
                         dag(L(m0, E(m1, 0), E(m1, 1), E(m1, 2), E(m1, 3))));
    K[0] = mul(A, dag(L(m1, 0, 0, 0, 0)));
    K[1] = mul(dag(A), dag(L(m0, 0, 0, 0, 0)));
  }
  // backward staples U_nu(x+mu-nu)^+ U_mu(x-nu)^+ U_nu(x-nu)
#pragma unroll
  for (int j = 0; j < 2; j++) {
    const int mu = m0 + j;
#pragma unroll
    for (int nu = 0; nu < 4; nu++) {
      if (nu == mu) continue;
      const Su2<T> e = L(nu, E(mu, 0) - E(nu, 0), E(mu, 1) - E(nu, 1), E(mu, 2) - E(nu, 2),
                         E(mu, 3) - E(nu, 3));
      const Su2<T> h = L(mu, -E(nu, 0), -E(nu, 1), -E(nu, 2), -E(nu, 3));
      const Su2<T> c = L(nu, -E(nu, 0), -E(nu, 1), -E(nu, 2), -E(nu, 3));
      K[j] = mul_acc(K[j], mul(dag(e), dag(h)), c);
    }
  }
  // the partner's cross products
  warp_pair_sync(bar_id);
  const Su2<T> Y0 = from_link(xs[0][t ^ 32]), Y1 = from_link(xs[1][t ^ 32]);
  if (HALF == 0) {  // K_0 += A_{0,k} U_k^+;  K_1 += A_{1,k} U_k^+ with A_{1,k} = Y^+  (k = 2, 3)
    const Su2<T> u2 = L(2, 0, 0, 0, 0), u3 = L(3, 0, 0, 0, 0);
    K[0] = mul_acc(K[0], X0, dag(u2));
    K[0] = mul_acc(K[0], X1, dag(u3));
    K[1] = mul_acc(K[1], dag(Y0), dag(u2));
    K[1] = mul_acc(K[1], dag(Y1), dag(u3));
  } else {  // K_k += A_{k,0} U_0^+ + A_{k,1} U_1^+ with A_{k,0} = A_{0,k}^+ = Y^+  (k = 2, 3)
    const Su2<T> u0 = L(0, 0, 0, 0, 0), u1 = L(1, 0, 0, 0, 0);
    K[0] = mul_acc(K[0], dag(Y0), dag(u0));
    K[0] = mul_acc(K[0], X0, dag(u1));
    K[1] = mul_acc(K[1], dag(Y1), dag(u0));
    K[1] = mul_acc(K[1], X1, dag(u1));
  }
  if (!valid) return 0.;
  const size_t self = (size_t)p * g.Vh + cb;
  double k2 = 0.;
#pragma unroll
  for (int j = 0; j < 2; j++)
    k2 += finish_link<T>(L(m0 + j, 0, 0, 0, 0), K[j], (m0 + j) * V + self, NL, P, extra, f,
                         scale_, mode, Uout, dt_upd);
  return k2;
}

// ReTr U_mu(x) U_nu(x+mu) (U_nu(x) U_mu(x+nu))^+ of one plaquette, in the storage precision:
// FP64 links in FP64; FP32 links (mixed precision) with the products in FP32 (the trace of
// one plaquette to about 1e-7 relative), returned in FP64 for the FP64 sums
template <class T>
__device__ __forceinline__ double plaq_trace(const Su2<T> &um, const Su2<T> &a,
                                             const Su2<T> &un, const Su2<T> &b) {
  return (double)retr_mul(mul(um, a), dag(mul(un, b)));
}

// plaquettes of one site: sums over planes mu<nu of ReTr U_mu(x) U_nu(x+mu) U_mu(x+nu)^+
// U_nu(x)^+ (flat-gauge_energy.hpp:31-94), each plaquette's trace in the storage precision
// (plaq_trace) and every sum in FP64; {full, spatial (mu >= 1), xi-weighted}.  The site's own
// links are read where each plane needs them (L1 hits after the first), so that no more than
// one plane's four links stay live.
template <class T, int ND>
__device__ __forceinline__ void plaq_site(const Geom &g, const LinkT<T> *__restrict__ U, int p,
                                          int cb, double xi, double &full, double &spat,
                                          double &wsum) {
  const Site s = site_from_eo(g, p, cb);
  const LinkT<T> *__restrict__ own = U + (size_t)p * g.Vh + cb;
#pragma unroll
  for (int mu = 0; mu < ND - 1; mu++) {
    const int lpm = s.lex + fwd(g, s, mu);
#pragma unroll
    for (int nu = mu + 1; nu < ND; nu++) {
      const int lpn = s.lex + fwd(g, s, nu);
      const Su2<T> A = ld_link(U + (size_t)nu * g.V + eo_of(g, lpm, 1 - p));
      const Su2<T> B = ld_link(U + (size_t)mu * g.V + eo_of(g, lpn, 1 - p));
      const double tr = plaq_trace<T>(ld_link(own + (size_t)mu * g.V), A,
                                      ld_link(own + (size_t)nu * g.V), B);
      full += tr;
      if (mu >= 1) spat += tr;
      wsum += (((mu == 0) ^ (nu == 0)) ? 1.0 / xi : xi) * tr;
    }
  }
}

// Box-Muller pair from one Philox draw: FP64 from two 53-bit uniforms (all four words).
__device__ __forceinline__ void gauss_pair64(const uint32_t r[4], double &a, double &b) {
  box_muller(u01_53(r[0], r[1]), u01_53(r[2], r[3]), a, b);
}
// The same pair in FP32 arithmetic: the same two 53-bit uniforms (exact integers scaled by
// 2^-53, rounded once to float) through FP32 log, sqrt and sincospi.  The radius keeps the
// FP64 pair's range: u1 >= 2^-53 is a normal float, so |z| reaches sqrt(106 ln 2) = 8.57
// sigma in both precisions (a 24-bit uniform would cut the tail at 5.77 sigma).  The normals
// agree with the FP64 pair to FP32 rounding, so both precisions draw the same momenta.
__device__ __forceinline__ void gauss_pair32(const uint32_t r[4], float &a, float &b) {
  const uint64_t k1 = ((uint64_t)r[0] << 21) ^ (uint64_t)(r[1] >> 11);
  const uint64_t k2 = ((uint64_t)r[2] << 21) ^ (uint64_t)(r[3] >> 11);
  const float u1 = (float)(k1 + 1) * 0x1p-53f;  // (0, 1]
  const float u2 = (float)(k2 + 1) * 0x1p-53f;
  const float rad = sqrtf(-2.0f * logf(u1));
  float sn, cs;
  sincospif(2.0f * u2, &sn, &cs);
  a = rad * cs;
  b = rad * sn;
}

// The three standard normals of the SU(2) momentum of link lref (reference link index) for
// trajectory traj: Philox(seed; {lref, draw, traj, TAG_MOMENTA}), draws 0 and 1, one
// Box-Muller pair of 53-bit uniforms each; FP32 storage evaluates the same pairs in FP32
// arithmetic.  U(1) momenta use the first normal.
template <class T>
__device__ __forceinline__ void momentum_normals(uint32_t lref, uint32_t traj, uint64_t seed,
                                                 int na, T &n0, T &n1, T &n2);
template <>
__device__ __forceinline__ void momentum_normals<double>(uint32_t lref, uint32_t traj,
                                                         uint64_t seed, int na, double &n0,
                                                         double &n1, double &n2) {
  uint32_t r[4];
  double n3;
  philox(lref, 0u, traj, TAG_MOMENTA, seed, r);
  gauss_pair64(r, n0, n1);
  if (na == 3) {
    philox(lref, 1u, traj, TAG_MOMENTA, seed, r);
    gauss_pair64(r, n2, n3);
  }
}
template <>
__device__ __forceinline__ void momentum_normals<float>(uint32_t lref, uint32_t traj,
                                                        uint64_t seed, int na, float &n0,
                                                        float &n1, float &n2) {
  uint32_t r[4];
  float n3;
  philox(lref, 0u, traj, TAG_MOMENTA, seed, r);
  gauss_pair32(r, n0, n1);
  if (na == 3) {
    philox(lref, 1u, traj, TAG_MOMENTA, seed, r);
    gauss_pair32(r, n2, n3);
  }
}

}  // namespace su2b
