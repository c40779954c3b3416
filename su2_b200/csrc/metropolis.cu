// metropolis.cu -- checkerboard Metropolis pass (flat-sweep.hh:64-164 update rule).
//
// One launch updates every link (x, mu) with parity(x) = p for one direction mu.  Such links
// share no staple: the staple of U_mu(x) contains U_mu(x +- nu) (opposite parity) and links
// of other directions only, so all of them update independently and in any order.  A sweep
// is 2*nd launches.  Per link: staples once (get_staples.hh:26-80), then N_hit proposals
// U -> U R with R = random_element(delta) (random_element.hh:9-34), dS = beta/Nc (ReTr(U K) -
// ReTr(U R K)), accept with min(1, exp(-dS)), restoreSU after each accepted hit.
//   FP64 links: all arithmetic in FP64.
//   FP32 links (mixed precision): the staple sum, the proposal R and the product U R in FP32;
//   the action change dS (the traces of the FP32 values, in FP64), the accept test and the
//   reunitarisation in FP64.
// In both, the accept test u < exp(-dS) goes through accept_fp64, which takes the FP64
// test's decisions (FP32 exp with a guard band, FP64 exp inside the band).  Random numbers:
// one Philox4x32-10 draw per hit, counter {reference link index, hit, sweep, TAG_METRO}:
// 32-bit uniforms for alpha, u, theta and the accept test, the same stream in both
// precisions.
#include "su2b_internal.h"

namespace su2b {
namespace {

template <class T> using LinkT = typename LinkOf<T>::type;

// The FP64 accept test u < exp(-dS) (dS >= 0), decided by FP32 exp where that is safe.  The
// FP32 value differs from the FP64 one by at most the rounding of dS to float (|dS| 2^-24
// relative to the result) plus expf's error (2 ulp); outside a guard band of twice that
// bound the FP32 comparison gives the FP64 decision, inside it (and where expf underflows)
// the test is taken in FP64.  The decisions are those of the FP64 test.
__device__ __forceinline__ bool accept_fp64(double u, double dS) {
  const float ef = expf(-(float)dS);
  if (!(ef > 1e-30f)) return u < exp(-dS);
  const double band = (double)ef * (2.0 * (double)dS * 0x1p-24 + 8.0 * 0x1p-24);
  if (u < (double)ef - band) return true;
  if (u >= (double)ef + band) return false;
  return u < exp(-dS);
}

// One link of a pass with FP32 storage (see the file comment); returns its accepted hits.
template <int ND>
__device__ __forceinline__ unsigned metro_link_fp32(const Geom &g, Link32 *__restrict__ U, int mu,
                                                    int p, int cb, double beta_nc, double delta,
                                                    int N_hit, uint64_t seed, uint32_t sweep,
                                                    float wt, float ws) {
  const Site s = site_from_eo(g, p, cb);
  const int lpm = s.lex + fwd_rt(g, s, mu);  // mu is known at run time only
  Su2<float> K = zero_su2<float>();
#pragma unroll
  for (int nu = 0; nu < ND; nu++) {
    if (nu == mu) continue;
    const int lpn = s.lex + fwd(g, s, nu);
    const Su2<float> A = ld_link_rw(U + (size_t)nu * g.V + eo_of(g, lpm, 1 - p));
    const Su2<float> B = ld_link_rw(U + (size_t)mu * g.V + eo_of(g, lpn, 1 - p));
    const Su2<float> D = ld_link_rw(U + (size_t)nu * g.V + eo_of(g, s.lex, p));
    K = mul_acc(K, scale((nu == 0 || mu == 0) ? wt : ws, mul(A, dag(B))), dag(D));
  }
#pragma unroll
  for (int nu = 0; nu < ND; nu++) {
    if (nu == mu) continue;
    const int b = bwd(g, s, nu);
    const Su2<float> A = ld_link_rw(U + (size_t)nu * g.V + eo_of(g, lpm + b, p));
    const Su2<float> B = ld_link_rw(U + (size_t)mu * g.V + eo_of(g, s.lex + b, 1 - p));
    const Su2<float> D = ld_link_rw(U + (size_t)nu * g.V + eo_of(g, s.lex + b, 1 - p));
    K = mul_acc(K, scale((nu == 0 || mu == 0) ? wt : ws, mul(dag(A), dag(B))), D);
  }
  const Su2<double> K64 = to64(K);
  const size_t l = (size_t)mu * g.V + (size_t)p * g.Vh + cb;
  Su2<float> u = ld_link_rw(U + l);
  double tr_u = retr_mul(to64(u), K64);
  const uint32_t lref = (uint32_t)(s.lex + g.lex0) * (uint32_t)g.nd + (uint32_t)mu;
  const float d2 = (float)(2.0 * delta);
  unsigned acc = 0;
  for (int n = 0; n < N_hit; n++) {
    uint32_t r[4];
    philox(lref, (uint32_t)n, sweep, TAG_METRO, seed, r);
    float sa, ca, st, ct;
    sincospif(d2 * (float)u01_32(r[0]), &sa, &ca);
    const float uu = fmaf(2.0f, (float)u01_32(r[1]), -1.0f);
    sincospif(2.0f * (float)u01_32(r[2]), &st, &ct);
    const float rr = sqrtf(fmaxf(0.0f, fmaf(-uu, uu, 1.0f)));
    const Su2<float> R{ca, sa * uu, sa * rr * st, sa * rr * ct};
    const Su2<float> uR = mul(u, R);
    const double tr_uR = retr_mul(to64(uR), K64);
    const double dS = beta_nc * (tr_u - tr_uR);
    bool a = dS < 0;
    if (!a) a = accept_fp64(u01_32(r[3]), dS);
    if (a) {
      u = from64<float>(restore_su(to64(uR)));
      tr_u = retr_mul(to64(u), K64);
      acc++;
    }
  }
  st_link(U + l, u);
  return acc;
}

// eight resident blocks of 128 threads (64 registers, no spills): the FP64 pass takes 3 %
// less time than with the compiler's free choice of 78 registers; FP32 links use 61 anyway
template <class T, int ND, int NT>
__global__ void __launch_bounds__(NT, 1024 / NT)
  k_metro_su2(Geom g, LinkT<T> *__restrict__ U, int mu, int p, double beta_nc, double delta,
              int N_hit, uint64_t seed, uint32_t sweep, unsigned long long *counts, double wt,
              double ws) {
  __shared__ unsigned int sh_acc;
  if (threadIdx.x == 0) sh_acc = 0;
  __syncthreads();
  // the sites cb0 .. cb0 + ncb - 1 of parity p (all of them but in a time slab)
  const int cb = g.cb0 + blockIdx.x * NT + threadIdx.x;
  unsigned int acc = 0;
  if constexpr (sizeof(T) == 4) {
    if (cb < g.cb0 + g.ncb)
      acc = metro_link_fp32<ND>(g, (Link32 *)U, mu, p, cb, beta_nc, delta, N_hit, seed, sweep,
                                (float)wt, (float)ws);
  } else if (cb < g.cb0 + g.ncb) {
    const Site s = site_from_eo(g, p, cb);
    // staple sum in FP64
    const int lpm = s.lex + fwd_rt(g, s, mu);  // mu is known at run time only
    Su2<double> K = zero_su2<double>();
#pragma unroll
    for (int nu = 0; nu < ND; nu++) {
      if (nu == mu) continue;
      const int lpn = s.lex + fwd(g, s, nu);
      const Su2<double> A = to64(ld_link_rw(U + (size_t)nu * g.V + eo_of(g, lpm, 1 - p)));
      const Su2<double> B = to64(ld_link_rw(U + (size_t)mu * g.V + eo_of(g, lpn, 1 - p)));
      const Su2<double> D = to64(ld_link_rw(U + (size_t)nu * g.V + eo_of(g, s.lex, p)));
      K = add(K, scale((nu == 0 || mu == 0) ? wt : ws, mul(mul(A, dag(B)), dag(D))));
    }
#pragma unroll
    for (int nu = 0; nu < ND; nu++) {
      if (nu == mu) continue;
      const int b = bwd(g, s, nu);
      const Su2<double> A = to64(ld_link_rw(U + (size_t)nu * g.V + eo_of(g, lpm + b, p)));
      const Su2<double> B = to64(ld_link_rw(U + (size_t)mu * g.V + eo_of(g, s.lex + b, 1 - p)));
      const Su2<double> D = to64(ld_link_rw(U + (size_t)nu * g.V + eo_of(g, s.lex + b, 1 - p)));
      K = add(K, scale((nu == 0 || mu == 0) ? wt : ws, mul(mul(dag(A), dag(B)), D)));
    }
    const size_t l = (size_t)mu * g.V + (size_t)p * g.Vh + cb;
    Su2<double> u = to64(ld_link_rw(U + l));
    const uint32_t lref = (uint32_t)(s.lex + g.lex0) * (uint32_t)g.nd + (uint32_t)mu;
    for (int n = 0; n < N_hit; n++) {
      uint32_t r[4];
      philox(lref, (uint32_t)n, sweep, TAG_METRO, seed, r);
      double sa, ca, st, ct;
      sincospi(2.0 * delta * u01_32(r[0]), &sa, &ca);
      const double uu = 2.0 * u01_32(r[1]) - 1.0;
      sincospi(2.0 * u01_32(r[2]), &st, &ct);
      const double rr = sqrt(1.0 - uu * uu);
      const Su2<double> R{ca, sa * uu, sa * rr * st, sa * rr * ct};
      const Su2<double> uR = mul(u, R);
      const double dS = beta_nc * (retr_mul(u, K) - retr_mul(uR, K));
      bool a = dS < 0;
      if (!a) a = accept_fp64(u01_32(r[3]), dS);
      if (a) {
        u = restore_su(uR);
        acc++;
      }
    }
    st_link(U + l, from64<T>(u));
  }
  if (acc) atomicAdd(&sh_acc, acc);
  __syncthreads();
  if (threadIdx.x == 0 && sh_acc) {
    atomicAdd(counts, (unsigned long long)sh_acc);
    if (mu == 0) atomicAdd(counts + 1, (unsigned long long)sh_acc);
  }
}

template <int ND, int NT>
__global__ void __launch_bounds__(NT)
  k_metro_u1(Geom g, double *__restrict__ U, int mu, int p, double beta, double delta,
             int N_hit, uint64_t seed, uint32_t sweep, unsigned long long *counts, double wt,
             double ws) {
  __shared__ unsigned int sh_acc;
  if (threadIdx.x == 0) sh_acc = 0;
  __syncthreads();
  const int cb = blockIdx.x * NT + threadIdx.x;
  unsigned int acc = 0;
  if (cb < g.Vh) {
    const Site s = site_from_eo(g, p, cb);
    const int lpm = s.lex + fwd_rt(g, s, mu);  // mu is known at run time only
    double Kr = 0., Ki = 0.;
#pragma unroll
    for (int nu = 0; nu < ND; nu++) {
      if (nu == mu) continue;
      const int lpn = s.lex + fwd(g, s, nu);
      const double A = U[(size_t)nu * g.V + eo_of(g, lpm, 1 - p)];
      const double B = U[(size_t)mu * g.V + eo_of(g, lpn, 1 - p)];
      const double D = U[(size_t)nu * g.V + eo_of(g, s.lex, p)];
      double sn, cs;
      sincospi(((A + (-B)) + (-D)) * M_1_PI_D, &sn, &cs);
      const double w = (nu == 0 || mu == 0) ? wt : ws;
      Kr += w * cs;
      Ki += w * sn;
    }
#pragma unroll
    for (int nu = 0; nu < ND; nu++) {
      if (nu == mu) continue;
      const int b = bwd(g, s, nu);
      const double A = U[(size_t)nu * g.V + eo_of(g, lpm + b, p)];
      const double B = U[(size_t)mu * g.V + eo_of(g, s.lex + b, 1 - p)];
      const double D = U[(size_t)nu * g.V + eo_of(g, s.lex + b, 1 - p)];
      double sn, cs;
      sincospi((((-A) + (-B)) + D) * M_1_PI_D, &sn, &cs);
      const double w = (nu == 0 || mu == 0) ? wt : ws;
      Kr += w * cs;
      Ki += w * sn;
    }
    const size_t l = (size_t)mu * g.V + (size_t)p * g.Vh + cb;
    double u = U[l];
    const uint32_t lref = (uint32_t)s.lex * (uint32_t)g.nd + (uint32_t)mu;
    for (int n = 0; n < N_hit; n++) {
      uint32_t r[4];
      philox(lref, (uint32_t)n, sweep, TAG_METRO, seed, r);
      const double th = M_PI * delta * (2.0 * u01_32(r[0]) - 1.0);
      double s0, c0, s1, c1;
      sincospi(u * M_1_PI_D, &s0, &c0);
      sincospi((u + th) * M_1_PI_D, &s1, &c1);
      const double dS = beta * ((c0 * Kr - s0 * Ki) - (c1 * Kr - s1 * Ki));
      bool a = dS < 0;
      if (!a) a = u01_32(r[1]) < exp(-dS);
      if (a) {
        u = u + th;
        acc++;
      }
    }
    U[l] = u;
  }
  if (acc) atomicAdd(&sh_acc, acc);
  __syncthreads();
  if (threadIdx.x == 0 && sh_acc) {
    atomicAdd(counts, (unsigned long long)sh_acc);
    if (mu == 0) atomicAdd(counts + 1, (unsigned long long)sh_acc);
  }
}

}  // namespace

template <class T>
cudaError_t metropolis_pass(const Geom &g, void *U, int group, int mu, int parity, double beta,
                            double xi, double delta, int N_hit, uint64_t seed, uint32_t sweep,
                            unsigned long long *counts, cudaStream_t s) {
  constexpr int NT = 128;
  // anisotropic weights of get_staples (get_staples.hh:58-79): 1/xi for planes with
  // direction 0, xi otherwise; both 1 (exactly) for the isotropic action
  const double wt = xi == 1.0 ? 1.0 : 1.0 / xi, ws = xi;
  const int grid = ((group == 0 ? g.ncb : g.Vh) + NT - 1) / NT;
  if (group == 0) {
    LinkT<T> *u = (LinkT<T> *)U;
    const double bn = beta / 2.0;
    switch (g.nd) {
      case 2:
        k_metro_su2<T, 2, NT><<<grid, NT, 0, s>>>(g, u, mu, parity, bn, delta, N_hit, seed,
                                                  sweep, counts, wt, ws);
        break;
      case 3:
        k_metro_su2<T, 3, NT><<<grid, NT, 0, s>>>(g, u, mu, parity, bn, delta, N_hit, seed,
                                                  sweep, counts, wt, ws);
        break;
      default:
        k_metro_su2<T, 4, NT><<<grid, NT, 0, s>>>(g, u, mu, parity, bn, delta, N_hit, seed,
                                                  sweep, counts, wt, ws);
        break;
    }
  } else {
    double *u = (double *)U;
    switch (g.nd) {
      case 2:
        k_metro_u1<2, NT><<<grid, NT, 0, s>>>(g, u, mu, parity, beta, delta, N_hit, seed, sweep,
                                              counts, wt, ws);
        break;
      case 3:
        k_metro_u1<3, NT><<<grid, NT, 0, s>>>(g, u, mu, parity, beta, delta, N_hit, seed, sweep,
                                              counts, wt, ws);
        break;
      default:
        k_metro_u1<4, NT><<<grid, NT, 0, s>>>(g, u, mu, parity, beta, delta, N_hit, seed, sweep,
                                              counts, wt, ws);
        break;
    }
  }
  return cudaGetLastError();
}

template cudaError_t metropolis_pass<double>(const Geom &, void *, int, int, int, double, double,
                                             double, int, uint64_t, uint32_t,
                                             unsigned long long *, cudaStream_t);
template cudaError_t metropolis_pass<float>(const Geom &, void *, int, int, int, double, double,
                                            double, int, uint64_t, uint32_t,
                                            unsigned long long *, cudaStream_t);

}  // namespace su2b
