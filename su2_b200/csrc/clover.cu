// clover.cu -- clover-leaf energy density and topological charge
// (flat-energy_density.hh:57-164), FP64 arithmetic whatever the link storage.
//
// Per site and plane mu<nu the four leaves
//   U_mu(x) U_nu(x+mu) U_mu(x+nu)^+ U_nu(x)^+            (the plaquette)
//   U_nu(x) U_mu(x-mu+nu)^+ U_nu(x-mu)^+ U_mu(x-mu)
//   U_mu(x-mu)^+ U_nu(x-mu-nu)^+ U_mu(x-mu-nu) U_nu(x-nu)
//   U_nu(x-nu)^+ U_mu(x-nu) U_nu(x+mu-nu) U_mu(x)^+
// are summed (cloverdef) or only the first is used, G = traceless_antiherm(leaf sum),
// E += ReTr(G G), and for d = 4 Q += eps_{i1 i2 i3 i4} ReTr(G_{i1 i2} G_{i3 i4}) over the
// terms with i1<i2, i3<i4; for U(1) in d = 2, Q += -Im G_01.  Per-block partials
// {sum E (all planes), sum E (planes mu >= 1), sum Q}.  This kernel is FP64-compute bound:
// about 2000 flop per site against 32*d bytes of links.
#include "su2b_internal.h"

namespace su2b {
namespace {

template <class T> using LinkT = typename LinkOf<T>::type;

template <class T>
__device__ __forceinline__ Su2<double> L(const Geom &g, const LinkT<T> *U, int mu, int lex,
                                         int p) {
  return to64(ld_link(U + (size_t)mu * g.V + eo_of(g, lex, p)));
}

// FP64 links: six resident blocks per SM (80 registers, 80 bytes of spills) beat the
// compiler's free choice of 104 registers and four blocks (155 against 169 us per call at
// 32^4); with FP32 links four blocks (128 registers, no spills) are as fast as any cap
template <class T, int NT> constexpr int clover_min_blocks() { return sizeof(T) == 8 ? 6 : 4; }

template <class T, int ND, int NT>
__global__ void __launch_bounds__(NT, clover_min_blocks<T, NT>())
  k_clover_su2(Geom g, const LinkT<T> *__restrict__ U, int cloverdef, double *part) {
  __shared__ double shk[4 * (NT / 32)];
  const int p = blockIdx.x & 1;
  // the sites cb0 .. cb0 + ncb - 1 of each parity (all of them but in a time slab)
  const int cb = g.cb0 + (blockIdx.x >> 1) * NT + threadIdx.x;
  double e_all = 0., e_ss = 0., q = 0.;
  if (cb < g.cb0 + g.ncb) {
    const Site s = site_from_eo(g, p, cb);
    Su2<double> G[ND][ND];
#pragma unroll
    for (int mu = 0; mu < ND - 1; mu++)
#pragma unroll
      for (int nu = mu + 1; nu < ND; nu++) {
        const int fm = fwd(g, s, mu), bm = bwd(g, s, mu), fn = fwd(g, s, nu),
                  bn = bwd(g, s, nu);
        const int x = s.lex;
        const int q_ = 1 - p;
        const Su2<double> umu = L<T>(g, U, mu, x, p), unu = L<T>(g, U, nu, x, p);
        Su2<double> leaf =
          mul(mul(umu, L<T>(g, U, nu, x + fm, q_)), dag(mul(unu, L<T>(g, U, mu, x + fn, q_))));
        if (cloverdef) {
          // U_nu(x) U_mu(x-mu+nu)^+ U_nu(x-mu)^+ U_mu(x-mu)
          leaf = add(leaf, mul(mul(unu, dag(L<T>(g, U, mu, x + bm + fn, p))),
                               mul(dag(L<T>(g, U, nu, x + bm, q_)), L<T>(g, U, mu, x + bm, q_))));
          // U_mu(x-mu)^+ U_nu(x-mu-nu)^+ U_mu(x-mu-nu) U_nu(x-nu)
          leaf = add(leaf, mul(mul(dag(L<T>(g, U, mu, x + bm, q_)),
                                   dag(L<T>(g, U, nu, x + bm + bn, p))),
                               mul(L<T>(g, U, mu, x + bm + bn, p), L<T>(g, U, nu, x + bn, q_))));
          // U_nu(x-nu)^+ U_mu(x-nu) U_nu(x+mu-nu) U_mu(x)^+
          leaf = add(leaf, mul(mul(dag(L<T>(g, U, nu, x + bn, q_)), L<T>(g, U, mu, x + bn, q_)),
                               mul(L<T>(g, U, nu, x + fm + bn, p), dag(umu))));
        }
        // traceless_antiherm (su2.hh:83-85): a -> i Im a, b unchanged
        G[mu][nu] = Su2<double>{0.0, leaf.ai, leaf.br, leaf.bi};
        const double t = retr_mul(G[mu][nu], G[mu][nu]);
        e_all += t;
        if (mu >= 1) e_ss += t;
      }
    if (ND == 4) {
      // eps terms with i1<i2, i3<i4 in tensors.hh order
      q += retr_mul(G[0][1], G[2][3]);
      q -= retr_mul(G[0][2], G[1][3]);
      q += retr_mul(G[0][3], G[1][2]);
      q += retr_mul(G[1][2], G[0][3]);
      q -= retr_mul(G[1][3], G[0][2]);
      q += retr_mul(G[2][3], G[0][1]);
    }
  }
  const int b = blockIdx.x;
  double v[3] = {e_all, e_ss, q};
  block_sums<NT, 3>(v, shk);
  if (threadIdx.x == 0) {
    part[3 * b] = v[0];
    part[3 * b + 1] = v[1];
    part[3 * b + 2] = v[2];
  }
}

template <int ND, int NT>
__global__ void __launch_bounds__(NT)
  k_clover_u1(Geom g, const double *__restrict__ U, int cloverdef, double *part) {
  __shared__ double shk[4 * (NT / 32)];
  const int p = blockIdx.x & 1;
  const int cb = (blockIdx.x >> 1) * NT + threadIdx.x;
  double e_all = 0., e_ss = 0., q = 0.;
  if (cb < g.Vh) {
    const Site s = site_from_eo(g, p, cb);
    double G[ND][ND];
    auto A = [&](int mu, int lex, int par) { return U[(size_t)mu * g.V + eo_of(g, lex, par)]; };
#pragma unroll
    for (int mu = 0; mu < ND - 1; mu++)
#pragma unroll
      for (int nu = mu + 1; nu < ND; nu++) {
        const int fm = fwd(g, s, mu), bm = bwd(g, s, mu), fn = fwd(g, s, nu),
                  bn = bwd(g, s, nu);
        const int x = s.lex, q_ = 1 - p;
        double im = sin_pi_scaled(((A(mu, x, p) + A(nu, x + fm, q_)) + (-A(mu, x + fn, q_))) +
                        (-A(nu, x, p)));
        if (cloverdef) {
          im += sin_pi_scaled(((A(nu, x, p) + (-A(mu, x + bm + fn, p))) + (-A(nu, x + bm, q_))) +
                    A(mu, x + bm, q_));
          im += sin_pi_scaled((((-A(mu, x + bm, q_)) + (-A(nu, x + bm + bn, p))) + A(mu, x + bm + bn, p)) +
                    A(nu, x + bn, q_));
          im += sin_pi_scaled((((-A(nu, x + bn, q_)) + A(mu, x + bn, q_)) + A(nu, x + fm + bn, p)) +
                    (-A(mu, x, p)));
        }
        G[mu][nu] = im;  // G = i*im (u1.hh:201-203)
        const double t = -im * im;
        e_all += t;
        if (mu >= 1) e_ss += t;
      }
    if (ND == 4) {
      q += -(G[0][1] * G[2][3]);
      q -= -(G[0][2] * G[1][3]);
      q += -(G[0][3] * G[1][2]);
      q += -(G[1][2] * G[0][3]);
      q -= -(G[1][3] * G[0][2]);
      q += -(G[2][3] * G[0][1]);
    }
    if (ND == 2) q += -G[0][1];
  }
  const int b = blockIdx.x;
  double v[3] = {e_all, e_ss, q};
  block_sums<NT, 3>(v, shk);
  if (threadIdx.x == 0) {
    part[3 * b] = v[0];
    part[3 * b + 1] = v[1];
    part[3 * b + 2] = v[2];
  }
}

}  // namespace

template <class T>
cudaError_t clover_partials(const Geom &g, const void *U, int group, int cloverdef,
                            double *part, int *nblocks, cudaStream_t s) {
  constexpr int NT = 128;
  const dim3 grid(2 * (((group == 0 ? g.ncb : g.Vh) + NT - 1) / NT));
  *nblocks = grid.x;
  if (group == 0) {
    const LinkT<T> *u = (const LinkT<T> *)U;
    switch (g.nd) {
      case 2: k_clover_su2<T, 2, NT><<<grid, NT, 0, s>>>(g, u, cloverdef, part); break;
      case 3: k_clover_su2<T, 3, NT><<<grid, NT, 0, s>>>(g, u, cloverdef, part); break;
      default: k_clover_su2<T, 4, NT><<<grid, NT, 0, s>>>(g, u, cloverdef, part); break;
    }
  } else {
    const double *u = (const double *)U;
    switch (g.nd) {
      case 2: k_clover_u1<2, NT><<<grid, NT, 0, s>>>(g, u, cloverdef, part); break;
      case 3: k_clover_u1<3, NT><<<grid, NT, 0, s>>>(g, u, cloverdef, part); break;
      default: k_clover_u1<4, NT><<<grid, NT, 0, s>>>(g, u, cloverdef, part); break;
    }
  }
  return cudaGetLastError();
}

template cudaError_t clover_partials<double>(const Geom &, const void *, int, int, double *,
                                             int *, cudaStream_t);
template cudaError_t clover_partials<float>(const Geom &, const void *, int, int, double *, int *,
                                            cudaStream_t);

}  // namespace su2b
