// observables.cu -- gauge observables measured between trajectories: the spatially averaged
// Polyakov loop, planar Wilson loops and APE smearing of the links.
//
// All three read the device links in the even/odd layout; products are accumulated in FP64
// whatever the link storage (FP32 links of a mixed-precision context are promoted), and sums
// go through per-block partials reduced in a fixed order.
#include <utility>
#include "site_ops.cuh"
#include "su2b.h"
#include "su2b_ctx.h"

namespace su2b {
namespace {

// link U_mu at lexicographic site lex (parity from the coordinates' sum), as FP64
template <class T>
__device__ __forceinline__ Su2<double> link_at(const Geom &g, const LinkT<T> *__restrict__ U,
                                               int mu, int lex, int par) {
  return to64(ld_link(U + (size_t)mu * g.V + (size_t)par * g.Vh + (lex >> 1)));
}
__device__ __forceinline__ double angle_at(const Geom &g, const double *__restrict__ U, int mu,
                                           int lex, int par) {
  return U[(size_t)mu * g.V + (size_t)par * g.Vh + (lex >> 1)];
}
__device__ __forceinline__ double2 cmul2(double2 x, double2 y) {
  return make_double2(x.x * y.x - x.y * y.y, x.x * y.y + x.y * y.x);
}
// e^{i a} through sincospi(a/pi): exact argument reduction, and no local-memory frame (the
// slow reduction path of sincos keeps one, which every kernel using it then carries)
__device__ __forceinline__ double2 phase(double a) {
  double s, c;
  sincospi(a * 0.318309886183790671537767526745, &s, &c);
  return make_double2(c, s);
}

// A lattice point held as four scalar coordinates.  Steps take the direction at run time;
// with an int[4] indexed by a variable the point (and the geometry) would live in local
// memory, with scalars and a selection it stays in registers.
struct Point {
  int c0, c1, c2, c3;
  __device__ __forceinline__ explicit Point(const Site &s)
    : c0(s.c[0]), c1(s.c[1]), c2(s.c[2]), c3(s.c[3]) {}
  __device__ __forceinline__ static int wrap(int v, int L) {
    return v < 0 ? v + L : (v >= L ? v - L : v);
  }
  __device__ __forceinline__ void step(const Geom &g, int d, int dir) {
    if (d == 0)
      c0 = wrap(c0 + dir, g.L[0]);
    else if (d == 1)
      c1 = wrap(c1 + dir, g.L[1]);
    else if (d == 2)
      c2 = wrap(c2 + dir, g.L[2]);
    else
      c3 = wrap(c3 + dir, g.L[3]);
  }
  __device__ __forceinline__ int lex(const Geom &g) const {
    return ((c0 * g.L[1] + c1) * g.L[2] + c2) * g.L[3] + c3;
  }
  __device__ __forceinline__ int par() const { return (c0 + c1 + c2 + c3) & 1; }
};

// polyakov_loop (polyakov_loop.hh:26-38): one thread per spatial point, the product of the
// temporal links along t, ReTr (SU(2): 2 Re a; U(1): Re of the phase product)
template <class T, int NT>
__global__ void __launch_bounds__(NT)
  k_polyakov(Geom g, const void *__restrict__ Uv, int group, double *part) {
  __shared__ double sh[NT / 32];
  const int V3 = g.L[1] * g.L[2] * g.L[3];
  const int s3 = blockIdx.x * NT + threadIdx.x;
  double v = 0.;
  if (s3 < V3) {
    const int z = s3 % g.L[3], y = (s3 / g.L[3]) % g.L[2], x = s3 / (g.L[3] * g.L[2]);
    if (group == 0) {
      const LinkT<T> *U = (const LinkT<T> *)Uv;
      Su2<double> P{1.0, 0.0, 0.0, 0.0};
      for (int t = 0; t < g.L[0]; t++) P = mul(P, link_at<T>(g, U, 0, t * V3 + s3, (t + x + y + z) & 1));
      v = retr(P);
    } else {
      const double *U = (const double *)Uv;
      double2 P = make_double2(1.0, 0.0);
      for (int t = 0; t < g.L[0]; t++)
        P = cmul2(P, phase(angle_at(g, U, 0, t * V3 + s3, (t + x + y + z) & 1)));
      v = P.x;
    }
  }
  const double r = block_sum<NT>(v, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = r;
}

// planar_wilsonloop_dir (wilsonloop.hh:51-91) summed over the planes (mu, 0), mu >= 1, by
// wilsonloop (wilsonloop.hh:147-157): one thread per site, loop x -> +t e_0 -> +r e_mu ->
// -t e_0 -> -r e_mu
template <class T, int NT>
__global__ void __launch_bounds__(NT)
  k_wilson(Geom g, const void *__restrict__ Uv, int group, int R, int Tt, double *part) {
  __shared__ double sh[NT / 32];
  const int lex0 = blockIdx.x * NT + threadIdx.x;
  double v = 0.;
  if (lex0 < g.V) {
    const Site s0 = site_from_lex(g, lex0);
    for (int mu = 1; mu < g.nd; mu++) {
      Point c(s0);
      auto step = [&](int d, int dir) { c.step(g, d, dir); };
      auto here = [&]() { return c.lex(g); };
      auto par = [&]() { return c.par(); };
      if (group == 0) {
        const LinkT<T> *U = (const LinkT<T> *)Uv;
        Su2<double> L{1.0, 0.0, 0.0, 0.0};
        for (int k = 0; k < Tt; k++) {
          L = mul(L, link_at<T>(g, U, 0, here(), par()));
          step(0, 1);
        }
        for (int k = 0; k < R; k++) {
          L = mul(L, link_at<T>(g, U, mu, here(), par()));
          step(mu, 1);
        }
        for (int k = 0; k < Tt; k++) {
          step(0, -1);
          L = mul(L, dag(link_at<T>(g, U, 0, here(), par())));
        }
        for (int k = 0; k < R; k++) {
          step(mu, -1);
          L = mul(L, dag(link_at<T>(g, U, mu, here(), par())));
        }
        v += retr(L);
      } else {
        const double *U = (const double *)Uv;
        double2 L = make_double2(1.0, 0.0);
        for (int k = 0; k < Tt; k++) {
          L = cmul2(L, phase(angle_at(g, U, 0, here(), par())));
          step(0, 1);
        }
        for (int k = 0; k < R; k++) {
          L = cmul2(L, phase(angle_at(g, U, mu, here(), par())));
          step(mu, 1);
        }
        for (int k = 0; k < Tt; k++) {
          step(0, -1);
          L = cmul2(L, phase(-angle_at(g, U, 0, here(), par())));
        }
        for (int k = 0; k < R; k++) {
          step(mu, -1);
          L = cmul2(L, phase(-angle_at(g, U, mu, here(), par())));
        }
        v += L.x;
      }
    }
  }
  const double r = block_sum<NT>(v, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = r;
}

// APEsmearing (smearape.hh:97-131) with get_staples_APE (get_staples.hh:89-110), one thread
// per link (site, i >= start), reading Uin and writing Uout; links i < start are copied:
//   U'_i(x) = restoreSU(alpha U_i(x) + beta sum_{nu >= start, nu != i}
//              [U_nu(x) U_i(x+nu) U_nu(x+i)^+ + U_nu(x-nu)^+ U_i(x-nu) U_nu(x+i-nu)])
template <class T, int NT>
__global__ void __launch_bounds__(NT)
  k_ape(Geom g, const void *__restrict__ Uin, void *__restrict__ Uout, int group, double alpha,
        double beta, int start) {
  // consecutive blocks take the directions of one band of sites, so the neighbour links a
  // band reads for one direction are still in L2 when the next direction reads them
  const int i = blockIdx.x % g.nd;
  const int lex = (blockIdx.x / g.nd) * NT + threadIdx.x;
  if (lex >= g.V) return;
  const Site s = site_from_lex(g, lex);
  const size_t self = (size_t)i * g.V + (size_t)s.p * g.Vh + (lex >> 1);
  auto at = [&](int d0, int d1, int dir0, int dir1, int *lx, int *pr) {
    Point c(s);
    c.step(g, d0, dir0);
    c.step(g, d1, dir1);
    *lx = c.lex(g);
    *pr = c.par();
  };
  if (group == 0) {
    const LinkT<T> *U = (const LinkT<T> *)Uin;
    LinkT<T> *Uo = (LinkT<T> *)Uout;
    if (i < start) {
      Uo[self] = U[self];
      return;
    }
    Su2<double> K{0.0, 0.0, 0.0, 0.0};
    for (int nu = start; nu < g.nd; nu++) {
      if (nu == i) continue;
      int ln, pn, li, pi, lm, pm, lim, pim;
      at(nu, nu, 1, 0, &ln, &pn);    // x + nu
      at(i, i, 1, 0, &li, &pi);      // x + i
      at(nu, nu, -1, 0, &lm, &pm);   // x - nu
      at(i, nu, 1, -1, &lim, &pim);  // x + i - nu
      K = add(K, mul(mul(link_at<T>(g, U, nu, lex, s.p), link_at<T>(g, U, i, ln, pn)),
                     dag(link_at<T>(g, U, nu, li, pi))));
      K = add(K, mul(mul(dag(link_at<T>(g, U, nu, lm, pm)), link_at<T>(g, U, i, lm, pm)),
                     link_at<T>(g, U, nu, lim, pim)));
    }
    const Su2<double> up = add(scale(alpha, link_at<T>(g, U, i, lex, s.p)), scale(beta, K));
    st_link(Uo + self, from64<T>(restore_su(up)));
  } else {
    const double *U = (const double *)Uin;
    double *Uo = (double *)Uout;
    if (i < start) {
      Uo[self] = U[self];
      return;
    }
    double2 K = make_double2(0.0, 0.0);
    for (int nu = start; nu < g.nd; nu++) {
      if (nu == i) continue;
      int ln, pn, li, pi, lm, pm, lim, pim;
      at(nu, nu, 1, 0, &ln, &pn);
      at(i, i, 1, 0, &li, &pi);
      at(nu, nu, -1, 0, &lm, &pm);
      at(i, nu, 1, -1, &lim, &pim);
      // U(1) products are angle sums; K += exp(i angle)
      const double a1 = (angle_at(g, U, nu, lex, s.p) + angle_at(g, U, i, ln, pn)) +
                        (-angle_at(g, U, nu, li, pi));
      const double a2 = ((-angle_at(g, U, nu, lm, pm)) + angle_at(g, U, i, lm, pm)) +
                        angle_at(g, U, nu, lim, pim);
      const double2 e1 = phase(a1), e2 = phase(a2);
      K = make_double2(K.x + e1.x, K.y + e1.y);
      K = make_double2(K.x + e2.x, K.y + e2.y);
    }
    const double2 e = phase(angle_at(g, U, i, lex, s.p));
    const double2 up = make_double2(alpha * e.x + beta * K.x, alpha * e.y + beta * K.y);
    Uo[self] = atan2(up.y, up.x);
  }
}

constexpr int NT_O = 256;

}  // namespace
}  // namespace su2b

using namespace su2b;

static int enter_ctx(su2b_ctx *ctx) {
  if (!ctx) return SU2B_ERR_INVALID;
  ctx->begin_call();
  SU2B_CK(cudaSetDevice(ctx->device));
  return SU2B_OK;
}

// polyakov_loop_spatial_average (polyakov_loop.hh:48-63): the sum over spatial points divided
// by the full volume, as the reference normalises it
extern "C" int su2b_polyakov_loop(su2b_ctx *ctx, double *out) {
  SU2B_CKS(enter_ctx(ctx));
  SU2B_NEED(out, "out is NULL");
  const int V3 = ctx->g.L[1] * ctx->g.L[2] * ctx->g.L[3];
  const int nb = (V3 + NT_O - 1) / NT_O;
  double *part = ctx->part_slot(0);
  if (ctx->link64)
    k_polyakov<double, NT_O><<<nb, NT_O, 0, ctx->stream>>>(ctx->g, ctx->U, ctx->group, part);
  else
    k_polyakov<float, NT_O><<<nb, NT_O, 0, ctx->stream>>>(ctx->g, ctx->U, ctx->group, part);
  SU2B_CK(cudaGetLastError());
  ctx->launches++;
  SU2B_LAUNCH(SU2B_K_OTHER, reduce_final(part, nb, 1, ctx->red + 48, ctx->stream));
  SU2B_CKS(su2b_fetch_red(ctx, 49));
  *out = ctx->h_red[48] / (double)ctx->V;
  return SU2B_OK;
}

// wilsonloop(U, r, t) (wilsonloop.hh:147-157): the r x t planar loops in the (mu, 0) planes,
// summed over sites and mu >= 1, divided by V Nc ndims
extern "C" int su2b_wilson_loop(su2b_ctx *ctx, int r, int t, double *out) {
  SU2B_CKS(enter_ctx(ctx));
  SU2B_NEED(out, "out is NULL");
  SU2B_NEED(r >= 0 && t >= 0, "loop extents must be non-negative");
  const int nb = (ctx->g.V + NT_O - 1) / NT_O;
  double *part = ctx->part_slot(0);
  if (ctx->link64)
    k_wilson<double, NT_O><<<nb, NT_O, 0, ctx->stream>>>(ctx->g, ctx->U, ctx->group, r, t, part);
  else
    k_wilson<float, NT_O><<<nb, NT_O, 0, ctx->stream>>>(ctx->g, ctx->U, ctx->group, r, t, part);
  SU2B_CK(cudaGetLastError());
  ctx->launches++;
  SU2B_LAUNCH(SU2B_K_OTHER, reduce_final(part, nb, 1, ctx->red + 48, ctx->stream));
  SU2B_CKS(su2b_fetch_red(ctx, 49));
  *out = ctx->h_red[48] / (double)ctx->V / (double)ctx->Nc() / (double)ctx->g.nd;
  return SU2B_OK;
}

// APEsmearing<double>(U, alpha, spatial) (smearape.hh:97-131), in place on the context's field
extern "C" int su2b_ape_smear(su2b_ctx *ctx, double alpha, int spatial) {
  SU2B_CKS(enter_ctx(ctx));
  const int start = spatial ? 1 : 0;
  // the reference refuses d = 2 whatever the choice of directions (smearape.hh:101-104)
  if (ctx->g.nd == 2)
    return su2b_fail(ctx, SU2B_ERR_INVALID, "APE smearing is not possible in 2 dimensions");
  SU2B_CKS(su2b_ensure_aux(ctx));
  const double beta = (1.0 - alpha) / (double)(2 * (ctx->g.nd - 1 - start));
  const dim3 grid(((ctx->g.V + NT_O - 1) / NT_O) * ctx->g.nd);
  if (ctx->link64)
    k_ape<double, NT_O><<<grid, NT_O, 0, ctx->stream>>>(ctx->g, ctx->U, ctx->U_aux, ctx->group,
                                                        alpha, beta, start);
  else
    k_ape<float, NT_O><<<grid, NT_O, 0, ctx->stream>>>(ctx->g, ctx->U, ctx->U_aux, ctx->group,
                                                       alpha, beta, start);
  SU2B_CK(cudaGetLastError());
  ctx->launches++;
  // the smeared field becomes the context's field by exchanging the two buffers (no copy)
  std::swap(ctx->U, ctx->U_aux);
  SU2B_CK(cudaStreamSynchronize(ctx->stream));
  ctx->phases_valid = false;
  return SU2B_OK;
}
