// adjoint.cu -- reverse-mode derivatives of the Wilson action and of the Wilson flow (SU(2)).
//
// Conventions (those of the reference): the algebra element (a, b, c) of adjointsu2
// (adjointfield.hh:12-51) is X = i(a s_x + b s_y + c s_z) (s = Pauli matrices) and exp_gauge.cc
// computes exp(X); in the (a, b) storage of an SU(2) element, X itself is {a: i c, b: b + i a}.
// get_deriv(S)_k = -ReTr(i s_k S) (adjointfield.hh:53-56).  Derivatives are left derivatives:
// grad O(x, mu)_k = d/dw O(exp(i w s_k) U_mu(x)) at w = 0; with them the derivative of
// get_S_G_hmc is gaugemonomial::derivative (flat-gaugemonomial.hh:105-131).
//
// Force field g(x, mu) = get_deriv(U_mu(x) K_mu(x)) (K = staple sum, get_staples.hh:26-80).
// Its vector-Jacobian product for a cotangent field mu is
//   VJP(x, nu) = get_deriv( U_nu(x) * sum_staples D ),
// where for a staple A B C of the link (A, B, C links or their daggers) the decorated sum is
//   D = A B C M_l + [A] B C + A [B] C + A B [C],   M = i mu.s = {a: i mu_c, b: mu_b + i mu_a},
//   [X] = +M_X X when X is a link traversed forwards, -X M_X when traversed backwards,
// M_l being the cotangent of the link itself.  (Derivation: mu.g = -sum ReTr(M U K); each
// staple term is a plaquette with M inserted at the front of one of its links.)
//
// One RK3 flow step (flat-gradient_flow.hh:17-50): Z_0 = a_0 g(W_0), W_1 = exp(b_0 Z_0) W_0,
// Z_1 = Z_0 + a_1 g(W_1), W_2 = exp(b_1 Z_1) W_1, Z_2 = Z_1 + a_2 g(W_2), W_3 = exp(b_2 Z_2) W_2.
// Reverse through W' = exp(x) W, x = b Z: the cotangent of W is R(x)^T lam' and that of Z is
// b J(x)^T lam', with R the rotation of the adjoint action of exp(x) and J the
// left-trivialised differential of exp (for su(2): ad_x v = -2 x cross v, theta = 2|x|,
// J = 1 + (1 - cos th)/th^2 ad + (th - sin th)/th^3 ad^2).
#include <cmath>
#include <utility>
#include <vector>

#include "su2b.h"
#include "su2b_ctx.h"

using namespace su2b;

namespace {

template <class T> using LinkT = typename LinkOf<T>::type;

template <class T> __device__ __forceinline__ Su2<T> alg(T ma, T mb, T mc) {
  return Su2<T>{T(0), mc, mb, ma};
}

// VJP of the force field, accumulated: lam(x,nu) += coef * VJP(x,nu).  One thread per link.
template <class T, int ND, int NT>
__global__ void __launch_bounds__(NT)
  k_force_vjp(Geom g, const LinkT<T> *__restrict__ U, const T *__restrict__ mu,
              T *__restrict__ lam, T coef, int accumulate) {
  const int nu = blockIdx.y >> 1, p = blockIdx.y & 1, q = 1 - p;
  const int cb = blockIdx.x * NT + threadIdx.x;
  if (cb >= g.Vh) return;
  const Site s = site_from_eo(g, p, cb);
  const size_t V = (size_t)g.V, NL = V * ND;
  auto M = [&](size_t l) { return alg<T>(mu[l], mu[NL + l], mu[2 * NL + l]); };
  const size_t ll = nu * V + (size_t)p * g.Vh + cb;
  const Su2<T> ul = ld_link(U + ll);
  const Su2<T> Ml = M(ll);
  const int lpn = s.lex + fwd(g, s, nu);
  Su2<T> D = zero_su2<T>();
#pragma unroll
  for (int rho = 0; rho < ND; rho++) {
    if (rho == nu) continue;
    // forward: A = U_rho(x+nu), B = U_nu(x+rho)^+, C = U_rho(x)^+
    {
      const size_t la = rho * V + eo_of(g, lpn, q);
      const size_t lb = nu * V + eo_of(g, s.lex + fwd(g, s, rho), q);
      const size_t lc = rho * V + (size_t)p * g.Vh + cb;
      const Su2<T> A = ld_link(U + la), B = dag(ld_link(U + lb)), C = dag(ld_link(U + lc));
      const Su2<T> BC = mul(B, C), AB = mul(A, B), ABC = mul(A, BC);
      D = add(D, mul(ABC, Ml));
      D = add(D, mul(mul(M(la), A), BC));              // A forward: +M A
      D = add(D, scale(T(-1), mul(A, mul(mul(B, M(lb)), C))));  // B backward: -B M
      D = add(D, scale(T(-1), mul(AB, mul(C, M(lc)))));        // C backward: -C M
    }
    // backward: A = U_rho(x+nu-rho)^+, B = U_nu(x-rho)^+, C = U_rho(x-rho)
    {
      const int b = bwd(g, s, rho);
      const size_t la = rho * V + eo_of(g, lpn + b, p);
      const size_t lb = nu * V + eo_of(g, s.lex + b, q);
      const size_t lc = rho * V + eo_of(g, s.lex + b, q);
      const Su2<T> A = dag(ld_link(U + la)), B = dag(ld_link(U + lb)), C = ld_link(U + lc);
      const Su2<T> BC = mul(B, C), AB = mul(A, B), ABC = mul(A, BC);
      D = add(D, mul(ABC, Ml));
      D = add(D, scale(T(-1), mul(mul(A, M(la)), BC)));  // A backward: -A M
      D = add(D, scale(T(-1), mul(A, mul(mul(B, M(lb)), C))));  // B backward: -B M
      D = add(D, mul(AB, mul(M(lc), C)));                // C forward: +M C
    }
  }
  const Su2<T> S = mul(ul, D);
  const T g0 = T(2) * S.bi, g1 = T(2) * S.br, g2 = T(2) * S.ai;
  if (accumulate) {
    lam[ll] += coef * g0;
    lam[NL + ll] += coef * g1;
    lam[2 * NL + ll] += coef * g2;
  } else {
    lam[ll] = coef * g0;
    lam[NL + ll] = coef * g1;
    lam[2 * NL + ll] = coef * g2;
  }
}

// reverse of W' = exp(b Z) W, per link: lam <- R(bZ)^T lam ; mu (+)= b J(bZ)^T lam
template <class T>
__global__ void k_exp_adjoint(size_t NL, const T *__restrict__ Z, T b, T *__restrict__ lam,
                              T *__restrict__ mu, int accumulate) {
  for (size_t l = blockIdx.x * (size_t)blockDim.x + threadIdx.x; l < NL;
       l += (size_t)gridDim.x * blockDim.x) {
    const double x0 = (double)b * Z[l], x1 = (double)b * Z[NL + l], x2 = (double)b * Z[2 * NL + l];
    const double l0 = lam[l], l1 = lam[NL + l], l2 = lam[2 * NL + l];
    const double a2 = x0 * x0 + x1 * x1 + x2 * x2, al = sqrt(a2), th = 2.0 * al;
    // ad v = -2 x cross v ; ad^2 v = 4 (x (x.v) - |x|^2 v)
    auto ad = [&](double v0, double v1, double v2, double &r0, double &r1, double &r2) {
      r0 = -2.0 * (x1 * v2 - x2 * v1);
      r1 = -2.0 * (x2 * v0 - x0 * v2);
      r2 = -2.0 * (x0 * v1 - x1 * v0);
    };
    double c1, c2, s1, s2;  // J = 1 + c1 ad + c2 ad^2 ; R = exp(ad) = 1 + s1 ad + s2 ad^2
    if (th < 1e-3) {
      const double t2 = th * th;
      c1 = 0.5 - t2 / 24.0;
      c2 = 1.0 / 6.0 - t2 / 120.0;
      s1 = 1.0 - t2 / 6.0;
      s2 = 0.5 - t2 / 24.0;
    } else {
      double sn, cs;
      sincospi(th * M_1_PI_D, &sn, &cs);
      c1 = (1.0 - cs) / (th * th);
      c2 = (th - sn) / (th * th * th);
      s1 = sn / th;
      s2 = (1.0 - cs) / (th * th);
    }
    // transposes: ad^T = -ad (skew), (ad^2)^T = ad^2
    double a0, a1, a2v, b0, b1, b2;
    ad(l0, l1, l2, a0, a1, a2v);
    ad(a0, a1, a2v, b0, b1, b2);
    const double r0 = l0 - s1 * a0 + s2 * b0, r1 = l1 - s1 * a1 + s2 * b1,
                 r2 = l2 - s1 * a2v + s2 * b2;
    const double j0 = (double)b * (l0 - c1 * a0 + c2 * b0),
                 j1 = (double)b * (l1 - c1 * a1 + c2 * b1),
                 j2 = (double)b * (l2 - c1 * a2v + c2 * b2);
    lam[l] = (T)r0;
    lam[NL + l] = (T)r1;
    lam[2 * NL + l] = (T)r2;
    if (accumulate) {
      mu[l] += (T)j0;
      mu[NL + l] += (T)j1;
      mu[2 * NL + l] += (T)j2;
    } else {
      mu[l] = (T)j0;
      mu[NL + l] = (T)j1;
      mu[2 * NL + l] = (T)j2;
    }
  }
}

template <class T>
cudaError_t force_vjp(const Geom &g, const void *U, const T *mu, T *lam, double coef, int acc,
                      cudaStream_t s) {
  constexpr int NT = 128;
  const dim3 grid((g.Vh + NT - 1) / NT, 2 * g.nd);
  const LinkT<T> *u = (const LinkT<T> *)U;
  switch (g.nd) {
    case 2: k_force_vjp<T, 2, NT><<<grid, NT, 0, s>>>(g, u, mu, lam, (T)coef, acc); break;
    case 3: k_force_vjp<T, 3, NT><<<grid, NT, 0, s>>>(g, u, mu, lam, (T)coef, acc); break;
    default: k_force_vjp<T, 4, NT><<<grid, NT, 0, s>>>(g, u, mu, lam, (T)coef, acc); break;
  }
  return cudaGetLastError();
}
template <class T>
cudaError_t exp_adjoint(const Geom &g, const T *Z, double b, T *lam, T *mu, int acc,
                        cudaStream_t s) {
  const size_t NL = (size_t)g.V * g.nd;
  const int grid = (int)std::min<size_t>((NL + 255) / 256, 148 * 32);
  k_exp_adjoint<T><<<grid, 256, 0, s>>>(NL, Z, (T)b, lam, mu, acc);
  return cudaGetLastError();
}

// device scratch of one adjoint computation, freed on return
// Scratch carved from the context's arena.  The arena stays allocated between calls (one
// gradient at 24^4 needs about 1.4 GB; allocating and freeing that per call costs
// milliseconds, and cudaFree synchronises the device) and only grows.
struct Scratch {
  char *base = nullptr;
  size_t off = 0, cap = 0;
  void *get(size_t bytes) {
    const size_t b = (bytes + 255) & ~(size_t)255;
    if (off + b > cap) return nullptr;
    void *q = base + off;
    off += b;
    return q;
  }
};
int arena(su2b_ctx *ctx, size_t bytes, Scratch *sc) {
  if (ctx->arena_bytes < bytes) {
    if (ctx->arena) {
      cudaFree(ctx->arena);
      ctx->arena = nullptr;
      ctx->arena_bytes = 0;
    }
    const cudaError_t e = cudaMalloc(&ctx->arena, bytes);
    if (e != cudaSuccess) {
      ctx->arena = nullptr;
      return su2b_fail(ctx, SU2B_ERR_NOMEM, "flow adjoint scratch (%zu bytes): %s", bytes,
                       cudaGetErrorString(e));
    }
    ctx->arena_bytes = bytes;
  }
  sc->base = (char *)ctx->arena;
  sc->off = 0;
  sc->cap = ctx->arena_bytes;
  return SU2B_OK;
}

struct FlowCoef {
  double a[3], b[3];
};
FlowCoef flow_coef(const su2b_ctx *ctx, double eps) {
  // flat-gradient_flow.hh:20-47 via gaugemonomial::derivative's fac*beta/Nc
  const double zfac[3] = {(-17.0) / (36.0), (8.0) / (9.0), (-3.0) / (4.0)};
  const double expfac[3] = {-36.0 / 4. / 17.0, 1., -1.};
  const int Nc = 2;
  FlowCoef c;
  for (int f = 0; f < 3; f++) {
    const double fac = 2. * Nc * zfac[f] / ctx->beta;
    c.a[f] = fac * ctx->beta / (double)Nc;
    c.b[f] = -eps * expfac[f];
  }
  return c;
}

template <class T>
int flow_adjoint_t(su2b_ctx *ctx, double eps, int n, int every, double *objective,
                   double *grad_host) {
  cudaStream_t s = ctx->stream;
  const Geom &g = ctx->g;
  const size_t NL = ctx->NL, lb = ctx->link_bytes() * NL, ab = ctx->adj_bytes() * NL;
  if (every <= 0) every = std::max(1, (int)std::lround(std::sqrt((double)n)));
  const int nseg = (n + every - 1) / every;
  const size_t lb_a = (lb + 255) & ~(size_t)255, ab_a = (ab + 255) & ~(size_t)255;
  Scratch sc;
  SU2B_CKS(arena(ctx, (nseg + every + 3) * lb_a + 5 * ab_a, &sc));
  std::vector<void *> ck(nseg), seg(every);
  for (int i = 0; i < nseg; i++) ck[i] = sc.get(lb);
  for (int i = 0; i < every; i++) seg[i] = sc.get(lb);
  void *W1 = sc.get(lb), *W2 = sc.get(lb), *cur = sc.get(lb);
  T *Zs[3], *lam, *mu;
  for (int f = 0; f < 3; f++) Zs[f] = (T *)sc.get(ab);
  lam = (T *)sc.get(ab);
  mu = (T *)sc.get(ab);
  const FlowCoef c = flow_coef(ctx, eps);
  // Z = a g(W) (+ Z with FM_HAS_IN); with Wn, also Wn = exp(b Z) W from the same kernel
  auto force = [&](const void *W, T *Z, double a, int mode, void *Wn = nullptr,
                   double b = 0.0) {
    return su2b_q_force(ctx, W, Z, nullptr, a, 1.0, Wn ? (mode | FM_UPDATE) : mode, nullptr,
                        nullptr, Wn, b);
  };
  // forward with checkpoints every `every` steps; the field alternates between cur and W1
  // (W1 is free until the backward pass), so every stage is fused with its link update
  SU2B_CK(cudaMemcpyAsync(cur, ctx->U, lb, cudaMemcpyDeviceToDevice, s));
  void *fa = cur, *fb = W1;
  for (int st = 0; st < n; st++) {
    if (st % every == 0)
      SU2B_CK(cudaMemcpyAsync(ck[st / every], fa, lb, cudaMemcpyDeviceToDevice, s));
    SU2B_CKS(su2b_q_flow_step_to(ctx, fa, fb, eps));
    std::swap(fa, fb);
  }
  cur = fa;
  // objective t^2 E_p(t), E_p = d(d-1)/2 - P/(V Nc) (flat-gradient_flow.hh:151)
  SU2B_CKS(su2b_q_plaq(ctx, cur, 40));
  SU2B_CKS(su2b_fetch_red(ctx, 43));
  const double d = g.nd, t = n * eps, VNc = (double)ctx->V * ctx->Nc();
  if (objective) *objective = t * t * (d * (d - 1) / 2.0 - ctx->h_red[40] / VNc);
  if (!grad_host) return SU2B_OK;
  // d O / d V_T (left derivative) = t^2/(V Nc) g(V_T)
  SU2B_CKS(force(cur, lam, t * t / VNc, 0));
  for (int sg = nseg - 1; sg >= 0; sg--) {
    const int s0 = sg * every, s1 = std::min(n, s0 + every);
    SU2B_CK(cudaMemcpyAsync(seg[0], ck[sg], lb, cudaMemcpyDeviceToDevice, s));
    for (int j = 1; j < s1 - s0; j++) {  // seg[j-1] -> seg[j] through W2, seg[j-1] kept
      SU2B_CKS(force(seg[j - 1], Zs[0], c.a[0], 0, seg[j], c.b[0]));
      SU2B_CKS(force(seg[j], Zs[0], c.a[1], FM_HAS_IN, W2, c.b[1]));
      SU2B_CKS(force(W2, Zs[0], c.a[2], FM_HAS_IN, seg[j], c.b[2]));
      if (!ctx->link64) SU2B_CKS(su2b_q_restore(ctx, seg[j]));
    }
    for (int j = s1 - s0 - 1; j >= 0; j--) {
      const void *W0 = seg[j];
      // stages of this step, each fused with its link update
      SU2B_CKS(force(W0, Zs[0], c.a[0], 0, W1, c.b[0]));
      SU2B_CK(cudaMemcpyAsync(Zs[1], Zs[0], ab, cudaMemcpyDeviceToDevice, s));
      SU2B_CKS(force(W1, Zs[1], c.a[1], FM_HAS_IN, W2, c.b[1]));
      SU2B_CK(cudaMemcpyAsync(Zs[2], Zs[1], ab, cudaMemcpyDeviceToDevice, s));
      SU2B_CKS(force(W2, Zs[2], c.a[2], FM_HAS_IN));
      // reverse
      SU2B_LAUNCH(SU2B_K_OTHER, exp_adjoint<T>(g, Zs[2], c.b[2], lam, mu, 0, s));
      SU2B_LAUNCH(SU2B_K_FORCE, force_vjp<T>(g, W2, mu, lam, c.a[2], 1, s));
      SU2B_LAUNCH(SU2B_K_OTHER, exp_adjoint<T>(g, Zs[1], c.b[1], lam, mu, 1, s));
      SU2B_LAUNCH(SU2B_K_FORCE, force_vjp<T>(g, W1, mu, lam, c.a[1], 1, s));
      SU2B_LAUNCH(SU2B_K_OTHER, exp_adjoint<T>(g, Zs[0], c.b[0], lam, mu, 1, s));
      SU2B_LAUNCH(SU2B_K_FORCE, force_vjp<T>(g, W0, mu, lam, c.a[0], 1, s));
    }
  }
  return su2b_adj_download(ctx, lam, grad_host);
}

}  // namespace

extern "C" int su2b_action_backward(su2b_ctx *ctx, double grad_out, double *S, double *dS_host) {
  if (!ctx) return SU2B_ERR_INVALID;
  ctx->begin_call();
  SU2B_CK(cudaSetDevice(ctx->device));
  if (S) {
    SU2B_CKS(su2b_q_plaq(ctx, ctx->U, 40));
    SU2B_CKS(su2b_fetch_red(ctx, 43));
    *S = -ctx->beta * ctx->h_red[42] / ctx->Nc();
  }
  if (!dS_host) return SU2B_OK;
  SU2B_CKS(su2b_q_force(ctx, ctx->U, ctx->Z, nullptr, grad_out * ctx->beta / ctx->Nc(), 1.0, 0,
                        nullptr, nullptr));
  return su2b_adj_download(ctx, ctx->Z, dS_host);
}

extern "C" int su2b_force_vjp(su2b_ctx *ctx, const double *mu_host, double *out_host) {
  if (!ctx) return SU2B_ERR_INVALID;
  ctx->begin_call();
  SU2B_CK(cudaSetDevice(ctx->device));
  SU2B_NEED(mu_host && out_host, "NULL buffer");
  if (ctx->group != SU2B_GROUP_SU2)
    return su2b_fail(ctx, SU2B_ERR_UNSUPPORTED, "the force VJP is provided for SU(2)");
  SU2B_CKS(su2b_adj_upload(ctx, mu_host, ctx->P));
  if (ctx->link64)
    SU2B_LAUNCH(SU2B_K_FORCE, force_vjp<double>(ctx->g, ctx->U, (const double *)ctx->P,
                                                (double *)ctx->Z, 1.0, 0, ctx->stream));
  else
    SU2B_LAUNCH(SU2B_K_FORCE, force_vjp<float>(ctx->g, ctx->U, (const float *)ctx->P,
                                               (float *)ctx->Z, 1.0, 0, ctx->stream));
  return su2b_adj_download(ctx, ctx->Z, out_host);
}

extern "C" int su2b_flow_adjoint(su2b_ctx *ctx, double eps, int n_steps, int checkpoint_every,
                                 double *objective, double *grad_host) {
  if (!ctx) return SU2B_ERR_INVALID;
  ctx->begin_call();
  SU2B_CK(cudaSetDevice(ctx->device));
  SU2B_NEED(n_steps >= 1 && eps > 0, "n_steps >= 1 and eps > 0 required");
  if (ctx->group != SU2B_GROUP_SU2)
    return su2b_fail(ctx, SU2B_ERR_UNSUPPORTED, "the flow adjoint is provided for SU(2)");
  SU2B_NEED(ctx->xi == 1.0, "the flow adjoint needs the isotropic action (xi = 1)");
  const int rc = ctx->link64 ? flow_adjoint_t<double>(ctx, eps, n_steps, checkpoint_every,
                                                      objective, grad_host)
                             : flow_adjoint_t<float>(ctx, eps, n_steps, checkpoint_every,
                                                     objective, grad_host);
  if (rc == SU2B_OK) SU2B_CK(cudaStreamSynchronize(ctx->stream));
  return rc;
}
