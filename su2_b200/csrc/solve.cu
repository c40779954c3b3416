// solve.cu -- host drivers of the staggered operator and Krylov solvers (U(1) only) and of
// the det(D Ddag) pseudofermion monomial (detDDdag_monomial.hh).
//
// Each solver runs as one persistent cooperative launch (CG, mixed CG, BiCGStab in
// staggered.cu) that iterates until convergence behind bounded grid barriers.  Where a
// cooperative launch of one block per SM is not possible, the solvers queue CHUNK iterations
// of per-phase kernels at a time instead; every kernel of an iteration checks the
// device-side SolverState and returns at once after convergence, so the host reads the
// state back once per chunk.  After convergence the true residual |b - A x| is recomputed
// in FP64 and, as CG.hpp:76-84 / BiCGStab.hpp:79-94 do, the solve restarts from x while the
// iterated residual is smaller than the true one.
#include <cmath>
#include <random>
#include <vector>

#include "su2b.h"
#include "su2b_ctx.h"

using namespace su2b;

namespace {

constexpr int CHUNK = 16;

int dalloc2(su2b_ctx *ctx, void **p, size_t bytes) {
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    *p = nullptr;
    return su2b_fail(ctx, SU2B_ERR_NOMEM, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
  }
  ctx->allocs.push_back(*p);
  return SU2B_OK;
}

int put_spinor(su2b_ctx *ctx, const double *host, double2 *dev) {
  SU2B_CK(cudaMemcpyAsync(ctx->stage, host, 2 * ctx->V * sizeof(double), cudaMemcpyHostToDevice,
                          ctx->stream));
  SU2B_LAUNCH(SU2B_K_OTHER, spinor_from_host(ctx->g, ctx->stage, dev, ctx->stream));
  return SU2B_OK;
}
int get_spinor(su2b_ctx *ctx, const double2 *dev, double *host) {
  SU2B_LAUNCH(SU2B_K_OTHER, spinor_to_host(ctx->g, dev, ctx->stage, ctx->stream));
  SU2B_CK(cudaMemcpyAsync(host, ctx->stage, 2 * ctx->V * sizeof(double), cudaMemcpyDeviceToHost,
                          ctx->stream));
  SU2B_CK(cudaStreamSynchronize(ctx->stream));
  return SU2B_OK;
}

int upload_state(su2b_ctx *ctx, const SolverState &h) {
  *ctx->h_st = h;
  SU2B_CK(cudaMemcpyAsync(ctx->st, ctx->h_st, sizeof(SolverState), cudaMemcpyHostToDevice,
                          ctx->stream));
  return SU2B_OK;
}
int fetch_state(su2b_ctx *ctx) {
  SU2B_CK(cudaMemcpyAsync(ctx->h_st, ctx->st, sizeof(SolverState), cudaMemcpyDeviceToHost,
                          ctx->stream));
  SU2B_CK(cudaStreamSynchronize(ctx->stream));
  return SU2B_OK;
}

int ensure_phases(su2b_ctx *ctx, bool need32) {
  if (!ctx->phases_valid) {
    SU2B_LAUNCH(SU2B_K_OTHER, u1_phases(ctx->g, (const double *)ctx->U, ctx->ph, ctx->stream));
    ctx->phases_valid = true;
    ctx->phases32_valid = false;
  }
  if (need32 && !ctx->phases32_valid) {
    SU2B_LAUNCH(SU2B_K_OTHER, u1_phases_f32(ctx->g, (const double *)ctx->U, ctx->ph32, ctx->stream));
    ctx->phases32_valid = true;
  }
  return SU2B_OK;
}

// out = D Ddag in (uses SV_T as scratch)
int apply_ddag64(su2b_ctx *ctx, double m, const double2 *in, double2 *out) {
  SU2B_LAUNCH(SU2B_K_STAGGERED, hop64(ctx->g, ctx->ph, m, 1, in, ctx->sv[SV_T], nullptr, nullptr, nullptr, nullptr, 0,
                ctx->stream));
  SU2B_LAUNCH(SU2B_K_STAGGERED, hop64(ctx->g, ctx->ph, m, 0, ctx->sv[SV_T], out, nullptr, nullptr, nullptr, nullptr, 0,
                ctx->stream));
  return SU2B_OK;
}

// |b - A x|^2 into red[slot], residual into r;  A = D Ddag (ddag) or D
int true_residual(su2b_ctx *ctx, double m, bool ddag, const double2 *b, const double2 *x,
                  double2 *r, int slot) {
  const int n = (int)ctx->V;
  if (ddag)
    SU2B_CKS(apply_ddag64(ctx, m, x, ctx->sv[SV_AP]));
  else
    SU2B_LAUNCH(SU2B_K_STAGGERED, hop64(ctx->g, ctx->ph, m, 0, x, ctx->sv[SV_AP], nullptr, nullptr, nullptr, nullptr,
                  0, ctx->stream));
  SU2B_LAUNCH(SU2B_K_OTHER, resid64(n, b, ctx->sv[SV_AP], r, ctx->part_slot(4), ctx->stream));
  SU2B_LAUNCH(SU2B_K_OTHER, reduce_final(ctx->part_slot(4), vec_blocks(n), 1, ctx->red + slot, ctx->stream));
  return SU2B_OK;
}

int finish_status(su2b_ctx *ctx, int done) {
  if (done == 2)
    return su2b_fail(ctx, SU2B_ERR_NOT_CONVERGED, "solver reached the iteration limit");
  if (done == 3) return su2b_fail(ctx, SU2B_ERR_NOT_CONVERGED, "solver residual is NaN");
  return SU2B_OK;
}

// CG on D Ddag (CG.hpp:36-94), b in SV_B, x in SV_X (start in, solution out)
int cg64(su2b_ctx *ctx, double m, double tol, int max_iter, su2b_solve_stats *stats) {
  const int n = (int)ctx->V;
  const Geom &g = ctx->g;
  cudaStream_t s = ctx->stream;
  double2 *b = ctx->sv[SV_B], *x = ctx->sv[SV_X], *r = ctx->sv[SV_R], *p = ctx->sv[SV_P],
          *t = ctx->sv[SV_T], *Ap = ctx->sv[SV_AP];
  double *dp = ctx->part_slot(3), *np = ctx->part_slot(4);
  SU2B_CKS(true_residual(ctx, m, true, b, x, r, 20));
  SU2B_CKS(su2b_fetch_red(ctx, 21));
  double rr0 = ctx->h_red[20];
  SolverState h{};
  h.rr = make_double2(rr0, 0.0);
  h.rn = sqrt(rr0);
  h.tol = tol;
  h.max_iter = max_iter;
  h.done = (h.rn > tol) ? 0 : 1;
  long restarts = 0;
  for (;;) {
    SU2B_CK(cudaMemcpyAsync(p, r, n * sizeof(double2), cudaMemcpyDeviceToDevice, s));
    SU2B_CKS(upload_state(ctx, h));
    int done = h.done;
    if (!done) {
      // the whole solve in one cooperative launch (two grid barriers per iteration)
      double *slot = ctx->part_slot(5);
      void *bar = slot + 3 * ctx->part_cap - 4;
      const cudaError_t e = cg_persistent(g, ctx->ph, m, x, r, p, t, slot, ctx->st, bar,
                                          (int)(3 * ctx->part_cap - 8), s);
      if (e != cudaErrorNotSupported) {
        SU2B_CK(e);
        ctx->launches++;
        int failed = 0;
        if (cg_barrier_failed(bar, s, &failed))
          return su2b_fail(ctx, SU2B_ERR_CUDA, "persistent CG: %s",
                           cudaGetErrorString(cudaGetLastError()));
        if (failed)
          return su2b_fail(ctx, SU2B_ERR_TIMEOUT, "persistent CG: a grid barrier gave up");
        SU2B_CKS(fetch_state(ctx));
        done = ctx->h_st->done;
      }
    }
    while (!done) {
      for (int k = 0; k < CHUNK; k++) {
        SU2B_LAUNCH(SU2B_K_STAGGERED, hop64(g, ctx->ph, m, 1, p, t, nullptr, nullptr, nullptr, ctx->st, 0, s));
        SU2B_LAUNCH(SU2B_K_STAGGERED, hop64(g, ctx->ph, m, 0, t, Ap, p, dp, nullptr, ctx->st, 0, s));
        SU2B_LAUNCH(SU2B_K_OTHER, cg_alpha(dp, hop_blocks(g), ctx->st, s));
        SU2B_LAUNCH(SU2B_K_OTHER, cg_xr(n, x, r, p, Ap, ctx->st, np, s));
        SU2B_LAUNCH(SU2B_K_OTHER, cg_beta(np, vec_blocks(n), ctx->st, s));
        SU2B_LAUNCH(SU2B_K_OTHER, cg_p(n, r, p, ctx->st, s));
      }
      SU2B_CKS(fetch_state(ctx));
      done = ctx->h_st->done;
    }
    h = *ctx->h_st;
    if (done != 1) break;
    SU2B_CKS(true_residual(ctx, m, true, b, x, ctx->sv[SV_S], 20));
    SU2B_CKS(su2b_fetch_red(ctx, 21));
    const double ex = sqrt(ctx->h_red[20]);
    if (h.rn < ex && h.iters < h.max_iter) {
      restarts++;
      SU2B_CK(cudaMemcpyAsync(r, ctx->sv[SV_S], n * sizeof(double2), cudaMemcpyDeviceToDevice, s));
      h.rr = make_double2(ctx->h_red[20], 0.0);
      h.rn = ex;
      h.done = (h.rn > tol) ? 0 : 1;
      continue;
    }
    if (stats) stats->true_residual = ex;
    break;
  }
  if (stats) {
    stats->iterations = h.iters;
    stats->restarts = restarts;
    stats->residual = h.rn;
  }
  return finish_status(ctx, h.done);
}

// BiCGStab on D (BiCGStab.hpp:36-106)
int bicgstab64(su2b_ctx *ctx, double m, double tol, int max_iter, su2b_solve_stats *stats) {
  const int n = (int)ctx->V;
  const Geom &g = ctx->g;
  cudaStream_t s = ctx->stream;
  double2 *b = ctx->sv[SV_B], *x = ctx->sv[SV_X], *r = ctx->sv[SV_R], *p = ctx->sv[SV_P],
          *t = ctx->sv[SV_T], *Ap = ctx->sv[SV_AP], *sv = ctx->sv[SV_S], *r0 = ctx->sv[SV_R0];
  double *dp = ctx->part_slot(3), *np = ctx->part_slot(3) + 2 * ctx->part_cap;
  double *dp2 = ctx->part_slot(5), *np2 = ctx->part_slot(5) + 2 * ctx->part_cap;
  SU2B_CKS(true_residual(ctx, m, false, b, x, r0, 20));
  SU2B_CKS(su2b_fetch_red(ctx, 21));
  SolverState h{};
  h.r0r = make_double2(ctx->h_red[20], 0.0);
  h.rn = sqrt(ctx->h_red[20]);
  h.tol = tol;
  h.max_iter = max_iter;
  h.done = (h.rn > tol) ? 0 : 1;
  long restarts = 0;
  for (;;) {
    SU2B_CK(cudaMemcpyAsync(r, r0, n * sizeof(double2), cudaMemcpyDeviceToDevice, s));
    SU2B_CK(cudaMemcpyAsync(p, r0, n * sizeof(double2), cudaMemcpyDeviceToDevice, s));
    SU2B_CKS(upload_state(ctx, h));
    int done = h.done;
    if (!done) {
      // the whole solve in one cooperative launch (three grid barriers per iteration)
      double *slot = ctx->part_slot(5);
      void *bar = slot + 3 * ctx->part_cap - 4;
      const cudaError_t e =
        bicgstab_persistent(g, ctx->ph, m, x, r, r0, p, ctx->sv[SV_P2], Ap, ctx->sv[SV_AP2], sv,
                            t, slot, ctx->st, bar, (int)(3 * ctx->part_cap - 8), s);
      if (e != cudaErrorNotSupported) {
        SU2B_CK(e);
        ctx->launches++;
        int failed = 0;
        if (cg_barrier_failed(bar, s, &failed))
          return su2b_fail(ctx, SU2B_ERR_CUDA, "persistent BiCGStab: %s",
                           cudaGetErrorString(cudaGetLastError()));
        if (failed)
          return su2b_fail(ctx, SU2B_ERR_TIMEOUT, "persistent BiCGStab: a grid barrier gave up");
        SU2B_CKS(fetch_state(ctx));
        done = ctx->h_st->done;
      }
    }
    while (!done) {
      for (int k = 0; k < CHUNK; k++) {
        SU2B_LAUNCH(SU2B_K_STAGGERED, hop64(g, ctx->ph, m, 0, p, Ap, r0, dp, nullptr, ctx->st, 0, s));
        SU2B_LAUNCH(SU2B_K_OTHER, bi_alpha(dp, hop_blocks(g), ctx->st, s));
        SU2B_LAUNCH(SU2B_K_OTHER, bi_s(n, r, Ap, sv, ctx->st, s));
        SU2B_LAUNCH(SU2B_K_STAGGERED, hop64(g, ctx->ph, m, 0, sv, t, sv, dp, np, ctx->st, 0, s));
        SU2B_LAUNCH(SU2B_K_OTHER, bi_omega(dp, np, hop_blocks(g), ctx->st, s));
        SU2B_LAUNCH(SU2B_K_OTHER, bi_rx(n, x, r, sv, t, p, r0, ctx->st, dp2, np2, s));
        SU2B_LAUNCH(SU2B_K_OTHER, bi_beta(dp2, np2, vec_blocks(n), ctx->st, s));
        SU2B_LAUNCH(SU2B_K_OTHER, bi_p(n, r, p, Ap, ctx->st, s));
      }
      SU2B_CKS(fetch_state(ctx));
      done = ctx->h_st->done;
    }
    h = *ctx->h_st;
    if (done != 1) break;
    SU2B_CKS(true_residual(ctx, m, false, b, x, r0, 20));
    SU2B_CKS(su2b_fetch_red(ctx, 21));
    const double ex = sqrt(ctx->h_red[20]);
    if (h.rn < ex && h.iters < h.max_iter) {
      restarts++;
      h.r0r = make_double2(ctx->h_red[20], 0.0);
      h.rn = ex;
      h.done = (h.rn > tol) ? 0 : 1;
      continue;
    }
    if (stats) stats->true_residual = ex;
    break;
  }
  if (stats) {
    stats->iterations = h.iters;
    stats->restarts = restarts;
    stats->residual = h.rn;
  }
  return finish_status(ctx, h.done);
}

// CG on D Ddag with FP32 iterations and FP64 reliable updates: the FP64 residual
// b - A x is recomputed whenever the iterated FP32 residual has dropped by `delta` since the
// last update (or reached the tolerance); convergence is decided on that FP64 residual.
int cg_mixed(su2b_ctx *ctx, double m, double tol, int max_iter, double delta,
             su2b_solve_stats *stats) {
  const int n = (int)ctx->V;
  const Geom &g = ctx->g;
  cudaStream_t s = ctx->stream;
  double2 *b = ctx->sv[SV_B], *x = ctx->sv[SV_X], *r = ctx->sv[SV_R], *t = ctx->sv[SV_T],
          *Ap = ctx->sv[SV_AP];
  float2 *xs = ctx->sv32[SV32_XS], *rs = ctx->sv32[SV32_RS], *ps = ctx->sv32[SV32_PS],
         *ts = ctx->sv32[SV32_TS], *Aps = ctx->sv32[SV32_APS];
  const float m32 = (float)m;
  double *dp = ctx->part_slot(3), *np = ctx->part_slot(4), *np2 = ctx->part_slot(5);
  SU2B_CKS(true_residual(ctx, m, true, b, x, r, 20));
  SU2B_LAUNCH(SU2B_K_OTHER, to32(n, r, rs, s));
  SU2B_CK(cudaMemsetAsync(xs, 0, n * sizeof(float2), s));
  SU2B_CK(cudaMemcpyAsync(ps, rs, n * sizeof(float2), cudaMemcpyDeviceToDevice, s));
  SU2B_CKS(su2b_fetch_red(ctx, 21));
  SolverState h{};
  h.rr = make_double2(ctx->h_red[20], 0.0);
  h.rn = sqrt(ctx->h_red[20]);
  h.maxr = h.rn;
  h.delta = delta > 0 ? delta : 0.1;
  h.tol = tol;
  h.max_iter = max_iter;
  h.done = (h.rn > tol) ? 0 : 1;
  SU2B_CKS(upload_state(ctx, h));
  int done = h.done;
  if (!done) {
    // the whole solve in one cooperative launch
    double *slot = ctx->part_slot(5);
    void *bar = slot + 3 * ctx->part_cap - 4;
    const cudaError_t e = cg_mixed_persistent(g, ctx->ph, ctx->ph32, m, b, x, r, t, xs, rs, ps,
                                              ts, slot, ctx->st, bar,
                                              (int)(3 * ctx->part_cap - 8), s);
    if (e != cudaErrorNotSupported) {
      SU2B_CK(e);
      ctx->launches++;
      int failed = 0;
      if (cg_barrier_failed(bar, s, &failed))
        return su2b_fail(ctx, SU2B_ERR_CUDA, "persistent mixed CG: %s",
                         cudaGetErrorString(cudaGetLastError()));
      if (failed)
        return su2b_fail(ctx, SU2B_ERR_TIMEOUT, "persistent mixed CG: a grid barrier gave up");
      SU2B_CKS(fetch_state(ctx));
      h = *ctx->h_st;
      if (stats) {
        stats->iterations = h.iters;
        stats->restarts = h.updates;
        stats->residual = h.rn;
        stats->true_residual = h.rn;
      }
      return finish_status(ctx, h.done);
    }
  }
  while (!done) {
    for (int k = 0; k < CHUNK; k++) {
      SU2B_LAUNCH(SU2B_K_STAGGERED, hop32(g, ctx->ph32, m32, 1, ps, ts, nullptr, nullptr, nullptr, ctx->st, s));
      SU2B_LAUNCH(SU2B_K_STAGGERED, hop32(g, ctx->ph32, m32, 0, ts, Aps, ps, dp, nullptr, ctx->st, s));
      SU2B_LAUNCH(SU2B_K_OTHER, cg_alpha(dp, hop_blocks(g), ctx->st, s));
      SU2B_LAUNCH(SU2B_K_OTHER, m_xr(n, xs, rs, ps, Aps, ctx->st, np, s));
      SU2B_LAUNCH(SU2B_K_OTHER, m_check(np, vec_blocks(n), ctx->st, s));
      SU2B_LAUNCH(SU2B_K_OTHER, m_accum(n, x, xs, ctx->st, s));
      SU2B_LAUNCH(SU2B_K_STAGGERED, hop64(g, ctx->ph, m, 1, x, t, nullptr, nullptr, nullptr, ctx->st, 1, s));
      SU2B_LAUNCH(SU2B_K_STAGGERED, hop64(g, ctx->ph, m, 0, t, Ap, nullptr, nullptr, nullptr, ctx->st, 1, s));
      SU2B_LAUNCH(SU2B_K_OTHER, m_resid(n, b, Ap, r, rs, ctx->st, np2, s));
      SU2B_LAUNCH(SU2B_K_OTHER, m_after(np2, vec_blocks(n), ctx->st, s));
      SU2B_LAUNCH(SU2B_K_OTHER, m_p(n, rs, ps, ctx->st, s));
    }
    SU2B_CKS(fetch_state(ctx));
    done = ctx->h_st->done;
  }
  h = *ctx->h_st;
  if (done == 2 || done == 3) {
    // fold the FP32 correction into x before returning
    h.do_update = 1;
    h.done = 0;
    SU2B_CKS(upload_state(ctx, h));
    SU2B_LAUNCH(SU2B_K_OTHER, m_accum(n, x, xs, ctx->st, s));
  }
  if (stats) {
    stats->iterations = h.iters;
    stats->restarts = h.updates;
    stats->residual = h.rn;
    stats->true_residual = h.rn;
  }
  return finish_status(ctx, done);
}

// the reference's CG start: real Gaussian, sigma = 10, std::mt19937(seed)
// (staggered.hpp:175-193, 267-268), generated with the same <random> engine
int reference_start(su2b_ctx *ctx, long seed) {
  if (ctx->x0_seed == seed) return SU2B_OK;
  std::vector<double> v(2 * ctx->V);
  std::mt19937 gen((size_t)seed);
  std::normal_distribution<double> dis{0.0, 10.0};
  for (size_t i = 0; i < ctx->V; i++) {
    v[2 * i] = dis(gen);
    v[2 * i + 1] = 0.0;
  }
  SU2B_CKS(put_spinor(ctx, v.data(), ctx->sv[SV_X0]));
  SU2B_CK(cudaStreamSynchronize(ctx->stream));
  ctx->x0_seed = seed;
  return SU2B_OK;
}

int set_start(su2b_ctx *ctx, int cg_start, long seed) {
  if (cg_start == SU2B_CG_START_ZERO) {
    SU2B_CK(cudaMemsetAsync(ctx->sv[SV_X], 0, ctx->V * sizeof(double2), ctx->stream));
    return SU2B_OK;
  }
  SU2B_CKS(reference_start(ctx, seed));
  SU2B_CK(cudaMemcpyAsync(ctx->sv[SV_X], ctx->sv[SV_X0], ctx->V * sizeof(double2),
                          cudaMemcpyDeviceToDevice, ctx->stream));
  return SU2B_OK;
}

// chi = (D Ddag)^-1 phi into SV_X (b = phi copied to SV_B)
int solve_phi(su2b_ctx *ctx, double mass, double tol, int max_iter, long *iters) {
  SU2B_CK(cudaMemcpyAsync(ctx->sv[SV_B], ctx->sv[SV_PHI], ctx->V * sizeof(double2),
                          cudaMemcpyDeviceToDevice, ctx->stream));
  su2b_solve_stats st{};
  int rc;
  if (ctx->prec == SU2B_PREC_MIXED) {
    SU2B_CKS(ensure_phases(ctx, true));
    rc = cg_mixed(ctx, mass, tol, max_iter, 0.1, &st);
  } else {
    rc = cg64(ctx, mass, tol, max_iter, &st);
  }
  *iters += st.iterations;
  return rc;
}

}  // namespace

// ===================================================================================
int su2b_fermion_setup(su2b_ctx *ctx, bool need32) {
  if (ctx->group != SU2B_GROUP_U1)
    return su2b_fail(ctx, SU2B_ERR_UNSUPPORTED,
                     "staggered fermions are not supported for SU(2) (staggered.hpp:343-350)");
  if (!ctx->ph) {
    SU2B_CKS(dalloc2(ctx, (void **)&ctx->ph, ctx->NL * sizeof(double2)));
    SU2B_CKS(dalloc2(ctx, (void **)&ctx->fderiv, ctx->NL * sizeof(double)));
    SU2B_CKS(dalloc2(ctx, (void **)&ctx->st, sizeof(SolverState)));
    for (int k = 0; k < SV_N; k++)
      SU2B_CKS(dalloc2(ctx, (void **)&ctx->sv[k], ctx->V * sizeof(double2)));
    ctx->phases_valid = false;
  }
  if (need32 && !ctx->ph32) {
    SU2B_CKS(dalloc2(ctx, (void **)&ctx->ph32, ctx->NL * sizeof(float2)));
    for (int k = 0; k < SV32_N; k++)
      SU2B_CKS(dalloc2(ctx, (void **)&ctx->sv32[k], ctx->V * sizeof(float2)));
    ctx->phases32_valid = false;
  }
  return ensure_phases(ctx, need32);
}

// derivative of the pseudofermion action into ctx->fderiv (phi in SV_PHI)
int su2b_fermion_deriv_q(su2b_ctx *ctx, double mass, double tol, int max_iter, int cg_start,
                         long seed, long *iters) {
  SU2B_CKS(su2b_fermion_setup(ctx, ctx->prec == SU2B_PREC_MIXED));
  SU2B_CKS(set_start(ctx, cg_start, seed));
  SU2B_CKS(solve_phi(ctx, mass, tol, max_iter, iters));
  SU2B_LAUNCH(SU2B_K_STAGGERED, hop64(ctx->g, ctx->ph, mass, 1, ctx->sv[SV_X], ctx->sv[SV_CHI1], nullptr, nullptr,
                nullptr, nullptr, 0, ctx->stream));
  SU2B_LAUNCH(SU2B_K_STAGGERED, fermion_force(ctx->g, ctx->ph, ctx->sv[SV_X], ctx->sv[SV_CHI1], ctx->fderiv,
                        ctx->stream));
  return SU2B_OK;
}

// Re phi^+ (D Ddag)^-1 phi into red[red_slot]
int su2b_fermion_action_q(su2b_ctx *ctx, double mass, double tol, int max_iter, int cg_start,
                          long seed, int red_slot, long *iters) {
  SU2B_CKS(su2b_fermion_setup(ctx, ctx->prec == SU2B_PREC_MIXED));
  SU2B_CKS(set_start(ctx, cg_start, seed));
  SU2B_CKS(solve_phi(ctx, mass, tol, max_iter, iters));
  const int n = (int)ctx->V;
  SU2B_LAUNCH(SU2B_K_OTHER, dot64(n, ctx->sv[SV_PHI], ctx->sv[SV_X], ctx->part_slot(4), ctx->stream));
  SU2B_LAUNCH(SU2B_K_OTHER, reduce_final(ctx->part_slot(4), vec_blocks(n), 2, ctx->red + 30, ctx->stream));
  SU2B_CK(cudaMemcpyAsync(ctx->red + red_slot, ctx->red + 30, sizeof(double),
                          cudaMemcpyDeviceToDevice, ctx->stream));
  return SU2B_OK;
}

// heatbath (detDDdag_monomial.hh:64-83): phi = D R into SV_PHI, |R|^2 into red[red_slot]
int su2b_fermion_heatbath_q(su2b_ctx *ctx, double mass, const double *R_host, uint64_t seed,
                            uint32_t traj, int cplx, int red_slot) {
  SU2B_CKS(su2b_fermion_setup(ctx, ctx->prec == SU2B_PREC_MIXED));
  double2 *R = ctx->sv[SV_S];
  if (R_host)
    SU2B_CKS(put_spinor(ctx, R_host, R));
  else
    SU2B_LAUNCH(SU2B_K_OTHER, pf_source(ctx->g, seed, traj, cplx, R, ctx->stream));
  SU2B_LAUNCH(SU2B_K_STAGGERED, hop64(ctx->g, ctx->ph, mass, 0, R, ctx->sv[SV_PHI], nullptr, nullptr, nullptr, nullptr,
                0, ctx->stream));
  const int n = (int)ctx->V;
  SU2B_LAUNCH(SU2B_K_OTHER, dot64(n, R, R, ctx->part_slot(4), ctx->stream));
  SU2B_LAUNCH(SU2B_K_OTHER, reduce_final(ctx->part_slot(4), vec_blocks(n), 2, ctx->red + 30, ctx->stream));
  SU2B_CK(cudaMemcpyAsync(ctx->red + red_slot, ctx->red + 30, sizeof(double),
                          cudaMemcpyDeviceToDevice, ctx->stream));
  return SU2B_OK;
}

extern "C" int su2b_staggered_apply(su2b_ctx *ctx, int op, double mass, const double *psi_host,
                                    double *out_host) {
  if (!ctx) return SU2B_ERR_INVALID;
  ctx->begin_call();
  SU2B_CK(cudaSetDevice(ctx->device));
  SU2B_NEED(psi_host && out_host, "NULL buffer");
  SU2B_NEED(op == SU2B_OP_D || op == SU2B_OP_DDAG || op == SU2B_OP_DDDAG, "bad op %d", op);
  SU2B_CKS(su2b_fermion_setup(ctx, false));
  SU2B_CKS(put_spinor(ctx, psi_host, ctx->sv[SV_B]));
  if (op == SU2B_OP_DDDAG)
    SU2B_CKS(apply_ddag64(ctx, mass, ctx->sv[SV_B], ctx->sv[SV_X]));
  else
    SU2B_LAUNCH(SU2B_K_STAGGERED, hop64(ctx->g, ctx->ph, mass, op == SU2B_OP_DDAG, ctx->sv[SV_B], ctx->sv[SV_X],
                  nullptr, nullptr, nullptr, nullptr, 0, ctx->stream));
  return get_spinor(ctx, ctx->sv[SV_X], out_host);
}

extern "C" int su2b_solve(su2b_ctx *ctx, const su2b_solve_params *prm, const double *b_host,
                          const double *x0_host, double *x_host, su2b_solve_stats *stats) {
  if (!ctx) return SU2B_ERR_INVALID;
  ctx->begin_call();
  SU2B_CK(cudaSetDevice(ctx->device));
  SU2B_NEED(prm && b_host && x_host, "NULL argument");
  SU2B_NEED(prm->max_iter > 0, "max_iter must be positive");
  const bool mixed = prm->solver == SU2B_SOLVER_CG_MIXED;
  if (prm->solver == SU2B_SOLVER_BICGSTAB)
    SU2B_NEED(prm->op == SU2B_OP_D, "BiCGStab solves D x = b (op = SU2B_OP_D)");
  else if (prm->solver == SU2B_SOLVER_CG || mixed)
    SU2B_NEED(prm->op == SU2B_OP_DDDAG, "CG solves D Ddag x = b (op = SU2B_OP_DDDAG)");
  else
    return su2b_fail(ctx, SU2B_ERR_INVALID, "unknown solver %d", prm->solver);
  SU2B_CKS(su2b_fermion_setup(ctx, mixed));
  SU2B_CKS(put_spinor(ctx, b_host, ctx->sv[SV_B]));
  if (x0_host)
    SU2B_CKS(put_spinor(ctx, x0_host, ctx->sv[SV_X]));
  else
    SU2B_CK(cudaMemsetAsync(ctx->sv[SV_X], 0, ctx->V * sizeof(double2), ctx->stream));
  double tol = prm->tol;
  if (prm->tol_mode == SU2B_TOL_REL) {
    const int n = (int)ctx->V;
    SU2B_LAUNCH(SU2B_K_OTHER, dot64(n, ctx->sv[SV_B], ctx->sv[SV_B], ctx->part_slot(4), ctx->stream));
    SU2B_LAUNCH(SU2B_K_OTHER, reduce_final(ctx->part_slot(4), vec_blocks(n), 2, ctx->red + 30, ctx->stream));
    SU2B_CKS(su2b_fetch_red(ctx, 32));
    tol = prm->tol * sqrt(ctx->h_red[30]);
  }
  su2b_solve_stats st{};
  int rc;
  if (prm->solver == SU2B_SOLVER_CG)
    rc = cg64(ctx, prm->mass, tol, prm->max_iter, &st);
  else if (mixed)
    rc = cg_mixed(ctx, prm->mass, tol, prm->max_iter, prm->delta, &st);
  else
    rc = bicgstab64(ctx, prm->mass, tol, prm->max_iter, &st);
  if (stats) *stats = st;
  if (rc != SU2B_OK && rc != SU2B_ERR_NOT_CONVERGED) return rc;
  SU2B_CKS(get_spinor(ctx, ctx->sv[SV_X], x_host));
  return rc;
}

static int fermion_common(su2b_ctx *ctx, double mass, const double *phi_host, double tol,
                          int max_iter, const double *x0_host, long seed, long *iters) {
  SU2B_NEED(phi_host, "phi_host is NULL");
  SU2B_NEED(max_iter > 0, "max_iter must be positive");
  SU2B_CKS(su2b_fermion_setup(ctx, ctx->prec == SU2B_PREC_MIXED));
  SU2B_CKS(put_spinor(ctx, phi_host, ctx->sv[SV_PHI]));
  if (x0_host)
    SU2B_CKS(put_spinor(ctx, x0_host, ctx->sv[SV_X]));
  else
    SU2B_CKS(set_start(ctx, SU2B_CG_START_REFERENCE, seed));
  return solve_phi(ctx, mass, tol, max_iter, iters);
}

extern "C" int su2b_fermion_force(su2b_ctx *ctx, double mass, const double *phi_host,
                                  double tol, int max_iter, const double *x0_host, long seed,
                                  double *deriv_host, long *cg_iterations) {
  if (!ctx) return SU2B_ERR_INVALID;
  ctx->begin_call();
  SU2B_CK(cudaSetDevice(ctx->device));
  SU2B_NEED(deriv_host, "deriv_host is NULL");
  long it = 0;
  SU2B_CKS(fermion_common(ctx, mass, phi_host, tol, max_iter, x0_host, seed, &it));
  SU2B_LAUNCH(SU2B_K_STAGGERED, hop64(ctx->g, ctx->ph, mass, 1, ctx->sv[SV_X], ctx->sv[SV_CHI1], nullptr, nullptr,
                nullptr, nullptr, 0, ctx->stream));
  SU2B_LAUNCH(SU2B_K_STAGGERED, fermion_force(ctx->g, ctx->ph, ctx->sv[SV_X], ctx->sv[SV_CHI1], ctx->fderiv,
                        ctx->stream));
  if (cg_iterations) *cg_iterations = it;
  return su2b_adj_download(ctx, ctx->fderiv, deriv_host);
}

extern "C" int su2b_fermion_action(su2b_ctx *ctx, double mass, const double *phi_host,
                                   double tol, int max_iter, const double *x0_host, long seed,
                                   double *out) {
  if (!ctx) return SU2B_ERR_INVALID;
  ctx->begin_call();
  SU2B_CK(cudaSetDevice(ctx->device));
  SU2B_NEED(out, "out is NULL");
  long it = 0;
  SU2B_CKS(fermion_common(ctx, mass, phi_host, tol, max_iter, x0_host, seed, &it));
  const int n = (int)ctx->V;
  SU2B_LAUNCH(SU2B_K_OTHER, dot64(n, ctx->sv[SV_PHI], ctx->sv[SV_X], ctx->part_slot(4), ctx->stream));
  SU2B_LAUNCH(SU2B_K_OTHER, reduce_final(ctx->part_slot(4), vec_blocks(n), 2, ctx->red + 30, ctx->stream));
  SU2B_CKS(su2b_fetch_red(ctx, 32));
  *out = ctx->h_red[30];
  return SU2B_OK;
}

// staggered::C_pion (propagator.hpp:25-65).  The reference solves (D D^+) R = delta_0 with
// DDdag_matrix_lat::inv -- always CG (its BiCGStab branch only declares a type,
// staggered.hpp:258-263), started from gaussian_spinor(0, 10, seed) -- once for every site
// with x0 >= 1, each time with the same source and start, then takes S = D^+ R at that site.
// One solve gives the same R; S = D^+ R over the whole lattice; C[t] sums |S|^2 over the
// time slice and divides by the spatial volume; C[0] stays 0 (the contact term is skipped).
extern "C" int su2b_pion_correlator(su2b_ctx *ctx, double mass, double tol, int max_iter,
                                    long seed, double *C_host, long *cg_iterations) {
  if (!ctx) return SU2B_ERR_INVALID;
  ctx->begin_call();
  SU2B_CK(cudaSetDevice(ctx->device));
  SU2B_NEED(C_host, "C_host is NULL");
  SU2B_NEED(max_iter > 0, "max_iter must be positive");
  SU2B_CKS(su2b_fermion_setup(ctx, false));
  cudaStream_t s = ctx->stream;
  double2 *b = ctx->sv[SV_B];
  SU2B_CK(cudaMemsetAsync(b, 0, ctx->V * sizeof(double2), s));
  const double2 one = make_double2(1.0, 0.0);  // the origin is even: eo index 0
  SU2B_CK(cudaMemcpyAsync(b, &one, sizeof(double2), cudaMemcpyHostToDevice, s));
  SU2B_CKS(set_start(ctx, SU2B_CG_START_REFERENCE, seed));
  su2b_solve_stats st{};
  const int rc = cg64(ctx, mass, tol, max_iter, &st);
  if (cg_iterations) *cg_iterations = st.iterations;
  if (rc != SU2B_OK) return rc;
  SU2B_LAUNCH(SU2B_K_STAGGERED, hop64(ctx->g, ctx->ph, mass, 1, ctx->sv[SV_X], ctx->sv[SV_T], nullptr, nullptr, nullptr, nullptr, 0, s));
  double *C = ctx->part_slot(4);
  SU2B_LAUNCH(SU2B_K_OTHER, pion_slices(ctx->g, ctx->sv[SV_T], C, s));
  SU2B_CK(cudaMemcpyAsync(C_host, C, sizeof(double) * ctx->g.L[0], cudaMemcpyDeviceToHost, s));
  SU2B_CK(cudaStreamSynchronize(s));
  return SU2B_OK;
}
