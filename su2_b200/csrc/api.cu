// api.cu -- the C ABI of libsu2b (include/su2b.h): contexts, transfers, reductions, the
// HMC trajectory driver, Metropolis sweeps, Wilson flow and the staggered solvers.
//
// Host code only orders kernels on the context's stream; every lattice-sized loop runs on
// the device.  Reductions are two-stage (per-block partials, then one block in a fixed
// order), so results do not depend on timing.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <utility>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "su2b.h"
#include "su2b_ctx.h"

using namespace su2b;

// ------------------------------------------------------------------------------------
// error helpers
int su2b_fail(su2b_ctx *ctx, int code, const char *fmt, ...) {
  if (ctx) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    ctx->err = buf;
  }
  return code;
}

#define CK(call)                                                                           \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess)                                                                 \
      return su2b_fail(ctx, SU2B_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call,     \
                       cudaGetErrorString(e_));                                            \
  } while (0)
#define CKS(expr)                                                                          \
  do {                                                                                     \
    int s_ = (expr);                                                                       \
    if (s_ != SU2B_OK) return s_;                                                          \
  } while (0)
#define NEED(cond, ...)                                                                    \
  do {                                                                                     \
    if (!(cond)) return su2b_fail(ctx, SU2B_ERR_INVALID, __VA_ARGS__);                     \
  } while (0)

static int enter(su2b_ctx *ctx) {
  if (!ctx) return SU2B_ERR_INVALID;
  ctx->begin_call();
  CK(cudaSetDevice(ctx->device));
  return SU2B_OK;
}

// ------------------------------------------------------------------------------------
// context
template <class P> static int dalloc(su2b_ctx *ctx, P **p, size_t bytes) {
  if (bytes == 0) bytes = 16;
  cudaError_t e = cudaMalloc((void **)p, bytes);
  if (e != cudaSuccess) {
    *p = nullptr;
    return su2b_fail(ctx, SU2B_ERR_NOMEM, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
  }
  ctx->allocs.push_back((void *)*p);
  return SU2B_OK;
}

int su2b_make_geom(int Lx, int Ly, int Lz, int Lt, int nd, Geom *g, std::string *why) {
  if (nd < 2 || nd > 4) {
    *why = "ndims must be 2, 3 or 4";
    return 0;
  }
  const int L[4] = {Lt, Lx, Ly, Lz};
  for (int k = 0; k < 4; k++) {
    if (k < nd) {
      if (L[k] < 2 || (L[k] & 1)) {
        *why = "active extents must be even and >= 2 (even/odd layout)";
        return 0;
      }
    } else if (L[k] != 1) {
      *why = "extents of inactive directions must be 1 (parse_input_file.cc:57-67)";
      return 0;
    }
  }
  // the volume formed one extent at a time against the limit, so no product can wrap
  long V = 1;
  for (int k = 0; k < 4; k++) {
    if (L[k] > (1l << 29) || (V *= L[k]) > (1l << 29)) {
      *why = "volume above 2^29 sites";
      return 0;
    }
  }
  g->nd = nd;
  for (int k = 0; k < 4; k++) g->L[k] = L[k];
  g->st[3] = 1;
  for (int k = 2; k >= 0; k--) g->st[k] = g->st[k + 1] * L[k + 1];
  g->V = (int)V;
  g->Vh = (int)(V / 2);
  for (int k = 0; k < 4; k++) g->dv[k] = make_fastdiv((uint32_t)L[k]);
  g->cb0 = 0;
  g->ncb = g->Vh;
  g->lex0 = 0;
  return 1;
}

extern "C" int su2b_ctx_create(int group, int Lx, int Ly, int Lz, int Lt, int ndims,
                               double beta, double xi, int precision, int device,
                               su2b_ctx **out) {
  if (!out) return SU2B_ERR_INVALID;
  *out = nullptr;
  if (group != SU2B_GROUP_SU2 && group != SU2B_GROUP_U1) return SU2B_ERR_INVALID;
  if (precision != SU2B_PREC_FP64 && precision != SU2B_PREC_MIXED) return SU2B_ERR_INVALID;
  if (!(xi > 0.0)) return SU2B_ERR_INVALID;
  Geom g;
  std::string why;
  if (!su2b_make_geom(Lx, Ly, Lz, Lt, ndims, &g, &why)) return SU2B_ERR_INVALID;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return SU2B_ERR_CUDA;
  if (device < 0 || device >= ndev) return SU2B_ERR_INVALID;
  su2b_ctx *ctx = new su2b_ctx();
  ctx->group = group;
  ctx->prec = precision;
  ctx->device = device;
  ctx->Lx = Lx;
  ctx->Ly = Ly;
  ctx->Lz = Lz;
  ctx->Lt = Lt;
  ctx->beta = beta;
  ctx->xi = xi;
  ctx->g = g;
  ctx->V = (size_t)g.V;
  ctx->NL = (size_t)g.V * ndims;
  ctx->link64 = !(group == SU2B_GROUP_SU2 && precision == SU2B_PREC_MIXED);
  ctx->tune_force = ctx->link64 ? 2 : 3;  // launch shape before any tuning: (128,4) / (128,6)
  int st = SU2B_OK;
  auto fin = [&](int s) -> int {
    if (s != SU2B_OK) {
      su2b_ctx_destroy(ctx);
      return s;
    }
    *out = ctx;
    return SU2B_OK;
  };
  if (cudaSetDevice(device) != cudaSuccess) return fin(SU2B_ERR_CUDA);
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess)
    return fin(SU2B_ERR_CUDA);
  const size_t NL = ctx->NL;
  const size_t lb = ctx->link_bytes();
  const size_t ab = ctx->adj_bytes();
  ctx->part_cap = (size_t)2 * ndims * ((g.Vh + 63) / 64) + 2048;
  if ((st = dalloc(ctx, &ctx->U, lb * NL)) || (st = dalloc(ctx, &ctx->U_old, lb * NL)) ||
      (st = dalloc(ctx, &ctx->U2, lb * NL)) ||
      (st = dalloc(ctx, &ctx->tparams, sizeof(TrajParams))) ||
      (st = dalloc(ctx, &ctx->P, ab * NL)) || (st = dalloc(ctx, &ctx->Z, ab * NL)) ||
      (st = dalloc(ctx, &ctx->stage, sizeof(double) * NL * (group == 0 ? 4 : 1))) ||
      (st = dalloc(ctx, &ctx->part, sizeof(double) * 3 * ctx->part_cap * NSLOT)) ||
      (st = dalloc(ctx, &ctx->red, sizeof(double) * 64)) ||
      (st = dalloc(ctx, &ctx->traj, sizeof(TrajDev))) ||
      (st = dalloc(ctx, &ctx->counts, sizeof(unsigned long long) * 4)))
    return fin(st);
  if (cudaMallocHost((void **)&ctx->h_red, sizeof(double) * 64) != cudaSuccess ||
      cudaMallocHost((void **)&ctx->h_traj, sizeof(TrajDev)) != cudaSuccess ||
      cudaMallocHost((void **)&ctx->h_counts, sizeof(unsigned long long) * 4) != cudaSuccess ||
      cudaMallocHost((void **)&ctx->h_st, sizeof(SolverState)) != cudaSuccess ||
      cudaMallocHost((void **)&ctx->h_tparams, sizeof(TrajParams)) != cudaSuccess)
    return fin(SU2B_ERR_NOMEM);
  if (cudaMemsetAsync(ctx->U, 0, lb * NL, ctx->stream) != cudaSuccess) return fin(SU2B_ERR_CUDA);
  if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return fin(SU2B_ERR_CUDA);
  return fin(SU2B_OK);
}

extern "C" int su2b_ctx_destroy(su2b_ctx *ctx) {
  if (!ctx) return SU2B_ERR_INVALID;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (auto &p : ctx->pend) {
    cudaEventDestroy(p.a);
    cudaEventDestroy(p.b);
  }
  for (cudaEvent_t e : ctx->ev_pool) cudaEventDestroy(e);
  for (auto &kv : ctx->graphs) cudaGraphExecDestroy(kv.second.exec);
  for (void *p : ctx->allocs) cudaFree(p);
  if (ctx->arena) cudaFree(ctx->arena);
  if (ctx->h_red) cudaFreeHost(ctx->h_red);
  if (ctx->h_traj) cudaFreeHost(ctx->h_traj);
  if (ctx->h_counts) cudaFreeHost(ctx->h_counts);
  if (ctx->h_st) cudaFreeHost(ctx->h_st);
  if (ctx->h_tparams) cudaFreeHost(ctx->h_tparams);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return SU2B_OK;
}

extern "C" const char *su2b_last_error(const su2b_ctx *ctx) {
  return ctx ? ctx->err.c_str() : "null context";
}
extern "C" int su2b_ctx_stream(su2b_ctx *ctx, void **stream) {
  if (!ctx) return SU2B_ERR_INVALID;
  if (!stream) return su2b_fail(ctx, SU2B_ERR_INVALID, "stream is NULL");
  *stream = (void *)ctx->stream;
  return SU2B_OK;
}
extern "C" int su2b_set_beta(su2b_ctx *ctx, double beta) {
  if (!ctx) return SU2B_ERR_INVALID;
  ctx->beta = beta;
  return SU2B_OK;
}
extern "C" int su2b_synchronize(su2b_ctx *ctx) {
  CKS(enter(ctx));
  CK(cudaStreamSynchronize(ctx->stream));
  return SU2B_OK;
}

// ------------------------------------------------------------------------------------
// device timers
cudaEvent_t su2b_ev_take(su2b_ctx *ctx) {
  if (ctx->ev_pool.empty()) {
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
  }
  cudaEvent_t e = ctx->ev_pool.back();
  ctx->ev_pool.pop_back();
  return e;
}
void su2b_ev_mark(su2b_ctx *ctx, int kclass, cudaEvent_t start) {
  cudaEvent_t b = su2b_ev_take(ctx);
  cudaEventRecord(b, ctx->stream);
  ctx->pend.push_back({kclass, start, b});
}
// resolve the recorded event pairs (synchronises the stream)
int su2b_prof_fold(su2b_ctx *ctx) {
  if (ctx->pend.empty()) return SU2B_OK;
  CK(cudaStreamSynchronize(ctx->stream));
  for (auto &p : ctx->pend) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
      ctx->prof_ms[p.k] += ms;
      ctx->prof_n[p.k]++;
    }
    ctx->ev_pool.push_back(p.a);
    ctx->ev_pool.push_back(p.b);
  }
  ctx->pend.clear();
  return SU2B_OK;
}
extern "C" int su2b_profile(su2b_ctx *ctx, int enable) {
  CKS(enter(ctx));
  CKS(su2b_prof_fold(ctx));
  ctx->prof = enable != 0;
  for (int k = 0; k < 16; k++) {
    ctx->prof_ms[k] = 0.;
    ctx->prof_n[k] = 0;
  }
  return SU2B_OK;
}
extern "C" int su2b_profile_read(su2b_ctx *ctx, int kclass, long *launches, double *total_ms) {
  CKS(enter(ctx));
  NEED(kclass >= 0 && kclass < SU2B_K_COUNT, "kernel class %d", kclass);
  CKS(su2b_prof_fold(ctx));
  if (launches) *launches = ctx->prof_n[kclass];
  if (total_ms) *total_ms = ctx->prof_ms[kclass];
  return SU2B_OK;
}
extern "C" int su2b_kernel_launches(su2b_ctx *ctx, long *count) {
  if (!ctx) return SU2B_ERR_INVALID;
  if (!count) return su2b_fail(ctx, SU2B_ERR_INVALID, "count is NULL");
  *count = ctx->launches;
  return SU2B_OK;
}

// ------------------------------------------------------------------------------------
// transfers
extern "C" int su2b_upload_gauge(su2b_ctx *ctx, const double *U_host) {
  CKS(enter(ctx));
  NEED(U_host, "U_host is NULL");
  const size_t n = ctx->NL * (ctx->group == 0 ? 4 : 1);
  CK(cudaMemcpyAsync(ctx->stage, U_host, n * sizeof(double), cudaMemcpyHostToDevice,
                     ctx->stream));
  if (ctx->link64)
    SU2B_LAUNCH(SU2B_K_OTHER, links_from_host<double>(ctx->g, ctx->stage, ctx->U, ctx->group, ctx->stream));
  else
    SU2B_LAUNCH(SU2B_K_OTHER, links_from_host<float>(ctx->g, ctx->stage, ctx->U, ctx->group, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->phases_valid = false;
  return SU2B_OK;
}

int su2b_links_to_stage(su2b_ctx *ctx, const void *U) {
  if (ctx->link64)
    SU2B_LAUNCH(SU2B_K_OTHER, links_to_host<double>(ctx->g, U, ctx->stage, ctx->group, ctx->stream));
  else
    SU2B_LAUNCH(SU2B_K_OTHER, links_to_host<float>(ctx->g, U, ctx->stage, ctx->group, ctx->stream));
  return SU2B_OK;
}

extern "C" int su2b_download_gauge(su2b_ctx *ctx, double *U_host) {
  CKS(enter(ctx));
  NEED(U_host, "U_host is NULL");
  const size_t n = ctx->NL * (ctx->group == 0 ? 4 : 1);
  CKS(su2b_links_to_stage(ctx, ctx->U));
  CK(cudaMemcpyAsync(U_host, ctx->stage, n * sizeof(double), cudaMemcpyDeviceToHost,
                     ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return SU2B_OK;
}

// adjoint field host <-> device (P or Z buffers, precision of the context)
int su2b_adj_upload(su2b_ctx *ctx, const double *host, void *dev) {
  const size_t n = ctx->NL * (ctx->group == 0 ? 3 : 1);
  CK(cudaMemcpyAsync(ctx->stage, host, n * sizeof(double), cudaMemcpyHostToDevice,
                     ctx->stream));
  if (ctx->link64)
    SU2B_LAUNCH(SU2B_K_OTHER, adj_from_host<double>(ctx->g, ctx->stage, (double *)dev, ctx->group, ctx->stream));
  else
    SU2B_LAUNCH(SU2B_K_OTHER, adj_from_host<float>(ctx->g, ctx->stage, (float *)dev, ctx->group, ctx->stream));
  return SU2B_OK;
}
int su2b_adj_download(su2b_ctx *ctx, const void *dev, double *host) {
  const size_t n = ctx->NL * (ctx->group == 0 ? 3 : 1);
  if (ctx->link64)
    SU2B_LAUNCH(SU2B_K_OTHER, adj_to_host<double>(ctx->g, (const double *)dev, ctx->stage, ctx->group, ctx->stream));
  else
    SU2B_LAUNCH(SU2B_K_OTHER, adj_to_host<float>(ctx->g, (const float *)dev, ctx->stage, ctx->group, ctx->stream));
  CK(cudaMemcpyAsync(host, ctx->stage, n * sizeof(double), cudaMemcpyDeviceToHost,
                     ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return SU2B_OK;
}

// ------------------------------------------------------------------------------------
// reductions (queued; results land in ctx->red[slot..])
int su2b_q_plaq(su2b_ctx *ctx, const void *U, int red_slot) {
  int nb = 0;
  double *part = ctx->part_slot(0);
  if (ctx->link64)
    SU2B_LAUNCH(SU2B_K_PLAQUETTE, plaq_partials<double>(ctx->g, U, ctx->group, ctx->xi, part, &nb, ctx->stream));
  else
    SU2B_LAUNCH(SU2B_K_PLAQUETTE, plaq_partials<float>(ctx->g, U, ctx->group, ctx->xi, part, &nb, ctx->stream));
  SU2B_LAUNCH(SU2B_K_OTHER, reduce_final(part, nb, 3, ctx->red + red_slot, ctx->stream));
  return SU2B_OK;
}
int su2b_q_clover(su2b_ctx *ctx, const void *U, int cloverdef, int red_slot) {
  int nb = 0;
  double *part = ctx->part_slot(2);
  if (ctx->link64)
    SU2B_LAUNCH(SU2B_K_CLOVER, clover_partials<double>(ctx->g, U, ctx->group, cloverdef, part, &nb, ctx->stream));
  else
    SU2B_LAUNCH(SU2B_K_CLOVER, clover_partials<float>(ctx->g, U, ctx->group, cloverdef, part, &nb, ctx->stream));
  SU2B_LAUNCH(SU2B_K_OTHER, reduce_final(part, nb, 3, ctx->red + red_slot, ctx->stream));
  return SU2B_OK;
}
int su2b_fetch_red(su2b_ctx *ctx, int n) {
  CK(cudaMemcpyAsync(ctx->h_red, ctx->red, n * sizeof(double), cudaMemcpyDeviceToHost,
                     ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return SU2B_OK;
}

extern "C" int su2b_gauge_energy(su2b_ctx *ctx, int spatial_only, double *out) {
  CKS(enter(ctx));
  NEED(out, "out is NULL");
  CKS(su2b_q_plaq(ctx, ctx->U, 0));
  CKS(su2b_fetch_red(ctx, 3));
  *out = ctx->h_red[spatial_only ? 1 : 0];
  return SU2B_OK;
}
extern "C" int su2b_retr_sum_plaquettes(su2b_ctx *ctx, int spatial_only, double *out) {
  CKS(enter(ctx));
  NEED(out, "out is NULL");
  if (ctx->xi == 1.0) return su2b_gauge_energy(ctx, spatial_only, out);
  NEED(!spatial_only, "anisotropic spatial-only plaquette sums are not provided");
  CKS(su2b_q_plaq(ctx, ctx->U, 0));
  CKS(su2b_fetch_red(ctx, 3));
  *out = ctx->h_red[2];
  return SU2B_OK;
}
extern "C" int su2b_gauge_action(su2b_ctx *ctx, double *out) {
  CKS(enter(ctx));
  NEED(out, "out is NULL");
  CKS(su2b_q_plaq(ctx, ctx->U, 0));
  CKS(su2b_fetch_red(ctx, 3));
  *out = -ctx->beta * ctx->h_red[2] / ctx->Nc();
  return SU2B_OK;
}

// E, Q from clover partial sums (flat-energy_density.hh:152-163)
void su2b_finish_clover(const double *r, double V, int cloverdef, int ss, double *E,
                        double *Q) {
  double e = -(ss ? r[1] : r[0]) / V;
  if (cloverdef) e /= 16.;
  double q = ss ? 0.0 : r[2];
  q = -4. * q / (32.0 * M_PI * M_PI);
  if (cloverdef) q /= 16.;
  *E = e;
  *Q = q;
}

extern "C" int su2b_energy_density(su2b_ctx *ctx, int cloverdef, int ss, double *E,
                                   double *Q) {
  CKS(enter(ctx));
  NEED(E && Q, "E or Q is NULL");
  CKS(su2b_q_clover(ctx, ctx->U, cloverdef, 0));
  CKS(su2b_fetch_red(ctx, 3));
  su2b_finish_clover(ctx->h_red, (double)ctx->V, cloverdef, ss, E, Q);
  return SU2B_OK;
}

// ------------------------------------------------------------------------------------
// force and updates
template <class T>
static int q_force(su2b_ctx *ctx, const void *U, T *P, const T *extra, double f, double scale,
                   int mode, double *kin_part, int *nb, void *Uout, double dt_upd) {
  SU2B_LAUNCH(SU2B_K_FORCE, force_update<T>(ctx->g, U, ctx->group, P, extra, f, scale, ctx->xi,
                                            mode, kin_part, nb, Uout, dt_upd, ctx->stream,
                                            ctx->tune_force));
  return SU2B_OK;
}
int su2b_q_force(su2b_ctx *ctx, const void *U, void *P, const void *extra, double f,
                 double scale, int mode, double *kin_part, int *nb, void *Uout, double dt_upd) {
  if (ctx->link64)
    return q_force<double>(ctx, U, (double *)P, (const double *)extra, f, scale, mode,
                           kin_part, nb, Uout, dt_upd);
  return q_force<float>(ctx, U, (float *)P, (const float *)extra, f, scale, mode, kin_part, nb,
                        Uout, dt_upd);
}
int su2b_q_update(su2b_ctx *ctx, void *U, const void *P, double dt, double round_dn) {
  if (ctx->link64)
    SU2B_LAUNCH(SU2B_K_UPDATE, link_update<double>(ctx->g, U, ctx->group, (const double *)P, dt,
                                                   ctx->stream, round_dn));
  else
    SU2B_LAUNCH(SU2B_K_UPDATE, link_update<float>(ctx->g, U, ctx->group, (const float *)P, dt,
                                                  ctx->stream, round_dn));
  ctx->phases_valid = false;
  return SU2B_OK;
}
int su2b_q_restore(su2b_ctx *ctx, void *U) {
  if (ctx->link64)
    SU2B_LAUNCH(SU2B_K_RESTORE, restore_links<double>(ctx->g, U, ctx->group, ctx->stream));
  else
    SU2B_LAUNCH(SU2B_K_RESTORE, restore_links<float>(ctx->g, U, ctx->group, ctx->stream));
  return SU2B_OK;
}

extern "C" int su2b_gauge_force(su2b_ctx *ctx, double fac, double *deriv_host) {
  CKS(enter(ctx));
  NEED(deriv_host, "deriv_host is NULL");
  const double f = fac * ctx->beta / ctx->Nc();
  CKS(su2b_q_force(ctx, ctx->U, ctx->Z, nullptr, f, 1.0, 0, nullptr, nullptr));
  return su2b_adj_download(ctx, ctx->Z, deriv_host);
}
extern "C" int su2b_restore_su(su2b_ctx *ctx) {
  CKS(enter(ctx));
  CKS(su2b_q_restore(ctx, ctx->U));
  CK(cudaStreamSynchronize(ctx->stream));
  return SU2B_OK;
}
extern "C" int su2b_update_gauge(su2b_ctx *ctx, const double *P_host, double dtau) {
  CKS(enter(ctx));
  NEED(P_host, "P_host is NULL");
  CKS(su2b_adj_upload(ctx, P_host, ctx->P));
  CKS(su2b_q_update(ctx, ctx->U, ctx->P, dtau));
  CK(cudaStreamSynchronize(ctx->stream));
  return SU2B_OK;
}

// ------------------------------------------------------------------------------------
// Metropolis
extern "C" int su2b_metropolis_sweep(su2b_ctx *ctx, double delta, int N_hit, uint64_t seed,
                                     uint32_t sweep, double *rates) {
  CKS(enter(ctx));
  NEED(rates, "rates is NULL");
  NEED(N_hit >= 0, "N_hit < 0");
  CK(cudaMemsetAsync(ctx->counts, 0, 2 * sizeof(unsigned long long), ctx->stream));
  for (int mu = 0; mu < ctx->g.nd; mu++)
    for (int p = 0; p < 2; p++) {
      if (ctx->link64)
        SU2B_LAUNCH(SU2B_K_METROPOLIS, metropolis_pass<double>(ctx->g, ctx->U, ctx->group, mu, p, ctx->beta, ctx->xi, delta, N_hit,
                                   seed, sweep, ctx->counts, ctx->stream));
      else
        SU2B_LAUNCH(SU2B_K_METROPOLIS, metropolis_pass<float>(ctx->g, ctx->U, ctx->group, mu, p, ctx->beta, ctx->xi, delta, N_hit,
                                  seed, sweep, ctx->counts, ctx->stream));
    }
  CK(cudaMemcpyAsync(ctx->h_counts, ctx->counts, 2 * sizeof(unsigned long long),
                     cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->phases_valid = false;
  if (ctx->pend.size() > 4096) CKS(su2b_prof_fold(ctx));
  const double nh = (double)(N_hit > 0 ? N_hit : 1);
  rates[0] = (double)ctx->h_counts[0] / nh / (double)ctx->NL;
  rates[1] = (double)ctx->h_counts[1] / nh / (double)ctx->V;
  return SU2B_OK;
}

// ------------------------------------------------------------------------------------
// Wilson flow: runge_kutta (flat-gradient_flow.hh:17-50)
int su2b_q_flow_step_to(su2b_ctx *ctx, void *src, void *dst, double eps) {
  const double zfac[3] = {(-17.0) / (36.0), (8.0) / (9.0), (-3.0) / (4.0)};
  const double expfac[3] = {-36.0 / 4. / 17.0, 1., -1.};
  const int Nc = ctx->group == 0 ? 2 : 1;
  // SU(2): a stage's link update W' = exp(c Z) W is written by the force kernel itself into
  // the other link buffer, as the fused trajectory steps do, so W is read once per stage
  // instead of twice.  src != dst: all three stages fused, src -> dst -> src -> dst (src is
  // left holding W2).  In place: src -> U2 -> src fused, then the third stage's force and
  // update in place (U2 holds no field between calls: it is the trajectory's spare).  The
  // update arithmetic is the separate update kernel's, so the flowed field is the same bit
  // for bit either way.
  const bool su2 = ctx->group == SU2B_GROUP_SU2;
  if (!su2 && src != dst) {  // U(1): the steps run in place, on a copy in dst
    CK(cudaMemcpyAsync(dst, src, ctx->link_bytes() * ctx->NL, cudaMemcpyDeviceToDevice,
                       ctx->stream));
    src = dst;
  }
  const bool in_place = src == dst;
  void *other = in_place ? ctx->U2 : dst;
  const int nfused = !su2 || (in_place && src == ctx->U2) ? 0 : (in_place ? 2 : 3);
  void *W = src;
  for (int f = 0; f < 3; f++) {
    const double fac = 2. * Nc * zfac[f] / ctx->beta;
    const double ff = fac * ctx->beta / (double)Nc;
    const int mode = f == 0 ? 0 : FM_HAS_IN;
    if (f < nfused) {
      void *next = W == src ? other : src;
      CKS(su2b_q_force(ctx, W, ctx->Z, nullptr, ff, 1.0, mode | FM_UPDATE, nullptr, nullptr,
                       next, -eps * expfac[f]));
      W = next;
      ctx->phases_valid = false;
    } else {
      CKS(su2b_q_force(ctx, W, ctx->Z, nullptr, ff, 1.0, mode, nullptr, nullptr));
      CKS(su2b_q_update(ctx, W, ctx->Z, -eps * expfac[f]));
    }
  }
  // FP32 links: every exp(.)U product rounds |U| by about one ulp in a direction that does not
  // average out over hundreds of steps, and the flowed plaquette (close to 1) amplifies that
  // drift in E = d(d-1)/2 - P/(V Nc).  Reunitarise in FP64 after each step, as the trajectory
  // does at its end; FP64 links keep the reference's step unchanged.
  if (!ctx->link64 && su2) CKS(su2b_q_restore(ctx, W));
  return SU2B_OK;
}
int su2b_q_flow_step(su2b_ctx *ctx, void *U, double eps) {
  return su2b_q_flow_step_to(ctx, U, U, eps);
}

extern "C" int su2b_flow_step(su2b_ctx *ctx, double eps) {
  CKS(enter(ctx));
  if (ctx->group == SU2B_GROUP_SU2) {
    // all three stages fused, U -> U2 -> U -> U2; the spare buffer becomes the current field
    // (as a trajectory's accept rotates its buffers) and the old one the spare
    CKS(su2b_q_flow_step_to(ctx, ctx->U, ctx->U2, eps));
    std::swap(ctx->U, ctx->U2);
  } else {
    CKS(su2b_q_flow_step(ctx, ctx->U, eps));
  }
  CK(cudaStreamSynchronize(ctx->stream));
  return SU2B_OK;
}

int su2b_ensure_aux(su2b_ctx *ctx) {
  if (ctx->U_aux) return SU2B_OK;
  return dalloc(ctx, &ctx->U_aux, ctx->link_bytes() * ctx->NL);
}

extern "C" int su2b_gradient_flow(su2b_ctx *ctx, double tmax, double eps, double tstart,
                                  double *rows, int max_rows, int *n_rows) {
  CKS(enter(ctx));
  NEED(n_rows, "n_rows is NULL");
  NEED(eps > 0, "eps must be positive");
  NEED(max_rows >= 0 && (rows || max_rows == 0), "rows buffer");
  CKS(su2b_ensure_aux(ctx));
  void *Vt = ctx->U_aux;
  CK(cudaMemcpyAsync(Vt, ctx->U, ctx->link_bytes() * ctx->NL, cudaMemcpyDeviceToDevice,
                     ctx->stream));
  const size_t d = (size_t)ctx->g.nd;
  const double ndims_fact = (double)(d * (d - 1)) / 2.0;
  const double ndims_fact_ss = (double)((d - 1) * (d - 2)) / 2.0;
  const double den = (double)ctx->V * ctx->Nc();
  double t[3] = {tstart, tstart, tstart};
  int nr = 0;
  while (t[1] < tmax - eps) {
    t[0] = t[2];
    t[1] = t[0] + eps;
    // two steps per record, Vt -> U2 -> Vt, every stage fused with its link update
    CKS(su2b_q_flow_step_to(ctx, Vt, ctx->U2, eps));
    // the reference prints the observables of the middle step only
    CKS(su2b_q_plaq(ctx, ctx->U2, 0));
    CKS(su2b_q_clover(ctx, ctx->U2, 1, 3));
    t[2] = t[1] + eps;
    CKS(su2b_q_flow_step_to(ctx, ctx->U2, Vt, eps));
    CKS(su2b_fetch_red(ctx, 6));
    const double *r = ctx->h_red;
    const double P1 = r[0] / den, Pss1 = r[1] / den;
    double E1, Q1, Ess1, Qss1;
    su2b_finish_clover(r + 3, (double)ctx->V, 1, 0, &E1, &Q1);
    su2b_finish_clover(r + 3, (double)ctx->V, 1, 1, &Ess1, &Qss1);
    const double Ep = ndims_fact - P1;
    const double Ep_ss = ndims_fact_ss - Pss1;
    const double Ep_ts = Ep - Ep_ss;
    const double Ep_ts_bar = Ep_ts / (double)(d - 1);
    const double Ep_ss_bar = Ep_ss / ndims_fact_ss;
    const double xi_R = sqrt(Ep_ts_bar / Ep_ss_bar);
    if (nr < max_rows) {
      double *o = rows + 9 * (size_t)nr;
      o[0] = t[1];
      o[1] = xi_R;
      o[2] = P1;
      o[3] = Pss1;
      o[4] = Ep;
      o[5] = Ep_ss;
      o[6] = E1;
      o[7] = Ess1;
      o[8] = Q1;
    }
    nr++;
  }
  CK(cudaStreamSynchronize(ctx->stream));
  *n_rows = nr;
  return SU2B_OK;
}
