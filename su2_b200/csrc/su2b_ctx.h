// su2b_ctx.h -- the context object behind the opaque su2b_ctx handle (host side only).
#pragma once
#include <map>
#include <string>
#include <vector>

#include "solver.h"
#include "su2b_internal.h"

constexpr int NSLOT = 6;  // partial-sum slots: 0 plaquette, 1 kinetic, 2 clover, 3-5 solvers

// device spinor buffers (U(1) staggered fermions)
enum { SV_B, SV_X, SV_R, SV_P, SV_T, SV_AP, SV_S, SV_R0, SV_PHI, SV_CHI, SV_CHI1, SV_X0, SV_P2, SV_AP2, SV_N };
enum { SV32_XS, SV32_RS, SV32_PS, SV32_TS, SV32_APS, SV32_N };

struct su2b_ctx {
  int group = 0, prec = 0, device = 0;
  int Lx = 0, Ly = 0, Lz = 0, Lt = 0;
  double beta = 0., xi = 1.;
  su2b::Geom g{};
  size_t V = 0, NL = 0;
  bool link64 = true;  // links/momenta in FP64 (false: SU(2) mixed precision, FP32)
  cudaStream_t stream = nullptr;

  // gauge field, backups, momenta, flow/force accumulator
  // U is the current field; U_old and U2 are the other two link buffers of the fused
  // trajectory (the start configuration stays untouched in one of them until accept/reject)
  void *U = nullptr, *U_old = nullptr, *U2 = nullptr, *U_aux = nullptr, *U_rev = nullptr;
  void *P = nullptr, *Z = nullptr;
  // scratch arena of the flow adjoint, kept between calls and grown on demand
  void *arena = nullptr;
  size_t arena_bytes = 0;
  double *stage = nullptr;  // host-layout staging buffer on the device
  double *part = nullptr;   // NSLOT slots of 3*part_cap partial sums
  size_t part_cap = 0;
  double *red = nullptr;    // 64 reduced scalars
  su2b::TrajDev *traj = nullptr;
  su2b::TrajParams *tparams = nullptr, *h_tparams = nullptr;
  unsigned long long *counts = nullptr;

  // pinned host mirrors
  double *h_red = nullptr;
  su2b::TrajDev *h_traj = nullptr;
  unsigned long long *h_counts = nullptr;
  su2b::SolverState *h_st = nullptr;

  // staggered fermions
  double2 *ph = nullptr;
  float2 *ph32 = nullptr;
  bool phases_valid = false, phases32_valid = false;
  double2 *sv[SV_N] = {};
  float2 *sv32[SV32_N] = {};
  double *fderiv = nullptr;
  su2b::SolverState *st = nullptr;
  long x0_seed = -1;  // seed of the reference CG start held in sv[SV_X0]

  // set at the end of a fused trajectory: red[] then holds the plaquette sums of both the
  // trajectory's start field and its final field, so the next fused trajectory takes its
  // start plaquettes from there instead of summing them again.  Every entry point clears it
  // on entry (begin_call), so any call between trajectories forces a fresh sum.
  bool start_plaq_cached = false;
  void begin_call() {
    err.clear();
    start_plaq_cached = false;
  }

  // launch shape of the SU(2) force kernel (su2b_autotune)
  int tune_force = 3;  // (128 threads, 6 blocks/SM) until tuned; FP64 contexts start at 2
  int traj_path = 0;   // SU2B_TRAJ_FUSED_GRAPH or SU2B_TRAJ_PLAIN

  // kernel launch counter and the per-class device timers (su2b_profile)
  long launches = 0;
  bool prof = false;
  struct Pending {
    int k;
    cudaEvent_t a, b;
  };
  std::vector<Pending> pend;
  std::vector<cudaEvent_t> ev_pool;
  double prof_ms[16] = {};
  long prof_n[16] = {};

  struct GraphEntry {
    cudaGraphExec_t exec;
    long kernels;
  };
  std::map<std::string, GraphEntry> graphs;
  std::map<std::string, void *> graph_final;  // buffer holding the result of each graph
  std::vector<void *> allocs;
  std::string err;

  size_t link_bytes() const { return group == 0 ? (link64 ? 32 : 16) : 8; }
  size_t adj_bytes() const { return (group == 0 ? 3 : 1) * (link64 ? 8 : 4); }
  double Nc() const { return group == 0 ? 2.0 : 1.0; }
  double *part_slot(int k) { return part + (size_t)k * 3 * part_cap; }
};

// the integrator schedules (integrator.hh), shared by the single-lattice and slab drivers
struct HmcOp {
  int kind;  // 0 momenta: P -= c * deriv;  1 gauge: U = exp(c P) U
  double c;
};
struct HmcFusedOp {
  int kind;  // 0 momentum step, 1 momentum + gauge step, 2 gauge step alone
  double cm, cg;
  bool kinetic;  // the last momentum step: its launch also sums |P|^2
};
std::vector<HmcOp> su2b_schedule(int integ, int n, double tau);
std::vector<HmcFusedOp> su2b_fuse(const std::vector<HmcOp> &ops);

// helpers shared by the api*.cu files
int su2b_fail(su2b_ctx *ctx, int code, const char *fmt, ...);
int su2b_adj_upload(su2b_ctx *ctx, const double *host, void *dev);
int su2b_adj_download(su2b_ctx *ctx, const void *dev, double *host);
int su2b_q_plaq(su2b_ctx *ctx, const void *U, int red_slot);
int su2b_q_clover(su2b_ctx *ctx, const void *U, int cloverdef, int red_slot);
int su2b_fetch_red(su2b_ctx *ctx, int n);
// E and Q of energy_density (flat-energy_density.hh:57-164) from the clover sums r[0..2] of V sites
void su2b_finish_clover(const double *r, double V, int cloverdef, int ss, double *E, double *Q);
// E and Q of energy_density (flat-energy_density.hh:57-164) from the clover sums r[0..2] of V sites
void su2b_finish_clover(const double *r, double V, int cloverdef, int ss, double *E, double *Q);
// mode FM_UPDATE / FM_RESTORE: the force kernel also writes the next link buffer Uout
int su2b_q_force(su2b_ctx *ctx, const void *U, void *P, const void *extra, double f,
                 double scale, int mode, double *kin_part, int *nb, void *Uout = nullptr,
                 double dt_upd = 0.0);
int su2b_q_update(su2b_ctx *ctx, void *U, const void *P, double dt, double round_dn = 0.0);
int su2b_q_restore(su2b_ctx *ctx, void *U);
int su2b_q_flow_step(su2b_ctx *ctx, void *U, double eps);
// one flow step from src into dst (dst == src: in place); src != dst leaves src clobbered
int su2b_q_flow_step_to(su2b_ctx *ctx, void *src, void *dst, double eps);
int su2b_ensure_aux(su2b_ctx *ctx);
int su2b_links_to_stage(su2b_ctx *ctx, const void *U);
int su2b_prof_fold(su2b_ctx *ctx);
int su2b_make_geom(int Lx, int Ly, int Lz, int Lt, int nd, su2b::Geom *g, std::string *why);
// fermions (solve.cu)
int su2b_fermion_setup(su2b_ctx *ctx, bool need32);
int su2b_fermion_deriv_q(su2b_ctx *ctx, double mass, double tol, int max_iter, int cg_start,
                         long seed, long *iters);
int su2b_fermion_action_q(su2b_ctx *ctx, double mass, double tol, int max_iter, int cg_start,
                          long seed, int red_slot, long *iters);
int su2b_fermion_heatbath_q(su2b_ctx *ctx, double mass, const double *R_host, uint64_t seed,
                            uint32_t traj, int cplx, int red_slot);

cudaEvent_t su2b_ev_take(su2b_ctx *ctx);
void su2b_ev_mark(su2b_ctx *ctx, int kclass, cudaEvent_t start);
int su2b_prof_fold(su2b_ctx *ctx);

// launch a kernel through its launcher: counts it and, with profiling on, times it
#define SU2B_LAUNCH(kclass, call)                                                          \
  do {                                                                                     \
    cudaEvent_t a_ = nullptr;                                                              \
    if (ctx->prof) {                                                                       \
      a_ = su2b_ev_take(ctx);                                                              \
      cudaEventRecord(a_, ctx->stream);                                                    \
    }                                                                                      \
    SU2B_CK(call);                                                                         \
    ctx->launches++;                                                                       \
    if (ctx->prof) su2b_ev_mark(ctx, kclass, a_);                                          \
  } while (0)

#define SU2B_CK(call)                                                                      \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess)                                                                 \
      return su2b_fail(ctx, SU2B_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call,     \
                       cudaGetErrorString(e_));                                            \
  } while (0)
#define SU2B_CKS(expr)                                                                     \
  do {                                                                                     \
    int s_ = (expr);                                                                       \
    if (s_ != SU2B_OK) return s_;                                                          \
  } while (0)
#define SU2B_NEED(cond, ...)                                                               \
  do {                                                                                     \
    if (!(cond)) return su2b_fail(ctx, SU2B_ERR_INVALID, __VA_ARGS__);                     \
  } while (0)
