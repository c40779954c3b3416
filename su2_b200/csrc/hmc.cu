// hmc.cu -- the HMC trajectory on the device (md_update, md_update.hh:18-81).
//
// Sequence per trajectory, all on the context's stream:
//   momenta (Philox, or uploaded)  + sum P^2         -> H_kin old
//   [fermions: R, phi = D R, |R|^2]                  -> H_F old
//   plaquette partials                               -> S_G old
//   U_old = U
//   integrator schedule (integrator.hh): momentum steps are the fused staple/force/momentum
//     kernel (the last one also sums P^2), gauge steps the exp(dt P) U kernel
//   restoreSU, plaquettes (+ fermion action)         -> H new
//   accept/reject on the device (FP64), optional reversibility test, U = U_old on reject
//   plaquette of the resulting field; one device->host copy of the result.
#include <cmath>
#include <vector>

#include "su2b.h"
#include "su2b_ctx.h"

using namespace su2b;

// integrator.hh: the step sequence of each scheme, with the reference's coefficient
// arithmetic (dtau = tau/nsteps, omf2 lambda = 0.1938, omf4 Omelyan constants).
std::vector<HmcOp> su2b_schedule(int integ, int n, double tau) {
  using Op = HmcOp;
  std::vector<Op> o;
  const double dtau = tau / (double)n;
  auto M = [&](double c) { o.push_back({0, c}); };
  auto G = [&](double c) { o.push_back({1, c}); };
  if (integ == SU2B_OMF2) {  // integrator.hh:83-116
    const double lambda = 0.1938;
    const double om2l = (1. - 2. * lambda);
    M(lambda * dtau);
    for (int i = 0; i < n - 1; i++) {
      G(0.5 * dtau);
      M(om2l * dtau);
      G(0.5 * dtau);
      M(2 * lambda * dtau);
    }
    G(0.5 * dtau);
    M(om2l * dtau);
    G(0.5 * dtau);
    M(lambda * dtau);
  } else if (integ == SU2B_OMF4 || integ == SU2B_LP_OMF4) {
    // integrator.hh:119-156 and the same schedule of lp_omf4, :158-199 (loop from i = 1 as
    // there)
    const double rho = 0.2539785108410595, theta = -0.03230286765269967,
                 vartheta = 0.08398315262876693, lambda = 0.6822365335719091;
    const double eps[10] = {rho * dtau,
                            lambda * dtau,
                            theta * dtau,
                            0.5 * (1 - 2. * (lambda + vartheta)) * dtau,
                            (1 - 2. * (theta + rho)) * dtau,
                            0.5 * (1 - 2. * (lambda + vartheta)) * dtau,
                            theta * dtau,
                            lambda * dtau,
                            rho * dtau,
                            2 * vartheta * dtau};
    M(0.5 * eps[9]);
    for (int i = 1; i < n - 1; i++)
      for (int j = 0; j < 5; j++) {
        G(eps[2 * j]);
        M(eps[2 * j + 1]);
      }
    for (int j = 0; j < 4; j++) {
      G(eps[2 * j]);
      M(eps[2 * j + 1]);
    }
    G(eps[8]);
    M(0.5 * eps[9]);
  } else if (integ == SU2B_EULER) {  // integrator.hh:201-217
    for (int i = 0; i < n; i++) {
      M(dtau);
      G(dtau);
    }
  } else if (integ == SU2B_RUTH) {  // integrator.hh:220-241
    for (int i = 0; i < n; i++) {
      M(dtau);
      G(-1. / 24. * dtau);
      M(-2. / 3. * dtau);
      G(3. / 4. * dtau);
      M(2. / 3. * dtau);
      G(7. / 24. * dtau);
    }
  } else {  // leapfrog and lp_leapfrog (integrator.hh:26-80), the fallback (:274-277)
    M(dtau / 2.);
    G(dtau);
    for (int i = 0; i < n - 1; i++) {
      M(dtau);
      G(dtau);
    }
    M(dtau / 2.);
  }
  return o;
}

// a momentum step and the gauge step after it become one fused force launch
std::vector<HmcFusedOp> su2b_fuse(const std::vector<HmcOp> &ops) {
  int last_m = -1;
  for (int i = 0; i < (int)ops.size(); i++)
    if (ops[i].kind == 0) last_m = i;
  std::vector<HmcFusedOp> f;
  for (int i = 0; i < (int)ops.size(); i++) {
    if (ops[i].kind == 0 && i + 1 < (int)ops.size() && ops[i + 1].kind == 1) {
      f.push_back({1, ops[i].c, ops[i + 1].c, i == last_m});
      i++;
    } else if (ops[i].kind == 0) {
      f.push_back({0, ops[i].c, 0.0, i == last_m});
    } else {
      f.push_back({2, 0.0, ops[i].c, false});
    }
  }
  return f;
}

namespace {

using Op = HmcOp;
using FOp = HmcFusedOp;
std::vector<Op> schedule(int integ, int n, double tau) { return su2b_schedule(integ, n, tau); }
std::vector<FOp> fuse(const std::vector<Op> &ops) { return su2b_fuse(ops); }

int kinetic_now(su2b_ctx *ctx, int slot);

bool low_precision(int integ) { return integ == SU2B_LP_LEAPFROG || integ == SU2B_LP_OMF4; }

int integrate(su2b_ctx *ctx, const std::vector<Op> &ops, const su2b_hmc_params *prm,
              int kin_slot, long *cg_iters) {
  const bool ferm = prm->fermion_mass > 0.0;
  // lp_leapfrog / lp_omf4: dn = N = pow(10, exponent) as a size_t (integrator.hh:59, 168);
  // each momentum step rounds the summed derivative, each gauge step the links
  const bool lp = low_precision(prm->integrator);
  const double dn = lp ? (double)(size_t)std::pow(10.0, (double)prm->round_exponent) : 0.0;
  int last_m = -1;
  for (int i = 0; i < (int)ops.size(); i++)
    if (ops[i].kind == 0) last_m = i;
  const double f = ctx->beta / ctx->Nc();  // fac = 1 (update_momenta.hh:21)
  for (int i = 0; i < (int)ops.size(); i++) {
    if (ops[i].kind == 0) {
      int mode = FM_HAS_IN | (i == last_m ? FM_KINETIC : 0);
      const void *extra = nullptr;
      if (ferm) {
        long it = 0;
        SU2B_CKS(su2b_fermion_deriv_q(ctx, prm->fermion_mass, prm->cg_tol, prm->cg_max_iter,
                                      prm->cg_start, prm->pf_seed, &it));
        *cg_iters += it;
        extra = ctx->fderiv;
        mode |= FM_EXTRA;
      }
      if (lp) {  // the derivative into Z (no momentum input), then P -= c round(Z)
        SU2B_CKS(su2b_q_force(ctx, ctx->U, ctx->Z, extra, f, 1.0, mode & FM_EXTRA, nullptr,
                              nullptr));
        if (ctx->link64)
          SU2B_LAUNCH(SU2B_K_OTHER, adj_round_axpy<double>(ctx->g, (double *)ctx->P,
                                                           (const double *)ctx->Z, ctx->group,
                                                           ops[i].c, dn, ctx->stream));
        else
          SU2B_LAUNCH(SU2B_K_OTHER, adj_round_axpy<float>(ctx->g, (float *)ctx->P,
                                                          (const float *)ctx->Z, ctx->group,
                                                          ops[i].c, dn, ctx->stream));
        continue;
      }
      int nb = 0;
      SU2B_CKS(su2b_q_force(ctx, ctx->U, ctx->P, extra, f, -ops[i].c, mode, ctx->part_slot(1),
                            &nb));
      if (mode & FM_KINETIC)
        SU2B_LAUNCH(SU2B_K_OTHER, reduce_final(ctx->part_slot(1), nb, 1, ctx->red + kin_slot, ctx->stream));
    } else {
      SU2B_CKS(su2b_q_update(ctx, ctx->U, ctx->P, ops[i].c, dn));
    }
  }
  if (lp) SU2B_CKS(kinetic_now(ctx, kin_slot));
  return su2b_q_restore(ctx, ctx->U);  // integrator.hh:48
}

int kinetic_now(su2b_ctx *ctx, int slot) {
  int nb = 0;
  if (ctx->link64)
    SU2B_LAUNCH(SU2B_K_OTHER, kinetic_partials<double>(ctx->g, (const double *)ctx->P, ctx->group,
                                     ctx->part_slot(1), &nb, ctx->stream));
  else
    SU2B_LAUNCH(SU2B_K_OTHER, kinetic_partials<float>(ctx->g, (const float *)ctx->P, ctx->group,
                                    ctx->part_slot(1), &nb, ctx->stream));
  SU2B_LAUNCH(SU2B_K_OTHER, reduce_final(ctx->part_slot(1), nb, 1, ctx->red + slot, ctx->stream));
  return SU2B_OK;
}

// ------------------------------------------------------------------------------------
// fused SU(2) trajectory: a momentum step and the gauge step after it are one kernel that
// reads links from one buffer and writes the updated links to another.  The start field S
// is never written, so a rejected trajectory needs no copy; the two other buffers X, Y
// alternate.  The closing restoreSU writes the final field and sums its plaquettes.

// queues the trajectory; returns the buffer that holds the final field in *fin
// cached: the start plaquettes are those the previous trajectory left in red[] (its start
// or its end field, by its accept flag), so the start pass skips the plaquette sums
int enqueue_fused(su2b_ctx *ctx, const std::vector<FOp> &fops, bool host_momenta, bool cached,
                  void *S, void *X, void *Y, void **fin) {
  cudaStream_t s = ctx->stream;
  int nb = 0;
  // partial sums: the start pass in slot 1, the final kinetic energy in slot 2, the end
  // plaquettes in slot 0; all three are reduced by the accept launch
  int nb_start = 0, nb_kin = 0, nb_plaq = 0;
  SU2B_CK(cudaMemsetAsync(ctx->red + 8, 0, 2 * sizeof(double), s));
  if (!host_momenta) {
    // momenta, kinetic energy and the plaquettes of the start field in one pass
    if (ctx->link64)
      SU2B_LAUNCH(SU2B_K_MOMENTA, momenta_plaq<double>(ctx->g, S, (double *)ctx->P, ctx->tparams,
                                                       ctx->xi, ctx->part_slot(1), &nb_start, s,
                                                       !cached));
    else
      SU2B_LAUNCH(SU2B_K_MOMENTA, momenta_plaq<float>(ctx->g, S, (float *)ctx->P, ctx->tparams,
                                                      ctx->xi, ctx->part_slot(1), &nb_start, s,
                                                      !cached));
  } else {
    SU2B_CKS(su2b_q_plaq(ctx, S, 1));
  }
  const double f = ctx->beta / ctx->Nc();
  void *cur = S;
  auto next = [&](void *c) { return c == X ? Y : X; };
  void *F = nullptr;
  // site pairs (FP32 links, isotropic, d = 4, T % 4 == 0, a schedule of fused steps closed by
  // a momentum step): the start field copied into the paired layout in X, the force launches
  // on paired buffers, the final field written back in the standard layout
  bool paired = !ctx->link64 && ctx->tune_force == FORCE_PAIR && ctx->xi == 1.0 &&
                pairs_apply(ctx->g) && !fops.empty();
  for (size_t i = 0; paired && i < fops.size(); i++)
    if (fops[i].kind != (i + 1 == fops.size() ? 0 : 1)) paired = false;
  if (paired) {
    SU2B_LAUNCH(SU2B_K_OTHER, to_pairs(ctx->g, S, X, s));
    cur = X;
  }
  for (size_t i = 0; i < fops.size(); i++) {
    const FOp &o = fops[i];
    const bool last = i + 1 == fops.size();
    if (o.kind == 2) {  // a gauge step that no momentum step precedes
      void *out = next(cur);
      SU2B_CK(cudaMemcpyAsync(out, cur, ctx->link_bytes() * ctx->NL, cudaMemcpyDeviceToDevice,
                              s));
      SU2B_CKS(su2b_q_update(ctx, out, ctx->P, o.cg));
      cur = out;
      continue;
    }
    int mode = FM_HAS_IN | (o.kinetic ? FM_KINETIC : 0);
    void *out = nullptr;
    if (o.kind == 1) {
      mode |= FM_UPDATE;
      out = next(cur);
    } else if (last) {
      // the closing restoreSU (integrator.hh:48) written by the last momentum step
      mode |= FM_RESTORE;
      out = F = (cur == S) ? X : next(cur);
    }
    // chained force launches overlap the next one's launch with the previous one's tail
    // (programmatic dependent launch; every access waits for the previous launch)
    const bool pdl = !ctx->prof;
    if (paired)
      SU2B_LAUNCH(SU2B_K_FORCE, force_pair(ctx->g, cur, (float *)ctx->P, f, -o.cm, mode,
                                           ctx->part_slot(2), &nb, out, o.cg, s, pdl));
    else if (ctx->link64)
      SU2B_LAUNCH(SU2B_K_FORCE,
                  force_update<double>(ctx->g, cur, 0, (double *)ctx->P, nullptr, f, -o.cm,
                                       ctx->xi, mode, ctx->part_slot(2), &nb, out, o.cg, s,
                                       ctx->tune_force, pdl));
    else
      SU2B_LAUNCH(SU2B_K_FORCE,
                  force_update<float>(ctx->g, cur, 0, (float *)ctx->P, nullptr, f, -o.cm,
                                      ctx->xi, mode, ctx->part_slot(2), &nb, out, o.cg, s,
                                      ctx->tune_force, pdl));
    if (o.kinetic) nb_kin = nb;
    if (o.kind == 1) cur = out;
  }
  if (!F) {  // the schedule ended with a gauge step: restore in place in a scratch buffer
    if (cur == S) {
      SU2B_CK(cudaMemcpyAsync(X, S, ctx->link_bytes() * ctx->NL, cudaMemcpyDeviceToDevice, s));
      cur = X;
    }
    SU2B_CKS(su2b_q_restore(ctx, cur));
    F = cur;
  }
  if (ctx->link64)
    SU2B_LAUNCH(SU2B_K_PLAQUETTE, plaq_partials<double>(ctx->g, F, ctx->group, ctx->xi,
                                                        ctx->part_slot(0), &nb_plaq, s));
  else
    SU2B_LAUNCH(SU2B_K_PLAQUETTE, plaq_partials<float>(ctx->g, F, ctx->group, ctx->xi,
                                                       ctx->part_slot(0), &nb_plaq, s));
  SU2B_LAUNCH(SU2B_K_OTHER, reduce_accept(ctx->part_slot(1), nb_start, ctx->part_slot(2), nb_kin,
                                          ctx->part_slot(0), nb_plaq, ctx->red, ctx->tparams,
                                          ctx->traj, cached && !host_momenta, s));
  SU2B_CK(cudaMemcpyAsync(ctx->h_traj, ctx->traj, sizeof(TrajDev), cudaMemcpyDeviceToHost, s));
  SU2B_CK(cudaMemcpyAsync(ctx->h_red, ctx->red, 20 * sizeof(double), cudaMemcpyDeviceToHost, s));
  *fin = F;
  return SU2B_OK;
}

int traj_fused(su2b_ctx *ctx, const su2b_hmc_params *prm, bool cached, su2b_traj_result *res) {
  cudaStream_t s = ctx->stream;
  const std::vector<FOp> fops = fuse(schedule(prm->integrator, prm->n_steps, prm->tau));
  void *S = ctx->U, *X = ctx->U_old, *Y = ctx->U2, *F = nullptr;
  const bool host_momenta = prm->momenta_host != nullptr;
  if (host_momenta) {
    SU2B_CKS(su2b_adj_upload(ctx, prm->momenta_host, ctx->P));
    SU2B_CKS(kinetic_now(ctx, 0));
  }
  if (ctx->prof || host_momenta) {
    SU2B_CKS(enqueue_fused(ctx, fops, host_momenta, cached && !host_momenta, S, X, Y, &F));
  } else {
    // one CUDA graph per schedule, coupling and buffer assignment; seed, trajectory index
    // and accept uniform come from ctx->tparams, so the graph replays for every trajectory
    char key[256];
    snprintf(key, sizeof key, "%d/%d/%.17g/%.17g/%p/%p/%p/%d/%d", prm->integrator, prm->n_steps,
             prm->tau, ctx->beta, S, X, Y, ctx->tune_force, (int)cached);
    auto it = ctx->graphs.find(key);
    if (it == ctx->graphs.end()) {
      const long n0 = ctx->launches;
      cudaGraph_t graph = nullptr;
      SU2B_CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      const int rc = enqueue_fused(ctx, fops, false, cached, S, X, Y, &F);
      const cudaError_t ec = cudaStreamEndCapture(s, &graph);
      if (rc != SU2B_OK) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
      }
      SU2B_CK(ec);
      su2b_ctx::GraphEntry e{nullptr, ctx->launches - n0};
      ctx->launches = n0;
      const cudaError_t ei = cudaGraphInstantiate(&e.exec, graph, 0);
      cudaGraphDestroy(graph);
      SU2B_CK(ei);
      it = ctx->graphs.emplace(key, e).first;
      ctx->graph_final[key] = F;
    }
    F = ctx->graph_final[key];
    SU2B_CK(cudaGraphLaunch(it->second.exec, s));
    ctx->launches += it->second.kernels;
  }
  SU2B_CK(cudaStreamSynchronize(s));
  const TrajDev &t = *ctx->h_traj;
  const double *r = ctx->h_red;
  if (t.accepted) {  // the final field becomes current; S and the spare become scratch
    ctx->U = F;
    ctx->U_old = S;
    ctx->U2 = (F == X) ? Y : X;
  }
  res->accepted = t.accepted;
  res->dH = t.dH;
  for (int k = 0; k < 3; k++) {
    res->H_old[k] = t.H_old[k];
    res->H_new[k] = t.H_new[k];
  }
  res->ddH = 0.0;
  res->plaquette = t.accepted ? r[5] : r[1];
  res->cg_iterations = 0;
  if (ctx->pend.size() > 4096) SU2B_CKS(su2b_prof_fold(ctx));
  // red[1..3] and red[5..7] now hold the start and end plaquettes; the next trajectory of an
  // uninterrupted sequence takes its start plaquettes from them (any other call clears this)
  ctx->start_plaq_cached = true;
  return SU2B_OK;
}

}  // namespace

extern "C" int su2b_hmc_trajectory(su2b_ctx *ctx, const su2b_hmc_params *prm,
                                   su2b_traj_result *res) {
  if (!ctx) return SU2B_ERR_INVALID;
  const bool cached = ctx->start_plaq_cached;
  ctx->begin_call();
  SU2B_CK(cudaSetDevice(ctx->device));
  SU2B_NEED(prm && res, "params or result is NULL");
  SU2B_NEED(prm->n_steps >= 1, "n_steps must be >= 1");
  const bool lp = low_precision(prm->integrator);
  SU2B_NEED(!lp || (prm->round_exponent >= 0 && prm->round_exponent <= 19),
            "round_exponent must be in 0..19 (10^e as a size_t)");
  // the rounding to 10^-e is defined on FP64 links and momenta (integrator.hh:53-80,
  // 158-199); on FP32 storage it would round nothing past e = 7
  if (lp && !ctx->link64)
    return su2b_fail(ctx, SU2B_ERR_UNSUPPORTED,
                     "lp_leapfrog / lp_omf4 need FP64 links (SU2B_PREC_FP64)");
  const bool ferm = prm->fermion_mass > 0.0;
  if (ferm && ctx->group != SU2B_GROUP_U1)
    return su2b_fail(ctx, SU2B_ERR_UNSUPPORTED,
                     "staggered fermions are U(1) only (detDDdag_monomial.hh:170-192)");
  cudaStream_t s = ctx->stream;
  TrajParams tp;
  tp.beta = ctx->beta;
  tp.Nc = ctx->Nc();
  tp.u_host = prm->uniform_host;
  tp.seed = prm->seed;
  tp.traj = prm->traj;
  tp.accept_reject = prm->accept_reject;
  *ctx->h_tparams = tp;
  SU2B_CK(cudaMemcpyAsync(ctx->tparams, ctx->h_tparams, sizeof(TrajParams),
                          cudaMemcpyHostToDevice, s));
  if (ctx->group == SU2B_GROUP_SU2 && !ferm && !prm->revtest && !lp &&
      ctx->traj_path == SU2B_TRAJ_FUSED_GRAPH)
    return traj_fused(ctx, prm, cached, res);

  // generic path: U(1), fermions, reversibility test, the low-precision integrators and the
  // plain form (SU2B_TRAJ_PLAIN)
  const std::vector<Op> ops = schedule(prm->integrator, prm->n_steps, prm->tau);
  long cg_iters = 0;
  int nb = 0;
  // momenta + H_kin old -> red[0]
  if (prm->momenta_host) {
    SU2B_CKS(su2b_adj_upload(ctx, prm->momenta_host, ctx->P));
    SU2B_CKS(kinetic_now(ctx, 0));
  } else {
    if (ctx->link64)
      SU2B_LAUNCH(SU2B_K_MOMENTA, momenta_philox<double>(ctx->g, (double *)ctx->P, ctx->group,
                                                         ctx->tparams, ctx->part_slot(1), &nb, s));
    else
      SU2B_LAUNCH(SU2B_K_MOMENTA, momenta_philox<float>(ctx->g, (float *)ctx->P, ctx->group,
                                                        ctx->tparams, ctx->part_slot(1), &nb, s));
    SU2B_LAUNCH(SU2B_K_OTHER, reduce_final(ctx->part_slot(1), nb, 1, ctx->red + 0, s));
  }
  SU2B_CK(cudaMemsetAsync(ctx->red + 8, 0, 2 * sizeof(double), s));
  if (ferm)
    SU2B_CKS(su2b_fermion_heatbath_q(ctx, prm->fermion_mass, prm->pf_source_host, prm->seed,
                                     prm->traj, prm->pf_complex, 8));
  // S_G old -> red[1..3]
  SU2B_CKS(su2b_q_plaq(ctx, ctx->U, 1));
  SU2B_CK(cudaMemcpyAsync(ctx->U_old, ctx->U, ctx->link_bytes() * ctx->NL,
                          cudaMemcpyDeviceToDevice, s));
  SU2B_CKS(integrate(ctx, ops, prm, 4, &cg_iters));
  SU2B_CKS(su2b_q_plaq(ctx, ctx->U, 5));
  if (ferm) {
    long it = 0;
    SU2B_CKS(su2b_fermion_action_q(ctx, prm->fermion_mass, prm->cg_tol, prm->cg_max_iter,
                                   prm->cg_start, prm->pf_seed, 9, &it));
    cg_iters += it;
  }
  SU2B_LAUNCH(SU2B_K_OTHER, accept_step(ctx->red, ctx->tparams, ctx->traj, s));

  if (prm->revtest) {  // md_update.hh:62-74
    if (!ctx->U_rev) {
      SU2B_CK(cudaMalloc(&ctx->U_rev, ctx->link_bytes() * ctx->NL));
      ctx->allocs.push_back(ctx->U_rev);
    }
    SU2B_CK(cudaMemcpyAsync(ctx->U_rev, ctx->U, ctx->link_bytes() * ctx->NL,
                            cudaMemcpyDeviceToDevice, s));
    if (ctx->link64)
      SU2B_LAUNCH(SU2B_K_OTHER, negate_adj<double>(ctx->g, (double *)ctx->P, ctx->group, s));
    else
      SU2B_LAUNCH(SU2B_K_OTHER, negate_adj<float>(ctx->g, (float *)ctx->P, ctx->group, s));
    SU2B_CKS(integrate(ctx, ops, prm, 10, &cg_iters));
    SU2B_CKS(su2b_q_plaq(ctx, ctx->U, 11));
    SU2B_CK(cudaMemsetAsync(ctx->red + 14, 0, sizeof(double), s));
    if (ferm) {
      long it = 0;
      SU2B_CKS(su2b_fermion_action_q(ctx, prm->fermion_mass, prm->cg_tol, prm->cg_max_iter,
                                     prm->cg_start, prm->pf_seed, 14, &it));
      cg_iters += it;
    }
    SU2B_CK(cudaMemcpyAsync(ctx->U, ctx->U_rev, ctx->link_bytes() * ctx->NL,
                            cudaMemcpyDeviceToDevice, s));
    ctx->phases_valid = ctx->phases32_valid = false;
  }
  if (ctx->link64)
    SU2B_LAUNCH(SU2B_K_OTHER,
                cond_restore<double>(ctx->g, ctx->U, ctx->U_old, ctx->group, ctx->traj, s));
  else
    SU2B_LAUNCH(SU2B_K_OTHER,
                cond_restore<float>(ctx->g, ctx->U, ctx->U_old, ctx->group, ctx->traj, s));
  ctx->phases_valid = ctx->phases32_valid = false;
  SU2B_CK(cudaMemcpyAsync(ctx->h_traj, ctx->traj, sizeof(TrajDev), cudaMemcpyDeviceToHost, s));
  SU2B_CKS(su2b_fetch_red(ctx, 20));
  const TrajDev &t = *ctx->h_traj;
  const double *r = ctx->h_red;
  res->accepted = t.accepted;
  res->dH = t.dH;
  for (int k = 0; k < 3; k++) {
    res->H_old[k] = t.H_old[k];
    res->H_new[k] = t.H_new[k];
  }
  res->ddH = 0.0;
  if (prm->revtest) {
    double d = 0.;
    d += 0.5 * r[10] - t.H_old[0];
    d += (-ctx->beta * r[13] / ctx->Nc()) - t.H_old[1];
    d += r[14] - t.H_old[2];
    res->ddH = d;
  }
  res->plaquette = t.accepted ? r[5] : r[1];
  res->cg_iterations = cg_iters;
  if (ctx->pend.size() > 4096) SU2B_CKS(su2b_prof_fold(ctx));
  return SU2B_OK;
}
