// solver.h -- device-resident Krylov solver state and kernel launchers (staggered.cu).
#pragma once
#include <cuda_runtime.h>

#include "su2b_common.cuh"

namespace su2b {

// Scalars of one solve, kept in device memory so iterations run without host round trips.
// done: 0 running, 1 converged, 2 iteration limit, 3 NaN residual.
struct SolverState {
  double2 rr;      // <r, r> (CG) of the current residual
  double2 alpha, beta, omega, r0r;
  double rr_new;   // mixed CG: |r_s|^2 after the update / true |r|^2 after a reliable update
  double rn;       // residual norm
  double tol;
  double maxr;     // mixed CG: |r| at the last reliable update
  double delta;    // mixed CG: reliable-update threshold
  long iters, max_iter, updates;
  int done;
  int do_update;
};

int hop_blocks(const Geom &g);
int vec_blocks(int n);
cudaError_t hop64(const Geom &g, const double2 *ph, double m, int dag, const double2 *in,
                  double2 *out, const double2 *a, double *dpart, double *npart,
                  const SolverState *st, int gate_update, cudaStream_t s);
cudaError_t hop32(const Geom &g, const float2 *ph, float m, int dag, const float2 *in,
                  float2 *out, const float2 *a, double *dpart, double *npart,
                  const SolverState *st, cudaStream_t s);
cudaError_t cg_alpha(const double *part, int n, SolverState *st, cudaStream_t s);
cudaError_t cg_xr(int n, double2 *x, double2 *r, const double2 *p, const double2 *Ap,
                  const SolverState *st, double *part, cudaStream_t s);
cudaError_t cg_beta(const double *part, int n, SolverState *st, cudaStream_t s);
cudaError_t cg_p(int n, const double2 *r, double2 *p, const SolverState *st, cudaStream_t s);
cudaError_t bi_alpha(const double *part, int n, SolverState *st, cudaStream_t s);
cudaError_t bi_s(int n, const double2 *r, const double2 *Ap, double2 *sv, const SolverState *st,
                 cudaStream_t s);
cudaError_t bi_omega(const double *dpart, const double *npart, int n, SolverState *st,
                     cudaStream_t s);
cudaError_t bi_rx(int n, double2 *x, double2 *r, const double2 *sv, const double2 *t,
                  const double2 *p, const double2 *r0, const SolverState *st, double *dpart,
                  double *npart, cudaStream_t s);
cudaError_t bi_beta(const double *dpart, const double *npart, int n, SolverState *st,
                    cudaStream_t s);
cudaError_t bi_p(int n, const double2 *r, double2 *p, const double2 *Ap, const SolverState *st,
                 cudaStream_t s);
cudaError_t m_xr(int n, float2 *xs, float2 *rs, const float2 *ps, const float2 *Aps,
                 const SolverState *st, double *part, cudaStream_t s);
cudaError_t m_check(const double *part, int n, SolverState *st, cudaStream_t s);
cudaError_t m_accum(int n, double2 *x, float2 *xs, const SolverState *st, cudaStream_t s);
cudaError_t m_resid(int n, const double2 *b, const double2 *Ax, double2 *r, float2 *rs,
                    const SolverState *st, double *part, cudaStream_t s);
cudaError_t m_after(const double *part, int n, SolverState *st, cudaStream_t s);
cudaError_t m_p(int n, const float2 *rs, float2 *ps, SolverState *st, cudaStream_t s);

cudaError_t cg_persistent(const Geom &g, const double2 *ph, double m, double2 *x, double2 *r,
                          double2 *p, double2 *t, double *part, SolverState *st, void *bar_mem,
                          int part_cap, cudaStream_t s);
cudaError_t cg_mixed_persistent(const Geom &g, const double2 *ph, const float2 *ph32, double m,
                                const double2 *b, double2 *x, double2 *r, double2 *t64,
                                float2 *xs, float2 *rs, float2 *ps, float2 *ts, double *part,
                                SolverState *st, void *bar_mem, int part_cap, cudaStream_t s);
cudaError_t bicgstab_persistent(const Geom &g, const double2 *ph, double m, double2 *x,
                                double2 *r, const double2 *r0, double2 *p, double2 *p2,
                                double2 *Ap, double2 *Ap2, double2 *sv, double2 *t,
                                double *part, SolverState *st, void *bar_mem, int part_cap,
                                cudaStream_t s);
int cg_barrier_failed(const void *bar_mem, cudaStream_t s, int *failed);
size_t cg_barrier_bytes();

cudaError_t pion_slices(const Geom &g, const double2 *S, double *C, cudaStream_t s);

cudaError_t resid64(int n, const double2 *b, const double2 *Ax, double2 *r, double *part,
                    cudaStream_t s);
cudaError_t to32(int n, const double2 *a, float2 *b, cudaStream_t s);
cudaError_t dot64(int n, const double2 *a, const double2 *b, double *part, cudaStream_t s);

}  // namespace su2b
