// staggered.cu -- U(1) staggered operator, fermion force and the Krylov-solver kernels.
//
// Operator (staggered.hpp:305-389), eta_mu(x) = (-1)^(sum_{nu<mu} x_nu) (staggered.hpp:41-48):
//   D psi(x)    = m psi(x) + 1/2 sum_mu eta_mu(x) [e^{i th_mu(x)} psi(x+mu)
//                                                 - e^{-i th_mu(x-mu)} psi(x-mu)]
//   Ddag psi(x) = m psi(x) - (the same hopping sum)
// Spinors are complex per site in even/odd order; links enter as a phase field
// (cos th, sin th) rebuilt whenever the angles change.  Bytes per site and application in
// FP64: psi in 16 + out 16 + 2*nd phases 16 (plus neighbour re-reads served by L1/L2).
//
// Solvers: every kernel below reads a SolverState in device memory and returns at once when
// the state says the solve has finished, so the host can queue many iterations and read
// the state back only every few of them.  Scalars (alpha, beta, omega) are computed on the
// device in FP64 with the reference's complex arithmetic (CG.hpp:51-64,
// BiCGStab.hpp:49-66).
#include "su2b_internal.h"
#include "solver.h"

namespace su2b {
namespace {

template <class R> struct C2;
template <> struct C2<double> { typedef double2 type; };
template <> struct C2<float> { typedef float2 type; };

__device__ __forceinline__ double2 cm(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cmc(double2 a, double2 b) {  // conj(a) * b
  return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
// libgcc's complex division for ordinary magnitudes (Smith, CACM 5 (1962) 435)
__device__ __forceinline__ double2 cdivs(double2 x, double2 y) {
  const double a = x.x, b = x.y, c = y.x, d = y.y;
  if (fabs(c) < fabs(d)) {
    const double ratio = c / d, denom = (c * ratio) + d;
    return make_double2(((a * ratio) + b) / denom, ((b * ratio) - a) / denom);
  }
  const double ratio = d / c, denom = (d * ratio) + c;
  return make_double2(((b * ratio) + a) / denom, (b - (a * ratio)) / denom);
}

__device__ __forceinline__ bool finished(const SolverState *st) {
  return st != nullptr && st->done != 0;
}

__global__ void k_phases(size_t NL, const double *__restrict__ th, double2 *ph) {
  for (size_t l = blockIdx.x * (size_t)blockDim.x + threadIdx.x; l < NL;
       l += (size_t)gridDim.x * blockDim.x) {
    double s, c;
    sincos(th[l], &s, &c);
    ph[l] = make_double2(c, s);
  }
}
__global__ void k_phases32(size_t NL, const double *__restrict__ th, float2 *ph) {
  for (size_t l = blockIdx.x * (size_t)blockDim.x + threadIdx.x; l < NL;
       l += (size_t)gridDim.x * blockDim.x) {
    double s, c;
    sincos(th[l], &s, &c);
    ph[l] = make_float2((float)c, (float)s);
  }
}

// out = m*in + sgn*hop(in); optional per-block partial of sum conj(a) * out (dot) and
// sum |out|^2 (nrm).  gate: skip when the solve finished (or when gate_update says so).
template <class R, int NT>
__global__ void __launch_bounds__(NT)
  k_hop(Geom g, const typename C2<R>::type *__restrict__ ph, R m, R sgn,
        const typename C2<R>::type *__restrict__ in, typename C2<R>::type *__restrict__ out,
        const typename C2<R>::type *__restrict__ a, double *dot_part, double *nrm_part,
        const SolverState *st, int gate_update) {
  typedef typename C2<R>::type cR;
  if (finished(st) || (gate_update && !st->do_update)) return;
  __shared__ double sh[NT / 32];
  const int p = blockIdx.y;
  const int cb = blockIdx.x * NT + threadIdx.x;
  double dr = 0., di = 0., nn = 0.;
  if (cb < g.Vh) {
    const Site s = site_from_eo(g, p, cb);
    R accr = 0, acci = 0;
    int esum = 0;
    // a compile-time bound with a guard keeps every index constant: with the runtime bound the
    // loop indexes the site's coordinates and the geometry by a variable, which puts both in
    // local memory
#pragma unroll
    for (int mu = 0; mu < 4; mu++) {
      if (mu >= g.nd) break;
      const R eta = (esum & 1) ? R(-0.5) : R(0.5);
      esum += s.c[mu];
      const int lp = s.lex + fwd(g, s, mu), lm = s.lex + bwd(g, s, mu);
      const cR up = ph[(size_t)mu * g.V + (size_t)p * g.Vh + cb];
      const cR um = ph[(size_t)mu * g.V + eo_of(g, lm, 1 - p)];
      const cR fp = in[eo_of(g, lp, 1 - p)], fm = in[eo_of(g, lm, 1 - p)];
      // e^{i th(x)} psi(x+mu) - e^{-i th(x-mu)} psi(x-mu)
      const R tr = (up.x * fp.x - up.y * fp.y) - (um.x * fm.x + um.y * fm.y);
      const R ti = (up.x * fp.y + up.y * fp.x) - (um.x * fm.y - um.y * fm.x);
      accr += eta * tr;
      acci += eta * ti;
    }
    const cR self = in[(size_t)p * g.Vh + cb];
    cR o;
    o.x = m * self.x + sgn * accr;
    o.y = m * self.y + sgn * acci;
    out[(size_t)p * g.Vh + cb] = o;
    if (dot_part) {
      const cR av = a[(size_t)p * g.Vh + cb];
      dr = (double)av.x * o.x + (double)av.y * o.y;
      di = (double)av.x * o.y - (double)av.y * o.x;
    }
    if (nrm_part) nn = (double)o.x * o.x + (double)o.y * o.y;
  }
  const int b = blockIdx.y * gridDim.x + blockIdx.x;
  if (dot_part) {
    double r = block_sum<NT>(dr, sh);
    if (threadIdx.x == 0) dot_part[2 * b] = r;
    r = block_sum<NT>(di, sh);
    if (threadIdx.x == 0) dot_part[2 * b + 1] = r;
  }
  if (nrm_part) {
    const double r = block_sum<NT>(nn, sh);
    if (threadIdx.x == 0) nrm_part[b] = r;
  }
}

// fermion force per link (detDDdag_monomial.hh:124-164)
__global__ void k_fforce(Geom g, const double2 *__restrict__ ph, const double2 *__restrict__ chi,
                         const double2 *__restrict__ chi1, double *deriv) {
  const int mu = blockIdx.y >> 1, p = blockIdx.y & 1;
  const int cb = blockIdx.x * blockDim.x + threadIdx.x;
  if (cb >= g.Vh) return;
  const Site s = site_from_eo(g, p, cb);
  int esum = 0;
#pragma unroll
  for (int nu = 0; nu < 3; nu++) esum += nu < mu ? s.c[nu] : 0;  // constant indexes
  const double eta = (esum & 1) ? -1.0 : 1.0;
  const size_t l = (size_t)mu * g.V + (size_t)p * g.Vh + cb;
  const int sx = p * g.Vh + cb, sp = eo_of(g, s.lex + fwd_rt(g, s, mu), 1 - p);
  const double2 u = ph[l], ud = make_double2(u.x, -u.y);
  // v_xp = (1/2 eta i) U chi1(x+mu);  v_x = (-1/2 eta (-i)) U^+ chi1(x)
  const double2 v_xp = cm(cm(make_double2(0.0, 0.5 * eta), u), chi1[sp]);
  const double2 v_x = cm(cm(make_double2(0.0, 0.5 * eta), ud), chi1[sx]);
  const double2 d = make_double2(cmc(chi[sx], v_xp).x + cmc(chi[sp], v_x).x,
                                 cmc(chi[sx], v_xp).y + cmc(chi[sp], v_x).y);
  // get_deriv(-2 i d) = Im(-2 i d) = -2 Re d
  deriv[l] = -2.0 * d.x;
}

__global__ void k_pf_source(Geom g, uint64_t seed, uint32_t traj, int cplx, double2 *R) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.V; i += gridDim.x * blockDim.x) {
    const Site s = site_from_lex(g, i);
    uint32_t r[4];
    philox((uint32_t)i, 0u, traj, TAG_PF, seed, r);
    double n0, n1;
    box_muller(u01_53(r[0], r[1]), u01_53(r[2], r[3]), n0, n1);
    const double sg = 0.7071067811865476;  // 1/sqrt(2)
    R[eo_of(g, i, s.p)] = make_double2(sg * n0, cplx ? sg * n1 : 0.0);
  }
}

// ---------------- solver scalar steps (one block) ----------------
template <int NT>
__device__ __forceinline__ double2 sum2(const double *part, int n, double *sh) {
  double a = 0., b = 0.;
  for (int i = threadIdx.x; i < n; i += NT) {
    a += part[2 * i];
    b += part[2 * i + 1];
  }
  const double ra = block_sum<NT>(a, sh);
  const double rb = block_sum<NT>(b, sh);
  return make_double2(ra, rb);
}
template <int NT>
__device__ __forceinline__ double sum1(const double *part, int n, double *sh) {
  double a = 0.;
  for (int i = threadIdx.x; i < n; i += NT) a += part[i];
  return block_sum<NT>(a, sh);
}

__device__ __forceinline__ void check_iter(SolverState *st) {
  st->iters++;
  if (st->rn != st->rn) st->done = 3;
  else if (!(st->rn > st->tol)) st->done = 1;
  else if (st->iters >= st->max_iter) st->done = 2;
}

// CG: alpha = rr / <p, A p>
template <int NT> __global__ void k_cg_alpha(const double *part, int n, SolverState *st) {
  if (finished(st)) return;
  __shared__ double sh[NT / 32];
  const double2 pAp = sum2<NT>(part, n, sh);
  if (threadIdx.x == 0) st->alpha = cdivs(st->rr, pAp);
}
// CG: rr_new = <r, r>; beta = rr_new / rr; rr = rr_new; rn = |r|
template <int NT> __global__ void k_cg_beta(const double *part, int n, SolverState *st) {
  if (finished(st)) return;
  __shared__ double sh[NT / 32];
  const double rr = sum1<NT>(part, n, sh);
  if (threadIdx.x == 0) {
    const double2 rrn = make_double2(rr, 0.0);
    st->beta = cdivs(rrn, st->rr);
    st->rr = rrn;
    st->rn = sqrt(rr);
    check_iter(st);
  }
}

// x += alpha p; r -= alpha Ap; partial |r|^2
template <int NT>
__global__ void __launch_bounds__(NT)
  k_cg_xr(int n, double2 *__restrict__ x, double2 *__restrict__ r, const double2 *__restrict__ p,
          const double2 *__restrict__ Ap, const SolverState *st, double *part) {
  if (finished(st)) return;
  __shared__ double sh[NT / 32];
  const double2 al = st->alpha;
  double nn = 0.;
  for (int i = blockIdx.x * NT + threadIdx.x; i < n; i += gridDim.x * NT) {
    const double2 ap = cm(al, p[i]), aq = cm(al, Ap[i]);
    x[i] = make_double2(x[i].x + 1.0 * ap.x, x[i].y + 1.0 * ap.y);
    const double2 rn = make_double2(r[i].x + (-1.0) * aq.x, r[i].y + (-1.0) * aq.y);
    r[i] = rn;
    nn += rn.x * rn.x + rn.y * rn.y;
  }
  const double t = block_sum<NT>(nn, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}
// p = r + beta p
__global__ void k_cg_p(int n, const double2 *__restrict__ r, double2 *__restrict__ p,
                       const SolverState *st) {
  if (finished(st)) return;
  const double2 be = st->beta;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double2 bp = cm(be, p[i]);
    p[i] = make_double2(r[i].x + 1.0 * bp.x, r[i].y + 1.0 * bp.y);
  }
}

// pion correlator: C[t] = sum over the spatial sites of time slice t of |S(t, x)|^2 / Vs,
// one block per t summing its slice in a fixed order (propagator.hpp:43-60)
template <int NT>
__global__ void __launch_bounds__(NT)
  k_pion_slices(Geom g, const double2 *__restrict__ S, double *C) {
  __shared__ double sh[NT / 32];
  const int t = blockIdx.x;
  const int Vs = g.V / g.L[0];
  double acc = 0.;
  for (int i = threadIdx.x; i < Vs; i += NT) {
    const int lex = t * Vs + i;
    const Site s = site_from_lex(g, lex);
    const double2 v = S[eo_of(g, lex, s.p)];
    acc += v.x * v.x + v.y * v.y;
  }
  const double r = block_sum<NT>(acc, sh);
  if (threadIdx.x == 0) C[t] = t == 0 ? 0.0 : r / (double)Vs;
}

// ---- persistent CG on D D^+ (one cooperative launch for the whole solve) ----
//
// For small lattices every CG iteration is a handful of microsecond-long kernels and the
// launches dominate.  This kernel keeps all blocks resident (cooperative launch: the runtime
// refuses the launch unless every block can be resident at once) and separates the phases by
// a grid barrier.  It uses D D^+ = A with <p, A p> = |D^+ p|^2 and, by linearity,
// D^+ p_new = D^+ r + beta D^+ p, so one iteration needs two barriers:
//   [t = D^+ p held]  alpha = rr / |t|^2;  Ap = D t;  x += alpha p;  r -= alpha Ap   | barrier
//   beta = |r|^2 / rr;  p = r + beta p;  t = D^+ r + beta t                         | barrier
// The scalars follow CG.hpp:51-64 in FP64 (complex alpha/beta with zero imaginary parts).
// Every block reduces the per-block partials itself in one fixed order, so all blocks take
// the same decisions and leave the loop together.  Barrier waits are bounded: a wait that
// gives up sets *err and every block returns.
// m*in + sgn*hop(in) at one site, with in(j) the input vector's value at even/odd index j
template <class In>
__device__ __forceinline__ double2 hop_site64_f(const Geom &g, const double2 *__restrict__ ph,
                                                double m, double sgn, In in, int p, int cb) {
  const Site s = site_from_eo(g, p, cb);
  double accr = 0, acci = 0;
  int esum = 0;
#pragma unroll
  for (int mu = 0; mu < 4; mu++) {  // constant indexes (see k_hop)
    if (mu >= g.nd) break;
    const double eta = (esum & 1) ? -0.5 : 0.5;
    esum += s.c[mu];
    const int lp = s.lex + fwd(g, s, mu), lm = s.lex + bwd(g, s, mu);
    const double2 up = ph[(size_t)mu * g.V + (size_t)p * g.Vh + cb];
    const double2 um = ph[(size_t)mu * g.V + eo_of(g, lm, 1 - p)];
    const double2 fp = in(eo_of(g, lp, 1 - p)), fm = in(eo_of(g, lm, 1 - p));
    const double tr = (up.x * fp.x - up.y * fp.y) - (um.x * fm.x + um.y * fm.y);
    const double ti = (up.x * fp.y + up.y * fp.x) - (um.x * fm.y - um.y * fm.x);
    accr += eta * tr;
    acci += eta * ti;
  }
  const double2 self = in((size_t)p * g.Vh + cb);
  return make_double2(m * self.x + sgn * accr, m * self.y + sgn * acci);
}
__device__ __forceinline__ double2 hop_site64(const Geom &g, const double2 *__restrict__ ph,
                                              double m, double sgn,
                                              const double2 *__restrict__ in, int p, int cb) {
  // neighbours belong to other blocks and change every iteration: read through L2 only
  // (the SM's L1 is not coherent with the other SMs' stores)
  return hop_site64_f(g, ph, m, sgn, [in](size_t j) { return __ldcg(&in[j]); }, p, cb);
}

__device__ __forceinline__ float2 hop_site32(const Geom &g, const float2 *__restrict__ ph,
                                             float m, float sgn, const float2 *__restrict__ in,
                                             int p, int cb) {
  const Site s = site_from_eo(g, p, cb);
  float accr = 0.f, acci = 0.f;
  int esum = 0;
#pragma unroll
  for (int mu = 0; mu < 4; mu++) {  // constant indexes (see k_hop)
    if (mu >= g.nd) break;
    const float eta = (esum & 1) ? -0.5f : 0.5f;
    esum += s.c[mu];
    const int lp = s.lex + fwd(g, s, mu), lm = s.lex + bwd(g, s, mu);
    const float2 up = ph[(size_t)mu * g.V + (size_t)p * g.Vh + cb];
    const float2 um = ph[(size_t)mu * g.V + eo_of(g, lm, 1 - p)];
    const float2 fp = __ldcg(&in[eo_of(g, lp, 1 - p)]), fm = __ldcg(&in[eo_of(g, lm, 1 - p)]);
    const float tr = (up.x * fp.x - up.y * fp.y) - (um.x * fm.x + um.y * fm.y);
    const float ti = (up.x * fp.y + up.y * fp.x) - (um.x * fm.y - um.y * fm.x);
    accr += eta * tr;
    acci += eta * ti;
  }
  const float2 self = __ldcg(&in[(size_t)p * g.Vh + cb]);
  return make_float2(m * self.x + sgn * accr, m * self.y + sgn * acci);
}

struct GridBarrier {
  unsigned long long count;  // arrivals since the launch; the host zeroes it before each launch
  int err;
};

constexpr long BARRIER_SPIN_LIMIT = 1L << 24;  // x >= 32 ns: gives up after about a second

// One atomic per block and barrier: block b's k-th arrival draws a ticket from the running
// 64-bit count, and the barrier of that round is complete when the count reaches the
// round's end, (ticket / G + 1) G.  The arrival has release semantics (after the block barrier it
// publishes every write of the block), the polling load acquire semantics.  No block resets
// anything, so no second round trip is needed.
__device__ __forceinline__ bool grid_sync(GridBarrier *b) {
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long ticket;
    asm volatile("atom.add.release.gpu.u64 %0, [%1], 1;"
                 : "=l"(ticket)
                 : "l"(&b->count)
                 : "memory");
    const unsigned long long target = (ticket / gridDim.x + 1) * gridDim.x;
    long spins = 0;
    for (;;) {
      unsigned long long cur;
      asm volatile("ld.acquire.gpu.u64 %0, [%1];" : "=l"(cur) : "l"(&b->count) : "memory");
      if (cur >= target) break;
      // another block's wait gave up: checked every 64 polls (a load per poll costs time)
      if ((++spins & 63) == 0 && *(volatile int *)&b->err != 0) break;
      if (spins > BARRIER_SPIN_LIMIT) {
        atomicExch(&b->err, 1);
        break;
      }
      __nanosleep(32);
    }
  }
  __syncthreads();
  return *(volatile int *)&b->err == 0;
}

// sum of part[0..n) in one fixed order (lane-strided, then a fixed warp tree), by warp 0;
// the result is broadcast through shared memory
// (n <= 32 * FIXED_SUM_PER_LANE; all loads are issued before the first add, so the sum costs
// one L2 round trip)
constexpr int FIXED_SUM_PER_LANE = 16;
template <int NT> __device__ __forceinline__ double fixed_sum(const double *part, int n) {
  __shared__ double bc;
  if (threadIdx.x < 32) {
    double v[FIXED_SUM_PER_LANE];
#pragma unroll
    for (int k = 0; k < FIXED_SUM_PER_LANE; k++) {
      const int i = threadIdx.x + 32 * k;
      v[k] = i < n ? __ldcg(&part[i]) : 0.0;
    }
    double a = 0.;
#pragma unroll
    for (int k = 0; k < FIXED_SUM_PER_LANE; k++) a += v[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (threadIdx.x == 0) bc = a;
  }
  __syncthreads();
  const double r = bc;
  __syncthreads();
  return r;
}

template <int NT>
__global__ void __launch_bounds__(NT, 1)
  k_cg_persistent(Geom g, const double2 *__restrict__ ph, double m, double2 *x, double2 *r,
                  double2 *p, double2 *t, double *part_t, double *part_r, SolverState *st,
                  GridBarrier *bar) {
  __shared__ double sh[NT / 32];
  const int n = g.V, G = gridDim.x;
  const int first = blockIdx.x * NT + threadIdx.x, stride = G * NT;
  double2 rr = st->rr;
  double rn = st->rn;
  long iters = st->iters;
  const long max_iter = st->max_iter;
  const double tol = st->tol;
  int done = st->done;
  // t = D^+ p, |t|^2
  double acc = 0.;
  for (int i = first; i < n; i += stride) {
    const int pp = i >= g.Vh, cb = i - pp * g.Vh;
    const double2 v = hop_site64(g, ph, m, -1.0, p, pp, cb);
    t[i] = v;
    acc += v.x * v.x + v.y * v.y;
  }
  double bs = block_sum<NT>(acc, sh);
  if (threadIdx.x == 0) part_t[blockIdx.x] = bs;
  if (!grid_sync(bar)) return;
  // Each phase reads its first site's stencil and own values before the global sum it
  // waits for, so the two L2 round trips overlap (at 256^2 every thread has one site).
  const bool has0 = first < n;
  const int pp0 = first >= g.Vh, cb0 = first - pp0 * g.Vh;
  while (!done) {
    double2 ap0{}, pv0{}, xv0{}, rv0{};
    if (has0) {
      ap0 = hop_site64(g, ph, m, 1.0, t, pp0, cb0);  // A p = D t
      pv0 = p[first];
      xv0 = x[first];
      rv0 = r[first];
    }
    const double2 alpha = cdivs(rr, make_double2(fixed_sum<NT>(part_t, G), 0.0));
    acc = 0.;
    for (int i = first; i < n; i += stride) {
      double2 ap, pv, xv, rv;
      if (i == first) {
        ap = ap0, pv = pv0, xv = xv0, rv = rv0;
      } else {
        const int pp = i >= g.Vh, cb = i - pp * g.Vh;
        ap = hop_site64(g, ph, m, 1.0, t, pp, cb);
        pv = p[i], xv = x[i], rv = r[i];
      }
      const double2 a1 = cm(alpha, pv), a2 = cm(alpha, ap);
      x[i] = make_double2(xv.x + a1.x, xv.y + a1.y);
      const double2 rnw = make_double2(rv.x - a2.x, rv.y - a2.y);
      r[i] = rnw;
      acc += rnw.x * rnw.x + rnw.y * rnw.y;
    }
    bs = block_sum<NT>(acc, sh);
    if (threadIdx.x == 0) part_r[blockIdx.x] = bs;
    if (!grid_sync(bar)) return;
    double2 dr0{}, rw0{}, pw0{}, tw0{};
    if (has0) {
      dr0 = hop_site64(g, ph, m, -1.0, r, pp0, cb0);  // D^+ r
      rw0 = r[first];
      pw0 = p[first];
      tw0 = t[first];
    }
    const double rr_new = fixed_sum<NT>(part_r, G);
    const double2 beta = cdivs(make_double2(rr_new, 0.0), rr);
    rr = make_double2(rr_new, 0.0);
    rn = sqrt(rr_new);
    iters++;
    if (rn != rn) done = 3;
    else if (!(rn > tol)) done = 1;
    else if (iters >= max_iter) done = 2;
    if (done) break;
    acc = 0.;
    for (int i = first; i < n; i += stride) {
      double2 dr, rv, pv, tv;
      if (i == first) {
        dr = dr0, rv = rw0, pv = pw0, tv = tw0;
      } else {
        const int pp = i >= g.Vh, cb = i - pp * g.Vh;
        dr = hop_site64(g, ph, m, -1.0, r, pp, cb);
        rv = r[i], pv = p[i], tv = t[i];
      }
      const double2 bp = cm(beta, pv), bt = cm(beta, tv);
      p[i] = make_double2(rv.x + bp.x, rv.y + bp.y);
      const double2 tn = make_double2(dr.x + bt.x, dr.y + bt.y);
      t[i] = tn;
      acc += tn.x * tn.x + tn.y * tn.y;
    }
    bs = block_sum<NT>(acc, sh);
    if (threadIdx.x == 0) part_t[blockIdx.x] = bs;
    if (!grid_sync(bar)) return;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->rr = rr;
    st->rn = rn;
    st->iters = iters;
    st->done = done;
  }
}

// ---- persistent mixed-precision CG: FP32 iterations, FP64 reliable updates ----
// The iteration of k_cg_persistent in FP32 vectors (ts = D^+ ps kept by linearity).  When the
// iterated |rs| falls below delta times |r| at the last update, or below the tolerance, every
// block takes a reliable update: x += xs, xs = 0; r = b - D D^+ x in FP64 (two stencil
// phases); rs = (float) r; convergence is decided on that true residual.  The decisions come
// from sums every block forms in the same order, so all blocks take them together.
template <int NT>
__global__ void __launch_bounds__(NT, 1)
  k_cg_mixed_persistent(Geom g, const double2 *__restrict__ ph, const float2 *__restrict__ ph32,
                        double m, const double2 *__restrict__ b, double2 *x, double2 *r,
                        double2 *t64, float2 *xs, float2 *rs, float2 *ps, float2 *ts,
                        double *part_t, double *part_r, SolverState *st, GridBarrier *bar) {
  __shared__ double sh[NT / 32];
  const int n = g.V, G = gridDim.x;
  const int first = blockIdx.x * NT + threadIdx.x, stride = G * NT;
  const float m32 = (float)m;
  double rr = st->rr.x, rn = st->rn, maxr = st->maxr;
  const double delta = st->delta, tol = st->tol;
  long iters = st->iters, updates = st->updates;
  const long max_iter = st->max_iter;
  int done = st->done;
  // ts = D^+ ps, |ts|^2
  double acc = 0.;
  for (int i = first; i < n; i += stride) {
    const int pp = i >= g.Vh, cb = i - pp * g.Vh;
    const float2 v = hop_site32(g, ph32, m32, -1.f, ps, pp, cb);
    ts[i] = v;
    acc += (double)v.x * v.x + (double)v.y * v.y;
  }
  double bs = block_sum<NT>(acc, sh);
  if (threadIdx.x == 0) part_t[blockIdx.x] = bs;
  if (!grid_sync(bar)) return;
  // as in k_cg_persistent, each phase reads its first site's stencil and own values before
  // the global sum it waits for
  const bool has0 = first < n;
  const int pp0 = first >= g.Vh, cb0 = first - pp0 * g.Vh;
  while (!done) {
    float2 aq0{}, pv0{}, xv0{}, rv0{};
    if (has0) {
      aq0 = hop_site32(g, ph32, m32, 1.f, ts, pp0, cb0);  // A ps = D ts
      pv0 = ps[first];
      xv0 = xs[first];
      rv0 = rs[first];
    }
    const float alpha = (float)(rr / fixed_sum<NT>(part_t, G));
    acc = 0.;
    for (int i = first; i < n; i += stride) {
      float2 aq, pv, xv, rv;
      if (i == first) {
        aq = aq0, pv = pv0, xv = xv0, rv = rv0;
      } else {
        const int pp = i >= g.Vh, cb = i - pp * g.Vh;
        aq = hop_site32(g, ph32, m32, 1.f, ts, pp, cb);
        pv = ps[i], xv = xs[i], rv = rs[i];
      }
      xv.x += alpha * pv.x;
      xv.y += alpha * pv.y;
      rv.x -= alpha * aq.x;
      rv.y -= alpha * aq.y;
      xs[i] = xv;
      rs[i] = rv;
      acc += (double)rv.x * rv.x + (double)rv.y * rv.y;
    }
    bs = block_sum<NT>(acc, sh);
    if (threadIdx.x == 0) part_r[blockIdx.x] = bs;
    if (!grid_sync(bar)) return;
    // read before the sum; a reliable update below rewrites rs and forces a re-read
    float2 dr0{}, rw0{}, pw0{}, tw0{};
    if (has0) {
      dr0 = hop_site32(g, ph32, m32, -1.f, rs, pp0, cb0);
      rw0 = rs[first];
      pw0 = ps[first];
      tw0 = ts[first];
    }
    double rr_new = fixed_sum<NT>(part_r, G);
    rn = sqrt(rr_new);
    iters++;
    if (rn != rn) {
      done = 3;
      break;
    }
    const bool update = rn < delta * maxr || !(rn > tol);
    if (!update && iters >= max_iter) {
      done = 2;
      break;
    }
    if (update) {
      for (int i = first; i < n; i += stride) {  // x += xs; xs = 0
        const float2 v = xs[i];
        x[i] = make_double2(x[i].x + (double)v.x, x[i].y + (double)v.y);
        xs[i] = make_float2(0.f, 0.f);
      }
      if (!grid_sync(bar)) return;
      for (int i = first; i < n; i += stride) {  // t64 = D^+ x
        const int pp = i >= g.Vh, cb = i - pp * g.Vh;
        t64[i] = hop_site64(g, ph, m, -1.0, x, pp, cb);
      }
      if (!grid_sync(bar)) return;
      acc = 0.;
      for (int i = first; i < n; i += stride) {  // r = b - D t64; rs = (float) r
        const int pp = i >= g.Vh, cb = i - pp * g.Vh;
        const double2 ax = hop_site64(g, ph, m, 1.0, t64, pp, cb);
        const double2 v = make_double2(b[i].x - ax.x, b[i].y - ax.y);
        r[i] = v;
        rs[i] = make_float2((float)v.x, (float)v.y);
        acc += v.x * v.x + v.y * v.y;
      }
      bs = block_sum<NT>(acc, sh);
      if (threadIdx.x == 0) part_r[blockIdx.x] = bs;
      if (!grid_sync(bar)) return;
      rr_new = fixed_sum<NT>(part_r, G);
      rn = sqrt(rr_new);
      maxr = rn;
      updates++;
      if (!(rn > tol)) {
        done = 1;
        break;
      }
      if (iters >= max_iter) {
        done = 2;
        break;
      }
      if (has0) {  // rs changed everywhere
        dr0 = hop_site32(g, ph32, m32, -1.f, rs, pp0, cb0);
        rw0 = rs[first];
      }
    }
    const float beta = (float)(rr_new / rr);
    rr = rr_new;
    acc = 0.;
    for (int i = first; i < n; i += stride) {  // ps = rs + beta ps; ts = D^+ rs + beta ts
      float2 dr, rv, pv, tv;
      if (i == first) {
        dr = dr0, rv = rw0, pv = pw0, tv = tw0;
      } else {
        const int pp = i >= g.Vh, cb = i - pp * g.Vh;
        dr = hop_site32(g, ph32, m32, -1.f, rs, pp, cb);
        rv = rs[i], pv = ps[i], tv = ts[i];
      }
      ps[i] = make_float2(rv.x + beta * pv.x, rv.y + beta * pv.y);
      const float2 tn = make_float2(dr.x + beta * tv.x, dr.y + beta * tv.y);
      ts[i] = tn;
      acc += (double)tn.x * tn.x + (double)tn.y * tn.y;
    }
    bs = block_sum<NT>(acc, sh);
    if (threadIdx.x == 0) part_t[blockIdx.x] = bs;
    if (!grid_sync(bar)) return;
  }
  if (done == 2 || done == 3)  // fold the FP32 correction into x
    for (int i = first; i < n; i += stride) {
      const float2 v = xs[i];
      x[i] = make_double2(x[i].x + (double)v.x, x[i].y + (double)v.y);
    }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->rr = make_double2(rr, 0.0);
    st->rn = rn;
    st->maxr = maxr;
    st->iters = iters;
    st->updates = updates;
    st->done = done;
  }
}

// ---- persistent BiCGStab ----
// fixed_sum of K arrays part[k*n .. k*n+n) at once: one L2 round trip for all of them
template <int K> __device__ __forceinline__ void fixed_sums(const double *part, int n,
                                                           double (&out)[K]) {
  __shared__ double bc[K];
  if (threadIdx.x < 32) {
    double v[K][FIXED_SUM_PER_LANE];
#pragma unroll
    for (int k = 0; k < K; k++)
#pragma unroll
      for (int j = 0; j < FIXED_SUM_PER_LANE; j++) {
        const int i = threadIdx.x + 32 * j;
        v[k][j] = i < n ? __ldcg(&part[k * n + i]) : 0.0;
      }
#pragma unroll
    for (int k = 0; k < K; k++) {
      double a = 0.;
#pragma unroll
      for (int j = 0; j < FIXED_SUM_PER_LANE; j++) a += v[k][j];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
      if (threadIdx.x == 0) bc[k] = a;
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < K; k++) out[k] = bc[k];
  __syncthreads();
}

// BiCGStab on D (BiCGStab.hpp:50-77) in one cooperative launch: three grid barriers per
// iteration, one per global reduction.  Where the vector a stencil phase applies D to is a
// combination of vectors the previous phase left, the combination is formed at every
// neighbour as it is read instead of being stored first (storing it would cost a barrier):
//   P1  p = r + beta p - (beta omega) Ap  (formed per site);  Ap = D p;  partial <r0, Ap>
//   P2  alpha = r0r / <r0, Ap>;  s = r - alpha Ap (formed per site);  t = D s;
//       partials <t, s>, <t, t>
//   P3  omega = <t, s> / <t, t>;  r = s - omega t;  x = x + omega s + alpha p;
//       partials <r0, r>, |r|^2;  beta = (<r0, r> / r0r)(alpha / omega)
// so A p and A s are applied directly, as in the reference, not carried by recurrences.  P1
// writes p and Ap while the neighbours still read the previous ones, so both alternate
// between two buffers.  In the first iteration p is the start residual as given.  The
// per-element arithmetic is that of the per-phase kernels below (k_bi_s, k_bi_rx, k_bi_p).
__device__ __forceinline__ double2 bi_comb_p(double2 rv, double2 pv, double2 qv, double2 be,
                                             double2 bo) {
  const double2 bp = cm(be, pv), bq = cm(bo, qv);
  const double2 t = make_double2(rv.x + 1.0 * bp.x, rv.y + 1.0 * bp.y);
  return make_double2(t.x + (-1.0) * bq.x, t.y + (-1.0) * bq.y);
}
__device__ __forceinline__ double2 bi_comb_s(double2 rv, double2 qv, double2 al) {
  const double2 aq = cm(al, qv);
  return make_double2(rv.x + (-1.0) * aq.x, rv.y + (-1.0) * aq.y);
}

template <int NT>
__global__ void __launch_bounds__(NT)
  k_bicgstab_persistent(Geom g, const double2 *__restrict__ ph, double m, double2 *x,
                        double2 *r, const double2 *__restrict__ r0, double2 *p, double2 *pn,
                        double2 *Ap, double2 *Apn, double2 *s, double2 *t, double *part,
                        SolverState *st, GridBarrier *bar) {
  __shared__ double sh[3 * (NT / 32)];
  const int n = g.V, G = gridDim.x;
  const int first = blockIdx.x * NT + threadIdx.x, stride = G * NT;
  // per-phase partial arrays: consecutive phases never share one (a block may write the next
  // phase's partials while another still reads the previous phase's)
  double *part1 = part, *part2 = part + 2 * G, *part3 = part + 5 * G;
  double2 r0r = st->r0r, alpha = make_double2(0., 0.), omega = make_double2(0., 0.),
          beta = make_double2(0., 0.);
  double rn = st->rn;
  long iters = st->iters;
  const long max_iter = st->max_iter;
  const double tol = st->tol;
  int done = st->done;
  bool start = true;
  while (!done) {
    {  // P1
      double v[2] = {0., 0.};
      const double2 be = beta, bo = cm(beta, omega);
      for (int i = first; i < n; i += stride) {
        const int pp = i >= g.Vh, cb = i - pp * g.Vh;
        double2 ap, pv;
        if (start) {
          ap = hop_site64(g, ph, m, 1.0, p, pp, cb);
          pv = p[i];
        } else {
          const auto pf = [=](size_t j) {
            return bi_comb_p(__ldcg(&r[j]), __ldcg(&p[j]), __ldcg(&Ap[j]), be, bo);
          };
          ap = hop_site64_f(g, ph, m, 1.0, pf, pp, cb);
          pv = pf(i);
        }
        pn[i] = pv;
        Apn[i] = ap;
        const double2 d = cmc(r0[i], ap);
        v[0] += d.x;
        v[1] += d.y;
      }
      block_sums<NT, 2>(v, sh);
      if (threadIdx.x == 0) {
        part1[blockIdx.x] = v[0];
        part1[G + blockIdx.x] = v[1];
      }
      if (!grid_sync(bar)) return;
      double2 *tmp = p;
      p = pn;
      pn = tmp;
      tmp = Ap;
      Ap = Apn;
      Apn = tmp;
      start = false;
    }
    {  // P2
      double q[2];
      fixed_sums<2>(part1, G, q);
      alpha = cdivs(r0r, make_double2(q[0], q[1]));
      const double2 al = alpha;
      double v[3] = {0., 0., 0.};
      const auto sf = [=](size_t j) { return bi_comb_s(__ldcg(&r[j]), __ldcg(&Ap[j]), al); };
      for (int i = first; i < n; i += stride) {
        const int pp = i >= g.Vh, cb = i - pp * g.Vh;
        const double2 tv = hop_site64_f(g, ph, m, 1.0, sf, pp, cb);
        const double2 sv = sf(i);
        s[i] = sv;
        t[i] = tv;
        const double2 d = cmc(tv, sv);
        v[0] += d.x;
        v[1] += d.y;
        v[2] += tv.x * tv.x + tv.y * tv.y;
      }
      block_sums<NT, 3>(v, sh);
      if (threadIdx.x == 0) {
        part2[blockIdx.x] = v[0];
        part2[G + blockIdx.x] = v[1];
        part2[2 * G + blockIdx.x] = v[2];
      }
      if (!grid_sync(bar)) return;
    }
    {  // P3
      double q[3];
      fixed_sums<3>(part2, G, q);
      omega = cdivs(make_double2(q[0], q[1]), make_double2(q[2], 0.0));
      const double2 om = omega, al = alpha;
      double v[3] = {0., 0., 0.};
      for (int i = first; i < n; i += stride) {
        const double2 sv = s[i], tv = t[i], pv = p[i], xv = x[i];
        const double2 ot = cm(om, tv);
        const double2 rnw = make_double2(sv.x + (-1.0) * ot.x, sv.y + (-1.0) * ot.y);
        r[i] = rnw;
        const double2 os = cm(om, sv), ap = cm(al, pv);
        const double2 x1 = make_double2(xv.x + 1.0 * os.x, xv.y + 1.0 * os.y);
        x[i] = make_double2(x1.x + 1.0 * ap.x, x1.y + 1.0 * ap.y);
        const double2 d = cmc(r0[i], rnw);
        v[0] += d.x;
        v[1] += d.y;
        v[2] += rnw.x * rnw.x + rnw.y * rnw.y;
      }
      block_sums<NT, 3>(v, sh);
      if (threadIdx.x == 0) {
        part3[blockIdx.x] = v[0];
        part3[G + blockIdx.x] = v[1];
        part3[2 * G + blockIdx.x] = v[2];
      }
      if (!grid_sync(bar)) return;
      fixed_sums<3>(part3, G, q);
      const double2 r0r_new = make_double2(q[0], q[1]);
      beta = cm(cdivs(r0r_new, r0r), cdivs(alpha, omega));
      r0r = r0r_new;
      rn = sqrt(q[2]);
      iters++;
      if (rn != rn) done = 3;
      else if (!(rn > tol)) done = 1;
      else if (iters >= max_iter) done = 2;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->r0r = r0r;
    st->alpha = alpha;
    st->omega = omega;
    st->beta = beta;
    st->rn = rn;
    st->iters = iters;
    st->done = done;
  }
}

// ---- BiCGStab ----
template <int NT> __global__ void k_bi_alpha(const double *part, int n, SolverState *st) {
  if (finished(st)) return;
  __shared__ double sh[NT / 32];
  const double2 r0Ap = sum2<NT>(part, n, sh);
  if (threadIdx.x == 0) st->alpha = cdivs(st->r0r, r0Ap);
}
__global__ void k_bi_s(int n, const double2 *__restrict__ r, const double2 *__restrict__ Ap,
                       double2 *__restrict__ s, const SolverState *st) {
  if (finished(st)) return;
  const double2 al = st->alpha;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double2 aq = cm(al, Ap[i]);
    s[i] = make_double2(r[i].x + (-1.0) * aq.x, r[i].y + (-1.0) * aq.y);
  }
}
// omega = <t, s> / <t, t>; partials: tpart = <s-side dot> written by k_hop with a = t?
// k_hop writes sum conj(a) out with a = s, out = t  ->  <s, t>; <t, s> = conj(<s, t>)
template <int NT>
__global__ void k_bi_omega(const double *dpart, const double *npart, int n, SolverState *st) {
  if (finished(st)) return;
  __shared__ double sh[NT / 32];
  const double2 st_ = sum2<NT>(dpart, n, sh);
  const double tt = sum1<NT>(npart, n, sh);
  if (threadIdx.x == 0) st->omega = cdivs(make_double2(st_.x, -st_.y), make_double2(tt, 0.0));
}
// r = s - omega t; x = x + omega s + alpha p; partials <r0, r>, |r|^2
template <int NT>
__global__ void __launch_bounds__(NT)
  k_bi_rx(int n, double2 *__restrict__ x, double2 *__restrict__ r, const double2 *__restrict__ s,
          const double2 *__restrict__ t, const double2 *__restrict__ p,
          const double2 *__restrict__ r0, const SolverState *st, double *dpart, double *npart) {
  if (finished(st)) return;
  __shared__ double sh[NT / 32];
  const double2 om = st->omega, al = st->alpha;
  double dr = 0., di = 0., nn = 0.;
  for (int i = blockIdx.x * NT + threadIdx.x; i < n; i += gridDim.x * NT) {
    const double2 ot = cm(om, t[i]);
    const double2 rn = make_double2(s[i].x + (-1.0) * ot.x, s[i].y + (-1.0) * ot.y);
    r[i] = rn;
    const double2 os = cm(om, s[i]), ap = cm(al, p[i]);
    const double2 x1 = make_double2(x[i].x + 1.0 * os.x, x[i].y + 1.0 * os.y);
    x[i] = make_double2(x1.x + 1.0 * ap.x, x1.y + 1.0 * ap.y);
    const double2 d = cmc(r0[i], rn);
    dr += d.x;
    di += d.y;
    nn += rn.x * rn.x + rn.y * rn.y;
  }
  const int b = blockIdx.x;
  double q = block_sum<NT>(dr, sh);
  if (threadIdx.x == 0) dpart[2 * b] = q;
  q = block_sum<NT>(di, sh);
  if (threadIdx.x == 0) dpart[2 * b + 1] = q;
  q = block_sum<NT>(nn, sh);
  if (threadIdx.x == 0) npart[b] = q;
}
template <int NT>
__global__ void k_bi_beta(const double *dpart, const double *npart, int n, SolverState *st) {
  if (finished(st)) return;
  __shared__ double sh[NT / 32];
  const double2 r0r = sum2<NT>(dpart, n, sh);
  const double rr = sum1<NT>(npart, n, sh);
  if (threadIdx.x == 0) {
    st->beta = cm(cdivs(r0r, st->r0r), cdivs(st->alpha, st->omega));
    st->r0r = r0r;
    st->rn = sqrt(rr);
    check_iter(st);
  }
}
// p = r + beta p - (beta omega) Ap
__global__ void k_bi_p(int n, const double2 *__restrict__ r, double2 *__restrict__ p,
                       const double2 *__restrict__ Ap, const SolverState *st) {
  if (finished(st)) return;
  const double2 be = st->beta, bo = cm(st->beta, st->omega);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double2 bp = cm(be, p[i]), bq = cm(bo, Ap[i]);
    const double2 t = make_double2(r[i].x + 1.0 * bp.x, r[i].y + 1.0 * bp.y);
    p[i] = make_double2(t.x + (-1.0) * bq.x, t.y + (-1.0) * bq.y);
  }
}

// ---- mixed-precision CG (FP32 iterations, FP64 reliable updates) ----
// xs += alpha ps; rs -= alpha Aps; partial |rs|^2
template <int NT>
__global__ void __launch_bounds__(NT)
  k_m_xr(int n, float2 *__restrict__ xs, float2 *__restrict__ rs, const float2 *__restrict__ ps,
         const float2 *__restrict__ Aps, const SolverState *st, double *part) {
  if (finished(st)) return;
  __shared__ double sh[NT / 32];
  const float ar = (float)st->alpha.x, ai = (float)st->alpha.y;
  double nn = 0.;
  for (int i = blockIdx.x * NT + threadIdx.x; i < n; i += gridDim.x * NT) {
    const float2 pv = ps[i], qv = Aps[i];
    float2 xv = xs[i], rv = rs[i];
    xv.x += ar * pv.x - ai * pv.y;
    xv.y += ar * pv.y + ai * pv.x;
    rv.x -= ar * qv.x - ai * qv.y;
    rv.y -= ar * qv.y + ai * qv.x;
    xs[i] = xv;
    rs[i] = rv;
    nn += (double)rv.x * rv.x + (double)rv.y * rv.y;
  }
  const double t = block_sum<NT>(nn, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}
// decide on a reliable update: iterated |rs| fell below delta * (|r| at the last update) or
// below the tolerance (then the true residual decides convergence)
template <int NT> __global__ void k_m_check(const double *part, int n, SolverState *st) {
  if (finished(st)) return;
  __shared__ double sh[NT / 32];
  const double rr = sum1<NT>(part, n, sh);
  if (threadIdx.x == 0) {
    st->rr_new = rr;
    st->rn = sqrt(rr);
    st->iters++;
    st->do_update = (st->rn < st->delta * st->maxr || !(st->rn > st->tol)) ? 1 : 0;
    if (st->rn != st->rn) st->done = 3;
    else if (!st->do_update && st->iters >= st->max_iter) st->done = 2;
  }
}
// x += xs; xs = 0 (only on a reliable update)
__global__ void k_m_accum(int n, double2 *__restrict__ x, float2 *__restrict__ xs,
                          const SolverState *st) {
  if (finished(st) || !st->do_update) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float2 v = xs[i];
    x[i] = make_double2(x[i].x + (double)v.x, x[i].y + (double)v.y);
    xs[i] = make_float2(0.f, 0.f);
  }
}
// r = b - Ax (FP64); rs = (float) r; partial |r|^2
template <int NT>
__global__ void __launch_bounds__(NT)
  k_m_resid(int n, const double2 *__restrict__ b, const double2 *__restrict__ Ax,
            double2 *__restrict__ r, float2 *__restrict__ rs, const SolverState *st,
            double *part) {
  if (finished(st) || !st->do_update) return;
  __shared__ double sh[NT / 32];
  double nn = 0.;
  for (int i = blockIdx.x * NT + threadIdx.x; i < n; i += gridDim.x * NT) {
    const double2 v = make_double2(b[i].x - Ax[i].x, b[i].y - Ax[i].y);
    r[i] = v;
    rs[i] = make_float2((float)v.x, (float)v.y);
    nn += v.x * v.x + v.y * v.y;
  }
  const double t = block_sum<NT>(nn, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}
template <int NT> __global__ void k_m_after(const double *part, int n, SolverState *st) {
  if (finished(st) || !st->do_update) return;
  __shared__ double sh[NT / 32];
  const double rr = sum1<NT>(part, n, sh);
  if (threadIdx.x == 0) {
    st->rr_new = rr;
    st->rn = sqrt(rr);
    st->maxr = st->rn;
    st->updates++;
    if (!(st->rn > st->tol)) st->done = 1;
    else if (st->iters >= st->max_iter) st->done = 2;
  }
}
// beta = rr_new / rr; ps = rs + beta ps; rr = rr_new
__global__ void k_m_p(int n, const float2 *__restrict__ rs, float2 *__restrict__ ps,
                      SolverState *st) {
  if (finished(st)) return;
  const double be = st->rr_new / st->rr.x;
  const float b = (float)be;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float2 r = rs[i], p = ps[i];
    ps[i] = make_float2(r.x + b * p.x, r.y + b * p.y);
  }
}
// rr = rr_new, in its own launch so that no block of k_m_p can read the new value
__global__ void k_m_commit(SolverState *st) {
  if (finished(st)) return;
  st->rr = make_double2(st->rr_new, 0.0);
}

// r = b + (-1)*Ax (a_plus_lambda_b, staggered.hpp:144-154); partial |r|^2
template <int NT>
__global__ void __launch_bounds__(NT)
  k_resid64(int n, const double2 *__restrict__ b, const double2 *__restrict__ Ax,
            double2 *__restrict__ r, double *part) {
  __shared__ double sh[NT / 32];
  double nn = 0.;
  for (int i = blockIdx.x * NT + threadIdx.x; i < n; i += gridDim.x * NT) {
    const double2 v = make_double2(b[i].x + (-1.0) * Ax[i].x, b[i].y + (-1.0) * Ax[i].y);
    r[i] = v;
    nn += v.x * v.x + v.y * v.y;
  }
  const double t = block_sum<NT>(nn, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}
__global__ void k_to32(int n, const double2 *__restrict__ a, float2 *__restrict__ b) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    b[i] = make_float2((float)a[i].x, (float)a[i].y);
}
// sum conj(a) b, partials
template <int NT>
__global__ void __launch_bounds__(NT)
  k_dot64(int n, const double2 *__restrict__ a, const double2 *__restrict__ b, double *part) {
  __shared__ double sh[NT / 32];
  double dr = 0., di = 0.;
  for (int i = blockIdx.x * NT + threadIdx.x; i < n; i += gridDim.x * NT) {
    const double2 d = cmc(a[i], b[i]);
    dr += d.x;
    di += d.y;
  }
  double t = block_sum<NT>(dr, sh);
  if (threadIdx.x == 0) part[2 * blockIdx.x] = t;
  t = block_sum<NT>(di, sh);
  if (threadIdx.x == 0) part[2 * blockIdx.x + 1] = t;
}

}  // namespace

// ===================================================================================
cudaError_t u1_phases(const Geom &g, const double *theta, double2 *ph, cudaStream_t s) {
  const size_t NL = (size_t)g.V * g.nd;
  k_phases<<<(int)((NL + 255) / 256), 256, 0, s>>>(NL, theta, ph);
  return cudaGetLastError();
}
cudaError_t u1_phases_f32(const Geom &g, const double *theta, float2 *ph, cudaStream_t s) {
  const size_t NL = (size_t)g.V * g.nd;
  k_phases32<<<(int)((NL + 255) / 256), 256, 0, s>>>(NL, theta, ph);
  return cudaGetLastError();
}

constexpr int NT_H = 128;
static dim3 hop_grid(const Geom &g) { return dim3((g.Vh + NT_H - 1) / NT_H, 2); }
int hop_blocks(const Geom &g) {
  const dim3 d = hop_grid(g);
  return d.x * d.y;
}

cudaError_t staggered_D(const Geom &g, const double2 *ph, double m, int dag, const double2 *in,
                        double2 *out, cudaStream_t s) {
  k_hop<double, NT_H><<<hop_grid(g), NT_H, 0, s>>>(g, ph, m, dag ? -1.0 : 1.0, in, out, nullptr,
                                                   nullptr, nullptr, nullptr, 0);
  return cudaGetLastError();
}
cudaError_t staggered_D(const Geom &g, const float2 *ph, float m, int dag, const float2 *in,
                        float2 *out, cudaStream_t s) {
  k_hop<float, NT_H><<<hop_grid(g), NT_H, 0, s>>>(g, ph, m, dag ? -1.f : 1.f, in, out, nullptr,
                                                  nullptr, nullptr, nullptr, 0);
  return cudaGetLastError();
}
cudaError_t hop64(const Geom &g, const double2 *ph, double m, int dag, const double2 *in,
                  double2 *out, const double2 *a, double *dpart, double *npart,
                  const SolverState *st, int gate_update, cudaStream_t s) {
  k_hop<double, NT_H><<<hop_grid(g), NT_H, 0, s>>>(g, ph, m, dag ? -1.0 : 1.0, in, out, a,
                                                   dpart, npart, st, gate_update);
  return cudaGetLastError();
}
cudaError_t hop32(const Geom &g, const float2 *ph, float m, int dag, const float2 *in,
                  float2 *out, const float2 *a, double *dpart, double *npart,
                  const SolverState *st, cudaStream_t s) {
  k_hop<float, NT_H><<<hop_grid(g), NT_H, 0, s>>>(g, ph, m, dag ? -1.f : 1.f, in, out, a, dpart,
                                                  npart, st, 0);
  return cudaGetLastError();
}

cudaError_t fermion_force(const Geom &g, const double2 *ph, const double2 *chi,
                          const double2 *chi1, double *deriv, cudaStream_t s) {
  const dim3 grid((g.Vh + 127) / 128, 2 * g.nd);
  k_fforce<<<grid, 128, 0, s>>>(g, ph, chi, chi1, deriv);
  return cudaGetLastError();
}
cudaError_t pf_source(const Geom &g, uint64_t seed, uint32_t traj, int complex_source,
                      double2 *R, cudaStream_t s) {
  k_pf_source<<<(g.V + 255) / 256, 256, 0, s>>>(g, seed, traj, complex_source, R);
  return cudaGetLastError();
}

constexpr int NT_V = 256;
int vec_blocks(int n) {
  const int b = (n + NT_V - 1) / NT_V;
  return b < 1184 ? b : 1184;  // 148 SMs x 8
}

cudaError_t cg_alpha(const double *part, int n, SolverState *st, cudaStream_t s) {
  k_cg_alpha<512><<<1, 512, 0, s>>>(part, n, st);
  return cudaGetLastError();
}
cudaError_t cg_xr(int n, double2 *x, double2 *r, const double2 *p, const double2 *Ap,
                  const SolverState *st, double *part, cudaStream_t s) {
  k_cg_xr<NT_V><<<vec_blocks(n), NT_V, 0, s>>>(n, x, r, p, Ap, st, part);
  return cudaGetLastError();
}
cudaError_t cg_beta(const double *part, int n, SolverState *st, cudaStream_t s) {
  k_cg_beta<512><<<1, 512, 0, s>>>(part, n, st);
  return cudaGetLastError();
}
cudaError_t cg_p(int n, const double2 *r, double2 *p, const SolverState *st, cudaStream_t s) {
  k_cg_p<<<vec_blocks(n), NT_V, 0, s>>>(n, r, p, st);
  return cudaGetLastError();
}
cudaError_t bi_alpha(const double *part, int n, SolverState *st, cudaStream_t s) {
  k_bi_alpha<512><<<1, 512, 0, s>>>(part, n, st);
  return cudaGetLastError();
}
cudaError_t bi_s(int n, const double2 *r, const double2 *Ap, double2 *sv, const SolverState *st,
                 cudaStream_t s) {
  k_bi_s<<<vec_blocks(n), NT_V, 0, s>>>(n, r, Ap, sv, st);
  return cudaGetLastError();
}
cudaError_t bi_omega(const double *dpart, const double *npart, int n, SolverState *st,
                     cudaStream_t s) {
  k_bi_omega<512><<<1, 512, 0, s>>>(dpart, npart, n, st);
  return cudaGetLastError();
}
cudaError_t bi_rx(int n, double2 *x, double2 *r, const double2 *sv, const double2 *t,
                  const double2 *p, const double2 *r0, const SolverState *st, double *dpart,
                  double *npart, cudaStream_t s) {
  k_bi_rx<NT_V><<<vec_blocks(n), NT_V, 0, s>>>(n, x, r, sv, t, p, r0, st, dpart, npart);
  return cudaGetLastError();
}
cudaError_t bi_beta(const double *dpart, const double *npart, int n, SolverState *st,
                    cudaStream_t s) {
  k_bi_beta<512><<<1, 512, 0, s>>>(dpart, npart, n, st);
  return cudaGetLastError();
}
cudaError_t bi_p(int n, const double2 *r, double2 *p, const double2 *Ap, const SolverState *st,
                 cudaStream_t s) {
  k_bi_p<<<vec_blocks(n), NT_V, 0, s>>>(n, r, p, Ap, st);
  return cudaGetLastError();
}
cudaError_t m_xr(int n, float2 *xs, float2 *rs, const float2 *ps, const float2 *Aps,
                 const SolverState *st, double *part, cudaStream_t s) {
  k_m_xr<NT_V><<<vec_blocks(n), NT_V, 0, s>>>(n, xs, rs, ps, Aps, st, part);
  return cudaGetLastError();
}
cudaError_t m_check(const double *part, int n, SolverState *st, cudaStream_t s) {
  k_m_check<512><<<1, 512, 0, s>>>(part, n, st);
  return cudaGetLastError();
}
cudaError_t m_accum(int n, double2 *x, float2 *xs, const SolverState *st, cudaStream_t s) {
  k_m_accum<<<vec_blocks(n), NT_V, 0, s>>>(n, x, xs, st);
  return cudaGetLastError();
}
cudaError_t m_resid(int n, const double2 *b, const double2 *Ax, double2 *r, float2 *rs,
                    const SolverState *st, double *part, cudaStream_t s) {
  k_m_resid<NT_V><<<vec_blocks(n), NT_V, 0, s>>>(n, b, Ax, r, rs, st, part);
  return cudaGetLastError();
}
cudaError_t m_after(const double *part, int n, SolverState *st, cudaStream_t s) {
  k_m_after<512><<<1, 512, 0, s>>>(part, n, st);
  return cudaGetLastError();
}
cudaError_t m_p(int n, const float2 *rs, float2 *ps, SolverState *st, cudaStream_t s) {
  k_m_p<<<vec_blocks(n), NT_V, 0, s>>>(n, rs, ps, st);
  k_m_commit<<<1, 1, 0, s>>>(st);
  return cudaGetLastError();
}

cudaError_t resid64(int n, const double2 *b, const double2 *Ax, double2 *r, double *part,
                    cudaStream_t s) {
  k_resid64<NT_V><<<vec_blocks(n), NT_V, 0, s>>>(n, b, Ax, r, part);
  return cudaGetLastError();
}
cudaError_t to32(int n, const double2 *a, float2 *b, cudaStream_t s) {
  k_to32<<<vec_blocks(n), NT_V, 0, s>>>(n, a, b);
  return cudaGetLastError();
}
cudaError_t dot64(int n, const double2 *a, const double2 *b, double *part, cudaStream_t s) {
  k_dot64<NT_V><<<vec_blocks(n), NT_V, 0, s>>>(n, a, b, part);
  return cudaGetLastError();
}

// One block per SM on the current device when it supports cooperative launches and one
// block of `nt` threads of `kern` fits an SM, else 0.  Computed once per device and kernel:
// slots[dev] holds the grid + 1 (0: not yet known).
constexpr int COOP_MAX_DEVICES = 64;
static int coop_blocks(const void *kern, int nt, int *slots) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= COOP_MAX_DEVICES) return 0;
  if (slots[dev] == 0) {
    int coop = 0, sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, nt, 0);
    slots[dev] = 1 + ((coop && per_sm >= 1) ? sms : 0);
  }
  return slots[dev] - 1;
}

// the persistent CG: one cooperative launch until convergence or the iteration limit;
// returns cudaErrorNotSupported where cooperative launches are unavailable (the caller then
// queues the per-phase kernels) and cudaErrorTimeout when a barrier wait gave up
cudaError_t cg_persistent(const Geom &g, const double2 *ph, double m, double2 *x, double2 *r,
                          double2 *p, double2 *t, double *part, SolverState *st, void *bar_mem,
                          int part_cap, cudaStream_t s) {
  // one block of 512 threads per SM: the fewer blocks arrive at a barrier, the shorter it is
  constexpr int NT = 512;
  static int slots[COOP_MAX_DEVICES];
  const int grid = coop_blocks((const void *)k_cg_persistent<NT>, NT, slots);
  const int G = std::min(grid, std::max(1, (g.V + NT - 1) / NT));
  if (G <= 0 || 2 * G > part_cap || G > 32 * FIXED_SUM_PER_LANE) return cudaErrorNotSupported;
  GridBarrier *bar = (GridBarrier *)bar_mem;
  cudaError_t e = cudaMemsetAsync(bar, 0, sizeof(GridBarrier), s);
  if (e != cudaSuccess) return e;
  double *part_t = part, *part_r = part + G;
  Geom gg = g;
  double mm = m;
  void *args[] = {&gg, (void *)&ph, &mm, &x, &r, &p, &t, &part_t, &part_r, &st, &bar};
  e = cudaLaunchCooperativeKernel((const void *)k_cg_persistent<NT>, dim3(G), dim3(NT), args, 0,
                                  s);
  if (e == cudaErrorCooperativeLaunchTooLarge) {  // fewer SMs available (shared GPU): queue
    cudaGetLastError();                           // the per-phase kernels instead
    return cudaErrorNotSupported;
  }
  return e;
}

// the persistent mixed-precision CG (k_cg_mixed_persistent); the same launch rules as
// cg_persistent
cudaError_t cg_mixed_persistent(const Geom &g, const double2 *ph, const float2 *ph32, double m,
                                const double2 *b, double2 *x, double2 *r, double2 *t64,
                                float2 *xs, float2 *rs, float2 *ps, float2 *ts, double *part,
                                SolverState *st, void *bar_mem, int part_cap, cudaStream_t s) {
  constexpr int NT = 512;
  static int slots[COOP_MAX_DEVICES];
  const int grid = coop_blocks((const void *)k_cg_mixed_persistent<NT>, NT, slots);
  const int G = std::min(grid, std::max(1, (g.V + NT - 1) / NT));
  if (G <= 0 || 2 * G > part_cap || G > 32 * FIXED_SUM_PER_LANE) return cudaErrorNotSupported;
  GridBarrier *bar = (GridBarrier *)bar_mem;
  cudaError_t e = cudaMemsetAsync(bar, 0, sizeof(GridBarrier), s);
  if (e != cudaSuccess) return e;
  double *part_t = part, *part_r = part + G;
  Geom gg = g;
  double mm = m;
  void *args[] = {&gg, (void *)&ph, (void *)&ph32, &mm, (void *)&b, &x, &r, &t64,
                  &xs, &rs, &ps, &ts, &part_t, &part_r, &st, &bar};
  e = cudaLaunchCooperativeKernel((const void *)k_cg_mixed_persistent<NT>, dim3(G), dim3(NT),
                                  args, 0, s);
  if (e == cudaErrorCooperativeLaunchTooLarge) {
    cudaGetLastError();
    return cudaErrorNotSupported;
  }
  return e;
}

// the persistent BiCGStab (k_bicgstab_persistent); the same launch rules as cg_persistent.
// p holds the start direction; p2 and Ap2 are the second buffers of p and Ap.
cudaError_t bicgstab_persistent(const Geom &g, const double2 *ph, double m, double2 *x,
                                double2 *r, const double2 *r0, double2 *p, double2 *p2,
                                double2 *Ap, double2 *Ap2, double2 *sv, double2 *t,
                                double *part, SolverState *st, void *bar_mem, int part_cap,
                                cudaStream_t s) {
  constexpr int NT = 512;
  static int slots[COOP_MAX_DEVICES];
  const int grid = coop_blocks((const void *)k_bicgstab_persistent<NT>, NT, slots);
  const int G = std::min(grid, std::max(1, (g.V + NT - 1) / NT));
  if (G <= 0 || 8 * G > part_cap || G > 32 * FIXED_SUM_PER_LANE) return cudaErrorNotSupported;
  GridBarrier *bar = (GridBarrier *)bar_mem;
  cudaError_t e = cudaMemsetAsync(bar, 0, sizeof(GridBarrier), s);
  if (e != cudaSuccess) return e;
  Geom gg = g;
  double mm = m;
  void *args[] = {&gg, (void *)&ph, &mm, &x, &r, (void *)&r0, &p, &p2, &Ap, &Ap2,
                  &sv, &t, &part, &st, &bar};
  e = cudaLaunchCooperativeKernel((const void *)k_bicgstab_persistent<NT>, dim3(G), dim3(NT),
                                  args, 0, s);
  if (e == cudaErrorCooperativeLaunchTooLarge) {
    cudaGetLastError();
    return cudaErrorNotSupported;
  }
  return e;
}

int cg_barrier_failed(const void *bar_mem, cudaStream_t s, int *failed) {
  GridBarrier h{};
  if (cudaMemcpyAsync(&h, bar_mem, sizeof h, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return 1;
  *failed = h.err;
  return 0;
}
size_t cg_barrier_bytes() { return sizeof(GridBarrier); }

cudaError_t pion_slices(const Geom &g, const double2 *S, double *C, cudaStream_t s) {
  k_pion_slices<256><<<g.L[0], 256, 0, s>>>(g, S, C);
  return cudaGetLastError();
}

}  // namespace su2b
