// pairs.cu -- the FP32 force step on site pairs in packed FP32 (FFMA2), d = 4.
//
// Each site x of the lower half of the lattice in t (t < T/2) is paired with its partner
// x + (T/2) t^, the site half the lattice away.  The pair's links are stored component by
// component side by side (the "paired layout"): for direction mu, parity p and pair index
// q = the lower site's even/odd index (0 <= q < Vh/2), 32 bytes
//   {ar_lo, ar_hi, ai_lo, ai_hi, br_lo, br_hi, bi_lo, bi_hi}
// at ((mu * 2 + p) * Vh/2 + q) * 32.  The partner map is a translation, so the neighbour of
// a pair in any direction is again a pair: one 32-byte load brings the same link of both
// sites, each component already as the two lanes of a float2.  A neighbour across the
// half-lattice boundary in t belongs to the upper half; its pair then arrives with the
// lanes exchanged (warp-uniform: a warp covers one t).  T/2 is even, so a site and its
// partner have the same parity.
//
// One thread per link of a site pair (warp mu of a block, 32 consecutive pairs of one
// parity): the six staples of link mu at both sites, then the link's tail (force, momentum
// step, the next gauge step or the closing restoreSU) -- the arithmetic of the one-thread-
// per-link kernel (force_link_impl) with every FP32 operation issued as a packed FFMA2 /
// FMUL2 / FADD2 on the pair.  Each lane runs the same sequence of correctly rounded
// operations as the scalar code, so both sites get bit for bit the links and momenta that
// the one-thread-per-link kernel gives them.  The momenta stay in the standard layout.
//
// Within a trajectory only: the start field is copied into the paired layout once
// (to_pairs), the force launches read and write paired buffers, and the last launch writes
// the reunitarised final field in the standard layout.
#include "su2b_internal.h"

namespace su2b {
namespace {

struct Q2 {  // one SU(2) element at both sites of a pair
  float2 ar, ai, br, bi;
};

__device__ __forceinline__ float2 neg(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 fm2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }

// mul, mul_acc, dag of su2b_common.cuh, operation for operation
__device__ __forceinline__ Q2 qmul(const Q2 &u, const Q2 &v) {
  Q2 r;
  r.ar = fm2(u.ar, v.ar, fm2(neg(u.ai), v.ai, fm2(neg(u.br), v.br, mul2(neg(u.bi), v.bi))));
  r.ai = fm2(u.ar, v.ai, fm2(u.ai, v.ar, fm2(neg(u.bi), v.br, mul2(u.br, v.bi))));
  r.br = fm2(u.ar, v.br, fm2(neg(u.ai), v.bi, fm2(u.br, v.ar, mul2(u.bi, v.ai))));
  r.bi = fm2(u.ar, v.bi, fm2(u.ai, v.br, fm2(u.bi, v.ar, mul2(neg(u.br), v.ai))));
  return r;
}
__device__ __forceinline__ Q2 qmul_acc(const Q2 &k, const Q2 &u, const Q2 &v) {
  Q2 r;
  r.ar = fm2(u.ar, v.ar, fm2(neg(u.ai), v.ai, fm2(neg(u.br), v.br, fm2(neg(u.bi), v.bi, k.ar))));
  r.ai = fm2(u.ar, v.ai, fm2(u.ai, v.ar, fm2(neg(u.bi), v.br, fm2(u.br, v.bi, k.ai))));
  r.br = fm2(u.ar, v.br, fm2(neg(u.ai), v.bi, fm2(u.br, v.ar, fm2(u.bi, v.ai, k.br))));
  r.bi = fm2(u.ar, v.bi, fm2(u.ai, v.br, fm2(u.bi, v.ar, fm2(neg(u.br), v.ai, k.bi))));
  return r;
}
__device__ __forceinline__ Q2 qdag(const Q2 &u) { return Q2{u.ar, neg(u.ai), neg(u.br), neg(u.bi)}; }


template <bool SWAPPED>
__device__ __forceinline__ Q2 ld_pair(const float4 *__restrict__ Upl, size_t at) {
  const float4 a = __ldg(Upl + 2 * at), b = __ldg(Upl + 2 * at + 1);
  if (SWAPPED)
    return Q2{make_float2(a.y, a.x), make_float2(a.w, a.z), make_float2(b.y, b.x),
              make_float2(b.w, b.z)};
  return Q2{make_float2(a.x, a.y), make_float2(a.z, a.w), make_float2(b.x, b.y),
            make_float2(b.z, b.w)};
}
__device__ __forceinline__ void st_pair(float4 *__restrict__ Upl, size_t at, const Q2 &u) {
  Upl[2 * at] = make_float4(u.ar.x, u.ar.y, u.ai.x, u.ai.y);
  Upl[2 * at + 1] = make_float4(u.br.x, u.br.y, u.bi.x, u.bi.y);
}
__device__ __forceinline__ Su2<float> lane(const Q2 &u, int hi) {
  return hi ? Su2<float>{u.ar.y, u.ai.y, u.br.y, u.bi.y}
            : Su2<float>{u.ar.x, u.ai.x, u.br.x, u.bi.x};
}

// exp_alg (su2b_common.cuh) of both lanes: the Taylor series in packed arithmetic when both
// arguments are small (every molecular-dynamics step in practice), else lane by lane
__device__ __forceinline__ Q2 qexp(float2 a, float2 b, float2 c) {
  const float2 t2 = fm2(a, a, fm2(b, b, mul2(c, c)));
  if (t2.x <= 0.25f && t2.y <= 0.25f) {
    float2 co = make_float2((float)detail::Coef<4>::c, (float)detail::Coef<4>::c);
    float2 f = make_float2((float)detail::Coef<4>::s, (float)detail::Coef<4>::s);
#define SU2B_HORNER(k)                                                                        \
  co = fm2(co, t2, make_float2((float)detail::Coef<k>::c, (float)detail::Coef<k>::c));      \
  f = fm2(f, t2, make_float2((float)detail::Coef<k>::s, (float)detail::Coef<k>::s))
    SU2B_HORNER(3);
    SU2B_HORNER(2);
    SU2B_HORNER(1);
    SU2B_HORNER(0);
#undef SU2B_HORNER
    return Q2{co, mul2(f, c), mul2(f, b), mul2(f, a)};
  }
  const Su2<float> lo = exp_alg(a.x, b.x, c.x), hi = exp_alg(a.y, b.y, c.y);
  return Q2{make_float2(lo.ar, hi.ar), make_float2(lo.ai, hi.ai), make_float2(lo.br, hi.br),
            make_float2(lo.bi, hi.bi)};
}

// the standard layout into the paired one: thread = (mu, parity, pair)
__global__ void __launch_bounds__(256) k_to_pairs(Geom g, const float4 *__restrict__ U,
                                                  float4 *__restrict__ Upl) {
  const long Vh2 = g.Vh / 2, n = 8 * Vh2;
  for (long i = blockIdx.x * 256l + threadIdx.x; i < n; i += (long)gridDim.x * 256) {
    const long mp = i / Vh2, q = i - mp * Vh2;  // mp = mu * 2 + p
    const size_t lo = (size_t)(mp >> 1) * g.V + (size_t)(mp & 1) * g.Vh + q;
    const float4 a = __ldg(U + lo), b = __ldg(U + lo + Vh2);
    Upl[2 * i] = make_float4(a.x, b.x, a.y, b.y);
    Upl[2 * i + 1] = make_float4(a.z, b.z, a.w, b.w);
  }
}

__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// the fused force step on site pairs: warp mu of block b takes link mu of the 32 pairs
// (b >> 1) * 32 .. of parity b & 1.  TB: the pair's lower site sits next to the half-lattice
// boundary in t, where its t neighbours belong to the upper half and their pairs arrive with
// the lanes exchanged: +1 at t = T/2 - 1 (forward t neighbours), -1 at t = 0 (backward), 0
// elsewhere.  A warp covers one t, so the three forms are warp-uniform code paths.
template <int mu, int TB>
__device__ __forceinline__ double pair_link(const Geom &g, const Site &s,
                                            const float4 *__restrict__ Upl,
                                            float *__restrict__ P, float f, float scale_,
                                            int mode, void *__restrict__ Uout, float dt_upd,
                                            int p, int q) {
  const int Vh2 = g.Vh / 2;
  int fo[4], bo[4];
#pragma unroll
  for (int d = 0; d < 4; d++) {
    fo[d] = fwd(g, s, d);
    bo[d] = bwd(g, s, d);
  }
  // link nu of the pair displaced by o (components in {-1, 0, 1})
  auto L = [&](int nu, int o0, int o1, int o2, int o3) -> Q2 {
    const int o[4] = {o0, o1, o2, o3};
    int lex = s.lex, odd = 0;
#pragma unroll
    for (int d = 0; d < 4; d++) {
      if (o[d] > 0) lex += fo[d];
      if (o[d] < 0) lex += bo[d];
      odd ^= (o[d] != 0);
    }
    int qn = lex >> 1;
    const size_t mp = (size_t)(nu * 2 + (p ^ odd)) * Vh2;
    if ((TB > 0 && o0 > 0) || (TB < 0 && o0 < 0))  // across t = T/2: the lanes swapped
      return ld_pair<true>(Upl, mp + qn - Vh2);
    return ld_pair<false>(Upl, mp + qn);
  };
  auto E = [](int d, int k) { return d == k ? 1 : 0; };
  Q2 K{make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f),
       make_float2(0.f, 0.f)};
#pragma unroll
  for (int nu = 0; nu < 4; nu++) {
    if (nu == mu) continue;
    const Q2 a = L(nu, E(mu, 0), E(mu, 1), E(mu, 2), E(mu, 3));  // U_nu(x+mu)
    const Q2 b = L(mu, E(nu, 0), E(nu, 1), E(nu, 2), E(nu, 3));  // U_mu(x+nu)
    const Q2 c = L(nu, 0, 0, 0, 0);                              // U_nu(x)
    K = qmul_acc(K, qmul(a, qdag(b)), qdag(c));
    const Q2 e = L(nu, E(mu, 0) - E(nu, 0), E(mu, 1) - E(nu, 1), E(mu, 2) - E(nu, 2),
                   E(mu, 3) - E(nu, 3));                                 // U_nu(x+mu-nu)
    const Q2 h = L(mu, -E(nu, 0), -E(nu, 1), -E(nu, 2), -E(nu, 3));  // U_mu(x-nu)
    const Q2 d = L(nu, -E(nu, 0), -E(nu, 1), -E(nu, 2), -E(nu, 3));  // U_nu(x-nu)
    K = qmul_acc(K, qmul(qdag(e), qdag(h)), d);
  }
  // the link's tail (finish_link of site_ops.cuh, operation for operation)
  const Q2 u = L(mu, 0, 0, 0, 0);
  const Q2 &k = K;
  const float2 sbi = fm2(u.ar, k.bi, fm2(u.ai, k.br, fm2(u.bi, k.ar, mul2(neg(u.br), k.ai))));
  const float2 sbr = fm2(u.ar, k.br, fm2(neg(u.ai), k.bi, fm2(u.br, k.ar, mul2(u.bi, k.ai))));
  const float2 sai = fm2(u.ar, k.ai, fm2(u.ai, k.ar, fm2(neg(u.bi), k.br, mul2(u.br, k.bi))));
  const float f2s = 2.0f * f;
  const float2 f2 = make_float2(f2s, f2s), sc = make_float2(scale_, scale_);
  const float2 d0 = mul2(f2, sbi), d1 = mul2(f2, sbr), d2 = mul2(f2, sai);
  const size_t NL = 4 * (size_t)g.V;
  const size_t l = (size_t)mu * g.V + (size_t)p * g.Vh + q, l2 = l + Vh2;
  float2 p0 = make_float2(0.f, 0.f), p1 = p0, p2 = p0;
  if (mode & FM_HAS_IN) {
    p0 = make_float2(P[l], P[l2]);
    p1 = make_float2(P[NL + l], P[NL + l2]);
    p2 = make_float2(P[2 * NL + l], P[2 * NL + l2]);
  }
  p0 = fm2(sc, d0, p0);
  p1 = fm2(sc, d1, p1);
  p2 = fm2(sc, d2, p2);
  P[l] = p0.x;
  P[l2] = p0.y;
  P[NL + l] = p1.x;
  P[NL + l2] = p1.y;
  P[2 * NL + l] = p2.x;
  P[2 * NL + l2] = p2.y;
  if (mode & FM_UPDATE) {
    const float2 dt = make_float2(dt_upd, dt_upd);
    st_pair((float4 *)Uout, (size_t)(mu * 2 + p) * Vh2 + q,
            qmul(qexp(mul2(dt, p0), mul2(dt, p1), mul2(dt, p2)), u));
  } else if (mode & FM_RESTORE) {  // the final field, in the standard layout
    float4 *out = (float4 *)Uout;
    const Su2<float> lo = from64<float>(restore_su(to64(lane(u, 0))));
    const Su2<float> hi = from64<float>(restore_su(to64(lane(u, 1))));
    out[l] = make_float4(lo.ar, lo.ai, lo.br, lo.bi);
    out[l2] = make_float4(hi.ar, hi.ai, hi.br, hi.bi);
  }
  if (!(mode & FM_KINETIC)) return 0.;
  return ((double)p0.x * p0.x + (double)p1.x * p1.x + (double)p2.x * p2.x) +
         ((double)p0.y * p0.y + (double)p1.y * p1.y + (double)p2.y * p2.y);
}

template <int MINB>
__global__ void __launch_bounds__(128, MINB)
  k_force_su2_pair(Geom g, const float4 *__restrict__ Upl, float *__restrict__ P, float f,
                   float scale_, int mode, double *kin_part, void *__restrict__ Uout,
                   float dt_upd) {
  __shared__ double sh[4];
  pdl_trigger();
  pdl_wait();
  const int w = threadIdx.x >> 5, p = blockIdx.x & 1;
  const int q = (blockIdx.x >> 1) * 32 + (threadIdx.x & 31);
  double k2 = 0.;
  if (q < g.Vh / 2) {
    const Site s = site_from_eo(g, p, q);
    const int tb = s.c[0] == g.L[0] / 2 - 1 ? 1 : (s.c[0] == 0 ? -1 : 0);
#define SU2B_PAIR_LINK(M, TB) k2 = pair_link<M, TB>(g, s, Upl, P, f, scale_, mode, Uout, dt_upd, p, q)
#define SU2B_PAIR_DIR(M)            \
  if (tb == 0)                      \
    SU2B_PAIR_LINK(M, 0);           \
  else if (tb > 0)                  \
    SU2B_PAIR_LINK(M, 1);           \
  else                              \
    SU2B_PAIR_LINK(M, -1)
    switch (w) {
      case 0: SU2B_PAIR_DIR(0); break;
      case 1: SU2B_PAIR_DIR(1); break;
      case 2: SU2B_PAIR_DIR(2); break;
      default: SU2B_PAIR_DIR(3); break;
    }
#undef SU2B_PAIR_DIR
#undef SU2B_PAIR_LINK
  }
  if (mode & FM_KINETIC) {
    const double r = block_sum<128>(k2, sh);
    if (threadIdx.x == 0) kin_part[blockIdx.x] = r;
  }
}

}  // namespace

bool pairs_apply(const Geom &g) {
  return g.nd == 4 && g.L[0] % 4 == 0 && g.cb0 == 0 && g.ncb == g.Vh;
}

cudaError_t to_pairs(const Geom &g, const void *U, void *Upl, cudaStream_t s) {
  const long n = 8l * (g.Vh / 2);
  const long blocks = (n + 255) / 256;
  k_to_pairs<<<(unsigned)(blocks < 148 * 16 ? blocks : 148 * 16), 256, 0, s>>>(
    g, (const float4 *)U, (float4 *)Upl);
  return cudaGetLastError();
}

cudaError_t force_pair(const Geom &g, const void *Upl, float *P, double f, double scale, int mode,
                       double *kin_part, int *nblocks, void *Uout, double dt_upd, cudaStream_t s,
                       bool pdl) {
  const dim3 grid(2 * ((g.Vh / 2 + 31) / 32));
  if (nblocks) *nblocks = grid.x;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = dim3(128);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, k_force_su2_pair<PAIR_MINB>, g, (const float4 *)Upl, P,
                            (float)f, (float)scale, mode, kin_part, Uout, (float)dt_upd);
}

}  // namespace su2b
