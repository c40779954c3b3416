// su2b_common.cuh -- device-side building blocks shared by every kernel of libsu2b.
//
// Data layout in HBM (one lattice):
//   site order  : even/odd.  eo(x) = parity(x)*V/2 + lex(x)/2 where
//                 lex(x) = ((t*Lx + x)*Ly + y)*Lz + z is the reference's site order
//                 (gaugeconfig.hh:211-222) and parity(x) = (t+x+y+z) mod 2.
//   links       : U[mu*V + eo(x)]; SU(2) as 4 reals {Re a, Im a, Re b, Im b}
//                 (su2.hh:11-70, U = [[a, b], [-b*, a*]]): 32 B (FP64) or 16 B (FP32);
//                 U(1) as one angle (u1.hh:58).
//   adjoint     : structure of arrays P_k[mu*V + eo(x)], k = 0..2 for SU(2)
//                 (adjointsu2 {a, b, c}, adjointfield.hh:12-51), k = 0 for U(1).
//   spinors     : complex per site in eo order (staggered, U(1) only).
// All active extents must be even so that the pair {2k, 2k+1} of lexicographic sites has
// opposite parities and the checkerboard is consistent across the periodic boundary.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace su2b {

// ------------------------------------------------------------------------------------
// integer division by a runtime constant, valid for numerators below 2^31:
// q = umulhi(n, m) >> s with m = ceil(2^(31+l)/d), l = ceil(log2 d), s = l - 1.
struct FastDiv {
  uint32_t d, m, s;
};

inline FastDiv make_fastdiv(uint32_t d) {
  FastDiv f{d, 0u, 0u};
  if (d <= 1) return f;
  uint32_t l = 0;
  while ((1ull << l) < d) l++;
  const unsigned __int128 num = (unsigned __int128)1 << (31 + l);
  f.m = (uint32_t)((num + d - 1) / d);
  f.s = l - 1;
  return f;
}

__device__ __forceinline__ uint32_t fdiv(uint32_t n, const FastDiv &f) {
  return f.m ? (__umulhi(n, f.m) >> f.s) : n;
}

// ------------------------------------------------------------------------------------
struct Geom {
  int nd;       // number of active directions (2..4)
  int L[4];     // extents by direction: 0 = t, 1 = x, 2 = y, 3 = z (1 if inactive)
  int st[4];    // lexicographic stride of each direction (st[3] = 1)
  int V, Vh;    // volume, half volume
  FastDiv dv[4];
  // The sites the trajectory kernels (force, plaquettes, momenta) cover: even/odd indices
  // cb0 .. cb0 + ncb - 1 of each parity.  0 and Vh for a whole lattice; for a time slab with
  // one ghost slice on each side, the slab's own slices.
  int cb0, ncb;
  // index in the whole lattice of the local site with lexicographic index 0 (the slab's
  // first ghost slice; may be negative), added to a site's index for its Philox stream
  int lex0;
};

// a site held in registers: coordinates, lexicographic index and parity
struct Site {
  int c[4];
  int lex;
  int p;
};

__device__ __forceinline__ Site site_from_eo(const Geom &g, int p, int cb) {
  Site s;
  const uint32_t lex0 = 2u * (uint32_t)cb;
  uint32_t q = lex0;
#pragma unroll
  for (int k = 3; k >= 1; k--) {
    const uint32_t qq = fdiv(q, g.dv[k]);
    s.c[k] = (int)(q - qq * (uint32_t)g.L[k]);
    q = qq;
  }
  s.c[0] = (int)q;
  s.lex = (int)lex0;
  if (((s.c[0] + s.c[1] + s.c[2] + s.c[3]) & 1) != p) {
    s.c[g.nd - 1] += 1;  // fastest active direction, stride 1, even extent
    s.lex += 1;
  }
  s.p = p;
  return s;
}

__device__ __forceinline__ Site site_from_lex(const Geom &g, int lex) {
  Site s;
  uint32_t q = (uint32_t)lex;
#pragma unroll
  for (int k = 3; k >= 1; k--) {
    const uint32_t qq = fdiv(q, g.dv[k]);
    s.c[k] = (int)(q - qq * (uint32_t)g.L[k]);
    q = qq;
  }
  s.c[0] = (int)q;
  s.lex = lex;
  s.p = (s.c[0] + s.c[1] + s.c[2] + s.c[3]) & 1;
  return s;
}

// lexicographic offset of the forward / backward neighbour in direction mu (periodic)
__device__ __forceinline__ int fwd(const Geom &g, const Site &s, int mu) {
  return s.c[mu] == g.L[mu] - 1 ? -(g.L[mu] - 1) * g.st[mu] : g.st[mu];
}
__device__ __forceinline__ int bwd(const Geom &g, const Site &s, int mu) {
  return s.c[mu] == 0 ? (g.L[mu] - 1) * g.st[mu] : -g.st[mu];
}
// The same for a direction known only at run time.  Selecting among the four entries keeps
// every array index constant; indexing the site's coordinates or the geometry by a variable
// would place both in local memory.
__device__ __forceinline__ int pick4(int k, int a0, int a1, int a2, int a3) {
  return k == 0 ? a0 : k == 1 ? a1 : k == 2 ? a2 : a3;
}
__device__ __forceinline__ int coord_rt(const Site &s, int mu) {
  return pick4(mu, s.c[0], s.c[1], s.c[2], s.c[3]);
}
__device__ __forceinline__ int fwd_rt(const Geom &g, const Site &s, int mu) {
  const int L = pick4(mu, g.L[0], g.L[1], g.L[2], g.L[3]);
  const int st = pick4(mu, g.st[0], g.st[1], g.st[2], g.st[3]);
  return coord_rt(s, mu) == L - 1 ? -(L - 1) * st : st;
}
__device__ __forceinline__ int bwd_rt(const Geom &g, const Site &s, int mu) {
  const int L = pick4(mu, g.L[0], g.L[1], g.L[2], g.L[3]);
  const int st = pick4(mu, g.st[0], g.st[1], g.st[2], g.st[3]);
  return coord_rt(s, mu) == 0 ? (L - 1) * st : -st;
}
// even/odd index of the site with lexicographic index lex and parity p
__device__ __forceinline__ int eo_of(const Geom &g, int lex, int p) {
  return p * g.Vh + (lex >> 1);
}

// ------------------------------------------------------------------------------------
// storage types
struct __align__(32) Link64 {
  double ar, ai, br, bi;
};
typedef float4 Link32;

template <class T> struct LinkOf;
template <> struct LinkOf<double> { typedef Link64 type; };
template <> struct LinkOf<float> { typedef Link32 type; };

template <class T> struct Su2 {
  T ar, ai, br, bi;
};

// The loads carry no side effect, so they are not volatile: the compiler may hoist and
// overlap them.
__device__ __forceinline__ Su2<double> ld_link(const Link64 *p) {
  Su2<double> r;
  asm("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];"
               : "=d"(r.ar), "=d"(r.ai), "=d"(r.br), "=d"(r.bi)
               : "l"(p));
  return r;
}
// coherent load (for kernels that also write the links they read)
__device__ __forceinline__ Su2<double> ld_link_rw(const Link64 *p) {
  Su2<double> r;
  asm volatile("ld.global.v4.f64 {%0,%1,%2,%3}, [%4];"
               : "=d"(r.ar), "=d"(r.ai), "=d"(r.br), "=d"(r.bi)
               : "l"(p)
               : "memory");
  return r;
}
__device__ __forceinline__ void st_link(Link64 *p, const Su2<double> &u) {
  asm volatile("st.global.v4.f64 [%0], {%1,%2,%3,%4};" ::"l"(p), "d"(u.ar), "d"(u.ai),
               "d"(u.br), "d"(u.bi)
               : "memory");
}
// The FP32 load is left to the compiler (__ldg) rather than written as inline PTX: a link it
// can no longer keep in a register it may then load again (an L1 hit) instead of spilling.
__device__ __forceinline__ Su2<float> ld_link(const Link32 *p) {
  const float4 v = __ldg(p);
  return Su2<float>{v.x, v.y, v.z, v.w};
}
__device__ __forceinline__ Su2<float> ld_link_rw(const Link32 *p) {
  const float4 v = *p;
  return Su2<float>{v.x, v.y, v.z, v.w};
}
__device__ __forceinline__ void st_link(Link32 *p, const Su2<float> &u) {
  *p = make_float4(u.ar, u.ai, u.br, u.bi);
}

template <class T> __device__ __forceinline__ Su2<double> to64(const Su2<T> &u) {
  return Su2<double>{(double)u.ar, (double)u.ai, (double)u.br, (double)u.bi};
}
template <class T> __device__ __forceinline__ Su2<T> from64(const Su2<double> &u) {
  return Su2<T>{(T)u.ar, (T)u.ai, (T)u.br, (T)u.bi};
}

// ------------------------------------------------------------------------------------
// SU(2) algebra in the (a, b) form (su2.hh:87-113).  u*v:
//   a = u.a v.a - u.b conj(v.b),  b = u.a v.b + u.b conj(v.a)
// written as chains of fused multiply-adds (one multiply and three FMAs per component; the
// sign flips of dag() fold into the FMA operands).
__device__ __forceinline__ float fm(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double fm(double a, double b, double c) { return fma(a, b, c); }

template <class T> __device__ __forceinline__ Su2<T> mul(const Su2<T> &u, const Su2<T> &v) {
  Su2<T> r;
  r.ar = fm(u.ar, v.ar, fm(-u.ai, v.ai, fm(-u.br, v.br, -u.bi * v.bi)));
  r.ai = fm(u.ar, v.ai, fm(u.ai, v.ar, fm(-u.bi, v.br, u.br * v.bi)));
  r.br = fm(u.ar, v.br, fm(-u.ai, v.bi, fm(u.br, v.ar, u.bi * v.ai)));
  r.bi = fm(u.ar, v.bi, fm(u.ai, v.br, fm(u.bi, v.ar, -u.br * v.ai)));
  return r;
}
// k + u*v, sixteen FMAs
template <class T>
__device__ __forceinline__ Su2<T> mul_acc(const Su2<T> &k, const Su2<T> &u, const Su2<T> &v) {
  Su2<T> r;
  r.ar = fm(u.ar, v.ar, fm(-u.ai, v.ai, fm(-u.br, v.br, fm(-u.bi, v.bi, k.ar))));
  r.ai = fm(u.ar, v.ai, fm(u.ai, v.ar, fm(-u.bi, v.br, fm(u.br, v.bi, k.ai))));
  r.br = fm(u.ar, v.br, fm(-u.ai, v.bi, fm(u.br, v.ar, fm(u.bi, v.ai, k.br))));
  r.bi = fm(u.ar, v.bi, fm(u.ai, v.br, fm(u.bi, v.ar, fm(-u.br, v.ai, k.bi))));
  return r;
}
template <class T> __device__ __forceinline__ Su2<T> dag(const Su2<T> &u) {
  return Su2<T>{u.ar, -u.ai, -u.br, -u.bi};
}
template <class T> __device__ __forceinline__ Su2<T> add(const Su2<T> &u, const Su2<T> &v) {
  return Su2<T>{u.ar + v.ar, u.ai + v.ai, u.br + v.br, u.bi + v.bi};
}
template <class T> __device__ __forceinline__ Su2<T> scale(T s, const Su2<T> &u) {
  return Su2<T>{s * u.ar, s * u.ai, s * u.br, s * u.bi};
}
template <class T> __device__ __forceinline__ T retr(const Su2<T> &u) { return T(2) * u.ar; }
// ReTr(u*v) = 2 Re(u.a v.a - u.b conj(v.b))
template <class T> __device__ __forceinline__ T retr_mul(const Su2<T> &u, const Su2<T> &v) {
  return T(2) * (u.ar * v.ar - u.ai * v.ai - (u.br * v.br + u.bi * v.bi));
}
template <class T> __device__ __forceinline__ Su2<T> zero_su2() { return Su2<T>{0, 0, 0, 0}; }

// restoreSU (su2.hh:62-66), always evaluated in FP64
__device__ __forceinline__ Su2<double> restore_su(const Su2<double> &u) {
  const double r = sqrt(u.ar * u.ar + u.ai * u.ai + u.br * u.br + u.bi * u.bi);
  const double ir = 1.0 / r;
  return Su2<double>{u.ar * ir, u.ai * ir, u.br * ir, u.bi * ir};
}

// exp of an algebra element (exp_gauge.cc:8-18): alpha = |x|, n = x/alpha,
// exp = (cos alpha + i sin(alpha) n2, sin(alpha) (n1 + i n0)).  Both cos(alpha) and
// sin(alpha)/alpha are even functions of alpha, so for alpha^2 <= 1/4 (every molecular-dynamics
// and flow step in practice) they are summed directly as their Taylor series in alpha^2,
// Horner form, with no square root, division or argument reduction:
//   cos a = sum_k (-1)^k a^2k/(2k)!,   sin(a)/a = sum_k (-1)^k a^2k/(2k+1)!.
// FP64 keeps k <= 7 (first omitted terms below 1e-18), FP32 k <= 4 (below 3e-10).  Larger
// arguments take the square root and sincos.  At alpha = 0 the reference divides 0/0; here
// the limit (the identity) is returned.  The large-argument branch evaluates sincospi(alpha/pi):
// the pi-scaled reduction is exact, whereas sincos keeps a local array for its slow
// reduction path, whose stack frame costs every thread local-memory traffic even when the
// branch is never taken.
namespace detail {
// n! is exact in double for n <= 18, so (+-1)/n! below is the correctly rounded coefficient
__host__ __device__ constexpr double fact(int n) { return n <= 1 ? 1.0 : n * fact(n - 1); }
template <int k> struct Coef {
  static constexpr double c = ((k & 1) ? -1.0 : 1.0) / fact(2 * k);      // cos
  static constexpr double s = ((k & 1) ? -1.0 : 1.0) / fact(2 * k + 1);  // sin(x)/x
};
template <class T, int k> struct Horner {
  static __device__ __forceinline__ void run(T t2, T &c, T &s) {
    c = fm(c, t2, T(Coef<k>::c));
    s = fm(s, t2, T(Coef<k>::s));
    Horner<T, k - 1>::run(t2, c, s);
  }
};
template <class T> struct Horner<T, -1> {
  static __device__ __forceinline__ void run(T, T &, T &) {}
};
template <class T, int K>
__device__ __forceinline__ void cos_sinc_series(T t2, T &co, T &sc) {
  co = T(Coef<K>::c);
  sc = T(Coef<K>::s);
  Horner<T, K - 1>::run(t2, co, sc);
}
}  // namespace detail

__device__ __forceinline__ Su2<double> exp_alg(double a, double b, double c) {
  const double t2 = fma(a, a, fma(b, b, c * c));
  double co, f;
  if (t2 <= 0.25) {
    detail::cos_sinc_series<double, 7>(t2, co, f);
  } else {
    const double alpha = sqrt(t2);
    double s;
    sincospi(alpha * 0.318309886183790671537767526745, &s, &co);
    f = s / alpha;
  }
  return Su2<double>{co, f * c, f * b, f * a};
}
__device__ __forceinline__ Su2<float> exp_alg(float a, float b, float c) {
  const float t2 = fmaf(a, a, fmaf(b, b, c * c));
  float co, f;
  if (t2 <= 0.25f) {
    detail::cos_sinc_series<float, 4>(t2, co, f);
  } else {
    const float alpha = sqrtf(t2);
    float s;
    sincospif(alpha * 0.318309886183790671538f, &s, &co);
    f = s / alpha;
  }
  return Su2<float>{co, f * c, f * b, f * a};
}

// FP64 trigonometry of an angle through the pi-scaled functions (sincospi(a/pi) etc.): their
// argument reduction is exact, and unlike sin/cos/sincos they carry no local-memory frame
// for a slow reduction path (the product a * (1/pi) rounds once, 1e-16 relative)
constexpr double M_1_PI_D = 0.318309886183790671537767526745;
__device__ __forceinline__ double sin_pi_scaled(double a) { return sinpi(a * M_1_PI_D); }

// ------------------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11); counter {index, draw, step, tag}
enum : uint32_t {
  TAG_MOMENTA = 0x4D4F4D31u,
  TAG_ACCEPT = 0x41434331u,
  TAG_METRO = 0x4D455431u,
  TAG_PF = 0x50465331u,
  TAG_CG0 = 0x43473031u
};

__host__ __device__ __forceinline__ void philox(uint32_t c0, uint32_t c1, uint32_t c2,
                                                uint32_t c3, uint64_t seed, uint32_t out[4]) {
  uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
#pragma unroll
  for (int r = 0; r < 10; r++) {
#ifdef __CUDA_ARCH__
    const uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
    const uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
#else
    const uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
    const uint32_t lo0 = (uint32_t)p0, hi0 = (uint32_t)(p0 >> 32);
    const uint32_t lo1 = (uint32_t)p1, hi1 = (uint32_t)(p1 >> 32);
#endif
    const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}
// (0,1] with 53 random bits
__device__ __forceinline__ double u01_53(uint32_t hi, uint32_t lo) {
  const uint64_t k = ((uint64_t)hi << 21) ^ (uint64_t)(lo >> 11);
  return ((double)k + 1.0) * 0x1p-53;
}
// [0,1) with 32 random bits
__device__ __forceinline__ double u01_32(uint32_t x) { return (double)x * 0x1p-32; }
__device__ __forceinline__ void box_muller(double u1, double u2, double &n0, double &n1) {
  const double r = sqrt(-2.0 * log(u1));
  double s, c;
  sincospi(2.0 * u2, &s, &c);
  n0 = r * c;
  n1 = r * s;
}

// ------------------------------------------------------------------------------------
// deterministic block reduction of doubles (fixed shape -> fixed summation order)
template <int NT> __device__ __forceinline__ double block_sum(double v, double *sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  double r = 0.0;
  if (w == 0) {
    r = (l < NT / 32) ? sh[l] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
  }
  __syncthreads();
  return r;  // valid in thread 0
}
// K block sums with one pair of barriers instead of K: each component is summed exactly as
// block_sum sums it (the same shuffle tree, then the warp sums in order), so the results are
// those of K calls of block_sum.  sh holds K * NT / 32 doubles; the sums are in thread 0.
template <int NT, int K> __device__ __forceinline__ void block_sums(double (&v)[K], double *sh) {
#pragma unroll
  for (int k = 0; k < K; k++)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0)
#pragma unroll
    for (int k = 0; k < K; k++) sh[k * (NT / 32) + w] = v[k];
  __syncthreads();
  if (w == 0)
#pragma unroll
    for (int k = 0; k < K; k++) {
      double r = (l < NT / 32) ? sh[k * (NT / 32) + l] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
      v[k] = r;
    }
  __syncthreads();
}

}  // namespace su2b
