/* su2_oracle.c -- plain-C restatement of the su2 reference hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA library, never the thing measured or
 * shipped.  Each function names the reference file:line it restates.  Floating-point
 * operations are written in the reference's evaluation order (std::complex<double> products
 * as (ac - bd, ad + bc), left-to-right SU(2) chains), so with the same compiler flags most
 * results agree with the reference bit for bit.
 *
 * Third-party algorithm restated here: libstdc++ (GCC 13.3) <random>
 *   - std::mt19937 (Matsumoto & Nishimura 1998, 32-bit MT19937 with the standard
 *     initialisation multiplier 1812433253 and tempering),
 *   - std::generate_canonical<double,53> (two 32-bit draws: (g1 + g2*2^32) / 2^64),
 *   - std::uniform_real_distribution (a + (b-a)*canonical),
 *   - std::normal_distribution (Marsaglia polar method with one cached deviate).
 * These fix the reference's random streams (hotstart, random_gauge_trafo, initnormal,
 * gaussian_spinor, md_update's accept uniform), so the reference chain can be replayed.
 *
 * Also restated: Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), the counter-based
 * generator the CUDA library uses; with it the oracle reproduces the device's own
 * momentum, pseudofermion and Metropolis streams.
 */
#define _GNU_SOURCE
#include "su2_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ===================================================================================== */
/* random numbers                                                                        */
/* ===================================================================================== */

void orc_mt_seed(orc_mt19937 *g, uint32_t seed) {
  g->mt[0] = seed;
  for (int i = 1; i < 624; i++)
    g->mt[i] = 1812433253u * (g->mt[i - 1] ^ (g->mt[i - 1] >> 30)) + (uint32_t)i;
  g->idx = 624;
}

static void mt_twist(orc_mt19937 *g) {
  for (int i = 0; i < 624; i++) {
    const uint32_t y = (g->mt[i] & 0x80000000u) | (g->mt[(i + 1) % 624] & 0x7fffffffu);
    uint32_t v = g->mt[(i + 397) % 624] ^ (y >> 1);
    if (y & 1u) v ^= 0x9908b0dfu;
    g->mt[i] = v;
  }
  g->idx = 0;
}

uint32_t orc_mt_next(orc_mt19937 *g) {
  if (g->idx >= 624) mt_twist(g);
  uint32_t y = g->mt[g->idx++];
  y ^= y >> 11;
  y ^= (y << 7) & 0x9d2c5680u;
  y ^= (y << 15) & 0xefc60000u;
  y ^= y >> 18;
  return y;
}

/* std::generate_canonical<double, 53>(mt19937): k = 2 draws */
double orc_canonical(orc_mt19937 *g) {
  const double r = 4294967296.0;
  double sum = (double)orc_mt_next(g);
  sum += (double)orc_mt_next(g) * r;
  double ret = sum / (r * r);
  if (ret >= 1.0) ret = nextafter(1.0, 0.0);
  return ret;
}

static double uniform_ab(orc_mt19937 *g, double a, double b) {
  return orc_canonical(g) * (b - a) + a;
}

/* std::normal_distribution<double>, one object = one cache slot */
typedef struct {
  double mean, stddev, saved;
  int have_saved;
} normal_dist;

static double normal_draw(normal_dist *n, orc_mt19937 *g) {
  double ret;
  if (n->have_saved) {
    n->have_saved = 0;
    ret = n->saved;
  } else {
    double x, y, r2;
    do {
      x = 2.0 * orc_canonical(g) - 1.0;
      y = 2.0 * orc_canonical(g) - 1.0;
      r2 = x * x + y * y;
    } while (r2 > 1.0 || r2 == 0.0);
    const double mult = sqrt(-2 * log(r2) / r2);
    n->saved = x * mult;
    n->have_saved = 1;
    ret = y * mult;
  }
  return ret * n->stddev + n->mean;
}

static inline uint32_t mulhilo32(uint32_t a, uint32_t b, uint32_t *hi) {
  const uint64_t p = (uint64_t)a * (uint64_t)b;
  *hi = (uint32_t)(p >> 32);
  return (uint32_t)p;
}

void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; r++) {
    uint32_t hi0, hi1;
    const uint32_t lo0 = mulhilo32(0xD2511F53u, c0, &hi0);
    const uint32_t lo1 = mulhilo32(0xCD9E8D57u, c2, &hi1);
    c0 = hi1 ^ c1 ^ k0;
    c1 = lo1;
    c2 = hi0 ^ c3 ^ k1;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

/* stream tags of the device library's counter layout {index, draw, step, tag} */
#define TAG_MOMENTA 0x4D4F4D31u
#define TAG_ACCEPT 0x41434331u
#define TAG_METRO 0x4D455431u
#define TAG_PF 0x50465331u

static void philox_draw(uint64_t seed, uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                        uint32_t out[4]) {
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  const uint32_t ctr[4] = {c0, c1, c2, c3};
  orc_philox4x32_10(ctr, key, out);
}
/* (0,1] with 53 random bits */
static double u01_53(uint32_t hi, uint32_t lo) {
  const uint64_t k = ((uint64_t)hi << 21) ^ (uint64_t)(lo >> 11);
  return ((double)k + 1.0) * 0x1p-53;
}
/* [0,1) with 32 random bits */
static double u01_32(uint32_t x) { return (double)x * 0x1p-32; }

static void box_muller(double u1, double u2, double *n0, double *n1) {
  const double r = sqrt(-2.0 * log(u1));
  *n0 = r * cos(2.0 * M_PI * u2);
  *n1 = r * sin(2.0 * M_PI * u2);
}

/* ===================================================================================== */
/* complex / SU(2) / U(1) arithmetic                                                     */
/* ===================================================================================== */

typedef struct {
  double r, i;
} cplx;
typedef struct {
  cplx a, b;
} su2;

static inline cplx C(double r, double i) {
  cplx c = {r, i};
  return c;
}
static inline cplx cmul(cplx x, cplx y) {
  return C(x.r * y.r - x.i * y.i, x.r * y.i + x.i * y.r);
}
static inline cplx cadd(cplx x, cplx y) { return C(x.r + y.r, x.i + y.i); }
static inline cplx csub(cplx x, cplx y) { return C(x.r - y.r, x.i - y.i); }
static inline cplx cconj(cplx x) { return C(x.r, -x.i); }
static inline cplx cscale(double s, cplx x) { return C(s * x.r, s * x.i); }
static inline cplx cexpi(double t) { return C(cos(t), sin(t)); }
/* std::complex<double> division as libgcc's __divdc3 evaluates it for operands of
 * ordinary magnitude: Smith's algorithm (R. L. Smith, CACM 5 (1962) 435, "Algorithm 116").
 * The extra rescaling branches of libgcc only matter near overflow/underflow. */
static inline cplx cdiv(cplx x, cplx y) {
  const double a = x.r, b = x.i, c = y.r, d = y.i;
  if (fabs(c) < fabs(d)) {
    const double ratio = c / d, denom = (c * ratio) + d;
    return C(((a * ratio) + b) / denom, ((b * ratio) - a) / denom);
  }
  const double ratio = d / c, denom = (d * ratio) + c;
  return C(((b * ratio) + a) / denom, (b - (a * ratio)) / denom);
}

/* su2.hh:87-92 */
static inline su2 smul(su2 u, su2 v) {
  su2 r;
  r.a = csub(cmul(u.a, v.a), cmul(u.b, cconj(v.b)));
  r.b = cadd(cmul(u.a, v.b), cmul(u.b, cconj(v.a)));
  return r;
}
/* su2.hh:53-55 */
static inline su2 sdag(su2 u) {
  su2 r;
  r.a = cconj(u.a);
  r.b = C(-u.b.r, -u.b.i);
  return r;
}
static inline su2 sadd(su2 u, su2 v) {
  su2 r;
  r.a = cadd(u.a, v.a);
  r.b = cadd(u.b, v.b);
  return r;
}
/* Complex(s, 0) * su2 (su2.hh:108-113) as used for anisotropy factors */
static inline su2 sscale(double s, su2 u) {
  su2 r;
  r.a = cmul(u.a, C(s, 0.));
  r.b = cmul(u.b, C(s, 0.));
  return r;
}
static inline double sretr(su2 u) { return 2. * u.a.r; }
/* su2.hh:62-66 (std::abs(complex) is hypot) */
static inline su2 srestore(su2 u) {
  const double ha = hypot(u.a.r, u.a.i), hb = hypot(u.b.r, u.b.i);
  const double r = sqrt(ha * ha + hb * hb);
  su2 o;
  o.a = C(u.a.r / r, u.a.i / r);
  o.b = C(u.b.r / r, u.b.i / r);
  return o;
}
/* su2.hh:83-85 */
static inline su2 stla(su2 x) {
  su2 r;
  const cplx d = csub(x.a, cconj(x.a));
  r.a = cscale(0.5, d);
  r.b = x.b;
  return r;
}
static inline su2 sload(const double *U, size_t l) {
  su2 u;
  u.a = C(U[4 * l], U[4 * l + 1]);
  u.b = C(U[4 * l + 2], U[4 * l + 3]);
  return u;
}
static inline void sstore(double *U, size_t l, su2 u) {
  U[4 * l] = u.a.r;
  U[4 * l + 1] = u.a.i;
  U[4 * l + 2] = u.b.r;
  U[4 * l + 3] = u.b.i;
}

/* exp_gauge.cc:8-18 */
void orc_exp_su2(const double x[3], double out[4]) {
  const double a = x[0], b = x[1], c = x[2];
  const double alpha = sqrt(a * a + b * b + c * c);
  const double n0 = a / alpha, n1 = b / alpha, n2 = c / alpha;
  const double salpha = sin(alpha);
  out[0] = cos(alpha);
  out[1] = salpha * n2;
  out[2] = salpha * n1;
  out[3] = salpha * n0;
}
static inline su2 sexp(double a, double b, double c) {
  const double x[3] = {a, b, c};
  double o[4];
  orc_exp_su2(x, o);
  su2 r;
  r.a = C(o[0], o[1]);
  r.b = C(o[2], o[3]);
  return r;
}

/* ===================================================================================== */
/* lattice geometry (gaugeconfig.hh:211-222)                                             */
/* ===================================================================================== */

typedef struct {
  int nd;
  long L[4]; /* t, x, y, z */
  size_t V;
} lat_t;

static lat_t mklat(int Lx, int Ly, int Lz, int Lt, int nd) {
  lat_t l;
  l.nd = nd;
  l.L[0] = Lt;
  l.L[1] = Lx;
  l.L[2] = Ly;
  l.L[3] = Lz;
  l.V = (size_t)Lx * Ly * Lz * Lt;
  return l;
}
static inline long wrap(long c, long L) { return ((c % L) + L) % L; }
static inline size_t site(const lat_t *l, const long c[4]) {
  return (size_t)(((wrap(c[0], l->L[0]) * l->L[1] + wrap(c[1], l->L[1])) * l->L[2] +
                   wrap(c[2], l->L[2])) *
                    l->L[3] +
                  wrap(c[3], l->L[3]));
}
static inline size_t link(const lat_t *l, const long c[4], int mu) {
  return site(l, c) * (size_t)l->nd + (size_t)mu;
}
static inline void coords(const lat_t *l, size_t s, long c[4]) {
  c[3] = (long)(s % (size_t)l->L[3]);
  s /= (size_t)l->L[3];
  c[2] = (long)(s % (size_t)l->L[2]);
  s /= (size_t)l->L[2];
  c[1] = (long)(s % (size_t)l->L[1]);
  s /= (size_t)l->L[1];
  c[0] = (long)s;
}
static inline size_t nlinks(const lat_t *l) { return l->V * (size_t)l->nd; }

/* ===================================================================================== */
/* random elements, hotstart, gauge transformation                                        */
/* ===================================================================================== */

static const double PI = 3.141592653589793; /* random_element.hh:7 atan(1)*4 */

/* random_element.hh:9-25 */
static su2 random_su2(orc_mt19937 *g, double delta) {
  const double alpha = uniform_ab(g, 0., delta * 2 * PI);
  const double u = uniform_ab(g, -1., 1.);
  const double theta = uniform_ab(g, 0., 2 * PI);
  const double r = sqrt(1 - u * u);
  const double salpha = sin(alpha);
  su2 R;
  R.a = C(cos(alpha), salpha * u);
  R.b = cscale(salpha * r, C(sin(theta), cos(theta)));
  return R;
}
/* random_element.hh:27-34 */
static double random_u1(orc_mt19937 *g, double delta) {
  return uniform_ab(g, -PI * delta, PI * delta);
}

/* random_gauge_trafo.hh:10-33 */
void orc_random_gauge_trafo(int group, int Lx, int Ly, int Lz, int Lt, int nd, int seed,
                            double *U) {
  const lat_t l = mklat(Lx, Ly, Lz, Lt, nd);
  orc_mt19937 g;
  orc_mt_seed(&g, (uint32_t)seed);
  for (size_t s = 0; s < l.V; s++) {
    long c[4];
    coords(&l, s, c);
    if (group == 0) {
      const su2 r = random_su2(&g, 1.);
      for (int mu = 0; mu < nd; mu++) {
        const size_t i = link(&l, c, mu);
        sstore(U, i, smul(r, sload(U, i)));
        long cm[4] = {c[0], c[1], c[2], c[3]};
        cm[mu] -= 1;
        const size_t j = link(&l, cm, mu);
        sstore(U, j, smul(sload(U, j), sdag(r)));
      }
    } else {
      const double r = random_u1(&g, 1.);
      for (int mu = 0; mu < nd; mu++) {
        const size_t i = link(&l, c, mu);
        U[i] = r + U[i];
        long cm[4] = {c[0], c[1], c[2], c[3]};
        cm[mu] -= 1;
        const size_t j = link(&l, cm, mu);
        U[j] = U[j] + (-r);
      }
    }
  }
}

/* gaugeconfig.hh:277-289 (+ base_program.hpp:314 gauge rotation when trafo_seed >= 0) */
void orc_hotstart(int group, int Lx, int Ly, int Lz, int Lt, int nd, int seed, double delta,
                  int trafo_seed, double *out) {
  const lat_t l = mklat(Lx, Ly, Lz, Lt, nd);
  if (delta < 0.) delta = 0.;
  if (delta > 1.) delta = 1.;
  orc_mt19937 g;
  orc_mt_seed(&g, (uint32_t)seed);
  for (size_t i = 0; i < nlinks(&l); i++) {
    if (group == 0)
      sstore(out, i, random_su2(&g, delta));
    else
      out[i] = random_u1(&g, delta);
  }
  if (trafo_seed >= 0) orc_random_gauge_trafo(group, Lx, Ly, Lz, Lt, nd, trafo_seed, out);
}

/* ===================================================================================== */
/* plaquettes and action                                                                 */
/* ===================================================================================== */

static double plaq_retr(int group, const lat_t *l, const double *U, const long c[4], int mu,
                        int nu) {
  long cpm[4] = {c[0], c[1], c[2], c[3]}, cpn[4] = {c[0], c[1], c[2], c[3]};
  cpm[mu] += 1;
  cpn[nu] += 1;
  const size_t i0 = link(l, c, mu), i1 = link(l, cpm, nu), i2 = link(l, cpn, mu),
               i3 = link(l, c, nu);
  if (group == 0) {
    const su2 p =
      smul(smul(smul(sload(U, i0), sload(U, i1)), sdag(sload(U, i2))), sdag(sload(U, i3)));
    return sretr(p);
  }
  return cos(((U[i0] + U[i1]) + (-U[i2])) + (-U[i3]));
}

/* flat-gauge_energy.hpp:31-94 */
double orc_retr_sum_plaquettes(int group, int Lx, int Ly, int Lz, int Lt, int nd,
                               const double *U, double xi, int aniso, int spatial_only) {
  const lat_t l = mklat(Lx, Ly, Lz, Lt, nd);
  double res = 0.;
  const int startmu = spatial_only ? 1 : 0;
  for (size_t s = 0; s < l.V; s++) {
    long c[4];
    coords(&l, s, c);
    for (int mu = startmu; mu < nd - 1; mu++)
      for (int nu = mu + 1; nu < nd; nu++) {
        double eta = 1.;
        if (aniso) eta = ((mu == 0) ^ (nu == 0)) ? 1.0 / xi : xi;
        const double p = plaq_retr(group, &l, U, c, mu, nu);
        res += aniso ? eta * p : p;
      }
  }
  return res;
}

/* flat-gauge_energy.hpp:109-137 */
double orc_gauge_energy(int group, int Lx, int Ly, int Lz, int Lt, int nd, const double *U,
                        int spatial_only) {
  return orc_retr_sum_plaquettes(group, Lx, Ly, Lz, Lt, nd, U, 1.0, 0, spatial_only);
}

/* flat-gaugemonomial.hh:46-54 */
double orc_S_G_hmc(int group, int Lx, int Ly, int Lz, int Lt, int nd, double beta,
                   const double *U, double xi, int aniso) {
  const double Nc = group == 0 ? 2. : 1.;
  return -beta * orc_retr_sum_plaquettes(group, Lx, Ly, Lz, Lt, nd, U, xi, aniso, 0) / Nc;
}

/* ===================================================================================== */
/* staples and gauge force                                                               */
/* ===================================================================================== */

/* get_staples.hh:26-80 for SU(2); returns K */
static su2 staples_su2(const lat_t *l, const double *U, const long c[4], int mu, double xi,
                       int aniso) {
  su2 K;
  K.a = C(0., 0.);
  K.b = C(0., 0.);
  long x1[4] = {c[0], c[1], c[2], c[3]}, x2[4] = {c[0], c[1], c[2], c[3]};
  x1[mu] += 1;
  for (int nu = 0; nu < l->nd; nu++) {
    if (nu == mu) continue;
    x2[nu]++;
    const su2 A = sload(U, link(l, x1, nu)), B = sload(U, link(l, x2, mu)),
              D = sload(U, link(l, c, nu));
    if (aniso) {
      const double f = ((nu == 0) || (mu == 0)) ? 1.0 / xi : xi;
      K = sadd(K, smul(smul(sscale(f, A), sdag(B)), sdag(D)));
    } else
      K = sadd(K, smul(smul(A, sdag(B)), sdag(D)));
    x2[nu]--;
  }
  for (int nu = 0; nu < l->nd; nu++) {
    if (nu == mu) continue;
    x1[nu]--;
    x2[nu]--;
    const su2 A = sload(U, link(l, x1, nu)), B = sload(U, link(l, x2, mu)),
              D = sload(U, link(l, x2, nu));
    if (aniso) {
      const double f = ((nu == 0) || (mu == 0)) ? 1.0 / xi : xi;
      K = sadd(K, smul(smul(sscale(f, sdag(A)), sdag(B)), D));
    } else
      K = sadd(K, smul(smul(sdag(A), sdag(B)), D));
    x2[nu]++;
    x1[nu]++;
  }
  return K;
}

/* get_staples.hh:26-80 for U(1): K is the complex accumulator (u1.hh:73-75) */
static cplx staples_u1(const lat_t *l, const double *U, const long c[4], int mu, double xi,
                       int aniso) {
  cplx K = C(0., 0.);
  long x1[4] = {c[0], c[1], c[2], c[3]}, x2[4] = {c[0], c[1], c[2], c[3]};
  x1[mu] += 1;
  for (int nu = 0; nu < l->nd; nu++) {
    if (nu == mu) continue;
    x2[nu]++;
    const double A = U[link(l, x1, nu)], B = U[link(l, x2, mu)], D = U[link(l, c, nu)];
    if (aniso) {
      const double f = ((nu == 0) || (mu == 0)) ? 1.0 / xi : xi;
      K = cadd(K, cmul(cmul(cmul(C(f, 0.), cexpi(A)), cexpi(-B)), cexpi(-D)));
    } else
      K = cadd(K, cexpi((A + (-B)) + (-D)));
    x2[nu]--;
  }
  for (int nu = 0; nu < l->nd; nu++) {
    if (nu == mu) continue;
    x1[nu]--;
    x2[nu]--;
    const double A = U[link(l, x1, nu)], B = U[link(l, x2, mu)], D = U[link(l, x2, nu)];
    if (aniso) {
      const double f = ((nu == 0) || (mu == 0)) ? 1.0 / xi : xi;
      K = cadd(K, cmul(cmul(cmul(C(f, 0.), cexpi(-A)), cexpi(-B)), cexpi(D)));
    } else
      K = cadd(K, cexpi(((-A) + (-B)) + D));
    x2[nu]++;
    x1[nu]++;
  }
  return K;
}

/* flat-gaugemonomial.hh:105-131: deriv += fac*beta/Nc * get_deriv(U*K) */
void orc_gauge_derivative(int group, int Lx, int Ly, int Lz, int Lt, int nd, double beta,
                          double xi, const double *U, double fac, double *deriv) {
  const lat_t l = mklat(Lx, Ly, Lz, Lt, nd);
  const int aniso = (xi != 1.0);
  const double Nc = group == 0 ? 2. : 1.;
  const double f = fac * beta / Nc;
#pragma omp parallel for schedule(static)
  for (long s = 0; s < (long)l.V; s++) {
    long c[4];
    coords(&l, (size_t)s, c);
    for (int mu = 0; mu < nd; mu++) {
      const size_t i = link(&l, c, mu);
      if (group == 0) {
        const su2 S = smul(sload(U, i), staples_su2(&l, U, c, mu, xi, aniso));
        /* adjointfield.hh:53-56 */
        deriv[3 * i] += f * (2. * S.b.i);
        deriv[3 * i + 1] += f * (2. * S.b.r);
        deriv[3 * i + 2] += f * (2. * S.a.i);
      } else {
        const cplx S = cmul(cexpi(U[i]), staples_u1(&l, U, c, mu, xi, aniso));
        deriv[i] += f * S.i; /* adjointfield.hh:79-81 */
      }
    }
  }
}

/* gaugeconfig.hh:115-120 */
void orc_restore_su(int group, int Lx, int Ly, int Lz, int Lt, int nd, double *U) {
  if (group != 0) return; /* u1.hh:178-179 no-op */
  const lat_t l = mklat(Lx, Ly, Lz, Lt, nd);
  for (size_t i = 0; i < nlinks(&l); i++) sstore(U, i, srestore(sload(U, i)));
}

/* update_gauge.hh:8-16 */
void orc_update_gauge(int group, int Lx, int Ly, int Lz, int Lt, int nd, double *U,
                      const double *P, double dtau) {
  const lat_t l = mklat(Lx, Ly, Lz, Lt, nd);
  const size_t N = nlinks(&l);
#pragma omp parallel for schedule(static)
  for (long i = 0; i < (long)N; i++) {
    if (group == 0) {
      const su2 e = sexp(dtau * P[3 * i], dtau * P[3 * i + 1], dtau * P[3 * i + 2]);
      sstore(U, (size_t)i, smul(e, sload(U, (size_t)i)));
    } else {
      U[i] = dtau * P[i] + U[i];
    }
  }
}

/* ===================================================================================== */
/* staggered fermions (staggered.hpp)                                                    */
/* ===================================================================================== */

/* staggered.hpp:41-48 */
/* ===================================================================================== */
/* observables between trajectories                                                      */
/* ===================================================================================== */

/* exp(i a) as std::exp(a * Complex(0., 1.)) evaluates it: (e^0 cos a, e^0 sin a) */
static inline cplx u1_phase(double a) { return C(cos(a), sin(a)); }

/* polyakov_loop_spatial_average (polyakov_loop.hh:26-63): the product of the temporal links
 * along t at every spatial point, ReTr, summed and divided by the full volume */
double orc_polyakov_loop(int group, int Lx, int Ly, int Lz, int Lt, int nd, const double *U) {
  const lat_t l = mklat(Lx, Ly, Lz, Lt, nd);
  double ploop = 0.;
  for (long x1 = 0; x1 < l.L[1]; x1++)
    for (long x2 = 0; x2 < l.L[2]; x2++)
      for (long x3 = 0; x3 < l.L[3]; x3++) {
        long c[4] = {0, x1, x2, x3};
        if (group == 0) {
          su2 P;
          P.a = C(1., 0.);
          P.b = C(0., 0.);
          for (c[0] = 0; c[0] < l.L[0]; c[0]++) P = smul(P, sload(U, link(&l, c, 0)));
          ploop += sretr(P);
        } else {
          cplx P = C(1., 0.);
          for (c[0] = 0; c[0] < l.L[0]; c[0]++) P = cmul(P, u1_phase(U[link(&l, c, 0)]));
          ploop += P.r;
        }
      }
  return ploop / (double)l.V;
}

/* planar_wilsonloop_dir (wilsonloop.hh:51-91): sum over sites of ReTr of the r x t loop
 * x -> x + t nu -> + r mu -> - t nu -> - r mu */
static double planar_loop_dir(int group, const lat_t *l, const double *U, long r, long t,
                              int mu, int nu) {
  double loop = 0.;
  for (size_t s = 0; s < l->V; s++) {
    long x[4];
    coords(l, s, x);
    if (group == 0) {
      su2 L;
      L.a = C(1., 0.);
      L.b = C(0., 0.);
      for (long k = 0; k < t; k++) {
        L = smul(L, sload(U, link(l, x, nu)));
        x[nu] += 1;
      }
      for (long k = 0; k < r; k++) {
        L = smul(L, sload(U, link(l, x, mu)));
        x[mu] += 1;
      }
      for (long k = 0; k < t; k++) {
        x[nu] -= 1;
        L = smul(L, sdag(sload(U, link(l, x, nu))));
      }
      for (long k = 0; k < r; k++) {
        x[mu] -= 1;
        L = smul(L, sdag(sload(U, link(l, x, mu))));
      }
      loop += sretr(L);
    } else {
      cplx L = C(1., 0.);
      for (long k = 0; k < t; k++) {
        L = cmul(L, u1_phase(U[link(l, x, nu)]));
        x[nu] += 1;
      }
      for (long k = 0; k < r; k++) {
        L = cmul(L, u1_phase(U[link(l, x, mu)]));
        x[mu] += 1;
      }
      for (long k = 0; k < t; k++) {
        x[nu] -= 1;
        L = cmul(L, u1_phase(-U[link(l, x, nu)]));
      }
      for (long k = 0; k < r; k++) {
        x[mu] -= 1;
        L = cmul(L, u1_phase(-U[link(l, x, mu)]));
      }
      loop += L.r;
    }
  }
  return loop;
}

/* wilsonloop(U, r, t) (wilsonloop.hh:147-157): planar loops in the (mu, 0) planes, mu >= 1,
 * normalised by V Nc ndims */
double orc_wilson_loop(int group, int Lx, int Ly, int Lz, int Lt, int nd, const double *U,
                       int r, int t) {
  const lat_t l = mklat(Lx, Ly, Lz, Lt, nd);
  double loop = 0.;
  for (int mu = 1; mu < nd; mu++) loop += planar_loop_dir(group, &l, U, r, t, mu, 0);
  const double Nc = group == 0 ? 2. : 1.;
  return loop / (double)l.V / Nc / (double)nd;
}

/* APEsmearing<double>(U, alpha, spatial) (smearape.hh:97-131) with the staples of
 * get_staples_APE (get_staples.hh:89-110):
 *   K = sum_{nu != i} U_nu(x) U_i(x+nu) U_nu(x+i)^+ + U_nu(x-nu)^+ U_i(x-nu) U_nu(x+i-nu)
 *   U_i(x) <- restoreSU(alpha U_i(x) + beta K),  beta = (1 - alpha) / (2 (d - 1 - start))
 * over nu >= start, for the links i >= start (start = 1 for spatial smearing) */
void orc_ape_smear(int group, int Lx, int Ly, int Lz, int Lt, int nd, double alpha,
                   int spatial, double *U) {
  const lat_t l = mklat(Lx, Ly, Lz, Lt, nd);
  const size_t n = nlinks(&l) * (group == 0 ? 4 : 1);
  double *Uold = (double *)malloc(n * sizeof(double));
  memcpy(Uold, U, n * sizeof(double));
  const int start = spatial ? 1 : 0;
  const double beta = (1.0 - alpha) / ((double)(2 * (nd - 1 - start)));
  for (size_t s = 0; s < l.V; s++) {
    long x[4];
    coords(&l, s, x);
    for (int i = start; i < nd; i++) {
      long xi[4] = {x[0], x[1], x[2], x[3]};
      xi[i] += 1;
      if (group == 0) {
        su2 K;
        K.a = C(0., 0.);
        K.b = C(0., 0.);
        for (int nu = start; nu < nd; nu++) {
          if (nu == i) continue;
          long xn[4] = {x[0], x[1], x[2], x[3]}, xmn[4] = {x[0], x[1], x[2], x[3]},
               ximn[4] = {xi[0], xi[1], xi[2], xi[3]};
          xn[nu] += 1;
          xmn[nu] -= 1;
          ximn[nu] -= 1;
          K = sadd(K, smul(smul(sload(Uold, link(&l, x, nu)), sload(Uold, link(&l, xn, i))),
                           sdag(sload(Uold, link(&l, xi, nu)))));
          K = sadd(K, smul(smul(sdag(sload(Uold, link(&l, xmn, nu))),
                                sload(Uold, link(&l, xmn, i))),
                           sload(Uold, link(&l, ximn, nu))));
        }
        const su2 up = sadd(sscale(alpha, sload(Uold, link(&l, x, i))), sscale(beta, K));
        sstore(U, link(&l, x, i), srestore(up));
      } else {
        cplx K = C(0., 0.);
        for (int nu = start; nu < nd; nu++) {
          if (nu == i) continue;
          long xn[4] = {x[0], x[1], x[2], x[3]}, xmn[4] = {x[0], x[1], x[2], x[3]},
               ximn[4] = {xi[0], xi[1], xi[2], xi[3]};
          xn[nu] += 1;
          xmn[nu] -= 1;
          ximn[nu] -= 1;
          /* _u1 products are angle sums; K += exp(i angle) */
          K = cadd(K, u1_phase((Uold[link(&l, x, nu)] + Uold[link(&l, xn, i)]) +
                               (-Uold[link(&l, xi, nu)])));
          K = cadd(K, u1_phase(((-Uold[link(&l, xmn, nu)]) + Uold[link(&l, xmn, i)]) +
                               Uold[link(&l, ximn, nu)]));
        }
        const cplx up = cadd(cmul(C(alpha, 0.), u1_phase(Uold[link(&l, x, i)])),
                             cmul(C(beta, 0.), K));
        U[link(&l, x, i)] = atan2(up.i, up.r);
      }
    }
  }
  free(Uold);
}

double orc_eta(int t, int x, int y, int z, int mu) {
  const int c[4] = {t, x, y, z};
  double s = 0;
  for (int nu = 0; nu < mu; nu++) s += c[nu];
  return pow(-1.0, s);
}
static double eta_c(const long c[4], int mu) {
  double s = 0;
  for (int nu = 0; nu < mu; nu++) s += (double)c[nu];
  return pow(-1.0, s);
}

static inline cplx ld_c(const double *v, size_t i) { return C(v[2 * i], v[2 * i + 1]); }
static inline void st_c(double *v, size_t i, cplx z) {
  v[2 * i] = z.r;
  v[2 * i + 1] = z.i;
}

/* staggered.hpp:305-341 (op 0) and :353-389 (op 1) */
static void apply_D_or_Ddag(const lat_t *l, const double *U, double m, int dag,
                            const double *psi, double *phi) {
#pragma omp parallel for schedule(static)
  for (long s = 0; s < (long)l->V; s++) {
    long c[4];
    coords(l, (size_t)s, c);
    cplx acc = C(0., 0.);
    for (int mu = 0; mu < l->nd; mu++) {
      long xm[4] = {c[0], c[1], c[2], c[3]}, xp[4] = {c[0], c[1], c[2], c[3]};
      xm[mu]--;
      xp[mu]++;
      const size_t sm = site(l, xm), sp = site(l, xp);
      if (!dag) {
        const double e = eta_c(c, mu);
        const cplx t1 = cmul(cmul(C(+(1.0 / 2.0) * e, 0.), cexpi(U[link(l, c, mu)])),
                             ld_c(psi, sp));
        acc = cadd(acc, t1);
        const cplx t2 = cmul(cmul(C(-(1.0 / 2.0) * e, 0.), cexpi(-U[link(l, xm, mu)])),
                             ld_c(psi, sm));
        acc = cadd(acc, t2);
      } else {
        const double em = eta_c(xm, mu), ep = eta_c(xp, mu);
        const cplx t1 = cmul(cmul(C(+(1.0 / 2.0) * em, 0.), cexpi(-U[link(l, xm, mu)])),
                             ld_c(psi, sm));
        acc = cadd(acc, t1);
        const cplx t2 = cmul(cmul(C(-(1.0 / 2.0) * ep, 0.), cexpi(U[link(l, c, mu)])),
                             ld_c(psi, sp));
        acc = cadd(acc, t2);
      }
    }
    acc = cadd(acc, cscale(m, ld_c(psi, (size_t)s)));
    st_c(phi, (size_t)s, acc);
  }
}

/* op: 0 D, 1 Ddag, 2 D Ddag (staggered.hpp:290-302) */
void orc_staggered_apply(int Lx, int Ly, int Lz, int Lt, int nd, const double *U, double m,
                         int op, const double *in, double *out) {
  const lat_t l = mklat(Lx, Ly, Lz, Lt, nd);
  if (op == 0 || op == 1) {
    apply_D_or_Ddag(&l, U, m, op, in, out);
    return;
  }
  double *tmp = (double *)malloc(2 * l.V * sizeof(double));
  apply_D_or_Ddag(&l, U, m, 1, in, tmp);
  apply_D_or_Ddag(&l, U, m, 0, tmp, out);
  free(tmp);
}

/* ---- generic Krylov solvers (CG.hpp:36-94, BiCGStab.hpp:36-106) --------------------- */

typedef void (*matvec_fn)(const void *ctx, const double *in, double *out);

static cplx vdot(size_t n, const double *a, const double *b) {
  cplx s = C(0., 0.);
  for (size_t i = 0; i < n; i++) s = cadd(s, cmul(cconj(ld_c(a, i)), ld_c(b, i)));
  return s;
}
static double vnorm(size_t n, const double *a) { return sqrt(vdot(n, a, a).r); }
/* c = a + (real)lam * b via double*Complex (used for +1/-1 combinations) */
static void vaxpy_r(size_t n, const double *a, double lam, const double *b, double *c) {
  for (size_t i = 0; i < n; i++) st_c(c, i, cadd(ld_c(a, i), cscale(lam, ld_c(b, i))));
}
/* lambda * psi = 0 + lambda*psi (staggered.hpp:215-220) */
static void vscal(size_t n, cplx lam, const double *b, double *c) {
  for (size_t i = 0; i < n; i++) st_c(c, i, cadd(C(0., 0.), cmul(lam, ld_c(b, i))));
}

static long last_solve_calls = 0;
long orc_last_solve_calls(void) { return last_solve_calls; }

static long cg_solve(size_t n, matvec_fn A, const void *ctx, const double *b, double *x,
                     double tol) {
  last_solve_calls = 0;
  double *r = malloc(2 * n * sizeof(double)), *p = malloc(2 * n * sizeof(double)),
         *ap = malloc(2 * n * sizeof(double)), *t = malloc(2 * n * sizeof(double)),
         *t2 = malloc(2 * n * sizeof(double));
  long iters = 0;
  for (;;) {
    last_solve_calls++;
    A(ctx, x, t);
    vaxpy_r(n, b, -1.0, t, r);
    memcpy(p, r, 2 * n * sizeof(double));
    double rn = vnorm(n, r);
    while (rn > tol) {
      A(ctx, p, ap);
      const cplx rr = vdot(n, r, r);
      const cplx alpha = cdiv(vdot(n, r, r), vdot(n, p, ap));
      vscal(n, alpha, p, t);
      vaxpy_r(n, x, 1.0, t, t2);
      memcpy(x, t2, 2 * n * sizeof(double));
      vscal(n, alpha, ap, t);
      vaxpy_r(n, r, -1.0, t, t2);
      memcpy(r, t2, 2 * n * sizeof(double));
      const cplx beta = cdiv(vdot(n, r, r), rr);
      vscal(n, beta, p, t);
      vaxpy_r(n, r, 1.0, t, p);
      iters++;
      rn = vnorm(n, r);
    }
    A(ctx, x, t);
    vaxpy_r(n, b, -1.0, t, t2);
    const double ex = vnorm(n, t2);
    if (!(rn < ex)) break; /* CG.hpp:78-84: restart from x while the true residual is larger */
  }
  free(r);
  free(p);
  free(ap);
  free(t);
  free(t2);
  return iters;
}

static long bicgstab_solve(size_t n, matvec_fn A, const void *ctx, const double *b, double *x,
                           double tol) {
  last_solve_calls = 0;
  const size_t B = 2 * n * sizeof(double);
  double *r0 = malloc(B), *r = malloc(B), *p = malloc(B), *ap = malloc(B), *s = malloc(B),
         *t = malloc(B), *w = malloc(B), *w2 = malloc(B);
  long iters = 0;
  for (;;) {
    last_solve_calls++;
    A(ctx, x, w);
    vaxpy_r(n, b, -1.0, w, r0);
    memcpy(r, r0, B);
    memcpy(p, r, B);
    double rn = vnorm(n, r);
    while (rn > tol) {
      A(ctx, p, ap);
      const cplx r0r = vdot(n, r0, r);
      const cplx alpha = cdiv(vdot(n, r0, r), vdot(n, r0, ap));
      vscal(n, alpha, ap, w);
      vaxpy_r(n, r, -1.0, w, s);
      A(ctx, s, t);
      const cplx omega = cdiv(vdot(n, t, s), vdot(n, t, t));
      vscal(n, omega, t, w); /* A*s recomputed in the reference; same values */
      vaxpy_r(n, s, -1.0, w, r);
      vscal(n, omega, s, w);
      vaxpy_r(n, x, 1.0, w, w2);
      vscal(n, alpha, p, w);
      vaxpy_r(n, w2, 1.0, w, x);
      const cplx beta = cmul(cdiv(vdot(n, r0, r), r0r), cdiv(alpha, omega));
      vscal(n, beta, p, w);
      vaxpy_r(n, r, 1.0, w, w2);
      vscal(n, cmul(beta, omega), ap, w);
      vaxpy_r(n, w2, -1.0, w, p);
      iters++;
      rn = vnorm(n, r);
    }
    A(ctx, x, w);
    vaxpy_r(n, b, -1.0, w, w2);
    const double ex = vnorm(n, w2);
    if (!(rn < ex)) break;
  }
  free(r0);
  free(r);
  free(p);
  free(ap);
  free(s);
  free(t);
  free(w);
  free(w2);
  return iters;
}

typedef struct {
  lat_t l;
  const double *U;
  double m;
  int op;
} stag_ctx;

static void stag_mv(const void *vctx, const double *in, double *out) {
  const stag_ctx *c = (const stag_ctx *)vctx;
  if (c->op == 2) {
    double *tmp = malloc(2 * c->l.V * sizeof(double));
    apply_D_or_Ddag(&c->l, c->U, c->m, 1, in, tmp);
    apply_D_or_Ddag(&c->l, c->U, c->m, 0, tmp, out);
    free(tmp);
  } else
    apply_D_or_Ddag(&c->l, c->U, c->m, c->op, in, out);
}

long orc_cg_ddag(int Lx, int Ly, int Lz, int Lt, int nd, const double *U, double m,
                 const double *b, const double *x0, double tol, double *x) {
  stag_ctx c = {mklat(Lx, Ly, Lz, Lt, nd), U, m, 2};
  memcpy(x, x0, 2 * c.l.V * sizeof(double));
  return cg_solve(c.l.V, stag_mv, &c, b, x, tol);
}

long orc_bicgstab_d(int Lx, int Ly, int Lz, int Lt, int nd, const double *U, double m,
                    const double *b, const double *x0, double tol, double *x) {
  stag_ctx c = {mklat(Lx, Ly, Lz, Lt, nd), U, m, 0};
  memcpy(x, x0, 2 * c.l.V * sizeof(double));
  return bicgstab_solve(c.l.V, stag_mv, &c, b, x, tol);
}

typedef struct {
  int n;
  const double *A;
} dense_ctx;
/* LA.hpp operator*(LAmatrix, LAvector): w[i] += A[i][k]*v[k] */
static void dense_mv(const void *vctx, const double *in, double *out) {
  const dense_ctx *c = (const dense_ctx *)vctx;
  for (int i = 0; i < c->n; i++) {
    cplx w = C(0., 0.);
    for (int k = 0; k < c->n; k++)
      w = cadd(w, cmul(ld_c(c->A, (size_t)(i * c->n + k)), ld_c(in, (size_t)k)));
    st_c(out, (size_t)i, w);
  }
}
long orc_cg_dense(int n, const double *A, const double *b, const double *x0, double tol,
                  double *x) {
  dense_ctx c = {n, A};
  memcpy(x, x0, 2 * (size_t)n * sizeof(double));
  return cg_solve((size_t)n, dense_mv, &c, b, x, tol);
}
long orc_bicgstab_dense(int n, const double *A, const double *b, const double *x0, double tol,
                        double *x) {
  dense_ctx c = {n, A};
  memcpy(x, x0, 2 * (size_t)n * sizeof(double));
  return bicgstab_solve((size_t)n, dense_mv, &c, b, x, tol);
}

/* staggered.hpp:175-193: real Gaussian per site from std::mt19937(seed) */
void orc_gaussian_spinor(int Lx, int Ly, int Lz, int Lt, double avr, double sigma, long seed,
                         double *out) {
  const size_t V = (size_t)Lx * Ly * Lz * Lt;
  orc_mt19937 g;
  orc_mt_seed(&g, (uint32_t)seed);
  normal_dist nd = {avr, sigma, 0., 0};
  for (size_t i = 0; i < V; i++) {
    out[2 * i] = normal_draw(&nd, &g);
    out[2 * i + 1] = 0.;
  }
}

/* DDdag_matrix_lat::inv (staggered.hpp:249-276) */
void orc_ddag_inv(int Lx, int Ly, int Lz, int Lt, int nd, const double *U, double m,
                  const double *psi, double tol, long seed, double *x) {
  const size_t V = (size_t)Lx * Ly * Lz * Lt;
  double *x0 = malloc(2 * V * sizeof(double));
  orc_gaussian_spinor(Lx, Ly, Lz, Lt, 0.0, 10.0, seed, x0);
  orc_cg_ddag(Lx, Ly, Lz, Lt, nd, U, m, psi, x0, tol, x);
  free(x0);
}

/* staggered::C_pion (propagator.hpp:25-65): R = (D D^+)^-1 delta_0 by DDdag.inv (CG from
 * gaussian_spinor(0, 10, seed)), S = D^+ R, C[t] = sum_{x in slice t} |S(x)|^2 / Vs for t >= 1,
 * C[0] = 0.  The reference repeats the identical solve for every site; once is the same. */
void orc_pion_correlator(int Lx, int Ly, int Lz, int Lt, int nd, const double *U, double m,
                         double tol, long seed, double *C) {
  const size_t V = (size_t)Lx * Ly * Lz * Lt, Vs = V / (size_t)Lt;
  double *src = calloc(2 * V, sizeof(double)), *R = malloc(2 * V * sizeof(double)),
         *S = malloc(2 * V * sizeof(double));
  src[0] = 1.0;
  orc_ddag_inv(Lx, Ly, Lz, Lt, nd, U, m, src, tol, seed, R);
  orc_staggered_apply(Lx, Ly, Lz, Lt, nd, U, m, 1, R, S);
  for (int t = 0; t < Lt; t++) {
    C[t] = 0.0;
    if (t == 0) continue;
    for (size_t i = 0; i < Vs; i++) {
      const size_t x = (size_t)t * Vs + i;
      C[t] += S[2 * x] * S[2 * x] + S[2 * x + 1] * S[2 * x + 1];
    }
    C[t] /= (double)Vs;
  }
  free(src);
  free(R);
  free(S);
}

/* detDDdag_monomial.hh:64-83 with n_traj = 0 */
double orc_fermion_heatbath(int Lx, int Ly, int Lz, int Lt, int nd, const double *U, double m,
                            long seed_pf, double *phi) {
  const lat_t l = mklat(Lx, Ly, Lz, Lt, nd);
  double *R = malloc(2 * l.V * sizeof(double));
  orc_gaussian_spinor(Lx, Ly, Lz, Lt, 0.0, 1.0 / sqrt(2), seed_pf, R);
  apply_D_or_Ddag(&l, U, m, 0, R, phi);
  const double h = vdot(l.V, R, R).r;
  free(R);
  return h;
}

/* detDDdag_monomial.hh:93-103 */
double orc_fermion_accept(int Lx, int Ly, int Lz, int Lt, int nd, const double *U, double m,
                          const double *phi, double tol, long seed) {
  const size_t V = (size_t)Lx * Ly * Lz * Lt;
  double *chi = malloc(2 * V * sizeof(double));
  orc_ddag_inv(Lx, Ly, Lz, Lt, nd, U, m, phi, tol, seed, chi);
  const double h = vdot(V, phi, chi).r;
  free(chi);
  return h;
}

/* detDDdag_monomial.hh:124-164: the per-link contraction given chi = (D Ddag)^-1 phi */
void orc_fermion_force_from_chi(int Lx, int Ly, int Lz, int Lt, int nd, const double *U,
                                double m, const double *chi, double *deriv) {
  const lat_t l = mklat(Lx, Ly, Lz, Lt, nd);
  double *chi1 = malloc(2 * l.V * sizeof(double));
  apply_D_or_Ddag(&l, U, m, 1, chi, chi1);
  const cplx I = C(0.0, 1.0), mI = C(-0.0, -1.0), m2I = C(-2.0 * 0.0, -2.0 * 1.0);
  for (size_t s = 0; s < l.V; s++) {
    long c[4];
    coords(&l, s, c);
    for (int mu = 0; mu < nd; mu++) {
      long xp[4] = {c[0], c[1], c[2], c[3]};
      xp[mu]++;
      const size_t sp = site(&l, xp), i = link(&l, c, mu);
      const double ex = eta_c(c, mu), exp_ = eta_c(xp, mu);
      const cplx v_xp =
        cmul(cmul(cscale((1.0 / 2.0) * ex, I), cexpi(U[i])), ld_c(chi1, sp));
      const cplx v_x =
        cmul(cmul(cscale(-(1.0 / 2.0) * exp_, mI), cexpi(-U[i])), ld_c(chi1, s));
      cplx d = cadd(cmul(cconj(ld_c(chi, s)), v_xp), cmul(cconj(ld_c(chi, sp)), v_x));
      d = cmul(m2I, d);
      deriv[i] += d.i;
    }
  }
  free(chi1);
}

/* detDDdag_monomial.hh:112-167 */
void orc_fermion_derivative(int Lx, int Ly, int Lz, int Lt, int nd, const double *U, double m,
                            const double *phi, double tol, long seed, double *deriv) {
  const size_t V = (size_t)Lx * Ly * Lz * Lt;
  double *chi = malloc(2 * V * sizeof(double));
  orc_ddag_inv(Lx, Ly, Lz, Lt, nd, U, m, phi, tol, seed, chi);
  orc_fermion_force_from_chi(Lx, Ly, Lz, Lt, nd, U, m, chi, deriv);
  free(chi);
}

/* ===================================================================================== */
/* molecular dynamics                                                                    */
/* ===================================================================================== */

typedef struct {
  int group;
  lat_t l;
  double beta, xi;
  /* optional staggered monomial (U(1) only) */
  int fermions;
  double m, tol;
  long seed;
  const double *phi;
  /* lp_leapfrog / lp_omf4: 10^exponent (> 0), else 0 */
  double round_dn;
} md_sys;

/* x.round(n) of the low-precision integrators, componentwise std::round(x*dn)/dn:
 * adjointsu2 / adjointu1 (adjointfield.hh:28-31, 67-69) and _su2 (su2.hh:29-33) */
static inline double round_dn(double x, double dn) { return round(x * dn) / dn; }
/* _u1::round (u1.hh:31-33) rounds the angle before scaling: (round(a)*dn)/dn */
static inline double round_u1_link(double a, double dn) { return (round(a) * dn) / dn; }

/* update_momenta.hh:10-33: deriv = 0; gauge (+ fermion) derivative; P -= dtau*deriv */
static void md_update_momenta(const md_sys *s, double *U, double *P, double dtau) {
  const lat_t *l = &s->l;
  const size_t N = nlinks(l), na = s->group == 0 ? 3 : 1;
  double *deriv = calloc(N * na, sizeof(double));
  orc_gauge_derivative(s->group, (int)l->L[1], (int)l->L[2], (int)l->L[3], (int)l->L[0],
                       l->nd, s->beta, s->xi, U, 1., deriv);
  if (s->fermions)
    orc_fermion_derivative((int)l->L[1], (int)l->L[2], (int)l->L[3], (int)l->L[0], l->nd, U,
                           s->m, s->phi, s->tol, s->seed, deriv);
  if (s->round_dn > 0.) /* round_and_update_momenta (update_momenta.hh:36-58) */
    for (size_t i = 0; i < N * na; i++) P[i] -= dtau * round_dn(deriv[i], s->round_dn);
  else
    for (size_t i = 0; i < N * na; i++) P[i] -= dtau * deriv[i];
  free(deriv);
}
static void md_update_gauge(const md_sys *s, double *U, const double *P, double dtau) {
  const lat_t *l = &s->l;
  if (s->round_dn > 0.) { /* round_and_update_gauge (update_gauge.hh:20-26): U = e * round(U) */
    const size_t N = nlinks(l);
    for (size_t i = 0; i < N; i++) {
      if (s->group == 0)
        for (int k = 0; k < 4; k++) U[4 * i + k] = round_dn(U[4 * i + k], s->round_dn);
      else
        U[i] = round_u1_link(U[i], s->round_dn);
    }
  }
  orc_update_gauge(s->group, (int)l->L[1], (int)l->L[2], (int)l->L[3], (int)l->L[0], l->nd, U,
                   P, dtau);
}

/* integrator.hh:26-50 (0), :83-116 (6), :119-156 (2), :201-217 (4), :220-241 (5); the
 * low-precision lp_leapfrog (1, :53-80) and lp_omf4 (3, :158-199) take the schedules of 0 and
 * 2 with the rounding of md_sys.round_dn */
static void md_integrate(const md_sys *s, int integ, int nsteps, double tau, double *U,
                         double *P) {
  const double dtau = tau / (double)nsteps;
  if (integ == 6) { /* omf2 */
    const double lambda = 0.1938;
    const double om2l = (1. - 2. * lambda);
    md_update_momenta(s, U, P, lambda * dtau);
    for (int i = 0; i < nsteps - 1; i++) {
      md_update_gauge(s, U, P, 0.5 * dtau);
      md_update_momenta(s, U, P, om2l * dtau);
      md_update_gauge(s, U, P, 0.5 * dtau);
      md_update_momenta(s, U, P, 2 * lambda * dtau);
    }
    md_update_gauge(s, U, P, 0.5 * dtau);
    md_update_momenta(s, U, P, om2l * dtau);
    md_update_gauge(s, U, P, 0.5 * dtau);
    md_update_momenta(s, U, P, lambda * dtau);
  } else if (integ == 2 || integ == 3) { /* omf4, lp_omf4 */
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
    md_update_momenta(s, U, P, 0.5 * eps[9]);
    for (int i = 1; i < nsteps - 1; i++)
      for (int j = 0; j < 5; j++) {
        md_update_gauge(s, U, P, eps[2 * j]);
        md_update_momenta(s, U, P, eps[2 * j + 1]);
      }
    for (int j = 0; j < 4; j++) {
      md_update_gauge(s, U, P, eps[2 * j]);
      md_update_momenta(s, U, P, eps[2 * j + 1]);
    }
    md_update_gauge(s, U, P, eps[8]);
    md_update_momenta(s, U, P, 0.5 * eps[9]);
  } else if (integ == 4) { /* euler */
    for (int i = 0; i < nsteps; i++) {
      md_update_momenta(s, U, P, dtau);
      md_update_gauge(s, U, P, dtau);
    }
  } else if (integ == 5) { /* ruth */
    for (int i = 0; i < nsteps; i++) {
      md_update_momenta(s, U, P, dtau);
      md_update_gauge(s, U, P, -1. / 24. * dtau);
      md_update_momenta(s, U, P, -2. / 3. * dtau);
      md_update_gauge(s, U, P, 3. / 4. * dtau);
      md_update_momenta(s, U, P, 2. / 3. * dtau);
      md_update_gauge(s, U, P, 7. / 24. * dtau);
    }
  } else { /* leapfrog (also the reference's fallback for unknown ids) */
    md_update_momenta(s, U, P, dtau / 2.);
    md_update_gauge(s, U, P, dtau);
    for (int i = 0; i < nsteps - 1; i++) {
      md_update_momenta(s, U, P, dtau);
      md_update_gauge(s, U, P, dtau);
    }
    md_update_momenta(s, U, P, dtau / 2.);
  }
  const lat_t *l = &s->l;
  orc_restore_su(s->group, (int)l->L[1], (int)l->L[2], (int)l->L[3], (int)l->L[0], l->nd, U);
}

static void integrate_r(int group, int Lx, int Ly, int Lz, int Lt, int nd, double beta,
                        double xi, int integ, int nsteps, double tau, double *U, double *P,
                        double dn) {
  md_sys s = {group, mklat(Lx, Ly, Lz, Lt, nd), beta, xi, 0, 0., 0., 0, NULL, dn};
  md_integrate(&s, integ, nsteps, tau, U, P);
}
void orc_integrate(int group, int Lx, int Ly, int Lz, int Lt, int nd, double beta, double xi,
                   int integ, int nsteps, double tau, double *U, double *P) {
  integrate_r(group, Lx, Ly, Lz, Lt, nd, beta, xi, integ, nsteps, tau, U, P, 0.);
}

/* adjointfield.hh:219-238: P*P */
static double pp(const double *P, size_t n) {
  double r = 0.;
  for (size_t i = 0; i < n; i++) r += P[i] * P[i];
  return r;
}
static double pp3(const double *P, size_t nl) {
  double r = 0.;
  for (size_t i = 0; i < nl; i++)
    r += P[3 * i] * P[3 * i] + P[3 * i + 1] * P[3 * i + 1] + P[3 * i + 2] * P[3 * i + 2];
  return r;
}
static double kinetic(int group, const double *P, size_t nl) {
  return 0.5 * (group == 0 ? pp3(P, nl) : pp(P, nl));
}

/* md_update.hh:18-61 with injected momenta, without the accept/reject */
static double md_injected_r(int group, int Lx, int Ly, int Lz, int Lt, int nd, double beta,
                            double xi, int integ, int nsteps, double tau, double *U, double *P,
                            double *H, double dn) {
  const lat_t l = mklat(Lx, Ly, Lz, Lt, nd);
  const int aniso = (xi != 1.0);
  H[0] = kinetic(group, P, nlinks(&l));
  H[1] = orc_S_G_hmc(group, Lx, Ly, Lz, Lt, nd, beta, U, xi, aniso);
  integrate_r(group, Lx, Ly, Lz, Lt, nd, beta, xi, integ, nsteps, tau, U, P, dn);
  H[2] = kinetic(group, P, nlinks(&l));
  H[3] = orc_S_G_hmc(group, Lx, Ly, Lz, Lt, nd, beta, U, xi, aniso);
  double dH = 0.;
  dH += H[2] - H[0];
  dH += H[3] - H[1];
  return dH;
}
double orc_md_injected(int group, int Lx, int Ly, int Lz, int Lt, int nd, double beta,
                       double xi, int integ, int nsteps, double tau, double *U, double *P,
                       double *H) {
  return md_injected_r(group, Lx, Ly, Lz, Lt, nd, beta, xi, integ, nsteps, tau, U, P, H, 0.);
}
/* md_injected with a low-precision integrator (1 or 3): N = pow(10, exponent) converted to
 * size_t as integrator.hh:59,168 does, so dn = 10^exponent exactly for exponent <= 19 */
double orc_md_injected_lp(int group, int Lx, int Ly, int Lz, int Lt, int nd, double beta,
                          double xi, int integ, int nsteps, double tau, double *U, double *P,
                          double *H, int exponent) {
  const double dn = (double)(size_t)pow(10, exponent);
  return md_injected_r(group, Lx, Ly, Lz, Lt, nd, beta, xi, integ, nsteps, tau, U, P, H, dn);
}

/* initnormal (adjointfield.hh:240-258) from std::mt19937(seed) + the next uniform draw */
double orc_initnormal(int group, int Lx, int Ly, int Lz, int Lt, int nd, long seed, double *P) {
  const lat_t l = mklat(Lx, Ly, Lz, Lt, nd);
  orc_mt19937 g;
  orc_mt_seed(&g, (uint32_t)seed);
  normal_dist n = {0., 1., 0., 0};
  const size_t na = group == 0 ? 3 : 1;
  for (size_t i = 0; i < nlinks(&l) * na; i++) P[i] = normal_draw(&n, &g);
  return uniform_ab(&g, 0., 1.);
}

/* hmc.hpp:86-101 + md_update.hh:18-81 (gauge monomial only, no reversibility test) */
void orc_hmc_run(int group, int Lx, int Ly, int Lz, int Lt, int nd, double beta, double xi,
                 int integ, int nsteps, double tau, long seed, int i0, int ntraj, double *U,
                 int *acc, double *dH, double *plaq) {
  const lat_t l = mklat(Lx, Ly, Lz, Lt, nd);
  const size_t N = nlinks(&l), na = group == 0 ? 3 : 1, nu = group == 0 ? 4 : 1;
  double *P = malloc(N * na * sizeof(double));
  double *U_old = malloc(N * nu * sizeof(double));
  for (int k = 0; k < ntraj; k++) {
    const size_t i = (size_t)(i0 + k);
    orc_mt19937 g;
    orc_mt_seed(&g, (uint32_t)((size_t)seed + i));
    normal_dist n = {0., 1., 0., 0};
    for (size_t j = 0; j < N * na; j++) P[j] = normal_draw(&n, &g);
    memcpy(U_old, U, N * nu * sizeof(double));
    double H[4];
    const double d = orc_md_injected(group, Lx, Ly, Lz, Lt, nd, beta, xi, integ, nsteps, tau, U,
                                     P, H);
    int accept = 1;
    if (d > 0) {
      if (uniform_ab(&g, 0., 1.) > exp(-d)) accept = 0;
    }
    if (!accept) memcpy(U, U_old, N * nu * sizeof(double));
    acc[k] = accept;
    dH[k] = d;
    plaq[k] = orc_gauge_energy(group, Lx, Ly, Lz, Lt, nd, U, 0);
  }
  free(P);
  free(U_old);
}

/* U(1) gauge + staggered pseudofermion trajectory with injected P and R; dn > 0 rounds as
 * the low-precision integrators do (the summed gauge + fermion derivative and the links) */
static double md_injected_fermion_r(int Lx, int Ly, int Lz, int Lt, int nd, double beta,
                                    double m, double tol, long seed, int integ, int nsteps,
                                    double tau, double *U, double *P, const double *R,
                                    double *H, double dn) {
  const lat_t l = mklat(Lx, Ly, Lz, Lt, nd);
  double *phi = malloc(2 * l.V * sizeof(double));
  apply_D_or_Ddag(&l, U, m, 0, R, phi);
  H[0] = kinetic(1, P, nlinks(&l));
  H[1] = orc_S_G_hmc(1, Lx, Ly, Lz, Lt, nd, beta, U, 1.0, 0);
  H[2] = vdot(l.V, R, R).r;
  md_sys s = {1, l, beta, 1.0, 1, m, tol, seed, phi, dn};
  md_integrate(&s, integ, nsteps, tau, U, P);
  H[3] = kinetic(1, P, nlinks(&l));
  H[4] = orc_S_G_hmc(1, Lx, Ly, Lz, Lt, nd, beta, U, 1.0, 0);
  H[5] = orc_fermion_accept(Lx, Ly, Lz, Lt, nd, U, m, phi, tol, seed);
  free(phi);
  double dH = 0.;
  dH += H[3] - H[0];
  dH += H[4] - H[1];
  dH += H[5] - H[2];
  return dH;
}
double orc_md_injected_fermion(int Lx, int Ly, int Lz, int Lt, int nd, double beta, double m,
                               double tol, long seed, int integ, int nsteps, double tau,
                               double *U, double *P, const double *R, double *H) {
  return md_injected_fermion_r(Lx, Ly, Lz, Lt, nd, beta, m, tol, seed, integ, nsteps, tau, U, P,
                               R, H, 0.);
}
/* the same with a low-precision integrator (1 or 3) and N = pow(10, exponent) as a size_t
 * (integrator.hh:59,168) */
double orc_md_injected_fermion_lp(int Lx, int Ly, int Lz, int Lt, int nd, double beta,
                                  double m, double tol, long seed, int integ, int nsteps,
                                  double tau, double *U, double *P, const double *R, double *H,
                                  int exponent) {
  const double dn = (double)(size_t)pow(10, exponent);
  return md_injected_fermion_r(Lx, Ly, Lz, Lt, nd, beta, m, tol, seed, integ, nsteps, tau, U, P,
                               R, H, dn);
}

/* ===================================================================================== */
/* clover energy density and topological charge (flat-energy_density.hh:57-164)           */
/* ===================================================================================== */

/* Levi-Civita entries (tensors.hh:23-58): permutations of {0,1,2,3} with sign */
static int eps4_N = 0;
static int eps4_idx[24][4];
static double eps4_val[24];
static void eps4_init(void) {
  if (eps4_N) return;
  int k = 0;
  for (int i1 = 1; i1 <= 4; i1++)
    for (int i2 = 1; i2 <= 4; i2++)
      for (int i3 = 1; i3 <= 4; i3++)
        for (int i4 = 1; i4 <= 4; i4++) {
          const int p = (i1 - i2) * (i1 - i3) * (i1 - i4) * (i2 - i3) * (i2 - i4) * (i3 - i4);
          if (p != 0) {
            eps4_val[k] = p > 0 ? 1 : -1;
            eps4_idx[k][0] = i1 - 1;
            eps4_idx[k][1] = i2 - 1;
            eps4_idx[k][2] = i3 - 1;
            eps4_idx[k][3] = i4 - 1;
            k++;
          }
        }
  eps4_N = k;
}

static void add4(long *d, const long *s) {
  for (int i = 0; i < 4; i++) d[i] = s[i];
}

void orc_energy_density(int group, int Lx, int Ly, int Lz, int Lt, int nd, const double *U,
                        int cloverdef, int ss, double *E, double *Q) {
  const lat_t l = mklat(Lx, Ly, Lz, Lt, nd);
  eps4_init();
  const int mu_start = ss ? 1 : 0;
  double res = 0., q = 0.;
  for (size_t s = 0; s < l.V; s++) {
    long c[4], x1[4], x2[4], x3[4];
    coords(&l, s, c);
    add4(x1, c);
    add4(x2, c);
    add4(x3, c);
    su2 G[4][4];
    double g1[4][4]; /* U(1): G = i*g */
    memset(G, 0, sizeof(G));
    memset(g1, 0, sizeof(g1));
    for (int mu = mu_start; mu < nd - 1; mu++)
      for (int nu = mu + 1; nu < nd; nu++) {
        x1[mu] += 1;
        x2[nu] += 1;
        if (group == 0) {
          su2 leaf = smul(smul(smul(sload(U, link(&l, c, mu)), sload(U, link(&l, x1, nu))),
                               sdag(sload(U, link(&l, x2, mu)))),
                          sdag(sload(U, link(&l, c, nu))));
          x1[mu] -= 1;
          x2[nu] -= 1;
          if (cloverdef) {
            x1[mu] -= 1;
            x1[nu] += 1;
            x2[mu] -= 1;
            leaf = sadd(leaf, smul(smul(smul(sload(U, link(&l, c, nu)),
                                             sdag(sload(U, link(&l, x1, mu)))),
                                        sdag(sload(U, link(&l, x2, nu)))),
                                   sload(U, link(&l, x2, mu))));
            x1[mu] += 1;
            x1[nu] -= 1;
            x2[mu] += 1;

            x1[mu] -= 1;
            x2[mu] -= 1;
            x2[nu] -= 1;
            x3[nu] -= 1;
            leaf = sadd(leaf, smul(smul(smul(sdag(sload(U, link(&l, x1, mu))),
                                             sdag(sload(U, link(&l, x2, nu)))),
                                        sload(U, link(&l, x2, mu))),
                                   sload(U, link(&l, x3, nu))));
            x1[mu] += 1;
            x2[mu] += 1;
            x2[nu] += 1;
            x3[nu] += 1;

            x1[nu] -= 1;
            x2[nu] -= 1;
            x2[mu] += 1;
            leaf = sadd(leaf, smul(smul(smul(sdag(sload(U, link(&l, x1, nu))),
                                             sload(U, link(&l, x1, mu))),
                                        sload(U, link(&l, x2, nu))),
                                   sdag(sload(U, link(&l, c, mu)))));
            x1[nu] += 1;
            x2[nu] += 1;
            x2[mu] -= 1;
          }
          G[mu][nu] = stla(leaf);
          res += sretr(smul(G[mu][nu], G[mu][nu]));
        } else {
          cplx leaf = cexpi(((U[link(&l, c, mu)] + U[link(&l, x1, nu)]) +
                             (-U[link(&l, x2, mu)])) +
                            (-U[link(&l, c, nu)]));
          x1[mu] -= 1;
          x2[nu] -= 1;
          if (cloverdef) {
            x1[mu] -= 1;
            x1[nu] += 1;
            x2[mu] -= 1;
            leaf = cadd(leaf, cexpi(((U[link(&l, c, nu)] + (-U[link(&l, x1, mu)])) +
                                     (-U[link(&l, x2, nu)])) +
                                    U[link(&l, x2, mu)]));
            x1[mu] += 1;
            x1[nu] -= 1;
            x2[mu] += 1;

            x1[mu] -= 1;
            x2[mu] -= 1;
            x2[nu] -= 1;
            x3[nu] -= 1;
            leaf = cadd(leaf, cexpi((((-U[link(&l, x1, mu)]) + (-U[link(&l, x2, nu)])) +
                                     U[link(&l, x2, mu)]) +
                                    U[link(&l, x3, nu)]));
            x1[mu] += 1;
            x2[mu] += 1;
            x2[nu] += 1;
            x3[nu] += 1;

            x1[nu] -= 1;
            x2[nu] -= 1;
            x2[mu] += 1;
            leaf = cadd(leaf, cexpi((((-U[link(&l, x1, nu)]) + U[link(&l, x1, mu)]) +
                                     U[link(&l, x2, nu)]) +
                                    (-U[link(&l, c, mu)])));
            x1[nu] += 1;
            x2[nu] += 1;
            x2[mu] -= 1;
          }
          g1[mu][nu] = leaf.i; /* u1.hh:201-203 */
          res += cmul(C(0., leaf.i), C(0., leaf.i)).r;
        }
      }
    if (nd == 4) {
      for (int k = 0; k < eps4_N; k++) {
        const int i1 = eps4_idx[k][0], i2 = eps4_idx[k][1], i3 = eps4_idx[k][2],
                  i4 = eps4_idx[k][3];
        if (i2 < i1) continue;
        if (i4 < i3) continue;
        const double tr = group == 0
                            ? sretr(smul(G[i1][i2], G[i3][i4]))
                            : cmul(C(0., g1[i1][i2]), C(0., g1[i3][i4])).r;
        q += eps4_val[k] * tr;
      }
    }
    if (nd == 2) {
      /* su2 trace is real (su2.hh:77-80); U(1) trace is the identity (u1.hh:193-195) */
      if (group == 1) q += -(g1[0][1] - g1[1][0]);
    }
  }
  res = -res / (double)l.V;
  if (cloverdef) res /= 16.;
  q = -4. * q / (32.0 * M_PI * M_PI);
  if (cloverdef) q /= 16.;
  *E = res;
  *Q = q;
}

/* ===================================================================================== */
/* Wilson gradient flow (flat-gradient_flow.hh)                                           */
/* ===================================================================================== */

/* flat-gradient_flow.hh:17-50 */
void orc_runge_kutta(int group, int Lx, int Ly, int Lz, int Lt, int nd, double beta,
                     double xi, double eps, double *U) {
  const lat_t l = mklat(Lx, Ly, Lz, Lt, nd);
  const double zfac[3] = {(-17.0) / (36.0), (8.0) / (9.0), (-3.0) / (4.0)};
  const double expfac[3] = {-36.0 / 4. / 17.0, 1., -1.};
  const size_t na = group == 0 ? 3 : 1;
  const int Nc = group == 0 ? 2 : 1;
  double *Z = calloc(nlinks(&l) * na, sizeof(double));
  for (int f = 0; f < 3; f++) {
    orc_gauge_derivative(group, Lx, Ly, Lz, Lt, nd, beta, xi, U, 2. * Nc * zfac[f] / beta, Z);
    orc_update_gauge(group, Lx, Ly, Lz, Lt, nd, U, Z, -eps * expfac[f]);
  }
  free(Z);
}

/* flat-gradient_flow.hh:70-197 */
int orc_gradient_flow(int group, int Lx, int Ly, int Lz, int Lt, int nd, double beta,
                      double xi, const double *U0, double tmax, double eps, double tstart,
                      double *rows, int max_rows) {
  const lat_t l = mklat(Lx, Ly, Lz, Lt, nd);
  const size_t d = (size_t)nd;
  const double ndims_fact = (double)(d * (d - 1)) / 2.0;
  const double ndims_fact_ss = (double)((d - 1) * (d - 2)) / 2.0;
  const double Nc = group == 0 ? 2. : 1.;
  const double den = (double)l.V * Nc;
  const size_t nu = group == 0 ? 4 : 1;
  double *Vt = malloc(nlinks(&l) * nu * sizeof(double));
  memcpy(Vt, U0, nlinks(&l) * nu * sizeof(double));
  double t[3] = {tstart, tstart, tstart}, P[3] = {0}, E[3] = {0}, Q[3] = {0}, P_ss[3] = {0},
         E_ss[3] = {0};
  double dens, topQ, dens_ss, topQ_ss;
  P[2] = orc_gauge_energy(group, Lx, Ly, Lz, Lt, nd, Vt, 0) / den;
  P_ss[2] = orc_gauge_energy(group, Lx, Ly, Lz, Lt, nd, Vt, 1) / den;
  orc_energy_density(group, Lx, Ly, Lz, Lt, nd, Vt, 1, 0, &dens, &topQ);
  E[2] = dens;
  orc_energy_density(group, Lx, Ly, Lz, Lt, nd, Vt, 1, 1, &dens_ss, &topQ_ss);
  E_ss[2] = dens_ss;
  int nrows = 0;
  while (t[1] < tmax - eps) {
    t[0] = t[2];
    P[0] = P[2];
    E[0] = E[2];
    Q[0] = Q[2];
    P_ss[0] = P_ss[2];
    E_ss[0] = E_ss[2];
    for (int x0 = 1; x0 < 3; x0++) {
      t[x0] = t[x0 - 1] + eps;
      orc_runge_kutta(group, Lx, Ly, Lz, Lt, nd, beta, xi, eps, Vt);
      P[x0] = orc_gauge_energy(group, Lx, Ly, Lz, Lt, nd, Vt, 0) / den;
      P_ss[x0] = orc_gauge_energy(group, Lx, Ly, Lz, Lt, nd, Vt, 1) / den;
      orc_energy_density(group, Lx, Ly, Lz, Lt, nd, Vt, 1, 0, &dens, &topQ);
      E[x0] = dens;
      Q[x0] = topQ;
      orc_energy_density(group, Lx, Ly, Lz, Lt, nd, Vt, 1, 1, &dens_ss, &topQ_ss);
      E_ss[x0] = dens_ss;
    }
    const double Ep = ndims_fact - P[1];
    const double Ep_ss = ndims_fact_ss - P_ss[1];
    const double Ep_ts = Ep - Ep_ss;
    const double Ep_ts_bar = Ep_ts / (double)(d - 1);
    const double Ep_ss_bar = Ep_ss / ndims_fact_ss;
    const double xi_R = sqrt(Ep_ts_bar / Ep_ss_bar);
    if (nrows < max_rows) {
      double *r = rows + 9 * nrows;
      r[0] = t[1];
      r[1] = xi_R;
      r[2] = P[1];
      r[3] = P_ss[1];
      r[4] = Ep;
      r[5] = Ep_ss;
      r[6] = E[1];
      r[7] = E_ss[1];
      r[8] = Q[1];
    }
    nrows++;
  }
  free(Vt);
  return nrows;
}

/* ===================================================================================== */
/* the device library's own random streams and Metropolis order                          */
/* ===================================================================================== */

/* momenta: per link l (reference link order), draws j = 0, 1 give 4 normals */
void orc_philox_momenta(int group, int Lx, int Ly, int Lz, int Lt, int nd, uint64_t seed,
                        uint32_t traj, double *P) {
  const lat_t l = mklat(Lx, Ly, Lz, Lt, nd);
  for (size_t i = 0; i < nlinks(&l); i++) {
    uint32_t r[4];
    double n0, n1, n2, n3;
    philox_draw(seed, (uint32_t)i, 0u, traj, TAG_MOMENTA, r);
    box_muller(u01_53(r[0], r[1]), u01_53(r[2], r[3]), &n0, &n1);
    if (group == 0) {
      philox_draw(seed, (uint32_t)i, 1u, traj, TAG_MOMENTA, r);
      box_muller(u01_53(r[0], r[1]), u01_53(r[2], r[3]), &n2, &n3);
      P[3 * i] = n0;
      P[3 * i + 1] = n1;
      P[3 * i + 2] = n2;
    } else
      P[i] = n0;
  }
}

double orc_philox_accept_uniform(uint64_t seed, uint32_t traj) {
  uint32_t r[4];
  philox_draw(seed, 0u, 0u, traj, TAG_ACCEPT, r);
  return u01_53(r[0], r[1]) - 0x1p-53; /* [0,1) */
}

/* pseudofermion source R: sigma = 1/sqrt(2) per real component */
void orc_philox_pf_source(int Lx, int Ly, int Lz, int Lt, uint64_t seed, uint32_t traj,
                          int complex_source, double *R) {
  const size_t V = (size_t)Lx * Ly * Lz * Lt;
  const double s = 1.0 / sqrt(2.0);
  for (size_t i = 0; i < V; i++) {
    uint32_t r[4];
    double n0, n1;
    philox_draw(seed, (uint32_t)i, 0u, traj, TAG_PF, r);
    box_muller(u01_53(r[0], r[1]), u01_53(r[2], r[3]), &n0, &n1);
    R[2 * i] = s * n0;
    R[2 * i + 1] = complex_source ? s * n1 : 0.;
  }
}

/* Site-parity checkerboard sweep: for mu, for parity p, every link (x, mu) with
 * parity(x) = p gets N_hit proposals U -> U R (flat-sweep.hh:97-117 update rule). */
void orc_metropolis_checkerboard(int group, int Lx, int Ly, int Lz, int Lt, int nd,
                                 double beta, double xi, double delta, int N_hit, uint64_t seed,
                                 uint32_t sweep, double *U, double *rates) {
  const lat_t l = mklat(Lx, Ly, Lz, Lt, nd);
  const double Nc = group == 0 ? 2. : 1.;
  long rate = 0, rate_t = 0;
  for (int mu = 0; mu < nd; mu++)
    for (int p = 0; p < 2; p++)
      for (size_t s = 0; s < l.V; s++) {
        long c[4];
        coords(&l, s, c);
        if (((c[0] + c[1] + c[2] + c[3]) & 1) != p) continue;
        const size_t i = link(&l, c, mu);
        if (group == 0) {
          const su2 K = staples_su2(&l, U, c, mu, xi, xi != 1.0);
          su2 u = sload(U, i);
          for (int n = 0; n < N_hit; n++) {
            uint32_t r[4];
            philox_draw(seed, (uint32_t)i, (uint32_t)n, sweep, TAG_METRO, r);
            const double alpha = 2.0 * M_PI * delta * u01_32(r[0]);
            const double uu = 2.0 * u01_32(r[1]) - 1.0;
            const double theta = 2.0 * M_PI * u01_32(r[2]);
            const double sa = sin(alpha), rr = sqrt(1 - uu * uu);
            su2 R;
            R.a = C(cos(alpha), sa * uu);
            R.b = C(sa * rr * sin(theta), sa * rr * cos(theta));
            const double dS =
              beta / Nc * (sretr(smul(u, K)) - sretr(smul(smul(u, R), K)));
            int acc = (dS < 0);
            if (!acc) acc = (u01_32(r[3]) < exp(-dS));
            if (acc) {
              u = srestore(smul(u, R));
              rate++;
              if (mu == 0) rate_t++;
            }
          }
          sstore(U, i, u);
        } else {
          const cplx K = staples_u1(&l, U, c, mu, xi, xi != 1.0);
          double u = U[i];
          for (int n = 0; n < N_hit; n++) {
            uint32_t r[4];
            philox_draw(seed, (uint32_t)i, (uint32_t)n, sweep, TAG_METRO, r);
            const double th = M_PI * delta * (2.0 * u01_32(r[0]) - 1.0);
            const double dS = beta / Nc * (cmul(cexpi(u), K).r - cmul(cexpi(u + th), K).r);
            int acc = (dS < 0);
            if (!acc) acc = (u01_32(r[1]) < exp(-dS));
            if (acc) {
              u = u + th;
              rate++;
              if (mu == 0) rate_t++;
            }
          }
          U[i] = u;
        }
      }
  rates[0] = (double)rate / (double)N_hit / (double)nlinks(&l);
  rates[1] = (double)rate_t / (double)N_hit / (double)l.V;
}
