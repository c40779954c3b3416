// gauge.cu -- gauge-field kernels of libsu2b: layout conversion, plaquette reductions, the
// fused staple/force/momentum kernel, link update, reunitarisation, Philox momenta, the
// deterministic final reduction and the HMC accept/reject.
//
// Roofline per link (FP64 / FP32 storage), algorithmic bytes:
//   force+momentum  read U 32/16, read+write P 48/24            = 80 / 40 B
//   link update     read P 24/12, read+write U 64/32            = 88 / 44 B
//   plaquette       read U once                                 = 32 / 16 B
#include "site_ops.cuh"

namespace su2b {

namespace {

inline int cdiv(long a, long b) { return (int)((a + b - 1) / b); }

// ------------------------------------------------------------------------------------
// layout conversion: thread i walks the reference order i = lex*nd + mu
template <class T>
__global__ void k_links_from_host_su2(Geom g, const double *__restrict__ aos, LinkT<T> *U) {
  const long n = (long)g.V * g.nd;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x) {
    const int lex = (int)(i / g.nd), mu = (int)(i - (long)lex * g.nd);
    const Site s = site_from_lex(g, lex);
    const double *src = aos + 4 * i;
    Su2<double> u{src[0], src[1], src[2], src[3]};
    st_link(U + (size_t)mu * g.V + eo_of(g, lex, s.p), from64<T>(u));
  }
}
template <class T>
__global__ void k_links_to_host_su2(Geom g, const LinkT<T> *__restrict__ U, double *aos) {
  const long n = (long)g.V * g.nd;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x) {
    const int lex = (int)(i / g.nd), mu = (int)(i - (long)lex * g.nd);
    const Site s = site_from_lex(g, lex);
    const Su2<double> u = to64(ld_link_rw(U + (size_t)mu * g.V + eo_of(g, lex, s.p)));
    double *dst = aos + 4 * i;
    dst[0] = u.ar;
    dst[1] = u.ai;
    dst[2] = u.br;
    dst[3] = u.bi;
  }
}
// U(1) angles and adjoint fields: na reals per link, SoA on the device
template <class T>
__global__ void k_adj_from_host(Geom g, const double *__restrict__ aos, T *P, int na) {
  const long n = (long)g.V * g.nd;
  const size_t NL = (size_t)g.V * g.nd;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x) {
    const int lex = (int)(i / g.nd), mu = (int)(i - (long)lex * g.nd);
    const Site s = site_from_lex(g, lex);
    const size_t l = (size_t)mu * g.V + eo_of(g, lex, s.p);
    for (int k = 0; k < na; k++) P[k * NL + l] = (T)aos[na * i + k];
  }
}
template <class T>
__global__ void k_adj_to_host(Geom g, const T *__restrict__ P, double *aos, int na) {
  const long n = (long)g.V * g.nd;
  const size_t NL = (size_t)g.V * g.nd;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x) {
    const int lex = (int)(i / g.nd), mu = (int)(i - (long)lex * g.nd);
    const Site s = site_from_lex(g, lex);
    const size_t l = (size_t)mu * g.V + eo_of(g, lex, s.p);
    for (int k = 0; k < na; k++) aos[na * i + k] = (double)P[k * NL + l];
  }
}
__global__ void k_spinor_from_host(Geom g, const double2 *__restrict__ aos, double2 *psi) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.V; i += gridDim.x * blockDim.x) {
    const Site s = site_from_lex(g, i);
    psi[eo_of(g, i, s.p)] = aos[i];
  }
}
__global__ void k_spinor_to_host(Geom g, const double2 *__restrict__ psi, double2 *aos) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.V; i += gridDim.x * blockDim.x) {
    const Site s = site_from_lex(g, i);
    aos[i] = psi[eo_of(g, i, s.p)];
  }
}

// ------------------------------------------------------------------------------------
// plaquettes: per site, sum over planes mu<nu of ReTr U_mu(x) U_nu(x+mu) U_mu(x+nu)^+ U_nu(x)^+
// (flat-gauge_energy.hpp:31-94), FP64 products.  Partials {full, spatial, xi-weighted}.
template <class T, int ND, int NT>
__global__ void __launch_bounds__(NT)
  k_plaq_su2(Geom g, const LinkT<T> *__restrict__ U, double xi, double *part) {
  __shared__ double sh[NT / 32];
  const int w = threadIdx.x >> 5, p = w & 1;
  const int cb = blockIdx.x * (NT / 2) + (w >> 1) * 32 + (threadIdx.x & 31);
  double full = 0., spat = 0., wsum = 0.;
  if (cb < g.Vh) plaq_site<T, ND>(g, U, p, cb, xi, full, spat, wsum);
  const int b = blockIdx.x;
  double r = block_sum<NT>(full, sh);
  if (threadIdx.x == 0) part[3 * b] = r;
  r = block_sum<NT>(spat, sh);
  if (threadIdx.x == 0) part[3 * b + 1] = r;
  r = block_sum<NT>(wsum, sh);
  if (threadIdx.x == 0) part[3 * b + 2] = r;
}

template <int ND, int NT>
__global__ void __launch_bounds__(NT)
  k_plaq_u1(Geom g, const double *__restrict__ U, double xi, double *part) {
  __shared__ double sh[NT / 32];
  const int w = threadIdx.x >> 5, p = w & 1;
  const int cb = blockIdx.x * (NT / 2) + (w >> 1) * 32 + (threadIdx.x & 31);
  double full = 0., spat = 0., wsum = 0.;
  if (cb < g.Vh) {
    const Site s = site_from_eo(g, p, cb);
    double u[ND];
#pragma unroll
    for (int mu = 0; mu < ND; mu++) u[mu] = U[(size_t)mu * g.V + p * g.Vh + cb];
#pragma unroll
    for (int mu = 0; mu < ND - 1; mu++) {
      const int lpm = s.lex + fwd(g, s, mu);
#pragma unroll
      for (int nu = mu + 1; nu < ND; nu++) {
        const int lpn = s.lex + fwd(g, s, nu);
        const double A = U[(size_t)nu * g.V + eo_of(g, lpm, 1 - p)];
        const double B = U[(size_t)mu * g.V + eo_of(g, lpn, 1 - p)];
        const double tr = cos(((u[mu] + A) + (-B)) + (-u[nu]));
        full += tr;
        if (mu >= 1) spat += tr;
        wsum += (((mu == 0) ^ (nu == 0)) ? 1.0 / xi : xi) * tr;
      }
    }
  }
  const int b = blockIdx.x;
  double r = block_sum<NT>(full, sh);
  if (threadIdx.x == 0) part[3 * b] = r;
  r = block_sum<NT>(spat, sh);
  if (threadIdx.x == 0) part[3 * b + 1] = r;
  r = block_sum<NT>(wsum, sh);
  if (threadIdx.x == 0) part[3 * b + 2] = r;
}

template <int NT>
__global__ void __launch_bounds__(NT)
  k_reduce_final(const double *__restrict__ part, int n, int ncomp, double *out) {
  __shared__ double sh[NT / 32];
  for (int k = 0; k < ncomp; k++) {
    double v = 0.;
    for (int b = threadIdx.x; b < n; b += NT) v += part[(size_t)b * ncomp + k];
    const double r = block_sum<NT>(v, sh);
    if (threadIdx.x == 0) out[k] = r;
  }
}

// fused staple/force/momentum(/link update) kernel: one thread per site, force_site body
template <class T, int ND, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB)
  k_force_su2(Geom g, const LinkT<T> *__restrict__ U, T *__restrict__ P,
              const T *__restrict__ extra, T f, T scale_, int mode, int aniso, T wt, T ws,
              double *kin_part, LinkT<T> *__restrict__ Uout, T dt_upd) {
  __shared__ double sh[NT / 32];
  // warps alternate between the parities of one band of NT/2 sites per parity, so the
  // +-z / +-y neighbours of a site are mostly the own links of another warp of the block
  const int w = threadIdx.x >> 5;
  const int p = w & 1;
  const int cb = blockIdx.x * (NT / 2) + (w >> 1) * 32 + (threadIdx.x & 31);
  double k2 = 0.;
  if (cb < g.Vh)
    k2 = force_site<T, ND>(g, U, P, extra, f, scale_, mode, aniso, wt, ws, Uout, dt_upd, p, cb);
  if (mode & FM_KINETIC) {
    const double r = block_sum<NT>(k2, sh);
    if (threadIdx.x == 0) kin_part[blockIdx.x] = r;
  }
}

// The same fused force step (d = 4) with the links staged in shared memory, 2.5D-blocked.
// A block owns a BX x BY x BZ brick of (x, y, z) and marches along t over a contiguous range
// of (brick, t) units; the units of the whole lattice are split evenly over the resident
// blocks, so the grid is one wave.  Three time slices (t-1, t, t+1) of the brick with a
// one-site halo in x, y and z are held in shared memory as a ring; moving to t+1 loads one
// new slice (cp.async, periodic wrap) into the slot of t-2.  Every staple of the site is then
// read from shared memory: each link crosses L2 -> SM about (BX+2)(BY+2)(BZ+2)/(BX BY BZ)
// times per launch instead of the 11 times of the gather kernel.
// Two threads share a site: half h updates the links mu = 2h, 2h+1.  The forward product A
// of a plane inside the half is shared by its two links; the four planes that cross the halves
// compute A in both (64 FMAs more per site), which halves the registers per thread and gives
// twice the warps for the same brick.
namespace tile {
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}
__device__ __forceinline__ int wrap(int c, int L) { return c < 0 ? c + L : (c >= L ? c - L : c); }
}  // namespace tile

template <int BX, int BY, int BZ> struct Brick {
  static constexpr int NS = BX * BY * BZ;  // sites per slice
  static constexpr int NT = 2 * NS;        // threads
  static constexpr int HY = BY + 2, HZ = BZ + 2, H = (BX + 2) * HY * HZ;
};

template <class T, int BX, int BY, int BZ> constexpr size_t tile_smem() {
  return (size_t)4 * 4 * Brick<BX, BY, BZ>::H * sizeof(LinkT<T>) +
         (size_t)Brick<BX, BY, BZ>::H * sizeof(int);
}

template <class T, int BX, int BY, int BZ, int HALF, bool ANISO>
__device__ __forceinline__ double tile_site(const Geom &g, const float4 *sm, const int slot[4],
                                            int hc, size_t self, T *__restrict__ P,
                                            const T *__restrict__ extra, T f, T scale_,
                                            int mode, T wt, T ws,
                                            LinkT<T> *__restrict__ Uout, T dt_upd) {
  using B = Brick<BX, BY, BZ>;
  constexpr int W = (int)(sizeof(LinkT<T>) / 16);
  // link U_mu at offset (dt, dx, dy, dz) from the site, dt in {-1, 0, 1}
  auto L = [&](int mu, int dt, int dx, int dy, int dz) -> Su2<T> {
    const float4 *q = sm + ((size_t)(slot[dt + 1] * 4 + mu) * B::H + hc + (dx * B::HY + dy) * B::HZ + dz) * W;
    if constexpr (W == 1) {
      const float4 v = *q;
      return Su2<T>{(T)v.x, (T)v.y, (T)v.z, (T)v.w};
    } else {
      const double2 a = *reinterpret_cast<const double2 *>(q);
      const double2 b = *reinterpret_cast<const double2 *>(q + 1);
      return Su2<T>{(T)a.x, (T)a.y, (T)b.x, (T)b.y};
    }
  };
  // unit offset of direction d (0 = t, 1 = x, 2 = y, 3 = z)
  auto E = [](int d, int k) { return d == k ? 1 : 0; };
  constexpr int m0 = 2 * HALF, m1 = 2 * HALF + 1;
  Su2<T> K[2] = {zero_su2<T>(), zero_su2<T>()};
  // forward staples: U_nu(x+mu) U_mu(x+nu)^+ U_nu(x)^+
#pragma unroll
  for (int j = 0; j < 2; j++) {
    const int mu = m0 + j;
#pragma unroll
    for (int nu = 0; nu < 4; nu++) {
      if (nu == mu) continue;
      const bool both = (nu == m0 || nu == m1);
      if (both && nu < mu) continue;  // the plane was done from the other link
      const Su2<T> a = L(nu, E(mu, 0), E(mu, 1), E(mu, 2), E(mu, 3));  // U_nu(x+mu)
      const Su2<T> b = L(mu, E(nu, 0), E(nu, 1), E(nu, 2), E(nu, 3));  // U_mu(x+nu)
      Su2<T> A = mul(a, dag(b));
      if (ANISO) A = scale((mu == 0 || nu == 0) ? wt : ws, A);
      K[j] = mul_acc(K[j], A, dag(L(nu, 0, 0, 0, 0)));
      if (both) K[nu - m0] = mul_acc(K[nu - m0], dag(A), dag(L(mu, 0, 0, 0, 0)));
    }
  }
  // backward staples U_nu(x+mu-nu)^+ U_mu(x-nu)^+ U_nu(x-nu)
#pragma unroll
  for (int j = 0; j < 2; j++) {
    const int mu = m0 + j;
#pragma unroll
    for (int nu = 0; nu < 4; nu++) {
      if (nu == mu) continue;
      const Su2<T> e = L(nu, E(mu, 0) - E(nu, 0), E(mu, 1) - E(nu, 1), E(mu, 2) - E(nu, 2),
                         E(mu, 3) - E(nu, 3));
      const Su2<T> h = L(mu, -E(nu, 0), -E(nu, 1), -E(nu, 2), -E(nu, 3));
      const Su2<T> c = L(nu, -E(nu, 0), -E(nu, 1), -E(nu, 2), -E(nu, 3));
      Su2<T> eh = mul(dag(e), dag(h));
      if (ANISO) eh = scale((mu == 0 || nu == 0) ? wt : ws, eh);
      K[j] = mul_acc(K[j], eh, c);
    }
  }
  const size_t V = (size_t)g.V, NL = 4 * V;
  double k2 = 0.;
#pragma unroll
  for (int j = 0; j < 2; j++)
    k2 += finish_link<T>(L(m0 + j, 0, 0, 0, 0), K[j], (m0 + j) * V + self, NL, P, extra, f,
                         scale_, mode, Uout, dt_upd);
  return k2;
}

template <class T, int BX, int BY, int BZ, int MINB>
__global__ void __launch_bounds__(Brick<BX, BY, BZ>::NT, MINB)
  k_force_su2_tile(Geom g, const LinkT<T> *__restrict__ U, T *__restrict__ P,
                   const T *__restrict__ extra, T f, T scale_, int mode, int aniso, T wt, T ws,
                   double *kin_part, LinkT<T> *__restrict__ Uout, T dt_upd) {
  using B = Brick<BX, BY, BZ>;
  constexpr int W = (int)(sizeof(LinkT<T>) / 16);
  extern __shared__ float4 sm[];
  __shared__ double sh[B::NT / 32];
  // spatial part of every halo site of the brick: lexicographic offset within a time slice,
  // parity of x+y+z in bit 31
  int *soff = reinterpret_cast<int *>(sm + (size_t)4 * 4 * B::H * W);
  const int tid = threadIdx.x;
  const int half = tid / B::NS, sidx = tid % B::NS;
  const int sx = sidx / (BY * BZ), sy = (sidx / BZ) % BY, sz = sidx % BZ;
  const int hc = ((sx + 1) * B::HY + (sy + 1)) * B::HZ + (sz + 1);
  const int LT = g.L[0], LX = g.L[1], LY = g.L[2], LZ = g.L[3];
  const int V3 = LX * LY * LZ;
  const int nbx = LX / BX, nby = LY / BY, nbz = LZ / BZ;
  const long units = (long)nbx * nby * nbz * LT;
  const long u0 = units * blockIdx.x / gridDim.x, u1 = units * (blockIdx.x + 1) / gridDim.x;
  // copy time slice t of the brick (halo included) into ring slot sl
  auto load = [&](int sl, int t) {
    const int tb = t * V3;
#pragma unroll 2
    for (int i = tid; i < 4 * B::H * W; i += B::NT) {
      const int part = i % W, hm = i / W;
      const int mu = hm / B::H, h = hm % B::H;
      const int so = soff[h];
      const int lex = tb + (so & 0x7fffffff);
      const int eo = ((t + (int)((unsigned)so >> 31)) & 1) * g.Vh + (lex >> 1);
      tile::cp_async16(sm + ((size_t)(sl * 4 + mu) * B::H + h) * W + part,
                       reinterpret_cast<const float4 *>(U + (size_t)mu * g.V + eo) + part);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  // ring: slot[0..2] hold t-1, t, t+1; slot[3] receives t+2 while t is computed
  int slot[4] = {0, 1, 2, 3};
  long cur_brick = -1;
  double k2 = 0.;
  for (long u = u0; u < u1; u++) {
    const long brick = u / LT;
    const int t = (int)(u % LT);
    const int bz = (int)(brick % nbz), by = (int)((brick / nbz) % nby),
              bx = (int)(brick / (nbz * nby));
    const int x0 = bx * BX, y0 = by * BY, z0 = bz * BZ;
    if (brick != cur_brick) {
      tile::cp_async_wait_all();
      __syncthreads();  // nothing in flight or being read before the table and ring restart
      for (int h = tid; h < B::H; h += B::NT) {
        const int hz = h % B::HZ, hy = (h / B::HZ) % B::HY, hx = h / (B::HZ * B::HY);
        const int x = tile::wrap(x0 - 1 + hx, LX), y = tile::wrap(y0 - 1 + hy, LY),
                  z = tile::wrap(z0 - 1 + hz, LZ);
        soff[h] = ((x * LY + y) * LZ + z) | (int)((unsigned)((x + y + z) & 1) << 31);
      }
      __syncthreads();
      slot[0] = 0;
      slot[1] = 1;
      slot[2] = 2;
      slot[3] = 3;
      load(slot[0], tile::wrap(t - 1, LT));
      load(slot[1], t);
      load(slot[2], tile::wrap(t + 1, LT));
      cur_brick = brick;
    }
    load(slot[3], tile::wrap(t + 2, LT));            // prefetch, overlaps the compute of t
    asm volatile("cp.async.wait_group 1;\n" ::: "memory");  // all but the prefetch landed
    __syncthreads();
    const int x = x0 + sx, y = y0 + sy, z = z0 + sz;
    const int lex = t * V3 + (x * LY + y) * LZ + z;
    const size_t self = (size_t)((t + x + y + z) & 1) * g.Vh + (lex >> 1);
    if (half == 0)
      k2 += aniso ? tile_site<T, BX, BY, BZ, 0, true>(g, sm, slot, hc, self, P, extra, f, scale_,
                                                      mode, wt, ws, Uout, dt_upd)
                  : tile_site<T, BX, BY, BZ, 0, false>(g, sm, slot, hc, self, P, extra, f,
                                                       scale_, mode, wt, ws, Uout, dt_upd);
    else
      k2 += aniso ? tile_site<T, BX, BY, BZ, 1, true>(g, sm, slot, hc, self, P, extra, f, scale_,
                                                      mode, wt, ws, Uout, dt_upd)
                  : tile_site<T, BX, BY, BZ, 1, false>(g, sm, slot, hc, self, P, extra, f,
                                                       scale_, mode, wt, ws, Uout, dt_upd);
    __syncthreads();  // the slot of t-1 is free: it takes the prefetch of the next step
    const int fr = slot[0];
    slot[0] = slot[1];
    slot[1] = slot[2];
    slot[2] = slot[3];
    slot[3] = fr;
  }
  tile::cp_async_wait_all();
  if (mode & FM_KINETIC) {
    const double r = block_sum<B::NT>(k2, sh);
    if (threadIdx.x == 0) kin_part[blockIdx.x] = r;
  }
}

template <class T, int BX, int BY, int BZ>
bool tile_fits(const Geom &g) {
  return g.nd == 4 && g.L[1] % BX == 0 && g.L[2] % BY == 0 && g.L[3] % BZ == 0;
}

// resident blocks of a tile kernel on this device (one wave), cached per instantiation
template <class T, int BX, int BY, int BZ, int MINB> int tile_grid() {
  static int grid = 0;
  if (!grid) {
    int per_sm = 0, dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_force_su2_tile<T, BX, BY, BZ, MINB>,
                                                  Brick<BX, BY, BZ>::NT,
                                                  tile_smem<T, BX, BY, BZ>());
    grid = std::max(1, per_sm) * std::max(1, sms);
  }
  return grid;
}

template <int ND, int NT>
__global__ void __launch_bounds__(NT)
  k_force_u1(Geom g, const double *__restrict__ U, double *__restrict__ P,
             const double *__restrict__ extra, double f, double scale_, int mode, int aniso,
             double wt, double ws, double *kin_part) {
  __shared__ double sh[NT / 32];
  const int mu = blockIdx.y >> 1, p = blockIdx.y & 1;
  const int cb = blockIdx.x * NT + threadIdx.x;
  double k2 = 0.;
  if (cb < g.Vh) {
    const Site s = site_from_eo(g, p, cb);
    const int lpm = s.lex + fwd(g, s, mu);
    double Kr = 0., Ki = 0.;
#pragma unroll
    for (int nu = 0; nu < ND; nu++) {
      if (nu == mu) continue;
      const int lpn = s.lex + fwd(g, s, nu);
      const double A = U[(size_t)nu * g.V + eo_of(g, lpm, 1 - p)];
      const double B = U[(size_t)mu * g.V + eo_of(g, lpn, 1 - p)];
      const double D = U[(size_t)nu * g.V + eo_of(g, s.lex, p)];
      double sn, cs;
      sincos((A + (-B)) + (-D), &sn, &cs);
      const double w = aniso ? ((nu == 0 || mu == 0) ? wt : ws) : 1.0;
      Kr += w * cs;
      Ki += w * sn;
    }
#pragma unroll
    for (int nu = 0; nu < ND; nu++) {
      if (nu == mu) continue;
      const int b = bwd(g, s, nu);
      const double A = U[(size_t)nu * g.V + eo_of(g, lpm + b, p)];
      const double B = U[(size_t)mu * g.V + eo_of(g, s.lex + b, 1 - p)];
      const double D = U[(size_t)nu * g.V + eo_of(g, s.lex + b, 1 - p)];
      double sn, cs;
      sincos(((-A) + (-B)) + D, &sn, &cs);
      const double w = aniso ? ((nu == 0 || mu == 0) ? wt : ws) : 1.0;
      Kr += w * cs;
      Ki += w * sn;
    }
    const size_t l = (size_t)mu * g.V + (size_t)p * g.Vh + cb;
    double su, cu;
    sincos(U[l], &su, &cu);
    double d = f * (cu * Ki + su * Kr);  // Im(e^{i theta} K), adjointfield.hh:79-81
    if (mode & FM_EXTRA) d += extra[l];
    const double pn = (mode & FM_HAS_IN) ? P[l] + scale_ * d : scale_ * d;
    P[l] = pn;
    k2 = pn * pn;
  }
  if (mode & FM_KINETIC) {
    const double r = block_sum<NT>(k2, sh);
    if (threadIdx.x == 0) kin_part[blockIdx.y * gridDim.x + blockIdx.x] = r;
  }
}

// ------------------------------------------------------------------------------------
// U <- exp(dt P) U (update_gauge.hh:8-16)
template <class T>
__global__ void k_update_su2(size_t NL, LinkT<T> *__restrict__ U, const T *__restrict__ P,
                             T dt) {
  for (size_t l = blockIdx.x * (size_t)blockDim.x + threadIdx.x; l < NL;
       l += (size_t)gridDim.x * blockDim.x) {
    const Su2<T> e = exp_alg(dt * P[l], dt * P[NL + l], dt * P[2 * NL + l]);
    st_link(U + l, mul(e, ld_link_rw(U + l)));
  }
}
__global__ void k_update_u1(size_t NL, double *__restrict__ U, const double *__restrict__ P,
                            double dt) {
  for (size_t l = blockIdx.x * (size_t)blockDim.x + threadIdx.x; l < NL;
       l += (size_t)gridDim.x * blockDim.x)
    U[l] = dt * P[l] + U[l];
}
// restoreSU in FP64 (gaugeconfig.hh:115-120)
template <class T> __global__ void k_restore(size_t NL, LinkT<T> *__restrict__ U) {
  for (size_t l = blockIdx.x * (size_t)blockDim.x + threadIdx.x; l < NL;
       l += (size_t)gridDim.x * blockDim.x)
    st_link(U + l, from64<T>(restore_su(to64(ld_link_rw(U + l)))));
}

// ------------------------------------------------------------------------------------
// ------------------------------------------------------------------------------------
// momenta: standard normal per component from Philox(seed; {ref link, draw, traj, MOM})
template <class T, int NT>
__global__ void __launch_bounds__(NT)
  k_momenta(Geom g, T *__restrict__ P, int na, const TrajParams *__restrict__ tp,
            double *kin_part) {
  __shared__ double sh[NT / 32];
  const uint64_t seed = tp->seed;
  const uint32_t traj = tp->traj;
  const int mu = blockIdx.y >> 1, p = blockIdx.y & 1;
  const int cb = blockIdx.x * NT + threadIdx.x;
  double k2 = 0.;
  if (cb < g.Vh) {
    const Site s = site_from_eo(g, p, cb);
    const uint32_t lref = (uint32_t)s.lex * (uint32_t)g.nd + (uint32_t)mu;
    const size_t NL = (size_t)g.V * g.nd;
    const size_t l = (size_t)mu * g.V + (size_t)p * g.Vh + cb;
    uint32_t r[4];
    T n0, n1, n2, n3;
    philox(lref, 0u, traj, TAG_MOMENTA, seed, r);
    gauss_pair<T>(r, n0, n1);
    P[l] = n0;
    k2 = (double)n0 * n0;
    if (na == 3) {
      philox(lref, 1u, traj, TAG_MOMENTA, seed, r);
      gauss_pair<T>(r, n2, n3);
      P[NL + l] = n1;
      P[2 * NL + l] = n2;
      k2 += (double)n1 * n1 + (double)n2 * n2;
    }
  }
  const double rr = block_sum<NT>(k2, sh);
  if (threadIdx.x == 0) kin_part[blockIdx.y * gridDim.x + blockIdx.x] = rr;
}

template <class T, int NT>
__global__ void __launch_bounds__(NT)
  k_kinetic(Geom g, const T *__restrict__ P, int na, double *part) {
  __shared__ double sh[NT / 32];
  const int mu = blockIdx.y >> 1, p = blockIdx.y & 1;
  const int cb = blockIdx.x * NT + threadIdx.x;
  double k2 = 0.;
  if (cb < g.Vh) {
    const size_t NL = (size_t)g.V * g.nd;
    const size_t l = (size_t)mu * g.V + (size_t)p * g.Vh + cb;
    for (int k = 0; k < na; k++) {
      const double v = (double)P[k * NL + l];
      k2 += v * v;
    }
  }
  const double rr = block_sum<NT>(k2, sh);
  if (threadIdx.x == 0) part[blockIdx.y * gridDim.x + blockIdx.x] = rr;
}

template <class T> __global__ void k_negate(size_t n, T *P) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    P[i] = -P[i];
}

// ------------------------------------------------------------------------------------
// accept/reject (md_update.hh:45-60), one thread
__global__ void k_accept(const double *__restrict__ red, const TrajParams *__restrict__ tp,
                         TrajDev *out) {
  const TrajParams in = *tp;
  TrajDev t;
  t.H_old[0] = 0.5 * red[0];
  t.H_old[1] = -in.beta * red[3] / in.Nc;
  t.H_old[2] = red[8];
  t.H_new[0] = 0.5 * red[4];
  t.H_new[1] = -in.beta * red[7] / in.Nc;
  t.H_new[2] = red[9];
  double dH = 0.;
  dH += t.H_new[0] - t.H_old[0];
  dH += t.H_new[1] - t.H_old[1];
  dH += t.H_new[2] - t.H_old[2];
  t.dH = dH;
  t.accepted = 1;
  t.u = -1.0;
  if (in.accept_reject && dH > 0) {
    double u = in.u_host;
    if (u < 0.0) {
      uint32_t r[4];
      philox(0u, 0u, in.traj, TAG_ACCEPT, in.seed, r);
      u = u01_53(r[0], r[1]) - 0x1p-53;
    }
    t.u = u;
    if (u > exp(-dH)) t.accepted = 0;
  }
  t.pad = 0;
  *out = t;
}

template <class T>
__global__ void k_cond_restore(size_t n, T *__restrict__ U, const T *__restrict__ U_old,
                               const TrajDev *__restrict__ flag) {
  if (flag->accepted) return;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    U[i] = U_old[i];
}

constexpr int NT_RED = 256;

inline int flat_grid(size_t n, int nt) {
  const size_t b = (n + nt - 1) / nt;
  return (int)(b < 148u * 32u ? (b > 0 ? b : 1) : 148u * 32u);
}

}  // namespace

// =====================================================================================
// launchers
// =====================================================================================

template <class T>
cudaError_t links_from_host(const Geom &g, const double *aos, void *U, int group,
                            cudaStream_t s) {
  const size_t n = (size_t)g.V * g.nd;
  if (group == 0)
    k_links_from_host_su2<T><<<flat_grid(n, 256), 256, 0, s>>>(g, aos, (LinkT<T> *)U);
  else
    k_adj_from_host<double><<<flat_grid(n, 256), 256, 0, s>>>(g, aos, (double *)U, 1);
  return cudaGetLastError();
}
template <class T>
cudaError_t links_to_host(const Geom &g, const void *U, double *aos, int group,
                          cudaStream_t s) {
  const size_t n = (size_t)g.V * g.nd;
  if (group == 0)
    k_links_to_host_su2<T><<<flat_grid(n, 256), 256, 0, s>>>(g, (const LinkT<T> *)U, aos);
  else
    k_adj_to_host<double><<<flat_grid(n, 256), 256, 0, s>>>(g, (const double *)U, aos, 1);
  return cudaGetLastError();
}
template <class T>
cudaError_t adj_from_host(const Geom &g, const double *aos, T *P, int group, cudaStream_t s) {
  const size_t n = (size_t)g.V * g.nd;
  k_adj_from_host<T><<<flat_grid(n, 256), 256, 0, s>>>(g, aos, P, group == 0 ? 3 : 1);
  return cudaGetLastError();
}
template <class T>
cudaError_t adj_to_host(const Geom &g, const T *P, double *aos, int group, cudaStream_t s) {
  const size_t n = (size_t)g.V * g.nd;
  k_adj_to_host<T><<<flat_grid(n, 256), 256, 0, s>>>(g, P, aos, group == 0 ? 3 : 1);
  return cudaGetLastError();
}
cudaError_t spinor_from_host(const Geom &g, const double *aos, double2 *psi, cudaStream_t s) {
  k_spinor_from_host<<<flat_grid(g.V, 256), 256, 0, s>>>(g, (const double2 *)aos, psi);
  return cudaGetLastError();
}
cudaError_t spinor_to_host(const Geom &g, const double2 *psi, double *aos, cudaStream_t s) {
  k_spinor_to_host<<<flat_grid(g.V, 256), 256, 0, s>>>(g, psi, (double2 *)aos);
  return cudaGetLastError();
}

template <class T>
cudaError_t plaq_partials(const Geom &g, const void *U, int group, double xi, double *part,
                          int *nblocks, cudaStream_t s) {
  constexpr int NT = 256;
  const dim3 grid(cdiv(g.Vh, NT / 2));
  *nblocks = grid.x;
  if (group == 0) {
    const LinkT<T> *u = (const LinkT<T> *)U;
    switch (g.nd) {
      case 2: k_plaq_su2<T, 2, NT><<<grid, NT, 0, s>>>(g, u, xi, part); break;
      case 3: k_plaq_su2<T, 3, NT><<<grid, NT, 0, s>>>(g, u, xi, part); break;
      default: k_plaq_su2<T, 4, NT><<<grid, NT, 0, s>>>(g, u, xi, part); break;
    }
  } else {
    const double *u = (const double *)U;
    switch (g.nd) {
      case 2: k_plaq_u1<2, NT><<<grid, NT, 0, s>>>(g, u, xi, part); break;
      case 3: k_plaq_u1<3, NT><<<grid, NT, 0, s>>>(g, u, xi, part); break;
      default: k_plaq_u1<4, NT><<<grid, NT, 0, s>>>(g, u, xi, part); break;
    }
  }
  return cudaGetLastError();
}

cudaError_t reduce_final(const double *part, int nblocks, int ncomp, double *out,
                         cudaStream_t s) {
  k_reduce_final<512><<<1, 512, 0, s>>>(part, nblocks, ncomp, out);
  return cudaGetLastError();
}

template <class T>
cudaError_t force_update(const Geom &g, const void *U, int group, T *P, const T *extra, double f,
                         double scale, double xi, int mode, double *kin_part, int *nblocks,
                         void *Uout, double dt_upd, cudaStream_t s, int variant) {
  constexpr int NT = 128;
  const int aniso = xi != 1.0;
  if (group == 0) {
    const LinkT<T> *u = (const LinkT<T> *)U;
    const T wt = (T)(1.0 / xi), ws = (T)xi;
    LinkT<T> *uo = (LinkT<T> *)Uout;
    int nb = 0;
    const int v = (variant >= 0 && variant < FORCE_VARIANTS) ? variant : 1;
#define SU2B_FORCE_LAUNCH(NTV, MB)                                                           \
  do {                                                                                     \
    const dim3 grid(cdiv(g.Vh, NTV / 2));                                                  \
    nb = grid.x;                                                                           \
    switch (g.nd) {                                                                        \
      case 2:                                                                              \
        k_force_su2<T, 2, NTV, MB><<<grid, NTV, 0, s>>>(g, u, P, extra, (T)f, (T)scale, mode, \
                                                        aniso, wt, ws, kin_part, uo,          \
                                                        (T)dt_upd);                           \
        break;                                                                             \
      case 3:                                                                              \
        k_force_su2<T, 3, NTV, MB><<<grid, NTV, 0, s>>>(g, u, P, extra, (T)f, (T)scale, mode, \
                                                        aniso, wt, ws, kin_part, uo,          \
                                                        (T)dt_upd);                           \
        break;                                                                             \
      default:                                                                             \
        k_force_su2<T, 4, NTV, MB><<<grid, NTV, 0, s>>>(g, u, P, extra, (T)f, (T)scale, mode, \
                                                        aniso, wt, ws, kin_part, uo,          \
                                                        (T)dt_upd);                           \
        break;                                                                             \
    }                                                                                      \
  } while (0)
#define SU2B_FORCE_TILE(BX, BY, BZ, MB)                                                     \
  do {                                                                                     \
    if (!tile_fits<T, BX, BY, BZ>(g)) {                                                    \
      SU2B_FORCE_LAUNCH(128, 6);                                                           \
      break;                                                                               \
    }                                                                                      \
    const int grid = tile_grid<T, BX, BY, BZ, MB>();                                       \
    nb = grid;                                                                             \
    k_force_su2_tile<T, BX, BY, BZ, MB>                                                    \
      <<<grid, Brick<BX, BY, BZ>::NT, tile_smem<T, BX, BY, BZ>(), s>>>(                    \
        g, u, P, extra, (T)f, (T)scale, mode, aniso, wt, ws, kin_part, uo, (T)dt_upd);     \
  } while (0)
    switch (v) {
      case 0: SU2B_FORCE_LAUNCH(256, 4); break;
      case 1: SU2B_FORCE_LAUNCH(128, 8); break;
      case 2: SU2B_FORCE_LAUNCH(128, 4); break;
      case 3: SU2B_FORCE_LAUNCH(128, 6); break;
      case 4: SU2B_FORCE_LAUNCH(256, 2); break;
      case 5: SU2B_FORCE_LAUNCH(256, 3); break;
      case 6: SU2B_FORCE_TILE(4, 4, 8, (sizeof(T) == 4 ? 2 : 1)); break;
      default: SU2B_FORCE_TILE(2, 4, 16, (sizeof(T) == 4 ? 2 : 1)); break;
    }
#undef SU2B_FORCE_LAUNCH
#undef SU2B_FORCE_TILE
    if (nblocks) *nblocks = nb;
  } else {
    if (sizeof(T) != 8) return cudaErrorNotSupported;
    const dim3 grid(cdiv(g.Vh, NT), 2 * g.nd);
    if (nblocks) *nblocks = grid.x * grid.y;
    const double *u = (const double *)U;
    double *PP = (double *)P;
    const double *ex = (const double *)extra;
    switch (g.nd) {
      case 2:
        k_force_u1<2, NT><<<grid, NT, 0, s>>>(g, u, PP, ex, f, scale, mode, aniso, 1.0 / xi, xi,
                                              kin_part);
        break;
      case 3:
        k_force_u1<3, NT><<<grid, NT, 0, s>>>(g, u, PP, ex, f, scale, mode, aniso, 1.0 / xi, xi,
                                              kin_part);
        break;
      default:
        k_force_u1<4, NT><<<grid, NT, 0, s>>>(g, u, PP, ex, f, scale, mode, aniso, 1.0 / xi, xi,
                                              kin_part);
        break;
    }
  }
  return cudaGetLastError();
}

template <class T>
cudaError_t link_update(const Geom &g, void *U, int group, const T *P, double dt,
                        cudaStream_t s) {
  const size_t NL = (size_t)g.V * g.nd;
  if (group == 0)
    k_update_su2<T><<<flat_grid(NL, 256), 256, 0, s>>>(NL, (LinkT<T> *)U, P, (T)dt);
  else {
    if (sizeof(T) != 8) return cudaErrorNotSupported;
    k_update_u1<<<flat_grid(NL, 256), 256, 0, s>>>(NL, (double *)U, (const double *)P, dt);
  }
  return cudaGetLastError();
}

template <class T> cudaError_t restore_links(const Geom &g, void *U, int group, cudaStream_t s) {
  if (group != 0) return cudaSuccess;  // u1.hh:178-179
  const size_t NL = (size_t)g.V * g.nd;
  k_restore<T><<<flat_grid(NL, 256), 256, 0, s>>>(NL, (LinkT<T> *)U);
  return cudaGetLastError();
}

template <class T>
cudaError_t momenta_philox(const Geom &g, T *P, int group, const TrajParams *tp,
                           double *kin_part, int *nblocks, cudaStream_t s) {
  constexpr int NT = NT_RED;
  const dim3 grid(cdiv(g.Vh, NT), 2 * g.nd);
  *nblocks = grid.x * grid.y;
  k_momenta<T, NT><<<grid, NT, 0, s>>>(g, P, group == 0 ? 3 : 1, tp, kin_part);
  return cudaGetLastError();
}

template <class T>
cudaError_t kinetic_partials(const Geom &g, const T *P, int group, double *part, int *nblocks,
                             cudaStream_t s) {
  constexpr int NT = NT_RED;
  const dim3 grid(cdiv(g.Vh, NT), 2 * g.nd);
  *nblocks = grid.x * grid.y;
  k_kinetic<T, NT><<<grid, NT, 0, s>>>(g, P, group == 0 ? 3 : 1, part);
  return cudaGetLastError();
}

template <class T> cudaError_t negate_adj(const Geom &g, T *P, int group, cudaStream_t s) {
  const size_t n = (size_t)g.V * g.nd * (group == 0 ? 3 : 1);
  k_negate<T><<<flat_grid(n, 256), 256, 0, s>>>(n, P);
  return cudaGetLastError();
}

cudaError_t accept_step(const double *red, const TrajParams *tp, TrajDev *out, cudaStream_t s) {
  k_accept<<<1, 1, 0, s>>>(red, tp, out);
  return cudaGetLastError();
}

template <class T>
cudaError_t cond_restore(const Geom &g, void *U, const void *U_old, int group,
                         const TrajDev *flag, cudaStream_t s) {
  const size_t NL = (size_t)g.V * g.nd;
  if (group == 0) {
    // copy as 16-byte words
    const size_t n = NL * sizeof(LinkT<T>) / sizeof(float4);
    k_cond_restore<float4><<<flat_grid(n, 256), 256, 0, s>>>(n, (float4 *)U,
                                                             (const float4 *)U_old, flag);
  } else {
    k_cond_restore<double><<<flat_grid(NL, 256), 256, 0, s>>>(NL, (double *)U,
                                                              (const double *)U_old, flag);
  }
  return cudaGetLastError();
}

// raise the dynamic shared-memory limit of the tiled force kernels (once per process)
template <class T> cudaError_t force_prepare_t() {
  cudaError_t e = cudaFuncSetAttribute(k_force_su2_tile<T, 4, 4, 8, (sizeof(T) == 4 ? 2 : 1)>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)tile_smem<T, 4, 4, 8>());
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_force_su2_tile<T, 2, 4, 16, (sizeof(T) == 4 ? 2 : 1)>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)tile_smem<T, 2, 4, 16>());
  return e;
}
cudaError_t force_prepare() {
  cudaError_t e = force_prepare_t<float>();
  if (e == cudaSuccess) e = force_prepare_t<double>();
  return e;
}

#define INST(T)                                                                              \
  template cudaError_t links_from_host<T>(const Geom &, const double *, void *, int,         \
                                          cudaStream_t);                                      \
  template cudaError_t links_to_host<T>(const Geom &, const void *, double *, int,           \
                                        cudaStream_t);                                        \
  template cudaError_t adj_from_host<T>(const Geom &, const double *, T *, int, cudaStream_t); \
  template cudaError_t adj_to_host<T>(const Geom &, const T *, double *, int, cudaStream_t);   \
  template cudaError_t plaq_partials<T>(const Geom &, const void *, int, double, double *,   \
                                        int *, cudaStream_t);                                 \
  template cudaError_t force_update<T>(const Geom &, const void *, int, T *, const T *,      \
                                       double, double, double, int, double *, int *, void *,  \
                                       double, cudaStream_t, int);                            \
  template cudaError_t link_update<T>(const Geom &, void *, int, const T *, double,          \
                                      cudaStream_t);                                          \
  template cudaError_t restore_links<T>(const Geom &, void *, int, cudaStream_t);            \
  template cudaError_t momenta_philox<T>(const Geom &, T *, int, const TrajParams *,         \
                                         double *, int *, cudaStream_t);                      \
  template cudaError_t kinetic_partials<T>(const Geom &, const T *, int, double *, int *,    \
                                           cudaStream_t);                                     \
  template cudaError_t negate_adj<T>(const Geom &, T *, int, cudaStream_t);                  \
  template cudaError_t cond_restore<T>(const Geom &, void *, const void *, int,              \
                                       const TrajDev *, cudaStream_t);
INST(double)
INST(float)
#undef INST

}  // namespace su2b
