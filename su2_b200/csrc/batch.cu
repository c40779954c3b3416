// batch.cu -- an ensemble of independent SU(2) chains (different geometries, dimensions and
// couplings) advanced together: every stage of an HMC trajectory is ONE persistent launch
// over a tile list that spans all chains, and the whole trajectory is one CUDA graph.
//
// Storage: the links of all chains are concatenated in each of three link buffers, the
// momenta in one adjoint buffer (per chain the single-lattice layout, see su2b_common.cuh).
// Each chain's triple-buffer rotation (which buffer holds its current field) lives in device
// memory and is advanced by the per-chain accept kernel, so replaying the graph needs no host
// decision.  A tile is NT/2 sites of each parity of one chain; block b finds its chain in the
// tile prefix table.  The per-site arithmetic is force_site / plaq_site, shared with the
// single-lattice kernels, so a chain gives the same trajectory alone or in a batch.
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <string>
#include <vector>

#include "site_ops.cuh"
#include "su2b.h"

using namespace su2b;

namespace {

struct ChainDev {
  Geom g;
  double beta;
  uint64_t seed;
  size_t off_link;  // offset of the chain in the link buffers (in links)
  size_t off_adj;   // offset of the chain's momenta (3 * NL reals)
  int tile0, ntiles;
};

constexpr int RS = 16;  // reduced scalars per chain

// the chain that owns a tile: the last chain whose first tile is <= tile (binary search)
__device__ __forceinline__ int chain_of(const ChainDev *__restrict__ ch, int n, int tile) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(&ch[mid].tile0) <= tile)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// threads per block of the batched launch shapes (a tile is NT/2 sites of each parity of one
// chain); the force kernel's minimum resident blocks per SM are 8, 4, 6, 3 (enqueue_batch)
constexpr int BATCH_NT[SU2B_BATCH_VARIANTS] = {64, 128, 128, 256};

template <class T> struct Bufs {
  LinkT<T> *b[3];
  // buffer k by selection: indexing the kernel-parameter array by a variable would copy it
  // to local memory
  __device__ __forceinline__ LinkT<T> *at(int k) const { return k == 0 ? b[0] : k == 1 ? b[1] : b[2]; }
};

template <class T, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB)
  k_batch_force(const ChainDev *__restrict__ ch, int nchains, int ntiles, Bufs<T> bufs,
                T *__restrict__ Pall, const int *__restrict__ cur, int rel_in, int rel_out,
                double cm, double cg, int mode, double *kin_part) {
  __shared__ double sh[NT / 32];
  const int w = threadIdx.x >> 5, p = w & 1;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int c = chain_of(ch, nchains, tile);
    const ChainDev &d = ch[c];
    const int cb = (tile - d.tile0) * (NT / 2) + (w >> 1) * 32 + (threadIdx.x & 31);
    const int S = cur[c];
    const LinkT<T> *U = bufs.at((S + rel_in) % 3) + d.off_link;
    LinkT<T> *Uo = rel_out >= 0 ? bufs.at((S + rel_out) % 3) + d.off_link : nullptr;
    T *P = Pall + d.off_adj;
    const T f = (T)(d.beta / 2.0);
    double k2 = 0.;
    if (cb < d.g.Vh) {
      if (d.g.nd == 4)
        k2 = force_site_impl<T, 4, false>(d.g, U, P, nullptr, f, (T)(-cm), mode, T(1), T(1), Uo, (T)cg, p,
                              cb);
      else
        k2 = force_site_impl<T, 3, false>(d.g, U, P, nullptr, f, (T)(-cm), mode, T(1), T(1), Uo, (T)cg, p,
                              cb);
    }
    if (mode & FM_KINETIC) {
      const double r = block_sum<NT>(k2, sh);
      if (threadIdx.x == 0) kin_part[tile] = r;
    }
  }
}

// momenta of the batch: the single-lattice Philox stream of each chain (its own seed)
template <class T, int NT>
__global__ void __launch_bounds__(NT)
  k_batch_momenta(const ChainDev *__restrict__ ch, int nchains, int ntiles, T *__restrict__ Pall,
                  const uint32_t *__restrict__ traj, double *kin_part) {
  __shared__ double sh[NT / 32];
  const int w = threadIdx.x >> 5, p = w & 1;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int c = chain_of(ch, nchains, tile);
    const ChainDev &d = ch[c];
    const int cb = (tile - d.tile0) * (NT / 2) + (w >> 1) * 32 + (threadIdx.x & 31);
    double k2 = 0.;
    if (cb < d.g.Vh) {
      const Site s = site_from_eo(d.g, p, cb);
      const size_t NL = (size_t)d.g.V * d.g.nd;
      T *P = Pall + d.off_adj;
      for (int mu = 0; mu < d.g.nd; mu++) {
        const uint32_t lref = (uint32_t)s.lex * (uint32_t)d.g.nd + (uint32_t)mu;
        const size_t l = (size_t)mu * d.g.V + (size_t)p * d.g.Vh + cb;
        T a, b, cc;
        momentum_normals<T>(lref, *traj, d.seed, 3, a, b, cc);
        P[l] = a;
        P[NL + l] = b;
        P[2 * NL + l] = cc;
        k2 += (double)a * a + (double)b * b + (double)cc * cc;
      }
    }
    const double rr = block_sum<NT>(k2, sh);
    if (threadIdx.x == 0) kin_part[tile] = rr;
  }
}

template <class T, int NT>
__global__ void __launch_bounds__(NT)
  k_batch_plaq(const ChainDev *__restrict__ ch, int nchains, int ntiles, Bufs<T> bufs,
               const int *__restrict__ cur, int rel, double *part) {
  __shared__ double sh[NT / 32];
  const int w = threadIdx.x >> 5, p = w & 1;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int c = chain_of(ch, nchains, tile);
    const ChainDev &d = ch[c];
    const int cb = (tile - d.tile0) * (NT / 2) + (w >> 1) * 32 + (threadIdx.x & 31);
    const LinkT<T> *U = bufs.at((cur[c] + rel) % 3) + d.off_link;
    double full = 0., spat = 0., wsum = 0.;
    if (cb < d.g.Vh) {
      if (d.g.nd == 4)
        plaq_site<T, 4>(d.g, U, p, cb, 1.0, full, spat, wsum);
      else
        plaq_site<T, 3>(d.g, U, p, cb, 1.0, full, spat, wsum);
    }
    double r = block_sum<NT>(full, sh);
    if (threadIdx.x == 0) part[3 * tile] = r;
    r = block_sum<NT>(spat, sh);
    if (threadIdx.x == 0) {
      part[3 * tile + 1] = r;
      part[3 * tile + 2] = 0.0;
    }
  }
}

// the start of a batched trajectory in one pass, as in the single-lattice path: each
// site's Philox momenta with their |P|^2 and its start plaquettes; per tile the partials
// {sum |P|^2, plaquettes, spatial plaquettes}.  Without PLAQ the momenta only (the start
// plaquettes are carried over from the previous trajectory; the plaquette partials are 0)
template <class T, int NT, bool PLAQ>
__global__ void __launch_bounds__(NT)
  k_batch_momenta_plaq(const ChainDev *__restrict__ ch, int nchains, int ntiles, Bufs<T> bufs,
                       const int *__restrict__ cur, T *__restrict__ Pall,
                       const uint32_t *__restrict__ traj, double *part) {
  __shared__ double shk[3 * (NT / 32)];
  const int w = threadIdx.x >> 5, p = w & 1;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int c = chain_of(ch, nchains, tile);
    const ChainDev &d = ch[c];
    const int cb = (tile - d.tile0) * (NT / 2) + (w >> 1) * 32 + (threadIdx.x & 31);
    double v[3] = {0., 0., 0.};
    if (cb < d.g.Vh) {
      const Site s = site_from_eo(d.g, p, cb);
      const size_t NL = (size_t)d.g.V * d.g.nd;
      T *P = Pall + d.off_adj;
      for (int mu = 0; mu < d.g.nd; mu++) {
        const uint32_t lref = (uint32_t)s.lex * (uint32_t)d.g.nd + (uint32_t)mu;
        const size_t l = (size_t)mu * d.g.V + (size_t)p * d.g.Vh + cb;
        T a, b, cc;
        momentum_normals<T>(lref, *traj, d.seed, 3, a, b, cc);
        P[l] = a;
        P[NL + l] = b;
        P[2 * NL + l] = cc;
        v[0] += (double)a * a + (double)b * b + (double)cc * cc;
      }
      if (PLAQ) {
        const LinkT<T> *U = bufs.at(cur[c] % 3) + d.off_link;
        double wsum = 0.;
        if (d.g.nd == 4)
          plaq_site<T, 4>(d.g, U, p, cb, 1.0, v[1], v[2], wsum);
        else
          plaq_site<T, 3>(d.g, U, p, cb, 1.0, v[1], v[2], wsum);
      }
    }
    block_sums<NT, 3>(v, shk);
    if (threadIdx.x == 0) {
      part[3 * tile] = v[0];
      part[3 * tile + 1] = v[1];
      part[3 * tile + 2] = v[2];
    }
  }
}

// the closing reductions and the accept/reject of every chain in one launch, one block per
// chain: the start partials (3 per tile) into red[0..2], the final kinetic partials into
// red[4], the end plaquette partials (3 per tile, the third unused) into red[5..7], each in
// a fixed order; then the chain's accept step (accept_chain) on thread 0.
// cached: the start pass summed no plaquettes; the chain's start field is the previous
// trajectory's result, whose plaquette sums are still in red -- red[5..6] if that
// trajectory was accepted (out[c].accepted, not yet overwritten), else red[1..2].  The end
// pass and the start pass add the same per-tile partials in the same order, so the carried
// sums equal recomputed ones bit for bit.
__device__ __forceinline__ void accept_chain(const ChainDev &d, const double *r,
                                             const uint32_t *__restrict__ traj, int rel_final,
                                             int *cur_c, TrajDev *out) {
  TrajDev t;
  t.H_old[0] = 0.5 * r[0];
  t.H_old[1] = -d.beta * r[1] / 2.0;
  t.H_old[2] = 0.0;
  t.H_new[0] = 0.5 * r[4];
  t.H_new[1] = -d.beta * r[5] / 2.0;
  t.H_new[2] = 0.0;
  double dH = 0.;
  dH += t.H_new[0] - t.H_old[0];
  dH += t.H_new[1] - t.H_old[1];
  t.dH = dH;
  t.accepted = 1;
  t.u = -1.0;
  if (dH > 0) {
    uint32_t rr[4];
    philox(0u, 0u, *traj, TAG_ACCEPT, d.seed, rr);
    t.u = u01_53(rr[0], rr[1]) - 0x1p-53;
    if (t.u > exp(-dH)) t.accepted = 0;
  }
  t.pad = 0;
  *out = t;
  if (t.accepted) *cur_c = (*cur_c + rel_final) % 3;
}
__global__ void __launch_bounds__(256)
  k_batch_reduce_accept(const ChainDev *__restrict__ ch, const double *__restrict__ ps,
                        const double *__restrict__ pk, const double *__restrict__ pe,
                        double *red, const uint32_t *__restrict__ traj, int rel_final, int *cur,
                        TrajDev *out, int cached) {
  __shared__ double shk[7 * 8];
  const int c = blockIdx.x;
  const ChainDev &d = ch[c];
  double v[7] = {0., 0., 0., 0., 0., 0., 0.};
  for (int t = threadIdx.x; t < d.ntiles; t += 256) {
    const size_t tt = (size_t)(d.tile0 + t);
#pragma unroll
    for (int k = 0; k < 3; k++) v[k] += ps[tt * 3 + k];
    v[3] += pk[tt];
#pragma unroll
    for (int k = 0; k < 3; k++) v[4 + k] += pe[tt * 3 + k];
  }
  block_sums<256, 7>(v, shk);
  if (threadIdx.x == 0) {
    double *r = red + c * RS;
    if (cached) {
      const bool acc = out[c].accepted;
      v[1] = acc ? r[5] : r[1];
      v[2] = acc ? r[6] : r[2];
    }
    r[0] = v[0];
    r[1] = v[1];
    r[2] = v[2];
    r[4] = v[3];
    r[5] = v[4];
    r[6] = v[5];
    r[7] = v[6];
    accept_chain(d, r, traj, rel_final, cur + c, out + c);
  }
}

}  // namespace

// =====================================================================================
struct su2b_batch {
  int n = 0, prec = 0, device = 0;
  bool link64 = true;
  cudaStream_t stream = nullptr;
  std::vector<su2b_chain_desc> desc;
  std::vector<ChainDev> hch[SU2B_BATCH_VARIANTS];  // tile tables per launch shape
  ChainDev *ch[SU2B_BATCH_VARIANTS] = {};
  int ntiles[SU2B_BATCH_VARIANTS] = {};
  int variant = 2;
  size_t total_links = 0;
  int maxtiles = 0;  // tiles of the launch shape with the most (sizes the partial buffer)
  void *buf[3] = {};
  void *P = nullptr;
  double *part = nullptr, *red = nullptr, *stage = nullptr;
  int *cur = nullptr;
  uint32_t *traj = nullptr, *h_traj = nullptr;
  TrajDev *res = nullptr, *h_res = nullptr;
  double *h_red = nullptr;
  int *h_cur = nullptr;
  struct Graph {
    std::string key;
    cudaGraphExec_t exec;
    long kernels;
  };
  std::vector<Graph> graphs;
  std::vector<void *> allocs;
  std::string err;
  long launches = 0;
  // set by a batched trajectory: red holds every chain's start and end plaquette sums, so
  // the next trajectory takes its start plaquettes from there; an upload or a retune clears it
  bool carry = false;
};

static int bfail(su2b_batch *b, int code, const char *fmt, ...) {
  if (b) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    b->err = buf;
  }
  return code;
}
#define BCK(call)                                                                          \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess)                                                                 \
      return bfail(b, SU2B_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call,            \
                   cudaGetErrorString(e_));                                                \
  } while (0)

int su2b_make_geom(int Lx, int Ly, int Lz, int Lt, int nd, Geom *g, std::string *why);

extern "C" int su2b_batch_create(int n_chains, const su2b_chain_desc *chains, int precision,
                                 int device, su2b_batch **out) {
  if (!out || !chains || n_chains < 1) return SU2B_ERR_INVALID;
  *out = nullptr;
  if (precision != SU2B_PREC_FP64 && precision != SU2B_PREC_MIXED) return SU2B_ERR_INVALID;
  su2b_batch *b = new su2b_batch();
  b->n = n_chains;
  b->prec = precision;
  b->device = device;
  b->link64 = precision == SU2B_PREC_FP64;
  b->desc.assign(chains, chains + n_chains);
  auto fin = [&](int s) -> int {
    if (s != SU2B_OK) {
      su2b_batch_destroy(b);
      return s;
    }
    *out = b;
    return SU2B_OK;
  };
  b->variant = b->link64 ? 1 : 2;
  size_t off_l = 0, off_a = 0;
  int maxtiles = 0;
  for (int v = 0; v < SU2B_BATCH_VARIANTS; v++) {
    const int half = BATCH_NT[v] / 2;
    off_l = off_a = 0;
    int tile = 0;
    for (int c = 0; c < n_chains; c++) {
      const su2b_chain_desc &d = chains[c];
      ChainDev cd{};
      std::string why;
      if (d.ndims < 3 || !su2b_make_geom(d.Lx, d.Ly, d.Lz, d.Lt, d.ndims, &cd.g, &why))
        return fin(bfail(b, SU2B_ERR_INVALID, "chain %d: %s", c,
                         d.ndims < 3 ? "batches hold d = 3 or 4 chains" : why.c_str()));
      cd.beta = d.beta;
      cd.seed = d.seed;
      cd.off_link = off_l;
      cd.off_adj = off_a;
      cd.tile0 = tile;
      cd.ntiles = (cd.g.Vh + half - 1) / half;
      const size_t NL = (size_t)cd.g.V * d.ndims;
      off_l += NL;
      off_a += 3 * NL;
      tile += cd.ntiles;
      b->hch[v].push_back(cd);
    }
    b->ntiles[v] = tile;
    maxtiles = std::max(maxtiles, tile);
  }
  b->total_links = off_l;
  b->maxtiles = maxtiles;
  const int tile = maxtiles;
  if (cudaSetDevice(device) != cudaSuccess) return fin(SU2B_ERR_CUDA);
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess)
    return fin(SU2B_ERR_CUDA);
  const size_t lb = b->link64 ? 32 : 16, ab = b->link64 ? 8 : 4;
  auto dal = [&](void **p, size_t bytes) -> bool {
    if (cudaMalloc(p, bytes) != cudaSuccess) return false;
    b->allocs.push_back(*p);
    return true;
  };
  size_t maxNL = 0;
  for (auto &c : b->hch[0]) maxNL = std::max(maxNL, (size_t)c.g.V * c.g.nd);
  bool ok = dal(&b->buf[0], lb * off_l) && dal(&b->buf[1], lb * off_l) &&
            dal(&b->buf[2], lb * off_l) && dal(&b->P, ab * off_a) &&
            dal((void **)&b->part, sizeof(double) * 7 * (size_t)tile) &&
            dal((void **)&b->red, sizeof(double) * RS * n_chains) &&
            dal((void **)&b->stage, sizeof(double) * 4 * maxNL) &&
            dal((void **)&b->cur, sizeof(int) * n_chains) &&
            dal((void **)&b->traj, sizeof(uint32_t)) &&
            dal((void **)&b->res, sizeof(TrajDev) * n_chains);
  for (int v = 0; v < SU2B_BATCH_VARIANTS && ok; v++)
    ok = dal((void **)&b->ch[v], sizeof(ChainDev) * n_chains);
  if (!ok) return fin(bfail(b, SU2B_ERR_NOMEM, "device allocation failed"));
  if (cudaMallocHost((void **)&b->h_traj, sizeof(uint32_t)) != cudaSuccess ||
      cudaMallocHost((void **)&b->h_res, sizeof(TrajDev) * n_chains) != cudaSuccess ||
      cudaMallocHost((void **)&b->h_red, sizeof(double) * RS * n_chains) != cudaSuccess ||
      cudaMallocHost((void **)&b->h_cur, sizeof(int) * n_chains) != cudaSuccess)
    return fin(SU2B_ERR_NOMEM);
  for (int v = 0; v < SU2B_BATCH_VARIANTS; v++)
    if (cudaMemcpy(b->ch[v], b->hch[v].data(), sizeof(ChainDev) * n_chains,
                   cudaMemcpyHostToDevice) != cudaSuccess)
      return fin(SU2B_ERR_CUDA);
  if (cudaMemset(b->cur, 0, sizeof(int) * n_chains) != cudaSuccess ||
      cudaMemset(b->buf[0], 0, lb * off_l) != cudaSuccess ||
      cudaMemset(b->P, 0, ab * off_a) != cudaSuccess)
    return fin(SU2B_ERR_CUDA);
  return fin(SU2B_OK);
}

extern "C" int su2b_batch_destroy(su2b_batch *b) {
  if (!b) return SU2B_ERR_INVALID;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  for (auto &g : b->graphs) cudaGraphExecDestroy(g.exec);
  for (void *p : b->allocs) cudaFree(p);
  if (b->h_traj) cudaFreeHost(b->h_traj);
  if (b->h_res) cudaFreeHost(b->h_res);
  if (b->h_red) cudaFreeHost(b->h_red);
  if (b->h_cur) cudaFreeHost(b->h_cur);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return SU2B_OK;
}

extern "C" const char *su2b_batch_last_error(const su2b_batch *b) {
  return b ? b->err.c_str() : "null batch";
}
extern "C" int su2b_batch_stream(su2b_batch *b, void **stream) {
  if (!b) return SU2B_ERR_INVALID;
  if (!stream) return bfail(b, SU2B_ERR_INVALID, "stream is NULL");
  *stream = (void *)b->stream;
  return SU2B_OK;
}
extern "C" int su2b_batch_kernel_launches(su2b_batch *b, long *count) {
  if (!b) return SU2B_ERR_INVALID;
  if (!count) return bfail(b, SU2B_ERR_INVALID, "count is NULL");
  *count = b->launches;
  return SU2B_OK;
}

static int chain_transfer(su2b_batch *b, int chain, double *host, bool up) {
  if (chain < 0 || chain >= b->n || !host) return bfail(b, SU2B_ERR_INVALID, "bad chain/buffer");
  BCK(cudaSetDevice(b->device));
  const ChainDev &c = b->hch[0][chain];
  const size_t NL = (size_t)c.g.V * c.g.nd;
  BCK(cudaMemcpy(b->h_cur, b->cur, sizeof(int) * b->n, cudaMemcpyDeviceToHost));
  const size_t lb = b->link64 ? 32 : 16;
  char *U = (char *)b->buf[b->h_cur[chain]] + lb * c.off_link;
  if (up) {
    BCK(cudaMemcpyAsync(b->stage, host, 4 * NL * sizeof(double), cudaMemcpyHostToDevice,
                        b->stream));
    if (b->link64)
      BCK(links_from_host<double>(c.g, b->stage, U, 0, b->stream));
    else
      BCK(links_from_host<float>(c.g, b->stage, U, 0, b->stream));
  } else {
    if (b->link64)
      BCK(links_to_host<double>(c.g, U, b->stage, 0, b->stream));
    else
      BCK(links_to_host<float>(c.g, U, b->stage, 0, b->stream));
    BCK(cudaMemcpyAsync(host, b->stage, 4 * NL * sizeof(double), cudaMemcpyDeviceToHost,
                        b->stream));
  }
  b->launches++;
  BCK(cudaStreamSynchronize(b->stream));
  return SU2B_OK;
}

extern "C" int su2b_batch_upload(su2b_batch *b, int chain, const double *U_host) {
  if (!b) return SU2B_ERR_INVALID;
  b->carry = false;  // a new field: its plaquettes are summed afresh
  return chain_transfer(b, chain, const_cast<double *>(U_host), true);
}
extern "C" int su2b_batch_download(su2b_batch *b, int chain, double *U_host) {
  return b ? chain_transfer(b, chain, U_host, false) : SU2B_ERR_INVALID;
}

namespace {

struct BOp {
  int kind;  // 0 momentum step, 1 momentum + gauge step
  double cm, cg;
  bool kinetic;
};

std::vector<BOp> batch_schedule(int integ, int n, double tau, bool *ok) {
  // the reference's leapfrog and omf2 (integrator.hh:26-50, 83-116), fused as in hmc.cu
  std::vector<std::pair<int, double>> ops;
  const double dtau = tau / (double)n;
  *ok = true;
  if (integ == SU2B_OMF2) {
    const double lambda = 0.1938, om2l = (1. - 2. * lambda);
    ops.push_back({0, lambda * dtau});
    for (int i = 0; i < n - 1; i++) {
      ops.push_back({1, 0.5 * dtau});
      ops.push_back({0, om2l * dtau});
      ops.push_back({1, 0.5 * dtau});
      ops.push_back({0, 2 * lambda * dtau});
    }
    ops.push_back({1, 0.5 * dtau});
    ops.push_back({0, om2l * dtau});
    ops.push_back({1, 0.5 * dtau});
    ops.push_back({0, lambda * dtau});
  } else if (integ == SU2B_LEAPFROG) {
    ops.push_back({0, dtau / 2.});
    ops.push_back({1, dtau});
    for (int i = 0; i < n - 1; i++) {
      ops.push_back({0, dtau});
      ops.push_back({1, dtau});
    }
    ops.push_back({0, dtau / 2.});
  } else {
    *ok = false;
    return {};
  }
  std::vector<BOp> f;
  for (size_t i = 0; i < ops.size(); i++) {
    if (ops[i].first == 0 && i + 1 < ops.size() && ops[i + 1].first == 1) {
      f.push_back({1, ops[i].second, ops[i + 1].second, false});
      i++;
    } else {
      f.push_back({0, ops[i].second, 0.0, false});
    }
  }
  if (!f.empty()) f.back().kinetic = true;
  return f;
}

template <int NT> int grid_for(const void *kernel, int ntiles) {
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, NT, 0);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return std::max(1, std::min(ntiles, std::max(1, per_sm) * sms));
}

// queues one batched trajectory; *nl receives the number of kernels queued
template <class T, int NT, int MINB>
int enqueue_batch_v(su2b_batch *b, const std::vector<BOp> &ops, int *rel_final, bool cached,
                    long *nl_out) {
  cudaStream_t s = b->stream;
  const int v = b->variant;
  const ChainDev *ch = b->ch[v];
  const int ntiles = b->ntiles[v];
  Bufs<T> bufs{{(LinkT<T> *)b->buf[0], (LinkT<T> *)b->buf[1], (LinkT<T> *)b->buf[2]}};
  T *P = (T *)b->P;
  const int gF = grid_for<NT>((const void *)k_batch_force<T, NT, MINB>, ntiles);
  const int gM = grid_for<NT>((const void *)k_batch_momenta_plaq<T, NT, true>, ntiles);
  const int gP = grid_for<NT>((const void *)k_batch_plaq<T, NT>, ntiles);
  // partial sums: the start pass, the final kinetic energy and the end plaquettes in three
  // regions, all reduced by the closing accept launch
  double *ps = b->part, *pk = b->part + 3 * (size_t)b->maxtiles,
         *pe = b->part + 4 * (size_t)b->maxtiles;
  long nl = 0;
  if (cached)
    k_batch_momenta_plaq<T, NT, false><<<gM, NT, 0, s>>>(ch, b->n, ntiles, bufs, b->cur, P,
                                                         b->traj, ps);
  else
    k_batch_momenta_plaq<T, NT, true><<<gM, NT, 0, s>>>(ch, b->n, ntiles, bufs, b->cur, P,
                                                        b->traj, ps);
  nl += 1;
  int cur = 0;
  auto next = [](int c) { return c == 1 ? 2 : 1; };
  int fin = -1;
  for (size_t i = 0; i < ops.size(); i++) {
    const BOp &o = ops[i];
    int mode = FM_HAS_IN | (o.kinetic ? FM_KINETIC : 0);
    int out = -1;
    if (o.kind == 1) {
      mode |= FM_UPDATE;
      out = next(cur);
    } else if (i + 1 == ops.size()) {
      mode |= FM_RESTORE;
      out = fin = (cur == 0) ? 1 : next(cur);
    }
    k_batch_force<T, NT, MINB><<<gF, NT, 0, s>>>(ch, b->n, ntiles, bufs, P, b->cur, cur, out,
                                                 o.cm, o.cg, mode, pk);
    nl++;
    if (o.kind == 1) cur = out;
  }
  if (fin < 0) return bfail(b, SU2B_ERR_UNSUPPORTED, "schedule must end with a momentum step");
  k_batch_plaq<T, NT><<<gP, NT, 0, s>>>(ch, b->n, ntiles, bufs, b->cur, fin, pe);
  k_batch_reduce_accept<<<b->n, 256, 0, s>>>(ch, ps, pk, pe, b->red, b->traj, fin, b->cur,
                                             b->res, (int)cached);
  nl += 2;
  BCK(cudaGetLastError());
  BCK(cudaMemcpyAsync(b->h_res, b->res, sizeof(TrajDev) * b->n, cudaMemcpyDeviceToHost, s));
  BCK(cudaMemcpyAsync(b->h_red, b->red, sizeof(double) * RS * b->n, cudaMemcpyDeviceToHost, s));
  *rel_final = fin;
  *nl_out = nl;
  return SU2B_OK;
}

template <class T>
int enqueue_batch(su2b_batch *b, const std::vector<BOp> &ops, int *rel_final, bool cached,
                  long *nl) {
  switch (b->variant) {
    case 0: return enqueue_batch_v<T, 64, 8>(b, ops, rel_final, cached, nl);
    case 1: return enqueue_batch_v<T, 128, 4>(b, ops, rel_final, cached, nl);
    case 2: return enqueue_batch_v<T, 128, 6>(b, ops, rel_final, cached, nl);
    default: return enqueue_batch_v<T, 256, 3>(b, ops, rel_final, cached, nl);
  }
}

// Times the batched force step (momentum step + link update of every chain, one persistent
// launch) of one launch shape: fresh momenta from the Philox stream, then `reps` launches
// that read each chain's current field and write the update into a buffer the chain does
// not use, so the chains' states are untouched.  Returns microseconds per launch.
template <class T, int NT, int MINB> int time_force_v(su2b_batch *b, int v, double *us) {
  cudaStream_t s = b->stream;
  const ChainDev *ch = b->ch[v];
  const int ntiles = b->ntiles[v];
  Bufs<T> bufs{{(LinkT<T> *)b->buf[0], (LinkT<T> *)b->buf[1], (LinkT<T> *)b->buf[2]}};
  T *P = (T *)b->P;
  const int gF = grid_for<NT>((const void *)k_batch_force<T, NT, MINB>, ntiles);
  const int gM = grid_for<NT>((const void *)k_batch_momenta<T, NT>, ntiles);
  k_batch_momenta<T, NT><<<gM, NT, 0, s>>>(ch, b->n, ntiles, P, b->traj, b->part);
  const int mode = FM_HAS_IN | FM_UPDATE;
  auto launch = [&]() {
    k_batch_force<T, NT, MINB><<<gF, NT, 0, s>>>(ch, b->n, ntiles, bufs, P, b->cur, 0, 1, 0.01,
                                                 0.01, mode, b->part);
  };
  launch();  // warm-up
  cudaEvent_t e0, e1;
  BCK(cudaEventCreate(&e0));
  BCK(cudaEventCreate(&e1));
  const int reps = 5;
  cudaEventRecord(e0, s);
  for (int r = 0; r < reps; r++) launch();
  cudaEventRecord(e1, s);
  const cudaError_t e = cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  BCK(e);
  BCK(cudaGetLastError());
  b->launches += reps + 2;
  *us = 1e3 * (double)ms / reps;
  return SU2B_OK;
}

template <class T> int time_force(su2b_batch *b, int v, double *us) {
  switch (v) {
    case 0: return time_force_v<T, 64, 8>(b, v, us);
    case 1: return time_force_v<T, 128, 4>(b, v, us);
    case 2: return time_force_v<T, 128, 6>(b, v, us);
    default: return time_force_v<T, 256, 3>(b, v, us);
  }
}

}  // namespace

extern "C" int su2b_batch_hmc(su2b_batch *b, int integrator, int n_steps, double tau,
                              uint32_t traj, su2b_traj_result *results) {
  if (!b) return SU2B_ERR_INVALID;
  b->err.clear();
  BCK(cudaSetDevice(b->device));
  if (!results || n_steps < 1) return bfail(b, SU2B_ERR_INVALID, "bad arguments");
  bool ok = true;
  const std::vector<BOp> ops = batch_schedule(integrator, n_steps, tau, &ok);
  if (!ok)
    return bfail(b, SU2B_ERR_UNSUPPORTED, "batched trajectories support leapfrog and omf2");
  *b->h_traj = traj;
  BCK(cudaMemcpyAsync(b->traj, b->h_traj, sizeof(uint32_t), cudaMemcpyHostToDevice, b->stream));
  const bool cached = b->carry;
  b->carry = false;  // set again only by a trajectory that completes
  char key[128];
  snprintf(key, sizeof key, "%d/%d/%.17g/v%d/%d", integrator, n_steps, tau, b->variant,
           (int)cached);
  cudaGraphExec_t exec = nullptr;
  long kernels = 0;
  for (auto &g : b->graphs)
    if (g.key == key) {
      exec = g.exec;
      kernels = g.kernels;
    }
  if (!exec) {
    cudaGraph_t graph = nullptr;
    BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    int rel = 0;
    long nl = 0;
    const int rc = b->link64 ? enqueue_batch<double>(b, ops, &rel, cached, &nl)
                             : enqueue_batch<float>(b, ops, &rel, cached, &nl);
    const cudaError_t ec = cudaStreamEndCapture(b->stream, &graph);
    if (rc != SU2B_OK) {
      if (graph) cudaGraphDestroy(graph);
      return rc;
    }
    BCK(ec);
    const cudaError_t ei = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    BCK(ei);
    kernels = nl;
    b->graphs.push_back({key, exec, kernels});
  }
  BCK(cudaGraphLaunch(exec, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  b->launches += kernels;
  b->carry = true;
  for (int c = 0; c < b->n; c++) {
    const TrajDev &t = b->h_res[c];
    su2b_traj_result &r = results[c];
    r.accepted = t.accepted;
    r.dH = t.dH;
    for (int k = 0; k < 3; k++) {
      r.H_old[k] = t.H_old[k];
      r.H_new[k] = t.H_new[k];
    }
    r.ddH = 0.0;
    r.plaquette = t.accepted ? b->h_red[c * RS + 5] : b->h_red[c * RS + 1];
    r.cg_iterations = 0;
  }
  return SU2B_OK;
}

extern "C" int su2b_batch_autotune(su2b_batch *b, double *times_us) {
  if (!b) return SU2B_ERR_INVALID;
  b->err.clear();
  b->carry = false;  // the tile tables change with the launch shape, and with them the order
                     // in which the carried plaquette sums were added
  BCK(cudaSetDevice(b->device));
  double t[SU2B_BATCH_VARIANTS], fastest = 0.;
  for (int v = 0; v < SU2B_BATCH_VARIANTS; v++) {
    double us = 0.;
    const int rc = b->link64 ? time_force<double>(b, v, &us) : time_force<float>(b, v, &us);
    if (rc != SU2B_OK) return rc;
    if (times_us) times_us[v] = us;
    t[v] = us;
    fastest = (v == 0 || us < fastest) ? us : fastest;
  }
  // as su2b_autotune: the first shape within 1 % of the fastest, so ties resolve alike
  int bv = 0;
  while (t[bv] > 1.01 * fastest) bv++;
  b->variant = bv;
  return SU2B_OK;
}

extern "C" int su2b_batch_tune_get(su2b_batch *b, int *variant) {
  if (!b) return SU2B_ERR_INVALID;
  if (!variant) return bfail(b, SU2B_ERR_INVALID, "variant is NULL");
  *variant = b->variant;
  return SU2B_OK;
}

extern "C" int su2b_batch_tune_set(su2b_batch *b, int variant) {
  if (!b) return SU2B_ERR_INVALID;
  if (variant < 0 || variant >= SU2B_BATCH_VARIANTS)
    return bfail(b, SU2B_ERR_INVALID, "batch launch shape %d out of range", variant);
  if (variant != b->variant) b->carry = false;
  b->variant = variant;
  return SU2B_OK;
}
