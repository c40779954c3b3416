// slabs.cu -- one lattice over time slabs: the t-slab decomposition of the HMC trajectory.
//
// The reference runs one lattice per process and splits the site loops over OpenMP threads
// along t (flat-sweep.hh:83,128; flat-gaugemonomial.hh:105-131).  Here the lattice (extent Lt
// in t, the slowest index of both the host order and the even/odd layout) is cut into
// nslabs slabs of Tl = Lt / nslabs slices.  A slab is an ordinary context over Tl + 2
// slices: its own slices 1 .. Tl and a ghost slice on each side (local slice 0 is the global
// slice t0 - 1, local slice Tl + 1 the global slice t0 + Tl, periodically), with the
// geometry's site range (cb0, ncb) set to its own slices and lex0 to the global index of its
// local site 0.  The trajectory kernels then run on a slab unchanged:
//   - a site's force step reads neighbours at most one slice away, so the ghost slices hold
//     everything the slab's own sites read;
//   - after each force launch that writes a link buffer, the ghost slices of that buffer are
//     refreshed from the neighbouring slabs (the halo exchange);
//   - the momenta are the Philox streams of the whole lattice (keyed by lex + lex0), and the
//     plaquette and kinetic partials cover the slab's own sites; the sums add over the slabs
//     before the accept/reject, which every slab then takes identically.
// So a trajectory gives the links and accept decisions of a single-lattice context with the
// same seed and trajectory index; the energies agree to rounding (the sums add in another
// order).
//
// In a slab the sites of local slice t and parity p are the even/odd indices
// t S/2 .. (t+1) S/2 - 1 (S sites per slice, even), so a face is 2 nd contiguous pieces of S/2
// links, one per direction and parity.  Tl is even, so a global site has the same local
// parity in every slab that holds it and the pieces map one to one.
//
// Transport.  Slabs on one device (count == nslabs) exchange faces with one copy kernel
// over a table of pieces and add their sums with a kernel over the slabs' reduction
// buffers, all queued on one stream, one CUDA graph per trajectory.  Slabs in separate
// processes (one GPU each, count == 1) pack their two faces, exchange them with NCCL
// send/recv and add the sums with an NCCL all-reduce; NCCL is loaded at run time.
#include <dlfcn.h>
#include <nccl.h>

#include <array>
#include <cmath>
#include <utility>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "su2b.h"
#include "su2b_ctx.h"

using namespace su2b;

namespace {

struct Piece {
  const uint4 *src;
  uint4 *dst;
};

// every piece of the table: n 16-byte words from src to dst (piece = blockIdx.y)
__global__ void __launch_bounds__(256) k_copy_pieces(const Piece *__restrict__ pc, long n) {
  const Piece q = pc[blockIdx.y];
  for (long i = blockIdx.x * 256l + threadIdx.x; i < n; i += (long)gridDim.x * 256)
    q.dst[i] = q.src[i];
}

// red[r][i] = sum over the slabs in slab order, for i < n, written back to every slab
__global__ void k_sum_slabs(double *const *__restrict__ red, int nslab, int n) {
  const int i = threadIdx.x;
  if (i < n) {
    double v = 0.;
    for (int r = 0; r < nslab; r++) v += red[r][i];
    for (int r = 0; r < nslab; r++) red[r][i] = v;
  }
}

// ---- NCCL, resolved from libnccl.so.2 when the first handle connects ----
struct NcclApi {
  ncclResult_t (*get_unique_id)(ncclUniqueId *);
  ncclResult_t (*comm_init_rank)(ncclComm_t *, int, ncclUniqueId, int);
  ncclResult_t (*comm_destroy)(ncclComm_t);
  ncclResult_t (*send)(const void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t);
  ncclResult_t (*recv)(void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t);
  ncclResult_t (*group_start)();
  ncclResult_t (*group_end)();
  ncclResult_t (*all_reduce)(const void *, void *, size_t, ncclDataType_t, ncclRedOp_t,
                             ncclComm_t, cudaStream_t);
  const char *(*error_string)(ncclResult_t);
};

const NcclApi *nccl_api(std::string *why) {
  static std::mutex m;
  static NcclApi api;
  static int state = 0;  // 0 not tried, 1 loaded, -1 failed
  static std::string err;
  std::lock_guard<std::mutex> lock(m);
  if (state == 0) {
    void *h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
    if (!h) h = dlopen("libnccl.so", RTLD_NOW | RTLD_GLOBAL);
    state = -1;
    if (!h) {
      err = std::string("libnccl.so.2 not found: ") + dlerror();
    } else {
      bool ok = true;
      auto sym = [&](const char *name) {
        void *p = dlsym(h, name);
        if (!p) ok = false;
        return p;
      };
      api.get_unique_id = (decltype(api.get_unique_id))sym("ncclGetUniqueId");
      api.comm_init_rank = (decltype(api.comm_init_rank))sym("ncclCommInitRank");
      api.comm_destroy = (decltype(api.comm_destroy))sym("ncclCommDestroy");
      api.send = (decltype(api.send))sym("ncclSend");
      api.recv = (decltype(api.recv))sym("ncclRecv");
      api.group_start = (decltype(api.group_start))sym("ncclGroupStart");
      api.group_end = (decltype(api.group_end))sym("ncclGroupEnd");
      api.all_reduce = (decltype(api.all_reduce))sym("ncclAllReduce");
      api.error_string = (decltype(api.error_string))sym("ncclGetErrorString");
      if (ok)
        state = 1;
      else
        err = "libnccl.so.2 lacks a symbol (ncclSend / ncclRecv need NCCL >= 2.7)";
    }
  }
  if (state == 1) return &api;
  *why = err;
  return nullptr;
}

}  // namespace

struct su2b_slabs {
  int nslabs = 0, first = 0, count = 0, device = 0;
  int Lt = 0, nd = 4, Tl = 0;
  long S = 0;  // sites per time slice
  bool link64 = true;
  std::vector<su2b_ctx *> sl;
  std::vector<cudaStream_t> own;  // the streams the slab contexts were created with
  cudaStream_t s = nullptr;       // every slab's work is queued here
  // overlap: each force step updates the boundary slices first and exchanges them on
  // stream xs while the interior slices are updated on s
  bool overlap = false;
  cudaStream_t xs = nullptr;
  cudaEvent_t ev_b = nullptr, ev_x = nullptr;
  std::vector<std::array<void *, 3>> buf;  // each slab's three link buffers
  int role[3] = {0, 1, 2};  // the buffers that hold the current field, and the two others
  long piece_n = 0;         // 16-byte words per piece (S/2 links)
  int npieces = 0;          // pieces per exchange table
  Piece *xchg[3] = {};      // one device: the exchange of buffer k between all slabs
  double **reds = nullptr;  // one device: the slabs' reduction buffers
  // NCCL (one slab per process)
  const NcclApi *nc = nullptr;
  ncclComm_t comm = nullptr;
  int nranks = 1, rank = 0;
  uint4 *sendbuf = nullptr, *recvbuf = nullptr;  // [lower face | upper face]
  double *tune_dev = nullptr;  // the tuner's times per force shape, reduced over the ranks
  Piece *pack[3] = {}, *unpack[3] = {};
  std::vector<void *> allocs;
  struct Graph {
    cudaGraphExec_t exec;
    int fin;
    long kernels;
  };
  std::map<std::string, Graph> graphs;
  long launches = 0;
  std::string err;
};

namespace {

int fail(su2b_slabs *h, int code, const std::string &msg) {
  h->err = msg;
  return code;
}
// the first slab context's error becomes the handle's, unless the handle has its own
int from_ctx(su2b_slabs *h, int rc) {
  if (rc != SU2B_OK && h->err.empty())
    for (const su2b_ctx *c : h->sl)
      if (!c->err.empty()) {
        h->err = c->err;
        break;
      }
  return rc;
}
#define SLAB_CUDA(call)                                                                    \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess)                                                                 \
      return fail(h, SU2B_ERR_CUDA,                                                        \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                     \
  } while (0)

// the 16-byte word offset of piece (mu, p) of local slice ts in a link buffer of c
size_t slice_word(const su2b_ctx *c, long S, int mu, int p, int ts) {
  const size_t l = (size_t)mu * c->g.V + (size_t)p * c->g.Vh + (size_t)ts * (S / 2);
  return l * (c->link_bytes() / 16);
}
uint4 *piece_at(su2b_slabs *h, int r, int k, int mu, int p, int ts) {
  return (uint4 *)h->buf[r][k] + slice_word(h->sl[r], h->S, mu, p, ts);
}

int upload_table(su2b_slabs *h, const std::vector<Piece> &v, Piece **dev) {
  void *p = nullptr;
  SLAB_CUDA(cudaMalloc(&p, sizeof(Piece) * v.size()));
  h->allocs.push_back(p);
  SLAB_CUDA(cudaMemcpy(p, v.data(), sizeof(Piece) * v.size(), cudaMemcpyHostToDevice));
  *dev = (Piece *)p;
  return SU2B_OK;
}

// Exchange tables are ordered by piece (mu, p) first, so the entries of one piece -- all a
// checkerboard pass changes -- are one contiguous run: entries (2 mu + p) * per_piece ..
// One device: per piece, for every slab r, its first slice goes to the upper ghost slice of
// slab r - 1 and its last slice to the lower ghost slice of slab r + 1 (periodically).
int build_local_tables(su2b_slabs *h) {
  const int R = h->count;
  for (int k = 0; k < 3; k++) {
    std::vector<Piece> v;
    for (int mu = 0; mu < h->nd; mu++)
      for (int p = 0; p < 2; p++)
        for (int r = 0; r < R; r++) {
          const int dn = (r + R - 1) % R, up = (r + 1) % R;
          v.push_back({piece_at(h, r, k, mu, p, 1), piece_at(h, dn, k, mu, p, h->Tl + 1)});
          v.push_back({piece_at(h, r, k, mu, p, h->Tl), piece_at(h, up, k, mu, p, 0)});
        }
    h->npieces = (int)v.size();
    SU2B_CKS(upload_table(h, v, &h->xchg[k]));
  }
  std::vector<double *> reds;
  for (su2b_ctx *c : h->sl) reds.push_back(c->red);
  void *p = nullptr;
  SLAB_CUDA(cudaMalloc(&p, sizeof(double *) * reds.size()));
  h->allocs.push_back(p);
  SLAB_CUDA(cudaMemcpy(p, reds.data(), sizeof(double *) * reds.size(), cudaMemcpyHostToDevice));
  h->reds = (double **)p;
  return SU2B_OK;
}

// NCCL: the send buffer holds [first slice | last slice], each as its 2 nd pieces in (mu, p)
// order; the receive buffer [from the slab below | from the slab above] goes to
// [ghost 0 | ghost Tl + 1].  The pack and unpack tables list per piece its two faces.
int build_nccl_tables(su2b_slabs *h) {
  const long face = 2l * h->nd * h->piece_n;
  for (int k = 0; k < 3; k++) {
    std::vector<Piece> pk, up;
    for (int mu = 0; mu < h->nd; mu++)
      for (int p = 0; p < 2; p++) {
        const long at = (2 * mu + p) * h->piece_n;
        pk.push_back({piece_at(h, 0, k, mu, p, 1), h->sendbuf + at});
        pk.push_back({piece_at(h, 0, k, mu, p, h->Tl), h->sendbuf + face + at});
        up.push_back({h->recvbuf + at, piece_at(h, 0, k, mu, p, 0)});
        up.push_back({h->recvbuf + face + at, piece_at(h, 0, k, mu, p, h->Tl + 1)});
      }
    SU2B_CKS(upload_table(h, pk, &h->pack[k]));
    SU2B_CKS(upload_table(h, up, &h->unpack[k]));
  }
  return SU2B_OK;
}

cudaError_t copy_pieces(const Piece *tab, int npieces, long n, cudaStream_t s) {
  const long blocks = (n + 255) / 256;
  k_copy_pieces<<<dim3((unsigned)(blocks < 64 ? blocks : 64), npieces), 256, 0, s>>>(tab, n);
  return cudaGetLastError();
}

#define NCCL_CK(call)                                                                      \
  do {                                                                                     \
    ncclResult_t r_ = (call);                                                              \
    if (r_ != ncclSuccess)                                                                 \
      return fail(h, SU2B_ERR_CUDA, std::string(#call) + ": " + h->nc->error_string(r_));  \
  } while (0)

// a kernel launch through a slab context, its failure reported as the handle's error
#define SLAB_LAUNCH(ctx_, kclass, call)                                                    \
  do {                                                                                     \
    su2b_ctx *ctx = (ctx_);                                                                \
    const int rc_ = [&]() -> int {                                                         \
      SU2B_LAUNCH(kclass, call);                                                           \
      return SU2B_OK;                                                                      \
    }();                                                                                   \
    if (rc_ != SU2B_OK) return from_ctx(h, rc_);                                           \
  } while (0)

// refresh the ghost slices of buffer k of every slab: every piece (piece < 0) or only
// piece 2 mu + p
int exchange(su2b_slabs *h, int k, int piece = -1, cudaStream_t st = nullptr) {
  if (!st) st = h->s;
  const int n_of = piece < 0 ? 2 * h->nd : 1, first = piece < 0 ? 0 : piece;
  if (!h->comm) {
    const int per = 2 * h->count;  // table entries per piece
    SLAB_CUDA(copy_pieces(h->xchg[k] + first * per, n_of * per, h->piece_n, st));
    h->launches++;
    return SU2B_OK;
  }
  const long face = 2l * h->nd * h->piece_n;
  const long at = first * h->piece_n;  // the pieces' place in each face of the buffers
  const size_t bytes = (size_t)n_of * h->piece_n * 16;
  const int up = (h->rank + 1) % h->nranks, dn = (h->rank + h->nranks - 1) % h->nranks;
  SLAB_CUDA(copy_pieces(h->pack[k] + 2 * first, 2 * n_of, h->piece_n, st));
  // with two slabs both neighbours are one process: sends and receives to one peer match
  // in the order they are posted, so the order is the same on every rank
  NCCL_CK(h->nc->group_start());
  NCCL_CK(h->nc->send(h->sendbuf + face + at, bytes, ncclUint8, up, h->comm, st));
  NCCL_CK(h->nc->send(h->sendbuf + at, bytes, ncclUint8, dn, h->comm, st));
  NCCL_CK(h->nc->recv(h->recvbuf + at, bytes, ncclUint8, dn, h->comm, st));
  NCCL_CK(h->nc->recv(h->recvbuf + face + at, bytes, ncclUint8, up, h->comm, st));
  NCCL_CK(h->nc->group_end());
  SLAB_CUDA(copy_pieces(h->unpack[k] + 2 * first, 2 * n_of, h->piece_n, st));
  h->launches += 2;
  return SU2B_OK;
}

// red[0 .. n-1] of every slab becomes the sum over all slabs
int sum_over_slabs(su2b_slabs *h, int n) {
  if (!h->comm) {
    k_sum_slabs<<<1, 32, 0, h->s>>>(h->reds, h->count, n);
    SLAB_CUDA(cudaGetLastError());
    h->launches++;
    return SU2B_OK;
  }
  NCCL_CK(h->nc->all_reduce(h->sl[0]->red, h->sl[0]->red, (size_t)n, ncclFloat64, ncclSum,
                            h->comm, h->s));
  return SU2B_OK;
}

bool connected(const su2b_slabs *h) { return h->count == h->nslabs || h->comm != nullptr; }

void set_roles(su2b_slabs *h) {
  for (int r = 0; r < h->count; r++) {
    h->sl[r]->U = h->buf[r][h->role[0]];
    h->sl[r]->U_old = h->buf[r][h->role[1]];
    h->sl[r]->U2 = h->buf[r][h->role[2]];
  }
}

// the fused trajectory over all slabs (the single-lattice form is enqueue_fused in hmc.cu):
// S (buffer role[0]) is never written; X and Y alternate; *fin receives the buffer that holds
// the final field
template <class T>
int enqueue(su2b_slabs *h, const std::vector<HmcFusedOp> &fops, int *fin) {
  const int R = h->count;
  const int iS = h->role[0], iX = h->role[1], iY = h->role[2];
  cudaStream_t s = h->s;
  std::vector<int> nb_start(R, 0), nb_kin(R, 0), nb_plaq(R, 0);
  for (int r = 0; r < R; r++) {
    su2b_ctx *ctx = h->sl[r];
    SU2B_LAUNCH(SU2B_K_MOMENTA, momenta_plaq<T>(ctx->g, h->buf[r][iS], (T *)ctx->P,
                                                ctx->tparams, ctx->xi, ctx->part_slot(1),
                                                &nb_start[r], s, true));
  }
  const double f = h->sl[0]->beta / h->sl[0]->Nc();
  int cur = iS, F = -1;
  auto next = [&](int c) { return c == iX ? iY : iX; };
  for (size_t i = 0; i < fops.size(); i++) {
    const HmcFusedOp &o = fops[i];
    int mode = FM_HAS_IN | (o.kinetic ? FM_KINETIC : 0);
    int out;
    if (o.kind == 1) {
      mode |= FM_UPDATE;
      out = next(cur);
    } else {  // the last momentum step writes the reunitarised final field
      mode |= FM_RESTORE;
      out = F = (cur == iS) ? iX : next(cur);
    }
    // the force step on sites cb0 .. cb0 + ncb - 1 of slab r, its kinetic partials at kin
    auto launch = [&](int r, int cb0, int ncb, double *kin, int *nb) -> int {
      su2b_ctx *ctx = h->sl[r];
      Geom gr = ctx->g;
      gr.cb0 = cb0;
      gr.ncb = ncb;
      SU2B_LAUNCH(SU2B_K_FORCE,
                  force_update<T>(gr, h->buf[r][cur], 0, (T *)ctx->P, nullptr, f, -o.cm,
                                  ctx->xi, mode, kin, nb, h->buf[r][out], o.cg, s,
                                  ctx->tune_force, false));
      return SU2B_OK;
    };
    const int half = (int)(h->S / 2);  // sites of one parity in one slice
    if (h->overlap && h->Tl > 2) {
      // the two boundary slices first; their faces travel on the exchange stream while
      // the interior slices are updated; the next step waits for the ghost slices
      std::vector<int> nb0(R, 0), nb1(R, 0);
      for (int r = 0; r < R; r++) {
        double *kin = h->sl[r]->part_slot(2);
        SU2B_CKS(launch(r, half, half, kin, &nb0[r]));
        SU2B_CKS(launch(r, h->Tl * half, half, kin + nb0[r], &nb1[r]));
      }
      {
        su2b_ctx *ctx = h->sl[0];
        SU2B_CK(cudaEventRecord(h->ev_b, s));
        SU2B_CK(cudaStreamWaitEvent(h->xs, h->ev_b, 0));
      }
      SU2B_CKS(exchange(h, out, -1, h->xs));
      for (int r = 0; r < R; r++) {
        int nb2 = 0;
        SU2B_CKS(launch(r, 2 * half, (h->Tl - 2) * half,
                        h->sl[r]->part_slot(2) + nb0[r] + nb1[r], &nb2));
        if (o.kinetic) nb_kin[r] = nb0[r] + nb1[r] + nb2;
      }
      {
        su2b_ctx *ctx = h->sl[0];
        SU2B_CK(cudaEventRecord(h->ev_x, h->xs));
        SU2B_CK(cudaStreamWaitEvent(s, h->ev_x, 0));
      }
    } else {
      for (int r = 0; r < R; r++) {
        int nb = 0;
        SU2B_CKS(launch(r, h->sl[r]->g.cb0, h->sl[r]->g.ncb, h->sl[r]->part_slot(2), &nb));
        if (o.kinetic) nb_kin[r] = nb;
      }
      SU2B_CKS(exchange(h, out));
    }
    if (o.kind == 1) cur = out;
  }
  for (int r = 0; r < R; r++) {
    su2b_ctx *ctx = h->sl[r];
    SU2B_LAUNCH(SU2B_K_PLAQUETTE, plaq_partials<T>(ctx->g, h->buf[r][F], 0, ctx->xi,
                                                   ctx->part_slot(0), &nb_plaq[r], s));
    SU2B_CK(cudaMemsetAsync(ctx->red, 0, 10 * sizeof(double), s));
    SU2B_LAUNCH(SU2B_K_OTHER, reduce_final(ctx->part_slot(1), nb_start[r], 4, ctx->red, s));
    SU2B_LAUNCH(SU2B_K_OTHER, reduce_final(ctx->part_slot(2), nb_kin[r], 1, ctx->red + 4, s));
    SU2B_LAUNCH(SU2B_K_OTHER, reduce_final(ctx->part_slot(0), nb_plaq[r], 3, ctx->red + 5, s));
  }
  SU2B_CKS(sum_over_slabs(h, 8));
  for (int r = 0; r < R; r++) {
    su2b_ctx *ctx = h->sl[r];
    SU2B_LAUNCH(SU2B_K_OTHER, accept_step(ctx->red, ctx->tparams, ctx->traj, s));
  }
  su2b_ctx *ctx = h->sl[0];
  SU2B_CK(cudaMemcpyAsync(ctx->h_traj, ctx->traj, sizeof(TrajDev), cudaMemcpyDeviceToHost, s));
  SU2B_CK(cudaMemcpyAsync(ctx->h_red, ctx->red, 10 * sizeof(double), cudaMemcpyDeviceToHost, s));
  *fin = F;
  return SU2B_OK;
}

long ctx_launches(const su2b_slabs *h) {
  long n = 0;
  for (const su2b_ctx *c : h->sl) n += c->launches;
  return n;
}
void reset_launches(su2b_slabs *h, const std::vector<long> &ctx_n, long own_n) {
  for (size_t r = 0; r < h->sl.size(); r++) h->sl[r]->launches = ctx_n[r];
  h->launches = own_n;
}

int trajectory(su2b_slabs *h, const su2b_hmc_params *prm, su2b_traj_result *res) {
  if (!prm || !res) return fail(h, SU2B_ERR_INVALID, "params or result is NULL");
  if (prm->n_steps < 1) return fail(h, SU2B_ERR_INVALID, "n_steps must be >= 1");
  if (!connected(h))
    return fail(h, SU2B_ERR_INVALID,
                "the handle holds a part of the slabs: connect it to the others first");
  if (prm->momenta_host || prm->revtest || prm->fermion_mass > 0.0)
    return fail(h, SU2B_ERR_UNSUPPORTED,
                "slabs take Philox momenta, no reversibility test and no fermions");
  const std::vector<HmcFusedOp> fops =
    su2b_fuse(su2b_schedule(prm->integrator, prm->n_steps, prm->tau));
  const bool fused_form = prm->integrator == SU2B_LEAPFROG || prm->integrator == SU2B_OMF2 ||
                          prm->integrator == SU2B_OMF4;
  for (size_t i = 0; i < fops.size(); i++)
    if (!fused_form || fops[i].kind != (i + 1 == fops.size() ? 0 : 1))
      return fail(h, SU2B_ERR_UNSUPPORTED,
                  "slabs run leapfrog, omf2 and omf4 (momentum steps with fused gauge steps)");
  for (su2b_ctx *c : h->sl) c->begin_call();
  cudaStream_t s = h->s;
  for (su2b_ctx *c : h->sl) {
    TrajParams &tp = *c->h_tparams;
    tp.beta = c->beta;
    tp.Nc = c->Nc();
    tp.u_host = prm->uniform_host;
    tp.seed = prm->seed;
    tp.traj = prm->traj;
    tp.accept_reject = prm->accept_reject;
    SLAB_CUDA(cudaMemcpyAsync(c->tparams, c->h_tparams, sizeof(TrajParams),
                              cudaMemcpyHostToDevice, s));
  }
  int F = -1;
  if (h->comm) {  // NCCL: launched directly
    const int rc = h->link64 ? enqueue<double>(h, fops, &F) : enqueue<float>(h, fops, &F);
    if (rc != SU2B_OK) return from_ctx(h, rc);
  } else {
    char key[192];
    snprintf(key, sizeof key, "%d/%d/%.17g/%d%d%d/%d/%d", prm->integrator, prm->n_steps,
             prm->tau, h->role[0], h->role[1], h->role[2], h->sl[0]->tune_force,
             (int)h->overlap);
    auto it = h->graphs.find(key);
    if (it == h->graphs.end()) {
      // the capture counts the graph's kernels; each replay adds them
      std::vector<long> ctx_n;
      for (const su2b_ctx *c : h->sl) ctx_n.push_back(c->launches);
      const long own_n = h->launches, n0 = ctx_launches(h) + own_n;
      cudaGraph_t graph = nullptr;
      SLAB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      const int rc = h->link64 ? enqueue<double>(h, fops, &F) : enqueue<float>(h, fops, &F);
      const cudaError_t ec = cudaStreamEndCapture(s, &graph);
      const long kernels = ctx_launches(h) + h->launches - n0;
      reset_launches(h, ctx_n, own_n);
      if (rc != SU2B_OK) {
        if (graph) cudaGraphDestroy(graph);
        return from_ctx(h, rc);
      }
      SLAB_CUDA(ec);
      su2b_slabs::Graph gr{nullptr, F, kernels};
      const cudaError_t ei = cudaGraphInstantiate(&gr.exec, graph, 0);
      cudaGraphDestroy(graph);
      SLAB_CUDA(ei);
      it = h->graphs.emplace(key, gr).first;
    }
    F = it->second.fin;
    SLAB_CUDA(cudaGraphLaunch(it->second.exec, s));
    h->launches += it->second.kernels;
  }
  SLAB_CUDA(cudaStreamSynchronize(s));
  const TrajDev &t = *h->sl[0]->h_traj;
  const double *red = h->sl[0]->h_red;
  if (t.accepted) {  // the final field becomes current
    const int S0 = h->role[0], X0 = h->role[1], Y0 = h->role[2];
    h->role[0] = F;
    h->role[1] = S0;
    h->role[2] = (F == X0) ? Y0 : X0;
    set_roles(h);
  }
  res->accepted = t.accepted;
  res->dH = t.dH;
  for (int k = 0; k < 3; k++) {
    res->H_old[k] = t.H_old[k];
    res->H_new[k] = t.H_new[k];
  }
  res->ddH = 0.0;
  res->plaquette = t.accepted ? red[5] : red[1];
  res->cg_iterations = 0;
  return SU2B_OK;
}

}  // namespace

extern "C" int su2b_slabs_create(int Lx, int Ly, int Lz, int Lt, int ndims, double beta,
                                 double xi, int precision, int nslabs, int first, int count,
                                 int device, su2b_slabs **out) {
  if (!out) return SU2B_ERR_INVALID;
  *out = nullptr;
  if (ndims < 2 || ndims > 4 || nslabs < 1 || count < 1 || first < 0 ||
      first + count > nslabs)
    return SU2B_ERR_INVALID;
  // slabs of an even, positive number of slices (Lt = 0 would leave no slice to wrap to)
  if (Lt < 2 || Lt % nslabs != 0 || (Lt / nslabs) % 2 != 0) return SU2B_ERR_INVALID;
  // the whole lattice within the single lattice's 2^29 sites: the Philox keys and lex0 are
  // global site indices (the volume formed one extent at a time, so no product can wrap)
  long Vg = 1;
  for (const int Lk : {Lx, Ly, Lz, Lt})
    if (Lk < 1 || Lk > (1l << 29) || (Vg *= Lk) > (1l << 29)) return SU2B_ERR_INVALID;
  su2b_slabs *h = new su2b_slabs();
  h->nslabs = nslabs;
  h->first = first;
  h->count = count;
  h->device = device;
  h->Lt = Lt;
  h->nd = ndims;
  h->Tl = Lt / nslabs;
  h->S = (long)Lx * Ly * Lz;
  auto fin = [&](int rc) -> int {
    if (rc != SU2B_OK) {
      su2b_slabs_destroy(h);
      return rc;
    }
    *out = h;
    return SU2B_OK;
  };
  for (int r = 0; r < count; r++) {
    su2b_ctx *c = nullptr;
    const int rc = su2b_ctx_create(SU2B_GROUP_SU2, Lx, Ly, Lz, h->Tl + 2, ndims, beta, xi,
                                   precision, device, &c);
    if (rc != SU2B_OK) return fin(rc);
    h->sl.push_back(c);
    h->own.push_back(c->stream);
    const int t0 = (first + r) * h->Tl;
    c->g.cb0 = (int)(h->S / 2);
    c->g.ncb = (int)(h->Tl * h->S / 2);
    c->g.lex0 = (int)((long)(t0 - 1) * h->S);
    h->buf.push_back({c->U, c->U_old, c->U2});
  }
  h->link64 = h->sl[0]->link64;
  h->s = h->sl[0]->stream;
  for (su2b_ctx *c : h->sl) c->stream = h->s;
  h->piece_n = (h->S / 2) * (long)(h->sl[0]->link_bytes() / 16);
  if (cudaSetDevice(device) != cudaSuccess) return fin(fail(h, SU2B_ERR_CUDA, "cudaSetDevice"));
  // the exchange stream at the highest priority, so that its copy and NCCL blocks take SMs
  // as the interior update's blocks retire instead of waiting for the whole launch
  int prio_lo = 0, prio_hi = 0;
  cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
  if (cudaStreamCreateWithPriority(&h->xs, cudaStreamNonBlocking, prio_hi) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->ev_b, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->ev_x, cudaEventDisableTiming) != cudaSuccess)
    return fin(fail(h, SU2B_ERR_CUDA, "exchange stream or events"));
  if (count == nslabs) return fin(build_local_tables(h));
  return fin(SU2B_OK);
}

extern "C" int su2b_slabs_destroy(su2b_slabs *h) {
  if (!h) return SU2B_ERR_INVALID;
  cudaSetDevice(h->device);
  if (h->s) cudaStreamSynchronize(h->s);
  if (h->xs) cudaStreamSynchronize(h->xs);
  for (auto &kv : h->graphs) cudaGraphExecDestroy(kv.second.exec);
  if (h->ev_b) cudaEventDestroy(h->ev_b);
  if (h->ev_x) cudaEventDestroy(h->ev_x);
  if (h->xs) cudaStreamDestroy(h->xs);
  if (h->comm && h->nc) h->nc->comm_destroy(h->comm);
  for (void *p : h->allocs) cudaFree(p);
  for (size_t r = 0; r < h->sl.size(); r++) {
    h->sl[r]->stream = h->own[r];
    su2b_ctx_destroy(h->sl[r]);
  }
  delete h;
  return SU2B_OK;
}

extern "C" const char *su2b_slabs_last_error(const su2b_slabs *h) {
  return h ? h->err.c_str() : "null handle";
}

extern "C" int su2b_slabs_info(const su2b_slabs *h, int *nslabs, int *first, int *count,
                               int *slices) {
  if (!h) return SU2B_ERR_INVALID;
  if (nslabs) *nslabs = h->nslabs;
  if (first) *first = h->first;
  if (count) *count = h->count;
  if (slices) *slices = h->Tl;
  return SU2B_OK;
}

extern "C" int su2b_slabs_nccl_id(void *id) {
  if (!id) return SU2B_ERR_INVALID;
  std::string why;
  const NcclApi *nc = nccl_api(&why);
  if (!nc) return SU2B_ERR_UNSUPPORTED;
  ncclUniqueId u;
  if (nc->get_unique_id(&u) != ncclSuccess) return SU2B_ERR_CUDA;
  memcpy(id, &u, sizeof u);
  return SU2B_OK;
}

extern "C" int su2b_slabs_connect(su2b_slabs *h, const void *id, int nranks, int rank) {
  if (!h) return SU2B_ERR_INVALID;
  h->err.clear();
  if (!id) return fail(h, SU2B_ERR_INVALID, "id is NULL");
  if (h->comm) return fail(h, SU2B_ERR_INVALID, "already connected");
  if (h->count != 1 || nranks != h->nslabs || rank != h->first)
    return fail(h, SU2B_ERR_INVALID,
                "connect wants one slab per process: nranks = nslabs, rank = first");
  std::string why;
  h->nc = nccl_api(&why);
  if (!h->nc) return fail(h, SU2B_ERR_UNSUPPORTED, why);
  SLAB_CUDA(cudaSetDevice(h->device));
  ncclUniqueId u;
  memcpy(&u, id, sizeof u);
  ncclComm_t comm = nullptr;
  NCCL_CK(h->nc->comm_init_rank(&comm, nranks, u, rank));
  h->comm = comm;
  h->nranks = nranks;
  h->rank = rank;
  // the faces travel through NCCL while the interior slices are updated: with the exchange
  // stream at the highest priority this beats the plain exchange (one rank on one B200:
  // 304 against 299 traj/s at 32^4), where for device copies the split launches lose
  h->overlap = true;
  const size_t bytes = (size_t)4 * h->nd * h->piece_n * 16;  // two faces
  void *a = nullptr, *b = nullptr;
  SLAB_CUDA(cudaMalloc(&a, bytes));
  h->allocs.push_back(a);
  SLAB_CUDA(cudaMalloc(&b, bytes));
  h->allocs.push_back(b);
  h->sendbuf = (uint4 *)a;
  h->recvbuf = (uint4 *)b;
  void *t = nullptr;
  SLAB_CUDA(cudaMalloc(&t, sizeof(double) * FORCE_VARIANTS));
  h->allocs.push_back(t);
  h->tune_dev = (double *)t;
  return build_nccl_tables(h);
}

// host field of the whole lattice (reference order, t slowest): rows of S nd links
extern "C" int su2b_slabs_upload(su2b_slabs *h, const double *U_host) {
  if (!h) return SU2B_ERR_INVALID;
  h->err.clear();
  if (!U_host) return fail(h, SU2B_ERR_INVALID, "U_host is NULL");
  SLAB_CUDA(cudaSetDevice(h->device));
  const size_t row = (size_t)h->S * h->nd * 4;  // doubles per time slice
  for (int r = 0; r < h->count; r++) {
    su2b_ctx *c = h->sl[r];
    c->begin_call();
    const int t0 = (h->first + r) * h->Tl;
    const int lo = (t0 + h->Lt - 1) % h->Lt, hi = (t0 + h->Tl) % h->Lt;
    SLAB_CUDA(cudaMemcpyAsync(c->stage, U_host + lo * row, row * 8, cudaMemcpyHostToDevice,
                              h->s));
    SLAB_CUDA(cudaMemcpyAsync(c->stage + row, U_host + t0 * row, h->Tl * row * 8,
                              cudaMemcpyHostToDevice, h->s));
    SLAB_CUDA(cudaMemcpyAsync(c->stage + (h->Tl + 1) * row, U_host + hi * row, row * 8,
                              cudaMemcpyHostToDevice, h->s));
    if (h->link64)
      SLAB_LAUNCH(c, SU2B_K_OTHER, links_from_host<double>(c->g, c->stage, c->U, 0, h->s));
    else
      SLAB_LAUNCH(c, SU2B_K_OTHER, links_from_host<float>(c->g, c->stage, c->U, 0, h->s));
  }
  SLAB_CUDA(cudaStreamSynchronize(h->s));
  return SU2B_OK;
}

extern "C" int su2b_slabs_download(su2b_slabs *h, double *U_host) {
  if (!h) return SU2B_ERR_INVALID;
  h->err.clear();
  if (!U_host) return fail(h, SU2B_ERR_INVALID, "U_host is NULL");
  SLAB_CUDA(cudaSetDevice(h->device));
  const size_t row = (size_t)h->S * h->nd * 4;
  for (int r = 0; r < h->count; r++) {
    su2b_ctx *c = h->sl[r];
    c->begin_call();
    const int t0 = (h->first + r) * h->Tl;
    if (h->link64)
      SLAB_LAUNCH(c, SU2B_K_OTHER, links_to_host<double>(c->g, c->U, c->stage, 0, h->s));
    else
      SLAB_LAUNCH(c, SU2B_K_OTHER, links_to_host<float>(c->g, c->U, c->stage, 0, h->s));
    SLAB_CUDA(cudaMemcpyAsync(U_host + t0 * row, c->stage + row, h->Tl * row * 8,
                              cudaMemcpyDeviceToHost, h->s));
  }
  SLAB_CUDA(cudaStreamSynchronize(h->s));
  return SU2B_OK;
}

extern "C" int su2b_slabs_hmc_trajectory(su2b_slabs *h, const su2b_hmc_params *prm,
                                         su2b_traj_result *res) {
  if (!h) return SU2B_ERR_INVALID;
  h->err.clear();
  SLAB_CUDA(cudaSetDevice(h->device));
  return trajectory(h, prm, res);
}

extern "C" int su2b_slabs_gauge_energy(su2b_slabs *h, int spatial_only, double *out) {
  if (!h) return SU2B_ERR_INVALID;
  h->err.clear();
  if (!out) return fail(h, SU2B_ERR_INVALID, "out is NULL");
  if (!connected(h))
    return fail(h, SU2B_ERR_INVALID,
                "the handle holds a part of the slabs: connect it to the others first");
  SLAB_CUDA(cudaSetDevice(h->device));
  for (su2b_ctx *c : h->sl) {
    c->begin_call();
    int nb = 0;
    if (h->link64)
      SLAB_LAUNCH(c, SU2B_K_PLAQUETTE, plaq_partials<double>(c->g, c->U, 0, c->xi,
                                                             c->part_slot(0), &nb, h->s));
    else
      SLAB_LAUNCH(c, SU2B_K_PLAQUETTE, plaq_partials<float>(c->g, c->U, 0, c->xi,
                                                            c->part_slot(0), &nb, h->s));
    SLAB_LAUNCH(c, SU2B_K_OTHER, reduce_final(c->part_slot(0), nb, 3, c->red, h->s));
  }
  SU2B_CKS(sum_over_slabs(h, 3));
  su2b_ctx *c = h->sl[0];
  SLAB_CUDA(cudaMemcpyAsync(c->h_red, c->red, 3 * sizeof(double), cudaMemcpyDeviceToHost, h->s));
  SLAB_CUDA(cudaStreamSynchronize(h->s));
  *out = c->h_red[spatial_only ? 1 : 0];
  return SU2B_OK;
}

// flat_spacetime::sweep (flat-sweep.hh:64-164) over the slabs, in the single lattice's
// order of passes: direction mu, then parity p of the whole lattice.  A slab's own slices
// start at local slice 1 and at an even global slice, so its local parity of a site is the
// global one flipped: the slabs run local parity p ^ 1.  A pass changes the links of one
// direction and parity only, so after it only that piece of the faces is exchanged.  The
// links' Philox streams are keyed by their global index: the sweep is the single lattice's.
extern "C" int su2b_slabs_metropolis_sweep(su2b_slabs *h, double delta, int N_hit,
                                           uint64_t seed, uint32_t sweep, double *rates) {
  if (!h) return SU2B_ERR_INVALID;
  h->err.clear();
  if (!rates) return fail(h, SU2B_ERR_INVALID, "rates is NULL");
  if (N_hit < 0) return fail(h, SU2B_ERR_INVALID, "N_hit < 0");
  if (!connected(h))
    return fail(h, SU2B_ERR_INVALID,
                "the handle holds a part of the slabs: connect it to the others first");
  SLAB_CUDA(cudaSetDevice(h->device));
  for (su2b_ctx *c : h->sl) {
    c->begin_call();
    SLAB_CUDA(cudaMemsetAsync(c->counts, 0, 2 * sizeof(unsigned long long), h->s));
  }
  for (int mu = 0; mu < h->nd; mu++)
    for (int p = 0; p < 2; p++) {
      const int pl = p ^ 1;
      for (su2b_ctx *c : h->sl) {
        if (h->link64)
          SLAB_LAUNCH(c, SU2B_K_METROPOLIS,
                      metropolis_pass<double>(c->g, c->U, 0, mu, pl, c->beta, c->xi, delta,
                                              N_hit, seed, sweep, c->counts, h->s));
        else
          SLAB_LAUNCH(c, SU2B_K_METROPOLIS,
                      metropolis_pass<float>(c->g, c->U, 0, mu, pl, c->beta, c->xi, delta,
                                             N_hit, seed, sweep, c->counts, h->s));
      }
      SU2B_CKS(exchange(h, h->role[0], 2 * mu + pl));
    }
  if (h->comm)
    NCCL_CK(h->nc->all_reduce(h->sl[0]->counts, h->sl[0]->counts, 2, ncclUint64, ncclSum,
                              h->comm, h->s));
  for (su2b_ctx *c : h->sl)
    SLAB_CUDA(cudaMemcpyAsync(c->h_counts, c->counts, 2 * sizeof(unsigned long long),
                              cudaMemcpyDeviceToHost, h->s));
  SLAB_CUDA(cudaStreamSynchronize(h->s));
  // every slab's counts (one device), or the all-reduced counts of the first
  unsigned long long n0 = 0, n1 = 0;
  for (size_t r = 0; r < (h->comm ? 1 : h->sl.size()); r++) {
    n0 += h->sl[r]->h_counts[0];
    n1 += h->sl[r]->h_counts[1];
  }
  const double nh = (double)(N_hit > 0 ? N_hit : 1);
  const double V = (double)h->S * h->Lt;
  rates[0] = (double)n0 / nh / (V * h->nd);
  rates[1] = (double)n1 / nh / V;
  return SU2B_OK;
}

// ---- the Wilson flow over the slabs (flat-gradient_flow.hh:17-197) ----
namespace {

// one RK3 step (runge_kutta, flat-gradient_flow.hh:17-50) of every slab from link buffer a
// into buffer b (a != b; a is left holding the middle stage): each stage is the force launch
// with its link update fused (a -> b -> a -> b), followed by the exchange of the buffer it
// wrote; with FP32 links the result is reunitarised in FP64, ghost links included (the same
// elementwise operation as on the neighbour's own links, so the ghosts stay exact copies)
int flow_step(su2b_slabs *h, int a, int b, double eps) {
  const double zfac[3] = {(-17.0) / (36.0), (8.0) / (9.0), (-3.0) / (4.0)};
  const double expfac[3] = {-36.0 / 4. / 17.0, 1., -1.};
  int w = a;
  for (int f = 0; f < 3; f++) {
    const int nxt = w == a ? b : a;
    for (int r = 0; r < h->count; r++) {
      su2b_ctx *c = h->sl[r];
      const double Nc = c->Nc();
      const double ff = 2. * Nc * zfac[f] / c->beta * c->beta / Nc;
      const int mode = (f == 0 ? 0 : FM_HAS_IN) | FM_UPDATE;
      const int rc = su2b_q_force(c, h->buf[r][w], c->Z, nullptr, ff, 1.0, mode, nullptr, nullptr,
                                  h->buf[r][nxt], -eps * expfac[f]);
      if (rc != SU2B_OK) return from_ctx(h, rc);
    }
    SU2B_CKS(exchange(h, nxt));
    w = nxt;
  }
  if (!h->link64)
    for (int r = 0; r < h->count; r++) {
      const int rc = su2b_q_restore(h->sl[r], h->buf[r][w]);
      if (rc != SU2B_OK) return from_ctx(h, rc);
    }
  return SU2B_OK;
}

// plaquette sums into red[slot .. slot+2] and clover sums (cloverdef) into red[slot+3 ..
// slot+5] of buffer k on every slab
int measure(su2b_slabs *h, int k, int cloverdef, int slot) {
  for (int r = 0; r < h->count; r++) {
    su2b_ctx *c = h->sl[r];
    int rc = su2b_q_plaq(c, h->buf[r][k], slot);
    if (rc == SU2B_OK) rc = su2b_q_clover(c, h->buf[r][k], cloverdef, slot + 3);
    if (rc != SU2B_OK) return from_ctx(h, rc);
  }
  return SU2B_OK;
}

int begin(su2b_slabs *h) {
  h->err.clear();
  if (!connected(h))
    return fail(h, SU2B_ERR_INVALID,
                "the handle holds a part of the slabs: connect it to the others first");
  SLAB_CUDA(cudaSetDevice(h->device));
  for (su2b_ctx *c : h->sl) c->begin_call();
  return SU2B_OK;
}

}  // namespace

// runge_kutta on the current field (as su2b_flow_step: the flowed field becomes current)
extern "C" int su2b_slabs_flow_step(su2b_slabs *h, double eps) {
  if (!h) return SU2B_ERR_INVALID;
  SU2B_CKS(begin(h));
  SU2B_CKS(flow_step(h, h->role[0], h->role[2], eps));
  std::swap(h->role[0], h->role[2]);
  set_roles(h);
  SLAB_CUDA(cudaStreamSynchronize(h->s));
  return SU2B_OK;
}

// energy_density (flat-energy_density.hh:57-164) of the whole lattice
extern "C" int su2b_slabs_energy_density(su2b_slabs *h, int cloverdef, int ss, double *E,
                                         double *Q) {
  if (!h) return SU2B_ERR_INVALID;
  if (!E || !Q) return fail(h, SU2B_ERR_INVALID, "E or Q is NULL");
  SU2B_CKS(begin(h));
  SU2B_CKS(measure(h, h->role[0], cloverdef, 0));
  SU2B_CKS(sum_over_slabs(h, 6));
  su2b_ctx *c = h->sl[0];
  SLAB_CUDA(cudaMemcpyAsync(c->h_red, c->red, 6 * sizeof(double), cudaMemcpyDeviceToHost, h->s));
  SLAB_CUDA(cudaStreamSynchronize(h->s));
  su2b_finish_clover(c->h_red + 3, (double)h->S * h->Lt, cloverdef, ss, E, Q);
  return SU2B_OK;
}

// gradient_flow (flat-gradient_flow.hh:70-197) of the current field, which stays unchanged:
// the rows of su2b_gradient_flow, the flow running on a copy in the second link buffer
extern "C" int su2b_slabs_gradient_flow(su2b_slabs *h, double tmax, double eps, double tstart,
                                        double *rows, int max_rows, int *n_rows) {
  if (!h) return SU2B_ERR_INVALID;
  if (!n_rows) return fail(h, SU2B_ERR_INVALID, "n_rows is NULL");
  if (!(eps > 0)) return fail(h, SU2B_ERR_INVALID, "eps must be positive");
  if (max_rows < 0 || (!rows && max_rows > 0)) return fail(h, SU2B_ERR_INVALID, "rows buffer");
  SU2B_CKS(begin(h));
  const int S0 = h->role[0], Vt = h->role[1], W2 = h->role[2];
  for (int r = 0; r < h->count; r++)
    SLAB_CUDA(cudaMemcpyAsync(h->buf[r][Vt], h->buf[r][S0],
                              h->sl[r]->link_bytes() * h->sl[r]->NL, cudaMemcpyDeviceToDevice,
                              h->s));
  const double d = (double)h->nd, V = (double)h->S * h->Lt;
  const double ndims_fact = d * (d - 1) / 2.0, ndims_fact_ss = (d - 1) * (d - 2) / 2.0;
  const double den = V * h->sl[0]->Nc();
  su2b_ctx *c = h->sl[0];
  double t[3] = {tstart, tstart, tstart};
  int nr = 0;
  while (t[1] < tmax - eps) {
    t[0] = t[2];
    t[1] = t[0] + eps;
    // two steps per record; the reference prints the observables of the middle step
    SU2B_CKS(flow_step(h, Vt, W2, eps));
    SU2B_CKS(measure(h, W2, 1, 0));
    t[2] = t[1] + eps;
    SU2B_CKS(flow_step(h, W2, Vt, eps));
    SU2B_CKS(sum_over_slabs(h, 6));
    SLAB_CUDA(cudaMemcpyAsync(c->h_red, c->red, 6 * sizeof(double), cudaMemcpyDeviceToHost,
                              h->s));
    SLAB_CUDA(cudaStreamSynchronize(h->s));
    const double *rd = c->h_red;
    const double P1 = rd[0] / den, Pss1 = rd[1] / den;
    double E1, Q1, Ess1, Qss1;
    su2b_finish_clover(rd + 3, V, 1, 0, &E1, &Q1);
    su2b_finish_clover(rd + 3, V, 1, 1, &Ess1, &Qss1);
    const double Ep = ndims_fact - P1, Ep_ss = ndims_fact_ss - Pss1;
    const double Ep_ts_bar = (Ep - Ep_ss) / (d - 1), Ep_ss_bar = Ep_ss / ndims_fact_ss;
    if (nr < max_rows) {
      double *o = rows + 9 * (size_t)nr;
      o[0] = t[1];
      o[1] = sqrt(Ep_ts_bar / Ep_ss_bar);
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
  *n_rows = nr;
  return SU2B_OK;
}

// The first slab of the handle times the shapes.  Slabs in separate processes take the
// maximum of each shape's time over the ranks (a step waits for the slowest slab) and apply
// the tuner's rule to it, so every rank runs the same shape.
extern "C" int su2b_slabs_autotune(su2b_slabs *h, double *times_us) {
  if (!h) return SU2B_ERR_INVALID;
  h->err.clear();
  if (!connected(h))
    return fail(h, SU2B_ERR_INVALID,
                "the handle holds a part of the slabs: connect it to the others first");
  double t[FORCE_VARIANTS] = {};
  const int rc = su2b_autotune(h->sl[0], nullptr, 1, t);
  if (rc != SU2B_OK && !h->comm) return from_ctx(h, rc);
  if (h->comm) {
    // a rank whose timing failed still joins the all-reduce, with a time that marks the
    // failure on every rank, so that no rank is left waiting in the collective
    constexpr double FAILED = 1e300;
    if (rc != SU2B_OK)
      for (double &x : t) x = FAILED;
    SLAB_CUDA(cudaMemcpyAsync(h->tune_dev, t, sizeof t, cudaMemcpyHostToDevice, h->s));
    NCCL_CK(h->nc->all_reduce(h->tune_dev, h->tune_dev, FORCE_VARIANTS, ncclFloat64, ncclMax,
                              h->comm, h->s));
    SLAB_CUDA(cudaMemcpyAsync(t, h->tune_dev, sizeof t, cudaMemcpyDeviceToHost, h->s));
    SLAB_CUDA(cudaStreamSynchronize(h->s));
    if (rc != SU2B_OK) return from_ctx(h, rc);
    if (t[0] >= FAILED)
      return fail(h, SU2B_ERR_CUDA, "the launch-shape timing failed on another rank");
    double fastest = t[0];
    for (int v = 1; v < FORCE_VARIANTS; v++) fastest = t[v] < fastest ? t[v] : fastest;
    int best = 0;
    while (t[best] > 1.01 * fastest) best++;
    h->sl[0]->tune_force = best;
  }
  for (su2b_ctx *c : h->sl) c->tune_force = h->sl[0]->tune_force;
  if (times_us)
    for (int v = 0; v < FORCE_VARIANTS; v++) times_us[v] = t[v];
  return SU2B_OK;
}

extern "C" int su2b_slabs_tune_get(su2b_slabs *h, int *variant) {
  if (!h) return SU2B_ERR_INVALID;
  if (!variant) return fail(h, SU2B_ERR_INVALID, "variant is NULL");
  *variant = h->sl[0]->tune_force;
  return SU2B_OK;
}

extern "C" int su2b_slabs_tune_set(su2b_slabs *h, int variant) {
  if (!h) return SU2B_ERR_INVALID;
  h->err.clear();
  if (variant < 0 || variant >= FORCE_VARIANTS)
    return fail(h, SU2B_ERR_INVALID, "force variant out of range");
  for (su2b_ctx *c : h->sl) c->tune_force = variant;
  return SU2B_OK;
}

extern "C" int su2b_slabs_set_overlap(su2b_slabs *h, int on) {
  if (!h) return SU2B_ERR_INVALID;
  h->overlap = on != 0;
  return SU2B_OK;
}

extern "C" int su2b_slabs_get_overlap(const su2b_slabs *h, int *on) {
  if (!h || !on) return SU2B_ERR_INVALID;  // a const handle keeps no message
  *on = h->overlap ? 1 : 0;
  return SU2B_OK;
}

extern "C" int su2b_slabs_kernel_launches(su2b_slabs *h, long *count) {
  if (!h) return SU2B_ERR_INVALID;
  if (!count) return fail(h, SU2B_ERR_INVALID, "count is NULL");
  *count = ctx_launches(h) + h->launches;
  return SU2B_OK;
}

extern "C" int su2b_slabs_stream(su2b_slabs *h, void **stream) {
  if (!h) return SU2B_ERR_INVALID;
  if (!stream) return fail(h, SU2B_ERR_INVALID, "stream is NULL");
  *stream = (void *)h->s;
  return SU2B_OK;
}
