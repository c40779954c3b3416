// gaugeio.cu -- gauge configurations on disk in the reference's own binary format, written
// from and read into the device without a host-side layout pass.
//
// gaugeconfig<G>::save / load (gaugeconfig.hh:225-252) write the link vector's memory as it
// is: one object per link in the order ((((t*Lx+x)*Ly+y)*Lz+z)*ndims + mu).  An _su2 object
// (su2.hh:11-16) is {size_t N_c = 2; complex<double> a; complex<double> b;} = 40 bytes, an
// _u1 object (u1.hh:11-15) {size_t N_c = 1; double a;} = 16 bytes (x86-64 layout, no
// padding).  Here a conversion kernel produces these records directly from the even/odd
// device links into the device staging buffer, in chunks; the host only moves bytes:
// chunk k is copied into one of two pinned buffers while chunk k-1 is written to the file
// (load: read, copy in, convert, the same way round).  Loading checks every record's N_c.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "site_ops.cuh"
#include "su2b.h"
#include "su2b_ctx.h"

namespace su2b {
namespace {

constexpr int NT_IO = 256;

struct RecSu2 {
  unsigned long long nc;
  double ar, ai, br, bi;
};
struct RecU1 {
  unsigned long long nc;
  double a;
};
static_assert(sizeof(RecSu2) == 40 && sizeof(RecU1) == 16, "record layout");

// reference link index i -> device link index mu*V + eo(site)
__device__ __forceinline__ size_t dev_link(const Geom &g, size_t i) {
  const int nd = g.nd;
  const int lex = (int)(i / nd), mu = (int)(i % nd);
  const Site s = site_from_lex(g, lex);
  return (size_t)mu * g.V + (size_t)s.p * g.Vh + (lex >> 1);
}

template <class T>
__global__ void k_to_records(Geom g, const void *__restrict__ Uv, int group, size_t l0,
                             size_t n, void *out) {
  for (size_t k = blockIdx.x * (size_t)NT_IO + threadIdx.x; k < n;
       k += (size_t)gridDim.x * NT_IO) {
    const size_t d = dev_link(g, l0 + k);
    if (group == 0) {
      const Su2<double> u = to64(ld_link((const LinkT<T> *)Uv + d));
      ((RecSu2 *)out)[k] = RecSu2{2ull, u.ar, u.ai, u.br, u.bi};
    } else {
      ((RecU1 *)out)[k] = RecU1{1ull, ((const double *)Uv)[d]};
    }
  }
}

template <class T>
__global__ void k_from_records(Geom g, void *__restrict__ Uv, int group, size_t l0, size_t n,
                               const void *in, int *bad) {
  for (size_t k = blockIdx.x * (size_t)NT_IO + threadIdx.x; k < n;
       k += (size_t)gridDim.x * NT_IO) {
    const size_t d = dev_link(g, l0 + k);
    if (group == 0) {
      const RecSu2 r = ((const RecSu2 *)in)[k];
      if (r.nc != 2ull) atomicExch(bad, 1);
      st_link((LinkT<T> *)Uv + d, from64<T>(Su2<double>{r.ar, r.ai, r.br, r.bi}));
    } else {
      const RecU1 r = ((const RecU1 *)in)[k];
      if (r.nc != 1ull) atomicExch(bad, 1);
      ((double *)Uv)[d] = r.a;
    }
  }
}

int io_grid(size_t n) {
  const size_t b = (n + NT_IO - 1) / NT_IO;
  return (int)(b < 65536 ? (b ? b : 1) : 65536);
}

struct Pinned {
  void *p[2] = {nullptr, nullptr};
  cudaEvent_t ev[2] = {nullptr, nullptr};
  ~Pinned() {
    for (int k = 0; k < 2; k++) {
      if (ev[k]) cudaEventDestroy(ev[k]);
      if (p[k]) cudaFreeHost(p[k]);
    }
  }
};

struct File {
  FILE *f = nullptr;
  ~File() {
    if (f) fclose(f);
  }
};

}  // namespace
}  // namespace su2b

using namespace su2b;

static int io_enter(su2b_ctx *ctx) {
  if (!ctx) return SU2B_ERR_INVALID;
  ctx->begin_call();
  SU2B_CK(cudaSetDevice(ctx->device));
  return SU2B_OK;
}

// bytes per record, links per chunk (two chunks fit the staging buffer)
static void io_sizes(const su2b_ctx *ctx, size_t *rec, size_t *chunk) {
  *rec = ctx->group == 0 ? sizeof(RecSu2) : sizeof(RecU1);
  const size_t stage_bytes = sizeof(double) * ctx->NL * (ctx->group == 0 ? 4 : 1);
  *chunk = stage_bytes / 2 / *rec;  // >= 2 for every valid lattice (even extents, d >= 2)
}

extern "C" int su2b_save_gauge(su2b_ctx *ctx, const char *path) {
  SU2B_CKS(io_enter(ctx));
  SU2B_NEED(path, "path is NULL");
  size_t rec, chunk;
  io_sizes(ctx, &rec, &chunk);
  if (chunk == 0) return su2b_fail(ctx, SU2B_ERR_INVALID, "lattice too small for the I/O chunks");
  File out;
  out.f = fopen(path, "wb");
  if (!out.f) return su2b_fail(ctx, SU2B_ERR_INVALID, "cannot open %s for writing", path);
  Pinned pin;
  for (int k = 0; k < 2; k++) {
    SU2B_CK(cudaMallocHost(&pin.p[k], chunk * rec));
    SU2B_CK(cudaEventCreateWithFlags(&pin.ev[k], cudaEventDisableTiming));
  }
  char *stage = (char *)ctx->stage;
  const size_t nchunks = (ctx->NL + chunk - 1) / chunk;
  for (size_t c = 0; c <= nchunks; c++) {
    if (c < nchunks) {
      const size_t l0 = c * chunk, n = std::min(chunk, ctx->NL - l0);
      void *dst = stage + (c & 1) * chunk * rec;
      if (ctx->link64)
        k_to_records<double><<<io_grid(n), NT_IO, 0, ctx->stream>>>(ctx->g, ctx->U, ctx->group,
                                                                     l0, n, dst);
      else
        k_to_records<float><<<io_grid(n), NT_IO, 0, ctx->stream>>>(ctx->g, ctx->U, ctx->group,
                                                                    l0, n, dst);
      SU2B_CK(cudaGetLastError());
      ctx->launches++;
      SU2B_CK(cudaMemcpyAsync(pin.p[c & 1], dst, n * rec, cudaMemcpyDeviceToHost, ctx->stream));
      SU2B_CK(cudaEventRecord(pin.ev[c & 1], ctx->stream));
    }
    if (c > 0) {  // write the previous chunk while this one is copied
      const size_t p = c - 1, n = std::min(chunk, ctx->NL - p * chunk);
      SU2B_CK(cudaEventSynchronize(pin.ev[p & 1]));
      if (fwrite(pin.p[p & 1], rec, n, out.f) != n)
        return su2b_fail(ctx, SU2B_ERR_INVALID, "short write to %s", path);
    }
  }
  if (fclose(out.f) != 0) {
    out.f = nullptr;
    return su2b_fail(ctx, SU2B_ERR_INVALID, "closing %s failed", path);
  }
  out.f = nullptr;
  return SU2B_OK;
}

extern "C" int su2b_load_gauge(su2b_ctx *ctx, const char *path) {
  SU2B_CKS(io_enter(ctx));
  SU2B_NEED(path, "path is NULL");
  size_t rec, chunk;
  io_sizes(ctx, &rec, &chunk);
  if (chunk == 0) return su2b_fail(ctx, SU2B_ERR_INVALID, "lattice too small for the I/O chunks");
  File in;
  in.f = fopen(path, "rb");
  if (!in.f) return su2b_fail(ctx, SU2B_ERR_INVALID, "cannot open %s", path);
  Pinned pin;
  for (int k = 0; k < 2; k++) {
    SU2B_CK(cudaMallocHost(&pin.p[k], chunk * rec));
    SU2B_CK(cudaEventCreateWithFlags(&pin.ev[k], cudaEventDisableTiming));
  }
  int *bad = (int *)ctx->part_slot(5);  // a scratch word for the record check
  SU2B_CK(cudaMemsetAsync(bad, 0, sizeof(int), ctx->stream));
  char *stage = (char *)ctx->stage;
  const size_t nchunks = (ctx->NL + chunk - 1) / chunk;
  for (size_t c = 0; c < nchunks; c++) {
    const size_t l0 = c * chunk, n = std::min(chunk, ctx->NL - l0);
    if (c >= 2) SU2B_CK(cudaEventSynchronize(pin.ev[c & 1]));  // its buffer was copied in
    if (fread(pin.p[c & 1], rec, n, in.f) != n)
      return su2b_fail(ctx, SU2B_ERR_INVALID, "%s holds fewer links than the lattice", path);
    void *dst = stage + (c & 1) * chunk * rec;
    SU2B_CK(cudaMemcpyAsync(dst, pin.p[c & 1], n * rec, cudaMemcpyHostToDevice, ctx->stream));
    SU2B_CK(cudaEventRecord(pin.ev[c & 1], ctx->stream));
    if (ctx->link64)
      k_from_records<double><<<io_grid(n), NT_IO, 0, ctx->stream>>>(ctx->g, ctx->U, ctx->group,
                                                                     l0, n, dst, bad);
    else
      k_from_records<float><<<io_grid(n), NT_IO, 0, ctx->stream>>>(ctx->g, ctx->U, ctx->group,
                                                                    l0, n, dst, bad);
    SU2B_CK(cudaGetLastError());
    ctx->launches++;
  }
  int hbad = 0;
  SU2B_CK(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  SU2B_CK(cudaStreamSynchronize(ctx->stream));
  ctx->phases_valid = false;
  if (hbad)
    return su2b_fail(ctx, SU2B_ERR_INVALID,
                     "%s: a record's N_c does not match the group (not a %s configuration)",
                     path, ctx->group == 0 ? "SU(2)" : "U(1)");
  return SU2B_OK;
}

// ---- the restart counter (io.hh:251-305) ----
static const char *const NCONF_COUNTER = "nconf_counter.txt";

extern "C" int su2b_update_nconf_counter(const char *conf_dir, int heat, long i,
                                         const char *path_conf) {
  if (!conf_dir || !path_conf || (heat != 0 && heat != 1) || i < 0) return SU2B_ERR_INVALID;
  const std::string name = std::string(conf_dir) + NCONF_COUNTER;
  File out;
  out.f = fopen(name.c_str(), "w");
  if (!out.f) return SU2B_ERR_INVALID;
  const int w = fprintf(out.f, "heat i path_conf\n%d %ld %s", heat, i, path_conf);
  const int c = fclose(out.f);
  out.f = nullptr;
  return (w < 0 || c != 0) ? SU2B_ERR_INVALID : SU2B_OK;
}

extern "C" int su2b_read_nconf_counter(const char *conf_dir, int *heat, long *i, char *path_buf,
                                       size_t path_cap) {
  if (!conf_dir || !heat || !i || !path_buf || path_cap == 0) return SU2B_ERR_INVALID;
  const std::string name = std::string(conf_dir) + NCONF_COUNTER;
  File in;
  in.f = fopen(name.c_str(), "r");
  if (!in.f) return SU2B_ERR_INVALID;
  // the second line, whole
  std::string line[2];
  for (int k = 0; k < 2; k++) {
    int ch;
    while ((ch = fgetc(in.f)) != EOF && ch != '\n') line[k].push_back((char)ch);
    if (ch == EOF && k == 0) return SU2B_ERR_INVALID;
  }
  // split at every space, as boost::split(v, line, is_any_of(" ")) does (empty tokens kept)
  std::vector<std::string> v(1);
  for (char ch : line[1]) {
    if (ch == ' ')
      v.emplace_back();
    else
      v.back().push_back(ch);
  }
  if (v.size() < 3) return SU2B_ERR_INVALID;
  if (v[0] != "0" && v[0] != "1") return SU2B_ERR_INVALID;  // lexical_cast<bool>
  char *end = nullptr;
  const long iv = strtol(v[1].c_str(), &end, 10);  // std::stoi: leading digits
  if (end == v[1].c_str()) return SU2B_ERR_INVALID;
  if (v[2].size() + 1 > path_cap) return SU2B_ERR_INVALID;
  *heat = v[0] == "1";
  *i = iv;
  memcpy(path_buf, v[2].c_str(), v[2].size() + 1);
  return SU2B_OK;
}

extern "C" int su2b_restart(su2b_ctx *ctx, const char *conf_dir, int *heat, long *i) {
  if (!ctx) return SU2B_ERR_INVALID;
  SU2B_NEED(conf_dir && heat && i, "NULL argument");
  std::vector<char> path(4096);
  if (su2b_read_nconf_counter(conf_dir, heat, i, path.data(), path.size()) != SU2B_OK)
    return su2b_fail(ctx, SU2B_ERR_INVALID, "cannot read %s%s", conf_dir, NCONF_COUNTER);
  return su2b_load_gauge(ctx, path.data());
}
