// noalloc.cu -- plaquette sums without any device allocation.
//
// Some callers cannot allocate device memory: host frameworks that own every byte of the GPU
// through their own pool and forbid cudaMalloc inside plug-ins, or code running while a CUDA
// graph is being captured, where an allocation would break the capture.  For them,
// su2b_gauge_energy_noalloc computes gauge_energy(U) and gauge_energy(U, spatial_only) from a
// gauge field the caller already holds on the device, in the reference's host layout, and
// writes the two sums to a device buffer the caller provides.  It creates no context.
//
// Its only scratch is the file-scope array below (one partial sum pair per block).  The array
// lives in every GPU that loads this library until the process exits; its size bounds the
// lattice: at most NOALLOC_MAX_BLOCKS blocks of NOALLOC_NT sites, i.e. 4,194,304 sites.
// Every call overwrites the partials it reads, so nothing has to start at zero; but all calls
// share the one array, so calls that overlap on the GPU (different streams, or host threads
// without ordering) race on it and must be serialised by the caller.
//
// Host code cannot use the array's name as a device address (in host code it names a host
// shadow object).  The device address is looked up with cudaGetSymbolAddress, with the
// device current, on every call made outside a stream capture, and remembered per device;
// a call made while its stream is being captured uses the remembered address.  So the first
// call on a device should happen before any stream capture begins, and a capture uses the
// address of the context that was current at the last call outside a capture.
#include <mutex>

#include "su2b.h"
#include "su2b_common.cuh"

namespace {

constexpr int NOALLOC_NT = 256;
constexpr int NOALLOC_MAX_BLOCKS = 16384;
constexpr int NOALLOC_MAX_DEVICES = 64;

static __device__ __align__(256) double g_noalloc_partials[2 * NOALLOC_MAX_BLOCKS];

std::mutex g_mutex;
double *g_scratch[NOALLOC_MAX_DEVICES] = {};

using su2b::Geom;
using su2b::Site;

// one thread per site in the reference order; planes mu < nu as
// flat-gauge_energy.hpp:109-137, partials {all planes, planes with mu >= 1}
template <int GROUP, int ND>
__global__ void __launch_bounds__(NOALLOC_NT)
  k_plaq_reference_layout(Geom g, const double *__restrict__ U, double *part) {
  __shared__ double sh[NOALLOC_NT / 32];
  const int lex = blockIdx.x * NOALLOC_NT + threadIdx.x;
  double full = 0., spat = 0.;
  if (lex < g.V) {
    const Site s = su2b::site_from_lex(g, lex);
#pragma unroll
    for (int mu = 0; mu < ND - 1; mu++) {
      const long lpm = lex + su2b::fwd(g, s, mu);
#pragma unroll
      for (int nu = mu + 1; nu < ND; nu++) {
        const long lpn = lex + su2b::fwd(g, s, nu);
        double tr;
        if (GROUP == 0) {
          const double *a = U + 4 * ((long)lex * ND + mu), *b = U + 4 * (lpm * ND + nu),
                       *c = U + 4 * (lpn * ND + mu), *d = U + 4 * ((long)lex * ND + nu);
          const su2b::Su2<double> A{a[0], a[1], a[2], a[3]}, B{b[0], b[1], b[2], b[3]},
            Cc{c[0], c[1], c[2], c[3]}, D{d[0], d[1], d[2], d[3]};
          tr = su2b::retr_mul(su2b::mul(A, B), su2b::dag(su2b::mul(D, Cc)));
        } else {
          tr = cos(((U[(long)lex * ND + mu] + U[lpm * ND + nu]) + (-U[lpn * ND + mu])) +
                   (-U[(long)lex * ND + nu]));
        }
        full += tr;
        if (mu >= 1) spat += tr;
      }
    }
  }
  double r = su2b::block_sum<NOALLOC_NT>(full, sh);
  if (threadIdx.x == 0) part[2 * blockIdx.x] = r;
  r = su2b::block_sum<NOALLOC_NT>(spat, sh);
  if (threadIdx.x == 0) part[2 * blockIdx.x + 1] = r;
}

__global__ void __launch_bounds__(512) k_noalloc_final(const double *part, int n, double *out) {
  __shared__ double sh[512 / 32];
  for (int k = 0; k < 2; k++) {
    double v = 0.;
    for (int b = threadIdx.x; b < n; b += 512) v += part[2 * b + k];
    const double r = su2b::block_sum<512>(v, sh);
    if (threadIdx.x == 0) out[k] = r;
  }
}

// device address of the scratch array in the current context.  Outside a stream capture it
// is looked up afresh (a host-side lookup that allocates nothing), so a context recreated
// after cudaDeviceReset, or another context made current, gets its own address; during a
// capture the address remembered for the device is used.
int scratch_address(cudaStream_t s, double **ptr) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return SU2B_ERR_CUDA;
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return SU2B_ERR_UNSUPPORTED;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  const bool capturing =
    cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone;
  if (capturing) cudaGetLastError();  // a refused query leaves no sticky error behind
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!capturing || !g_scratch[dev]) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_partials) != cudaSuccess || !p)
      return SU2B_ERR_CUDA;
    g_scratch[dev] = (double *)p;
  }
  *ptr = g_scratch[dev];
  return SU2B_OK;
}

}  // namespace

extern "C" int su2b_gauge_energy_noalloc(int group, int Lx, int Ly, int Lz, int Lt, int ndims,
                                         const double *U_dev, double *out_dev, void *stream) {
  if (!U_dev || !out_dev) return SU2B_ERR_INVALID;
  if (group != SU2B_GROUP_SU2 && group != SU2B_GROUP_U1) return SU2B_ERR_INVALID;
  if (ndims < 2 || ndims > 4) return SU2B_ERR_INVALID;
  const int L[4] = {Lt, Lx, Ly, Lz};
  // the volume is formed one extent at a time and checked against the scratch array's
  // limit at each step, so no product of extents can wrap before the check
  constexpr long max_sites = (long)NOALLOC_MAX_BLOCKS * NOALLOC_NT;
  long V = 1;
  for (int k = 0; k < 4; k++) {
    if (L[k] < 1 || L[k] > max_sites) return SU2B_ERR_INVALID;
    if (k >= ndims && L[k] != 1) return SU2B_ERR_INVALID;
    V *= L[k];
    if (V > max_sites) return SU2B_ERR_INVALID;  // beyond the scratch array
  }
  const long nblocks = (V + NOALLOC_NT - 1) / NOALLOC_NT;
  Geom g{};
  g.nd = ndims;
  for (int k = 0; k < 4; k++) g.L[k] = L[k];
  g.st[3] = 1;
  for (int k = 2; k >= 0; k--) g.st[k] = g.st[k + 1] * L[k + 1];
  g.V = (int)V;
  g.Vh = (int)(V / 2);
  for (int k = 0; k < 4; k++) g.dv[k] = su2b::make_fastdiv((uint32_t)L[k]);
  cudaStream_t s = (cudaStream_t)stream;
  double *part = nullptr;
  const int rc = scratch_address(s, &part);
  if (rc != SU2B_OK) return rc;
  const int grid = (int)nblocks;
  switch (group * 8 + ndims) {
    case 2: k_plaq_reference_layout<0, 2><<<grid, NOALLOC_NT, 0, s>>>(g, U_dev, part); break;
    case 3: k_plaq_reference_layout<0, 3><<<grid, NOALLOC_NT, 0, s>>>(g, U_dev, part); break;
    case 4: k_plaq_reference_layout<0, 4><<<grid, NOALLOC_NT, 0, s>>>(g, U_dev, part); break;
    case 10: k_plaq_reference_layout<1, 2><<<grid, NOALLOC_NT, 0, s>>>(g, U_dev, part); break;
    case 11: k_plaq_reference_layout<1, 3><<<grid, NOALLOC_NT, 0, s>>>(g, U_dev, part); break;
    default: k_plaq_reference_layout<1, 4><<<grid, NOALLOC_NT, 0, s>>>(g, U_dev, part); break;
  }
  if (cudaGetLastError() != cudaSuccess) return SU2B_ERR_CUDA;
  k_noalloc_final<<<1, 512, 0, s>>>(part, grid, out_dev);
  if (cudaGetLastError() != cudaSuccess) return SU2B_ERR_CUDA;
  return SU2B_OK;
}
