// Bulk-flux reduction that allocates no device memory.
//
// Same quantity as c3d_compute_mean_mass_flow_u with Hu = 1
// (compute_mean_mass_flow_U, src/mass_flow.f90:24-53), for callers that
// cannot call cudaMalloc: for example a driver that runs the flux check
// inside its own time loop, where cudaMalloc's implicit device
// synchronisation would stall the stream, or a host program whose device
// memory is owned by a fixed pool of another runtime.  The caller passes
// device pointers to the field, to the y grid and to the one-double result.
//
// Scratch: one (sum, norm) pair per z plane in a file-scope __device__ array
// of kNoAllocMaxPlanes entries (64 KiB).  It is reserved on every GPU that
// loads the library until the process exits.  Host code cannot use the
// array's name as a device address; the first call on each device resolves
// the address with cudaGetSymbolAddress while that device is current (so
// that first call must come before any stream capture).  The address is kept
// for the life of the process, so the entry must not be used across a
// cudaDeviceReset of that device (the array then has a new address that the
// cached one does not follow).  All calls share the
// array: calls whose kernels overlap on a GPU race on it, so issue them on
// one stream or serialise them.  Each call writes every partial it later
// reads, so nothing needs clearing between calls.
#include <map>
#include <mutex>
#include <string>

#include "c3d_internal.cuh"

namespace c3d {

static constexpr int kNoAllocMaxPlanes = 4096;
static __device__ __align__(256) double2 g_flux_partials[kNoAllocMaxPlanes];

static std::mutex g_na_mu;
static std::map<int, double2*> g_na_ptr;   // device ordinal -> address of g_flux_partials

// one block per z plane k = 2..nzg-1: partial of sum_j sum_i (U(j)+U(j-1)) w(j)
// and of its norm sum_j sum_i 2 w(j), w(j) = 0.5*(yg(j)-yg(j-1)), j = 3..nyg-1
__global__ void __launch_bounds__(256) k_flux_plane_noalloc(const double* __restrict__ U, int nx,
                                                            int nyg, const double* __restrict__ yg,
                                                            double2* __restrict__ part) {
  const int k = 2 + blockIdx.x;
  const int ni = nx - 2, nj = nyg - 3;
  double s = 0.0, n = 0.0;
  for (int t = threadIdx.x; t < ni * nj; t += blockDim.x) {
    const int i = 2 + t % ni;
    const int j = 3 + t / ni;
    const double w = 0.5 * (yg[j - 1] - yg[j - 2]);   // yg is 0-based here: yg[j-1] = yg(j)
    const int64_t a = (int64_t)(i - 1) + (int64_t)nx * ((j - 1) + (int64_t)nyg * (k - 1));
    const int64_t b = a - nx;
    s += (U[a] + U[b]) * w;
    n += 2.0 * w;
  }
  __shared__ double ss[256], sn[256];
  ss[threadIdx.x] = s;
  sn[threadIdx.x] = n;
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) {
      ss[threadIdx.x] += ss[threadIdx.x + st];
      sn[threadIdx.x] += sn[threadIdx.x + st];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = make_double2(ss[0], sn[0]);
}

__global__ void k_flux_final_noalloc(const double2* __restrict__ part, int np, double* q) {
  __shared__ double ss[256], sn[256];
  double s = 0.0, n = 0.0;
  for (int t = threadIdx.x; t < np; t += blockDim.x) {
    s += part[t].x;
    n += part[t].y;
  }
  ss[threadIdx.x] = s;
  sn[threadIdx.x] = n;
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) {
      ss[threadIdx.x] += ss[threadIdx.x + st];
      sn[threadIdx.x] += sn[threadIdx.x + st];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) *q = ss[0] / sn[0];
}

static int resolve_scratch(double2** out, std::string& err) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) { err = std::string("cudaGetDevice: ") + cudaGetErrorString(e); return C3D_ERR_CUDA; }
  std::lock_guard<std::mutex> lk(g_na_mu);
  auto it = g_na_ptr.find(dev);
  if (it != g_na_ptr.end()) { *out = it->second; return 0; }
  double2* p = nullptr;
  e = cudaGetSymbolAddress((void**)&p, g_flux_partials);
  if (e != cudaSuccess || p == nullptr) {
    err = std::string("cudaGetSymbolAddress(g_flux_partials): ") + cudaGetErrorString(e);
    return C3D_ERR_CUDA;
  }
  g_na_ptr[dev] = p;
  *out = p;
  return 0;
}

}  // namespace c3d

extern "C" int c3d_mean_mass_flow_u_noalloc(const double* U, int nx, int nyg, int nzg,
                                            const double* yg, double* qflow, void* stream) {
  using namespace c3d;
  if (!U || !yg || !qflow) {
    set_global_error("c3d_mean_mass_flow_u_noalloc: null pointer argument");
    return C3D_ERR_PARAM;
  }
  if (nx < 3 || nyg < 4 || nzg < 3) {
    set_global_error("c3d_mean_mass_flow_u_noalloc: need nx >= 3, nyg >= 4, nzg >= 3");
    return C3D_ERR_PARAM;
  }
  const int nplanes = nzg - 2;   // k = 2..nzg-1
  if (nplanes > kNoAllocMaxPlanes) {
    set_global_error("c3d_mean_mass_flow_u_noalloc: nzg-2 = " + std::to_string(nplanes) +
                     " z planes exceed the static scratch of " +
                     std::to_string(kNoAllocMaxPlanes) + " planes");
    return C3D_ERR_PARAM;
  }
  // an error left pending by the caller's own earlier work is reported as
  // such and left in place (peek, not get), so it is not mistaken for a
  // failure of this call's launches
  cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess) {
    set_global_error(std::string("c3d_mean_mass_flow_u_noalloc: CUDA error pending before the call: ") +
                     cudaGetErrorString(e));
    return C3D_ERR_CUDA;
  }
  double2* part = nullptr;
  std::string err;
  int rc = resolve_scratch(&part, err);
  if (rc) { set_global_error(err); return rc; }
  cudaStream_t s = (cudaStream_t)stream;
  k_flux_plane_noalloc<<<nplanes, 256, 0, s>>>(U, nx, nyg, yg, part);
  k_flux_final_noalloc<<<1, 256, 0, s>>>(part, nplanes, qflow);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_global_error(std::string("c3d_mean_mass_flow_u_noalloc launch: ") + cudaGetErrorString(e));
    return C3D_ERR_CUDA;
  }
  return 0;
}
