// Scattered far field of device-resident currents without any device allocation.
//
// sie_farfield (the host-buffer entry point) allocates its device buffers per call
// and gathers the currents into the context's work vector.  Some callers can do
// neither: a host code that hands the whole HBM to its own pool allocator up front
// (cudaMalloc then fails or evicts that pool), and a pipeline that keeps several
// streams busy, where the implicit device-wide synchronisation of cudaFree would
// stall every other stream.  This entry point writes only into the caller's output
// buffers and into one fixed scratch array compiled into the library.
#include <mutex>

#include "sie_internal.h"

namespace sie {
__global__ void k_gather(const zc* ext, zc* in, const int* perm, int M, int nrhs);
__global__ void k_field(const FnD* fn, const zc* x, int M, Material mt, const double* pts,
                        int npts, zc* Eo, zc* Ho, double* Io);
}  // namespace sie

using namespace sie;

// Internal-layout copy of the currents: (J, M) interleaved per edge in leaf-box order,
// 2 * SIE_NOALLOC_MAX_EDGES complex values = 4 MiB.  Every element the field kernel
// reads is written by the gather of the same call first, so nothing here has to
// start at zero.  One array per device for the whole process.
static __device__ __align__(256) zc g_noalloc_x[2 * SIE_NOALLOC_MAX_EDGES];

namespace {
const int kMaxDevices = 64;
// Device address of g_noalloc_x per device ordinal, looked up by the first call on that
// device that succeeds; a failed lookup is not kept, so the next call tries again.  The
// address belongs to the module loaded in the device's primary context: after a
// cudaDeviceReset it is stale, and this entry point must not be called again in the
// process.
std::mutex g_sym_mu;
zc* g_sym_ptr[kMaxDevices];

// Restores the caller's current device when the call returns.
struct DeviceGuard {
  int prev = -1;
  DeviceGuard() {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};
}  // namespace

extern "C" int sie_farfield_device_noalloc(sie_ctx* c, const double* d_x, const double* d_pts,
                                           int npts, double* d_E, double* d_H, double* d_I,
                                           void* stream) {
  if (!c || !d_x || !d_pts || !d_E || !d_H || !d_I || npts < 1)
    return fail(SIE_ERR_ARG, "sie_farfield_device_noalloc: bad argument");
  if (c->M > SIE_NOALLOC_MAX_EDGES)
    return fail(SIE_ERR_ARG, "sie_farfield_device_noalloc: mesh has more than "
                             "SIE_NOALLOC_MAX_EDGES edges");
  if (!c->setup_done) return fail(SIE_ERR_STATE, "sie_farfield_device_noalloc: sie_setup not called");
  if (c->device < 0 || c->device >= kMaxDevices)
    return fail(SIE_ERR_ARG, "sie_farfield_device_noalloc: device ordinal out of range");
  DeviceGuard keep_device;
  SIE_CUDA(cudaSetDevice(c->device));
  zc* xi = nullptr;
  {
    // the scratch address is looked up once per device, with that device current
    std::lock_guard<std::mutex> lk(g_sym_mu);
    if (!g_sym_ptr[c->device]) {
      void* p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_x);
      if (e != cudaSuccess) return cuda_fail(e, "sie_farfield_device_noalloc: cudaGetSymbolAddress");
      g_sym_ptr[c->device] = (zc*)p;
    }
    xi = g_sym_ptr[c->device];
  }
  cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
  int M = c->M;
  k_gather<<<(M + 255) / 256, 256, 0, st>>>((const zc*)d_x, xi, c->d_perm, M, 1);
  count_launch();
  SIE_CUDA(cudaGetLastError());
  k_field<<<npts, 256, 0, st>>>(c->d_fn, xi, M, c->mt, d_pts, npts, (zc*)d_E, (zc*)d_H, d_I);
  count_launch();
  SIE_CUDA(cudaGetLastError());
  return SIE_OK;
}
