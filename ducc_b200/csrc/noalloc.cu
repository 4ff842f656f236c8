// Type-1 NUFFT entry point that allocates nothing.
//
// Some callers cannot allocate device memory while they run a transform:
// callbacks and plugins that run inside another framework which owns the
// whole device memory pool, and services that reserve a fixed memory budget
// up front and forbid allocation afterwards (cudaMalloc may also synchronise
// the device and stall other streams).  For them dnufft_nu2u_noalloc takes
// every temporary of the transform from one fixed area compiled into this
// library: a file-scope device array of NOALLOC_SCRATCH_BYTES bytes, which
// every GPU that loads the library holds until the process exits.
//
// The call waits on its stream once, part-way through, to read the number of
// point chunks back to the host (a 4-byte copy into a host variable), and it
// uploads the correction factors from host vectors; the host thread therefore
// returns only after the sort has run on the GPU.
#include <cuda_runtime.h>

#include <cuda_runtime.h>

#include <mutex>

#include "../../include/ducc_b200.h"
#include "dnufft_internal.h"

namespace dnufft {
int nu2u_in_scratch(const dnufft_array *points, const dnufft_array *coord, int forward,
                    double epsilon, dnufft_array *out, const dnufft_opts *opts, void *stream,
                    void *scratch, size_t scratch_bytes);
void set_last_error(const char *msg);
}  // namespace dnufft

namespace {

constexpr size_t NOALLOC_SCRATCH_BYTES = size_t(32) << 20;   // 32 MiB

// The scratch area.  Host code may not use this name as an address (on the
// host it denotes a stand-in, not device memory): its device address comes
// from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
void *g_scratch_ptr[MAX_DEVICES] = {nullptr};

// Device address of the scratch area on the current device, looked up once
// per device (with that device current) on its first call and kept for the
// life of the process: after cudaDeviceReset (or a reset of the primary
// context) the kept address is stale, so a process that resets a device must
// not call this entry point on it again.
int scratch_address(void **ptr) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    dnufft::set_last_error(cudaGetErrorString(e));
    return DNUFFT_ERR_CUDA;
  }
  if (dev < 0 || dev >= MAX_DEVICES) {
    dnufft::set_last_error("device index out of range");
    return DNUFFT_ERR_INTERNAL;
  }
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_ptr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      dnufft::set_last_error(cudaGetErrorString(e));
      return DNUFFT_ERR_CUDA;
    }
    g_scratch_ptr[dev] = p;
  }
  *ptr = g_scratch_ptr[dev];
  return DNUFFT_OK;
}

}  // namespace

extern "C" int dnufft_nu2u_noalloc(const dnufft_array *points, const dnufft_array *coord,
                                   int forward, double epsilon, dnufft_array *out,
                                   const dnufft_opts *opts, void *stream) {
  void *scratch = nullptr;
  int st = scratch_address(&scratch);
  if (st != DNUFFT_OK) return st;
  return dnufft::nu2u_in_scratch(points, coord, forward, epsilon, out, opts, stream, scratch,
                                 NOALLOC_SCRATCH_BYTES);
}

extern "C" size_t dnufft_noalloc_scratch_bytes(void) { return NOALLOC_SCRATCH_BYTES; }
