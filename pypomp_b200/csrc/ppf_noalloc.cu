// ppf_noalloc.cu -- ppf_pfilter for callers that cannot allocate device memory.
//
// Every other entry point takes its scratch memory from the caller
// (`workspace`).  Some callers have no way to provide it: a host runtime that
// owns the device's memory pool and forbids foreign allocations (pypomp's own
// JAX runtime preallocates most of the GPU for XLA by default), or plugin code
// that is not permitted to call the CUDA allocator at all.  For them this file
// keeps a fixed scratch area in the library itself, a file-scope __device__
// array of PPF_NOALLOC_SCRATCH_BYTES, and runs the ordinary batched filter on
// it.  Nothing here calls cudaMalloc, cudaFree or any allocating routine.
//
// Consequences a caller must know:
//  - every GPU that loads the library holds the array until the process exits;
//  - all calls on a device share the one array: calls whose work overlaps on
//    the GPU (different streams, or different host threads) race and corrupt
//    each other -- serialise them;
//  - the array keeps the previous call's contents; ppf_pfilter clears the part
//    that must start at zero (counters, accumulators, tile totals)
//    and fully writes the particle arrays before reading them;
//  - the first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (the host-side name is only a stand-in, not a device
//    pointer);
//  - the call is synchronous: it waits for the stream, then reads the status
//    word the kernels leave at the start of the scratch area, so a bounded
//    device-side wait that gave up is reported as PPF_ETIMEOUT.  A stream
//    wait cannot be recorded into a CUDA graph, so the call refuses to run
//    (PPF_EUNSUPPORTED, before any work) while its stream is capturing;
//  - PPF_F_GRAPH is ignored: replaying a cached graph would need a private
//    stream and graph objects, which the driver allocates, so the launches
//    always go directly onto the caller's stream.
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>
#include <string.h>

#include "ppf.h"

namespace {

constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[PPF_NOALLOC_SCRATCH_BYTES];

void* g_scratch_addr[kMaxDevices] = {nullptr};

// Device address of the scratch array on the current device (looked up once).
int scratch_address(void** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return PPF_ECUDA;
  if (dev < 0 || dev >= kMaxDevices) return PPF_EUNSUPPORTED;
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return PPF_ECUDA;
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return PPF_OK;
}

}  // namespace

extern "C" {

int ppf_pfilter_noalloc(const ppf_pfilter_desc* d, void* stream) {
  if (!d) return PPF_EINVAL;
  const size_t need = ppf_pfilter_workspace_bytes(d);
  if (need == 0) return PPF_EINVAL;
  if (need > PPF_NOALLOC_SCRATCH_BYTES) return PPF_ESCRATCH;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cap) != cudaSuccess) return PPF_ECUDA;
  if (cap != cudaStreamCaptureStatusNone) return PPF_EUNSUPPORTED;
  void* scratch = nullptr;
  const int rc = scratch_address(&scratch);
  if (rc != PPF_OK) return rc;
  ppf_pfilter_desc local;
  memcpy(&local, d, sizeof(local));
  local.workspace = scratch;
  local.ws_bytes = PPF_NOALLOC_SCRATCH_BYTES;
  local.flags &= ~PPF_F_GRAPH;   // direct launches only: no driver-side graph objects
  const int run = ppf_pfilter(&local, stream);
  if (run != PPF_OK) return run;
  uint32_t status = 0;   // first word of the scratch: device-side error bits
  if (cudaMemcpyAsync(&status, scratch, sizeof(status), cudaMemcpyDeviceToHost, s) != cudaSuccess)
    return PPF_ECUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return PPF_ECUDA;
  if (status & 1u) return PPF_ETIMEOUT;
  if (status) return PPF_EINTERNAL;
  return PPF_OK;
}

}  // extern "C"
