// Allocation-free variant of the copy engine's converting upload (host values of one type -> device array
// of another type).
//
// The runner's upload path stages host bytes in a scratch buffer that it grows with cudaMalloc on demand.
// Some callers cannot allow that: a host application that owns the whole device-memory budget (its own pool,
// a hard memory cap) and forbids allocations after start-up, or a time-stepping loop that cannot absorb the
// latency and device-wide synchronisation a cudaMalloc may bring.  This entry point stages through a fixed
// array that lives in the library's own device image instead, so it allocates nothing.
//
// Scratch: kNoAllocScratchBytes (8 MiB) in a file-scope __device__ array.  Every GPU that loads the library
// holds it until the process exits.  All calls share it and it keeps the last call's contents; each call
// overwrites exactly the bytes it uses before reading them, so nothing needs to start at zero.  Calls that
// overlap on the GPU (two streams, or two host threads) race on the shared array: serialise them.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "dgk.h"
#include "runner.hpp"

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(8) << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void *g_scratch_addr[kMaxDevices];  // device address of g_noalloc_scratch, resolved once per device

// Device address of the scratch array on the current device.  The host-side symbol g_noalloc_scratch is only
// a stand-in: handing it to a kernel would fault (or silently touch host memory on systems where the GPU can
// reach it), so the real address comes from cudaGetSymbolAddress, once per device, with that device current.
void *scratch_address() {
  int dev = 0;
  dgk::cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) throw dgk::Error(DGK_ERR_UNSUPPORTED, "device index beyond the scratch table");
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_addr[dev]) {
    void *p = nullptr;
    dgk::cuda_check(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress(scratch)");
    g_scratch_addr[dev] = p;
  }
  return g_scratch_addr[dev];
}

}  // namespace

extern "C" int dgk_convert_upload_noalloc(const void *host, int32_t host_dtype, void *device_dst, int32_t dev_dtype,
                                          int64_t count, void *cuda_stream) {
  try {
    if (count < 0 || (count > 0 && (!host || !device_dst)))
      throw dgk::Error(DGK_ERR_INVALID, "null buffer or negative count");
    const size_t esize = (size_t)dgk::dtype_size(host_dtype);
    dgk::dtype_size(dev_dtype);
    // compare counts, not byte products: count * esize could wrap around for a huge count
    if ((uint64_t)count > kNoAllocScratchBytes / esize)
      throw dgk::Error(DGK_ERR_INVALID, "dgk_convert_upload_noalloc: " + std::to_string(count) +
                                            " host values exceed the fixed 8 MiB staging area; split the "
                                            "upload into calls of at most 8 MiB of host data");
    const size_t bytes = (size_t)count * esize;
    if (count == 0) return DGK_OK;
    void *scratch = scratch_address();  // first call on a device resolves the address (do it before a capture)
    cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
    dgk::cuda_check(cudaMemcpyAsync(scratch, host, bytes, cudaMemcpyHostToDevice, st), "H2D into scratch");
    dgk::launch_convert(scratch, host_dtype, device_dst, dev_dtype, count, st);
    dgk::cuda_check(cudaGetLastError(), "convert kernel");
    dgk::cuda_check(cudaStreamSynchronize(st), "sync");  // the host buffer may be reused when this returns
    return DGK_OK;
  } catch (const dgk::Error &e) {
    dgk::set_global_error(e.what());  // readable through dgk_global_error()
    return e.code;
  } catch (const std::exception &e) {
    dgk::set_global_error(e.what());
    return DGK_ERR_INVALID;
  }
}
