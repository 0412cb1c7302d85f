// swc_solve_noalloc: the supernodal solve of swc_solve for callers that must not allocate
// device memory at solve time.
//
// Some callers cannot call cudaMalloc when they need a solve: applications that hand all
// device memory to their own pool or arena and forbid further CUDA allocations, plug-in
// hosts that only allow allocation during initialisation, and latency-critical loops where
// the implicit device-wide synchronisation of cudaMalloc/cudaFree is not acceptable.
// swc_solve allocates its workspace on first use; this entry point instead uses one
// fixed scratch array in device memory that is part of the library image, so the call
// itself allocates nothing.  The handle (created, analysed and factored earlier) keeps the
// factor and the solve plan; the caller passes the right-hand sides and the output.
//
// The scratch holds one double per off-diagonal row of L per right-hand side (the
// contributions the forward solve passes from each supernode to its ancestors).  Every
// entry is written before it is read within one call, so nothing has to be cleared
// between calls.  All calls on a GPU share the one array: calls that overlap on the GPU
// (from several host threads or streams) race on it and must be serialised by the caller.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/swcholesky_b200.h"
#include "swc_handle.h"

namespace {

// Fixed scratch: 2^20 doubles = 8 MiB, held by every GPU that loads the library until exit.
static __device__ __align__(256) double g_solve_scratch[SWC_SOLVE_NOALLOC_MAX];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double *g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch on the current device.  The host-side symbol is only a
// stand-in, so the address is looked up once per device (on the first call made with
// that device current) and cached.
bool scratch_address(int dev, double **out) {
  std::lock_guard<std::mutex> lock(g_mu);
  if (dev < 0 || dev >= kMaxDevices) {
    swc::set_last_error("device index out of range");
    return false;
  }
  if (!g_scratch_ptr[dev]) {
    double *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void **)&p, g_solve_scratch);
    if (e != cudaSuccess || !p) {
      swc::set_last_error(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      return false;
    }
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return true;
}

}  // namespace

extern "C" int swc_solve_noalloc(swc_handle_t h, const double *b, double *x, int nrhs) {
  if (!h) return swc::set_last_error("null handle"), SWC_INVALID_INPUT;
  if (!h->factored) return swc::set_last_error("solve before a successful factor"), SWC_NOT_READY;
  if (!b || !x || nrhs <= 0) return swc::set_last_error("bad solve arguments"), SWC_INVALID_INPUT;
  const cudaError_t e = cudaSetDevice(h->device);
  if (e != cudaSuccess)
    return swc::set_last_error(std::string("cudaSetDevice: ") + cudaGetErrorString(e)), SWC_CUDA_ERROR;
  double *scratch = nullptr;
  if (!scratch_address(h->device, &scratch)) return SWC_CUDA_ERROR;
  std::string err;
  if (!h->eng->solve_in_scratch(b, x, nrhs, scratch, SWC_SOLVE_NOALLOC_MAX, err)) {
    swc::set_last_error(err);
    if (err.rfind("solve needs", 0) == 0) return SWC_INVALID_INPUT;
    return err.rfind("timeout:", 0) == 0 ? SWC_TIMEOUT : SWC_CUDA_ERROR;
  }
  return SWC_OK;
}
