// sbdgpu_sigma_device_noalloc: the FP64 sigma build for callers that must not
// allocate device memory during the call.
//
// Such callers include code that runs between the set-up of a long job and its
// teardown under a strict memory budget (a pool or a pre-reserved arena owns
// all device memory, so a stray cudaMalloc would fail or fragment it), and
// code paths that must not synchronise the device, which cudaMalloc/cudaFree
// can do.  The regular sigma entry points allocate their transposed-vector
// scratch lazily on first use; this variant takes its scratch from one
// file-scope device array instead.
//
// Limits and behaviour:
//  - The array holds 3 x 524,288 doubles (12 MiB).  Every GPU on which a
//    context is created holds it until the process exits.  A basis of more
//    than 524,288 determinants (na * nb) is rejected with SBDGPU_ERR_LIMIT
//    before any launch.
//  - Creating a context (sbdgpu_create) prepares its device once: with that
//    device current it resolves the array's device address
//    (cudaGetSymbolAddress) and loads every kernel of the FP64 sigma build.
//    Under CUDA's lazy module loading the array's module, and each kernel's,
//    would otherwise be loaded (and device memory allocated for them) inside
//    the first call that touches them.  So the no-allocation call itself loads
//    nothing.
//  - The context's own set-up allocations must be done beforehand: call
//    sbdgpu_build_tables and sbdgpu_diag (or any sigma entry point) once.
//    Otherwise the call returns SBDGPU_ERR_STATE.
//  - All calls in the process share the array, and it keeps the previous
//    call's contents.  Every element the build reads from it is written by the
//    same call first, so nothing needs clearing; but two calls that overlap on
//    the GPU (different contexts on different host threads or streams) race
//    on it and corrupt each other's results.
#include <mutex>
#include <string>

#include "internal.cuh"

namespace {

constexpr size_t kNoAllocMaxDets = size_t(1) << 19;  // 524,288 determinants
constexpr int kMaxDevices = 64;

// staged input, transposed vector, transposed beta-part of sigma
static __device__ __align__(256) double g_sigma_scratch[3 * kNoAllocMaxDets];

std::mutex g_scratch_mu;
double* g_scratch_addr[kMaxDevices] = {};

// Device address of g_sigma_scratch on `device`, resolved by noalloc_prepare
// (the host-side name is only a stand-in and must never reach a kernel).
double* scratch_address(int device) {
  if (device < 0 || device >= kMaxDevices)
    throw sbdgpu::Error{SBDGPU_ERR_ARG, "device index out of range for the no-allocation scratch"};
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_addr[device])
    throw sbdgpu::Error{SBDGPU_ERR_STATE, "no-allocation scratch not prepared on this device (no context created)"};
  return g_scratch_addr[device];
}

}  // namespace

namespace sbdgpu {

// Once per device, with that device current: the array's device address, and
// every module the FP64 sigma build launches from, loaded now.
void noalloc_prepare(int device) {
  if (device < 0 || device >= kMaxDevices) return;  // the entry point then reports it
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (g_scratch_addr[device]) return;
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_sigma_scratch);
  if (e != cudaSuccess || !p)
    throw Error{SBDGPU_ERR_CUDA, std::string("cudaGetSymbolAddress(g_sigma_scratch): ") + cudaGetErrorString(e)};
  preload_fp64_sigma(device);
  g_scratch_addr[device] = static_cast<double*>(p);
}

}  // namespace sbdgpu

extern "C" int sbdgpu_sigma_device_noalloc(sbdgpu_ctx* c, const double* dC, double* dS) {
  if (!c) return SBDGPU_ERR_ARG;
  try {
    if (!dC || !dS) throw sbdgpu::Error{SBDGPU_ERR_ARG, "null vector"};
    if (!c->tables_ready || !c->hii_ready || !c->ja || !c->jb)
      throw sbdgpu::Error{SBDGPU_ERR_STATE,
                          "no-allocation sigma needs the set-up first: call sbdgpu_build_tables and sbdgpu_diag "
                          "(or one sigma) on this context"};
    if (c->N > kNoAllocMaxDets)
      throw sbdgpu::Error{SBDGPU_ERR_LIMIT, "no-allocation sigma supports at most 524288 determinants (na*nb = " +
                                                std::to_string(c->N) + ")"};
    SBD_CUDA(cudaSetDevice(c->device));
    double* base = scratch_address(c->device);
    double* io = base;
    double* ct = base + kNoAllocMaxDets;
    double* st = base + 2 * kNoAllocMaxDets;
    SBD_CUDA(cudaMemcpyAsync(io, dC, sizeof(double) * c->N, cudaMemcpyDeviceToDevice, c->stream));
    sbdgpu::apply_phase(c, io);
    sbdgpu::sigma_fp64_prepared(c, io, dS, ct, st);
    sbdgpu::apply_phase(c, dS);
    SBD_CUDA(cudaStreamSynchronize(c->stream));
    c->err.clear();
    return SBDGPU_OK;
  } catch (const sbdgpu::Error& e) {
    c->err = e.msg;
    return e.code;
  }
}
