// relax_noalloc.cu -- gfd_operator_relax_noalloc: relaxation sweeps that
// allocate no device memory.
//
// gfd_operator_relax needs one grid of device scratch (the second buffer of
// the Jacobi ping-pong, or the sweep-start copy that periodic Gauss-Seidel
// reads wrapped neighbours from) and allocates it with cudaMalloc on first
// use.  Some callers cannot allow that: code running while a CUDA graph is
// being captured, where an allocation would break or end the capture; hosts
// that hand the whole device memory to their own pool allocator and forbid
// other allocations; and real-time loops where an allocation's implicit
// device synchronisation is not acceptable.  This entry point uses a
// fixed scratch array compiled into the library instead.
//
// The scratch is a file-scope __device__ array of kNoAllocScratchBytes
// (16 MiB: up to 2,097,152 float64 points, a 128^3 grid, or 4,194,304
// float32 points).  Every GPU on which the library is loaded holds it until
// the process exits.  Host code must not pass the array's name to a kernel
// (on the host it names a stand-in, not device memory); the device address
// is looked up with cudaGetSymbolAddress, with the device current, on the
// first call in each CUDA context of a device, and cached.  A context that
// is destroyed and created again (cudaDeviceReset) gets a new lookup, since
// the module, and with it the array, may then sit at another address.
#include <mutex>
#include <string>

#include "common.cuh"
#include "internal.h"

namespace gfd {

constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;

static __device__ __align__(256) unsigned char g_relax_scratch[kNoAllocScratchBytes];

// Per device: the context the address was looked up in and the address.
struct ScratchAddr {
  void* ctx = nullptr;
  void* addr = nullptr;
};
static ScratchAddr g_scratch_addr[64];
static std::mutex g_scratch_mutex;

// The current context (CUcontext, as void*) through the driver entry point,
// so the library needs no link-time dependency on libcuda.
typedef int (*CtxGetCurrentFn)(void**);
static int current_context(void** ctx) {
  static CtxGetCurrentFn fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<CtxGetCurrentFn>(f);
  }();
  if (!fn) return set_error(GFD_ECUDA, "cuCtxGetCurrent is not available");
  *ctx = nullptr;
  if (fn(ctx) != 0 || !*ctx) return set_error(GFD_ECUDA, "no current CUDA context");
  return GFD_OK;
}

static int scratch_for_current_device(void** out) {
  int dev = 0;
  int st = check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
  if (st) return st;
  if (dev < 0 || dev >= 64) return set_error(GFD_EUNSUPPORTED, "device index out of range");
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  ScratchAddr& e = g_scratch_addr[dev];
  void* ctx = nullptr;
  // No current context yet (a first call before any other CUDA work on this
  // thread) reads as "not cached": the lookup below makes the runtime bind
  // the device's primary context, which is then recorded.
  if (current_context(&ctx) != GFD_OK) ctx = nullptr;
  if (!e.addr || !ctx || e.ctx != ctx) {
    void* p = nullptr;
    st = check_cuda(cudaGetSymbolAddress(&p, g_relax_scratch),
                    "cudaGetSymbolAddress(relaxation scratch)");
    if (st) return st;
    if ((st = current_context(&ctx))) return st;
    e.ctx = ctx;
    e.addr = p;
  }
  *out = e.addr;
  return GFD_OK;
}

}  // namespace gfd

using namespace gfd;

extern "C" int gfd_operator_relax_noalloc(gfd_operator* op, int dtype, int relax_method,
                                          void* func, const void* source, int nrelax, double w,
                                          void* stream) {
  if (!op) return set_error(GFD_EINVAL, "null operator");
  if (dtype != GFD_FLOAT64 && dtype != GFD_FLOAT32)
    return set_error(GFD_EINVAL, "relaxation works on real arrays only");
  if (!op->real) return set_error(GFD_EINVAL, "operator was built for complex arrays");
  if (!func || !source) return set_error(GFD_EINVAL, "null array pointer");
  if (nrelax < 0) return set_error(GFD_EINVAL, "negative sweep count");
  if (op->off[0] != 0 || op->off[1] != 0 || op->off[2] != 0)
    return set_error(GFD_EINVAL, "relaxation needs the diagonal (zero offset) as coefs[0]");
  const size_t bytes = (size_t)op->n[0] * op->n[1] * op->n[2] * dtype_size(dtype);
  if (bytes > kNoAllocScratchBytes)
    return set_error(GFD_EINVAL,
                     "grid needs " + std::to_string(bytes) +
                         " bytes of relaxation scratch; gfd_operator_relax_noalloc holds at most " +
                         std::to_string(kNoAllocScratchBytes) +
                         " bytes (2097152 float64 or 4194304 float32 points); use "
                         "gfd_operator_relax for larger grids");
  if (nrelax == 0) return GFD_OK;
  void* scratch = nullptr;
  int st = scratch_for_current_device(&scratch);
  if (st) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (relax_method == GFD_RELAX_GS)
    return op_gs_sweeps(op, dtype, func, source, nrelax, scratch, s);
  if (w == 0.0) return GFD_OK;
  // Weighted Jacobi ping-pong between func and the static scratch; the
  // scratch is fully overwritten by each sweep, so no clearing is needed.
  void* cur = func;
  void* nxt = scratch;
  for (int k = 0; k < nrelax; k++) {
    st = op_launch(op, dtype, OP_JACOBI, cur, nxt, source, 1, nullptr, w, nullptr, s);
    if (st) return st;
    void* tmp = cur;
    cur = nxt;
    nxt = tmp;
  }
  if (cur != func)
    return check_cuda(cudaMemcpyAsync(func, cur, bytes, cudaMemcpyDeviceToDevice, s),
                      "cudaMemcpyAsync(relax result)");
  return GFD_OK;
}
