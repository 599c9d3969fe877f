// Coupling matvec for callers that must not allocate device memory.
//
// Some host programs cannot call cudaMalloc at the point where they want a matvec: a code that
// reserves all of its device memory once at start-up and forbids allocation inside its time loop,
// an embedding runtime that owns the CUDA allocator, or a caller that only hands out fixed
// input/output buffers. yasf_coupling_matvec_noalloc computes the same y = W x as
// yasf_coupling_matvec, but its scratch (the per-source V stream, the per-chunk partial sums and
// the stage-timeout word) lives in one file-scope device array of YASF_STATIC_SCRATCH_BYTES, so
// the call allocates nothing. The caller still passes the plan, positions, x and y.
//
// Limits and sharing:
// - Problems whose scratch exceeds the array are rejected with YASF_ERR_SCRATCH_LIMIT before any
//   device work (yasf_coupling_workspace_size gives the bytes a problem needs).
// - Every call on a device uses the same array, which keeps the previous call's contents. The
//   only word that must start at zero (the stage-timeout flag) is cleared by each call; the
//   stream and partial sums are fully overwritten. Calls that overlap on the GPU (different
//   streams, or different host threads on one device) race on the array and corrupt each other;
//   order them on one stream.
// - The first call on each device looks up the array's device address with that device current
//   (cudaGetSymbolAddress, which may load the module); make that first call before any stream
//   capture begins. The address is cached together with the unique id of the CUDA context it was
//   looked up in: after cudaDeviceReset (or any other teardown of the primary context) the next
//   call sees a new context id and looks the address up again instead of using a stale one.
#include <cuda.h>

#include <mutex>

#include "capi_internal.h"

namespace yasf {

static __device__ __align__(256) unsigned char g_static_scratch[YASF_STATIC_SCRATCH_BYTES];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
void* g_scratch_ptr[kMaxDevices] = {nullptr};
unsigned long long g_scratch_ctx[kMaxDevices] = {0};

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// Unique id (for the life of the process) of the CUDA context current on this thread. The driver
// functions are fetched through the runtime, so the library needs no link against libcuda.
int current_context_id(unsigned long long* id) {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static int looked_up = 0;
  if (!looked_up) {
    cudaDriverEntryPointQueryResult q1 = cudaDriverEntryPointSymbolNotFound, q2 = q1;
    void* f1 = nullptr;
    void* f2 = nullptr;
    YASF_CUDA_TRY(cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1));
    YASF_CUDA_TRY(cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2));
    if (q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess || !f1 || !f2) {
      set_error_text("driver lacks cuCtxGetCurrent / cuCtxGetId");
      return YASF_ERR_CUDA;
    }
    get_current = reinterpret_cast<CtxGetCurrentFn>(f1);
    get_id = reinterpret_cast<CtxGetIdFn>(f2);
    looked_up = 1;
  }
  CUcontext ctx = nullptr;
  *id = 0;
  if (get_current(&ctx) != CUDA_SUCCESS) {
    set_error_text("cuCtxGetCurrent failed");
    return YASF_ERR_CUDA;
  }
  if (!ctx) return YASF_OK;  // no context bound to this thread yet: id 0
  if (get_id(ctx, id) != CUDA_SUCCESS) {
    set_error_text("cuCtxGetId failed");
    return YASF_ERR_CUDA;
  }
  return YASF_OK;
}

// Device address of the static scratch for the current device, looked up once per device and
// context (g_scratch_mu also guards the one-time driver lookup above).
int static_scratch(void** out) {
  int dev = -1;
  YASF_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return YASF_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  unsigned long long ctx = 0;
  if (int st = current_context_id(&ctx)) return st;
  if (ctx == 0 || !g_scratch_ptr[dev] || g_scratch_ctx[dev] != ctx) {
    void* p = nullptr;
    // binds the device's primary context to this thread if no runtime call did so yet
    YASF_CUDA_TRY(cudaGetSymbolAddress(&p, g_static_scratch));
    if (!p) return YASF_ERR_CUDA;
    if (ctx == 0) {
      if (int st = current_context_id(&ctx)) return st;
      if (ctx == 0) {
        set_error_text("no CUDA context current after the symbol lookup");
        return YASF_ERR_CUDA;
      }
    }
    g_scratch_ptr[dev] = p;
    g_scratch_ctx[dev] = ctx;
  }
  *out = g_scratch_ptr[dev];
  return YASF_OK;
}
}  // namespace

}  // namespace yasf

using namespace yasf;

extern "C" int yasf_coupling_matvec_noalloc(const yasf_plan* plan, int n_particles,
                                            const double* positions, double k_medium,
                                            const double* x, double* y, int precision,
                                            void* stream) {
  int st = validate_coupling(plan, n_particles, positions, k_medium, precision);
  if (st != YASF_OK) return st;
  if (!x || !y || x == y) return YASF_ERR_INVALID_ARGUMENT;
  if (!aligned16(x) || !aligned16(y)) return YASF_ERR_ALIGNMENT;
  const size_t need = coupling_layout(plan, n_particles, precision).total;
  if (need > (size_t)YASF_STATIC_SCRATCH_BYTES) {
    set_error_text("problem needs more scratch than the static array holds");
    return YASF_ERR_SCRATCH_LIMIT;
  }
  void* scratch = nullptr;
  if ((st = static_scratch(&scratch)) != YASF_OK) return st;
  return coupling_column(plan, n_particles, positions, k_medium, nullptr, x, y, precision, 0,
                         scratch, (size_t)YASF_STATIC_SCRATCH_BYTES,
                         static_cast<cudaStream_t>(stream));
}
