// Allocation-free variant of the global skeleton solve.
//
// mhm_skeleton_solve expects the caller to allocate its scratch workspace.
// Some callers have no way to do that: host codes that reach this library only
// through its C ABI from an environment without a CUDA allocator of their own
// (a Fortran or C simulation driver, an FFI binding), or a serving process that
// reserves all device memory at start-up and must not call cudaMalloc/cudaFree
// afterwards (both calls also synchronise the device and stall other streams).
// mhm_skeleton_solve_static gives them the same solve with its scratch held in
// a fixed file-scope device array instead.
#include <mutex>

#include "mhm_common.cuh"

namespace {

// Scratch of the allocation-free entry point: every GPU that loads the library
// holds these 4 MiB until the process exits.
constexpr int64_t kStaticScratchBytes = int64_t(4) << 20;
static __device__ __align__(256) unsigned char g_skeleton_scratch[kStaticScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
void* g_scratch_address[kMaxDevices] = {};

// Device address of the scratch array on the current device.  In host code the
// array's name is only a host-side stand-in, so the address is looked up once
// per device, with that device current, and cached.
int scratch_address(void** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return MHM_ERR_LAUNCH;
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (g_scratch_address[dev] == nullptr) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_skeleton_scratch) != cudaSuccess || p == nullptr) {
      cudaGetLastError();
      return MHM_ERR_LAUNCH;
    }
    g_scratch_address[dev] = p;
  }
  *out = g_scratch_address[dev];
  return MHM_OK;
}

}  // namespace

extern "C" int mhm_skeleton_solve_static(const mhm_skeleton_system* s, const double* rhs,
                                         const double* load_scale, double* x, double rtol,
                                         double inner_rtol, int32_t max_inner, int32_t max_outer,
                                         int32_t grid, int32_t* info, double* stats, void* stream) {
  if (!s) return MHM_ERR_ARGUMENT;
  const int64_t need = mhm_skeleton_workspace_bytes(s, grid);
  if (need < 0) return MHM_ERR_ARGUMENT;
  if (need > kStaticScratchBytes) return MHM_ERR_UNSUPPORTED;
  void* scratch = nullptr;
  const int rc = scratch_address(&scratch);
  if (rc != MHM_OK) return rc;
  // The solve zeroes its barrier counters and error flag itself on every call;
  // the remaining scratch is fully written before it is read.
  return mhm_skeleton_solve(s, rhs, load_scale, x, rtol, inner_rtol, max_inner, max_outer, grid,
                            scratch, kStaticScratchBytes, info, stats, stream);
}
