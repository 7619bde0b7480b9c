// reno_heff_apply_noalloc: the effective-Hamiltonian matvec for callers that
// cannot allocate device memory, using a fixed scratch array that is part of
// the library image instead of a caller-provided workspace.
//
// Who needs it: hosts that have handed all device memory to their own pool or
// arena and forbid third-party code from allocating (frameworks that reserve
// the whole GPU at start-up), and foreign-language hosts whose runtime cannot
// own a device allocation across calls.  They pass inputs and outputs only.
//
// Costs and rules:
//  - g_heff_noalloc_scratch is RENO_NOALLOC_SCRATCH_BYTES of device memory
//    that every GPU which loads the library holds until the process exits.
//  - Problems whose workspace (reno_heff_workspace_bytes) exceeds it are
//    rejected with RENO_ERR_WORKSPACE; use reno_heff_apply for those.
//  - Every call shares the one array and it keeps the previous call's
//    contents.  The matvec overwrites every scratch byte it reads, so nothing
//    has to start at zero.  Calls whose kernels can overlap on the GPU (two
//    streams, two host threads) race on the array: serialise them.
//  - The first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (with that device current); make that first call
//    before any stream capture.
#include <mutex>
#include "reno_common.cuh"

static __device__ __align__(256) unsigned char g_heff_noalloc_scratch[RENO_NOALLOC_SCRATCH_BYTES];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
void* g_scratch_addr[kMaxDevices] = {nullptr};

// device address of the scratch array on ctx's device (set up once per device)
int scratch_for(reno_ctx* ctx, void** out) {
  if (ctx->device < 0 || ctx->device >= kMaxDevices)
    return reno::set_error(ctx, RENO_ERR_INVALID, "reno_heff_apply_noalloc: device index out of range");
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_addr[ctx->device]) {
    int prev = -1;
    cudaError_t e = cudaGetDevice(&prev);
    if (e != cudaSuccess) return reno::check_cuda(ctx, e, "reno_heff_apply_noalloc: cudaGetDevice");
    if (prev != ctx->device) {
      e = cudaSetDevice(ctx->device);
      if (e != cudaSuccess) return reno::check_cuda(ctx, e, "reno_heff_apply_noalloc: cudaSetDevice");
    }
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_heff_noalloc_scratch);
    if (prev != ctx->device) {
      const cudaError_t er = cudaSetDevice(prev);
      if (er != cudaSuccess) return reno::check_cuda(ctx, er, "reno_heff_apply_noalloc: restoring the device");
    }
    if (e != cudaSuccess) return reno::check_cuda(ctx, e, "reno_heff_apply_noalloc: cudaGetSymbolAddress");
    g_scratch_addr[ctx->device] = p;
  }
  *out = g_scratch_addr[ctx->device];
  return RENO_OK;
}
}  // namespace

extern "C" int reno_heff_apply_noalloc(reno_ctx* ctx, const reno_heff_desc* desc, const void* L, const void* W1,
                                       const void* W2, const void* R, const void* psi, void* y) {
  if (!ctx) return RENO_ERR_INVALID;
  size_t need = 0;
  if (reno_heff_workspace_bytes(desc, &need) != RENO_OK)
    return reno::set_error(ctx, RENO_ERR_INVALID, "reno_heff_apply_noalloc: invalid descriptor");
  if (need > (size_t)RENO_NOALLOC_SCRATCH_BYTES)
    return reno::set_error(ctx, RENO_ERR_WORKSPACE,
                           "reno_heff_apply_noalloc: this matvec needs " + std::to_string(need) +
                               " bytes of scratch but the built-in array holds " +
                               std::to_string((size_t)RENO_NOALLOC_SCRATCH_BYTES) +
                               "; call reno_heff_apply with a workspace instead");
  // the kernels launch on the caller's current device: the scratch address
  // must belong to that device
  int cur = -1;
  const cudaError_t ce = cudaGetDevice(&cur);
  if (ce != cudaSuccess) return reno::check_cuda(ctx, ce, "reno_heff_apply_noalloc: cudaGetDevice");
  if (cur != ctx->device)
    return reno::set_error(ctx, RENO_ERR_INVALID,
                           "reno_heff_apply_noalloc: the current device (" + std::to_string(cur) +
                               ") is not the context's device (" + std::to_string(ctx->device) +
                               "); make the context's device current first");
  void* scratch = nullptr;
  const int st = scratch_for(ctx, &scratch);
  if (st != RENO_OK) return st;
  return reno_heff_apply(ctx, desc, L, W1, W2, R, psi, y, scratch, (size_t)RENO_NOALLOC_SCRATCH_BYTES);
}
