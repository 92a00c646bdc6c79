// noalloc.cu -- the tensor-core batch for callers that cannot allocate device
// memory.
//
// b200d2_diff2_coarse_batch needs a caller-provided workspace.  Some callers
// cannot provide one: a host program whose device memory is owned by another
// allocator (RELION's own caching allocator reserves most of the card up
// front, so a cudaMalloc from a plug-in fails or fragments its pool), a
// request path that must not pay cudaMalloc's implicit device
// synchronisation, or a plug-in interface that hands the library nothing but
// its input and output buffers.  For them this file keeps a fixed scratch
// area in the library's own device image and runs the same pipeline on it.
//
// The scratch is a file-scope static __device__ array of B200D2_STATIC_SCRATCH_BYTES
// (64 MiB): every GPU that loads the library holds it until the process
// exits.  Host code cannot use the array's name as a device address (on the
// host it names a stand-in object), so the device address is looked up with
// cudaGetSymbolAddress on the first call made while a device is current, and
// kept for that device's current CUDA context.  A new context (after
// cudaDeviceReset, or a host that destroys and recreates its primary
// context) reloads the library's device image, possibly elsewhere, so the
// address is looked up again whenever the current context differs from the
// one it was found in.  Make the first call on each device (and the first
// call after such a reset) before any stream capture.
//
// All calls share the one array, which keeps the previous call's contents:
// the pipeline's first stage resets everything that must start at zero (the
// status word and the per-particle min keys) and every later stage overwrites
// its whole section.  Calls that overlap on the GPU (concurrent streams, or
// several host threads on one device) race on the array and must be
// serialised by the caller.
//
// It calls no cudaMalloc, cudaFree or other allocating routine, and runs all
// stages in order on the caller's stream (the allocating entry point uses a
// side stream; this one creates none).
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "common.cuh"

namespace b200d2 {
size_t tc_workspace_bytes(const b200d2_view& view, const b200d2_batch& b, int precision,
                          bool allow_split = true);
int tc_run_stage(const b200d2_view& view, const b200d2_batch& b, int precision, int stage, void* ws,
                 size_t ws_bytes, cudaStream_t s, bool allow_split = true);
const char* tc_stage_name(int precision, int stage);
}  // namespace b200d2

namespace {

static __device__ __align__(256) unsigned char g_static_scratch[B200D2_STATIC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
void* g_scratch_ptr[kMaxDevices] = {nullptr};
unsigned long long g_scratch_ctx[kMaxDevices] = {0};  // unique id of the context the address was found in

// cuCtxGetCurrent and cuCtxGetId through the runtime's driver entry-point
// query (the library links no driver API import).
struct CtxApi {
  CUresult (*current)(CUcontext*) = nullptr;
  CUresult (*id)(CUcontext, unsigned long long*) = nullptr;
};
const CtxApi& ctx_api() {
  static CtxApi api;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      api.current = reinterpret_cast<CUresult (*)(CUcontext*)>(p);
    p = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      api.id = reinterpret_cast<CUresult (*)(CUcontext, unsigned long long*)>(p);
  });
  return api;
}

// Unique id (never reused within the process) of the current context, or 0
// when no context is current yet.
int current_ctx_id(unsigned long long* id) {
  const CtxApi& api = ctx_api();
  if (!api.current || !api.id) return B200D2_ERR_CUDA;
  CUcontext ctx = nullptr;
  if (api.current(&ctx) != CUDA_SUCCESS) return B200D2_ERR_CUDA;
  *id = 0;
  if (ctx && api.id(ctx, id) != CUDA_SUCCESS) return B200D2_ERR_CUDA;
  return B200D2_OK;
}

// Device address of g_static_scratch in the current device's current
// context (looked up once per context).
int static_scratch(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return b200d2::status_from_cuda(e);
  if (dev < 0 || dev >= kMaxDevices) return B200D2_ERR_UNSUPPORTED;
  unsigned long long ctx = 0;  // 0 until the runtime has made the device's context current
  int st = current_ctx_id(&ctx);
  if (st != B200D2_OK) return st;
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (!ctx || !g_scratch_ptr[dev] || g_scratch_ctx[dev] != ctx) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_static_scratch);  // also makes the primary context current
    if (e != cudaSuccess || !p) return b200d2::status_from_cuda(e == cudaSuccess ? cudaErrorInvalidSymbol : e);
    st = current_ctx_id(&ctx);
    if (st != B200D2_OK) return st;
    if (!ctx) return B200D2_ERR_CUDA;
    g_scratch_ptr[dev] = p;
    g_scratch_ctx[dev] = ctx;
  }
  *out = g_scratch_ptr[dev];
  return B200D2_OK;
}

}  // namespace

extern "C" int b200d2_diff2_coarse_batch_static(const b200d2_view* view, const b200d2_batch* batch,
                                                int precision, void* stream) {
  if (!view || !batch) return B200D2_ERR_INVALID;
  if (!b200d2::is_tc_precision(precision))
    return B200D2_ERR_UNSUPPORTED;  // the CUDA-core paths need no scratch: use b200d2_diff2_coarse_batch
  if (batch->O == 0 || batch->T == 0 || batch->P == 0) return B200D2_OK;
  // the allocating entry point's size query also validates the view and batch
  if (b200d2_diff2_coarse_batch_workspace(view, batch, precision) == 0) return B200D2_ERR_INVALID;
  // the scratch is sized for the contraction without k-splits (no partial sums)
  const size_t need = b200d2::tc_workspace_bytes(*view, *batch, precision, false);
  if (need > (size_t)B200D2_STATIC_SCRATCH_BYTES) return B200D2_ERR_TOO_LARGE;
  void* ws = nullptr;
  int st = static_scratch(&ws);
  if (st != B200D2_OK) return st;
  cudaStream_t s = (cudaStream_t)stream;
  for (int stage = 0; b200d2::tc_stage_name(precision, stage) != nullptr; ++stage) {
    st = b200d2::tc_run_stage(*view, *batch, precision, stage, ws, (size_t)B200D2_STATIC_SCRATCH_BYTES, s,
                              false);
    if (st != B200D2_OK) return st;
  }
  return B200D2_OK;
}
