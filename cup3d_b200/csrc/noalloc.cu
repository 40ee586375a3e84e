// cup_cnn_forward_host_noalloc: the network forward of cup_cnn_forward_host
// for callers that must not allocate device memory.
//
// cup_cnn_forward_host stages its host inputs and outputs in device buffers
// that it allocates and frees on every call.  cudaFree waits for the whole
// device to go idle, so a caller that evaluates the network from inside a
// running solve or time step (work queued on other streams) would stall all
// of it; and a caller whose device memory is owned by another allocator (a
// host framework that reserved the pool up front) may have none to give.
// This entry point stages the samples in one statically sized device array
// instead, so a call allocates no device memory and frees none.
//
// The staging array is a file-scope __device__ array: one copy per device
// per process, shared by every context on that device.  Two calls that used
// it at the same time would overwrite each other's samples, so calls hold a
// process-wide lock from the first copy in until their outputs are back on
// the host (the call synchronizes the context's stream before it returns).
//
// Set-up: the first call on a device looks the array's address up with
// cudaGetSymbolAddress, with that device current, and keeps it.  That first
// call belongs before any stream capture is begun on the device.
#include <mutex>

#include "context.h"

namespace cup3d {

namespace {

constexpr int kStageMaxSamples = CUP_CNN_FORWARD_NOALLOC_MAX;
constexpr int kInFloats = 1000;  // 10^3 input tile per sample
constexpr int kOutFloats = BN;   // 8^3 output block per sample
constexpr int kMaxDevices = 64;

// [kStageMaxSamples][1000] inputs, then [kStageMaxSamples][512] outputs:
// 64 * 1512 * 4 bytes = 387,072 bytes per device.
static __device__ __align__(256) float g_cnn_stage[kStageMaxSamples * (kInFloats + kOutFloats)];

std::mutex g_stage_lock;
float* g_stage_addr[kMaxDevices] = {};

// Address of g_cnn_stage on `device` (looked up once, with `device` current).
int stage_address(int device, float** out) {
  if (device < 0 || device >= kMaxDevices) return CUP_ERR_ARG;
  if (!g_stage_addr[device]) {
    int prev = -1;
    CUP_CUDA_TRY(cudaGetDevice(&prev));
    CUP_CUDA_TRY(cudaSetDevice(device));
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_cnn_stage);
    const cudaError_t e2 = cudaSetDevice(prev);
    if (e != cudaSuccess) return set_cuda_error(e, "cudaGetSymbolAddress(g_cnn_stage)", __FILE__, __LINE__);
    if (e2 != cudaSuccess) return set_cuda_error(e2, "cudaSetDevice (restore)", __FILE__, __LINE__);
    g_stage_addr[device] = static_cast<float*>(p);
  }
  *out = g_stage_addr[device];
  return 0;
}

}  // namespace

}  // namespace cup3d

using namespace cup3d;

extern "C" int cup_cnn_forward_host_noalloc(cup_ctx* c, const float* in, float* out, int32_t n) {
  if (!c || c->host_only || !in || !out || n <= 0)
    return ctx_fail(c, CUP_ERR_ARG, "cup_cnn_forward_host_noalloc: bad arguments");
  if (n > kStageMaxSamples)
    return ctx_fail(c, CUP_ERR_ARG,
                    "cup_cnn_forward_host_noalloc: " + std::to_string(n) +
                        " samples exceed the static staging capacity of " + std::to_string(kStageMaxSamples) +
                        " (CUP_CNN_FORWARD_NOALLOC_MAX); split the batch or use cup_cnn_forward_host");
  CnnState& S = c->cnn;
  if (!S.ready) return ctx_fail(c, CUP_ERR_STATE, "no weights");
  std::lock_guard<std::mutex> hold(g_stage_lock);
  float* stage = nullptr;
  if (int rc = stage_address(c->cfg.device, &stage)) return ctx_fail(c, rc, cup_last_error(nullptr));
  float* din = stage;
  float* dout = stage + size_t(kStageMaxSamples) * kInFloats;
  // Every return below happens with the lock held and, on an error after the
  // first copy was queued, after waiting for the stream: the next call (maybe
  // another context on another stream) must not find this call's copies or
  // kernel still reading or writing the shared array.
  auto fail_drained = [&](int rc) {
    cudaStreamSynchronize(c->stream);  // its own error is the one already recorded
    return ctx_fail(c, rc, cup_last_error(nullptr));
  };
  cudaError_t e = cudaMemcpyAsync(din, in, size_t(n) * kInFloats * sizeof(float), cudaMemcpyHostToDevice, c->stream);
  if (e != cudaSuccess) return fail_drained(set_cuda_error(e, "cnn_forward_noalloc in", __FILE__, __LINE__));
  if (int rc = cnn_forward_batch(S.W, din, dout, n, S.gpart, S.train_grid, c->stream)) return fail_drained(rc);
  e = cudaMemcpyAsync(out, dout, size_t(n) * kOutFloats * sizeof(float), cudaMemcpyDeviceToHost, c->stream);
  if (e != cudaSuccess) return fail_drained(set_cuda_error(e, "cnn_forward_noalloc out", __FILE__, __LINE__));
  e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess)
    return ctx_fail(c, set_cuda_error(e, "cnn_forward_noalloc sync", __FILE__, __LINE__), cup_last_error(nullptr));
  return 0;
}
