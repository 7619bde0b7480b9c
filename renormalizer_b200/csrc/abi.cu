// Context management of the C ABI (reno_b200.h).
#include "reno_common.cuh"

using namespace reno;

extern "C" int reno_version(void) { return 100; }

extern "C" int reno_ctx_create(int device, reno_ctx** out) {
  if (!out) return RENO_ERR_INVALID;
  *out = nullptr;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || device < 0 || device >= n) return RENO_ERR_CUDA;
  e = cudaSetDevice(device);
  if (e != cudaSuccess) return RENO_ERR_CUDA;
  reno_ctx* c = new reno_ctx();
  c->device = device;
  cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
  *out = c;
  return RENO_OK;
}

extern "C" int reno_ctx_destroy(reno_ctx* ctx) {
  delete ctx;
  return RENO_OK;
}

extern "C" int reno_ctx_set_stream(reno_ctx* ctx, void* stream) {
  if (!ctx) return RENO_ERR_INVALID;
  ctx->stream = static_cast<cudaStream_t>(stream);
  return RENO_OK;
}

extern "C" const char* reno_last_error(const reno_ctx* ctx) {
  if (!ctx) return "null context";
  return ctx->last_error.c_str();
}

extern "C" int reno_ctx_synchronize(reno_ctx* ctx) {
  if (!ctx) return RENO_ERR_INVALID;
  return check_cuda(ctx, cudaStreamSynchronize(ctx->stream), "reno_ctx_synchronize");
}

extern "C" int reno_launch_count(long long* count) {
  if (!count) return RENO_ERR_INVALID;
  *count = g_launches.load();
  return RENO_OK;
}

extern "C" int reno_set_wait_limit_ns(uint64_t ns) {
  if (ns < 1000000ull || ns > 60000000000ull) return RENO_ERR_INVALID;  // 1 ms .. 60 s
  g_wait_ns.store(ns, std::memory_order_relaxed);
  return RENO_OK;
}

extern "C" int reno_set_split_accumulation_chunk(int32_t k_elems) {
  if (k_elems < 0) return RENO_ERR_INVALID;
  g_split_chunk_k.store(k_elems, std::memory_order_relaxed);
  return RENO_OK;
}

extern "C" int reno_test_skip_arrival(int32_t kind, int32_t at) {
  if (at < -1) return RENO_ERR_INVALID;
  if (kind == RENO_SKIP_SPLIT_STAGE) g_skip_split_stage.store(at);
  else if (kind == RENO_SKIP_HETRD_ARRIVAL) g_skip_hetrd_column.store(at);
  else return RENO_ERR_INVALID;
  return RENO_OK;
}
