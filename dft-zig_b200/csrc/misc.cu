// Status strings, per-thread last-error message, pointer classification.
#include <atomic>
#include <string>

#include "kctx.cuh"

namespace dftcuda {

static std::atomic<uint64_t> g_launches{0};
uint64_t launches_total() { return g_launches.load(std::memory_order_relaxed); }
void count_launch(int n) { g_launches.fetch_add((uint64_t)n, std::memory_order_relaxed); }

cudaEvent_t Profiler::take() {
  if (!pool.empty()) {
    cudaEvent_t e = pool.back();
    pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}

void Profiler::resolve() {
  for (auto& ev : pending) {
    cudaEventSynchronize(ev.b);
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, ev.a, ev.b) == cudaSuccess) ns[ev.cat] += (double)ms * 1e6;
    pool.push_back(ev.a);
    pool.push_back(ev.b);
  }
  pending.clear();
}

void Profiler::clear() {
  resolve();
  for (double& v : ns) v = 0.0;
  for (uint64_t& v : launches) v = 0;
  calls = columns = 0;
}

void Profiler::destroy() {
  resolve();
  for (cudaEvent_t e : pool) cudaEventDestroy(e);
  pool.clear();
}

static thread_local std::string g_last_error;

void set_last_error(int status, const std::string& msg) {
  (void)status;
  g_last_error = msg;
}

bool is_device_pointer(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();  // clear the sticky-free error of an unregistered host pointer
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace dftcuda

extern "C" const char* dftcuda_status_string(int status) {
  switch (status) {
    case DFTCUDA_OK: return "ok";
    case DFTCUDA_ERR_INVALID_MATRIX_SIZE: return "InvalidMatrixSize";
    case DFTCUDA_ERR_INVALID_GRID: return "InvalidGrid";
    case DFTCUDA_ERR_EIGENSOLVER_FAILURE: return "LapackFailure";
    case DFTCUDA_ERR_OUT_OF_MEMORY: return "OutOfMemory";
    case DFTCUDA_ERR_CUDA: return "CudaError";
    case DFTCUDA_ERR_INVALID_ARGUMENT: return "InvalidArgument";
    case DFTCUDA_ERR_UNSUPPORTED: return "Unsupported";
    case DFTCUDA_ERR_TIMEOUT: return "Timeout";
    default: return "unknown";
  }
}

extern "C" const char* dftcuda_last_error_message(void) { return dftcuda::g_last_error.c_str(); }

extern "C" int dftcuda_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

extern "C" int dftcuda_kctx_set_profiling(dftcuda_kctx* c, int enable) {
  if (!c) return dftcuda::fail(DFTCUDA_ERR_INVALID_ARGUMENT, "set_profiling: null context");
  cudaStreamSynchronize(c->stream);
  c->prof.clear();
  c->prof.on = enable != 0;
  return DFTCUDA_OK;
}

extern "C" int dftcuda_kctx_get_profile(dftcuda_kctx* c, dftcuda_profile* out) {
  using namespace dftcuda;
  if (!c || !out) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "get_profile: null argument");
  cudaStreamSynchronize(c->stream);
  Profiler& p = c->prof;
  p.resolve();
  auto u = [](double v) { return (uint64_t)(v + 0.5); };
  dftcuda_profile r{};
  r.local_plane_inv_ns = u(p.ns[P_PLANE_INV]);
  r.local_xline_ns = u(p.ns[P_XLINE]);
  r.local_plane_fwd_ns = u(p.ns[P_PLANE_FWD]);
  r.local_plane_inv_launches = p.launches[P_PLANE_INV];
  r.local_xline_launches = p.launches[P_XLINE];
  r.local_plane_fwd_launches = p.launches[P_PLANE_FWD];
  r.nl_project_ns = u(p.ns[P_NL_PROJECT]);
  r.nl_dij_ns = u(p.ns[P_NL_DIJ]);
  r.nl_backproject_ns = u(p.ns[P_NL_BACK]);
  r.apply_local_ns = r.local_plane_inv_ns + r.local_xline_ns + r.local_plane_fwd_ns;
  r.apply_nonlocal_ns = r.nl_project_ns + r.nl_dij_ns + r.nl_backproject_ns;
  r.apply_h_ns = r.apply_local_ns + r.apply_nonlocal_ns;
  r.density_ns = u(p.ns[P_DENSITY]);
  r.subspace_ns = u(p.ns[P_SUBSPACE]);
  r.apply_h_calls = p.calls;
  r.apply_h_columns = p.columns;
  uint64_t l = 0;
  for (int i = 0; i < P_NCAT; ++i) l += p.launches[i];
  r.kernel_launches = l;
  *out = r;
  return DFTCUDA_OK;
}
