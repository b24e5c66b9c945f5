// Status strings, per-thread last-error message, pointer classification.
#include <atomic>
#include <mutex>
#include <map>
#include <string>
#include <utility>

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

int ensure_max_dynamic_smem(const void* kernel, int bytes) {
  // the limit only ever rises: a later, smaller request must not undercut a launch that needs more
  static std::mutex mu;
  static std::map<std::pair<int, const void*>, int> set_to;
  int dev = 0;
  DFT_CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  const auto key = std::make_pair(dev, kernel);
  auto it = set_to.find(key);
  if (it != set_to.end() && it->second >= bytes) return DFTCUDA_OK;
  const cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e != cudaSuccess)
    return fail(DFTCUDA_ERR_CUDA, std::string("cudaFuncSetAttribute(MaxDynamicSharedMemorySize): ") + cudaGetErrorString(e));
  set_to[key] = bytes;
  return DFTCUDA_OK;
}

static std::atomic<long> g_wait_polls{0};
static std::atomic<bool> g_wait_unreachable{false};
WaitLimits wait_limits() { return WaitLimits{g_wait_polls.load(), g_wait_unreachable.load()}; }

// -1: no failure planned; k >= 0: the k-th following allocation fails (then -1 again).
static std::atomic<long> g_fail_alloc{-1};
bool alloc_should_fail() {
  long v = g_fail_alloc.load(std::memory_order_relaxed);
  while (v >= 0) {
    if (g_fail_alloc.compare_exchange_weak(v, v - 1)) return v == 0;
  }
  return false;
}

DeviceGuard::DeviceGuard(int dev) {
  if (cudaGetDevice(&prev) != cudaSuccess) {
    cudaGetLastError();
    prev = -1;
  }
  if (dev >= 0 && dev != prev) {
    status = cudaSetDevice(dev) == cudaSuccess ? DFTCUDA_OK : fail(DFTCUDA_ERR_CUDA, "cudaSetDevice to the context's device");
    switched = status == DFTCUDA_OK;
  }
}
DeviceGuard::~DeviceGuard() {
  if (switched && prev >= 0) cudaSetDevice(prev);
}

}  // namespace dftcuda

extern "C" int dftcuda_debug_set_wait_limits(long polls, int unreachable) {
  if (polls < 0) return dftcuda::fail(DFTCUDA_ERR_INVALID_ARGUMENT, "debug_set_wait_limits: polls < 0");
  dftcuda::g_wait_polls.store(polls);
  dftcuda::g_wait_unreachable.store(unreachable != 0);
  return DFTCUDA_OK;
}

extern "C" int dftcuda_debug_fail_alloc(long after) {
  dftcuda::g_fail_alloc.store(after < 0 ? -1 : after);
  return DFTCUDA_OK;
}

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
  r.local_layout = c->last_layout < 0 ? 0 : (uint64_t)c->last_layout;
  *out = r;
  return DFTCUDA_OK;
}

// The library's complex GEMM for tests and benchmarks (zgemm.cu / tc_gemm.cu behind one call).
extern "C" int dftcuda_complex_gemm(int precision, size_t M, size_t N, size_t K, const double* a, long lda, int a_kc,
                                    int conj_a, const double* b, long ldb, int b_kc, int conj_b, double* out, long ldo_r,
                                    long ldo_c, double alpha, double beta) {
  using namespace dftcuda;
  if (M == 0 || N == 0) return DFTCUDA_OK;
  if (K == 0 || !a || !b || !out) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "complex_gemm: K == 0 or null pointer");
  if (M > INT32_MAX || N > INT32_MAX || K > INT32_MAX)
    return fail(DFTCUDA_ERR_INVALID_MATRIX_SIZE, "complex_gemm: dimension above 2^31 - 1");
  if (precision != DFTCUDA_PRECISION_FP64 && !precision_uses_tc(precision))
    return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "complex_gemm: precision must be FP64, TF32 or TF32X3");
  GemmArgs g{};
  g.M = (int)M; g.N = (int)N; g.K = (int)K;
  g.A = reinterpret_cast<const double2*>(a); g.lda = lda; g.a_kc = a_kc != 0; g.conj_a = conj_a != 0;
  g.B = reinterpret_cast<const double2*>(b); g.ldb = ldb; g.b_kc = b_kc != 0; g.conj_b = conj_b != 0;
  g.O = reinterpret_cast<double2*>(out); g.ldo_r = ldo_r; g.ldo_c = ldo_c;
  g.alpha = alpha; g.beta = beta;
  const bool tc = precision_uses_tc(precision);
  const size_t ws_elems = tc ? cgemm_tf32_workspace_elems(g.M, g.N, g.K) : zgemm_workspace_elems(g.M, g.N, g.K);
  int dev = 0;
  DFT_CUDA_TRY(cudaGetDevice(&dev));
  // One engine per device (stream, split-K workspace, error flag, pre-split operand tiles), kept for
  // the life of the process and grown on demand, so that a call costs its kernels and one sync.
  struct Engine {
    cudaStream_t s = nullptr;
    double2* ws = nullptr;
    size_t ws_cap = 0;
    int* err = nullptr;
    TcScratch tiles;
    std::mutex mu;
  };
  static std::mutex map_mu;
  static std::map<int, Engine*> engines;
  Engine* en = nullptr;
  {
    std::lock_guard<std::mutex> lock(map_mu);
    Engine*& slot = engines[dev];
    if (!slot) slot = new Engine();  // never freed: device memory is released at context teardown
    en = slot;
  }
  std::lock_guard<std::mutex> lock(en->mu);
  if (!en->s && (cudaStreamCreateWithFlags(&en->s, cudaStreamDefault) != cudaSuccess || dev_malloc(&en->err, sizeof(int)) != cudaSuccess)) {
    if (en->s) cudaStreamDestroy(en->s);
    en->s = nullptr;
    en->err = nullptr;
    return fail(DFTCUDA_ERR_CUDA, "complex_gemm: stream or error-flag allocation failed");
  }
  if (ws_elems > en->ws_cap) {
    cudaStreamSynchronize(en->s);
    if (en->ws) cudaFree(en->ws);
    en->ws = nullptr;
    en->ws_cap = 0;
    if (dev_malloc(&en->ws, sizeof(double2) * ws_elems) != cudaSuccess) return fail(DFTCUDA_ERR_OUT_OF_MEMORY, "complex_gemm: workspace");
    en->ws_cap = ws_elems;
  }
  DFT_CUDA_TRY(cudaMemsetAsync(en->err, 0, sizeof(int), en->s));
  en->tiles.valid = false;  // operands differ from call to call
  int rc = tc ? cgemm_tf32(g, en->s, en->ws, en->ws_cap, en->err, precision == DFTCUDA_PRECISION_TF32X3, &en->tiles)
              : zgemm(g, en->s, en->ws, en->ws_cap);
  int herr = 0;
  const cudaError_t e = rc == DFTCUDA_OK ? cudaMemcpyAsync(&herr, en->err, sizeof(int), cudaMemcpyDeviceToHost, en->s) : cudaSuccess;
  const cudaError_t e2 = cudaStreamSynchronize(en->s);
  if (rc == DFTCUDA_OK) {
    if (e != cudaSuccess || e2 != cudaSuccess) rc = fail(DFTCUDA_ERR_CUDA, std::string("complex_gemm: ") + cudaGetErrorString(e2));
    else if (herr) rc = fail(DFTCUDA_ERR_TIMEOUT, "complex_gemm: a tensor-core pipeline wait timed out");
  }
  return rc;
}
