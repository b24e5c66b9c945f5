// Autotuner for one k-point context's H|psi>: times candidate launch configurations of the real
// operator on the context's own data (its basis, V(r) and projectors) with CUDA events and keeps
// the fastest.  Knobs, tuned one after another (coordinate descent from the built-in defaults):
//   1. FFT passes: four-step register kernels (local4.cu) or the generic shared-memory passes;
//   2. the box workspace budget that sets how many columns one chunk of FFT passes carries
//      (L2 residency of the active-plane workspace against launch count);
//   3. split-K of the projection GEMM; 4. split-K of the back-projection GEMM.
// The reference sizes its FFT plans and BLAS calls once and never measures; here the shapes of
// every cell and k-point differ (uneven n_pw, box sizes 20^3 ... 108^3), so they are measured.
#include <algorithm>
#include <vector>

#include "kctx.cuh"

namespace dftcuda {
namespace {

__global__ void k_tune_fill(double2* __restrict__ x, long count) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= count) return;
  uint64_t z = (uint64_t)i * 0x9E3779B97F4A7C15ULL + 0x2545F4914F6CDD1DULL;
  z = (z ^ (z >> 31)) * 0xBF58476D1CE4E5B9ULL;
  z ^= z >> 29;
  x[i] = make_double2((double)(z & 0xFFFFF) / 1048576.0 - 0.5, (double)((z >> 20) & 0xFFFFF) / 1048576.0 - 0.5);
}

struct Timer {
  cudaEvent_t a = nullptr, b = nullptr;
  Timer() {
    cudaEventCreate(&a);
    cudaEventCreate(&b);
  }
  ~Timer() {
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  }
};

}  // namespace
}  // namespace dftcuda

using namespace dftcuda;

extern "C" int dftcuda_kctx_autotune(dftcuda_kctx* c, size_t ncols, dftcuda_tune_report* report) {
  if (!c || ncols == 0) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "kctx_autotune: null context or no columns");
  DeviceGuard dg(c->device);  // the context's device, whatever the caller has current
  DFT_TRY(dg.status);
  if (!c->has_vloc) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "kctx_autotune: local potential not set (dftcuda_set_vloc)");
  cudaStream_t s = c->stream;
  const size_t n = c->npw;
  double2* xy = nullptr;
  if (dev_malloc(&xy, sizeof(double2) * n * ncols * 2) != cudaSuccess)
    return fail(DFTCUDA_ERR_OUT_OF_MEMORY, "kctx_autotune: trial columns");
  double2* x = xy;
  double2* y = xy + n * ncols;
  k_tune_fill<<<ceil_div(n * ncols, 256), 256, 0, s>>>(x, (long)(n * ncols)); count_launch();
  const bool prof = c->prof.on;
  c->prof.on = false;
  Timer tm;
  int evaluated = 0;
  int st = DFTCUDA_OK;
  // median of three timed applications after one warm-up
  auto measure = [&](double* ms_out) -> int {
    DFT_TRY(kctx_apply_h_dev(c, x, y, ncols, s));
    float t[3];
    for (int r = 0; r < 3; ++r) {
      DFT_CUDA_TRY(cudaEventRecord(tm.a, s));
      DFT_TRY(kctx_apply_h_dev(c, x, y, ncols, s));
      DFT_CUDA_TRY(cudaEventRecord(tm.b, s));
      DFT_CUDA_TRY(cudaEventSynchronize(tm.b));
      DFT_CUDA_TRY(cudaEventElapsedTime(&t[r], tm.a, tm.b));
    }
    std::sort(t, t + 3);
    *ms_out = t[1];
    ++evaluated;
    return DFTCUDA_OK;
  };
  double best = 0.0;
  st = measure(&best);
  const double default_ms = best;
  // 1. local-operator layout: stick layout, plane layout (four-step passes), generic passes
  const bool fast_avail = (c->precision == DFTCUDA_PRECISION_FP64) ? c->fast64 : c->fast32;
  const bool sticks_avail = (c->precision == DFTCUDA_PRECISION_FP64) ? c->sticks64 : c->sticks32;
  if (st == DFTCUDA_OK && (fast_avail || sticks_avail)) {
    const bool keep_generic = c->fft_generic, keep_off = c->sticks_off;
    bool pick_generic = keep_generic, pick_off = keep_off;
    const bool cand[3][2] = {{false, false}, {false, true}, {true, true}};  // {generic, sticks_off}
    for (int i = 0; i < 3 && st == DFTCUDA_OK; ++i) {
      if (cand[i][0] == keep_generic && cand[i][1] == keep_off) continue;  // the default, timed above
      if (!cand[i][0] && !cand[i][1] && !sticks_avail) continue;
      if (!cand[i][0] && cand[i][1] && !fast_avail) continue;
      c->fft_generic = cand[i][0];
      c->sticks_off = cand[i][1];
      double t = 0.0;
      st = measure(&t);
      if (st == DFTCUDA_OK && t < best) {
        best = t;
        pick_generic = cand[i][0];
        pick_off = cand[i][1];
      }
    }
    c->fft_generic = pick_generic;
    c->sticks_off = pick_off;
  }
  // 2. box workspace budget
  if (st == DFTCUDA_OK) {
    const double keep = c->w_budget_bytes;
    double pick = keep;
    for (double mb : {24.0, 48.0, 192.0}) {
      c->w_budget_bytes = mb * 1024 * 1024;
      double t = 0.0;
      st = measure(&t);
      if (st != DFTCUDA_OK) break;
      if (t < best) {
        best = t;
        pick = c->w_budget_bytes;
      }
    }
    c->w_budget_bytes = pick;
  }
  // 3-4. projector GEMM split-K counts
  if (st == DFTCUDA_OK && c->nl.nproj > 0) {
    for (int which = 0; which < 2 && st == DFTCUDA_OK; ++which) {
      int& knob = which == 0 ? c->split_proj : c->split_back;
      const int keep = knob;
      int pick = keep;
      // the back-projection (M = columns, N = n_pw) already fills the GPU with output tiles: only
      // small split counts are worth their partial-sum traffic
      for (int sp : {1, 2, 4, 8, 16, 32}) {
        if (which == 1 && sp > 2) break;
        knob = sp;
        double t = 0.0;
        st = measure(&t);
        if (st != DFTCUDA_OK) break;
        if (t < best) {
          best = t;
          pick = sp;
        }
      }
      knob = pick;
    }
  }
  c->prof.on = prof;
  cudaFree(xy);
  if (st != DFTCUDA_OK) return st;
  DFT_TRY(kctx_check_error(c));
  if (report) {
    report->fft_path = c->fft_generic ? 0 : (sticks_avail && !c->sticks_off ? 2 : (fast_avail ? 1 : 0));
    report->box_budget_mb = c->w_budget_bytes / (1024.0 * 1024.0);
    report->proj_splits = c->split_proj;
    report->back_splits = c->split_back;
    report->default_ms = default_ms;
    report->tuned_ms = best;
    report->candidates = evaluated;
  }
  return DFTCUDA_OK;
}
