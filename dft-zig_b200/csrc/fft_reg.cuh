// Register-resident FFT building blocks for the fused local-potential passes.
//
// A length N = N1 * N2 line runs as a four-step transform:
//   step A (one thread per t < N2):  a_t[k1] = DFT_N1( x[j*N2 + t] )_j [k1] * w_N^{s t k1}
//   step B (one thread per k1 < N1): X[k1 + N1*k2] = DFT_N2( a_t[k1] )_t [k2]
// with w_N = exp(2 pi i / N) and s = +1 (inverse, FFTW_BACKWARD) or -1 (forward).  Each step's
// sub-DFT lives in registers (RegDft: recursive mixed radix 2/3/4/5 with compile-time indices), so a
// line crosses shared memory once per transform instead of once per radix stage.
//
// Twiddles: the sub-DFTs' internal roots have compile-time indices and are read from constant
// memory (uniform across the warp); the four-step twiddles w_N^{t k1} vary per thread and are read
// from a per-length global table (L1-cached).
#pragma once

#include <cmath>
#include <mutex>
#include <vector>

#include "common.cuh"

namespace dftcuda {

// Roots exp(2 pi i e / L) for the sub-DFT lengths, concatenated: L = 2,3,4,5,6,8,9,10,12,15,16.
constexpr int kRootLens[] = {2, 3, 4, 5, 6, 8, 9, 10, 12, 15, 16};
constexpr int kNumRootLens = sizeof(kRootLens) / sizeof(int);
__host__ __device__ constexpr int root_off(int L) {
  return L == 2 ? 0 : L == 3 ? 2 : L == 4 ? 5 : L == 5 ? 9 : L == 6 ? 14 : L == 8 ? 20 : L == 9 ? 28
       : L == 10 ? 37 : L == 12 ? 47 : L == 15 ? 59 : L == 16 ? 74 : -1;
}
constexpr int kRootTotal = root_off(16) + 16;

// Defined here (not extern): the library is compiled without relocatable device code, so every
// translation unit that includes this header has its own copy of the tables, and must fill it with
// init_root_tables_here() (idempotent per device) before its first kernel that uses RegDft runs.
static __constant__ double2 c_roots64[kRootTotal];
static __constant__ float2 c_roots32[kRootTotal];

// Loads this translation unit's root tables into constant memory on the current device.
static int init_root_tables_here() {
  static std::mutex mu;
  static bool done[128] = {};
  int dev = 0;
  DFT_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 128) return fail(DFTCUDA_ERR_UNSUPPORTED, "device ordinal above 127");
  std::lock_guard<std::mutex> lock(mu);
  if (done[dev]) return DFTCUDA_OK;
  std::vector<double2> r64(kRootTotal);
  std::vector<float2> r32(kRootTotal);
  for (int i = 0; i < kNumRootLens; ++i) {
    const int L = kRootLens[i], off = root_off(L);
    for (int e = 0; e < L; ++e) {
      const double a = 2.0 * M_PI * (double)e / (double)L;
      r64[off + e] = make_double2(std::cos(a), std::sin(a));
      r32[off + e] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
  }
  DFT_CUDA_TRY(cudaMemcpyToSymbol(c_roots64, r64.data(), sizeof(double2) * kRootTotal));
  DFT_CUDA_TRY(cudaMemcpyToSymbol(c_roots32, r32.data(), sizeof(float2) * kRootTotal));
  DFT_CUDA_TRY(cudaDeviceSynchronize());
  done[dev] = true;
  return DFTCUDA_OK;
}

template <typename T> __device__ __forceinline__ cplx<T> root(int idx);
template <> __device__ __forceinline__ double2 root<double>(int idx) { return c_roots64[idx]; }
template <> __device__ __forceinline__ float2 root<float>(int idx) { return c_roots32[idx]; }

template <int L> struct RadixOf {
  static constexpr int value = (L % 4 == 0 && L != 8) ? 4 : (L % 2 == 0) ? 2 : (L % 3 == 0) ? 3 : 5;
};

// r-point DFT (r = 2, 3, 4, 5) on a register array, y_q = sum_p x_p exp(s 2 pi i p q / r).
template <typename T, int R>
__device__ __forceinline__ void butterfly(cplx<T>* x, T sg) {
  using C = cplx<T>;
  if (R == 2) {
    C a = x[0], b = x[1];
    x[0] = cadd(a, b);
    x[1] = csub(a, b);
  } else if (R == 4) {
    C a0 = cadd(x[0], x[2]), a1 = csub(x[0], x[2]);
    C b0 = cadd(x[1], x[3]), b1 = cmuli(csub(x[1], x[3]), sg);
    x[0] = cadd(a0, b0);
    x[2] = csub(a0, b0);
    x[1] = cadd(a1, b1);
    x[3] = csub(a1, b1);
  } else if (R == 3) {
    const T h = (T)0.86602540378443864676;
    C t = cadd(x[1], x[2]);
    C d = cmuli(csub(x[1], x[2]), sg * h);
    C a = x[0];
    x[0] = cadd(a, t);
    C base = csub(a, cscale(t, (T)0.5));
    x[1] = cadd(base, d);
    x[2] = csub(base, d);
  } else {
    const T c1 = (T)0.30901699437494742410, c2 = (T)-0.80901699437494742410;
    const T s1 = (T)0.95105651629515357212, s2 = (T)0.58778525229247312917;
    C t1 = cadd(x[1], x[4]), t2 = cadd(x[2], x[3]);
    C t3 = csub(x[1], x[4]), t4 = csub(x[2], x[3]);
    C x0 = x[0];
    C a1 = cadd(x0, cadd(cscale(t1, c1), cscale(t2, c2)));
    C a2 = cadd(x0, cadd(cscale(t1, c2), cscale(t2, c1)));
    C b1 = cmuli(cadd(cscale(t3, s1), cscale(t4, s2)), sg);
    C b2 = cmuli(csub(cscale(t3, s2), cscale(t4, s1)), sg);
    x[0] = cadd(x0, cadd(t1, t2));
    x[1] = cadd(a1, b1);
    x[4] = csub(a1, b1);
    x[2] = cadd(a2, b2);
    x[3] = csub(a2, b2);
  }
}

// In-place natural-order DFT of length L on a register array (all indices compile-time).
template <typename T, int L>
struct RegDft {
  using C = cplx<T>;
  static __device__ __forceinline__ void run(C* x, T sg) {
    constexpr int R = RadixOf<L>::value;
    constexpr int M = L / R;
    if constexpr (M == 1) {
      butterfly<T, R>(x, sg);
      return;
    } else {
    C sub[R][M];
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int m = 0; m < M; ++m) sub[r][m] = x[m * R + r];
#pragma unroll
    for (int r = 0; r < R; ++r) RegDft<T, M>::run(sub[r], sg);
    constexpr int off = root_off(L);
#pragma unroll
    for (int k = 0; k < M; ++k) {
      C t[R];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        if (r == 0 || k == 0) {
          t[r] = sub[r][k];
        } else {
          C w = root<T>(off + (r * k) % L);
          w.y *= sg;
          t[r] = cmul(sub[r][k], w);
        }
      }
      butterfly<T, R>(t, sg);
#pragma unroll
      for (int q = 0; q < R; ++q) x[k + M * q] = t[q];
    }
    }
  }
};
template <typename T>
struct RegDft<T, 1> {
  static __device__ __forceinline__ void run(cplx<T>*, T) {}
};

// Factorisation N = N1 * N2 used by the four-step kernels (N1 >= N2, both <= 16).
template <int N> struct Split;
#define DFTCUDA_SPLIT(N, A, B) \
  template <> struct Split<N> { static constexpr int N1 = A, N2 = B; };
DFTCUDA_SPLIT(20, 5, 4)
DFTCUDA_SPLIT(24, 6, 4)
DFTCUDA_SPLIT(27, 9, 3)
DFTCUDA_SPLIT(30, 6, 5)
DFTCUDA_SPLIT(32, 8, 4)
DFTCUDA_SPLIT(36, 6, 6)
DFTCUDA_SPLIT(40, 8, 5)
DFTCUDA_SPLIT(45, 9, 5)
DFTCUDA_SPLIT(48, 8, 6)
DFTCUDA_SPLIT(60, 12, 5)
DFTCUDA_SPLIT(64, 8, 8)
DFTCUDA_SPLIT(72, 9, 8)
DFTCUDA_SPLIT(75, 15, 5)
DFTCUDA_SPLIT(80, 10, 8)
DFTCUDA_SPLIT(90, 10, 9)
DFTCUDA_SPLIT(96, 12, 8)
DFTCUDA_SPLIT(100, 10, 10)
DFTCUDA_SPLIT(108, 12, 9)
DFTCUDA_SPLIT(120, 12, 10)
DFTCUDA_SPLIT(128, 16, 8)
#undef DFTCUDA_SPLIT

// Lengths with a four-step kernel (keep in sync with the Split table and the dispatch switches).
#define DFTCUDA_FOUR_STEP_LENGTHS(X) \
  X(20) X(24) X(27) X(30) X(32) X(36) X(40) X(45) X(48) X(60) X(64) X(72) X(75) X(80) X(90) X(96) X(100) X(108) X(120) X(128)

bool four_step_supported(int n);

}  // namespace dftcuda
