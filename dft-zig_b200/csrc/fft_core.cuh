// In-place mixed-radix (2, 3, 4, 5) 1D FFTs over lines held in shared memory.
//
// A length n = r_0 r_1 ... r_{s-1} transform runs as s butterfly stages over the whole set of
// lines in shared memory, one __syncthreads() per stage:
//  * DIT (decimation in time) takes its input in digit-reversed order -- element x sits at
//    position pinv[x] -- and leaves the result in natural order.  Stage t (m = r_0..r_{t-1},
//    L = m r_t) combines a_q = base + k + q m as y_q = sum_p (x_p w_L^{pk}) w_r^{pq}.
//  * DIF (decimation in frequency) runs the stages in reverse with the twiddle applied after the
//    r-point DFT; natural-order input, digit-reversed output (X[x] at position pinv[x]).
// The inverse 3D transform uses DIT along every axis (inputs are scattered straight into
// digit-reversed positions) and the forward transform uses DIF (outputs are read back through
// pinv), so no separate permutation pass exists.  sign = +1 is e^{+i} (FFTW_BACKWARD), -1 is
// e^{-i} (FFTW_FORWARD); no 1/N normalisation is applied here.
#pragma once

#include <vector>

#include "common.cuh"

namespace dftcuda {

constexpr int kMaxStages = 8;
constexpr int kMaxFftLen = 128;

// Device view of a 1D plan, passed to kernels by value.
struct Fft1d {
  int n;
  int nstages;
  int radix[kMaxStages];
  int m[kMaxStages];       // product of the radices of earlier stages
  int tw_off[kMaxStages];  // offset of stage t's twiddles: entry k*(r-1) + (p-1) = exp(+2 pi i p k / L)
  const double2* tw64;
  const float2* tw32;
  const int* pinv;  // natural index -> digit-reversed position
};

// Host-owned plan with its device tables.
struct Fft1dPlan {
  Fft1d dev{};
  std::vector<int> radices;
  std::vector<int> pinv;  // host copy
  void* d_buf = nullptr;
  int create(int n);
  void destroy();
};

bool fft_len_supported(int n);

template <typename T> __device__ __forceinline__ cplx<T> tw_load(const Fft1d& p, int i);
template <> __device__ __forceinline__ double2 tw_load<double>(const Fft1d& p, int i) { return __ldg(p.tw64 + i); }
template <> __device__ __forceinline__ float2 tw_load<float>(const Fft1d& p, int i) { return __ldg(p.tw32 + i); }

// r-point DFT in registers, y_q = sum_p x_p exp(sign 2 pi i p q / r).
template <typename T>
__device__ __forceinline__ void dft_small(cplx<T>* x, int r, T sg) {
  using C = cplx<T>;
  if (r == 2) {
    C a = x[0], b = x[1];
    x[0] = cadd(a, b);
    x[1] = csub(a, b);
  } else if (r == 4) {
    C a0 = cadd(x[0], x[2]), a1 = csub(x[0], x[2]);
    C b0 = cadd(x[1], x[3]), b1 = cmuli(csub(x[1], x[3]), sg);
    x[0] = cadd(a0, b0);
    x[2] = csub(a0, b0);
    x[1] = cadd(a1, b1);
    x[3] = csub(a1, b1);
  } else if (r == 3) {
    const T h = (T)0.86602540378443864676;  // sin(2 pi / 3)
    C t = cadd(x[1], x[2]);
    C d = cmuli(csub(x[1], x[2]), sg * h);
    C a = x[0];
    x[0] = cadd(a, t);
    C base = csub(a, cscale(t, (T)0.5));
    x[1] = cadd(base, d);
    x[2] = csub(base, d);
  } else {  // r == 5
    const T c1 = (T)0.30901699437494742410;   // cos(2 pi / 5)
    const T c2 = (T)-0.80901699437494742410;  // cos(4 pi / 5)
    const T s1 = (T)0.95105651629515357212;   // sin(2 pi / 5)
    const T s2 = (T)0.58778525229247312917;   // sin(4 pi / 5)
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

// One butterfly stage over `nlines` lines.  Element e of line l sits at s[l*line_stride + e*elem_stride].
// line_fast selects whether consecutive threads walk lines (for strided elements) or butterflies.
template <typename T, bool DIT>
__device__ __forceinline__ void fft_stage(cplx<T>* s, const Fft1d& p, int t, int elem_stride, int line_stride,
                                          int nlines, T sg, bool line_fast) {
  using C = cplx<T>;
  const int r = p.radix[t];
  const int m = p.m[t];
  const int L = m * r;
  const int nb = p.n / r;
  const int total = nb * nlines;
  const int two = p.tw_off[t];
  for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
    int line, b;
    if (line_fast) {
      b = idx / nlines;
      line = idx - b * nlines;
    } else {
      line = idx / nb;
      b = idx - line * nb;
    }
    const int blk = b / m;
    const int k = b - blk * m;
    C* base = s + line * line_stride + (blk * L + k) * elem_stride;
    const int step = m * elem_stride;
    C x[5];
#pragma unroll
    for (int q = 0; q < 5; ++q)
      if (q < r) x[q] = base[q * step];
    if (DIT) {
      if (k != 0) {
#pragma unroll
        for (int q = 1; q < 5; ++q)
          if (q < r) {
            C w = tw_load<T>(p, two + k * (r - 1) + (q - 1));
            w.y *= sg;
            x[q] = cmul(x[q], w);
          }
      }
      dft_small<T>(x, r, sg);
    } else {
      dft_small<T>(x, r, sg);
      if (k != 0) {
#pragma unroll
        for (int q = 1; q < 5; ++q)
          if (q < r) {
            C w = tw_load<T>(p, two + k * (r - 1) + (q - 1));
            w.y *= sg;
            x[q] = cmul(x[q], w);
          }
      }
    }
#pragma unroll
    for (int q = 0; q < 5; ++q)
      if (q < r) base[q * step] = x[q];
  }
}

// Full 1D transform of every line (DIT: digit-reversed in, natural out; DIF: the converse).
template <typename T, bool DIT>
__device__ __forceinline__ void fft_lines(cplx<T>* s, const Fft1d& p, int elem_stride, int line_stride, int nlines,
                                          T sg, bool line_fast) {
  if (DIT) {
    for (int t = 0; t < p.nstages; ++t) {
      fft_stage<T, true>(s, p, t, elem_stride, line_stride, nlines, sg, line_fast);
      __syncthreads();
    }
  } else {
    for (int t = p.nstages - 1; t >= 0; --t) {
      fft_stage<T, false>(s, p, t, elem_stride, line_stride, nlines, sg, line_fast);
      __syncthreads();
    }
  }
}

}  // namespace dftcuda
