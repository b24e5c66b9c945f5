// FP64 complex GEMM over strided operands, used for the Kleinman-Bylander projections
// (apply.zig:1143-1183, 1278-1336) and the Rayleigh-Ritz contractions V^H W and V C
// (lobpcg/common.zig:113-143, 231-259).  B200 has no FP64 tcgen05 kind, so the FP64 path runs on
// the FP64 tensor cores through mma.sync m8n8k4 .f64 with three real products per complex one
// (k_zgemm_dmma3m, the default: the FP64 MMA pipe is the bound, and it does a quarter less work),
// with the plain four products (k_zgemm_dmma, DFTCUDA_ZGEMM=dmma8) or on the m16n8k8 shape
// (k_zgemm_dmma16, DFTCUDA_ZGEMM=dmma16: the same throughput as m8n8k4), or on the FP64 FMA pipe
// (k_zgemm, DFTCUDA_ZGEMM=fma):
// 64x64 output tiles per 256-thread CTA, K staged through
// shared memory in slices of 16 with cp.async double buffering, and split-K with a deterministic
// second-pass reduction when the output has too few tiles to fill the 148 SMs.
#include <algorithm>
#include <cstdlib>
#include <string>

#include "kctx.cuh"

namespace dftcuda {

constexpr int BM = 64, BN = 64, BK = 16;

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool pred) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int sz = pred ? 16 : 0;  // 0 source bytes: the 16 destination bytes are zero-filled
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::); }

// One BK-deep slice of A and B into shared memory with cp.async (4 x 16 B per thread each).
template <bool AKC, bool BKC, int PAD = 1>
__device__ __forceinline__ void zgemm_fetch(double2 (*As)[BM + PAD], double2 (*Bs)[BN + PAD], int M, int N, int kend, int r0,
                                            int c0, int k0, const double2* __restrict__ A, long lda,
                                            const double2* __restrict__ B, long ldb, int tid) {
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int i = tid + 256 * q;
    int r, kk;
    if (AKC) { kk = i % BK; r = i / BK; } else { r = i % BM; kk = i / BM; }
    const int gr = r0 + r, gk = k0 + kk;
    const bool ok = gr < M && gk < kend;
    const double2* src = ok ? (AKC ? A + (long)gr * lda + gk : A + (long)gk * lda + gr) : A;
    cp_async16(&As[kk][r], src, ok);
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int i = tid + 256 * q;
    int cc, kk;
    if (BKC) { kk = i % BK; cc = i / BK; } else { cc = i % BN; kk = i / BN; }
    const int gc = c0 + cc, gk = k0 + kk;
    const bool ok = gc < N && gk < kend;
    const double2* src = ok ? (BKC ? B + (long)gc * ldb + gk : B + (long)gk * ldb + gc) : B;
    cp_async16(&Bs[kk][cc], src, ok);
  }
  cp_async_commit();
}

// Double-buffered: the next K slice streams into the other shared-memory buffer with cp.async
// while the current one is multiplied; conjugation is applied as the operands leave shared memory.
// At most 128 registers per thread so two CTAs share an SM.
template <bool AKC, bool BKC, bool CJA, bool CJB>
__global__ void __launch_bounds__(256, 2) k_zgemm(int M, int N, int K, const double2* __restrict__ A, long lda,
                                                  const double2* __restrict__ B, long ldb, double2* __restrict__ O,
                                                  long ldo_r, long ldo_c, double alpha, double beta, int kps,
                                                  double2* __restrict__ part) {
  extern __shared__ __align__(16) unsigned char zsm[];
  double2(*As)[BK][BM + 1] = reinterpret_cast<double2(*)[BK][BM + 1]>(zsm);
  double2(*Bs)[BK][BN + 1] = reinterpret_cast<double2(*)[BK][BN + 1]>(zsm + 2 * sizeof(double2) * BK * (BM + 1));
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;
  const int r0 = blockIdx.y * BM, c0 = blockIdx.x * BN;
  const int kbeg = blockIdx.z * kps;
  const int kend = min(K, kbeg + kps);
  const double sa = CJA ? -1.0 : 1.0, sb = CJB ? -1.0 : 1.0;
  double2 acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = make_double2(0.0, 0.0);
  if (kbeg < kend) zgemm_fetch<AKC, BKC>(As[0], Bs[0], M, N, kend, r0, c0, kbeg, A, lda, B, ldb, tid);
  int buf = 0;
  for (int k0 = kbeg; k0 < kend; k0 += BK) {
    cp_async_wait_all();
    __syncthreads();
    if (k0 + BK < kend) zgemm_fetch<AKC, BKC>(As[buf ^ 1], Bs[buf ^ 1], M, N, kend, r0, c0, k0 + BK, A, lda, B, ldb, tid);
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      double2 a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        a[i] = As[buf][kk][ty + 16 * i];
        a[i].y *= sa;
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        b[j] = Bs[buf][kk][tx + 16 * j];
        b[j].y *= sb;
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          acc[i][j].x = fma(a[i].x, b[j].x, acc[i][j].x);
          acc[i][j].x = fma(-a[i].y, b[j].y, acc[i][j].x);
          acc[i][j].y = fma(a[i].x, b[j].y, acc[i][j].y);
          acc[i][j].y = fma(a[i].y, b[j].x, acc[i][j].y);
        }
    }
    buf ^= 1;
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int r = r0 + ty + 16 * i, c = c0 + tx + 16 * j;
      if (r >= M || c >= N) continue;
      if (part) {
        part[((long)blockIdx.z * M + r) * N + c] = acc[i][j];
      } else {
        double2* o = O + (long)r * ldo_r + (long)c * ldo_c;
        double2 v;
        v.x = alpha * acc[i][j].x;
        v.y = alpha * acc[i][j].y;
        if (beta != 0.0) {
          const double2 old = *o;
          v.x += beta * old.x;
          v.y += beta * old.y;
        }
        *o = v;
      }
    }
}

static const size_t kZgemmSmem = 2 * sizeof(double2) * BK * (BM + 1) + 2 * sizeof(double2) * BK * (BN + 1);

// The same contraction on the FP64 tensor cores (mma.sync m8n8k4 .f64; tcgen05 has no f64 kind):
// one warp instruction is 256 FMAs instead of 32, which relieves the issue pressure of the FMA
// kernel above.  Fragments of mma.m8n8k4.row.col.f64, lane = 4 g + t:
//   A (8 x 4): A[g][t];  B (4 x 8): B[t][g];  C (8 x 8): C[g][2t], C[g][2t + 1].
// The 8 warps tile the 64 x 64 output as 4 x 2 blocks of 16 x 32 (2 x 4 tiles of 8 x 8); a complex
// product is four real MMAs (the negated imaginary A fragment gives -Ai Bi).  Shared memory holds
// the slices as [k][row] complex with a row stride of 66: the 8 lanes of a 16-byte load phase
// (g in {0,1}, t in 0..3) then fall on 8 distinct 16-byte bank groups.
constexpr int kZmPad = 2;
static const size_t kZgemmDmmaSmem = 2 * sizeof(double2) * BK * (BM + kZmPad) + 2 * sizeof(double2) * BK * (BN + kZmPad);

__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

template <bool AKC, bool BKC, bool CJA, bool CJB>
__global__ void __launch_bounds__(256, 2) k_zgemm_dmma(int M, int N, int K, const double2* __restrict__ A, long lda,
                                                       const double2* __restrict__ B, long ldb, double2* __restrict__ O,
                                                       long ldo_r, long ldo_c, double alpha, double beta, int kps,
                                                       double2* __restrict__ part) {
  extern __shared__ __align__(16) unsigned char zsm[];
  double2(*As)[BK][BM + kZmPad] = reinterpret_cast<double2(*)[BK][BM + kZmPad]>(zsm);
  double2(*Bs)[BK][BN + kZmPad] = reinterpret_cast<double2(*)[BK][BN + kZmPad]>(zsm + 2 * sizeof(double2) * BK * (BM + kZmPad));
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wr = warp >> 1, wc = warp & 1;  // warp block: rows 16 wr .., columns 32 wc ..
  const int r0 = blockIdx.y * BM, c0 = blockIdx.x * BN;
  const int kbeg = blockIdx.z * kps;
  const int kend = min(K, kbeg + kps);
  const double sa = CJA ? -1.0 : 1.0, sb = CJB ? -1.0 : 1.0;
  double cre[2][4][2], cim[2][4][2];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) cre[i][j][0] = cre[i][j][1] = cim[i][j][0] = cim[i][j][1] = 0.0;
  if (kbeg < kend) zgemm_fetch<AKC, BKC, kZmPad>(As[0], Bs[0], M, N, kend, r0, c0, kbeg, A, lda, B, ldb, tid);
  int buf = 0;
  for (int k0 = kbeg; k0 < kend; k0 += BK) {
    cp_async_wait_all();
    __syncthreads();
    if (k0 + BK < kend) zgemm_fetch<AKC, BKC, kZmPad>(As[buf ^ 1], Bs[buf ^ 1], M, N, kend, r0, c0, k0 + BK, A, lda, B, ldb, tid);
#pragma unroll
    for (int k4 = 0; k4 < BK; k4 += 4) {
      double ar[2], ai[2], nai[2], br[4], bi[4];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const double2 v = As[buf][k4 + t][wr * 16 + i * 8 + g];
        ar[i] = v.x;
        ai[i] = sa * v.y;
        nai[i] = -ai[i];
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const double2 v = Bs[buf][k4 + t][wc * 32 + j * 8 + g];
        br[j] = v.x;
        bi[j] = sb * v.y;
      }
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          dmma(cre[i][j][0], cre[i][j][1], ar[i], br[j]);
          dmma(cre[i][j][0], cre[i][j][1], nai[i], bi[j]);
          dmma(cim[i][j][0], cim[i][j][1], ar[i], bi[j]);
          dmma(cim[i][j][0], cim[i][j][1], ai[i], br[j]);
        }
    }
    buf ^= 1;
  }
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int r = r0 + wr * 16 + i * 8 + g, c = c0 + wc * 32 + j * 8 + 2 * t + h;
        if (r >= M || c >= N) continue;
        const double2 acc = make_double2(cre[i][j][h], cim[i][j][h]);
        if (part) {
          part[((long)blockIdx.z * M + r) * N + c] = acc;
        } else {
          double2* o = O + (long)r * ldo_r + (long)c * ldo_c;
          double2 v = make_double2(alpha * acc.x, alpha * acc.y);
          if (beta != 0.0) {
            const double2 old = *o;
            v.x += beta * old.x;
            v.y += beta * old.y;
          }
          *o = v;
        }
      }
}

// The same tiling on the m16n8k8 FP64 MMA (one instruction = 1,024 FMAs, four times the m8n8k4's,
// for the same operands).  Fragments of mma.m16n8k8.row.col.f64, lane = 4 g + t:
//   A (16 x 8): a0 = A[g][t], a1 = A[g + 8][t], a2 = A[g][t + 4], a3 = A[g + 8][t + 4];
//   B (8 x 8):  b0 = B[t][g], b1 = B[t + 4][g];
//   C (16 x 8): c0 = C[g][2t], c1 = C[g][2t + 1], c2 = C[g + 8][2t], c3 = C[g + 8][2t + 1].
// Each warp owns 16 x 32 outputs (four 16 x 8 tiles); a complex product is four real MMAs.
__device__ __forceinline__ void dmma16(double (&c)[4], const double (&a)[4], double b0, double b1) {
  asm volatile("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
               : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
               : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b0), "d"(b1));
}

template <bool AKC, bool BKC, bool CJA, bool CJB>
__global__ void __launch_bounds__(256, 2) k_zgemm_dmma16(int M, int N, int K, const double2* __restrict__ A, long lda,
                                                         const double2* __restrict__ B, long ldb, double2* __restrict__ O,
                                                         long ldo_r, long ldo_c, double alpha, double beta, int kps,
                                                         double2* __restrict__ part) {
  extern __shared__ __align__(16) unsigned char zsm[];
  double2(*As)[BK][BM + kZmPad] = reinterpret_cast<double2(*)[BK][BM + kZmPad]>(zsm);
  double2(*Bs)[BK][BN + kZmPad] = reinterpret_cast<double2(*)[BK][BN + kZmPad]>(zsm + 2 * sizeof(double2) * BK * (BM + kZmPad));
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wr = warp >> 1, wc = warp & 1;  // warp block: rows 16 wr .., columns 32 wc ..
  const int r0 = blockIdx.y * BM, c0 = blockIdx.x * BN;
  const int kbeg = blockIdx.z * kps;
  const int kend = min(K, kbeg + kps);
  const double sa = CJA ? -1.0 : 1.0, sb = CJB ? -1.0 : 1.0;
  double cre[4][4], cim[4][4];
#pragma unroll
  for (int j = 0; j < 4; ++j)
#pragma unroll
    for (int e = 0; e < 4; ++e) cre[j][e] = cim[j][e] = 0.0;
  if (kbeg < kend) zgemm_fetch<AKC, BKC, kZmPad>(As[0], Bs[0], M, N, kend, r0, c0, kbeg, A, lda, B, ldb, tid);
  int buf = 0;
  for (int k0 = kbeg; k0 < kend; k0 += BK) {
    cp_async_wait_all();
    __syncthreads();
    if (k0 + BK < kend) zgemm_fetch<AKC, BKC, kZmPad>(As[buf ^ 1], Bs[buf ^ 1], M, N, kend, r0, c0, k0 + BK, A, lda, B, ldb, tid);
#pragma unroll
    for (int k8 = 0; k8 < BK; k8 += 8) {
      double ar[4], ai[4], nai[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const double2 v = As[buf][k8 + t + 4 * (e >> 1)][wr * 16 + g + 8 * (e & 1)];
        ar[e] = v.x;
        ai[e] = sa * v.y;
        nai[e] = -ai[e];
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const double2 u0 = Bs[buf][k8 + t][wc * 32 + j * 8 + g];
        const double2 u1 = Bs[buf][k8 + t + 4][wc * 32 + j * 8 + g];
        const double bi0 = sb * u0.y, bi1 = sb * u1.y;
        dmma16(cre[j], ar, u0.x, u1.x);
        dmma16(cre[j], nai, bi0, bi1);
        dmma16(cim[j], ar, bi0, bi1);
        dmma16(cim[j], ai, u0.x, u1.x);
      }
    }
    buf ^= 1;
  }
#pragma unroll
  for (int j = 0; j < 4; ++j)
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int r = r0 + wr * 16 + g + 8 * (e >> 1), c = c0 + wc * 32 + j * 8 + 2 * t + (e & 1);
      if (r >= M || c >= N) continue;
      const double2 acc = make_double2(cre[j][e], cim[j][e]);
      if (part) {
        part[((long)blockIdx.z * M + r) * N + c] = acc;
      } else {
        double2* o = O + (long)r * ldo_r + (long)c * ldo_c;
        double2 v = make_double2(alpha * acc.x, alpha * acc.y);
        if (beta != 0.0) {
          const double2 old = *o;
          v.x += beta * old.x;
          v.y += beta * old.y;
        }
        *o = v;
      }
    }
}

// Three real MMAs per complex product (Gauss): with a = ar + i ai, b = br + i bi,
//   T1 = ar (br + bi),  T2 = (ar + ai) bi,  T3 = (ai - ar) br;   Re = T1 - T2,  Im = T1 + T3.
// The m8n8k4 kernel's tiling and fragments with a third accumulator per 8 x 8 tile: a quarter
// fewer FP64 MMAs, the FP64 tensor pipe being the bound of the four-product form.
template <bool AKC, bool BKC, bool CJA, bool CJB>
__global__ void __launch_bounds__(256, 2) k_zgemm_dmma3m(int M, int N, int K, const double2* __restrict__ A, long lda,
                                                         const double2* __restrict__ B, long ldb, double2* __restrict__ O,
                                                         long ldo_r, long ldo_c, double alpha, double beta, int kps,
                                                         double2* __restrict__ part) {
  extern __shared__ __align__(16) unsigned char zsm[];
  double2(*As)[BK][BM + kZmPad] = reinterpret_cast<double2(*)[BK][BM + kZmPad]>(zsm);
  double2(*Bs)[BK][BN + kZmPad] = reinterpret_cast<double2(*)[BK][BN + kZmPad]>(zsm + 2 * sizeof(double2) * BK * (BM + kZmPad));
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wr = warp >> 1, wc = warp & 1;
  const int r0 = blockIdx.y * BM, c0 = blockIdx.x * BN;
  const int kbeg = blockIdx.z * kps;
  const int kend = min(K, kbeg + kps);
  const double sa = CJA ? -1.0 : 1.0, sb = CJB ? -1.0 : 1.0;
  double t1[2][4][2], t2[2][4][2], t3[2][4][2];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) t1[i][j][h] = t2[i][j][h] = t3[i][j][h] = 0.0;
  if (kbeg < kend) zgemm_fetch<AKC, BKC, kZmPad>(As[0], Bs[0], M, N, kend, r0, c0, kbeg, A, lda, B, ldb, tid);
  int buf = 0;
  for (int k0 = kbeg; k0 < kend; k0 += BK) {
    cp_async_wait_all();
    __syncthreads();
    if (k0 + BK < kend) zgemm_fetch<AKC, BKC, kZmPad>(As[buf ^ 1], Bs[buf ^ 1], M, N, kend, r0, c0, k0 + BK, A, lda, B, ldb, tid);
#pragma unroll
    for (int k4 = 0; k4 < BK; k4 += 4) {
      double ar[2], as_[2], ad[2], bs[4], bi[4], br[4];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const double2 v = As[buf][k4 + t][wr * 16 + i * 8 + g];
        const double ai = sa * v.y;
        ar[i] = v.x;
        as_[i] = v.x + ai;
        ad[i] = ai - v.x;
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const double2 v = Bs[buf][k4 + t][wc * 32 + j * 8 + g];
        br[j] = v.x;
        bi[j] = sb * v.y;
        bs[j] = v.x + bi[j];
      }
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          dmma(t1[i][j][0], t1[i][j][1], ar[i], bs[j]);
          dmma(t2[i][j][0], t2[i][j][1], as_[i], bi[j]);
          dmma(t3[i][j][0], t3[i][j][1], ad[i], br[j]);
        }
    }
    buf ^= 1;
  }
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int r = r0 + wr * 16 + i * 8 + g, c = c0 + wc * 32 + j * 8 + 2 * t + h;
        if (r >= M || c >= N) continue;
        const double2 acc = make_double2(t1[i][j][h] - t2[i][j][h], t1[i][j][h] + t3[i][j][h]);
        if (part) {
          part[((long)blockIdx.z * M + r) * N + c] = acc;
        } else {
          double2* o = O + (long)r * ldo_r + (long)c * ldo_c;
          double2 v = make_double2(alpha * acc.x, alpha * acc.y);
          if (beta != 0.0) {
            const double2 old = *o;
            v.x += beta * old.x;
            v.y += beta * old.y;
          }
          *o = v;
        }
      }
}

__global__ void k_zgemm_reduce(int M, int N, int splits, const double2* __restrict__ part, double2* __restrict__ O,
                               long ldo_r, long ldo_c, double alpha, double beta) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= (long)M * N) return;
  const int r = (int)(i / N), c = (int)(i - (long)r * N);
  double2 s = make_double2(0.0, 0.0);
  for (int z = 0; z < splits; ++z) {
    const double2 v = part[(long)z * M * N + i];
    s.x += v.x;
    s.y += v.y;
  }
  double2* o = O + (long)r * ldo_r + (long)c * ldo_c;
  double2 v = make_double2(alpha * s.x, alpha * s.y);
  if (beta != 0.0) {
    const double2 old = *o;
    v.x += beta * old.x;
    v.y += beta * old.y;
  }
  *o = v;
}

// Split K so that tiles x splits fills whole waves of 2 CTAs per SM on 148 SMs.
static int pick_splits(int M, int N, int K) {
  const long tiles = (long)ceil_div(M, BM) * ceil_div(N, BN);
  const long wave = 2 * 148;
  if (tiles >= wave || K < 4 * BK * 8) return 1;
  const long maxs = std::max<long>(1, K / (BK * 8));  // at least 8 K slices per split
  long best = 1;
  double best_eff = 0.0;
  for (long sp = 1; sp <= std::min<long>(maxs, 64); ++sp) {
    const long ctas = tiles * sp;
    const double eff = (double)ctas / (double)(((ctas + wave - 1) / wave) * wave);  // wave fill
    const double score = eff * std::min(1.0, (double)ctas / wave);
    if (score > best_eff + 1e-9) {
      best_eff = score;
      best = sp;
    }
  }
  return (int)best;
}

size_t zgemm_workspace_elems(int M, int N, int K) {
  const int s = pick_splits(M, N, K);
  return s > 1 ? (size_t)s * M * N : 0;
}

// DFTCUDA_ZGEMM=fma / dmma8 / dmma16 select the other kernels (A/B measurements); the
// three-product m8n8k4 kernel is the default.
static int zgemm_kind() {
  static const int v = [] {
    const char* e = std::getenv("DFTCUDA_ZGEMM");
    if (e && std::string(e) == "fma") return 0;
    if (e && std::string(e) == "dmma8") return 1;
    if (e && std::string(e) == "dmma16") return 2;
    return 3;
  }();
  return v;
}

template <bool AKC, bool BKC, bool CJA, bool CJB>
static void launch(const GemmArgs& g, dim3 grid, int kps, double2* part, cudaStream_t s) {
  if (zgemm_kind() == 3) {
    ensure_max_dynamic_smem((const void*)k_zgemm_dmma3m<AKC, BKC, CJA, CJB>, (int)kZgemmDmmaSmem);
    k_zgemm_dmma3m<AKC, BKC, CJA, CJB><<<grid, 256, kZgemmDmmaSmem, s>>>(g.M, g.N, g.K, g.A, g.lda, g.B, g.ldb, g.O, g.ldo_r,
                                                                        g.ldo_c, g.alpha, g.beta, kps, part);
    count_launch();
    return;
  }
  if (zgemm_kind() == 2) {
    ensure_max_dynamic_smem((const void*)k_zgemm_dmma16<AKC, BKC, CJA, CJB>, (int)kZgemmDmmaSmem);
    k_zgemm_dmma16<AKC, BKC, CJA, CJB><<<grid, 256, kZgemmDmmaSmem, s>>>(g.M, g.N, g.K, g.A, g.lda, g.B, g.ldb, g.O, g.ldo_r,
                                                                        g.ldo_c, g.alpha, g.beta, kps, part);
    count_launch();
    return;
  }
  if (zgemm_kind() == 1) {
    ensure_max_dynamic_smem((const void*)k_zgemm_dmma<AKC, BKC, CJA, CJB>, (int)kZgemmDmmaSmem);
    k_zgemm_dmma<AKC, BKC, CJA, CJB><<<grid, 256, kZgemmDmmaSmem, s>>>(g.M, g.N, g.K, g.A, g.lda, g.B, g.ldb, g.O, g.ldo_r,
                                                                      g.ldo_c, g.alpha, g.beta, kps, part);
    count_launch();
    return;
  }
  ensure_max_dynamic_smem((const void*)k_zgemm<AKC, BKC, CJA, CJB>, (int)kZgemmSmem);
  k_zgemm<AKC, BKC, CJA, CJB><<<grid, 256, kZgemmSmem, s>>>(g.M, g.N, g.K, g.A, g.lda, g.B, g.ldb, g.O, g.ldo_r, g.ldo_c, g.alpha,
                                                   g.beta, kps, part); count_launch();
}

int zgemm(const GemmArgs& g, cudaStream_t s, double2* ws, size_t ws_elems) {
  if (g.M <= 0 || g.N <= 0) return DFTCUDA_OK;
  if (g.K <= 0) {
    // out = beta * out
    return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "zgemm: K must be positive");
  }
  int splits = g.splits > 0 ? std::min(g.splits, std::max(1, g.K / 32)) : pick_splits(g.M, g.N, g.K);
  if (splits > 1) splits = (int)std::max<size_t>(1, std::min<size_t>(splits, ws_elems / ((size_t)g.M * g.N)));  // what fits the workspace
  int kps = (g.K + splits - 1) / splits;
  kps = ((kps + BK - 1) / BK) * BK;
  splits = (g.K + kps - 1) / kps;
  dim3 grid(ceil_div(g.N, BN), ceil_div(g.M, BM), splits);
  double2* part = splits > 1 ? ws : nullptr;
  const int key = (g.a_kc ? 8 : 0) | (g.b_kc ? 4 : 0) | (g.conj_a ? 2 : 0) | (g.conj_b ? 1 : 0);
  switch (key) {
    case 0: launch<false, false, false, false>(g, grid, kps, part, s); break;
    case 1: launch<false, false, false, true>(g, grid, kps, part, s); break;
    case 2: launch<false, false, true, false>(g, grid, kps, part, s); break;
    case 3: launch<false, false, true, true>(g, grid, kps, part, s); break;
    case 4: launch<false, true, false, false>(g, grid, kps, part, s); break;
    case 5: launch<false, true, false, true>(g, grid, kps, part, s); break;
    case 6: launch<false, true, true, false>(g, grid, kps, part, s); break;
    case 7: launch<false, true, true, true>(g, grid, kps, part, s); break;
    case 8: launch<true, false, false, false>(g, grid, kps, part, s); break;
    case 9: launch<true, false, false, true>(g, grid, kps, part, s); break;
    case 10: launch<true, false, true, false>(g, grid, kps, part, s); break;
    case 11: launch<true, false, true, true>(g, grid, kps, part, s); break;
    case 12: launch<true, true, false, false>(g, grid, kps, part, s); break;
    case 13: launch<true, true, false, true>(g, grid, kps, part, s); break;
    case 14: launch<true, true, true, false>(g, grid, kps, part, s); break;
    default: launch<true, true, true, true>(g, grid, kps, part, s); break;
  }
  if (part) {
    const long tot = (long)g.M * g.N;
    k_zgemm_reduce<<<ceil_div(tot, 256), 256, 0, s>>>(g.M, g.N, splits, part, g.O, g.ldo_r, g.ldo_c, g.alpha, g.beta); count_launch();
  }
  DFT_CUDA_TRY(cudaGetLastError());
  return DFTCUDA_OK;
}

}  // namespace dftcuda
