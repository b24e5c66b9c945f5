// Hermitian eigensolver for the Rayleigh-Ritz subspace problem: the zheev('V','U') calls of
// lobpcg/common.zig:440-537 and linalg/linalg.zig:141-151, restricted to the lowest nev eigenpairs
// (the Davidson loop reads only the first nbands, lobpcg/serial.zig:196-227).  FP64 throughout,
// m <= 2048:
//   1. Householder reduction to real symmetric tridiagonal form Q^H A Q = T, reflectors chosen as
//      in LAPACK's zlarfg so the off-diagonal of T is real.  One cooperative launch; the matrix
//      stays in L2 (m = 2048: 64 MB) and each column costs one grid barrier (bounded waits): the
//      rank-2 update of step k and the matrix-vector product of step k+1 share one sweep.
//   2. The nev lowest eigenvalues of T by Sturm-count multisection: one warp per eigenvalue, its
//      32 lanes evaluate the count at 32 interior points, so the bracket shrinks 33x per round.
//   3. Eigenvectors of T by inverse iteration on a row-pivoted LU of T - lambda I (three sweeps
//      from a hashed start vector), one warp per group of eigenvalues closer than 1e-5 ||T||: its
//      vectors are computed in order, re-orthogonalised (modified Gram-Schmidt, all lanes) after
//      each solve; one lane runs the recurrences out of shared memory.
//   4. Back-transformation E = H_0 H_1 ... H_{m-2} Z with the stored reflectors.  Small problems:
//      one warp per eigenvector, the vector held in shared memory.  From m = 192 and nev = 32 on:
//      blocks of 64 reflectors in compact WY form (I - V T V^H, as LAPACK's zlarft/zlarfb), each
//      block applied to all eigenvectors at once by three complex GEMMs.
#include <cfloat>
#include <cmath>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>

#include "kctx.cuh"

namespace dftcuda {

namespace {

constexpr int HT_THREADS = 512;              // tridiagonalisation block
constexpr int HT_WARPS = HT_THREADS / 32;
constexpr int BS_WARPS = 8;                  // bisection: eigenvalues per block
constexpr int BT_WARPS = 4;                  // back-transformation: eigenvectors per block
constexpr long kBarrierSpin = 1L << 24;      // polls (with 32 ns sleeps) before a barrier gives up
constexpr double kGroupTol = 1e-5;           // eigenvalue grouping, relative to ||T||
constexpr int kHtMaxSplit = 8;               // warps per trailing column (row chunks)
constexpr int kHtColRegs = 4;                // column entries per thread (m <= 4 HT_THREADS)
static_assert(kHtColRegs * HT_THREADS >= 2048, "k_hetrd1 holds a column of up to 2047 entries in registers");
constexpr int kIvChunk = 8;                  // inverse iteration: entries loaded ahead per sweep step

struct GridBarrier {
  unsigned* count;  // arrivals since the launch (zeroed by the host)
  int* err;
  unsigned nblocks;
  long spin = kBarrierSpin;  // polls before a wait gives up
  unsigned extra = 0;        // arrivals added to every target (failure injection: 1 = never reached)
};

// All blocks of the (co-resident, cooperative) grid meet here.  The arrival counter only grows
// (reset by the host before the launch): the t-th barrier is passed once it reaches t * nblocks, so
// arriving is one atomic and waiting one acquire-load poll.  Returns false for every thread of a
// block whose wait gave up (the error flag is then set); a block that gives up returns, and the
// others give up at their next barrier, which it never reaches.
__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ bool grid_sync(const GridBarrier& b, unsigned& epoch) {
  __shared__ int s_ok;
  __syncthreads();
  ++epoch;
  if (threadIdx.x == 0) {
    int ok = 1;
    const unsigned target = epoch * b.nblocks + b.extra;
    __threadfence();
    atomicAdd(b.count, 1u);
    long it = 0;
    while (ld_acquire_gpu(b.count) < target) {
      if (++it > b.spin) {
        atomicExch(b.err, kBarrierTimeoutFlag);
        ok = 0;
        break;
      }
      __nanosleep(32);
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sum over the block (HT_THREADS threads), returned to every thread.
__device__ double2 block_sum2(double2 v, double2* red) {
  v.x = warp_sum(v.x);
  v.y = warp_sum(v.y);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double2 t = make_double2(0.0, 0.0);
  for (int i = 0; i < HT_WARPS; ++i) {
    t.x += red[i].x;
    t.y += red[i].y;
  }
  return t;
}

// Step 1.  A: m x m Hermitian, column-major, both triangles.  Column k of the result holds the
// reflector v_k below the subdiagonal (v_k[0] = 1 implied at row k+1); d, e: T's diagonal and
// (real) subdiagonal; tau[k]: H_k = I - tau_k v_k v_k^H with H_k^H A[k+1:, k] = e_k e_1.
// The grid's warps cover the (column, row chunk) pairs of the trailing matrix.
__global__ void __launch_bounds__(HT_THREADS) k_hetrd(double2* __restrict__ A, int m, double* __restrict__ dd,
                                                      double* __restrict__ ee, double2* __restrict__ tau,
                                                      double2* __restrict__ y, GridBarrier bar) {
  extern __shared__ double2 hsm[];
  double2* sv = hsm;      // v_k, m - k - 1 entries
  double2* sw = hsm + m;  // w = tau A v + alpha v
  __shared__ double2 red[HT_WARPS];
  const int tid = threadIdx.x, lane = tid & 31;
  const int gw = blockIdx.x * HT_WARPS + (tid >> 5);
  const int W = gridDim.x * HT_WARPS;
  unsigned epoch = 0;
  for (int k = 0; k + 1 < m; ++k) {
    const int n1 = m - k - 1;
    const double2* col = A + (long)k * m + (k + 1);
    // Phase A (every block): the reflector of column k.
    double2 part = make_double2(0.0, 0.0);
    for (int i = tid; i < n1; i += HT_THREADS) {
      const double2 x = __ldcg(col + i);
      sv[i] = x;
      if (i > 0) part.x += x.x * x.x + x.y * x.y;
    }
    const double xnorm2 = block_sum2(part, red).x;
    const double2 alpha = sv[0];
    double2 t = make_double2(0.0, 0.0);
    double beta = alpha.x;
    if (!(xnorm2 == 0.0 && alpha.y == 0.0)) {
      beta = -copysign(sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xnorm2), alpha.x);
      t = make_double2((beta - alpha.x) / beta, -alpha.y / beta);
    }
    const bool active = !(t.x == 0.0 && t.y == 0.0);
    // 1 / (alpha - beta)
    const double2 den = make_double2(alpha.x - beta, alpha.y);
    const double dn2 = den.x * den.x + den.y * den.y;
    const double2 sc = active ? make_double2(den.x / dn2, -den.y / dn2) : make_double2(0.0, 0.0);
    __syncthreads();
    for (int i = tid; i < n1; i += HT_THREADS) sv[i] = i == 0 ? make_double2(1.0, 0.0) : cmul(sv[i], sc);
    if (blockIdx.x == 0 && tid == 0) {
      dd[k] = __ldcg(A + (long)k * m + k).x;
      ee[k] = beta;
      tau[k] = t;
    }
    __syncthreads();
    // Warps per column: S of them split the rows of each trailing column, so a step takes about
    // n1 / (32 S) dependent loads per lane; every block derives the same S.
    const int S = max(1, min(kHtMaxSplit, W / max(n1, 1)));
    const int chunk = (n1 + S - 1) / S;
    // Phase B: partial sums of (A22 v)_r = sum_c conj(A[c, r]) v_c over the rows of one chunk;
    // ypart[s][r] for chunk s (tau is applied in phase C).
    if (active) {
      for (int g = gw; g < n1 * S; g += W) {
        const int c = g / S, sidx = g - c * S;
        const int r = k + 1 + c;
        const int i0 = sidx * chunk, i1 = min(n1, i0 + chunk);
        const double2* ac = A + (long)r * m + (k + 1);
        double sx = 0.0, sy = 0.0;
        for (int i = i0 + lane; i < i1; i += 32) {
          const double2 a = __ldcg(ac + i), v = sv[i];
          sx += a.x * v.x + a.y * v.y;  // conj(a) v
          sy += a.x * v.y - a.y * v.x;
        }
        sx = warp_sum(sx);
        sy = warp_sum(sy);
        if (lane == 0) y[(long)sidx * m + r] = make_double2(sx, sy);
      }
    }
    if (!grid_sync(bar, epoch)) return;
    // Phase C: y = tau A22 v; w = y + alpha v with alpha = -tau (y^H v) / 2; A22 -= v w^H + w v^H.
    if (active) {
      double2 p2 = make_double2(0.0, 0.0);
      for (int i = tid; i < n1; i += HT_THREADS) {
        double2 acc = make_double2(0.0, 0.0);
        for (int q = 0; q < S; ++q) acc = cadd(acc, __ldcg(y + (long)q * m + k + 1 + i));
        const double2 yi = cmul(t, acc), vi = sv[i];
        sw[i] = yi;
        p2.x += yi.x * vi.x + yi.y * vi.y;
        p2.y += yi.x * vi.y - yi.y * vi.x;
      }
      const double2 sdot = block_sum2(p2, red);
      const double2 al = cscale(cmul(t, sdot), -0.5);
      for (int i = tid; i < n1; i += HT_THREADS) sw[i] = cadd(sw[i], cmul(al, sv[i]));
      __syncthreads();
      for (int g = gw; g < n1 * S; g += W) {
        const int c = g / S, sidx = g - c * S;
        const int r = k + 1 + c;
        const int i0 = sidx * chunk, i1 = min(n1, i0 + chunk);
        const double2 wr = cconj(sw[c]), vr = cconj(sv[c]);
        double2* ac = A + (long)r * m + (k + 1);
        for (int i = i0 + lane; i < i1; i += 32) {
          double2 a = __ldcg(ac + i);
          a = csub(a, cadd(cmul(sv[i], wr), cmul(sw[i], vr)));
          ac[i] = a;
        }
      }
    }
    if (blockIdx.x == 0) {
      double2* cw = A + (long)k * m + (k + 1);
      for (int i = tid; i < n1; i += HT_THREADS) cw[i] = i == 0 ? make_double2(beta, 0.0) : sv[i];
    }
    if (!grid_sync(bar, epoch)) return;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) dd[m - 1] = __ldcg(A + (long)(m - 1) * m + (m - 1)).x;
}

// Householder reflector of x[0 .. n) in shared memory (zlarfg: x[0] = alpha), by every thread of the
// block: x becomes v (v[0] = 1), returns tau and beta with H^H x = beta e_1, H = I - tau v v^H.
__device__ void block_reflector(double2* x, int n, double2* red, double2& t, double& beta) {
  const int tid = threadIdx.x;
  double2 part = make_double2(0.0, 0.0);
  for (int i = tid + 1; i < n; i += HT_THREADS) part.x += x[i].x * x[i].x + x[i].y * x[i].y;
  const double xnorm2 = block_sum2(part, red).x;
  const double2 alpha = x[0];
  t = make_double2(0.0, 0.0);
  beta = alpha.x;
  if (!(xnorm2 == 0.0 && alpha.y == 0.0)) {
    beta = -copysign(sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xnorm2), alpha.x);
    t = make_double2((beta - alpha.x) / beta, -alpha.y / beta);
  }
  const bool active = !(t.x == 0.0 && t.y == 0.0);
  const double2 den = make_double2(alpha.x - beta, alpha.y);  // v = x / (alpha - beta)
  const double dn2 = den.x * den.x + den.y * den.y;
  const double2 sc = active ? make_double2(den.x / dn2, -den.y / dn2) : make_double2(0.0, 0.0);
  __syncthreads();
  for (int i = tid; i < n; i += HT_THREADS) x[i] = i == 0 ? make_double2(1.0, 0.0) : cmul(x[i], sc);
  __syncthreads();
}

// Step 1 with one grid barrier per column.  The update of step k and the matrix-vector product of
// step k+1 share one sweep over the trailing matrix: every block first applies step k's rank-2
// update to column k+1 alone (redundantly, from the unmodified global copy) and forms reflector
// k+1 from it, so the warps that then update a (column, row chunk) pair of the trailing matrix
// can take its partial product with v_{k+1} while the updated entries are in registers.  Column
// k+1 itself is never updated in global memory: its reflector is written there instead.  The
// trailing matrix is read once and written once per column (the two-barrier form reads it twice).
// The partial products alternate between two halves of y by step parity: a block still summing
// step k's partials while another already writes step k+1's never shares a buffer with it.
__global__ void __launch_bounds__(HT_THREADS) k_hetrd1(double2* __restrict__ A, int m, double* __restrict__ dd,
                                                       double* __restrict__ ee, double2* __restrict__ tau,
                                                       double2* __restrict__ y, GridBarrier bar) {
  extern __shared__ double2 hsm[];
  double2* sv = hsm;          // v_k (n1 entries)
  double2* sw = hsm + m;      // w_k
  double2* sn = hsm + 2 * m;  // v_{k+1}
  __shared__ double2 red[HT_WARPS];
  const int tid = threadIdx.x, lane = tid & 31;
  const int gw = blockIdx.x * HT_WARPS + (tid >> 5);
  const int W = gridDim.x * HT_WARPS;
  unsigned epoch = 0;
  // prologue: reflector 0 and the partial products of step 0
  double2 t;
  double beta;
  {
    const int n1 = m - 1;
    for (int i = tid; i < n1; i += HT_THREADS) sv[i] = __ldcg(A + 1 + i);
    __syncthreads();
    block_reflector(sv, n1, red, t, beta);
    if (blockIdx.x == 0 && tid == 0) {
      dd[0] = __ldcg(A).x;
      ee[0] = beta;
      tau[0] = t;
    }
  }
  int S_prev;
  {
    const int n1 = m - 1;
    const int S = max(1, min(kHtMaxSplit, W / max(n1, 1)));
    const int chunk = (n1 + S - 1) / S;
    for (int g = gw; g < n1 * S; g += W) {
      const int c = g / S, sidx = g - c * S;
      const int r = 1 + c;
      const int i0 = sidx * chunk, i1 = min(n1, i0 + chunk);
      const double2* ac = A + (long)r * m + 1;
      double sx = 0.0, sy = 0.0;
#pragma unroll 4
      for (int i = i0 + lane; i < i1; i += 32) {
        const double2 a = __ldcg(ac + i), v = sv[i];
        sx += a.x * v.x + a.y * v.y;  // conj(a) v
        sy += a.x * v.y - a.y * v.x;
      }
      sx = warp_sum(sx);
      sy = warp_sum(sy);
      if (lane == 0) y[(long)sidx * m + r] = make_double2(sx, sy);
    }
    S_prev = S;
  }
  if (!grid_sync(bar, epoch)) return;
  for (int k = 0; k + 1 < m; ++k) {
    const int n1 = m - k - 1;
    const double2* yk = y + (size_t)(k & 1) * kHtMaxSplit * m;      // step k's partials
    double2* yn = y + (size_t)((k + 1) & 1) * kHtMaxSplit * m;      // step k+1's
    // column k+1 as the previous sweep left it (rows k+1 ..), loaded with step k's partials
    double2 colr[kHtColRegs];
    {
      const double2* col = A + (long)(k + 1) * m + (k + 1);
#pragma unroll
      for (int q = 0; q < kHtColRegs; ++q) {
        const int i = tid + q * HT_THREADS;
        colr[q] = i < n1 ? __ldcg(col + i) : make_double2(0.0, 0.0);
      }
    }
    // (1) y = tau A22 v from the partial products; w = y + alpha v, alpha = -tau (y^H v) / 2
    {
      double2 p2 = make_double2(0.0, 0.0);
      for (int i = tid; i < n1; i += HT_THREADS) {
        double2 acc = make_double2(0.0, 0.0);
#pragma unroll 8
        for (int q = 0; q < S_prev; ++q) acc = cadd(acc, __ldcg(yk + (long)q * m + k + 1 + i));
        const double2 yi = cmul(t, acc), vi = sv[i];
        sw[i] = yi;
        p2.x += yi.x * vi.x + yi.y * vi.y;
        p2.y += yi.x * vi.y - yi.y * vi.x;
      }
      const double2 sdot = block_sum2(p2, red);
      const double2 al = cscale(cmul(t, sdot), -0.5);
      for (int i = tid; i < n1; i += HT_THREADS) sw[i] = cadd(sw[i], cmul(al, sv[i]));
      if (blockIdx.x == 0) {
        // column k now holds its reflector (no block reads column k any more)
        double2* cw = A + (long)k * m + (k + 1);
        for (int i = tid; i < n1; i += HT_THREADS) cw[i] = i == 0 ? make_double2(beta, 0.0) : sv[i];
      }
      __syncthreads();
    }
    // (2) column k+1 after step k's update (rows k+1 .. m-1), its diagonal, and reflector k+1
    const bool next = k + 2 < m;  // a reflector k+1 exists
    double2 tn = make_double2(0.0, 0.0);
    double betan = 0.0;
    {
      const double2 w0c = cconj(sw[0]);  // v_0 = 1
#pragma unroll
      for (int q = 0; q < kHtColRegs; ++q) {
        const int i = tid + q * HT_THREADS;
        if (i >= n1) break;
        const double2 x = csub(colr[q], cadd(cmul(sv[i], w0c), sw[i]));
        if (i == 0) {
          if (blockIdx.x == 0) dd[k + 1] = x.x;
        } else {
          sn[i - 1] = x;
        }
      }
      __syncthreads();
      if (next) {
        block_reflector(sn, n1 - 1, red, tn, betan);
        if (blockIdx.x == 0 && tid == 0) {
          ee[k + 1] = betan;
          tau[k + 1] = tn;
        }
      }
    }
    if (!next) break;
    // (3) rank-2 update of columns k+2 .. m-1 (all rows k+1 .. m-1) and, on the updated entries,
    // the partial products of step k+1 (rows k+2 ..)
    {
      const int nc = n1 - 1;
      const int S = max(1, min(kHtMaxSplit, W / max(nc, 1)));
      const int chunk = (n1 + S - 1) / S;
      for (int g = gw; g < nc * S; g += W) {
        const int c = 1 + g / S, sidx = g - (c - 1) * S;
        const int r = k + 1 + c;
        const int i0 = sidx * chunk, i1 = min(n1, i0 + chunk);
        const double2 wr = cconj(sw[c]), vr = cconj(sv[c]);
        double2* ac = A + (long)r * m + (k + 1);
        double sx = 0.0, sy = 0.0;
#pragma unroll 8
        for (int i = i0 + lane; i < i1; i += 32) {
          double2 a = __ldcg(ac + i);
          a = csub(a, cadd(cmul(sv[i], wr), cmul(sw[i], vr)));
          ac[i] = a;
          if (i > 0) {
            const double2 v = sn[i - 1];
            sx += a.x * v.x + a.y * v.y;  // conj(a) v
            sy += a.x * v.y - a.y * v.x;
          }
        }
        sx = warp_sum(sx);
        sy = warp_sum(sy);
        if (lane == 0) yn[(long)sidx * m + r] = make_double2(sx, sy);
      }
      S_prev = S;
    }
    if (!grid_sync(bar, epoch)) return;
    double2* tmp = sv;
    sv = sn;
    sn = tmp;
    t = tn;
    beta = betan;
  }
}

// Number of eigenvalues of T below x (Sturm sequence of the LDL^T pivots).
__device__ __forceinline__ int sturm_count(const double* d, const double* e2, int m, double x, double pivmin) {
  double q = d[0] - x;
  if (fabs(q) < pivmin) q = -pivmin;
  int cnt = q < 0.0;
  for (int i = 1; i < m; ++i) {
    q = (d[i] - x) - e2[i - 1] / q;
    if (fabs(q) < pivmin) q = -pivmin;
    cnt += q < 0.0;
  }
  return cnt;
}

// Step 2.  w[j], j < nev: the j-th smallest eigenvalue of T.  Block 0 also writes ||T|| (the
// Gershgorin radius bound) to *tnorm_out for step 3.
__global__ void __launch_bounds__(BS_WARPS * 32) k_tridiag_bisect(const double* __restrict__ dd, const double* __restrict__ ee,
                                                                  int m, int nev, double* __restrict__ w,
                                                                  double* __restrict__ tnorm_out) {
  extern __shared__ double bsm[];
  double* d = bsm;
  double* e2 = bsm + m;
  __shared__ double red[3][BS_WARPS];
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  double lo = DBL_MAX, hi = -DBL_MAX, emax = 0.0;
  for (int i = tid; i < m; i += blockDim.x) {
    const double di = dd[i];
    const double el = i > 0 ? fabs(ee[i - 1]) : 0.0, er = i + 1 < m ? fabs(ee[i]) : 0.0;
    d[i] = di;
    if (i + 1 < m) e2[i] = ee[i] * ee[i];
    lo = fmin(lo, di - el - er);
    hi = fmax(hi, di + el + er);
    emax = fmax(emax, er * er);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    emax = fmax(emax, __shfl_xor_sync(0xffffffffu, emax, o));
  }
  if (lane == 0) {
    red[0][wid] = lo;
    red[1][wid] = hi;
    red[2][wid] = emax;
  }
  __syncthreads();
  lo = red[0][0];
  hi = red[1][0];
  emax = red[2][0];
  for (int i = 1; i < BS_WARPS; ++i) {
    lo = fmin(lo, red[0][i]);
    hi = fmax(hi, red[1][i]);
    emax = fmax(emax, red[2][i]);
  }
  const double tnorm = fmax(fabs(lo), fabs(hi));
  const double pivmin = DBL_MIN * fmax(1.0, emax);
  if (blockIdx.x == 0 && tid == 0) *tnorm_out = tnorm;
  const double fudge = 2.0 * DBL_EPSILON * tnorm + 4.0 * pivmin;
  lo -= fudge;
  hi += fudge;
  const int j = blockIdx.x * BS_WARPS + wid;
  if (j >= nev) return;
  const double abstol = DBL_EPSILON * tnorm;
  for (int it = 0; it < 64; ++it) {
    const double width = hi - lo;
    if (width <= fmax(abstol, 2.0 * DBL_EPSILON * fmax(fabs(lo), fabs(hi))) + pivmin) break;
    const double x = lo + width * (double)(lane + 1) / 33.0;
    const int c = sturm_count(d, e2, m, x, pivmin);
    const unsigned ball = __ballot_sync(0xffffffffu, c > j);
    if (ball) {
      const int f = __ffs(ball) - 1;
      const double nhi = __shfl_sync(0xffffffffu, x, f);
      const double nlo = f > 0 ? __shfl_sync(0xffffffffu, x, f > 0 ? f - 1 : 0) : lo;
      if (nhi >= hi && nlo <= lo) break;  // no progress: bracket at rounding level
      lo = nlo;
      hi = nhi;
    } else {
      const double nlo = __shfl_sync(0xffffffffu, x, 31);
      if (nlo <= lo) break;
      lo = nlo;
    }
  }
  if (lane == 0) w[j] = 0.5 * (lo + hi);
}

__device__ __forceinline__ double hashed_unit(uint64_t a, uint64_t b) {
  uint64_t z = a * 0x9E3779B97F4A7C15ULL + b + 0x632BE59BD9B4E019ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  z ^= z >> 31;
  return (double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;  // [-1, 1)
}

// Step 3.  Z[:, j] (m x nev, column-major, real) = unit eigenvector of T for w[j].  One warp (one
// block) per group of eigenvalues closer than kGroupTol ||T|| to their neighbour (a singleton is a
// group of one), run by the block whose j starts the group.  The group's vectors are computed in
// order; after every solve each is re-orthogonalised (modified Gram-Schmidt) against the group's
// earlier vectors, the 32 lanes sharing the dot products, the updates and the norm.  Lane 0 runs the
// three recurrences (row-pivoted elimination of T - lambda I, the forward and the back substitution)
// out of shared memory, which holds, m entries each: the reciprocal pivots, U's two superdiagonals,
// the multipliers, the working vector (doubles) and the row-swap flags (bytes).  Every sweep loads
// kIvChunk entries ahead of the recurrence that consumes them.
constexpr size_t invit_smem(int m) { return (size_t)m * (5 * sizeof(double) + 1); }

__global__ void __launch_bounds__(32) k_tridiag_invit(const double* __restrict__ dd, const double* __restrict__ ee, int m,
                                                      int nev, const double* __restrict__ w,
                                                      const double* __restrict__ tnorm_p, double* __restrict__ Z) {
  extern __shared__ double ism[];
  const int j = blockIdx.x, lane = threadIdx.x;
  if (j >= nev) return;
  const double tnorm = fmax(*tnorm_p, DBL_MIN);
  const double gtol = kGroupTol * tnorm;
  if (j > 0 && !(w[j] - w[j - 1] > gtol)) return;
  int jend = j + 1;
  while (jend < nev && !(w[jend] - w[jend - 1] > gtol)) ++jend;
  double* const rp = ism;      // 1 / U's diagonal
  double* const u1 = rp + m;   // U's first superdiagonal
  double* const u2 = u1 + m;   // U's second superdiagonal (nonzero after a row swap)
  double* const lm = u2 + m;   // elimination multipliers
  double* const zz = lm + m;   // working vector
  unsigned char* const swp = reinterpret_cast<unsigned char*>(zz + m);  // row i swapped with i+1
  const double tiny = DBL_EPSILON * tnorm;
  for (int p = j; p < jend; ++p) {
    const double lam = w[p];
    if (lane == 0) {
      // Row-pivoted elimination of T - lam I.  (a, b): the running row at columns (i, i+1).
      double a = dd[0] - lam, b = m > 1 ? ee[0] : 0.0;
      for (int i0 = 0; i0 + 1 < m; i0 += kIvChunk) {
        const int n = min(kIvChunk, m - 1 - i0);
        double sb[kIvChunk], dn[kIvChunk], up[kIvChunk];
#pragma unroll
        for (int c = 0; c < kIvChunk; ++c) {
          if (c < n) {
            const int i = i0 + c;
            sb[c] = __ldg(ee + i);
            dn[c] = __ldg(dd + i + 1) - lam;
            up[c] = i + 2 < m ? __ldg(ee + i + 1) : 0.0;
          }
        }
#pragma unroll
        for (int c = 0; c < kIvChunk; ++c) {
          if (c < n) {
            const int i = i0 + c;
            if (fabs(a) >= fabs(sb[c])) {
              const double piv = fabs(a) < tiny ? (a < 0.0 ? -tiny : tiny) : a;
              const double l = sb[c] / piv;
              rp[i] = 1.0 / piv; u1[i] = b; u2[i] = 0.0; lm[i] = l; swp[i] = 0;
              a = dn[c] - l * b;
              b = up[c];
            } else {
              const double l = a / sb[c];
              rp[i] = 1.0 / sb[c]; u1[i] = dn[c]; u2[i] = up[c]; lm[i] = l; swp[i] = 1;
              a = b - l * dn[c];
              b = -l * up[c];
            }
          }
        }
      }
      rp[m - 1] = 1.0 / (fabs(a) < tiny ? (a < 0.0 ? -tiny : tiny) : a);
      u1[m - 1] = 0.0;  // the back substitution reads row m-1's superdiagonals
      u2[m - 1] = 0.0;
    }
    // zz holds the vector up to the factor scl (the previous sweep's normalisation, applied as the
    // next sweep reads it); the first sweep starts from a hashed vector
    double scl = 1.0;
    for (int sweep = 0; sweep < 3; ++sweep) {
      double nrm = 0.0, bigv = 0.0;
      if (lane == 0) {
        auto rhs = [&](int i) { return sweep == 0 ? hashed_unit((uint64_t)p, (uint64_t)i) : zz[i] * scl; };
        // forward: the same row operations on the right-hand side (entry i+1 is read before entry
        // i is written, so a chunk's loads may all precede its stores)
        double cb = rhs(0);
        for (int i0 = 0; i0 + 1 < m; i0 += kIvChunk) {
          const int n = min(kIvChunk, m - 1 - i0);
          double zn[kIvChunk], lv[kIvChunk];
          unsigned char sv[kIvChunk];
#pragma unroll
          for (int c = 0; c < kIvChunk; ++c) {
            if (c < n) {
              zn[c] = rhs(i0 + c + 1);
              lv[c] = lm[i0 + c];
              sv[c] = swp[i0 + c];
            }
          }
#pragma unroll
          for (int c = 0; c < kIvChunk; ++c) {
            if (c < n) {
              if (sv[c] == 0) {
                zz[i0 + c] = cb;
                cb = zn[c] - lv[c] * cb;
              } else {
                zz[i0 + c] = zn[c];
                cb = cb - lv[c] * zn[c];
              }
            }
          }
        }
        zz[m - 1] = cb;
        // back substitution with U (diagonal + two superdiagonals), z[i+1], z[i+2] carried; the
        // squared norm and the entry of largest magnitude (first in index order) on the way
        double zp1 = 0.0, zp2 = 0.0, big = -1.0;
        for (int i1 = m; i1 > 0; i1 -= kIvChunk) {
          const int n = min(kIvChunk, i1);
          double zr[kIvChunk], r0[kIvChunk], d1[kIvChunk], d2[kIvChunk];
#pragma unroll
          for (int c = 0; c < kIvChunk; ++c) {
            if (c < n) {
              const int i = i1 - 1 - c;
              zr[c] = zz[i];
              r0[c] = rp[i];
              d1[c] = u1[i];
              d2[c] = u2[i];
            }
          }
#pragma unroll
          for (int c = 0; c < kIvChunk; ++c) {
            if (c < n) {
              const double x = (zr[c] - d1[c] * zp1 - d2[c] * zp2) * r0[c];
              zz[i1 - 1 - c] = x;
              nrm += x * x;
              if (fabs(x) >= big) { big = fabs(x); bigv = x; }
              zp2 = zp1;
              zp1 = x;
            }
          }
        }
      }
      __syncwarp();
      if (p > j) {
        // modified Gram-Schmidt against the group's earlier vectors (written by this warp), then the
        // norm and the first entry of largest magnitude again
        for (int q = j; q < p; ++q) {
          const double* zq = Z + (size_t)q * m;
          double dot = 0.0;
          for (int i = lane; i < m; i += 32) dot += zq[i] * zz[i];
          dot = warp_sum(dot);
          for (int i = lane; i < m; i += 32) zz[i] -= dot * zq[i];
          __syncwarp();
        }
        double big = -1.0;
        int bi = m;
        nrm = 0.0;
        bigv = 0.0;
        for (int i = lane; i < m; i += 32) {
          const double zi = zz[i];
          nrm += zi * zi;
          if (fabs(zi) > big) { big = fabs(zi); bigv = zi; bi = i; }
        }
        nrm = warp_sum(nrm);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          const double ob = __shfl_xor_sync(0xffffffffu, big, o), ov = __shfl_xor_sync(0xffffffffu, bigv, o);
          const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
          if (ob > big || (ob == big && oi < bi)) { big = ob; bigv = ov; bi = oi; }
        }
      } else {
        nrm = __shfl_sync(0xffffffffu, nrm, 0);
        bigv = __shfl_sync(0xffffffffu, bigv, 0);
      }
      scl = nrm > 0.0 ? 1.0 / sqrt(nrm) : 0.0;
      if (bigv < 0.0) scl = -scl;
    }
    double* z = Z + (size_t)p * m;
    for (int i = lane; i < m; i += 32) z[i] = zz[i] * scl;
    __syncwarp();
  }
}

// Step 4.  E[:, j] = H_0 H_1 ... H_{m-2} Z[:, j] (applied right to left), one warp per column.
__global__ void __launch_bounds__(BT_WARPS * 32) k_hetrd_back(const double2* __restrict__ A, const double2* __restrict__ tau,
                                                              int m, int nev, const double* __restrict__ Z,
                                                              double2* __restrict__ E, long lde) {
  extern __shared__ double2 esm[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int j = blockIdx.x * BT_WARPS + wid;
  if (j >= nev) return;
  double2* ev = esm + (size_t)wid * m;
  const double* zj = Z + (size_t)j * m;
  for (int i = lane; i < m; i += 32) ev[i] = make_double2(zj[i], 0.0);
  __syncwarp();
  for (int k = m - 2; k >= 0; --k) {
    const double2 t = tau[k];
    if (t.x == 0.0 && t.y == 0.0) continue;
    const int n1 = m - k - 1;
    const double2* vk = A + (long)k * m + (k + 1);
    double sx = 0.0, sy = 0.0;
    for (int i = lane; i < n1; i += 32) {
      const double2 v = i == 0 ? make_double2(1.0, 0.0) : __ldg(vk + i);
      const double2 x = ev[k + 1 + i];
      sx += v.x * x.x + v.y * x.y;  // conj(v) x
      sy += v.x * x.y - v.y * x.x;
    }
    sx = warp_sum(sx);
    sy = warp_sum(sy);
    const double2 ts = cmul(t, make_double2(sx, sy));
    for (int i = lane; i < n1; i += 32) {
      const double2 v = i == 0 ? make_double2(1.0, 0.0) : __ldg(vk + i);
      ev[k + 1 + i] = csub(ev[k + 1 + i], cmul(ts, v));
    }
    __syncwarp();
  }
  for (int i = lane; i < m; i += 32) E[(size_t)j * lde + i] = ev[i];
}

// ---- blocked back-transformation (compact WY) ----------------------------------------------------
// The reflectors k0 .. k0+nb-1 multiply to H_k0 ... H_{k0+nb-1} = I - V T V^H with T upper
// triangular, T[j][j] = tau_j and T[0:j, j] = -tau_j T[0:j, 0:j] (V[:, 0:j]^H v_j).  Then
// E <- E - V (T (V^H E)) is three GEMMs; the blocks are applied from the last to the first.
constexpr int kWyB = 64;

// Vb (m x nb, column-major): v_{k0+j} with its implicit unit at row k0+j+1 and zeros above.
__global__ void k_wy_v(const double2* __restrict__ A, int m, int k0, int nb, double2* __restrict__ Vb) {
  const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (idx >= (long)m * nb) return;
  const int j = (int)(idx / m), row = (int)(idx - (long)j * m);
  const int k = k0 + j;
  double2 v = make_double2(0.0, 0.0);
  if (row == k + 1) v = make_double2(1.0, 0.0);
  else if (row > k + 1) v = A[row + (long)k * m];
  Vb[idx] = v;
}

// Every block's triangular factor at once (the factors depend on the reflectors only): CTA b
// forms G = V_b^H V_b for reflectors k0 = b kWyB .. k0 + nb - 1 straight from the factored matrix
// (v_k = 1 at row k+1, A[row, k] below, 0 above), 4 x 4 outputs per thread (rows tr + 16 q,
// columns tc + 16 q) over row chunks staged in shared memory, then T_b (ld kWyB, at T + b kWyB^2) by the zlarft recurrence: column j needs
// T[0:j, 0:j] G[0:j, j]; its row i is summed by the four consecutive lanes of row group i and two
// shuffles.
constexpr int kWyTThreads = 4 * kWyB;
constexpr int kWyRows = 32;  // reflector rows per staged chunk
struct WyTSmem {
  double2 gs[kWyB][kWyB + 1];  // gs[col][row]
  double2 ts[kWyB][kWyB + 1];  // ts[col][row]
  double2 vc[kWyRows][kWyB + 1];  // a chunk of V_b's rows
};
constexpr size_t kWyTSmem = sizeof(WyTSmem);
__global__ void __launch_bounds__(kWyTThreads) k_wy_t_all(const double2* __restrict__ A, int m, const double2* __restrict__ tau,
                                                          int nref, double2* __restrict__ T) {
  extern __shared__ __align__(16) unsigned char wsm[];
  WyTSmem& S = *reinterpret_cast<WyTSmem*>(wsm);
  const int tid = threadIdx.x;
  const int k0 = blockIdx.x * kWyB, nb = min(kWyB, nref - k0);
  const int tr = tid >> 4, tc = tid & 15;  // G tile: rows tr + 16 q, columns tc + 16 q
  double2 acc[4][4];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[r][c] = make_double2(0.0, 0.0);
  for (int row0 = k0 + 1; row0 < m; row0 += kWyRows) {
    __syncthreads();
    for (int idx = tid; idx < kWyRows * kWyB; idx += kWyTThreads) {  // along each reflector's rows
      const int j = idx / kWyRows, rr = idx - j * kWyRows, row = row0 + rr, k = k0 + j;
      double2 v = make_double2(0.0, 0.0);
      if (j < nb && row < m) {
        if (row == k + 1) v = make_double2(1.0, 0.0);
        else if (row > k + 1) v = A[row + (long)k * m];
      }
      S.vc[rr][j] = v;
    }
    __syncthreads();
#pragma unroll 4
    for (int rr = 0; rr < kWyRows; ++rr) {
      double2 vr[4], vcol[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        vr[q] = S.vc[rr][tr + 16 * q];
        vcol[q] = S.vc[rr][tc + 16 * q];
      }
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) {  // acc += conj(vr) vcol
          acc[r][c].x += vr[r].x * vcol[c].x + vr[r].y * vcol[c].y;
          acc[r][c].y += vr[r].x * vcol[c].y - vr[r].y * vcol[c].x;
        }
    }
  }
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      S.gs[tc + 16 * c][tr + 16 * r] = acc[r][c];
      S.ts[tc + 16 * c][tr + 16 * r] = make_double2(0.0, 0.0);
    }
  __syncthreads();
  const int i = tid >> 2, q = tid & 3;
  for (int j = 0; j < nb; ++j) {
    double2 sum = make_double2(0.0, 0.0);
    if (i < j)
      for (int l = i + q; l < j; l += 4) sum = cadd(sum, cmul(S.ts[l][i], S.gs[j][l]));
    sum.x += __shfl_xor_sync(0xffffffffu, sum.x, 1);
    sum.y += __shfl_xor_sync(0xffffffffu, sum.y, 1);
    sum.x += __shfl_xor_sync(0xffffffffu, sum.x, 2);
    sum.y += __shfl_xor_sync(0xffffffffu, sum.y, 2);
    if (q == 0) {
      const double2 tj = tau[k0 + j];
      if (i < j) S.ts[j][i] = cscale(cmul(tj, sum), -1.0);
      else if (i == j) S.ts[j][i] = tj;
    }
    __syncthreads();
  }
  double2* Tb = T + (size_t)blockIdx.x * kWyB * kWyB;
  for (int idx = tid; idx < kWyB * kWyB; idx += kWyTThreads) {
    const int r = idx % kWyB, c = idx / kWyB;
    Tb[r + c * kWyB] = S.ts[c][r];
  }
}

__global__ void k_real_to_complex(const double* __restrict__ Z, int m, int nev, double2* __restrict__ E, long lde) {
  const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (idx >= (long)m * nev) return;
  const int j = (int)(idx / m), row = (int)(idx - (long)j * m);
  E[row + j * lde] = make_double2(Z[idx], 0.0);
}

int heev_back_blocked(const double2* A, const double2* tau, int m, int nev, const double* Z, double2* E, long lde,
                      const HeevWork& w, cudaStream_t s) {
  const int nref = m - 1;
  const int nblk = (nref + kWyB - 1) / kWyB;
  double2* Vb = w.wy;
  double2* T = Vb + (size_t)m * kWyB;  // nblk triangular factors
  double2* W = T + (size_t)nblk * kWyB * kWyB;
  double2* W2 = W + (size_t)kWyB * nev;
  double2* ws = W2 + (size_t)kWyB * nev;
  k_real_to_complex<<<ceil_div((size_t)m * nev, 256), 256, 0, s>>>(Z, m, nev, E, lde);
  count_launch();
  k_wy_t_all<<<nblk, kWyTThreads, kWyTSmem, s>>>(A, m, tau, nref, T);
  count_launch();
  for (int b = nblk - 1; b >= 0; --b) {
    const int k0 = b * kWyB, nb = std::min(kWyB, nref - k0);
    const int rows = m - k0 - 1;  // rows k0+1 .. m-1 hold the block's reflectors
    k_wy_v<<<ceil_div((size_t)m * nb, 256), 256, 0, s>>>(A, m, k0, nb, Vb);
    count_launch();
    // W = V^H E
    GemmArgs g{};
    g.M = nb; g.N = nev; g.K = rows;
    g.A = Vb + k0 + 1; g.lda = m; g.a_kc = true; g.conj_a = true;
    g.B = E + k0 + 1; g.ldb = lde; g.b_kc = true; g.conj_b = false;
    g.O = W; g.ldo_r = 1; g.ldo_c = kWyB; g.alpha = 1.0; g.beta = 0.0;
    DFT_TRY(zgemm(g, s, ws, w.wy_ws_elems));
    // W2 = T_b W
    g = GemmArgs{};
    g.M = nb; g.N = nev; g.K = nb;
    g.A = T + (size_t)b * kWyB * kWyB; g.lda = kWyB; g.a_kc = false; g.conj_a = false;
    g.B = W; g.ldb = kWyB; g.b_kc = true; g.conj_b = false;
    g.O = W2; g.ldo_r = 1; g.ldo_c = kWyB; g.alpha = 1.0; g.beta = 0.0;
    DFT_TRY(zgemm(g, s, ws, w.wy_ws_elems));
    // E[k0+1:, :] -= V W2
    g = GemmArgs{};
    g.M = rows; g.N = nev; g.K = nb;
    g.A = Vb + k0 + 1; g.lda = m; g.a_kc = false; g.conj_a = false;
    g.B = W2; g.ldb = kWyB; g.b_kc = true; g.conj_b = false;
    g.O = E + k0 + 1; g.ldo_r = 1; g.ldo_c = lde; g.alpha = -1.0; g.beta = 1.0;
    DFT_TRY(zgemm(g, s, ws, w.wy_ws_elems));
  }
  return DFTCUDA_OK;
}

__global__ void k_upper_to_full(const double2* __restrict__ src, long lds, double2* __restrict__ A, int m) {
  const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (idx >= (long)m * m) return;
  const int r = (int)(idx % m), c = (int)(idx / m);
  if (r < c) A[idx] = src[r + c * lds];
  else if (r == c) A[idx] = make_double2(src[r + c * lds].x, 0.0);
  else {
    const double2 u = src[c + r * lds];
    A[idx] = make_double2(u.x, -u.y);
  }
}

}  // namespace

// Split-K space of the blocked back-transformation's GEMMs: up to 32 partial kWyB x nev products.
static size_t wy_ws_elems(int nev) { return (size_t)32 * kWyB * std::max(nev, kWyB); }
static size_t wy_elems(int m, int nev) {
  const size_t nblk = (size_t)(std::max(m - 1, 1) + kWyB - 1) / kWyB;
  return (size_t)m * kWyB + nblk * kWyB * kWyB + 2 * (size_t)kWyB * nev + wy_ws_elems(nev);
}

size_t heev_work_bytes(int m, int nev) {
  const size_t mm = (size_t)m;
  return 256 * 8 + sizeof(double) * (3 * mm + 1) + sizeof(double2) * (1 + 2 * kHtMaxSplit) * mm + sizeof(double) * mm * nev +
         sizeof(double2) * wy_elems(m, nev);
}

void heev_bind(HeevWork& w, void* base, int m, int nev) {
  char* b = (char*)base;
  size_t off = 0;
  auto take = [&](size_t bytes) { char* p = b + off; off += (bytes + 255) / 256 * 256; return p; };
  w.bar = (unsigned*)take(4 * sizeof(unsigned));
  w.d = (double*)take(sizeof(double) * m);
  w.e = (double*)take(sizeof(double) * m);
  w.tnorm = (double*)take(sizeof(double));
  w.tau = (double2*)take(sizeof(double2) * m);
  w.y = (double2*)take(sizeof(double2) * m * 2 * kHtMaxSplit);  // two halves for the one-barrier form
  w.z = (double*)take(sizeof(double) * (size_t)m * nev);
  w.wy_ws_elems = wy_ws_elems(nev);
  w.wy = (double2*)take(sizeof(double2) * wy_elems(m, nev));
  w.m_cap = m;
  w.nev_cap = nev;
}

int heev_lowest(double2* A, int m, int nev, double* evals, double2* E, long lde, const HeevWork& w, int* status,
                cudaStream_t s) {
  if (m < 1 || m > 2048 || nev < 1 || nev > m || m > (int)w.m_cap || nev > (int)w.nev_cap)
    return fail(DFTCUDA_ERR_INVALID_MATRIX_SIZE, "heev: size outside the workspace");
  int dev = 0;
  DFT_CUDA_TRY(cudaGetDevice(&dev));
  // DFTCUDA_HETRD=2barrier selects the two-barrier tridiagonalisation (A/B measurements)
  static const bool two_barrier = [] {
    const char* e = std::getenv("DFTCUDA_HETRD");
    return e && std::string(e) == "2barrier";
  }();
  const void* hetrd_fn = two_barrier ? (const void*)k_hetrd : (const void*)k_hetrd1;
  const int hetrd_bufs = two_barrier ? 2 : 3;  // shared-memory vectors of m entries
  const size_t smem_tr = sizeof(double2) * hetrd_bufs * 2048;
  DFT_TRY(ensure_max_dynamic_smem(hetrd_fn, (int)smem_tr));
  DFT_TRY(ensure_max_dynamic_smem((const void*)k_hetrd_back, (int)(sizeof(double2) * BT_WARPS * 2048)));
  DFT_TRY(ensure_max_dynamic_smem((const void*)k_wy_t_all, (int)kWyTSmem));
  DFT_TRY(ensure_max_dynamic_smem((const void*)k_tridiag_invit, (int)invit_smem(2048)));
  // SM count and the reduction kernel's occupancy, per device (several host threads may ask at once)
  static std::mutex occ_mu;
  static std::map<int, std::pair<int, int>> occ;
  int n_sm = 0, per_sm = 0;
  {
    std::lock_guard<std::mutex> lock(occ_mu);
    auto it = occ.find(dev);
    if (it == occ.end()) {
      DFT_CUDA_TRY(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
      DFT_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, hetrd_fn, HT_THREADS, smem_tr));
      occ[dev] = {n_sm, per_sm};
    } else {
      n_sm = it->second.first;
      per_sm = it->second.second;
    }
  }
  if (per_sm < 1) return fail(DFTCUDA_ERR_UNSUPPORTED, "heev: tridiagonalisation kernel does not fit an SM");
  DFT_CUDA_TRY(cudaMemsetAsync(w.bar, 0, 2 * sizeof(unsigned), s));
  DFT_CUDA_TRY(cudaMemsetAsync(status, 0, sizeof(int), s));
  if (m > 1) {
    GridBarrier bar{w.bar, status, 0};
    const WaitLimits wl = wait_limits();
    if (wl.polls > 0) bar.spin = wl.polls;
    bar.extra = wl.unreachable ? 1u : 0u;
    // enough warps for kHtMaxSplit per column at the start, at most one block per SM
    // (DFTCUDA_HETRD_BPS=2 allows two where they fit, for measurements)
    static const int bps = [] {
      const char* e = std::getenv("DFTCUDA_HETRD_BPS");
      return e && std::atoi(e) == 2 ? 2 : 1;
    }();
    const int want = (m * kHtMaxSplit + HT_WARPS - 1) / HT_WARPS;
    bar.nblocks = (unsigned)std::max(1, std::min(want, n_sm * std::min(per_sm, bps)));
    double2* a_ = A;
    int m_ = m;
    double* d_ = w.d;
    double* e_ = w.e;
    double2* t_ = w.tau;
    double2* y_ = w.y;
    void* args[] = {&a_, &m_, &d_, &e_, &t_, &y_, &bar};
    DFT_CUDA_TRY(cudaLaunchCooperativeKernel(hetrd_fn, dim3(bar.nblocks), dim3(HT_THREADS), args,
                                             sizeof(double2) * hetrd_bufs * m, s));
    count_launch();
  } else {
    DFT_CUDA_TRY(cudaMemcpyAsync(w.d, A, sizeof(double), cudaMemcpyDeviceToDevice, s));
    DFT_CUDA_TRY(cudaMemsetAsync(w.tau, 0, sizeof(double2), s));
  }
  k_tridiag_bisect<<<ceil_div(nev, BS_WARPS), BS_WARPS * 32, sizeof(double) * 2 * m, s>>>(w.d, w.e, m, nev, evals, w.tnorm);
  count_launch();
  k_tridiag_invit<<<nev, 32, invit_smem(m), s>>>(w.d, w.e, m, nev, evals, w.tnorm, w.z);
  count_launch();
  if (m >= 192 && nev >= 32) {
    DFT_TRY(heev_back_blocked(A, w.tau, m, nev, w.z, E, lde, w, s));
  } else {
    k_hetrd_back<<<ceil_div(nev, BT_WARPS), BT_WARPS * 32, sizeof(double2) * BT_WARPS * m, s>>>(A, w.tau, m, nev, w.z, E, lde);
    count_launch();
  }
  DFT_CUDA_TRY(cudaGetLastError());
  return DFTCUDA_OK;
}

int hermitian_upper_to_full(const double2* src, long lds, double2* A, int m, cudaStream_t s) {
  k_upper_to_full<<<ceil_div((size_t)m * m, 256), 256, 0, s>>>(src, lds, A, m);
  count_launch();
  DFT_CUDA_TRY(cudaGetLastError());
  return DFTCUDA_OK;
}

}  // namespace dftcuda

using namespace dftcuda;

// linalg.hermitian_eigen_decomp (linalg/linalg.zig:141-151, zheev 'V','U'): the nev lowest
// eigenpairs of the n x n Hermitian matrix a (column-major, upper triangle read).
extern "C" int dftcuda_hermitian_eigen_decomp(size_t n, const double* a, size_t nev, double* values, double* vectors) {
  if (n == 0 || nev == 0) return DFTCUDA_OK;
  if (!a || !values || !vectors) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "hermitian_eigen_decomp: null argument");
  if (n > 2048 || nev > n) return fail(DFTCUDA_ERR_INVALID_MATRIX_SIZE, "hermitian_eigen_decomp: n > 2048 or nev > n");
  const int m = (int)n, k = (int)nev;
  cudaStream_t s = nullptr;
  DFT_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamDefault));
  struct Guard {
    cudaStream_t s;
    void* p[4] = {nullptr, nullptr, nullptr, nullptr};
    ~Guard() {
      for (void* q : p)
        if (q) cudaFree(q);
      cudaStreamDestroy(s);
    }
  } g{s};
  const size_t mat = sizeof(double2) * n * n;
  DFT_CUDA_TRY(dev_malloc(&g.p[0], mat));
  DFT_CUDA_TRY(dev_malloc(&g.p[1], mat + sizeof(double2) * n * nev + sizeof(double) * nev + 256));
  DFT_CUDA_TRY(dev_malloc(&g.p[2], heev_work_bytes(m, k)));
  DFT_CUDA_TRY(dev_malloc(&g.p[3], 256));
  double2* src = (double2*)g.p[0];
  double2* A = (double2*)g.p[1];
  double2* E = A + n * n;
  double* ev = (double*)(E + n * nev);
  HeevWork w;
  heev_bind(w, g.p[2], m, k);
  int* status = (int*)g.p[3];
  DFT_CUDA_TRY(cudaMemcpyAsync(src, a, mat, is_device_pointer(a) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
  DFT_TRY(hermitian_upper_to_full(src, (long)n, A, m, s));
  DFT_TRY(heev_lowest(A, m, k, ev, E, (long)n, w, status, s));
  int h_status = 0;
  DFT_CUDA_TRY(cudaMemcpyAsync(&h_status, status, sizeof(int), cudaMemcpyDeviceToHost, s));
  DFT_CUDA_TRY(cudaMemcpyAsync(values, ev, sizeof(double) * nev,
                               is_device_pointer(values) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s));
  DFT_CUDA_TRY(cudaMemcpyAsync(vectors, E, sizeof(double2) * n * nev,
                               is_device_pointer(vectors) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s));
  DFT_CUDA_TRY(cudaStreamSynchronize(s));
  if (h_status != 0) return fail(DFTCUDA_ERR_TIMEOUT, "hermitian_eigen_decomp: grid barrier timed out");
  return DFTCUDA_OK;
}
