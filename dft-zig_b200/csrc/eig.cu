// Block-Davidson ("LOBPCG") eigensolver on the device: src/features/linalg/lobpcg/serial.zig:55-307.
//
// Device data: V, W = H V (max_subspace columns), Ritz vectors, residuals.  The host keeps only the
// control flow of the reference loop (iteration count, which bands are added, restart), reading
// back nbands eigenvalues and residual norms per iteration.
//
// Steps and their reference counterparts:
//  * random start: the reference's LCG (common.zig:287-319) evaluated in closed form per element
//    (s_k = a^k s0 + sum_{j<k} a^j mod 2^64), so the device draws exactly the reference's numbers;
//  * T = V^H W, Hermitised (common.zig:231-259): FP64 complex GEMM on the new columns only + k_gram_finish;
//  * small eigenproblem (zheev, common.zig:440-508): cyclic two-sided complex Jacobi in one CTA
//    below 96 columns, the tridiagonal solver of heev.cu (lowest nbands pairs) from there on;
//  * Ritz vectors V C, W C and residuals r_b = W c_b - lambda_b V c_b with norms (serial.zig:201-227);
//  * new directions: r_b / (diag - lambda_b) clamped at |den| >= 1e-8 (common.zig:214-226), then
//    modified Gram-Schmidt against V with a drop when the remaining norm is < 1e-8
//    (common.zig:263-284, serial.zig:250-262).  The device does this for the whole block at once:
//    project out V, then a Cholesky of the new block's Gram matrix taken column by column in the
//    reference's order, dropping a column when its Cholesky pivot (= the MGS norm) is < 1e-8, then
//    project the kept vectors out of V once more and take a second Cholesky pass (CholQR2).  This spans exactly the vectors MGS
//    keeps, in the same order; only rounding differs.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <thread>
#include <cstdio>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "kctx.cuh"

namespace dftcuda {

static const uint64_t kLcgA = 6364136223846793005ULL;

// Affine map s -> A s + C applied k times for the step s -> a s + 1.
__host__ __device__ inline void lcg_jump(uint64_t k, uint64_t& A, uint64_t& C) {
  uint64_t ra = 1, rc = 0;  // accumulated map
  uint64_t ba = kLcgA, bc = 1;  // map for 2^i steps
  while (k) {
    if (k & 1) {  // r <- b o r
      rc = ba * rc + bc;
      ra = ba * ra;
    }
    bc = ba * bc + bc;
    ba = ba * ba;
    k >>= 1;
  }
  A = ra;
  C = rc;
}

// V[col][i] = (u(2e+1) - 0.5, u(2e+2) - 0.5), e = col*n + i, u(k) = (s_k >> 11) / 2^53.
__global__ void k_lcg_fill(double2* __restrict__ V, long count, uint64_t s0) {
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (e >= count) return;
  uint64_t A, C;
  lcg_jump((uint64_t)(2 * e + 1), A, C);
  const uint64_t s1 = A * s0 + C;
  const uint64_t s2 = kLcgA * s1 + 1;
  const double re = (double)(s1 >> 11) / 9007199254740992.0 - 0.5;
  const double im = (double)(s2 >> 11) / 9007199254740992.0 - 0.5;
  V[e] = make_double2(re, im);
}

// Rayleigh-Ritz matrix from the persistent Gram store Tk (leading dimension ld).  Columns
// [m_old, m) of Tk hold the fresh products V[0:m]^H W[m_old:m]; the rows [m_old, m) to their left
// are the conjugate mirror (H is Hermitian, so V_new^H W_old = (V_old^H W_new)^H), and the new
// diagonal block is hermitised as (T + T^H) / 2 (common.zig:231-259).  Writes T (ld m).
__global__ void k_gram_finish(const double2* __restrict__ Tk, long ld, int m_old, int m, double2* __restrict__ T) {
  const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (idx >= (long)m * m) return;
  const int i = (int)(idx % m), j = (int)(idx / m);
  double2 v;
  if (j < m_old && i < m_old) {
    v = Tk[i + j * ld];
  } else if (i < m_old) {
    v = Tk[i + j * ld];
  } else if (j < m_old) {
    v = cconj(Tk[j + i * ld]);
  } else if (i == j) {
    v = make_double2(Tk[i + j * ld].x, 0.0);
  } else {
    const double2 a = Tk[i + j * ld], b = Tk[j + i * ld];
    v = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y - b.y));
  }
  T[idx] = v;
}

__global__ void k_gram_store(const double2* __restrict__ T, int m, double2* __restrict__ Tk, long ld) {
  const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (idx >= (long)m * m) return;
  const int i = (int)(idx % m), j = (int)(idx / m);
  Tk[i + j * ld] = T[idx];
}

// Cyclic two-sided Jacobi for a Hermitian m x m matrix (column-major), one CTA.  Each round applies
// m/2 disjoint rotations chosen by the circle method.  Writes ascending eigenvalues and the
// matching eigenvectors (columns of E).  status: 0 ok, 1 not converged.
__global__ void __launch_bounds__(1024) k_jacobi(double2* __restrict__ A, double2* __restrict__ U,
                                                 double* __restrict__ evals, double2* __restrict__ E, int m,
                                                 int max_sweeps, double rel_tol, int* __restrict__ status) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int m2 = m + (m & 1);
  const int npair = m2 / 2;
  // 16-byte members first so every array stays aligned for any npair.
  double2* pe = reinterpret_cast<double2*>(smraw);  // e^{-i phi}
  double* pc = reinterpret_cast<double*>(smraw + sizeof(double2) * npair);
  double* ps = pc + npair;
  int2* pq = reinterpret_cast<int2*>(ps + npair);
  __shared__ double red[1024];
  __shared__ int conv;
  const int tid = threadIdx.x, nt = blockDim.x;
  for (long i = tid; i < (long)m * m; i += nt) {
    const int r = (int)(i % m), c = (int)(i / m);
    U[i] = make_double2(r == c ? 1.0 : 0.0, 0.0);
  }
  __syncthreads();
  int sweep = 0;
  for (; sweep <= max_sweeps; ++sweep) {
    double off = 0.0, tot = 0.0;
    for (long i = tid; i < (long)m * m; i += nt) {
      const int r = (int)(i % m), c = (int)(i / m);
      const double2 v = A[i];
      const double a2 = v.x * v.x + v.y * v.y;
      tot += a2;
      if (r != c) off += a2;
    }
    red[tid] = off;
    __syncthreads();
    for (int w = nt / 2; w > 0; w >>= 1) {
      if (tid < w) red[tid] += red[tid + w];
      __syncthreads();
    }
    const double off_s = red[0];
    __syncthreads();
    red[tid] = tot;
    __syncthreads();
    for (int w = nt / 2; w > 0; w >>= 1) {
      if (tid < w) red[tid] += red[tid + w];
      __syncthreads();
    }
    const double tot_s = red[0];
    if (tid == 0) conv = (off_s <= rel_tol * rel_tol * tot_s) || tot_s == 0.0;
    __syncthreads();
    if (conv || sweep == max_sweeps) break;
    for (int rnd = 0; rnd < m2 - 1; ++rnd) {
      for (int k = tid; k < npair; k += nt) {
        int p, q;
        if (k == 0) {
          p = rnd;
          q = m2 - 1;
        } else {
          p = (rnd + k) % (m2 - 1);
          q = (rnd - k + (m2 - 1)) % (m2 - 1);
        }
        if (p > q) { const int t = p; p = q; q = t; }
        pq[k] = make_int2(p, q);
        double c = 1.0, s = 0.0;
        double2 e = make_double2(1.0, 0.0);
        if (q < m) {
          const double app = A[p + (long)p * m].x, aqq = A[q + (long)q * m].x;
          const double2 apq = A[p + (long)q * m];
          const double b = hypot(apq.x, apq.y);
          if (b > 1e-300) {
            e = make_double2(apq.x / b, -apq.y / b);  // e^{-i phi}
            const double zeta = (aqq - app) / (2.0 * b);
            const double t = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
            c = 1.0 / sqrt(1.0 + t * t);
            s = t * c;
          }
        }
        pc[k] = c;
        ps[k] = s;
        pe[k] = e;
      }
      __syncthreads();
      // A <- A G and U <- U G (columns p, q)
      for (long i = tid; i < (long)m * npair; i += nt) {
        const int k = (int)(i / m), r = (int)(i - (long)k * m);
        const int2 ij = pq[k];
        if (ij.y >= m || ps[k] == 0.0) continue;
        const double c = pc[k], s = ps[k];
        const double2 e = pe[k];
        double2* ap = A + r + (long)ij.x * m;
        double2* aq = A + r + (long)ij.y * m;
        const double2 x = *ap, y = *aq;
        const double2 ey = cmul(e, y);
        *ap = make_double2(c * x.x - s * ey.x, c * x.y - s * ey.y);
        *aq = make_double2(s * x.x + c * ey.x, s * x.y + c * ey.y);
        double2* up = U + r + (long)ij.x * m;
        double2* uq = U + r + (long)ij.y * m;
        const double2 ux = *up, uy = *uq;
        const double2 euy = cmul(e, uy);
        *up = make_double2(c * ux.x - s * euy.x, c * ux.y - s * euy.y);
        *uq = make_double2(s * ux.x + c * euy.x, s * ux.y + c * euy.y);
      }
      __syncthreads();
      // A <- G^H A (rows p, q)
      for (long i = tid; i < (long)m * npair; i += nt) {
        const int k = (int)(i / m), col = (int)(i - (long)k * m);
        const int2 ij = pq[k];
        if (ij.y >= m || ps[k] == 0.0) continue;
        const double c = pc[k], s = ps[k];
        const double2 ec = cconj(pe[k]);  // e^{+i phi}
        double2* ap = A + ij.x + (long)col * m;
        double2* aq = A + ij.y + (long)col * m;
        const double2 x = *ap, y = *aq;
        const double2 ey = cmul(ec, y);
        *ap = make_double2(c * x.x - s * ey.x, c * x.y - s * ey.y);
        *aq = make_double2(s * x.x + c * ey.x, s * x.y + c * ey.y);
      }
      __syncthreads();
      for (int k = tid; k < npair; k += nt) {
        const int2 ij = pq[k];
        if (ij.y >= m || ps[k] == 0.0) continue;
        A[ij.x + (long)ij.y * m] = make_double2(0.0, 0.0);
        A[ij.y + (long)ij.x * m] = make_double2(0.0, 0.0);
        A[ij.x + (long)ij.x * m].y = 0.0;
        A[ij.y + (long)ij.y * m].y = 0.0;
      }
      __syncthreads();
    }
  }
  if (tid == 0) *status = conv ? 0 : 1;
  // rank sort (ascending, ties by index) and gather eigenvectors
  for (int i = tid; i < m; i += nt) {
    const double di = A[i + (long)i * m].x;
    int rank = 0;
    for (int j = 0; j < m; ++j) {
      const double dj = A[j + (long)j * m].x;
      rank += (dj < di) || (dj == di && j < i);
    }
    evals[rank] = di;
    for (int r = 0; r < m; ++r) E[r + (long)rank * m] = U[r + (long)i * m];
  }
}

// res[b] -= lambda_b ritz[b]; norms[b] = ||res[b]||   (serial.zig:218-227)
__global__ void k_residual(double2* __restrict__ res, const double2* __restrict__ ritz, const double* __restrict__ lam,
                           long n, double* __restrict__ norms) {
  const int b = blockIdx.x;
  const double l = lam[b];
  double2* r = res + (long)b * n;
  const double2* x = ritz + (long)b * n;
  double s = 0.0;
  for (long i = threadIdx.x; i < n; i += blockDim.x) {
    double2 v = r[i];
    const double2 xv = x[i];
    v.x -= l * xv.x;
    v.y -= l * xv.y;
    r[i] = v;
    s += v.x * v.x + v.y * v.y;
  }
  __shared__ double red[256];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) norms[b] = sqrt(red[0]);
}

// Q[j] = res[band[j]] / (diag - lambda[band[j]]), |den| clamped to 1e-8 keeping its sign (common.zig:214-226)
__global__ void k_precondition(double2* __restrict__ Q, const double2* __restrict__ res, const double* __restrict__ diag,
                               const double* __restrict__ lam, const int* __restrict__ band, int k, long n) {
  const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (idx >= (long)k * n) return;
  const int j = (int)(idx / n);
  const long i = idx - (long)j * n;
  const int b = band[j];
  double den = diag[i] - lam[b];
  if (fabs(den) < 1e-8) den = den >= 0.0 ? 1e-8 : -1e-8;
  const double inv = 1.0 / den;
  const double2 v = res[(long)b * n + i];
  Q[idx] = make_double2(v.x * inv, v.y * inv);
}

// Cholesky of the k x k Gram matrix G (column-major) in column order with the MGS drop rule: column
// j is dropped when its pivot sqrt(d) < drop, where d, the Schur-complement diagonal after the kept
// columns before j, is exactly the squared norm MGS leaves (common.zig:263-284).  Right-looking: each
// kept column scales its row and updates the whole trailing upper triangle in parallel; dropped
// columns update nothing.  A: k x k row-major workspace (its kept rows end up as R); kept[0..kk),
// *kk_out.  One CTA; the working triangle stays in L2.
__global__ void __launch_bounds__(1024) k_chol_right(const double2* __restrict__ G, int k, double drop,
                                                     double2* __restrict__ A, int* __restrict__ kept, int* __restrict__ kk_out) {
  __shared__ double s_piv;
  __shared__ int s_nk;
  const int tid = threadIdx.x, nt = blockDim.x;
  for (long idx = tid; idx < (long)k * k; idx += nt) {
    const int j = (int)(idx / k), l = (int)(idx - (long)j * k);
    if (l >= j) A[idx] = G[j + (long)l * k];
  }
  if (tid == 0) s_nk = 0;
  __syncthreads();
  for (int j = 0; j < k; ++j) {
    if (tid == 0) {
      const double d = A[(long)j * k + j].x;
      s_piv = d > 0.0 ? sqrt(d) : 0.0;
    }
    __syncthreads();
    const double piv = s_piv;
    if (!(piv >= drop) || piv == 0.0) {
      __syncthreads();
      continue;
    }
    const double inv = 1.0 / piv;
    double2* rj = A + (long)j * k;
    for (int l = j + 1 + tid; l < k; l += nt) rj[l] = make_double2(rj[l].x * inv, rj[l].y * inv);
    if (tid == 0) {
      rj[j] = make_double2(piv, 0.0);
      kept[s_nk] = j;
      s_nk = s_nk + 1;
    }
    __syncthreads();
    // A[l1][l2] -= conj(R[j][l1]) R[j][l2] for j < l1 <= l2 < k
    const int n = k - j - 1;
    for (long idx = tid; idx < (long)n * n; idx += nt) {
      const int a1 = (int)(idx / n), a2 = (int)(idx - (long)a1 * n);
      if (a1 > a2) continue;
      const int l1 = j + 1 + a1, l2 = j + 1 + a2;
      const double2 x = rj[l1], y = rj[l2];
      double2* t = A + (long)l1 * k + l2;
      double2 v = *t;
      v.x -= x.x * y.x + x.y * y.y;
      v.y -= x.x * y.y - x.y * y.x;
      *t = v;
    }
    __syncthreads();
  }
  if (tid == 0) *kk_out = s_nk;
}

// Blocked form of the same factorisation for larger blocks.  k_chol_init copies G's upper triangle
// into A (row-major) over the whole grid and resets the kept count; then per panel of rows
// [j0, j1) one CTA loads the panel's rows (columns j0 .. k-1) into shared memory, factors them there
// (pivots, drops, row scaling and the updates among the panel's own rows), and writes them back;
// the panel's rank-(j1 - j0) update of the trailing triangle is an FP64 GEMM.  Dropped rows are
// zeroed so they add nothing to the GEMM.  The panel width keeps its rows within kChPanelSmem.
constexpr int kChPanelMax = 32;
constexpr size_t kChPanelSmem = 200 * 1024;

__global__ void k_chol_init(const double2* __restrict__ G, int k, double2* __restrict__ A, int* __restrict__ kk) {
  const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (idx == 0) *kk = 0;
  if (idx >= (long)k * k) return;
  const int j = (int)(idx / k), l = (int)(idx - (long)j * k);
  if (l >= j) A[idx] = G[j + (long)l * k];
}

__global__ void __launch_bounds__(1024) k_chol_panel(double2* __restrict__ A, int k, double drop, int* __restrict__ kept,
                                                     int* __restrict__ kk, int j0, int j1) {
  extern __shared__ double2 cps[];  // [j1 - j0][k - j0]: row j0 + r, column j0 + c at cps[r * nc + c]
  __shared__ double s_piv;
  __shared__ int s_nk;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int nc = k - j0, rows = j1 - j0;
  for (long idx = tid; idx < (long)rows * nc; idx += nt) {
    const int r = (int)(idx / nc), c = (int)(idx - (long)r * nc);
    cps[idx] = A[(long)(j0 + r) * k + j0 + c];
  }
  if (tid == 0) s_nk = *kk;
  __syncthreads();
  for (int jl = 0; jl < rows; ++jl) {  // row j = j0 + jl; its diagonal at column jl
    double2* rj = cps + (long)jl * nc;
    if (tid == 0) {
      const double d = rj[jl].x;
      s_piv = d > 0.0 ? sqrt(d) : 0.0;
    }
    __syncthreads();
    const double piv = s_piv;
    if (!(piv >= drop) || piv == 0.0) {
      for (int c = jl + tid; c < nc; c += nt) rj[c] = make_double2(0.0, 0.0);
      __syncthreads();
      continue;
    }
    const double inv = 1.0 / piv;
    for (int c = jl + 1 + tid; c < nc; c += nt) rj[c] = make_double2(rj[c].x * inv, rj[c].y * inv);
    if (tid == 0) {
      rj[jl] = make_double2(piv, 0.0);
      kept[s_nk] = j0 + jl;
      s_nk = s_nk + 1;
    }
    __syncthreads();
    // the panel's rows after j: A[j'][l] -= conj(R[j][j']) R[j][l] for l >= j'
    const int nr = rows - jl - 1, nu = nc - jl - 1;
    for (long idx = tid; idx < (long)nr * nu; idx += nt) {
      const int a = (int)(idx / nu), b = (int)(idx - (long)a * nu);
      const int rr = jl + 1 + a, c = jl + 1 + b;
      if (c < rr) continue;
      const double2 x = rj[rr], y = rj[c];
      double2* t = cps + (long)rr * nc + c;
      double2 v = *t;
      v.x -= x.x * y.x + x.y * y.y;
      v.y -= x.x * y.y - x.y * y.x;
      *t = v;
    }
    __syncthreads();
  }
  for (long idx = tid; idx < (long)rows * nc; idx += nt) {
    const int r = (int)(idx / nc), c = (int)(idx - (long)r * nc);
    A[(long)(j0 + r) * k + j0 + c] = cps[idx];
  }
  if (tid == 0) *kk = s_nk;
}

// Z (k x k columns, ld k): column b < kk solves R_kept z = e_b on the kept rows (rows of dropped
// columns zero), so Q Z has orthonormal columns; columns b >= kk are zeroed.  One warp per column,
// the back substitution's dot products split over the lanes; the column being solved and the kept
// index table live in shared memory, so each of the (up to k - 1) dependent steps waits only on
// shared-memory and L1 latency.
constexpr int kCiWarps = 4;
__global__ void __launch_bounds__(kCiWarps * 32) k_chol_inv(const double2* __restrict__ A, int k, const int* __restrict__ kept,
                                                            const int* __restrict__ kk_p, double2* __restrict__ Z) {
  extern __shared__ __align__(16) unsigned char cism[];
  double2* zs = reinterpret_cast<double2*>(cism);                // [kCiWarps][k]
  int* skept = reinterpret_cast<int*>(zs + (size_t)kCiWarps * k);  // [k]
  const int kk = *kk_p;
  for (int i = threadIdx.x; i < kk; i += blockDim.x) skept[i] = kept[i];
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int b = blockIdx.x * kCiWarps + w;
  if (b >= k) return;
  double2* z = zs + (size_t)w * k;
  for (int i = lane; i < k; i += 32) z[i] = make_double2(0.0, 0.0);
  __syncwarp();
  if (b < kk) {
    const int kb = skept[b];
    if (lane == 0) z[kb] = make_double2(1.0 / A[(long)kb * k + kb].x, 0.0);
    __syncwarp();
    for (int a = b - 1; a >= 0; --a) {
      const int ka = skept[a];
      const double2* ra = A + (long)ka * k;
      double sx = 0.0, sy = 0.0;
      for (int u = a + 1 + lane; u <= b; u += 32) {
        const int ku = skept[u];
        const double2 r = __ldg(ra + ku), zz = z[ku];
        sx += r.x * zz.x - r.y * zz.y;
        sy += r.x * zz.y + r.y * zz.x;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        sx += __shfl_xor_sync(0xffffffffu, sx, o);
        sy += __shfl_xor_sync(0xffffffffu, sy, o);
      }
      if (lane == 0) {
        const double d = ra[ka].x;
        z[ka] = make_double2(-sx / d, -sy / d);
      }
      __syncwarp();
    }
  }
  double2* zo = Z + (long)b * k;
  for (int i = lane; i < k; i += 32) zo[i] = z[i];
}


// ------------------------------------------------------------------------------------------

constexpr size_t kVTileCacheBytes = (size_t)8 << 30;  // both V tile caches of one context

struct KCtxImpl {
  size_t n = 0, max_sub = 0, nb = 0, kmax = 0;
  double2 *V = nullptr, *W = nullptr, *ritz = nullptr, *res = nullptr, *Q = nullptr, *Q2 = nullptr;
  double2 *Tk = nullptr;  // persistent Rayleigh-Ritz matrix, leading dimension max_sub
  double2 *T = nullptr, *U = nullptr, *E = nullptr, *H = nullptr, *G = nullptr, *R = nullptr, *Z = nullptr;
  double *evals = nullptr, *norms = nullptr, *diag = nullptr, *ekin = nullptr;
  int *band = nullptr, *kept = nullptr, *status = nullptr;
  double2* ws = nullptr;
  size_t ws_elems = 0;
  void* all = nullptr;
  void* heev_mem = nullptr;
  HeevWork hw;
  bool rr_tc = false;  // Rayleigh-Ritz products on the tensor cores (3xTF32), TF32/TF32X3 contexts
  int* err = nullptr;  // the context's tensor-core error flag
  TcScratch* tcs = nullptr;  // the context's pre-split operand buffer
  // Pre-split tiles of V[0:m] in its two roles (the Gram operand V^H, and the combination V C), kept
  // while V[0:m] is unchanged: the Rayleigh-Ritz products and both orthonormalisation passes of an
  // iteration read the same V[0:m], so each role is split once per iteration instead of three times.
  // Used when both fit kVTileCacheBytes; invalidated wherever V's leading columns are rewritten.
  TcScratch vt_gram, vt_comb;
  bool v_cache = false;
  double tc_min_flops = 0.0;  // smaller products take the FP64 GEMM (dftcuda_kctx::tc_min_flops)
  // pinned host mirrors of the per-iteration read-backs
  void* pinned = nullptr;
  double *h_ev = nullptr, *h_nr = nullptr;
  int *h_st = nullptr, *h_kk = nullptr, *h_band = nullptr;
};

void eig_destroy(KCtxImpl* e) {
  if (!e) return;
  e->vt_gram.release();
  e->vt_comb.release();
  if (e->all) cudaFree(e->all);
  if (e->ws) cudaFree(e->ws);
  if (e->heev_mem) cudaFree(e->heev_mem);
  if (e->pinned) cudaFreeHost(e->pinned);
  delete e;
}

static int eig_alloc(dftcuda_kctx* c, size_t n, size_t max_sub, size_t nb) {
  KCtxImpl* e = c->eig;
  const size_t kmax = max_sub;
  if (e && e->n == n && e->max_sub >= max_sub && e->nb >= nb) return DFTCUDA_OK;
  eig_destroy(e);
  e = c->eig = new KCtxImpl();
  e->n = n; e->max_sub = max_sub; e->nb = nb; e->kmax = kmax;
  const size_t ms2 = max_sub * max_sub;
  size_t off = 0;
  auto take = [&](size_t bytes) { const size_t o = off; off += (bytes + 255) / 256 * 256; return o; };
  const size_t oV = take(sizeof(double2) * n * max_sub), oW = take(sizeof(double2) * n * max_sub);
  const size_t oRi = take(sizeof(double2) * n * nb), oRe = take(sizeof(double2) * n * nb);
  const size_t oQ = take(sizeof(double2) * n * kmax), oQ2 = take(sizeof(double2) * n * kmax);
  const size_t oT = take(sizeof(double2) * ms2), oU = take(sizeof(double2) * ms2), oE = take(sizeof(double2) * ms2);
  const size_t oH = take(sizeof(double2) * ms2), oG = take(sizeof(double2) * ms2), oR = take(sizeof(double2) * ms2);
  const size_t oZ = take(sizeof(double2) * ms2), oTk = take(sizeof(double2) * ms2);
  const size_t oev = take(sizeof(double) * max_sub), onr = take(sizeof(double) * nb), odg = take(sizeof(double) * n);
  const size_t oek = take(sizeof(double) * kmax);
  const size_t obd = take(sizeof(int) * kmax), okp = take(sizeof(int) * kmax), ost = take(sizeof(int) * 4);
  if (dev_malloc(&e->all, off) != cudaSuccess) {
    eig_destroy(e);
    c->eig = nullptr;
    return fail(DFTCUDA_ERR_OUT_OF_MEMORY, "eigensolver workspace");
  }
  char* b = (char*)e->all;
  e->V = (double2*)(b + oV); e->W = (double2*)(b + oW); e->ritz = (double2*)(b + oRi); e->res = (double2*)(b + oRe);
  e->Q = (double2*)(b + oQ); e->Q2 = (double2*)(b + oQ2); e->T = (double2*)(b + oT); e->U = (double2*)(b + oU);
  e->E = (double2*)(b + oE); e->H = (double2*)(b + oH); e->G = (double2*)(b + oG); e->R = (double2*)(b + oR);
  e->Z = (double2*)(b + oZ); e->Tk = (double2*)(b + oTk); e->evals = (double*)(b + oev); e->norms = (double*)(b + onr); e->diag = (double*)(b + odg); e->ekin = (double*)(b + oek);
  e->band = (int*)(b + obd); e->kept = (int*)(b + okp); e->status = (int*)(b + ost);
  size_t need = 0;
  const int ms = (int)max_sub;
  need = std::max(need, zgemm_workspace_elems(ms, ms, (int)n));
  need = std::max(need, zgemm_workspace_elems((int)nb, (int)n, ms));
  need = std::max(need, zgemm_workspace_elems(ms, (int)kmax, (int)n));
  need = std::max(need, zgemm_workspace_elems((int)kmax, (int)n, ms));
  need = std::max(need, zgemm_workspace_elems((int)kmax, (int)kmax, (int)n));
  need = std::max(need, cgemm_tf32_workspace_elems(ms, ms, (int)n));
  need = std::max(need, cgemm_tf32_workspace_elems((int)nb, (int)n, ms));
  need = std::max(need, cgemm_tf32_workspace_elems(ms, (int)kmax, (int)n));
  need = std::max(need, cgemm_tf32_workspace_elems((int)kmax, (int)n, ms));
  need = std::max(need, cgemm_tf32_workspace_elems((int)kmax, (int)kmax, (int)n));
  // a workspace that could not be completed is dropped, so the next call allocates it afresh
  auto out_of_memory = [&](const char* what) {
    eig_destroy(e);
    c->eig = nullptr;
    return fail(DFTCUDA_ERR_OUT_OF_MEMORY, what);
  };
  if (need) {
    if (dev_malloc(&e->ws, need * sizeof(double2)) != cudaSuccess) return out_of_memory("eig gemm ws");
    e->ws_elems = need;
  }
  if (dev_malloc(&e->heev_mem, heev_work_bytes(ms, (int)nb)) != cudaSuccess) return out_of_memory("eig heev ws");
  heev_bind(e->hw, e->heev_mem, ms, (int)nb);
  const size_t pin_bytes = sizeof(double) * 2 * nb + sizeof(int) * (8 + kmax);
  if (cudaMallocHost(&e->pinned, pin_bytes) != cudaSuccess) return out_of_memory("eig pinned host buffers");
  e->h_ev = (double*)e->pinned;
  e->h_nr = e->h_ev + nb;
  e->h_st = (int*)(e->h_nr + nb);
  e->h_kk = e->h_st + 4;
  e->h_band = e->h_st + 8;
  return DFTCUDA_OK;
}

// Gram products on blocks stored as rows of length n ("vector blocks", column-major [n x cols]).
// out[i + j*ldo] = sum_g conj(X[i][g]) Y[j][g]
// In TF32 / TF32X3 contexts every subspace product (Rayleigh-Ritz V^H W, V C, W C and the
// orthonormalisation's projections and block overlaps) runs on the tensor cores in the split-TF32
// form (FP32-class accuracy); the Cholesky factorisations, the subspace eigensolver and the residual
// norms stay FP64.  FP64 and FP32 contexts use the FP64 GEMM throughout.
static int gemm_dispatch(KCtxImpl* e, const GemmArgs& g, bool /*rr*/, cudaStream_t s) {
  if (e->rr_tc && tc_worthwhile(g.M, g.N, g.K, e->tc_min_flops)) return cgemm_tf32(g, s, e->ws, e->ws_elems, e->err, true, e->tcs);
  return zgemm(g, s, e->ws, e->ws_elems);
}

static int gram(KCtxImpl* e, const double2* X, int mx, const double2* Y, int my, double2* out, int ldo, cudaStream_t s,
                bool rr = false) {
  GemmArgs g{};
  g.M = mx; g.N = my; g.K = (int)e->n;
  g.A = X; g.lda = (long)e->n; g.a_kc = true; g.conj_a = true;
  if (e->v_cache && X == e->V) g.a_cache = &e->vt_gram;
  g.B = Y; g.ldb = (long)e->n; g.b_kc = true; g.conj_b = false;
  g.O = out; g.ldo_r = 1; g.ldo_c = ldo;
  g.alpha = 1.0; g.beta = 0.0;
  return gemm_dispatch(e, g, rr, s);
}

// Out[j][g] = alpha * sum_i X[i][g] C[i + j*ldc] + beta * Out[j][g]
static int combine(KCtxImpl* e, const double2* X, int mx, const double2* C, int ldc, int ncols, double2* out,
                   double alpha, double beta, cudaStream_t s, bool rr = false) {
  GemmArgs g{};
  g.M = ncols; g.N = (int)e->n; g.K = mx;
  g.A = C; g.lda = ldc; g.a_kc = true; g.conj_a = false;
  g.B = X; g.ldb = (long)e->n; g.b_kc = false; g.conj_b = false;
  if (e->v_cache && X == e->V) g.b_cache = &e->vt_comb;
  g.O = out; g.ldo_r = (long)e->n; g.ldo_c = 1;
  g.alpha = alpha; g.beta = beta;
  return gemm_dispatch(e, g, rr, s);
}

// Cholesky with the drop rule of the k x k Gram matrix G into e->R / e->kept, kept count at kk_dev,
// then Z = the inverse on the kept rows.  One CTA below 97 columns, the panel form above.
static int chol_drop(KCtxImpl* e, const double2* G, int k, double drop, int* kk_dev, cudaStream_t s) {
  if (k <= 96) {
    k_chol_right<<<1, 1024, 0, s>>>(G, k, drop, e->R, e->kept, kk_dev);
    count_launch();
  } else {
    k_chol_init<<<ceil_div((size_t)k * k, 256), 256, 0, s>>>(G, k, e->R, kk_dev);
    count_launch();
    DFT_TRY(ensure_max_dynamic_smem((const void*)k_chol_panel, (int)kChPanelSmem));
    for (int j0 = 0; j0 < k;) {
      const int w = (int)std::max<size_t>(1, std::min<size_t>(kChPanelMax, kChPanelSmem / (sizeof(double2) * (size_t)(k - j0))));
      const int j1 = std::min(k, j0 + w);
      k_chol_panel<<<1, 1024, sizeof(double2) * (size_t)(j1 - j0) * (k - j0), s>>>(e->R, k, drop, e->kept, kk_dev, j0, j1);
      count_launch();
      if (j1 < k) {
        // A[l1][l2] -= sum_{j in panel} conj(R[j][l1]) R[j][l2], l1, l2 >= j1 (the lower triangle
        // of A is scratch)
        GemmArgs g{};
        g.M = k - j1; g.N = k - j1; g.K = j1 - j0;
        g.A = e->R + (size_t)j0 * k + j1; g.lda = k; g.a_kc = false; g.conj_a = true;
        g.B = e->R + (size_t)j0 * k + j1; g.ldb = k; g.b_kc = false; g.conj_b = false;
        g.O = e->R + (size_t)j1 * k + j1; g.ldo_r = k; g.ldo_c = 1;
        g.alpha = -1.0; g.beta = 1.0;
        DFT_TRY(zgemm(g, s, e->ws, e->ws_elems));
      }
      j0 = j1;
    }
  }
  const size_t ci_smem = sizeof(double2) * kCiWarps * (size_t)k + sizeof(int) * (size_t)k;
  // k <= 1024: at most 68 KB
  DFT_TRY(ensure_max_dynamic_smem((const void*)k_chol_inv, (int)(sizeof(double2) * kCiWarps * 1024 + sizeof(int) * 1024)));
  k_chol_inv<<<ceil_div(k, kCiWarps), kCiWarps * 32, ci_smem, s>>>(e->R, k, e->kept, kk_dev, e->Z);
  count_launch();
  DFT_CUDA_TRY(cudaGetLastError());
  return DFTCUDA_OK;
}

// Orthonormalise the k vectors in Q against V[0:m] and among themselves (in order), writing the kept
// vectors to dst.  Two phases around one host read of the kept count: phase A projects out V once
// and takes the dropping Cholesky of the block's Gram matrix (kept count -> e->h_kk, pinned);
// phase B (after the stream is synchronised) forms the kept vectors and their second CholQR pass.
static int block_orth_a(KCtxImpl* e, int m, double2* Q, int k, cudaStream_t s) {
  if (k > 1024) return fail(DFTCUDA_ERR_UNSUPPORTED, "block_orthonormalize: more than 1024 new vectors");
  // One classical projection pass here; phase B projects the kept vectors once more before their
  // second Cholesky (classical Gram-Schmidt twice, with the drop test taken after the first pass:
  // the first pass leaves components along V of order eps ||q||, far below the 1e-8 drop norm).
  if (m > 0) {
    DFT_TRY(gram(e, e->V, m, Q, k, e->H, m, s));
    DFT_TRY(combine(e, e->V, m, e->H, m, k, Q, -1.0, 1.0, s));
  }
  DFT_TRY(gram(e, Q, k, Q, k, e->G, k, s));
  DFT_TRY(chol_drop(e, e->G, k, 1e-8, e->status + 1, s));
  DFT_CUDA_TRY(cudaMemcpyAsync(e->h_kk, e->status + 1, sizeof(int), cudaMemcpyDeviceToHost, s));
  return DFTCUDA_OK;
}

static int block_orth_b(KCtxImpl* e, int m, double2* Q, int k, double2* dst, int kk, cudaStream_t s) {
  if (kk <= 0) return DFTCUDA_OK;
  DFT_TRY(combine(e, Q, k, e->Z, k, kk, e->Q2, 1.0, 0.0, s));
  // second pass (CholQR2) without drops
  if (m > 0) {
    DFT_TRY(gram(e, e->V, m, e->Q2, kk, e->H, m, s));
    DFT_TRY(combine(e, e->V, m, e->H, m, kk, e->Q2, -1.0, 1.0, s));
  }
  DFT_TRY(gram(e, e->Q2, kk, e->Q2, kk, e->G, kk, s));
  DFT_TRY(chol_drop(e, e->G, kk, 0.0, e->status + 2, s));
  DFT_TRY(combine(e, e->Q2, kk, e->Z, kk, kk, dst, 1.0, 0.0, s));
  return DFTCUDA_OK;
}

// Both phases with the synchronisation in between; kept_host receives the kept indices (into Q).
static int block_orthonormalize(dftcuda_kctx* c, int m, double2* Q, int k, double2* dst, int* kk,
                                std::vector<int>& kept_host, cudaStream_t s) {
  KCtxImpl* e = c->eig;
  DFT_TRY(block_orth_a(e, m, Q, k, s));
  DFT_CUDA_TRY(cudaStreamSynchronize(s));
  const int h_kk = *e->h_kk;
  kept_host.assign(h_kk, 0);
  if (h_kk > 0) {
    DFT_CUDA_TRY(cudaMemcpyAsync(kept_host.data(), e->kept, sizeof(int) * h_kk, cudaMemcpyDeviceToHost, s));
    DFT_TRY(block_orth_b(e, m, Q, k, dst, h_kk, s));
    DFT_CUDA_TRY(cudaStreamSynchronize(s));
  }
  *kk = h_kk;
  return DFTCUDA_OK;
}

// Subspace sizes from which the tridiagonal solver replaces the one-CTA Jacobi sweeps (whose cost
// grows as m^3 on a single SM).  DFTCUDA_SUBSPACE_EIG=jacobi|tridiag forces either.
constexpr int kTridiagMinM = 96;

static int small_eig(KCtxImpl* e, int m, int nev, cudaStream_t s) {
  const char* force = std::getenv("DFTCUDA_SUBSPACE_EIG");
  const bool tri = force ? (std::strcmp(force, "tridiag") == 0) : (m >= kTridiagMinM);
  if (tri) return heev_lowest(e->T, m, nev, e->evals, e->E, m, e->hw, e->status, s);
  const int m2 = m + (m & 1);
  const size_t smem = (sizeof(int2) + 2 * sizeof(double) + sizeof(double2)) * (size_t)(m2 / 2);
  DFT_TRY(ensure_max_dynamic_smem((const void*)k_jacobi, 160 * 1024));
  k_jacobi<<<1, 1024, smem, s>>>(e->T, e->U, e->evals, e->E, m, 60, 1e-14, e->status); count_launch();
  DFT_CUDA_TRY(cudaGetLastError());
  return DFTCUDA_OK;
}

// V's leading columns were rewritten: the tiles cached from them are stale.
static void v_changed(KCtxImpl* e) {
  e->vt_gram.valid = false;
  e->vt_comb.valid = false;
}

// orthonormalize_all (common.zig:298-312) for V[0:m]: block Gram-Schmidt; columns that drop are
// replaced by fresh LCG vectors (the reference's retry) and the block is redone, at most 3 times.
// Every caller has just written V[0:m] (start, restart), and this rewrites it.
static int orthonormalize_all(dftcuda_kctx* c, int m, uint64_t& seed, cudaStream_t s) {
  KCtxImpl* e = c->eig;
  struct Invalidate {
    KCtxImpl* e;
    ~Invalidate() { v_changed(e); }
  } inv{e};
  v_changed(e);
  const long n = (long)e->n;
  for (int attempt = 0; attempt < 4; ++attempt) {
    DFT_CUDA_TRY(cudaMemcpyAsync(e->Q, e->V, sizeof(double2) * n * m, cudaMemcpyDeviceToDevice, s));
    int kk = 0;
    std::vector<int> kept;
    DFT_TRY(block_orthonormalize(c, 0, e->Q, m, e->V, &kk, kept, s));
    if (kk == m) return DFTCUDA_OK;
    if (attempt == 3) break;
    // Put kept vectors back in their slots, refill dropped slots with random vectors.
    std::vector<char> ok(m, 0);
    for (int t = 0; t < kk; ++t) ok[kept[t]] = 1;
    DFT_CUDA_TRY(cudaMemcpyAsync(e->Q2, e->V, sizeof(double2) * n * kk, cudaMemcpyDeviceToDevice, s));
    for (int t = 0; t < kk; ++t)
      DFT_CUDA_TRY(cudaMemcpyAsync(e->V + (long)kept[t] * n, e->Q2 + (long)t * n, sizeof(double2) * n,
                                   cudaMemcpyDeviceToDevice, s));
    for (int j = 0; j < m; ++j) {
      if (ok[j]) continue;
      k_lcg_fill<<<ceil_div(n, 256), 256, 0, s>>>(e->V + (long)j * n, n, seed); count_launch();
      uint64_t A, C;
      lcg_jump(2 * (uint64_t)n, A, C);
      seed = A * seed + C;
    }
  }
  return fail(DFTCUDA_ERR_INVALID_MATRIX_SIZE, "orthonormalize_all: could not build an orthonormal block");
}

}  // namespace dftcuda


namespace dftcuda {

// One k-point's Davidson run as a state machine, so that many k-points advance in lockstep on their
// own streams with one host synchronisation per phase for all of them (the reference runs k-points
// on worker threads, kpoint/workers.zig:133-180; here the GPU overlaps them instead).  The loop
// body follows serial.zig:55-307:
//   RR:      T = V^H W (new columns), small eigenproblem, Ritz vectors, residuals, norms  -> read-back
//   DECIDE:  convergence test; candidates ||r_b|| >= tol in band order; precondition; phase A of the
//            orthonormalisation of one chunk                                              -> read-back
//   ORTH:    phase B; more chunks while room is left; then restart or H on the new columns.
struct EigRun {
  dftcuda_kctx* c = nullptr;
  KCtxImpl* e = nullptr;
  cudaStream_t s = nullptr;
  size_t n = 0, nbands = 0, max_sub = 0, block = 0;
  dftcuda_eig_opts opts{};
  uint64_t seed = 0x6f3d3cbeULL;
  size_t m = 0, it = 0, applies = 0, t_valid = 0;
  bool done = false, converged = false, orth_pending = false;
  double max_res = 0.0;
  std::vector<int> cand;
  size_t added = 0, next = 0, take = 0;
  bool gram_full = false;
  double* values_out = nullptr;
  double* vectors_out = nullptr;
  dftcuda_eig_info* info = nullptr;
  int status = DFTCUDA_OK;
  size_t index = 0;     // position in the batch
  std::string err_msg;  // the failure message, recorded on the host thread that issued the failing call
};

static int run_init(EigRun& r, const double* diag, const double* init_vecs, size_t init_cols) {
  dftcuda_kctx* c = r.c;
  const size_t n = c->npw;
  r.n = n;
  if (r.info) *r.info = dftcuda_eig_info{0, 0, 1, 0.0};
  if (r.nbands == 0 || n == 0) {
    r.done = true;
    r.converged = true;
    return DFTCUDA_OK;
  }
  const dftcuda_eig_opts& opts = r.opts;
  r.max_sub = opts.max_subspace == 0 ? std::min(n, 4 * r.nbands + 8) : std::min(n, std::max(opts.max_subspace, r.nbands));
  r.block = opts.block_size == 0 ? std::min(r.max_sub, r.nbands + 4) : std::min(r.max_sub, std::max(opts.block_size, r.nbands));
  if (r.nbands > r.max_sub) return fail(DFTCUDA_ERR_INVALID_MATRIX_SIZE, "eig_solve: nbands exceeds the basis size");
  if (r.max_sub > 2048) return fail(DFTCUDA_ERR_UNSUPPORTED, "eig_solve: max_subspace above 2048");
  r.s = c->stream;
  cudaStream_t s = r.s;
  DFT_TRY(eig_alloc(c, n, r.max_sub, r.nbands));
  KCtxImpl* e = r.e = c->eig;
  e->rr_tc = precision_uses_tc(c->precision);
  if (e->rr_tc && !c->d_err) {
    DFT_CUDA_TRY(dev_malloc(&c->d_err, sizeof(int)));
    DFT_CUDA_TRY(cudaMemsetAsync(c->d_err, 0, sizeof(int), s));
  }
  e->err = c->d_err;
  e->tcs = &c->tc_scratch;
  v_changed(e);
  if (e->rr_tc && !e->v_cache) {
    const size_t bg = tc4_operand_bytes((int)e->max_sub, (int)n, true), bc = tc4_operand_bytes((int)n, (int)e->max_sub, true);
    if (bg + bc <= kVTileCacheBytes && e->vt_gram.ensure(bg) == DFTCUDA_OK && e->vt_comb.ensure(bc) == DFTCUDA_OK) {
      e->v_cache = true;
    } else {
      e->vt_gram.release();
      e->vt_comb.release();
    }
  }
  e->tc_min_flops = c->tc_min_flops;
  const char* gram_mode = std::getenv("DFTCUDA_GRAM");
  r.gram_full = gram_mode && std::strcmp(gram_mode, "full") == 0;
  DFT_CUDA_TRY(cudaMemcpyAsync(e->diag, diag, sizeof(double) * n,
                               is_device_pointer(diag) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
  const size_t m = r.block;
  size_t icols = 0;
  if (init_vecs) icols = std::min(m, init_cols == 0 ? r.nbands : init_cols);
  if (opts.init_diagonal) {
    std::vector<double> hd(n);
    DFT_CUDA_TRY(cudaMemcpyAsync(hd.data(), e->diag, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
    DFT_CUDA_TRY(cudaStreamSynchronize(s));
    std::vector<size_t> order(n);
    for (size_t i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return hd[a] < hd[b]; });
    DFT_CUDA_TRY(cudaMemsetAsync(e->V, 0, sizeof(double2) * n * m, s));
    const double2 one = make_double2(1.0, 0.0);
    for (size_t col = 0; col < m; ++col)
      DFT_CUDA_TRY(cudaMemcpyAsync(e->V + col * n + order[col], &one, sizeof(double2), cudaMemcpyHostToDevice, s));
    DFT_CUDA_TRY(cudaStreamSynchronize(s));
  } else {
    k_lcg_fill<<<ceil_div(n * m, 256), 256, 0, s>>>(e->V, (long)(n * m), r.seed); count_launch();
    uint64_t A, C;
    lcg_jump(2 * (uint64_t)(n * m), A, C);
    r.seed = A * r.seed + C;
  }
  if (icols) {
    DFT_CUDA_TRY(cudaMemcpyAsync(e->V, init_vecs, sizeof(double2) * n * icols,
                                 is_device_pointer(init_vecs) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
  }
  DFT_TRY(orthonormalize_all(c, (int)m, r.seed, s));
  DFT_TRY(kctx_apply_h_dev(c, e->V, e->W, m, s));
  r.applies = m;
  r.m = m;
  return DFTCUDA_OK;
}

// RR phase: everything up to the read-back of eigenvalues, residual norms and the solver status.
static int run_rr(EigRun& r) {
  KCtxImpl* e = r.e;
  cudaStream_t s = r.s;
  const size_t n = r.n;
  const int mi = (int)r.m;
  ProfScope ps_sub(r.c, P_SUBSPACE, s);
  const int m_old = r.gram_full ? 0 : (int)r.t_valid;
  const long ldt = (long)r.max_sub;
  DFT_TRY(gram(e, e->V, mi, e->W + (size_t)m_old * n, mi - m_old, e->Tk + (size_t)m_old * ldt, (int)ldt, s, true));
  k_gram_finish<<<ceil_div((size_t)mi * mi, 256), 256, 0, s>>>(e->Tk, ldt, m_old, mi, e->T); count_launch();
  k_gram_store<<<ceil_div((size_t)mi * mi, 256), 256, 0, s>>>(e->T, mi, e->Tk, ldt); count_launch();
  r.t_valid = r.m;
  DFT_TRY(small_eig(e, mi, (int)r.nbands, s));
  DFT_TRY(combine(e, e->V, mi, e->E, mi, (int)r.nbands, e->ritz, 1.0, 0.0, s, true));
  DFT_TRY(combine(e, e->W, mi, e->E, mi, (int)r.nbands, e->res, 1.0, 0.0, s, true));
  k_residual<<<(unsigned)r.nbands, 256, 0, s>>>(e->res, e->ritz, e->evals, (long)n, e->norms); count_launch();
  DFT_CUDA_TRY(cudaMemcpyAsync(e->h_ev, e->evals, sizeof(double) * r.nbands, cudaMemcpyDeviceToHost, s));
  DFT_CUDA_TRY(cudaMemcpyAsync(e->h_nr, e->norms, sizeof(double) * r.nbands, cudaMemcpyDeviceToHost, s));
  DFT_CUDA_TRY(cudaMemcpyAsync(e->h_st, e->status, sizeof(int), cudaMemcpyDeviceToHost, s));
  return DFTCUDA_OK;
}

// Precondition the next chunk of candidates and launch phase A of its orthonormalisation.
static int run_orth_a(EigRun& r) {
  KCtxImpl* e = r.e;
  cudaStream_t s = r.s;
  r.take = std::min(r.max_sub - (r.m + r.added), r.cand.size() - r.next);
  std::memcpy(e->h_band, r.cand.data() + r.next, sizeof(int) * r.take);
  DFT_CUDA_TRY(cudaMemcpyAsync(e->band, e->h_band, sizeof(int) * r.take, cudaMemcpyHostToDevice, s));
  ProfScope ps_sub(r.c, P_SUBSPACE, s);
  DFT_TRY(precondition_launch(r.c, e->Q, e->res, e->diag, e->evals, e->norms, e->ritz, e->band, (int)r.take, (long)r.n,
                              (double)r.it, e->ekin, s));
  DFT_TRY(block_orth_a(e, (int)(r.m + r.added), e->Q, (int)r.take, s));
  r.orth_pending = true;
  return DFTCUDA_OK;
}

// After the RR read-back: convergence and candidate selection (serial.zig:228-264).
static int run_decide(EigRun& r) {
  KCtxImpl* e = r.e;
  if (*e->h_st == kBarrierTimeoutFlag)
    return fail(DFTCUDA_ERR_TIMEOUT, "eig_solve: a grid barrier of the subspace eigensolver timed out");
  if (*e->h_st != 0)
    return fail(DFTCUDA_ERR_EIGENSOLVER_FAILURE, "eig_solve: subspace eigensolver failed (Jacobi not converged)");
  r.max_res = 0.0;
  for (size_t b = 0; b < r.nbands; ++b) r.max_res = std::max(r.max_res, e->h_nr[b]);
  if (r.max_res < r.opts.tol) {
    r.converged = true;
    r.done = true;
    ++r.it;
    return DFTCUDA_OK;
  }
  r.cand.clear();
  for (size_t b = 0; b < r.nbands; ++b)
    if (!(e->h_nr[b] < r.opts.tol)) r.cand.push_back((int)b);
  r.added = 0;
  r.next = 0;
  if (r.m + r.added < r.max_sub && r.next < r.cand.size()) return run_orth_a(r);
  return DFTCUDA_OK;
}

// After the phase-A read-back: finish the chunk; either another chunk, or the end of the iteration
// (no vector added: converged; subspace full: restart; else H on the new columns).
static int run_orth_b(EigRun& r) {
  KCtxImpl* e = r.e;
  cudaStream_t s = r.s;
  r.orth_pending = false;
  const int kk = *e->h_kk;
  {
    ProfScope ps_sub(r.c, P_SUBSPACE, s);
    DFT_TRY(block_orth_b(e, (int)(r.m + r.added), e->Q, (int)r.take, e->V + (r.m + r.added) * r.n, kk, s));
  }
  r.added += (size_t)std::max(kk, 0);
  r.next += r.take;
  if (r.m + r.added < r.max_sub && r.next < r.cand.size()) return run_orth_a(r);
  if (r.added == 0) {
    r.converged = true;
    r.done = true;
    ++r.it;
    return DFTCUDA_OK;
  }
  if (r.m + r.added >= r.max_sub) {
    // Restart (serial.zig:285-293).  The reference also applies H to the vectors it is about to
    // discard; that product is never read, so it is skipped here.
    DFT_CUDA_TRY(cudaMemcpyAsync(e->V, e->ritz, sizeof(double2) * r.n * r.nbands, cudaMemcpyDeviceToDevice, s));
    r.m = r.nbands;
    r.t_valid = 0;
    DFT_TRY(orthonormalize_all(r.c, (int)r.m, r.seed, s));
    DFT_TRY(kctx_apply_h_dev(r.c, e->V, e->W, r.m, s));
    r.applies += r.m;
  } else {
    DFT_TRY(kctx_apply_h_dev(r.c, e->V + r.m * r.n, e->W + r.m * r.n, r.added, s));
    r.applies += r.added;
    r.m += r.added;
  }
  ++r.it;
  return DFTCUDA_OK;
}

// values: last eigenvalues; vectors: last Ritz vectors (serial.zig:298-306).
static int run_finish(EigRun& r) {
  if (r.nbands == 0 || r.n == 0) return DFTCUDA_OK;
  KCtxImpl* e = r.e;
  cudaStream_t s = r.s;
  if (is_device_pointer(r.values_out))
    DFT_CUDA_TRY(cudaMemcpyAsync(r.values_out, e->evals, sizeof(double) * r.nbands, cudaMemcpyDeviceToDevice, s));
  else
    std::memcpy(r.values_out, e->h_ev, sizeof(double) * r.nbands);
  DFT_CUDA_TRY(cudaMemcpyAsync(r.vectors_out, e->ritz, sizeof(double2) * r.n * r.nbands,
                               is_device_pointer(r.vectors_out) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s));
  DFT_CUDA_TRY(cudaStreamSynchronize(s));
  DFT_TRY(kctx_check_error(r.c));
  if (r.info) {
    r.info->iterations = r.it;
    r.info->h_applies = r.applies;
    r.info->converged = r.converged ? 1 : 0;
    r.info->max_residual = r.max_res;
  }
  return DFTCUDA_OK;
}

static int sync_runs(std::vector<EigRun>& runs, bool only_pending) {
  for (EigRun& r : runs) {
    if (r.done || r.status != DFTCUDA_OK) continue;
    if (only_pending && !r.orth_pending) continue;
    const cudaError_t ce = cudaStreamSynchronize(r.s);
    if (ce != cudaSuccess) r.status = fail(DFTCUDA_ERR_CUDA, std::string("eig_solve: ") + cudaGetErrorString(ce));
  }
  return DFTCUDA_OK;
}

// Host-side phase timers of the lockstep driver, printed to stderr after each solve when
// DFTCUDA_EIG_TIMERS is set: host time spent issuing each phase and blocked in the syncs.
struct EigTimers {
  double t[6] = {0, 0, 0, 0, 0, 0};  // init, rr issue, sync after rr, decide issue, orth syncs, orth_b issue
  long syncs = 0;
};
static bool eig_timers_on() {
  static const bool on = std::getenv("DFTCUDA_EIG_TIMERS") != nullptr;
  return on;
}
static double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Host threads that issue the runs' kernels in each phase: many small runs (k-points, cells) spend
// most of their time in the host's launch calls, and the runs are independent (each has its own
// context, stream and workspace), so their issue spreads over threads.  DFTCUDA_ISSUE_THREADS
// overrides the default (up to 8 threads, one per 8 runs; 1 = issue serially).
static int issue_threads(size_t nruns) {
  static const int env = [] {
    const char* e = std::getenv("DFTCUDA_ISSUE_THREADS");
    return e ? std::max(1, std::atoi(e)) : 0;
  }();
  if (env > 0) return (int)std::min<size_t>(env, std::max<size_t>(nruns, 1));
  const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
  return (int)std::max<size_t>(1, std::min<size_t>({(size_t)8, (size_t)hw, nruns / 8}));
}

// fn(run) for every run, on up to issue_threads() host threads (dynamic assignment).
template <typename F>
static void for_each_run(std::vector<EigRun>& runs, F&& fn) {
  const int nt = issue_threads(runs.size());
  if (nt <= 1) {
    for (EigRun& r : runs) fn(r);
    return;
  }
  int dev = 0;
  cudaGetDevice(&dev);
  std::atomic<size_t> next{0};
  auto work = [&]() {
    cudaSetDevice(dev);  // the runtime's current device is per host thread
    for (size_t i; (i = next.fetch_add(1)) < runs.size();) {
      EigRun& r = runs[i];
      const int before = r.status;
      fn(r);
      if (before == DFTCUDA_OK && r.status != DFTCUDA_OK) r.err_msg = dftcuda_last_error_message();
    }
  };
  std::vector<std::thread> th;
  th.reserve(nt - 1);
  for (int t = 1; t < nt; ++t) th.emplace_back(work);
  work();
  for (std::thread& t : th) t.join();
}

// Lockstep driver: every active run does RR; one synchronisation; every run decides (and launches
// phase A of a chunk); one synchronisation; phase B for those with a chunk (repeated while chunks
// remain); loop.
static int eig_solve_runs(std::vector<EigRun>& runs, const std::vector<const double*>& diags,
                          const std::vector<const double*>& inits, const std::vector<size_t>& icols) {
  EigTimers tm;
  double t0 = now_s();
  for (size_t i = 0; i < runs.size(); ++i) runs[i].index = i;
  for_each_run(runs, [&](EigRun& r) {
    r.status = run_init(r, diags[r.index], inits[r.index], icols[r.index]);
    if (r.status != DFTCUDA_OK) r.done = true;
  });
  double t1 = now_s();
  tm.t[0] += t1 - t0;
  for (;;) {
    t0 = now_s();
    for (EigRun& r : runs)
      if (!r.done && r.status == DFTCUDA_OK && r.it >= r.opts.max_iter) r.done = true;
    bool any = false;
    for (EigRun& r : runs) any |= (!r.done && r.status == DFTCUDA_OK);
    if (!any) break;
    for_each_run(runs, [](EigRun& r) {
      if (!r.done && r.status == DFTCUDA_OK) r.status = run_rr(r);
    });
    t1 = now_s();
    tm.t[1] += t1 - t0;
    sync_runs(runs, false);
    ++tm.syncs;
    t0 = now_s();
    tm.t[2] += t0 - t1;
    for_each_run(runs, [](EigRun& r) {
      if (!r.done && r.status == DFTCUDA_OK) r.status = run_decide(r);
    });
    t1 = now_s();
    tm.t[3] += t1 - t0;
    for (;;) {
      bool pend = false;
      for (EigRun& r : runs) pend |= (!r.done && r.status == DFTCUDA_OK && r.orth_pending);
      if (!pend) break;
      t0 = now_s();
      sync_runs(runs, true);
      ++tm.syncs;
      t1 = now_s();
      tm.t[4] += t1 - t0;
      for_each_run(runs, [](EigRun& r) {
        if (!r.done && r.status == DFTCUDA_OK && r.orth_pending) r.status = run_orth_b(r);
      });
      tm.t[5] += now_s() - t1;
    }
  }
  if (eig_timers_on())
    std::fprintf(stderr,
                 "eig timers: init %.1f ms, rr issue %.1f, rr sync %.1f, decide issue %.1f, orth syncs %.1f, orth_b issue "
                 "%.1f (%ld syncs)\n",
                 1e3 * tm.t[0], 1e3 * tm.t[1], 1e3 * tm.t[2], 1e3 * tm.t[3], 1e3 * tm.t[4], 1e3 * tm.t[5], tm.syncs);
  int first = DFTCUDA_OK;
  std::string first_msg;
  for (EigRun& r : runs) {
    if (r.status == DFTCUDA_OK) {
      r.status = run_finish(r);
      if (r.status != DFTCUDA_OK) r.err_msg = dftcuda_last_error_message();
    }
    if (first == DFTCUDA_OK && r.status != DFTCUDA_OK) {
      first = r.status;
      first_msg = r.err_msg;
    }
  }
  if (first != DFTCUDA_OK && !first_msg.empty()) set_last_error(first, first_msg);  // on the caller's thread
  return first;
}

}  // namespace dftcuda

using namespace dftcuda;

extern "C" int dftcuda_eig_solve(dftcuda_kctx* c, const double* diag, size_t nbands, const dftcuda_eig_opts* opts_in,
                                 const double* init_vecs, size_t init_cols, double* values_out, double* vectors_out,
                                 dftcuda_eig_info* info) {
  return dftcuda_eig_solve_batch(1, &c, &diag, nbands, opts_in, init_vecs ? &init_vecs : nullptr,
                                 init_vecs ? &init_cols : nullptr, &values_out, &vectors_out, info);
}

extern "C" int dftcuda_eig_solve_batch(size_t nk, dftcuda_kctx* const* ctxs, const double* const* diags, size_t nbands,
                                       const dftcuda_eig_opts* opts_in, const double* const* init_vecs,
                                       const size_t* init_cols, double* const* values_out, double* const* vectors_out,
                                       dftcuda_eig_info* infos) {
  if (nk == 0) return DFTCUDA_OK;
  if (!ctxs || !diags || (nbands && (!values_out || !vectors_out)))
    return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "eig_solve: null argument");
  dftcuda_eig_opts opts{40, 1e-6, 0, 0, 0};
  if (opts_in) opts = *opts_in;
  std::vector<EigRun> runs(nk);
  std::vector<const double*> dg(nk), iv(nk, nullptr);
  std::vector<size_t> ic(nk, 0);
  for (size_t i = 0; i < nk; ++i) {
    if (!ctxs[i] || !diags[i] || (nbands && (!values_out[i] || !vectors_out[i])))
      return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "eig_solve: null argument");
    for (size_t j = 0; j < i; ++j)
      if (ctxs[j] == ctxs[i]) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "eig_solve_batch: a context appears twice");
    EigRun& r = runs[i];
    r.c = ctxs[i];
    r.nbands = nbands;
    r.opts = opts;
    r.values_out = values_out[i];
    r.vectors_out = vectors_out[i];
    r.info = infos ? infos + i : nullptr;
    dg[i] = diags[i];
    if (init_vecs) {
      iv[i] = init_vecs[i];
      ic[i] = init_cols ? init_cols[i] : 0;
    }
  }
  // every run's kernels go to its context's stream on that context's device: one device per batch
  for (size_t i = 1; i < nk; ++i)
    if (ctxs[i]->device != ctxs[0]->device)
      return fail(DFTCUDA_ERR_UNSUPPORTED, "eig_solve_batch: contexts of different devices in one batch");
  DeviceGuard guard(ctxs[0]->device);  // the contexts' device, whatever the caller has current
  DFT_TRY(guard.status);
  return eig_solve_runs(runs, dg, iv, ic);
}
