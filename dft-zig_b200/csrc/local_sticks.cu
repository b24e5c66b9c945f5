// Stick-layout local-potential passes: V_loc psi + kinetic for a chunk of columns in three kernels
// whose intermediate is the z-sticks of the G-sphere, not the full y-z planes.
//
// A stick is an (x, y) pair of Miller indices that holds plane waves (all sticks of one x-plane
// "slot" are consecutive, y ascending).  Per column the intermediate S[r][g] holds, for every stick
// g and every z row, one complex value: n_st * nz entries (Si216: 1,886 sticks x 108 = 3.3 MB FP64,
// against 9.1 MB for the 49 full 108 x 108 planes of the plane layout).
//
//  k_stick_inv   32 sticks per CTA: gather the plane waves (zero elsewhere) and run the inverse z
//                transform of each stick in shared memory; rows r of S in the four-step's
//                digit-permuted z order (r = (z mod N1) N2 + z / N1).
//  k_zplane      one z-plane per CTA (a few columns in turn): scatter the plane's stick values into
//                Q[slot][y], inverse y transform of every slot row, then per y line the inverse x
//                transform over the active slots, x V(r), the forward x transform back to the active
//                slots (one warp handles a few lines, exchanges through a per-warp buffer), then the
//                forward y transform and the gather of the stick values.  Everything between the
//                stick row load and store stays in shared memory.
//  k_stick_fwd   forward z transform of each stick, then per plane wave y = kinetic x + (1/N) psi(G).
//
// Each transform is the four-step register DFT of fft_reg.cuh.  The inverse runs with the split
// (N1, N2) and leaves frequency k1 + N1 k2 at index k1 N2 + k2; the forward runs with the split
// swapped (N2, N1), which reads exactly that permuted order and writes natural order, so every step
// works in place and the pair needs no separate un-permute pass.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <string>
#include <vector>

#include "fft_reg.cuh"
#include "kctx.cuh"

namespace dftcuda {

namespace {

constexpr int kStickTile = 32;    // sticks per CTA of the stick passes
constexpr int kStickPad = kStickTile + 1;
constexpr int kStickThreads = 256;
// warps of a z-plane CTA: FP64 lines need more registers per lane (launch bound 384 threads = 170
// registers), FP32 ones fit 512 threads
template <typename T> constexpr int plane_max_warps() { return sizeof(T) == 8 ? 12 : 16; }

template <typename T> __device__ __forceinline__ cplx<T> twl(const cplx<T>* tw, int e, T sg) {
  cplx<T> w = tw[e];
  w.y *= sg;
  return w;
}

// ------------------------------------------------------------------------------------------
// Pass 1: gather + inverse z transform per stick.
// ------------------------------------------------------------------------------------------
template <typename T, int NZ>
__global__ void __launch_bounds__(kStickThreads) k_stick_inv(const double2* __restrict__ x, long npw, cplx<T>* __restrict__ S,
                                                             int n_st, const int* __restrict__ st_map,
                                                             const cplx<T>* __restrict__ twz) {
  using C = cplx<T>;
  constexpr int N1 = Split<NZ>::N1, N2 = Split<NZ>::N2;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* Tl = reinterpret_cast<C*>(smraw);  // [NZ][kStickPad]
  const int g0 = blockIdx.x * kStickTile;
  const long b = blockIdx.y;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const double2* xb = x + b * npw;
  // gather: lanes over z (a stick's plane waves are contiguous in the reference's basis order)
  for (int s = warp; s < kStickTile; s += nwarp) {
    const int g = g0 + s;
    for (int z = lane; z < NZ; z += 32) {
      const int idx = g < n_st ? __ldg(st_map + (long)g * NZ + z) : -1;
      C v = mk<C>(0.0, 0.0);
      if (idx >= 0) {
        const double2 c = __ldg(xb + idx);
        v = mk<C>(c.x, c.y);
      }
      Tl[z * kStickPad + s] = v;
    }
  }
  __syncthreads();
  // step A: task (t, s), lanes over sticks
  for (int w = threadIdx.x; w < N2 * kStickTile; w += blockDim.x) {
    const int s = w % kStickTile, t = w / kStickTile;
    C v[N1];
#pragma unroll
    for (int j = 0; j < N1; ++j) v[j] = Tl[(j * N2 + t) * kStickPad + s];
    RegDft<T, N1>::run(v, (T)1);
#pragma unroll
    for (int k1 = 1; k1 < N1; ++k1)
      if (t) v[k1] = cmul(v[k1], twl<T>(twz, (t * k1) % NZ, (T)1));
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) Tl[(k1 * N2 + t) * kStickPad + s] = v[k1];
  }
  __syncthreads();
  // step B: task (k1, s); frequency k1 + N1 k2 stays at row k1 N2 + k2
  for (int w = threadIdx.x; w < N1 * kStickTile; w += blockDim.x) {
    const int s = w % kStickTile, k1 = w / kStickTile;
    C u[N2];
#pragma unroll
    for (int t = 0; t < N2; ++t) u[t] = Tl[(k1 * N2 + t) * kStickPad + s];
    RegDft<T, N2>::run(u, (T)1);
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) Tl[(k1 * N2 + k2) * kStickPad + s] = u[k2];
  }
  __syncthreads();
  // rows of S in storage (permuted) order, sticks contiguous
  C* Sb = S + b * (long)NZ * n_st;
  for (int r = warp; r < NZ; r += nwarp) {
    const int g = g0 + lane;
    if (g < n_st) Sb[(long)r * n_st + g] = Tl[r * kStickPad + lane];
  }
}

// ------------------------------------------------------------------------------------------
// Pass 3: forward z transform per stick (swapped split reads the permuted rows), then the gather
// into the output column with the 1/N normalisation and the kinetic term.
// ------------------------------------------------------------------------------------------
template <typename T, int NZ>
__global__ void __launch_bounds__(kStickThreads) k_stick_fwd(const cplx<T>* __restrict__ S, int n_st,
                                                             const int* __restrict__ st_map, const cplx<T>* __restrict__ twz,
                                                             const double2* __restrict__ x, double2* __restrict__ y_out,
                                                             long npw, const double* __restrict__ kinetic, double invN) {
  using C = cplx<T>;
  constexpr int N1 = Split<NZ>::N1, N2 = Split<NZ>::N2;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* Tl = reinterpret_cast<C*>(smraw);
  const int g0 = blockIdx.x * kStickTile;
  const long b = blockIdx.y;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const C* Sb = S + b * (long)NZ * n_st;
  for (int r = warp; r < NZ; r += nwarp) {
    const int g = g0 + lane;
    Tl[r * kStickPad + lane] = g < n_st ? Sb[(long)r * n_st + g] : mk<C>(0.0, 0.0);
  }
  __syncthreads();
  // forward step A (split N2 x N1): task (t < N1, s) reads rows t N2 + j, j < N2 (positions j N1 + t)
  for (int w = threadIdx.x; w < N1 * kStickTile; w += blockDim.x) {
    const int s = w % kStickTile, t = w / kStickTile;
    C v[N2];
#pragma unroll
    for (int j = 0; j < N2; ++j) v[j] = Tl[(t * N2 + j) * kStickPad + s];
    RegDft<T, N2>::run(v, (T)-1);
#pragma unroll
    for (int k = 1; k < N2; ++k)
      if (t) v[k] = cmul(v[k], twl<T>(twz, (t * k) % NZ, (T)-1));
#pragma unroll
    for (int k = 0; k < N2; ++k) Tl[(t * N2 + k) * kStickPad + s] = v[k];
  }
  __syncthreads();
  // forward step B: task (k < N2, s): DFT over t, frequency k + N2 m lands in row k + N2 m (natural)
  for (int w = threadIdx.x; w < N2 * kStickTile; w += blockDim.x) {
    const int s = w % kStickTile, k = w / kStickTile;
    C u[N1];
#pragma unroll
    for (int t = 0; t < N1; ++t) u[t] = Tl[(t * N2 + k) * kStickPad + s];
    RegDft<T, N1>::run(u, (T)-1);
#pragma unroll
    for (int m = 0; m < N1; ++m) Tl[(m * N2 + k) * kStickPad + s] = u[m];
  }
  __syncthreads();
  const double2* xb = x + b * npw;
  double2* yb = y_out + b * npw;
  for (int s = warp; s < kStickTile; s += nwarp) {
    const int g = g0 + s;
    if (g >= n_st) break;
    for (int z = lane; z < NZ; z += 32) {
      const int idx = __ldg(st_map + (long)g * NZ + z);
      if (idx >= 0) {
        const double2 xv = __ldg(xb + idx);
        const double kin = __ldg(kinetic + idx);
        const C u = Tl[z * kStickPad + s];
        double2 o;
        o.x = kin * xv.x + (double)u.x * invN;
        o.y = kin * xv.y + (double)u.y * invN;
        yb[idx] = o;
      }
    }
  }
}

// ------------------------------------------------------------------------------------------
// Pass 2: one z-plane per CTA.
// ------------------------------------------------------------------------------------------
// Exchange layout of the H|psi> z-plane pass's x lines.  The inverse half keeps the [N1][N2] layout
// (stride N2); the forward half stores its [N2][N1] intermediate with row stride R and each line's
// buffer spans SF entries, chosen per length so that the 16-byte accesses of a quarter warp fall on
// distinct bank groups (for 108: 222 wavefronts per line group against 330 with R = N1, S = 113; the
// forward read with stride N1 = 12 was 3.25-way conflicted).
struct XStrides {
  int R, SF;
};
constexpr XStrides xline_strides(int n) {
  switch (n) {
    case 20: return {5, 20};
    case 24: return {6, 27};
    case 27: return {9, 27};
    case 30: return {9, 45};
    case 32: return {9, 36};
    case 36: return {9, 54};
    case 40: return {9, 45};
    case 45: return {9, 45};
    case 48: return {9, 54};
    case 60: return {17, 85};
    case 64: return {9, 72};
    case 72: return {9, 72};
    case 75: return {17, 85};
    case 80: return {11, 88};
    case 90: return {17, 153};
    case 96: return {13, 104};
    case 100: return {13, 130};
    case 108: return {17, 153};
    case 120: return {13, 130};
    case 128: return {17, 136};
    default: return {0, 0};
  }
}

template <int NX> struct PlaneXGeom {
  static constexpr int N1 = Split<NX>::N1, N2 = Split<NX>::N2;
  static constexpr int LW = 32 / N2;                                 // lines per warp
  static constexpr int Q = (N1 + N2 - 1) / N2;                       // phase-2 rows per lane
  static constexpr int S = NX + ((N2 - NX) % 8 + 8) % 8;             // exchange stride per line
  static constexpr int R = xline_strides(NX).R;    // forward row stride (H|psi> pass)
  static constexpr int SF = xline_strides(NX).SF;  // per-line exchange entries (H|psi> pass)
  static_assert(R >= N1 && SF >= N2 * R && SF >= NX, "x-line exchange strides");
};

template <typename T, int N>
__global__ void __launch_bounds__(plane_max_warps<T>() * 32, 1) k_zplane(cplx<T>* __restrict__ S, int n_st, const int* __restrict__ st_sy,
                                                                     int n_act, const int* __restrict__ slot_of_x,
                                                                     const T* __restrict__ Vn, int n1z, int n2z, int ncols,
                                                                     int cols_per_cta, const cplx<T>* __restrict__ tw) {
  using C = cplx<T>;
  using G = PlaneXGeom<N>;
  constexpr int N1 = G::N1, N2 = G::N2, LW = G::LW, QR = G::Q, SX = G::SF, RF = G::R;
  constexpr int QS = N + 1;  // Q row stride: odd, so lanes over slots hit distinct banks
  extern __shared__ __align__(16) unsigned char smraw[];
  C* Q = reinterpret_cast<C*>(smraw);  // [n_act][QS]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  C* Bw = Q + (size_t)n_act * QS + (size_t)warp * LW * SX;  // this warp's exchange buffer [LW][SX]
  const int z = blockIdx.x;
  const int r = (z % n1z) * n2z + z / n1z;  // storage row of z in S
  const int c0 = blockIdx.y * cols_per_cta;
  const int c1 = min(ncols, c0 + cols_per_cta);
  const int nq = n_act * QS;
  const T* Vz = Vn + (long)z * N * N;
  const int L = lane / N2, t = lane - L * N2;
  const bool lane_ok = L < LW;
  C* B = Bw + (lane_ok ? L : 0) * SX;
  for (int c = c0; c < c1; ++c) {
    C* Srow = S + ((long)c * gridDim.x + r) * n_st;
    __syncthreads();  // the previous column's gather has read Q
    for (int i = threadIdx.x; i < nq; i += blockDim.x) Q[i] = mk<C>(0.0, 0.0);
    __syncthreads();
    for (int g = threadIdx.x; g < n_st; g += blockDim.x) {
      const int sy = __ldg(st_sy + g);
      Q[(sy >> 16) * QS + (sy & 0xffff)] = Srow[g];
    }
    __syncthreads();
    // inverse y, step A: task (t, slot), lanes over slots
    for (int w = threadIdx.x; w < N2 * n_act; w += blockDim.x) {
      const int sl = w % n_act, tt = w / n_act;
      C* q = Q + sl * QS;
      C v[N1];
#pragma unroll
      for (int j = 0; j < N1; ++j) v[j] = q[j * N2 + tt];
      RegDft<T, N1>::run(v, (T)1);
#pragma unroll
      for (int k1 = 1; k1 < N1; ++k1)
        if (tt) v[k1] = cmul(v[k1], twl<T>(tw, (tt * k1) % N, (T)1));
#pragma unroll
      for (int k1 = 0; k1 < N1; ++k1) q[k1 * N2 + tt] = v[k1];
    }
    __syncthreads();
    // inverse y, step B: position k1 + N1 k2 lands at column k1 N2 + k2
    for (int w = threadIdx.x; w < N1 * n_act; w += blockDim.x) {
      const int sl = w % n_act, k1 = w / n_act;
      C* q = Q + sl * QS + k1 * N2;
      C u[N2];
#pragma unroll
      for (int j = 0; j < N2; ++j) u[j] = q[j];
      RegDft<T, N2>::run(u, (T)1);
#pragma unroll
      for (int k2 = 0; k2 < N2; ++k2) q[k2] = u[k2];
    }
    __syncthreads();
    // x lines: LW lines per warp; line y sits in column col(y) of every active slot
    for (int lt = warp; lt * LW < N; lt += nwarp) {
      const int yl = lt * LW + L;
      const bool lv = lane_ok && yl < N;
      const int col = lv ? (yl % N1) * N2 + yl / N1 : 0;
      {  // inverse step A over x = t + N2 m
        C v[N1];
#pragma unroll
        for (int m = 0; m < N1; ++m) {
          const int sm = lv ? __ldg(slot_of_x + t + N2 * m) : -1;
          v[m] = sm >= 0 ? Q[sm * QS + col] : mk<C>(0.0, 0.0);
        }
        RegDft<T, N1>::run(v, (T)1);
#pragma unroll
        for (int k1 = 1; k1 < N1; ++k1)
          if (t) v[k1] = cmul(v[k1], twl<T>(tw, (t * k1) % N, (T)1));
        if (lane_ok) {
#pragma unroll
          for (int k1 = 0; k1 < N1; ++k1) B[k1 * N2 + t] = v[k1];
        }
      }
      __syncwarp();
      C u[QR][N2];
#pragma unroll
      for (int q = 0; q < QR; ++q) {
        const int k1 = t + N2 * q;
        if (lane_ok && k1 < N1) {
#pragma unroll
          for (int j = 0; j < N2; ++j) u[q][j] = B[k1 * N2 + j];
        }
      }
      __syncwarp();
#pragma unroll
      for (int q = 0; q < QR; ++q) {  // inverse step B, x V(r), forward step A (split swapped)
        const int k1 = t + N2 * q;
        if (lane_ok && k1 < N1) {
          RegDft<T, N2>::run(u[q], (T)1);
#pragma unroll
          for (int k2 = 0; k2 < N2; ++k2) u[q][k2] = cscale(u[q][k2], lv ? __ldg(Vz + (long)yl * N + k1 + N1 * k2) : (T)0);
          RegDft<T, N2>::run(u[q], (T)-1);
#pragma unroll
          for (int kf = 1; kf < N2; ++kf)
            if (k1) u[q][kf] = cmul(u[q][kf], twl<T>(tw, (k1 * kf) % N, (T)-1));
#pragma unroll
          for (int kf = 0; kf < N2; ++kf) B[kf * RF + k1] = u[q][kf];
        }
      }
      __syncwarp();
      {  // forward step B for frequency index t: outputs x = t + N2 m
        C v[N1];
#pragma unroll
        for (int tf = 0; tf < N1; ++tf) v[tf] = lane_ok ? B[t * RF + tf] : mk<C>(0.0, 0.0);
        RegDft<T, N1>::run(v, (T)-1);
#pragma unroll
        for (int m = 0; m < N1; ++m) {
          const int sm = lv ? __ldg(slot_of_x + t + N2 * m) : -1;
          if (sm >= 0) Q[sm * QS + col] = v[m];
        }
      }
      __syncwarp();
    }
    __syncthreads();
    // forward y (split swapped), step A: task (t < N1, slot) reads columns t N2 + j
    for (int w = threadIdx.x; w < N1 * n_act; w += blockDim.x) {
      const int sl = w % n_act, tt = w / n_act;
      C* q = Q + sl * QS + tt * N2;
      C v[N2];
#pragma unroll
      for (int j = 0; j < N2; ++j) v[j] = q[j];
      RegDft<T, N2>::run(v, (T)-1);
#pragma unroll
      for (int k = 1; k < N2; ++k)
        if (tt) v[k] = cmul(v[k], twl<T>(tw, (tt * k) % N, (T)-1));
#pragma unroll
      for (int k = 0; k < N2; ++k) q[k] = v[k];
    }
    __syncthreads();
    // forward y, step B: task (k < N2, slot), frequency k + N2 m lands at column k + N2 m
    for (int w = threadIdx.x; w < N2 * n_act; w += blockDim.x) {
      const int sl = w % n_act, k = w / n_act;
      C* q = Q + sl * QS;
      C u[N1];
#pragma unroll
      for (int tt = 0; tt < N1; ++tt) u[tt] = q[tt * N2 + k];
      RegDft<T, N1>::run(u, (T)-1);
#pragma unroll
      for (int m = 0; m < N1; ++m) q[m * N2 + k] = u[m];
    }
    __syncthreads();
    for (int g = threadIdx.x; g < n_st; g += blockDim.x) {
      const int sy = __ldg(st_sy + g);
      Srow[g] = Q[(sy >> 16) * QS + (sy & 0xffff)];
    }
  }
}

// Doubles reserved for the density kernel's N x N plane: rounded up to an even count, so the complex
// plane after it starts on a 16-byte boundary (N^2 is odd for odd N).
template <int N> __host__ __device__ constexpr int density_plane_words() { return (N * N + 1) & ~1; }

// ------------------------------------------------------------------------------------------
// Band density on the stick layout, pass 2: per z-plane, the inverse y and x transforms of each of
// the CTA's columns and rho(x, y, z) += w_c |psi_c|^2 / Omega accumulated in a shared-memory plane,
// added to the global density once at the end (several CTAs share a plane: atomics).
// ------------------------------------------------------------------------------------------
template <typename T, int N>
__global__ void __launch_bounds__(256, 1) k_zplane_density(const cplx<T>* __restrict__ S, int n_st, const int* __restrict__ st_sy,
                                                           int n_act, const int* __restrict__ slot_of_x, int n1z, int n2z, int ncols,
                                                           int cols_per_cta, const cplx<T>* __restrict__ tw,
                                                           const double* __restrict__ wgt, double inv_vol, double* __restrict__ rho) {
  using C = cplx<T>;
  using G = PlaneXGeom<N>;
  constexpr int N1 = G::N1, N2 = G::N2, LW = G::LW, QR = G::Q, SX = G::S;
  constexpr int QS = N + 1;
  extern __shared__ __align__(16) unsigned char smraw[];
  double* R = reinterpret_cast<double*>(smraw);               // [N][N] density plane, x fastest
  C* Q = reinterpret_cast<C*>(R + density_plane_words<N>());  // [n_act][QS], 16-byte aligned
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  C* Bw = Q + (size_t)n_act * QS + (size_t)warp * LW * SX;
  const int z = blockIdx.x;
  const int r = (z % n1z) * n2z + z / n1z;
  const int c0 = blockIdx.y * cols_per_cta;
  const int c1 = min(ncols, c0 + cols_per_cta);
  const int nq = n_act * QS;
  const int L = lane / N2, t = lane - L * N2;
  const bool lane_ok = L < LW;
  C* B = Bw + (lane_ok ? L : 0) * SX;
  for (int i = threadIdx.x; i < N * N; i += blockDim.x) R[i] = 0.0;
  for (int c = c0; c < c1; ++c) {
    const C* Srow = S + ((long)c * gridDim.x + r) * n_st;
    const double wc = __ldg(wgt + c) * inv_vol;
    __syncthreads();
    for (int i = threadIdx.x; i < nq; i += blockDim.x) Q[i] = mk<C>(0.0, 0.0);
    __syncthreads();
    for (int g = threadIdx.x; g < n_st; g += blockDim.x) {
      const int sy = __ldg(st_sy + g);
      Q[(sy >> 16) * QS + (sy & 0xffff)] = Srow[g];
    }
    __syncthreads();
    for (int w = threadIdx.x; w < N2 * n_act; w += blockDim.x) {
      const int sl = w % n_act, tt = w / n_act;
      C* q = Q + sl * QS;
      C v[N1];
#pragma unroll
      for (int j = 0; j < N1; ++j) v[j] = q[j * N2 + tt];
      RegDft<T, N1>::run(v, (T)1);
#pragma unroll
      for (int k1 = 1; k1 < N1; ++k1)
        if (tt) v[k1] = cmul(v[k1], twl<T>(tw, (tt * k1) % N, (T)1));
#pragma unroll
      for (int k1 = 0; k1 < N1; ++k1) q[k1 * N2 + tt] = v[k1];
    }
    __syncthreads();
    for (int w = threadIdx.x; w < N1 * n_act; w += blockDim.x) {
      const int sl = w % n_act, k1 = w / n_act;
      C* q = Q + sl * QS + k1 * N2;
      C u[N2];
#pragma unroll
      for (int j = 0; j < N2; ++j) u[j] = q[j];
      RegDft<T, N2>::run(u, (T)1);
#pragma unroll
      for (int k2 = 0; k2 < N2; ++k2) q[k2] = u[k2];
    }
    __syncthreads();
    for (int lt = warp; lt * LW < N; lt += nwarp) {
      const int yl = lt * LW + L;
      const bool lv = lane_ok && yl < N;
      const int col = lv ? (yl % N1) * N2 + yl / N1 : 0;
      {
        C v[N1];
#pragma unroll
        for (int m = 0; m < N1; ++m) {
          const int sm = lv ? __ldg(slot_of_x + t + N2 * m) : -1;
          v[m] = sm >= 0 ? Q[sm * QS + col] : mk<C>(0.0, 0.0);
        }
        RegDft<T, N1>::run(v, (T)1);
#pragma unroll
        for (int k1 = 1; k1 < N1; ++k1)
          if (t) v[k1] = cmul(v[k1], twl<T>(tw, (t * k1) % N, (T)1));
        if (lane_ok) {
#pragma unroll
          for (int k1 = 0; k1 < N1; ++k1) B[k1 * N2 + t] = v[k1];
        }
      }
      __syncwarp();
#pragma unroll
      for (int q = 0; q < QR; ++q) {  // inverse step B: x = k1 + N1 k2, then the density
        const int k1 = t + N2 * q;
        if (lv && k1 < N1) {
          C u[N2];
#pragma unroll
          for (int j = 0; j < N2; ++j) u[j] = B[k1 * N2 + j];
          RegDft<T, N2>::run(u, (T)1);
          double* Ry = R + (size_t)yl * N;
#pragma unroll
          for (int k2 = 0; k2 < N2; ++k2)
            Ry[k1 + N1 * k2] += wc * ((double)u[k2].x * (double)u[k2].x + (double)u[k2].y * (double)u[k2].y);
        }
      }
      __syncwarp();
    }
  }
  __syncthreads();
  double* rz = rho + (long)z * N * N;
  for (int i = threadIdx.x; i < N * N; i += blockDim.x) {
    const double v = R[i];
    if (v != 0.0) atomicAdd(rz + i, v);
  }
}

}  // namespace

// ------------------------------------------------------------------------------------------
// Host side
// ------------------------------------------------------------------------------------------

static constexpr int kSmemSticks = 227 * 1024;

static size_t stick_smem(size_t cs, int nz) { return cs * (size_t)nz * kStickPad; }

template <int N> static int plane_warps(size_t cs, int n_act) {
  using G = PlaneXGeom<N>;
  const size_t q = cs * (size_t)n_act * (N + 1);
  const size_t per_warp = cs * (size_t)G::LW * G::SF;
  const int maxw = cs == sizeof(double2) ? plane_max_warps<double>() : plane_max_warps<float>();
  if (q + per_warp > (size_t)kSmemSticks) return 0;
  return (int)std::min<size_t>(maxw, ((size_t)kSmemSticks - q) / per_warp);
}

static int plane_warps_rt(size_t cs, int n, int n_act) {
  switch (n) {
#define X(N) \
  case N: return plane_warps<N>(cs, n_act);
    DFTCUDA_FOUR_STEP_LENGTHS(X)
#undef X
    default: return 0;
  }
}

// Layout choice at context creation: DFTCUDA_LOCAL=planes or =sticks forces one; by default the
// stick layout serves boxes from 96 points along x on (Si216, 108^3: 12.0 against 14.2 ms per
// 452-column FP64 block) and the plane layout smaller ones (Si64, 75^3: the stick z-plane pass took
// 18.1 against 11.3 ms per step).  The autotuner times both either way.
static int local_layout_env() {
  const char* e = std::getenv("DFTCUDA_LOCAL");
  if (e && std::string(e) == "planes") return 1;
  if (e && std::string(e) == "sticks") return 2;
  return 0;
}

bool kctx_sticks_ok(const dftcuda_kctx* c, int precision) {
  if (local_layout_env() == 1) return false;
  if (!four_step_supported(c->nx) || !four_step_supported(c->nz) || c->nx != c->ny) return false;
  if (c->n_act > 0xffff || c->ny > 0xffff) return false;
  const size_t cs = precision == DFTCUDA_PRECISION_FP64 ? sizeof(double2) : sizeof(float2);
  return plane_warps_rt(cs, c->ny, c->n_act) >= 4 && stick_smem(cs, c->nz) <= (size_t)kSmemSticks;
}

size_t sticks_bytes_per_col(const dftcuda_kctx* c, size_t cs) { return cs * (size_t)c->nz * c->n_st; }

template <typename T, int NZ>
static int launch_stick_inv(dftcuda_kctx* c, const double2* x, cplx<T>* S, size_t ncols, cudaStream_t s) {
  const size_t smem = stick_smem(sizeof(cplx<T>), NZ);
  DFT_TRY(ensure_max_dynamic_smem((const void*)k_stick_inv<T, NZ>, (int)smem));
  const cplx<T>* tw = std::is_same<T, double>::value ? (const cplx<T>*)c->d_twz64 : (const cplx<T>*)c->d_twz32;
  dim3 g(ceil_div(c->n_st, kStickTile), (unsigned)ncols);
  k_stick_inv<T, NZ><<<g, kStickThreads, smem, s>>>(x, (long)c->npw, S, c->n_st, c->d_st_map, tw);
  count_launch();
  return DFTCUDA_OK;
}

template <typename T, int NZ>
static int launch_stick_fwd(dftcuda_kctx* c, const cplx<T>* S, const double2* x, double2* y, size_t ncols, cudaStream_t s) {
  const size_t smem = stick_smem(sizeof(cplx<T>), NZ);
  DFT_TRY(ensure_max_dynamic_smem((const void*)k_stick_fwd<T, NZ>, (int)smem));
  const cplx<T>* tw = std::is_same<T, double>::value ? (const cplx<T>*)c->d_twz64 : (const cplx<T>*)c->d_twz32;
  dim3 g(ceil_div(c->n_st, kStickTile), (unsigned)ncols);
  k_stick_fwd<T, NZ><<<g, kStickThreads, smem, s>>>(S, c->n_st, c->d_st_map, tw, x, y, (long)c->npw, c->d_kinetic,
                                                    1.0 / (double)c->N);
  count_launch();
  return DFTCUDA_OK;
}

template <typename T, int N>
static int launch_zplane(dftcuda_kctx* c, cplx<T>* S, size_t ncols, cudaStream_t s) {
  using G = PlaneXGeom<N>;
  const size_t cs = sizeof(cplx<T>);
  const int nw = plane_warps<N>(cs, c->n_act);
  if (nw < 1) return fail(DFTCUDA_ERR_UNSUPPORTED, "z-plane pass does not fit shared memory");
  const size_t smem = cs * ((size_t)c->n_act * (N + 1) + (size_t)nw * G::LW * G::SF);
  DFT_TRY(ensure_max_dynamic_smem((const void*)k_zplane<T, N>, (int)smem));
  const T* vn = std::is_same<T, double>::value ? (const T*)c->d_vn : (const T*)c->d_vn32;
  const cplx<T>* tw = std::is_same<T, double>::value ? (const cplx<T>*)c->d_twx64 : (const cplx<T>*)c->d_twx32;
  // a few columns per CTA: enough CTAs for two waves of one CTA per SM
  const int cpc = std::max(1, (int)std::min<size_t>(8, ncols * c->nz / 296));
  dim3 g((unsigned)c->nz, ceil_div(ncols, cpc));
  int n1z = 0, n2z = 0;
  switch (c->nz) {
#define X(L)            \
  case L:               \
    n1z = Split<L>::N1; \
    n2z = Split<L>::N2; \
    break;
    DFTCUDA_FOUR_STEP_LENGTHS(X)
#undef X
    default: return fail(DFTCUDA_ERR_UNSUPPORTED, "z length without a four-step split");
  }
  k_zplane<T, N><<<g, nw * 32, smem, s>>>(S, c->n_st, c->d_st_sy, c->n_act, c->d_st_sox, vn, n1z, n2z, (int)ncols, cpc, tw);
  count_launch();
  return DFTCUDA_OK;
}

static constexpr int kDensityWarps = 8;

template <int N> static size_t density_plane_smem(size_t cs, int n_act) {
  using G = PlaneXGeom<N>;
  return sizeof(double) * (size_t)density_plane_words<N>() + cs * ((size_t)n_act * (N + 1) + (size_t)kDensityWarps * G::LW * G::S);
}

template <typename T, int N>
static int launch_zplane_density(dftcuda_kctx* c, const cplx<T>* S, size_t ncols, const double* w, double* rho, cudaStream_t s) {
  const size_t smem = density_plane_smem<N>(sizeof(cplx<T>), c->n_act);
  if (smem > (size_t)kSmemSticks) return fail(DFTCUDA_ERR_UNSUPPORTED, "z-plane density pass does not fit shared memory");
  DFT_TRY(ensure_max_dynamic_smem((const void*)k_zplane_density<T, N>, (int)smem));
  const cplx<T>* tw = std::is_same<T, double>::value ? (const cplx<T>*)c->d_twx64 : (const cplx<T>*)c->d_twx32;
  // columns per CTA: every CTA sums its columns in shared memory before one atomic pass over its plane
  const int cpc = std::max(1, (int)((ncols * c->nz + 295) / 296));
  dim3 g((unsigned)c->nz, ceil_div(ncols, cpc));
  int n1z = 0, n2z = 0;
  switch (c->nz) {
#define X(L)            \
  case L:               \
    n1z = Split<L>::N1; \
    n2z = Split<L>::N2; \
    break;
    DFTCUDA_FOUR_STEP_LENGTHS(X)
#undef X
    default: return fail(DFTCUDA_ERR_UNSUPPORTED, "z length without a four-step split");
  }
  k_zplane_density<T, N><<<g, kDensityWarps * 32, smem, s>>>(S, c->n_st, c->d_st_sy, c->n_act, c->d_st_sox, n1z, n2z, (int)ncols, cpc, tw,
                                                              w, 1.0 / c->volume, rho);
  count_launch();
  return DFTCUDA_OK;
}

template <typename T>
static int dispatch_zplane_density(dftcuda_kctx* c, const cplx<T>* S, size_t ncols, const double* w, double* rho, cudaStream_t s) {
  switch (c->nx) {
#define X(N) \
  case N: return launch_zplane_density<T, N>(c, S, ncols, w, rho, s);
    DFTCUDA_FOUR_STEP_LENGTHS(X)
#undef X
    default: return fail(DFTCUDA_ERR_UNSUPPORTED, "x length without a four-step kernel");
  }
}

bool kctx_sticks_density_ok(const dftcuda_kctx* c, int precision) {
  if (!(precision == DFTCUDA_PRECISION_FP64 ? c->sticks64 : c->sticks32)) return false;
  const size_t cs = precision == DFTCUDA_PRECISION_FP64 ? sizeof(double2) : sizeof(float2);
  switch (c->nx) {
#define X(N) \
  case N: return density_plane_smem<N>(cs, c->n_act) <= (size_t)kSmemSticks;
    DFTCUDA_FOUR_STEP_LENGTHS(X)
#undef X
    default: return false;
  }
}

template <typename T>
static int dispatch_stick_inv(dftcuda_kctx* c, const double2* x, cplx<T>* S, size_t ncols, cudaStream_t s) {
  switch (c->nz) {
#define X(N) \
  case N: return launch_stick_inv<T, N>(c, x, S, ncols, s);
    DFTCUDA_FOUR_STEP_LENGTHS(X)
#undef X
    default: return fail(DFTCUDA_ERR_UNSUPPORTED, "z length without a four-step kernel");
  }
}
template <typename T>
static int dispatch_stick_fwd(dftcuda_kctx* c, const cplx<T>* S, const double2* x, double2* y, size_t ncols, cudaStream_t s) {
  switch (c->nz) {
#define X(N) \
  case N: return launch_stick_fwd<T, N>(c, S, x, y, ncols, s);
    DFTCUDA_FOUR_STEP_LENGTHS(X)
#undef X
    default: return fail(DFTCUDA_ERR_UNSUPPORTED, "z length without a four-step kernel");
  }
}
template <typename T>
static int dispatch_zplane(dftcuda_kctx* c, cplx<T>* S, size_t ncols, cudaStream_t s) {
  switch (c->nx) {
#define X(N) \
  case N: return launch_zplane<T, N>(c, S, ncols, s);
    DFTCUDA_FOUR_STEP_LENGTHS(X)
#undef X
    default: return fail(DFTCUDA_ERR_UNSUPPORTED, "x length without a four-step kernel");
  }
}

template <typename T>
int local_block_sticks(dftcuda_kctx* c, const double2* x, double2* y, size_t ncols, cudaStream_t s) {
  cplx<T>* S = reinterpret_cast<cplx<T>*>(c->d_box);
  {
    ProfScope ps(c, P_PLANE_INV, s);
    DFT_TRY(dispatch_stick_inv<T>(c, x, S, ncols, s));
  }
  {
    ProfScope ps(c, P_XLINE, s);
    DFT_TRY(dispatch_zplane<T>(c, S, ncols, s));
  }
  {
    ProfScope ps(c, P_PLANE_FWD, s);
    DFT_TRY(dispatch_stick_fwd<T>(c, S, x, y, ncols, s));
  }
  DFT_CUDA_TRY(cudaGetLastError());
  return DFTCUDA_OK;
}
template int local_block_sticks<double>(dftcuda_kctx*, const double2*, double2*, size_t, cudaStream_t);
template int local_block_sticks<float>(dftcuda_kctx*, const double2*, double2*, size_t, cudaStream_t);

template <typename T>
int density_block_sticks(dftcuda_kctx* c, const double2* x, size_t ncols, const double* w, double* rho, cudaStream_t s) {
  cplx<T>* S = reinterpret_cast<cplx<T>*>(c->d_box);
  ProfScope ps(c, P_DENSITY, s);
  DFT_TRY(dispatch_stick_inv<T>(c, x, S, ncols, s));
  DFT_TRY(dispatch_zplane_density<T>(c, S, ncols, w, rho, s));
  DFT_CUDA_TRY(cudaGetLastError());
  return DFTCUDA_OK;
}

template int density_block_sticks<double>(dftcuda_kctx*, const double2*, size_t, const double*, double*, cudaStream_t);
template int density_block_sticks<float>(dftcuda_kctx*, const double2*, size_t, const double*, double*, cudaStream_t);

// Stick tables: sticks in slot order (y ascending within a slot), the packed (slot, y) of each, the
// plane-wave index of every (stick, z) (or -1), and the z and x/y twiddle tables.
int kctx_setup_sticks(dftcuda_kctx* c, const std::vector<int>& slot_of_x, const std::vector<int>& xpos, const int32_t* hkl) {
  c->sticks64 = kctx_sticks_ok(c, DFTCUDA_PRECISION_FP64);
  c->sticks32 = kctx_sticks_ok(c, DFTCUDA_PRECISION_FP32);
  if (!c->sticks64 && !c->sticks32) return DFTCUDA_OK;
  c->sticks_off = local_layout_env() != 2 && c->nx < 96;
  DFT_TRY(init_root_tables_here());  // this file's copy of the sub-DFT roots
  const int ny = c->ny, nz = c->nz, n_act = c->n_act;
  std::vector<std::vector<int>> ys(n_act);
  std::vector<std::vector<char>> has(n_act, std::vector<char>(ny, 0));
  for (size_t i = 0; i < c->npw; ++i) {
    const int sl = slot_of_x[xpos[i]];
    const int yy = ((hkl[3 * i + 1] % ny) + ny) % ny;
    if (!has[sl][yy]) {
      has[sl][yy] = 1;
      ys[sl].push_back(yy);
    }
  }
  std::vector<int> first(n_act + 1, 0);
  std::vector<std::vector<int>> gidx(n_act, std::vector<int>(ny, -1));
  std::vector<int> sy;
  for (int sl = 0; sl < n_act; ++sl) {
    std::sort(ys[sl].begin(), ys[sl].end());
    first[sl + 1] = first[sl] + (int)ys[sl].size();
    for (size_t k = 0; k < ys[sl].size(); ++k) {
      gidx[sl][ys[sl][k]] = first[sl] + (int)k;
      sy.push_back((sl << 16) | ys[sl][k]);
    }
  }
  c->n_st = first[n_act];
  std::vector<int> map((size_t)c->n_st * nz, -1);
  for (size_t i = 0; i < c->npw; ++i) {
    const int sl = slot_of_x[xpos[i]];
    const int yy = ((hkl[3 * i + 1] % ny) + ny) % ny, zz = ((hkl[3 * i + 2] % nz) + nz) % nz;
    map[(size_t)gidx[sl][yy] * nz + zz] = (int)i;
  }
  auto roots = [](int n, std::vector<double2>& r64, std::vector<float2>& r32) {
    r64.resize(n);
    r32.resize(n);
    for (int e = 0; e < n; ++e) {
      const double a = 2.0 * M_PI * (double)e / (double)n;
      r64[e] = make_double2(std::cos(a), std::sin(a));
      r32[e] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
  };
  std::vector<double2> tz64, tx64;
  std::vector<float2> tz32, tx32;
  roots(nz, tz64, tz32);
  roots(c->nx, tx64, tx32);
  std::vector<int> sox(slot_of_x.begin(), slot_of_x.end());
  bool ok = dev_malloc(&c->d_st_sy, sizeof(int) * std::max<size_t>(sy.size(), 1)) == cudaSuccess &&
            dev_malloc(&c->d_st_map, sizeof(int) * std::max<size_t>(map.size(), 1)) == cudaSuccess &&
            dev_malloc(&c->d_st_sox, sizeof(int) * c->nx) == cudaSuccess &&
            dev_malloc(&c->d_twz64, sizeof(double2) * nz) == cudaSuccess &&
            dev_malloc(&c->d_twz32, sizeof(float2) * nz) == cudaSuccess &&
            dev_malloc(&c->d_twx64, sizeof(double2) * c->nx) == cudaSuccess &&
            dev_malloc(&c->d_twx32, sizeof(float2) * c->nx) == cudaSuccess &&
            dev_malloc(&c->d_vn, sizeof(double) * c->N) == cudaSuccess &&
            dev_malloc(&c->d_vn32, sizeof(float) * c->N) == cudaSuccess;
  if (!ok) return fail(DFTCUDA_ERR_OUT_OF_MEMORY, "stick tables");
  cudaStream_t st = c->stream;
  if (!sy.empty()) DFT_CUDA_TRY(cudaMemcpyAsync(c->d_st_sy, sy.data(), sizeof(int) * sy.size(), cudaMemcpyHostToDevice, st));
  if (!map.empty()) DFT_CUDA_TRY(cudaMemcpyAsync(c->d_st_map, map.data(), sizeof(int) * map.size(), cudaMemcpyHostToDevice, st));
  DFT_CUDA_TRY(cudaMemcpyAsync(c->d_st_sox, sox.data(), sizeof(int) * c->nx, cudaMemcpyHostToDevice, st));
  DFT_CUDA_TRY(cudaMemcpyAsync(c->d_twz64, tz64.data(), sizeof(double2) * nz, cudaMemcpyHostToDevice, st));
  DFT_CUDA_TRY(cudaMemcpyAsync(c->d_twz32, tz32.data(), sizeof(float2) * nz, cudaMemcpyHostToDevice, st));
  DFT_CUDA_TRY(cudaMemcpyAsync(c->d_twx64, tx64.data(), sizeof(double2) * c->nx, cudaMemcpyHostToDevice, st));
  DFT_CUDA_TRY(cudaMemcpyAsync(c->d_twx32, tx32.data(), sizeof(float2) * c->nx, cudaMemcpyHostToDevice, st));
  DFT_CUDA_TRY(cudaStreamSynchronize(st));
  return DFTCUDA_OK;
}

}  // namespace dftcuda
