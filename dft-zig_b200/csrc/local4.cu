// Four-step register FFT versions of the local-potential passes (see fft_reg.cuh), used when the
// box extents have a four-step kernel and two y-z planes fit in shared memory.  Same results as the
// generic passes in hpsi.cu (which remain for every other box), fewer shared-memory round trips:
//
//  k_plane_inv4  z transform on the plane's sticks (the y columns holding plane waves; step A
//                reads the plane waves straight from the wavefunction through a per-plane
//                (z, y) -> plane-wave map), then the y transform on every z row, plane to HBM.
//  k_xline4      per run of (z, y) lines: inverse x transform (step A gathers the active planes
//                from HBM), x V(r) in registers, forward x transform whose step A takes the inverse's
//                step-B registers directly, active x frequencies back to HBM.  Two barriers per
//                column; V(r) stays in registers for all the CTA's columns.
//  k_plane_fwd4  y transform on every row, z transform on the sticks, gather x 1/N + kinetic
//                straight into the output column.
//  k_xline_density4  inverse x transform and sum_b w_b |psi_b|^2 / Omega in registers.
#include <algorithm>
#include <cstdlib>
#include <string>
#include <cmath>
#include <mutex>
#include <vector>

#include "fft_reg.cuh"
#include "kctx.cuh"

namespace dftcuda {

bool four_step_supported(int n) {
  switch (n) {
#define X(N) case N:
    DFTCUDA_FOUR_STEP_LENGTHS(X)
#undef X
    return true;
    default:
      return false;
  }
}

template <typename T> __device__ __forceinline__ cplx<T> tw_ld(const cplx<T>* tw, int e, T sg) {
  cplx<T> w = tw[e];
  w.y *= sg;
  return w;
}

// ------------------------------------------------------------------------------------------

template <typename T, int NP>
__global__ void __launch_bounds__(512) k_plane_inv4(const double2* __restrict__ x, long npw, cplx<T>* __restrict__ W,
                                                    int n_act, const int* __restrict__ pwmap,
                                                    const int* __restrict__ stick_off, const int* __restrict__ stick_y,
                                                    const cplx<T>* __restrict__ tw) {
  using C = cplx<T>;
  constexpr int N1 = Split<NP>::N1, N2 = Split<NP>::N2, P = NP * NP;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* S1 = reinterpret_cast<C*>(smraw);
  C* S2 = S1 + P;
  int* sy = reinterpret_cast<int*>(S2 + P);
  unsigned char* isst = reinterpret_cast<unsigned char*>(sy + NP);
  const int slot = blockIdx.x;
  const long b = blockIdx.y;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int s0 = stick_off[slot], ns = stick_off[slot + 1] - s0;
  for (int i = tid; i < NP; i += nt) isst[i] = 0;
  __syncthreads();
  for (int i = tid; i < ns; i += nt) {
    const int y = stick_y[s0 + i];
    sy[i] = y;
    isst[y] = 1;
  }
  __syncthreads();
  const int* pm = pwmap + (long)slot * P;
  const double2* xb = x + b * npw;
  // z transform, step A: thread (t, stick)
  for (int w = tid; w < N2 * ns; w += nt) {
    const int s = w % ns, t = w / ns, y = sy[s];
    C v[N1];
#pragma unroll
    for (int j = 0; j < N1; ++j) {
      const int idx = __ldg(pm + (j * N2 + t) * NP + y);
      if (idx >= 0) {
        const double2 c = __ldg(xb + idx);
        v[j] = mk<C>(c.x, c.y);
      } else {
        v[j] = mk<C>(0.0, 0.0);
      }
    }
    RegDft<T, N1>::run(v, (T)1);
#pragma unroll
    for (int k1 = 1; k1 < N1; ++k1)
      if (t) v[k1] = cmul(v[k1], tw_ld<T>(tw, (t * k1) % NP, (T)1));
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) S1[(k1 * N2 + t) * NP + y] = v[k1];
  }
  __syncthreads();
  // z transform, step B: thread (k1, stick); natural z order into S2
  for (int w = tid; w < N1 * ns; w += nt) {
    const int s = w % ns, k1 = w / ns, y = sy[s];
    C u[N2];
#pragma unroll
    for (int t = 0; t < N2; ++t) u[t] = S1[(k1 * N2 + t) * NP + y];
    RegDft<T, N2>::run(u, (T)1);
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) S2[(k1 + N1 * k2) * NP + y] = u[k2];
  }
  __syncthreads();
  // y transform, step A: thread (t, z); columns without plane waves are zero
  for (int w = tid; w < N2 * NP; w += nt) {
    const int t = w % N2, z = w / N2;
    C v[N1];
#pragma unroll
    for (int j = 0; j < N1; ++j) {
      const int y = j * N2 + t;
      v[j] = isst[y] ? S2[z * NP + y] : mk<C>(0.0, 0.0);
    }
    RegDft<T, N1>::run(v, (T)1);
#pragma unroll
    for (int k1 = 1; k1 < N1; ++k1)
      if (t) v[k1] = cmul(v[k1], tw_ld<T>(tw, (t * k1) % NP, (T)1));
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) S1[z * NP + k1 * N2 + t] = v[k1];
  }
  __syncthreads();
  // y transform, step B: thread (k1, z); plane to HBM in natural (z, y) order
  C* Wp = W + (b * n_act + slot) * (long)P;
  for (int w = tid; w < N1 * NP; w += nt) {
    const int k1 = w % N1, z = w / N1;
    C u[N2];
#pragma unroll
    for (int t = 0; t < N2; ++t) u[t] = S1[z * NP + k1 * N2 + t];
    RegDft<T, N2>::run(u, (T)1);
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) Wp[z * NP + k1 + N1 * k2] = u[k2];
  }
}

template <typename T, int NP>
__global__ void __launch_bounds__(512) k_plane_fwd4(const cplx<T>* __restrict__ W, int n_act, const int* __restrict__ pwmap,
                                                    const int* __restrict__ stick_off, const int* __restrict__ stick_y,
                                                    const cplx<T>* __restrict__ tw, const double2* __restrict__ x,
                                                    double2* __restrict__ y_out, long npw,
                                                    const double* __restrict__ kinetic, double invN) {
  using C = cplx<T>;
  constexpr int N1 = Split<NP>::N1, N2 = Split<NP>::N2, P = NP * NP;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* S1 = reinterpret_cast<C*>(smraw);
  C* S2 = S1 + P;
  int* sy = reinterpret_cast<int*>(S2 + P);
  unsigned char* isst = reinterpret_cast<unsigned char*>(sy + NP);
  const int slot = blockIdx.x;
  const long b = blockIdx.y;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int s0 = stick_off[slot], ns = stick_off[slot + 1] - s0;
  for (int i = tid; i < NP; i += nt) isst[i] = 0;
  const C* Wp = W + (b * n_act + slot) * (long)P;
  for (int i = tid; i < P; i += nt) S2[i] = Wp[i];
  __syncthreads();
  for (int i = tid; i < ns; i += nt) {
    const int y = stick_y[s0 + i];
    sy[i] = y;
    isst[y] = 1;
  }
  // y transform, step A: thread (t, z)
  for (int w = tid; w < N2 * NP; w += nt) {
    const int t = w % N2, z = w / N2;
    C v[N1];
#pragma unroll
    for (int j = 0; j < N1; ++j) v[j] = S2[z * NP + j * N2 + t];
    RegDft<T, N1>::run(v, (T)-1);
#pragma unroll
    for (int k1 = 1; k1 < N1; ++k1)
      if (t) v[k1] = cmul(v[k1], tw_ld<T>(tw, (t * k1) % NP, (T)-1));
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) S1[z * NP + k1 * N2 + t] = v[k1];
  }
  __syncthreads();
  // y transform, step B: keep only the stick columns the z transform needs
  for (int w = tid; w < N1 * NP; w += nt) {
    const int k1 = w % N1, z = w / N1;
    C u[N2];
#pragma unroll
    for (int t = 0; t < N2; ++t) u[t] = S1[z * NP + k1 * N2 + t];
    RegDft<T, N2>::run(u, (T)-1);
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) {
      const int y = k1 + N1 * k2;
      if (isst[y]) S2[z * NP + y] = u[k2];
    }
  }
  __syncthreads();
  // z transform, step A: thread (t, stick)
  for (int w = tid; w < N2 * ns; w += nt) {
    const int s = w % ns, t = w / ns, y = sy[s];
    C v[N1];
#pragma unroll
    for (int j = 0; j < N1; ++j) v[j] = S2[(j * N2 + t) * NP + y];
    RegDft<T, N1>::run(v, (T)-1);
#pragma unroll
    for (int k1 = 1; k1 < N1; ++k1)
      if (t) v[k1] = cmul(v[k1], tw_ld<T>(tw, (t * k1) % NP, (T)-1));
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) S1[(k1 * N2 + t) * NP + y] = v[k1];
  }
  __syncthreads();
  // z transform, step B: thread (k1, stick); gather x 1/N plus kinetic into the output column
  const int* pm = pwmap + (long)slot * P;
  for (int w = tid; w < N1 * ns; w += nt) {
    const int s = w % ns, k1 = w / ns, y = sy[s];
    C u[N2];
#pragma unroll
    for (int t = 0; t < N2; ++t) u[t] = S1[(k1 * N2 + t) * NP + y];
    RegDft<T, N2>::run(u, (T)-1);
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) {
      const int z = k1 + N1 * k2;
      const int g = __ldg(pm + z * NP + y);
      if (g >= 0) {
        const double2 xv = __ldg(x + b * npw + g);
        const double kin = __ldg(kinetic + g);
        double2 o;
        o.x = kin * xv.x + (double)u[k2].x * invN;
        o.y = kin * xv.y + (double)u[k2].y * invN;
        y_out[b * npw + g] = o;
      }
    }
  }
}

// Single-buffer plane passes: every four-step phase works in place.  Step B of a transform writes
// its N2 outputs for row (or column) k1 into the slots k1 N2 + k2 it read, i.e. frequency
// k1 + N1 k2 sits at index perm(f) = (f mod N1) N2 + f / N1; later phases either work per row /
// column (where the order does not matter) or un-permute when they read or write HBM.  One P-sized
// shared buffer instead of two: two CTAs per SM at 75^2 in FP64, and planes up to 119^2 fit.
constexpr int kPlaneThreads = 384;  // two CTAs per SM at <= 85 registers
// Two CTAs per SM where two planes fit the 227 KB of shared memory; otherwise one, with the whole
// register file for it.
template <typename T, int NP> __host__ __device__ constexpr int plane_min_ctas() {
  return sizeof(cplx<T>) * NP * NP <= 113 * 1024 ? 2 : 1;
}

template <int NP> __device__ __forceinline__ int dperm(int f) {
  constexpr int N1 = Split<NP>::N1, N2 = Split<NP>::N2;
  return (f % N1) * N2 + f / N1;
}

template <typename T, int NP>
__global__ void __launch_bounds__(kPlaneThreads, plane_min_ctas<T, NP>()) k_plane_inv5(const double2* __restrict__ x, long npw, cplx<T>* __restrict__ W,
                                                    int n_act, const int* __restrict__ pwmap,
                                                    const int* __restrict__ stick_off, const int* __restrict__ stick_y,
                                                    const cplx<T>* __restrict__ tw) {
  using C = cplx<T>;
  constexpr int N1 = Split<NP>::N1, N2 = Split<NP>::N2, P = NP * NP;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* S = reinterpret_cast<C*>(smraw);
  int* sy = reinterpret_cast<int*>(S + P);
  unsigned char* isst = reinterpret_cast<unsigned char*>(sy + NP);
  const int slot = blockIdx.x;
  const long b = blockIdx.y;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int s0 = stick_off[slot], ns = stick_off[slot + 1] - s0;
  for (int i = tid; i < NP; i += nt) isst[i] = 0;
  __syncthreads();
  for (int i = tid; i < ns; i += nt) {
    const int y = stick_y[s0 + i];
    sy[i] = y;
    isst[y] = 1;
  }
  __syncthreads();
  const int* pm = pwmap + (long)slot * P;
  const double2* xb = x + b * npw;
  // z transform, step A: thread (t, stick), rows k1 N2 + t of column y
  for (int w = tid; w < N2 * ns; w += nt) {
    const int s = w % ns, t = w / ns, y = sy[s];
    C v[N1];
#pragma unroll
    for (int j = 0; j < N1; ++j) {
      const int idx = __ldg(pm + (j * N2 + t) * NP + y);
      if (idx >= 0) {
        const double2 c = __ldg(xb + idx);
        v[j] = mk<C>(c.x, c.y);
      } else {
        v[j] = mk<C>(0.0, 0.0);
      }
    }
    RegDft<T, N1>::run(v, (T)1);
#pragma unroll
    for (int k1 = 1; k1 < N1; ++k1)
      if (t) v[k1] = cmul(v[k1], tw_ld<T>(tw, (t * k1) % NP, (T)1));
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) S[(k1 * N2 + t) * NP + y] = v[k1];
  }
  __syncthreads();
  // z transform, step B in place: z frequency k1 + N1 k2 lands in row k1 N2 + k2
  for (int w = tid; w < N1 * ns; w += nt) {
    const int s = w % ns, k1 = w / ns, y = sy[s];
    C u[N2];
#pragma unroll
    for (int t = 0; t < N2; ++t) u[t] = S[(k1 * N2 + t) * NP + y];
    RegDft<T, N2>::run(u, (T)1);
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) S[(k1 * N2 + k2) * NP + y] = u[k2];
  }
  __syncthreads();
  // y transform, step A in place on every row r (a permuted z); columns without plane waves are zero
  for (int w = tid; w < N2 * NP; w += nt) {
    const int t = w % N2, r = w / N2;
    C v[N1];
#pragma unroll
    for (int j = 0; j < N1; ++j) {
      const int y = j * N2 + t;
      v[j] = isst[y] ? S[r * NP + y] : mk<C>(0.0, 0.0);
    }
    RegDft<T, N1>::run(v, (T)1);
#pragma unroll
    for (int k1 = 1; k1 < N1; ++k1)
      if (t) v[k1] = cmul(v[k1], tw_ld<T>(tw, (t * k1) % NP, (T)1));
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) S[r * NP + k1 * N2 + t] = v[k1];
  }
  __syncthreads();
  // y transform, step B: thread (k1, row); the plane to HBM in natural (z, y) order
  C* Wp = W + (b * n_act + slot) * (long)P;
  for (int w = tid; w < N1 * NP; w += nt) {
    const int k1 = w % N1, r = w / N1;
    const int z = (r / N2) + N1 * (r % N2);
    C u[N2];
#pragma unroll
    for (int t = 0; t < N2; ++t) u[t] = S[r * NP + k1 * N2 + t];
    RegDft<T, N2>::run(u, (T)1);
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) Wp[z * NP + k1 + N1 * k2] = u[k2];
  }
}

template <typename T, int NP>
__global__ void __launch_bounds__(kPlaneThreads, plane_min_ctas<T, NP>()) k_plane_fwd5(const cplx<T>* __restrict__ W, int n_act, const int* __restrict__ pwmap,
                                                    const int* __restrict__ stick_off, const int* __restrict__ stick_y,
                                                    const cplx<T>* __restrict__ tw, const double2* __restrict__ x,
                                                    double2* __restrict__ y_out, long npw,
                                                    const double* __restrict__ kinetic, double invN) {
  using C = cplx<T>;
  constexpr int N1 = Split<NP>::N1, N2 = Split<NP>::N2, P = NP * NP;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* S = reinterpret_cast<C*>(smraw);
  int* sy = reinterpret_cast<int*>(S + P);
  const int slot = blockIdx.x;
  const long b = blockIdx.y;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int s0 = stick_off[slot], ns = stick_off[slot + 1] - s0;
  const C* Wp = W + (b * n_act + slot) * (long)P;
  for (int i = tid; i < P; i += nt) S[i] = Wp[i];
  for (int i = tid; i < ns; i += nt) sy[i] = stick_y[s0 + i];
  __syncthreads();
  // y transform, step A in place: thread (t, z)
  for (int w = tid; w < N2 * NP; w += nt) {
    const int t = w % N2, z = w / N2;
    C v[N1];
#pragma unroll
    for (int j = 0; j < N1; ++j) v[j] = S[z * NP + j * N2 + t];
    RegDft<T, N1>::run(v, (T)-1);
#pragma unroll
    for (int k1 = 1; k1 < N1; ++k1)
      if (t) v[k1] = cmul(v[k1], tw_ld<T>(tw, (t * k1) % NP, (T)-1));
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) S[z * NP + k1 * N2 + t] = v[k1];
  }
  __syncthreads();
  // y transform, step B in place: y frequency k1 + N1 k2 lands in column k1 N2 + k2
  for (int w = tid; w < N1 * NP; w += nt) {
    const int k1 = w % N1, z = w / N1;
    C u[N2];
#pragma unroll
    for (int t = 0; t < N2; ++t) u[t] = S[z * NP + k1 * N2 + t];
    RegDft<T, N2>::run(u, (T)-1);
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) S[z * NP + k1 * N2 + k2] = u[k2];
  }
  __syncthreads();
  // z transform, step A in place on the stick columns (stick y sits at column dperm(y))
  for (int w = tid; w < N2 * ns; w += nt) {
    const int s = w % ns, t = w / ns, col = dperm<NP>(sy[s]);
    C v[N1];
#pragma unroll
    for (int j = 0; j < N1; ++j) v[j] = S[(j * N2 + t) * NP + col];
    RegDft<T, N1>::run(v, (T)-1);
#pragma unroll
    for (int k1 = 1; k1 < N1; ++k1)
      if (t) v[k1] = cmul(v[k1], tw_ld<T>(tw, (t * k1) % NP, (T)-1));
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) S[(k1 * N2 + t) * NP + col] = v[k1];
  }
  __syncthreads();
  // z transform, step B: thread (k1, stick); gather x 1/N plus kinetic into the output column
  const int* pm = pwmap + (long)slot * P;
  for (int w = tid; w < N1 * ns; w += nt) {
    const int s = w % ns, k1 = w / ns, y = sy[s], col = dperm<NP>(y);
    C u[N2];
#pragma unroll
    for (int t = 0; t < N2; ++t) u[t] = S[(k1 * N2 + t) * NP + col];
    RegDft<T, N2>::run(u, (T)-1);
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) {
      const int z = k1 + N1 * k2;
      const int g = __ldg(pm + z * NP + y);
      if (g >= 0) {
        const double2 xv = __ldg(x + b * npw + g);
        const double kin = __ldg(kinetic + g);
        double2 o;
        o.x = kin * xv.x + (double)u[k2].x * invN;
        o.y = kin * xv.y + (double)u[k2].y * invN;
        y_out[b * npw + g] = o;
      }
    }
  }
}

template <typename T, int NX>
__global__ void __launch_bounds__(256) k_xline4(cplx<T>* __restrict__ W, int n_act, const int* __restrict__ slot_of_x,
                                                const T* __restrict__ Vt, int P, int ncols, int cols_per_cta,
                                                const cplx<T>* __restrict__ tw) {
  using C = cplx<T>;
  constexpr int N1 = Split<NX>::N1, N2 = Split<NX>::N2;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int J = blockDim.x;
  C* B1 = reinterpret_cast<C*>(smraw);  // [N1*N2][J]
  C* B2 = B1 + NX * J;                   // [N2*N1][J]
  const int l = threadIdx.x, ky = threadIdx.y;
  const int j0 = blockIdx.x * J;
  const bool lv = (j0 + l) < P;
  const int c0 = blockIdx.y * cols_per_cta;
  const int c1 = min(ncols, c0 + cols_per_cta);
  T vr[N2];
#pragma unroll
  for (int k2 = 0; k2 < N2; ++k2) vr[k2] = lv ? __ldg(Vt + (long)(ky + N1 * k2) * P + j0 + l) : (T)0;
  for (int c = c0; c < c1; ++c) {
    C* Wc = W + (long)c * n_act * P + j0 + l;
    if (ky < N2) {  // inverse, step A
      C v[N1];
#pragma unroll
      for (int j = 0; j < N1; ++j) {
        const int s = __ldg(slot_of_x + j * N2 + ky);
        v[j] = (s >= 0 && lv) ? Wc[(long)s * P] : mk<C>(0.0, 0.0);
      }
      RegDft<T, N1>::run(v, (T)1);
#pragma unroll
      for (int k1 = 1; k1 < N1; ++k1)
        if (ky) v[k1] = cmul(v[k1], tw_ld<T>(tw, (ky * k1) % NX, (T)1));
#pragma unroll
      for (int k1 = 0; k1 < N1; ++k1) B1[(k1 * N2 + ky) * J + l] = v[k1];
    }
    __syncthreads();
    {  // inverse step B, x V(r), forward step A (lengths swapped: N1f = N2, N2f = N1)
      C u[N2];
#pragma unroll
      for (int t = 0; t < N2; ++t) u[t] = B1[(ky * N2 + t) * J + l];
      RegDft<T, N2>::run(u, (T)1);
#pragma unroll
      for (int k2 = 0; k2 < N2; ++k2) u[k2] = cscale(u[k2], vr[k2]);
      RegDft<T, N2>::run(u, (T)-1);
#pragma unroll
      for (int k1f = 1; k1f < N2; ++k1f)
        if (ky) u[k1f] = cmul(u[k1f], tw_ld<T>(tw, (ky * k1f) % NX, (T)-1));
#pragma unroll
      for (int k1f = 0; k1f < N2; ++k1f) B2[(k1f * N1 + ky) * J + l] = u[k1f];
    }
    __syncthreads();
    if (ky < N2) {  // forward step B: frequencies ky + N2 * k2f
      C v[N1];
#pragma unroll
      for (int t = 0; t < N1; ++t) v[t] = B2[(ky * N1 + t) * J + l];
      RegDft<T, N1>::run(v, (T)-1);
#pragma unroll
      for (int k2f = 0; k2f < N1; ++k2f) {
        const int s = __ldg(slot_of_x + ky + N2 * k2f);
        if (s >= 0 && lv) Wc[(long)s * P] = v[k2f];
      }
    }
  }
}

// Geometry of the warp-synchronous x-line pass: a line's x transform is done by N2 lanes of one
// warp (LW lines per warp).  Exchange-buffer stride S >= NX with S = N2 (mod 8), so the step-A writes
// of the N2 lanes of consecutive lines fall in distinct 16-byte bank groups.
template <int NX> struct XLineGeom {
  static constexpr int N1 = Split<NX>::N1, N2 = Split<NX>::N2;
  static constexpr int LW = 32 / N2;
  static constexpr int Q = (N1 + N2 - 1) / N2;
  static constexpr int S = NX + ((N2 - NX) % 8 + 8) % 8;
};
constexpr int kXlWarps = 3;

// x-line pass with every lane busy in every phase: lane t of a line
//   1. inverse step A for index t: DFT_N1 over the inputs x = m N2 + t (the active slots),
//   2. for its rows k1 = t, t + N2, ... < N1: inverse step B (DFT_N2), x V(r) at x = k1 + N1 k2,
//      forward step A (DFT_N2, lengths swapped) and its twiddles,
//   3. forward step B for frequency index t: DFT_N1, outputs x = t + N2 m back to the active slots.
// The exchanges go through two per-warp shared buffers with __syncwarp only (no block barriers);
// the input and output slot sets of a lane coincide ({t + N2 m}).  V(r) and the slot table are read
// through L1 (reused by the CTA's columns) instead of being held in registers.
template <typename T, int NX>
__global__ void __launch_bounds__(kXlWarps * 32, 5) k_xline5(cplx<T>* __restrict__ W, int n_act, const int* __restrict__ slot_of_x,
                                                             const T* __restrict__ Vt, int P, int ncols, int cols_per_cta,
                                                             const cplx<T>* __restrict__ tw) {
  using C = cplx<T>;
  using G = XLineGeom<NX>;
  constexpr int N1 = G::N1, N2 = G::N2, LW = G::LW, Q = G::Q, S = G::S;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int L = lane / N2, t = lane - L * N2;
  const bool lane_ok = L < LW;
  C* B1 = reinterpret_cast<C*>(smraw) + ((size_t)warp * LW + (lane_ok ? L : 0)) * S;
  C* B2 = B1 + (size_t)kXlWarps * LW * S;
  const int j = (blockIdx.x * kXlWarps + warp) * LW + L;
  const bool lv = lane_ok && j < P;
  const int c0 = blockIdx.y * cols_per_cta;
  const int c1 = min(ncols, c0 + cols_per_cta);
  const int* slt = slot_of_x + t;  // slot of x = t + N2 m at slt[N2 m]
  for (int c = c0; c < c1; ++c) {
    C* Wc = W + (long)c * n_act * P + j;
    {  // 1. inverse step A
      C v[N1];
#pragma unroll
      for (int m = 0; m < N1; ++m) {
        const int sm = lv ? __ldg(slt + N2 * m) : -1;
        v[m] = sm >= 0 ? Wc[(long)sm * P] : mk<C>(0.0, 0.0);
      }
      RegDft<T, N1>::run(v, (T)1);
#pragma unroll
      for (int k1 = 1; k1 < N1; ++k1)
        if (t) v[k1] = cmul(v[k1], tw_ld<T>(tw, (t * k1) % NX, (T)1));
      if (lane_ok) {
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1) B1[k1 * N2 + t] = v[k1];
      }
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < Q; ++q) {  // 2. inverse step B, x V(r), forward step A
      const int k1 = t + N2 * q;
      if (lane_ok && k1 < N1) {
        C u[N2];
#pragma unroll
        for (int tt = 0; tt < N2; ++tt) u[tt] = B1[k1 * N2 + tt];
        RegDft<T, N2>::run(u, (T)1);
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) u[k2] = cscale(u[k2], lv ? __ldg(Vt + (long)(k1 + N1 * k2) * P + j) : (T)0);
        RegDft<T, N2>::run(u, (T)-1);
#pragma unroll
        for (int k1f = 1; k1f < N2; ++k1f)
          if (k1) u[k1f] = cmul(u[k1f], tw_ld<T>(tw, (k1 * k1f) % NX, (T)-1));
#pragma unroll
        for (int k1f = 0; k1f < N2; ++k1f) B2[k1f * N1 + k1] = u[k1f];
      }
    }
    __syncwarp();
    {  // 3. forward step B for frequency index t
      C v[N1];
#pragma unroll
      for (int tf = 0; tf < N1; ++tf) v[tf] = lane_ok ? B2[t * N1 + tf] : mk<C>(0.0, 0.0);
      RegDft<T, N1>::run(v, (T)-1);
#pragma unroll
      for (int m = 0; m < N1; ++m) {
        const int sm = lv ? __ldg(slt + N2 * m) : -1;
        if (sm >= 0) Wc[(long)sm * P] = v[m];
      }
    }
    __syncwarp();
  }
}

template <typename T, int NX>
__global__ void __launch_bounds__(256) k_xline_density4(const cplx<T>* __restrict__ W, int n_act,
                                                        const int* __restrict__ slot_of_x, int P, int ncols,
                                                        const cplx<T>* __restrict__ tw, const double* __restrict__ wgt,
                                                        double inv_vol, double* __restrict__ rho) {
  using C = cplx<T>;
  constexpr int N1 = Split<NX>::N1, N2 = Split<NX>::N2;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int J = blockDim.x;
  C* B1 = reinterpret_cast<C*>(smraw);
  const int l = threadIdx.x, ky = threadIdx.y;
  const int j0 = blockIdx.x * J;
  const bool lv = (j0 + l) < P;
  double acc[N2];
#pragma unroll
  for (int k2 = 0; k2 < N2; ++k2) acc[k2] = 0.0;
  for (int c = 0; c < ncols; ++c) {
    const C* Wc = W + (long)c * n_act * P + j0 + l;
    if (ky < N2) {
      C v[N1];
#pragma unroll
      for (int j = 0; j < N1; ++j) {
        const int s = __ldg(slot_of_x + j * N2 + ky);
        v[j] = (s >= 0 && lv) ? Wc[(long)s * P] : mk<C>(0.0, 0.0);
      }
      RegDft<T, N1>::run(v, (T)1);
#pragma unroll
      for (int k1 = 1; k1 < N1; ++k1)
        if (ky) v[k1] = cmul(v[k1], tw_ld<T>(tw, (ky * k1) % NX, (T)1));
#pragma unroll
      for (int k1 = 0; k1 < N1; ++k1) B1[(k1 * N2 + ky) * J + l] = v[k1];
    }
    __syncthreads();
    C u[N2];
#pragma unroll
    for (int t = 0; t < N2; ++t) u[t] = B1[(ky * N2 + t) * J + l];
    RegDft<T, N2>::run(u, (T)1);
    const double wc = __ldg(wgt + c) * inv_vol;
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) acc[k2] += wc * ((double)u[k2].x * (double)u[k2].x + (double)u[k2].y * (double)u[k2].y);
    __syncthreads();
  }
  if (lv) {
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) rho[(long)(j0 + l) * NX + ky + N1 * k2] += acc[k2];
  }
}

// ------------------------------------------------------------------------------------------
// Host side
// ------------------------------------------------------------------------------------------

static constexpr size_t kSmem4 = 227 * 1024;

// Shared memory of a plane pass: `buffers` planes of N^2 complex plus the stick list and flags.
static size_t plane_smem_bytes(size_t cs, int N, int buffers) {
  return buffers * cs * (size_t)N * N + sizeof(int) * N + N + 16;
}
template <typename T, int N>
static size_t plane_smem(int buffers) {
  return plane_smem_bytes(sizeof(cplx<T>), N, buffers);
}

// DFTCUDA_FFT4=legacy selects the earlier two-buffer plane passes and the block-barrier x-line
// pass (for A/B measurements); the default single-buffer and warp-synchronous kernels fit planes up
// to 119^2 in FP64.
static bool fft4_legacy() {
  static const bool v = [] {
    const char* e = std::getenv("DFTCUDA_FFT4");
    return e && std::string(e) == "legacy";
  }();
  return v;
}

bool kctx_fast_path_ok(const dftcuda_kctx* c, int precision) {
  if (!four_step_supported(c->nx) || !four_step_supported(c->ny) || c->ny != c->nz) return false;
  const size_t cs = precision == DFTCUDA_PRECISION_FP32 ? sizeof(float2) : sizeof(double2);
  return plane_smem_bytes(cs, c->ny, fft4_legacy() ? 2 : 1) <= kSmem4;
}

template <typename T, int NP>
static int launch_plane_inv4(dftcuda_kctx* c, const double2* x, cplx<T>* W, size_t ncols, cudaStream_t s) {
  const cplx<T>* tw5 = std::is_same<T, double>::value ? (const cplx<T>*)c->d_tw4p64 : (const cplx<T>*)c->d_tw4p32;
  if (!fft4_legacy()) {
    DFT_TRY(ensure_max_dynamic_smem((const void*)k_plane_inv5<T, NP>, (int)kSmem4));
    dim3 g(c->n_act, (unsigned)ncols);
    k_plane_inv5<T, NP><<<g, kPlaneThreads, plane_smem<T, NP>(1), s>>>(x, (long)c->npw, W, c->n_act, c->d_pwmap, c->d_stick_off,
                                                              c->d_stick_y, tw5);
    count_launch();
    return DFTCUDA_OK;
  }
  const size_t smem = plane_smem<T, NP>(2);
  DFT_TRY(ensure_max_dynamic_smem((const void*)k_plane_inv4<T, NP>, (int)kSmem4));
  const cplx<T>* tw = std::is_same<T, double>::value ? (const cplx<T>*)c->d_tw4p64 : (const cplx<T>*)c->d_tw4p32;
  dim3 g(c->n_act, (unsigned)ncols);
  k_plane_inv4<T, NP><<<g, 512, smem, s>>>(x, (long)c->npw, W, c->n_act, c->d_pwmap, c->d_stick_off, c->d_stick_y, tw); count_launch();
  return DFTCUDA_OK;
}

template <typename T, int NP>
static int launch_plane_fwd4(dftcuda_kctx* c, const cplx<T>* W, const double2* x, double2* y, size_t ncols,
                             cudaStream_t s) {
  if (!fft4_legacy()) {
    DFT_TRY(ensure_max_dynamic_smem((const void*)k_plane_fwd5<T, NP>, (int)kSmem4));
    const cplx<T>* tw5 = std::is_same<T, double>::value ? (const cplx<T>*)c->d_tw4p64 : (const cplx<T>*)c->d_tw4p32;
    dim3 g(c->n_act, (unsigned)ncols);
    k_plane_fwd5<T, NP><<<g, kPlaneThreads, plane_smem<T, NP>(1), s>>>(W, c->n_act, c->d_pwmap, c->d_stick_off, c->d_stick_y, tw5, x, y,
                                                              (long)c->npw, c->d_kinetic, 1.0 / (double)c->N);
    count_launch();
    return DFTCUDA_OK;
  }
  const size_t smem = plane_smem<T, NP>(2);
  DFT_TRY(ensure_max_dynamic_smem((const void*)k_plane_fwd4<T, NP>, (int)kSmem4));
  const cplx<T>* tw = std::is_same<T, double>::value ? (const cplx<T>*)c->d_tw4p64 : (const cplx<T>*)c->d_tw4p32;
  dim3 g(c->n_act, (unsigned)ncols);
  k_plane_fwd4<T, NP><<<g, 512, smem, s>>>(W, c->n_act, c->d_pwmap, c->d_stick_off, c->d_stick_y, tw, x, y, (long)c->npw,
                                           c->d_kinetic, 1.0 / (double)c->N); count_launch();
  return DFTCUDA_OK;
}

template <typename T, int NX>
static int launch_xline4(dftcuda_kctx* c, cplx<T>* W, size_t ncols, cudaStream_t s) {
  constexpr int N1 = Split<NX>::N1;
  const T* vt = std::is_same<T, double>::value ? (const T*)c->d_vt : (const T*)c->d_vt32;
  const cplx<T>* tw = std::is_same<T, double>::value ? (const cplx<T>*)c->d_tw4x64 : (const cplx<T>*)c->d_tw4x32;
  if (!fft4_legacy()) {
    using G = XLineGeom<NX>;
    const size_t smem5 = 2 * sizeof(cplx<T>) * (size_t)kXlWarps * G::LW * G::S;
    DFT_TRY(ensure_max_dynamic_smem((const void*)k_xline5<T, NX>, (int)kSmem4));
    const int cpc = 4;
    dim3 g(ceil_div(c->P, kXlWarps * G::LW), ceil_div(ncols, cpc));
    k_xline5<T, NX><<<g, kXlWarps * 32, smem5, s>>>(W, c->n_act, c->d_slot_of_x, vt, c->P, (int)ncols, cpc, tw);
    count_launch();
    return DFTCUDA_OK;
  }
  const int J = N1 > 8 ? 16 : 32;
  DFT_TRY(ensure_max_dynamic_smem((const void*)k_xline4<T, NX>, (int)kSmem4));
  const size_t smem = 2 * sizeof(cplx<T>) * (size_t)NX * J;
  const int cpc = 4;
  dim3 g(ceil_div(c->P, J), ceil_div(ncols, cpc));
  dim3 b(J, N1);
  k_xline4<T, NX><<<g, b, smem, s>>>(W, c->n_act, c->d_slot_of_x, vt, c->P, (int)ncols, cpc, tw); count_launch();
  return DFTCUDA_OK;
}

template <typename T, int NX>
static int launch_xline_density4(dftcuda_kctx* c, const cplx<T>* W, size_t ncols, const double* w, double* rho,
                                 cudaStream_t s) {
  constexpr int N1 = Split<NX>::N1;
  const int J = N1 > 8 ? 16 : 32;
  DFT_TRY(ensure_max_dynamic_smem((const void*)k_xline_density4<T, NX>, (int)kSmem4));
  const size_t smem = sizeof(cplx<T>) * (size_t)NX * J;
  dim3 g(ceil_div(c->P, J));
  dim3 b(J, N1);
  const cplx<T>* tw = std::is_same<T, double>::value ? (const cplx<T>*)c->d_tw4x64 : (const cplx<T>*)c->d_tw4x32;
  k_xline_density4<T, NX><<<g, b, smem, s>>>(W, c->n_act, c->d_slot_of_x, c->P, (int)ncols, tw, w, 1.0 / c->volume, rho); count_launch();
  return DFTCUDA_OK;
}

template <typename T>
static int dispatch_plane_inv4(dftcuda_kctx* c, const double2* x, cplx<T>* W, size_t ncols, cudaStream_t s) {
  switch (c->ny) {
#define X(N) \
  case N: return launch_plane_inv4<T, N>(c, x, W, ncols, s);
    DFTCUDA_FOUR_STEP_LENGTHS(X)
#undef X
    default: return fail(DFTCUDA_ERR_UNSUPPORTED, "plane length without a four-step kernel");
  }
}
template <typename T>
static int dispatch_plane_fwd4(dftcuda_kctx* c, const cplx<T>* W, const double2* x, double2* y, size_t ncols,
                               cudaStream_t s) {
  switch (c->ny) {
#define X(N) \
  case N: return launch_plane_fwd4<T, N>(c, W, x, y, ncols, s);
    DFTCUDA_FOUR_STEP_LENGTHS(X)
#undef X
    default: return fail(DFTCUDA_ERR_UNSUPPORTED, "plane length without a four-step kernel");
  }
}
template <typename T>
static int dispatch_xline4(dftcuda_kctx* c, cplx<T>* W, size_t ncols, cudaStream_t s) {
  switch (c->nx) {
#define X(N) \
  case N: return launch_xline4<T, N>(c, W, ncols, s);
    DFTCUDA_FOUR_STEP_LENGTHS(X)
#undef X
    default: return fail(DFTCUDA_ERR_UNSUPPORTED, "x length without a four-step kernel");
  }
}
template <typename T>
static int dispatch_xline_density4(dftcuda_kctx* c, const cplx<T>* W, size_t ncols, const double* w, double* rho,
                                   cudaStream_t s) {
  switch (c->nx) {
#define X(N) \
  case N: return launch_xline_density4<T, N>(c, W, ncols, w, rho, s);
    DFTCUDA_FOUR_STEP_LENGTHS(X)
#undef X
    default: return fail(DFTCUDA_ERR_UNSUPPORTED, "x length without a four-step kernel");
  }
}

template <typename T>
int local_block4(dftcuda_kctx* c, const double2* x, double2* y, size_t ncols, cudaStream_t s) {
  cplx<T>* W = reinterpret_cast<cplx<T>*>(c->d_box);
  {
    ProfScope ps(c, P_PLANE_INV, s);
    DFT_TRY(dispatch_plane_inv4<T>(c, x, W, ncols, s));
  }
  {
    ProfScope ps(c, P_XLINE, s);
    DFT_TRY(dispatch_xline4<T>(c, W, ncols, s));
  }
  {
    ProfScope ps(c, P_PLANE_FWD, s);
    DFT_TRY(dispatch_plane_fwd4<T>(c, W, x, y, ncols, s));
  }
  DFT_CUDA_TRY(cudaGetLastError());
  return DFTCUDA_OK;
}
template int local_block4<double>(dftcuda_kctx*, const double2*, double2*, size_t, cudaStream_t);
template int local_block4<float>(dftcuda_kctx*, const double2*, double2*, size_t, cudaStream_t);

template <typename T>
int density_block4(dftcuda_kctx* c, const double2* x, size_t ncols, const double* w, double* rho, cudaStream_t s) {
  cplx<T>* W = reinterpret_cast<cplx<T>*>(c->d_box);
  ProfScope ps(c, P_DENSITY, s);
  DFT_TRY(dispatch_plane_inv4<T>(c, x, W, ncols, s));
  DFT_TRY(dispatch_xline_density4<T>(c, W, ncols, w, rho, s));
  DFT_CUDA_TRY(cudaGetLastError());
  return DFTCUDA_OK;
}
template int density_block4<double>(dftcuda_kctx*, const double2*, size_t, const double*, double*, cudaStream_t);
template int density_block4<float>(dftcuda_kctx*, const double2*, size_t, const double*, double*, cudaStream_t);

// Per-context tables of the four-step path: slot of every x frequency, per-plane (z, y) ->
// plane-wave map, stick lists and the four-step twiddles of the x and plane lengths.
int kctx_setup_fast_path(dftcuda_kctx* c, const std::vector<int>& slot_of_x, const std::vector<int>& xpos,
                         const int32_t* hkl) {
  c->fast64 = kctx_fast_path_ok(c, DFTCUDA_PRECISION_FP64);
  c->fast32 = kctx_fast_path_ok(c, DFTCUDA_PRECISION_FP32);
  if (!c->fast64 && !c->fast32) return DFTCUDA_OK;
  DFT_TRY(init_root_tables_here());
  const int nx = c->nx, ny = c->ny, nz = c->nz, P = c->P, n_act = c->n_act;
  std::vector<int> pwmap((size_t)n_act * P, -1);
  std::vector<std::vector<int>> sticks(n_act);
  std::vector<std::vector<char>> has(n_act, std::vector<char>(ny, 0));
  for (size_t i = 0; i < c->npw; ++i) {
    const int s = slot_of_x[xpos[i]];
    const int yy = ((hkl[3 * i + 1] % ny) + ny) % ny, zz = ((hkl[3 * i + 2] % nz) + nz) % nz;
    pwmap[(size_t)s * P + zz * ny + yy] = (int)i;
    if (!has[s][yy]) {
      has[s][yy] = 1;
      sticks[s].push_back(yy);
    }
  }
  std::vector<int> soff(n_act + 1, 0), sy;
  for (int s = 0; s < n_act; ++s) {
    std::sort(sticks[s].begin(), sticks[s].end());
    soff[s + 1] = soff[s] + (int)sticks[s].size();
    sy.insert(sy.end(), sticks[s].begin(), sticks[s].end());
  }
  std::vector<int> sox(nx, -1);
  for (int x = 0; x < nx; ++x) sox[x] = slot_of_x[x];
  auto roots = [](int n, std::vector<double2>& r64, std::vector<float2>& r32) {
    r64.resize(n);
    r32.resize(n);
    for (int e = 0; e < n; ++e) {
      const double a = 2.0 * M_PI * (double)e / (double)n;
      r64[e] = make_double2(std::cos(a), std::sin(a));
      r32[e] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
  };
  std::vector<double2> tx64, tp64;
  std::vector<float2> tx32, tp32;
  roots(nx, tx64, tx32);
  roots(ny, tp64, tp32);
  bool ok = dev_malloc(&c->d_pwmap, sizeof(int) * pwmap.size()) == cudaSuccess &&
            dev_malloc(&c->d_stick_off, sizeof(int) * soff.size()) == cudaSuccess &&
            dev_malloc(&c->d_stick_y, sizeof(int) * std::max<size_t>(sy.size(), 1)) == cudaSuccess &&
            dev_malloc(&c->d_slot_of_x, sizeof(int) * nx) == cudaSuccess &&
            dev_malloc(&c->d_tw4x64, sizeof(double2) * nx) == cudaSuccess &&
            dev_malloc(&c->d_tw4x32, sizeof(float2) * nx) == cudaSuccess &&
            dev_malloc(&c->d_tw4p64, sizeof(double2) * ny) == cudaSuccess &&
            dev_malloc(&c->d_tw4p32, sizeof(float2) * ny) == cudaSuccess;
  if (!ok) return fail(DFTCUDA_ERR_OUT_OF_MEMORY, "four-step tables");
  cudaStream_t st = c->stream;
  cudaMemcpyAsync(c->d_pwmap, pwmap.data(), sizeof(int) * pwmap.size(), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(c->d_stick_off, soff.data(), sizeof(int) * soff.size(), cudaMemcpyHostToDevice, st);
  if (!sy.empty()) cudaMemcpyAsync(c->d_stick_y, sy.data(), sizeof(int) * sy.size(), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(c->d_slot_of_x, sox.data(), sizeof(int) * nx, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(c->d_tw4x64, tx64.data(), sizeof(double2) * nx, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(c->d_tw4x32, tx32.data(), sizeof(float2) * nx, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(c->d_tw4p64, tp64.data(), sizeof(double2) * ny, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(c->d_tw4p32, tp32.data(), sizeof(float2) * ny, cudaMemcpyHostToDevice, st);
  DFT_CUDA_TRY(cudaStreamSynchronize(st));
  return DFTCUDA_OK;
}

}  // namespace dftcuda
