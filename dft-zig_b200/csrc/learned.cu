// Preconditioners for the Davidson correction step (the reference's is common.zig:214-226) and the
// training kernels of the learned one.
//
//   kind 0  reference:  q_i = r_i / (|k+G_i|^2 - lambda_b), |den| clamped at 1e-8 (eig.cu)
//   kind 1  Teter-Payne-Allan: q_i = K(x_i) r_i, x_i = |k+G_i|^2 / E_kin,b,
//           K(x) = (27 + 18x + 12x^2 + 8x^3) / (27 + 18x + 12x^2 + 8x^3 + 16x^4)
//           (Teter, Payne, Allan, Phys. Rev. B 40, 12255 (1989)); E_kin,b = <psi_b|T|psi_b>
//   kind 2  learned: q_i = m_theta(u_i) r_i with a per-plane-wave MLP, FP32 weights,
//           u_i = (log(x_i + 0.05), log(|r_i| / rms(r_b) + 1e-6), t / 20), t the iteration index,
//           h1 = tanh(W1 u + b1), h2 = tanh(W2 h1 + b2), z = w3 . h2 + b3 (3 -> 64 -> 64 -> 1),
//           m = K(x_i) exp(clamp(z, -8, 8)): a learned refinement of Teter-Payne-Allan.
//
// Training (dftcuda_precond_mlp_loss_grad / _train): samples are bands b with plane-wave data
// c_i = conj(r_i) delta_i, w_i = |r_i|^2 and D_b = ||delta_b||^2, where delta is the correction that
// would have taken the Ritz vector to the converged eigenvector.  The loss is scale-free, as the
// Davidson step is:  L = mean_b [1 - |A_b|^2 / (Q_b D_b)],  A_b = sum_i m_i c_i,  Q_b = sum_i m_i^2 w_i
// (one minus the squared cosine between the preconditioned residual and the ideal correction).
// One CTA per band for the forward sums; the backward pass recomputes the activations per tile of
// 128 plane waves and accumulates the weight gradients as small tile GEMMs in registers.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "kctx.cuh"

namespace dftcuda {

constexpr int MLP_H = 64;
constexpr int MLP_IN = 3;
// parameter layout: W1[64][3], b1[64], W2[64][64] (row = output), b2[64], w3[64], b3
constexpr int MLP_OFF_W1 = 0;
constexpr int MLP_OFF_B1 = MLP_OFF_W1 + MLP_H * MLP_IN;
constexpr int MLP_OFF_W2 = MLP_OFF_B1 + MLP_H;
constexpr int MLP_OFF_B2 = MLP_OFF_W2 + MLP_H * MLP_H;
constexpr int MLP_OFF_W3 = MLP_OFF_B2 + MLP_H;
constexpr int MLP_OFF_B3 = MLP_OFF_W3 + MLP_H;
constexpr int MLP_NPARAM = MLP_OFF_B3 + 1;  // 4481
static_assert(MLP_NPARAM == DFTCUDA_PRECOND_MLP_PARAMS, "parameter count");

// The learned multiplier refines Teter-Payne-Allan: m = K(x) exp(clamp(z)), x = exp(u0) - 0.05 the
// kinetic ratio recovered from the first feature; with zero output weights the network is TPA.
__device__ __forceinline__ double tpa_k(double x) {
  const double num = 27.0 + x * (18.0 + x * (12.0 + 8.0 * x));
  return num / (num + 16.0 * x * x * x * x);
}
__device__ __forceinline__ float zclamp(float z) { return fminf(fmaxf(z, -8.f), 8.f); }
__device__ __forceinline__ double mlp_multiplier(float u0, float z) {
  return tpa_k(fmax(exp((double)u0) - 0.05, 0.0)) * exp((double)zclamp(z));
}

// Forward for one input with the parameters in shared memory; returns z (the log of the multiplier
// relative to TPA) and
// optionally the two hidden layers.
__device__ __forceinline__ float mlp_forward(const float* __restrict__ p, const float u[3], float* h1, float* h2) {
  float a1[MLP_H];
#pragma unroll
  for (int j = 0; j < MLP_H; ++j) {
    const float* w = p + MLP_OFF_W1 + j * MLP_IN;
    a1[j] = tanhf(fmaf(w[0], u[0], fmaf(w[1], u[1], fmaf(w[2], u[2], p[MLP_OFF_B1 + j]))));
  }
  float z = p[MLP_OFF_B3];
#pragma unroll 4
  for (int j = 0; j < MLP_H; ++j) {
    const float* w = p + MLP_OFF_W2 + j * MLP_H;
    float s = p[MLP_OFF_B2 + j];
#pragma unroll
    for (int i = 0; i < MLP_H; ++i) s = fmaf(w[i], a1[i], s);
    const float t = tanhf(s);
    if (h2) h2[j] = t;
    z = fmaf(p[MLP_OFF_W3 + j], t, z);
  }
  if (h1) {
#pragma unroll
    for (int j = 0; j < MLP_H; ++j) h1[j] = a1[j];
  }
  return z;
}

__device__ __forceinline__ void mlp_features(double kin, double ekin, double rabs, double rms, double t, float u[3]) {
  const double x = kin / fmax(ekin, 1e-6);
  u[0] = (float)log(x + 0.05);
  u[1] = (float)log(rabs / fmax(rms, 1e-300) + 1e-6);
  u[2] = (float)fmin(t / 20.0, 2.0);
}

// E_kin,b = sum_i kin_i |psi_b,i|^2 for the bands in the list (one CTA per band).
__global__ void k_band_kinetic(const double2* __restrict__ ritz, const double* __restrict__ kin, const int* __restrict__ band,
                               long n, double* __restrict__ ekin) {
  __shared__ double red[256];
  const int b = band[blockIdx.x];
  const double2* v = ritz + (long)b * n;
  double s = 0.0;
  for (long i = threadIdx.x; i < n; i += blockDim.x) s += kin[i] * (v[i].x * v[i].x + v[i].y * v[i].y);
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) ekin[blockIdx.x] = red[0];
}

__global__ void k_precondition_tpa(double2* __restrict__ Q, const double2* __restrict__ res, const double* __restrict__ kin,
                                   const double* __restrict__ ekin, const int* __restrict__ band, int k, long n) {
  const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (idx >= (long)k * n) return;
  const int j = (int)(idx / n);
  const long i = idx - (long)j * n;
  const double x = kin[i] / fmax(ekin[j], 1e-6);
  const double num = 27.0 + x * (18.0 + x * (12.0 + 8.0 * x));
  const double f = num / (num + 16.0 * x * x * x * x);
  const double2 v = res[(long)band[j] * n + i];
  Q[idx] = make_double2(v.x * f, v.y * f);
}

// Inference through a table (the default).  The network's output z depends on the entry only through
// (u0, u1); u2 = t/20 is fixed within a call.  So each call (or the first call at a new t) tabulates z
// with the FP32 network of the training kernels (mlp_forward) on a kLutN0 x kLutN1 grid over
// u0 in [kLutU0, kLutU0Hi] (x from 0 to about 1100) and u1 in [kLutU1, kLutU1Hi] (|r_i| / rms(r) from
// 0 to about 1100), and every entry interpolates the table bilinearly: for the trained weights
// |dz| <= 5e-5 over the grid (the tensor-core form below moves z by ~1e-3).  An entry outside the
// grid evaluates the network itself.  DFTCUDA_MLP_INFER=tc selects the tensor-core form.
constexpr int kLutN0 = 256, kLutN1 = 512;
constexpr float kLutU0 = -3.0f, kLutU0Hi = 7.0f, kLutU1 = -13.85f, kLutU1Hi = 7.0f;
constexpr int kMlpParamPad = (MLP_NPARAM + 63) / 64 * 64;  // the table starts 256-byte aligned

__global__ void __launch_bounds__(128) k_mlp_table(const float* __restrict__ params, double t, float* __restrict__ lut) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= kLutN0 * kLutN1) return;
  const int a = idx / kLutN1, b = idx - a * kLutN1;
  float u[3];
  u[0] = kLutU0 + (kLutU0Hi - kLutU0) * (float)a / (float)(kLutN0 - 1);
  u[1] = kLutU1 + (kLutU1Hi - kLutU1) * (float)b / (float)(kLutN1 - 1);
  u[2] = (float)fmin(t / 20.0, 2.0);
  lut[idx] = mlp_forward(params, u, nullptr, nullptr);
}

// The network for an entry outside the table, kept out of line so that the table path keeps a small
// register footprint.
__device__ __noinline__ float mlp_forward_outside(const float* __restrict__ params, float u0, float u1, float u2) {
  const float u[3] = {u0, u1, u2};
  return mlp_forward(params, u, nullptr, nullptr);
}

__global__ void __launch_bounds__(256, 4) k_precondition_lut(double2* __restrict__ Q, const double2* __restrict__ res,
                                                          const double* __restrict__ kin, const double* __restrict__ ekin,
                                                          const double* __restrict__ norms, const int* __restrict__ band,
                                                          int k, long n, double t, const float* __restrict__ lut,
                                                          const float* __restrict__ params) {
  const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (idx >= (long)k * n) return;
  const int j = (int)(idx / n);
  const long i = idx - (long)j * n;
  const int b = band[j];
  const double2 v = res[(long)b * n + i];
  float u[3];
  mlp_features(kin[i], ekin[j], sqrt(v.x * v.x + v.y * v.y), norms[b] / sqrt((double)n), t, u);
  constexpr float s0 = (float)(kLutN0 - 1) / (kLutU0Hi - kLutU0), s1 = (float)(kLutN1 - 1) / (kLutU1Hi - kLutU1);
  const float f0 = (u[0] - kLutU0) * s0, f1 = (u[1] - kLutU1) * s1;
  float z;
  if (f0 >= 0.f && f0 < (float)(kLutN0 - 1) && f1 >= 0.f && f1 < (float)(kLutN1 - 1)) {
    const int i0 = (int)f0, i1 = (int)f1;
    const float a = f0 - (float)i0, c = f1 - (float)i1;
    const float* r0 = lut + i0 * kLutN1 + i1;
    const float z0 = fmaf(c, __ldg(r0 + 1) - __ldg(r0), __ldg(r0));
    const float z1 = fmaf(c, __ldg(r0 + kLutN1 + 1) - __ldg(r0 + kLutN1), __ldg(r0 + kLutN1));
    z = fmaf(a, z1 - z0, z0);
  } else {
    z = mlp_forward_outside(params, u[0], u[1], u[2]);
  }
  const double m = mlp_multiplier(u[0], z);
  Q[idx] = make_double2(v.x * m, v.y * m);
}

static bool mlp_infer_tc() {
  static const bool v = [] {
    const char* e = std::getenv("DFTCUDA_MLP_INFER");
    return e && std::strcmp(e, "tc") == 0;
  }();
  return v;
}

// Inference (the Davidson preconditioner) over tiles of MLP_TE plane-wave entries.  The first layer
// per entry, then the 64 x 64 second layer on the tensor cores (mma.sync m16n8k8, TF32 operands,
// FP32 accumulation; each warp takes 16 entries x 64 hidden units), its tanh and the output layer on
// the accumulator fragments, and a shuffle sum over the four lanes that share an entry.  TF32
// operands and the hardware tanh (tanh.approx.f32) move the learned multiplier by ~1e-3 relative
// from the FP32 network of mlp_forward (the training kernels); a preconditioner only steers the
// Davidson corrections, so the eigenpairs it converges to are unchanged.
constexpr int MLP_TE = 128;             // entries per tile
constexpr int MLP_IT = 256;             // threads: 8 warps x 16 entries
constexpr int MLP_AS = MLP_TE + 8;      // activation row stride (conflict-free fragment loads)
constexpr int MLP_WS = MLP_H + 8;       // transposed-weight row stride
struct MlpInferSmem {
  uint32_t a[MLP_H][MLP_AS];    // first-layer activations (TF32 bits), hidden unit major
  uint32_t w2t[MLP_H][MLP_WS];  // W2 transposed (TF32 bits): w2t[i][j] = W2[j][i]
  float w1[MLP_H * MLP_IN], b1[MLP_H], b2[MLP_H], w3[MLP_H];
  float u0[MLP_TE];
  double m[MLP_TE];
};

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float tanh_hw(float x) {
  float r;
  asm("tanh.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

__global__ void __launch_bounds__(MLP_IT) k_precondition_mlp(double2* __restrict__ Q, const double2* __restrict__ res,
                                                             const double* __restrict__ kin, const double* __restrict__ ekin,
                                                             const double* __restrict__ norms, const int* __restrict__ band,
                                                             int k, long n, double t, const float* __restrict__ params) {
  extern __shared__ __align__(16) unsigned char mlp_smraw[];
  MlpInferSmem& S = *reinterpret_cast<MlpInferSmem*>(mlp_smraw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int q = tid; q < MLP_H * MLP_H; q += MLP_IT) {
    const int j = q / MLP_H, i = q - j * MLP_H;
    S.w2t[i][j] = to_tf32(params[MLP_OFF_W2 + q]);
  }
  for (int q = tid; q < MLP_H * MLP_IN; q += MLP_IT) S.w1[q] = params[MLP_OFF_W1 + q];
  for (int q = tid; q < MLP_H; q += MLP_IT) {
    S.b1[q] = params[MLP_OFF_B1 + q];
    S.b2[q] = params[MLP_OFF_B2 + q];
    S.w3[q] = params[MLP_OFF_W3 + q];
  }
  const float b3 = params[MLP_OFF_B3];
  const long total = (long)k * n;
  const int e1 = tid % MLP_TE, half = tid / MLP_TE;  // first layer: entry, half of the hidden units
  const int g = lane >> 2, tq = lane & 3;            // mma fragment coordinates
  const int e0 = warp * 16;                          // this warp's entries in the tile
  for (long base = (long)blockIdx.x * MLP_TE; base < total; base += (long)gridDim.x * MLP_TE) {
    __syncthreads();  // the previous tile's shared data is consumed
    {
      const long idx = base + e1;
      float u[3] = {0.f, 0.f, 0.f};
      if (idx < total) {
        const int j = (int)(idx / n);
        const long i = idx - (long)j * n;
        const int b = band[j];
        const double2 v = res[(long)b * n + i];
        mlp_features(kin[i], ekin[j], sqrt(v.x * v.x + v.y * v.y), norms[b] / sqrt((double)n), t, u);
      }
      if (half == 0) S.u0[e1] = u[0];
#pragma unroll 4
      for (int h = half * (MLP_H / 2); h < (half + 1) * (MLP_H / 2); ++h) {
        const float* w = S.w1 + h * MLP_IN;
        S.a[h][e1] = to_tf32(tanh_hw(fmaf(w[0], u[0], fmaf(w[1], u[1], fmaf(w[2], u[2], S.b1[h])))));
      }
    }
    __syncthreads();
    // A fragments of the warp's 16 entries for the eight k steps
    uint32_t af[8][4];
#pragma unroll
    for (int ks = 0; ks < 8; ++ks) {
      af[ks][0] = S.a[8 * ks + tq][e0 + g];
      af[ks][1] = S.a[8 * ks + tq][e0 + g + 8];
      af[ks][2] = S.a[8 * ks + tq + 4][e0 + g];
      af[ks][3] = S.a[8 * ks + tq + 4][e0 + g + 8];
    }
    float zlo = 0.f, zhi = 0.f;  // output-layer partial sums of entries e0 + g and e0 + g + 8
#pragma unroll 2
    for (int nt = 0; nt < 8; ++nt) {
      float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
      for (int ks = 0; ks < 8; ++ks) {
        const uint32_t b0 = S.w2t[8 * ks + tq][8 * nt + g], b1 = S.w2t[8 * ks + tq + 4][8 * nt + g];
        asm volatile(
            "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
            "{%0, %1, %2, %3};"
            : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
            : "r"(af[ks][0]), "r"(af[ks][1]), "r"(af[ks][2]), "r"(af[ks][3]), "r"(b0), "r"(b1));
      }
      const int j0 = 8 * nt + 2 * tq;
      zlo = fmaf(S.w3[j0], tanh_hw(c[0] + S.b2[j0]), zlo);
      zlo = fmaf(S.w3[j0 + 1], tanh_hw(c[1] + S.b2[j0 + 1]), zlo);
      zhi = fmaf(S.w3[j0], tanh_hw(c[2] + S.b2[j0]), zhi);
      zhi = fmaf(S.w3[j0 + 1], tanh_hw(c[3] + S.b2[j0 + 1]), zhi);
    }
    zlo += __shfl_xor_sync(0xffffffffu, zlo, 1);
    zlo += __shfl_xor_sync(0xffffffffu, zlo, 2);
    zhi += __shfl_xor_sync(0xffffffffu, zhi, 1);
    zhi += __shfl_xor_sync(0xffffffffu, zhi, 2);
    if (tq == 0) {
      S.m[e0 + g] = mlp_multiplier(S.u0[e0 + g], zlo + b3);
      S.m[e0 + g + 8] = mlp_multiplier(S.u0[e0 + g + 8], zhi + b3);
    }
    __syncthreads();
    // scale the residual entries (two threads per entry: real and imaginary parts)
    {
      const int e = tid >> 1, part = tid & 1;
      const long idx = base + e;
      if (idx < total) {
        const int j = (int)(idx / n);
        const long i = idx - (long)j * n;
        const double* src = reinterpret_cast<const double*>(res + (long)band[j] * n + i);
        reinterpret_cast<double*>(Q + idx)[part] = src[part] * S.m[e];
      }
    }
  }
}

// The reference preconditioner (eig.cu).
__global__ void k_precondition(double2* __restrict__ Q, const double2* __restrict__ res, const double* __restrict__ diag,
                               const double* __restrict__ lam, const int* __restrict__ band, int k, long n);

// ---- training -----------------------------------------------------------------------------------

// Per band: A_b = sum m_i c_i (complex), Q_b = sum m_i^2 w_i.
__global__ void __launch_bounds__(256) k_mlp_band_sums(const int* __restrict__ off, const float* __restrict__ feat,
                                                       const float2* __restrict__ cc, const float* __restrict__ w,
                                                       const float* __restrict__ params, double* __restrict__ sums) {
  __shared__ float p[MLP_NPARAM];
  __shared__ double red[3][256];
  for (int i = threadIdx.x; i < MLP_NPARAM; i += blockDim.x) p[i] = params[i];
  __syncthreads();
  const int b = blockIdx.x;
  double ar = 0.0, ai = 0.0, q = 0.0;
  for (int i = off[b] + threadIdx.x; i < off[b + 1]; i += blockDim.x) {
    const float u[3] = {feat[3 * i], feat[3 * i + 1], feat[3 * i + 2]};
    const double m = mlp_multiplier(u[0], mlp_forward(p, u, nullptr, nullptr));
    ar += m * cc[i].x;
    ai += m * cc[i].y;
    q += m * m * w[i];
  }
  red[0][threadIdx.x] = ar;
  red[1][threadIdx.x] = ai;
  red[2][threadIdx.x] = q;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s)
      for (int r = 0; r < 3; ++r) red[r][threadIdx.x] += red[r][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    sums[3 * b] = red[0][0];
    sums[3 * b + 1] = red[1][0];
    sums[3 * b + 2] = red[2][0];
  }
}

constexpr int BW_TILE = 128;  // plane waves per backward tile (= threads per CTA)

// Gradient of L = (1/B) sum_b [1 - |A_b|^2 / (Q_b D_b)] with respect to the parameters, one CTA
// per band.  Thread t owns the dW2 entries (row t / 2, columns 32 (t % 2) ... + 31) and the
// first-layer / bias / w3 entries with index t (< 64).
__global__ void __launch_bounds__(BW_TILE) k_mlp_backward(const int* __restrict__ off, const float* __restrict__ feat,
                                                          const float2* __restrict__ cc, const float* __restrict__ w,
                                                          const float* __restrict__ dnorm, const double* __restrict__ sums,
                                                          const float* __restrict__ params, int nbands,
                                                          float* __restrict__ grad) {
  extern __shared__ float bsm[];
  float* p = bsm;                       // MLP_NPARAM
  float* H1 = p + MLP_NPARAM + 3;       // [BW_TILE][65] (padded)
  float* DA2 = H1 + BW_TILE * 65;       // [BW_TILE][65]
  float* DA1 = DA2 + BW_TILE * 65;      // [BW_TILE][65]
  float* U = DA1 + BW_TILE * 65;        // [BW_TILE][3]
  float* H2 = U + BW_TILE * 3;          // [BW_TILE][65]
  float* DZ = H2 + BW_TILE * 65;        // [BW_TILE]
  const int tid = threadIdx.x;
  for (int i = tid; i < MLP_NPARAM; i += blockDim.x) p[i] = params[i];
  __syncthreads();
  const int b = blockIdx.x;
  const double Ar = sums[3 * b], Ai = sums[3 * b + 1], Qb = fmax(sums[3 * b + 2], 1e-300), Db = fmax((double)dnorm[b], 1e-300);
  const double A2 = Ar * Ar + Ai * Ai;
  const double scale = 1.0 / (double)nbands;
  // owned accumulators
  const int row = tid >> 1, cbase = (tid & 1) * 32;
  float gW2[32];
#pragma unroll
  for (int q = 0; q < 32; ++q) gW2[q] = 0.f;
  float gW1[3] = {0.f, 0.f, 0.f}, gb1 = 0.f, gb2 = 0.f, gw3 = 0.f, gb3 = 0.f;
  for (int t0 = off[b]; t0 < off[b + 1]; t0 += BW_TILE) {
    const int i = t0 + tid;
    const bool live = i < off[b + 1];
    float* h1 = H1 + tid * 65;
    float* h2 = H2 + tid * 65;
    float* da2 = DA2 + tid * 65;
    float u[3] = {0.f, 0.f, 0.f};
    float dz = 0.f;
    if (live) {
      u[0] = feat[3 * i];
      u[1] = feat[3 * i + 1];
      u[2] = feat[3 * i + 2];
      const float z = mlp_forward(p, u, h1, h2);
      const double m = mlp_multiplier(u[0], z);
      // dL/dm_i = -(2 / (D Q)) [Re(conj(A) c_i) - (|A|^2 / Q) m_i w_i], times 1/B; dm/dz = m
      // inside the clamp, 0 outside
      const double re = Ar * cc[i].x + Ai * cc[i].y;
      const double dm = -2.0 / (Db * Qb) * (re - A2 / Qb * m * w[i]) * scale;
      dz = (z > -8.f && z < 8.f) ? (float)(dm * m) : 0.f;
    } else {
      for (int j = 0; j < MLP_H; ++j) h1[j] = h2[j] = 0.f;
    }
    // da2 = dz w3 (1 - h2^2); da1 = (W2^T da2) (1 - h1^2)
    for (int j = 0; j < MLP_H; ++j) da2[j] = dz * p[MLP_OFF_W3 + j] * (1.f - h2[j] * h2[j]);
    for (int i2 = 0; i2 < MLP_H; ++i2) {
      float sacc = 0.f;
      for (int j = 0; j < MLP_H; ++j) sacc = fmaf(p[MLP_OFF_W2 + j * MLP_H + i2], da2[j], sacc);
      DA1[tid * 65 + i2] = sacc * (1.f - h1[i2] * h1[i2]);
    }
    U[tid * 3] = u[0];
    U[tid * 3 + 1] = u[1];
    U[tid * 3 + 2] = u[2];
    DZ[tid] = dz;
    __syncthreads();
    // dW2[row][c] += sum_t DA2[t][row] H1[t][c]
    for (int t = 0; t < BW_TILE; ++t) {
      const float a = DA2[t * 65 + row];
#pragma unroll
      for (int q = 0; q < 32; ++q) gW2[q] = fmaf(a, H1[t * 65 + cbase + q], gW2[q]);
    }
    if (tid < MLP_H) {
      for (int t = 0; t < BW_TILE; ++t) {
        const float a1 = DA1[t * 65 + tid];
        gW1[0] = fmaf(a1, U[t * 3], gW1[0]);
        gW1[1] = fmaf(a1, U[t * 3 + 1], gW1[1]);
        gW1[2] = fmaf(a1, U[t * 3 + 2], gW1[2]);
        gb1 += a1;
        gb2 += DA2[t * 65 + tid];
        gw3 = fmaf(DZ[t], H2[t * 65 + tid], gw3);
      }
    }
    if (tid == 0)
      for (int t = 0; t < BW_TILE; ++t) gb3 += DZ[t];
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < 32; ++q) atomicAdd(&grad[MLP_OFF_W2 + row * MLP_H + cbase + q], gW2[q]);
  if (tid < MLP_H) {
    atomicAdd(&grad[MLP_OFF_W1 + tid * 3], gW1[0]);
    atomicAdd(&grad[MLP_OFF_W1 + tid * 3 + 1], gW1[1]);
    atomicAdd(&grad[MLP_OFF_W1 + tid * 3 + 2], gW1[2]);
    atomicAdd(&grad[MLP_OFF_B1 + tid], gb1);
    atomicAdd(&grad[MLP_OFF_B2 + tid], gb2);
    atomicAdd(&grad[MLP_OFF_W3 + tid], gw3);
  }
  if (tid == 0) atomicAdd(&grad[MLP_OFF_B3], gb3);
}

__global__ void k_mlp_loss(const double* __restrict__ sums, const float* __restrict__ dnorm, int nbands, double* __restrict__ loss) {
  __shared__ double red[256];
  double s = 0.0;
  for (int b = threadIdx.x; b < nbands; b += blockDim.x) {
    const double Ar = sums[3 * b], Ai = sums[3 * b + 1], Q = fmax(sums[3 * b + 2], 1e-300), D = fmax((double)dnorm[b], 1e-300);
    s += 1.0 - (Ar * Ar + Ai * Ai) / (Q * D);
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *loss = red[0] / nbands;
}

__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m1, float* __restrict__ m2,
                       int np, float lr, float b1, float b2, float eps, int step) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  const float gi = g[i];
  const float a = b1 * m1[i] + (1.f - b1) * gi, v = b2 * m2[i] + (1.f - b2) * gi * gi;
  m1[i] = a;
  m2[i] = v;
  const float ah = a / (1.f - powf(b1, (float)step)), vh = v / (1.f - powf(b2, (float)step));
  p[i] -= lr * ah / (sqrtf(vh) + eps);
}

constexpr size_t kBackwardSmem = sizeof(float) * (MLP_NPARAM + 3 + 4 * BW_TILE * 65 + BW_TILE * 3 + BW_TILE);

struct MlpData {
  int nb = 0;
  long np = 0;
  int* off = nullptr;
  float* feat = nullptr;
  float2* cc = nullptr;
  float* w = nullptr;
  float* dn = nullptr;
  double* sums = nullptr;
  double* loss = nullptr;
  float* params = nullptr;
  float* grad = nullptr;
  float* m1 = nullptr;
  float* m2 = nullptr;
  void* mem = nullptr;
  ~MlpData() {
    if (mem) cudaFree(mem);
  }
};

static int mlp_upload(MlpData& d, size_t nbands, size_t npw, const int* off, const float* feat, const float* cc, const float* w,
                      const float* dnorm, const float* params, cudaStream_t s) {
  d.nb = (int)nbands;
  d.np = (long)npw;
  size_t o = 0;
  auto take = [&](size_t bytes) { const size_t r = o; o += (bytes + 255) / 256 * 256; return r; };
  const size_t oo = take(sizeof(int) * (nbands + 1)), of = take(sizeof(float) * 3 * npw), oc = take(sizeof(float2) * npw),
               ow = take(sizeof(float) * npw), od = take(sizeof(float) * nbands), os = take(sizeof(double) * 3 * nbands),
               ol = take(sizeof(double)), op = take(sizeof(float) * MLP_NPARAM), og = take(sizeof(float) * MLP_NPARAM),
               o1 = take(sizeof(float) * MLP_NPARAM), o2 = take(sizeof(float) * MLP_NPARAM);
  if (dev_malloc(&d.mem, o) != cudaSuccess) return fail(DFTCUDA_ERR_OUT_OF_MEMORY, "precond_mlp: training data");
  char* b = (char*)d.mem;
  d.off = (int*)(b + oo); d.feat = (float*)(b + of); d.cc = (float2*)(b + oc); d.w = (float*)(b + ow);
  d.dn = (float*)(b + od); d.sums = (double*)(b + os); d.loss = (double*)(b + ol); d.params = (float*)(b + op);
  d.grad = (float*)(b + og); d.m1 = (float*)(b + o1); d.m2 = (float*)(b + o2);
  auto up = [&](void* dst, const void* src, size_t bytes) {
    return cudaMemcpyAsync(dst, src, bytes, is_device_pointer(src) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s);
  };
  DFT_CUDA_TRY(up(d.off, off, sizeof(int) * (nbands + 1)));
  DFT_CUDA_TRY(up(d.feat, feat, sizeof(float) * 3 * npw));
  DFT_CUDA_TRY(up(d.cc, cc, sizeof(float2) * npw));
  DFT_CUDA_TRY(up(d.w, w, sizeof(float) * npw));
  DFT_CUDA_TRY(up(d.dn, dnorm, sizeof(float) * nbands));
  DFT_CUDA_TRY(up(d.params, params, sizeof(float) * MLP_NPARAM));
  DFT_CUDA_TRY(cudaMemsetAsync(d.m1, 0, sizeof(float) * MLP_NPARAM, s));
  DFT_CUDA_TRY(cudaMemsetAsync(d.m2, 0, sizeof(float) * MLP_NPARAM, s));
  return DFTCUDA_OK;
}

static int mlp_loss_grad_dev(MlpData& d, cudaStream_t s) {
  DFT_TRY(ensure_max_dynamic_smem((const void*)k_mlp_backward, (int)kBackwardSmem));
  k_mlp_band_sums<<<d.nb, 256, 0, s>>>(d.off, d.feat, d.cc, d.w, d.params, d.sums); count_launch();
  k_mlp_loss<<<1, 256, 0, s>>>(d.sums, d.dn, d.nb, d.loss); count_launch();
  DFT_CUDA_TRY(cudaMemsetAsync(d.grad, 0, sizeof(float) * MLP_NPARAM, s));
  k_mlp_backward<<<d.nb, BW_TILE, kBackwardSmem, s>>>(d.off, d.feat, d.cc, d.w, d.dn, d.sums, d.params, d.nb, d.grad); count_launch();
  DFT_CUDA_TRY(cudaGetLastError());
  return DFTCUDA_OK;
}

}  // namespace dftcuda

using namespace dftcuda;

extern "C" int dftcuda_kctx_set_preconditioner(dftcuda_kctx* c, int kind, const float* params, size_t nparams) {
  if (!c) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "set_preconditioner: null context");
  DeviceGuard dg(c->device);  // the context's device, whatever the caller has current
  DFT_TRY(dg.status);
  if (kind < DFTCUDA_PRECOND_REFERENCE || kind > DFTCUDA_PRECOND_MLP)
    return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "set_preconditioner: unknown kind");
  if (kind == DFTCUDA_PRECOND_MLP) {
    if (!params || nparams != (size_t)MLP_NPARAM)
      return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "set_preconditioner: the MLP needs DFTCUDA_PRECOND_MLP_PARAMS weights");
    if (!c->d_mlp && dev_malloc(&c->d_mlp, sizeof(float) * (kMlpParamPad + (size_t)kLutN0 * kLutN1)) != cudaSuccess)
      return fail(DFTCUDA_ERR_OUT_OF_MEMORY, "set_preconditioner: weights");
    c->mlp_table_t = -1.0;
    DFT_CUDA_TRY(cudaMemcpyAsync(c->d_mlp, params, sizeof(float) * MLP_NPARAM,
                                 is_device_pointer(params) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, c->stream));
    DFT_CUDA_TRY(cudaStreamSynchronize(c->stream));
  }
  c->precond_kind = kind;
  return DFTCUDA_OK;
}

extern "C" int dftcuda_precond_mlp_loss_grad(size_t nbands, size_t npw, const int* band_off, const float* feat,
                                             const float* cc, const float* w, const float* dnorm, const float* params,
                                             double* loss, float* grad) {
  if (nbands == 0 || npw == 0 || !band_off || !feat || !cc || !w || !dnorm || !params || !loss || !grad)
    return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "precond_mlp_loss_grad: empty or null argument");
  cudaStream_t s = nullptr;
  DFT_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamDefault));
  int st;
  {
    MlpData d;
    st = mlp_upload(d, nbands, npw, band_off, feat, cc, w, dnorm, params, s);
    if (st == DFTCUDA_OK) st = mlp_loss_grad_dev(d, s);
    if (st == DFTCUDA_OK) {
      cudaMemcpyAsync(loss, d.loss, sizeof(double), is_device_pointer(loss) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s);
      cudaMemcpyAsync(grad, d.grad, sizeof(float) * MLP_NPARAM,
                      is_device_pointer(grad) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s);
      const cudaError_t ce = cudaStreamSynchronize(s);
      if (ce != cudaSuccess) st = fail(DFTCUDA_ERR_CUDA, cudaGetErrorString(ce));
    }
  }
  cudaStreamDestroy(s);
  return st;
}

extern "C" int dftcuda_precond_mlp_train(size_t nbands, size_t npw, const int* band_off, const float* feat, const float* cc,
                                         const float* w, const float* dnorm, float* params, size_t steps, float lr,
                                         double* loss_history) {
  if (nbands == 0 || npw == 0 || !band_off || !feat || !cc || !w || !dnorm || !params)
    return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "precond_mlp_train: empty or null argument");
  cudaStream_t s = nullptr;
  DFT_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamDefault));
  int st;
  {
    MlpData d;
    st = mlp_upload(d, nbands, npw, band_off, feat, cc, w, dnorm, params, s);
    std::vector<double> hist(steps, 0.0);
    double* dhist = nullptr;
    if (st == DFTCUDA_OK && steps && dev_malloc(&dhist, sizeof(double) * steps) != cudaSuccess)
      st = fail(DFTCUDA_ERR_OUT_OF_MEMORY, "precond_mlp_train: history");
    for (size_t it = 0; it < steps && st == DFTCUDA_OK; ++it) {
      st = mlp_loss_grad_dev(d, s);
      if (st != DFTCUDA_OK) break;
      cudaMemcpyAsync(dhist + it, d.loss, sizeof(double), cudaMemcpyDeviceToDevice, s);
      k_adam<<<ceil_div(MLP_NPARAM, 256), 256, 0, s>>>(d.params, d.grad, d.m1, d.m2, MLP_NPARAM, lr, 0.9f, 0.999f, 1e-8f,
                                                      (int)it + 1);
      count_launch();
    }
    if (st == DFTCUDA_OK) {
      cudaMemcpyAsync(params, d.params, sizeof(float) * MLP_NPARAM,
                      is_device_pointer(params) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s);
      if (steps) cudaMemcpyAsync(hist.data(), dhist, sizeof(double) * steps, cudaMemcpyDeviceToHost, s);
      const cudaError_t ce = cudaStreamSynchronize(s);
      if (ce != cudaSuccess) st = fail(DFTCUDA_ERR_CUDA, cudaGetErrorString(ce));
      if (st == DFTCUDA_OK && loss_history)
        for (size_t i = 0; i < steps; ++i) loss_history[i] = hist[i];
    }
    if (dhist) cudaFree(dhist);
  }
  cudaStreamDestroy(s);
  return st;
}

namespace dftcuda {

int precondition_launch(dftcuda_kctx* c, double2* Q, const double2* res, const double* kin, const double* lam,
                        const double* norms, const double2* ritz, const int* band, int take, long n, double t,
                        double* ekin_ws, cudaStream_t s) {
  const unsigned grid = ceil_div((size_t)take * n, 256);
  if (c->precond_kind == DFTCUDA_PRECOND_REFERENCE) {
    k_precondition<<<grid, 256, 0, s>>>(Q, res, kin, lam, band, take, n);
    count_launch();
  } else {
    k_band_kinetic<<<take, 256, 0, s>>>(ritz, kin, band, n, ekin_ws);
    count_launch();
    if (c->precond_kind == DFTCUDA_PRECOND_TPA)
      k_precondition_tpa<<<grid, 256, 0, s>>>(Q, res, kin, ekin_ws, band, take, n);
    else if (!mlp_infer_tc()) {
      float* lut = c->d_mlp + kMlpParamPad;
      if (c->mlp_table_t != t) {
        k_mlp_table<<<ceil_div((size_t)kLutN0 * kLutN1, 128), 128, 0, s>>>(c->d_mlp, t, lut);
        count_launch();
        c->mlp_table_t = t;
      }
      k_precondition_lut<<<grid, 256, 0, s>>>(Q, res, kin, ekin_ws, norms, band, take, n, t, lut, c->d_mlp);
    } else {
      // tiles of MLP_TE entries, up to eight blocks per SM (about three resident)
      int dev = 0, nsm = 148;
      DFT_CUDA_TRY(cudaGetDevice(&dev));
      DFT_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
      DFT_TRY(ensure_max_dynamic_smem((const void*)k_precondition_mlp, (int)sizeof(MlpInferSmem)));
      const size_t tiles = ((size_t)take * n + MLP_TE - 1) / MLP_TE;
      const unsigned g = (unsigned)std::min<size_t>(tiles, (size_t)nsm * 8);
      k_precondition_mlp<<<g, MLP_IT, sizeof(MlpInferSmem), s>>>(Q, res, kin, ekin_ws, norms, band, take, n, t, c->d_mlp);
    }
    count_launch();
  }
  DFT_CUDA_TRY(cudaGetLastError());
  return DFTCUDA_OK;
}

}  // namespace dftcuda
