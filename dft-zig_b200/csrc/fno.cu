// Fourier neural operator that maps the superposition-of-atoms density of a cell to a first SCF
// density (the learned start of the SCF loop; the reference starts from the atomic superposition
// or a uniform density, scf/density init).  Inference and training kernels, FP32.
//
//   input   u: 2 channels on the cell's FFT grid (x fastest), the Si-like and Ge-like atomic
//           superposition densities divided by the mean valence density;
//   lift    v0 = P u + p                                               (W = 8 channels)
//   layers  v_{l+1} = act(W_l v_l + b_l + Re IDFT_M(R_l . DFT_M(v_l)))   l = 0..3
//           act = GELU (tanh form, Hendrycks & Gimpel 2016) for l < 3, identity for l = 3
//   proj    d = q . v4 + q0: the predicted (rho_scf - rho_atomic) / mean density.
// DFT_M keeps the 16 lowest frequencies per axis (f = -8..7), computed as three separable partial
// DFTs (one small contraction per axis, any grid size >= 16) and divided by the grid size N, so the
// mode weights act on resolution-independent Fourier coefficients; IDFT_M is the matching partial
// inverse sum (no factor), of which the real part is kept (the mode weights R_l[k][o][i] are free
// complex numbers).  Gradients: the adjoint of DFT_M / N is Re IDFT_M / N and the adjoint of
// Re IDFT_M is DFT_M, so the backward pass reuses the same axis contractions.  Loss: mean over samples of the mean squared
// error over grid points.
#include <cmath>
#include <vector>

#include "kctx.cuh"

namespace dftcuda {

constexpr int FNO_W = 8;                // channels
constexpr int FNO_M = 16;               // modes per axis
constexpr int FNO_K = FNO_M * FNO_M * FNO_M;
constexpr int FNO_L = 4;                // Fourier layers
constexpr int FNO_IN = 2;
// parameter layout
constexpr long FNO_OFF_P = 0;                                   // P[W][2]
constexpr long FNO_OFF_PB = FNO_OFF_P + FNO_W * FNO_IN;         // p[W]
constexpr long FNO_OFF_LAYER = FNO_OFF_PB + FNO_W;              // per layer: R[K][W][W] complex, Wl[W][W], bl[W]
constexpr long FNO_LAYER_SIZE = 2L * FNO_K * FNO_W * FNO_W + FNO_W * FNO_W + FNO_W;
constexpr long FNO_OFF_Q = FNO_OFF_LAYER + FNO_L * FNO_LAYER_SIZE;  // q[W]
constexpr long FNO_OFF_Q0 = FNO_OFF_Q + FNO_W;
constexpr long FNO_NPARAM = FNO_OFF_Q0 + 1;
static_assert(FNO_NPARAM == DFTCUDA_FNO_PARAMS, "parameter count");

__host__ __device__ constexpr long fno_R(int l) { return FNO_OFF_LAYER + l * FNO_LAYER_SIZE; }
__host__ __device__ constexpr long fno_Wl(int l) { return fno_R(l) + 2L * FNO_K * FNO_W * FNO_W; }
__host__ __device__ constexpr long fno_bl(int l) { return fno_Wl(l) + FNO_W * FNO_W; }

__device__ __forceinline__ float gelu_t(float x, float* dgelu) {
  const float s = 0.7978845608028654f;  // sqrt(2 / pi)
  const float a = s * (x + 0.044715f * x * x * x);
  const float t = tanhf(a);
  if (dgelu) *dgelu = 0.5f * (1.f + t) + 0.5f * x * (1.f - t * t) * s * (1.f + 3.f * 0.044715f * x * x);
  return 0.5f * x * (1.f + t);
}

// Twiddles T[j][x] = exp(-2 pi i f_j x / n), f_j = j - 8, for one axis.
__global__ void k_fno_twiddles(float2* __restrict__ T, int n) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= FNO_M * n) return;
  const int j = idx / n, x = idx - j * n;
  const long f = j - FNO_M / 2;
  // reduce f x mod n exactly, then the angle -2 pi (f x mod n) / n
  long r = (f * x) % n;
  if (r < 0) r += n;
  double sn, cs;
  sincospi(-2.0 * (double)r / (double)n, &sn, &cs);
  T[idx] = make_float2((float)cs, (float)sn);
}

// out[o][k][i] = sum_l in[o][l][i] * T'(k, l), T'(k, l) = T[k][l] (trans = 0) or T[l][k] (trans = 1),
// conjugated when conj_t.  in real (real_in) or complex; out complex, or its real part (real_out).
__global__ void k_axis_contract(const void* __restrict__ in_, void* __restrict__ out_, long outer, int L, int inner, int K,
                                const float2* __restrict__ T, int ldt, bool trans, bool conj_t, bool real_in, bool real_out,
                                bool accumulate, float scale) {
  const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const long total = outer * K * inner;
  if (idx >= total) return;
  const int i = (int)(idx % inner);
  const long ok = idx / inner;
  const int k = (int)(ok % K);
  const long o = ok / K;
  float sr = 0.f, si = 0.f;
  for (int l = 0; l < L; ++l) {
    float2 t = trans ? T[(long)l * ldt + k] : T[(long)k * ldt + l];
    if (conj_t) t.y = -t.y;
    const long ii = (o * L + l) * inner + i;
    if (real_in) {
      const float v = reinterpret_cast<const float*>(in_)[ii];
      sr = fmaf(v, t.x, sr);
      si = fmaf(v, t.y, si);
    } else {
      const float2 v = reinterpret_cast<const float2*>(in_)[ii];
      sr = fmaf(v.x, t.x, fmaf(-v.y, t.y, sr));
      si = fmaf(v.x, t.y, fmaf(v.y, t.x, si));
    }
  }
  sr *= scale;
  si *= scale;
  if (real_out) {
    float* out = reinterpret_cast<float*>(out_);
    out[idx] = accumulate ? out[idx] + sr : sr;
  } else {
    float2* out = reinterpret_cast<float2*>(out_);
    if (accumulate) {
      const float2 v = out[idx];
      out[idx] = make_float2(v.x + sr, v.y + si);
    } else {
      out[idx] = make_float2(sr, si);
    }
  }
}

// What[o][k] = sum_i R[k][o][i] Vhat[i][k]
__global__ void k_fno_mix(const float2* __restrict__ Vh, const float2* __restrict__ R, float2* __restrict__ Wh) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= FNO_W * FNO_K) return;
  const int o = idx / FNO_K, k = idx - o * FNO_K;
  float sr = 0.f, si = 0.f;
  for (int i = 0; i < FNO_W; ++i) {
    const float2 r = R[((long)k * FNO_W + o) * FNO_W + i], v = Vh[(long)i * FNO_K + k];
    sr += r.x * v.x - r.y * v.y;
    si += r.x * v.y + r.y * v.x;
  }
  Wh[idx] = make_float2(sr, si);
}

// dR[k][o][i] += G[o][k] conj(Vhat[i][k]);  dVhat[i][k] = sum_o conj(R[k][o][i]) G[o][k]
// Vh and dVh may be the same buffer (the backward pass writes dVh over Vh): each thread reads its own
// Vh entry before it writes the same dVh entry, so neither pointer is restrict-qualified.
__global__ void k_fno_mix_bwd(const float2* __restrict__ G, const float2* Vh, const float2* __restrict__ R,
                              float2* __restrict__ dR, float2* dVh) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= FNO_W * FNO_K) return;
  const int i = idx / FNO_K, k = idx - i * FNO_K;
  const float2 v = Vh[(long)i * FNO_K + k];
  float sr = 0.f, si = 0.f;
  for (int o = 0; o < FNO_W; ++o) {
    const float2 g = G[(long)o * FNO_K + k];
    const long ri = ((long)k * FNO_W + o) * FNO_W + i;
    const float2 r = R[ri];
    float2 d = dR[ri];
    d.x += g.x * v.x + g.y * v.y;  // g conj(v)
    d.y += g.y * v.x - g.x * v.y;
    dR[ri] = d;
    sr += r.x * g.x + r.y * g.y;  // conj(r) g
    si += r.x * g.y - r.y * g.x;
  }
  dVh[idx] = make_float2(sr, si);
}

// y[o][r] (+)= sum_i W[o][i] x[i][r] + b[o]
__global__ void k_fno_pointwise(const float* __restrict__ x, int cin, const float* __restrict__ W, const float* __restrict__ b,
                                float* __restrict__ y, int cout, long N, bool accumulate) {
  const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (idx >= (long)cout * N) return;
  const int o = (int)(idx / N);
  const long r = idx - (long)o * N;
  float s = b ? b[o] : 0.f;
  for (int i = 0; i < cin; ++i) s = fmaf(W[o * cin + i], x[(long)i * N + r], s);
  y[idx] = accumulate ? y[idx] + s : s;
}

// dx[i][r] (+)= sum_o W[o][i] g[o][r]
__global__ void k_fno_pointwise_dx(const float* __restrict__ g, int cout, const float* __restrict__ W, float* __restrict__ dx,
                                   int cin, long N, bool accumulate) {
  const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (idx >= (long)cin * N) return;
  const int i = (int)(idx / N);
  const long r = idx - (long)i * N;
  float s = 0.f;
  for (int o = 0; o < cout; ++o) s = fmaf(W[o * cin + i], g[(long)o * N + r], s);
  dx[idx] = accumulate ? dx[idx] + s : s;
}

// dW[o][i] += sum_r g[o][r] x[i][r] (blocks o * cin + i); db[o] += sum_r g[o][r] (blocks cout*cin + o)
__global__ void k_fno_pointwise_dw(const float* __restrict__ g, int cout, const float* __restrict__ x, int cin, long N,
                                   float* __restrict__ dW, float* __restrict__ db) {
  __shared__ float red[256];
  const int blk = blockIdx.x;
  const bool bias = blk >= cout * cin;
  const int o = bias ? blk - cout * cin : blk / cin, i = bias ? 0 : blk % cin;
  float s = 0.f;
  for (long r = threadIdx.x; r < N; r += blockDim.x) s += g[(long)o * N + r] * (bias ? 1.f : x[(long)i * N + r]);
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    if (bias) db[o] += red[0];
    else dW[o * cin + i] += red[0];
  }
}

__global__ void k_fno_gelu(const float* __restrict__ pre, float* __restrict__ out, long n) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < n) out[i] = gelu_t(pre[i], nullptr);
}

__global__ void k_fno_gelu_bwd(const float* __restrict__ pre, float* __restrict__ g, long n) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  float d;
  gelu_t(pre[i], &d);
  g[i] *= d;
}

// g[r] = 2 (d[r] - t[r]) * scale; loss += scale * sum (d - t)^2
__global__ void k_fno_mse(const float* __restrict__ d, const float* __restrict__ t, long N, float scale, float* __restrict__ g,
                          double* __restrict__ loss) {
  __shared__ double red[256];
  double s = 0.0;
  for (long r = blockIdx.x * (long)blockDim.x + threadIdx.x; r < N; r += (long)gridDim.x * blockDim.x) {
    const float e = d[r] - t[r];
    g[r] = 2.f * e * scale;
    s += (double)e * e;
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(loss, red[0] * (double)scale);
}

__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m1, float* __restrict__ m2,
                       int np, float lr, float b1, float b2, float eps, int step);

// Workspace for one sample of up to nmax grid points.
struct FnoWork {
  long nmax = 0;
  int nx = 0, ny = 0, nz = 0;
  float* v[FNO_L + 1] = {};   // activations W x N
  float* pre[FNO_L] = {};     // pre-activations W x N
  float2* vh[FNO_L] = {};     // DFT_M(v_l), W x K
  float2* ca = nullptr;       // W x nz x ny x 16
  float2* cb = nullptr;       // W x nz x 16 x 16
  float2* wh = nullptr;       // W x K
  float* g = nullptr;         // W x N gradient scratch
  float* g2 = nullptr;        // W x N
  float* out = nullptr;       // N
  float2* tw = nullptr;       // 16 x (nx + ny + nz)
  void* mem = nullptr;
  ~FnoWork() {
    if (mem) cudaFree(mem);
  }
};

static int fno_alloc(FnoWork& w, long nmax, int dmax) {
  w.nmax = nmax;
  size_t o = 0;
  auto take = [&](size_t bytes) { const size_t r = o; o += (bytes + 255) / 256 * 256; return r; };
  size_t ov[FNO_L + 1], op[FNO_L], oh[FNO_L];
  for (int l = 0; l <= FNO_L; ++l) ov[l] = take(sizeof(float) * FNO_W * nmax);
  for (int l = 0; l < FNO_L; ++l) op[l] = take(sizeof(float) * FNO_W * nmax);
  for (int l = 0; l < FNO_L; ++l) oh[l] = take(sizeof(float2) * FNO_W * FNO_K);
  const size_t oca = take(sizeof(float2) * FNO_W * (size_t)dmax * dmax * FNO_M), ocb = take(sizeof(float2) * FNO_W * (size_t)dmax * FNO_M * FNO_M),
               owh = take(sizeof(float2) * FNO_W * FNO_K), og = take(sizeof(float) * FNO_W * nmax), og2 = take(sizeof(float) * FNO_W * nmax),
               oo = take(sizeof(float) * nmax), ot = take(sizeof(float2) * FNO_M * 3 * dmax);
  if (dev_malloc(&w.mem, o) != cudaSuccess) return fail(DFTCUDA_ERR_OUT_OF_MEMORY, "fno workspace");
  char* b = (char*)w.mem;
  for (int l = 0; l <= FNO_L; ++l) w.v[l] = (float*)(b + ov[l]);
  for (int l = 0; l < FNO_L; ++l) {
    w.pre[l] = (float*)(b + op[l]);
    w.vh[l] = (float2*)(b + oh[l]);
  }
  w.ca = (float2*)(b + oca); w.cb = (float2*)(b + ocb); w.wh = (float2*)(b + owh);
  w.g = (float*)(b + og); w.g2 = (float*)(b + og2); w.out = (float*)(b + oo); w.tw = (float2*)(b + ot);
  return DFTCUDA_OK;
}

static inline unsigned g256(long n) { return (unsigned)((n + 255) / 256); }

static int fno_set_grid(FnoWork& w, int nx, int ny, int nz, cudaStream_t s) {
  if (nx < FNO_M || ny < FNO_M || nz < FNO_M) return fail(DFTCUDA_ERR_INVALID_GRID, "fno: grid axes must be >= 16");
  if (w.nx == nx && w.ny == ny && w.nz == nz) return DFTCUDA_OK;
  w.nx = nx; w.ny = ny; w.nz = nz;
  k_fno_twiddles<<<g256(FNO_M * nx), 256, 0, s>>>(w.tw, nx); count_launch();
  k_fno_twiddles<<<g256(FNO_M * ny), 256, 0, s>>>(w.tw + FNO_M * nx, ny); count_launch();
  k_fno_twiddles<<<g256(FNO_M * nz), 256, 0, s>>>(w.tw + FNO_M * (nx + ny), nz); count_launch();
  return DFTCUDA_OK;
}

// Vh[c][k] = scale * DFT_M(v)[c][k] for C channels (real v, layout [c][z][y][x]).
static void fno_dft(FnoWork& w, const float* v, int C, float2* Vh, float scale, cudaStream_t s) {
  const int nx = w.nx, ny = w.ny, nz = w.nz;
  const float2 *tx = w.tw, *ty = w.tw + FNO_M * nx, *tz = w.tw + FNO_M * (nx + ny);
  long outer = (long)C * nz * ny;
  k_axis_contract<<<g256(outer * FNO_M), 256, 0, s>>>(v, w.ca, outer, nx, 1, FNO_M, tx, nx, false, false, true, false, false, 1.f);
  outer = (long)C * nz;
  k_axis_contract<<<g256(outer * FNO_M * FNO_M), 256, 0, s>>>(w.ca, w.cb, outer, ny, FNO_M, FNO_M, ty, ny, false, false, false, false, false,
                                                               1.f);
  outer = C;
  k_axis_contract<<<g256(outer * FNO_M * FNO_M * FNO_M), 256, 0, s>>>(w.cb, Vh, outer, nz, FNO_M * FNO_M, FNO_M, tz, nz, false, false, false,
                                                                      false, false, scale);
  count_launch(3);
}

// out[c][r] (+)= scale * Re IDFT_M(Wh)[c][r]
static void fno_idft(FnoWork& w, const float2* Wh, int C, float* out, bool accumulate, float scale, cudaStream_t s) {
  const int nx = w.nx, ny = w.ny, nz = w.nz;
  const float2 *tx = w.tw, *ty = w.tw + FNO_M * nx, *tz = w.tw + FNO_M * (nx + ny);
  long outer = C;
  k_axis_contract<<<g256(outer * nz * FNO_M * FNO_M), 256, 0, s>>>(Wh, w.cb, outer, FNO_M, FNO_M * FNO_M, nz, tz, nz, true, true, false, false,
                                                                   false, 1.f);
  outer = (long)C * nz;
  k_axis_contract<<<g256(outer * ny * FNO_M), 256, 0, s>>>(w.cb, w.ca, outer, FNO_M, FNO_M, ny, ty, ny, true, true, false, false, false, 1.f);
  outer = (long)C * nz * ny;
  k_axis_contract<<<g256(outer * nx), 256, 0, s>>>(w.ca, out, outer, FNO_M, 1, nx, tx, nx, true, true, false, true, accumulate, scale);
  count_launch(3);
}

// Forward for one sample: u [2][N] -> w.out [N]; keeps the activations for the backward pass.
static int fno_forward(FnoWork& w, const float* P, const float* u, cudaStream_t s) {
  const long N = (long)w.nx * w.ny * w.nz;
  k_fno_pointwise<<<g256(FNO_W * N), 256, 0, s>>>(u, FNO_IN, P + FNO_OFF_P, P + FNO_OFF_PB, w.v[0], FNO_W, N, false); count_launch();
  for (int l = 0; l < FNO_L; ++l) {
    fno_dft(w, w.v[l], FNO_W, w.vh[l], 1.f / (float)N, s);
    k_fno_mix<<<g256(FNO_W * FNO_K), 256, 0, s>>>(w.vh[l], reinterpret_cast<const float2*>(P + fno_R(l)), w.wh); count_launch();
    k_fno_pointwise<<<g256(FNO_W * N), 256, 0, s>>>(w.v[l], FNO_W, P + fno_Wl(l), P + fno_bl(l), w.pre[l], FNO_W, N, false); count_launch();
    fno_idft(w, w.wh, FNO_W, w.pre[l], true, 1.f, s);
    if (l < FNO_L - 1) {
      k_fno_gelu<<<g256(FNO_W * N), 256, 0, s>>>(w.pre[l], w.v[l + 1], FNO_W * N); count_launch();
    } else {
      DFT_CUDA_TRY(cudaMemcpyAsync(w.v[l + 1], w.pre[l], sizeof(float) * FNO_W * N, cudaMemcpyDeviceToDevice, s));
    }
  }
  k_fno_pointwise<<<g256(N), 256, 0, s>>>(w.v[FNO_L], FNO_W, P + FNO_OFF_Q, P + FNO_OFF_Q0, w.out, 1, N, false); count_launch();
  return DFTCUDA_OK;
}

// Backward for one sample given dL/dout in gout [N]; adds the parameter gradient into dP.
static int fno_backward(FnoWork& w, const float* P, const float* u, const float* gout, float* dP, cudaStream_t s) {
  const long N = (long)w.nx * w.ny * w.nz;
  // projection
  k_fno_pointwise_dw<<<FNO_W + 1, 256, 0, s>>>(gout, 1, w.v[FNO_L], FNO_W, N, dP + FNO_OFF_Q, dP + FNO_OFF_Q0); count_launch();
  k_fno_pointwise_dx<<<g256(FNO_W * N), 256, 0, s>>>(gout, 1, P + FNO_OFF_Q, w.g, FNO_W, N, false); count_launch();
  // w.g = dL/dv_{l+1}
  for (int l = FNO_L - 1; l >= 0; --l) {
    if (l < FNO_L - 1) {
      k_fno_gelu_bwd<<<g256(FNO_W * N), 256, 0, s>>>(w.pre[l], w.g, FNO_W * N); count_launch();
    }
    // w.g = dL/dpre_l.  Pointwise branch.
    k_fno_pointwise_dw<<<FNO_W * FNO_W + FNO_W, 256, 0, s>>>(w.g, FNO_W, w.v[l], FNO_W, N, dP + fno_Wl(l), dP + fno_bl(l)); count_launch();
    k_fno_pointwise_dx<<<g256(FNO_W * N), 256, 0, s>>>(w.g, FNO_W, P + fno_Wl(l), w.g2, FNO_W, N, false); count_launch();
    // Spectral branch: G = DFT_M(g); dR += G conj(Vh); dVh = R^H G; dv += Re IDFT_M(dVh)
    fno_dft(w, w.g, FNO_W, w.wh, 1.f, s);
    k_fno_mix_bwd<<<g256(FNO_W * FNO_K), 256, 0, s>>>(w.wh, w.vh[l], reinterpret_cast<const float2*>(P + fno_R(l)),
                                                       reinterpret_cast<float2*>(dP + fno_R(l)), w.vh[l]);
    count_launch();
    fno_idft(w, w.vh[l], FNO_W, w.g2, true, 1.f / (float)N, s);
    std::swap(w.g, w.g2);
  }
  // lift: w.g = dL/dv0
  k_fno_pointwise_dw<<<FNO_W * FNO_IN + FNO_W, 256, 0, s>>>(w.g, FNO_W, u, FNO_IN, N, dP + FNO_OFF_P, dP + FNO_OFF_PB); count_launch();
  DFT_CUDA_TRY(cudaGetLastError());
  return DFTCUDA_OK;
}

struct FnoSet {
  size_t ns = 0;
  std::vector<int> dims;
  std::vector<size_t> offs;
  float* u = nullptr;
  float* t = nullptr;
  float* P = nullptr;
  float* dP = nullptr;
  float* m1 = nullptr;
  float* m2 = nullptr;
  double* loss = nullptr;
  void* mem = nullptr;
  long nmax = 0;
  int dmax = 0;
  ~FnoSet() {
    if (mem) cudaFree(mem);
  }
};

static int fno_upload(FnoSet& d, size_t ns, const int* dims, const size_t* offs, const float* u, const float* t,
                      const float* params, cudaStream_t s) {
  d.ns = ns;
  d.dims.assign(dims, dims + 3 * ns);
  d.offs.assign(offs, offs + ns + 1);
  for (size_t i = 0; i < ns; ++i) {
    const long N = (long)dims[3 * i] * dims[3 * i + 1] * dims[3 * i + 2];
    if ((long)(offs[i + 1] - offs[i]) != N) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "fno: sample size != nx ny nz");
    d.nmax = std::max(d.nmax, N);
    for (int a = 0; a < 3; ++a) d.dmax = std::max(d.dmax, dims[3 * i + a]);
  }
  const size_t tot = offs[ns];
  size_t o = 0;
  auto take = [&](size_t bytes) { const size_t r = o; o += (bytes + 255) / 256 * 256; return r; };
  const size_t ou = take(sizeof(float) * FNO_IN * tot), ot = t ? take(sizeof(float) * tot) : 0, oP = take(sizeof(float) * FNO_NPARAM),
               odP = take(sizeof(float) * FNO_NPARAM), o1 = take(sizeof(float) * FNO_NPARAM), o2 = take(sizeof(float) * FNO_NPARAM),
               ol = take(sizeof(double));
  if (dev_malloc(&d.mem, o) != cudaSuccess) return fail(DFTCUDA_ERR_OUT_OF_MEMORY, "fno data");
  char* b = (char*)d.mem;
  d.u = (float*)(b + ou); d.t = t ? (float*)(b + ot) : nullptr; d.P = (float*)(b + oP); d.dP = (float*)(b + odP);
  d.m1 = (float*)(b + o1); d.m2 = (float*)(b + o2); d.loss = (double*)(b + ol);
  auto up = [&](void* dst, const void* src, size_t bytes) {
    return cudaMemcpyAsync(dst, src, bytes, is_device_pointer(src) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s);
  };
  DFT_CUDA_TRY(up(d.u, u, sizeof(float) * FNO_IN * tot));
  if (t) DFT_CUDA_TRY(up(d.t, t, sizeof(float) * tot));
  DFT_CUDA_TRY(up(d.P, params, sizeof(float) * FNO_NPARAM));
  DFT_CUDA_TRY(cudaMemsetAsync(d.m1, 0, sizeof(float) * FNO_NPARAM, s));
  DFT_CUDA_TRY(cudaMemsetAsync(d.m2, 0, sizeof(float) * FNO_NPARAM, s));
  return DFTCUDA_OK;
}

// loss = mean_s mean_r (out - t)^2 and its gradient (dP) over the whole set
static int fno_loss_grad(FnoSet& d, FnoWork& w, cudaStream_t s) {
  DFT_CUDA_TRY(cudaMemsetAsync(d.dP, 0, sizeof(float) * FNO_NPARAM, s));
  DFT_CUDA_TRY(cudaMemsetAsync(d.loss, 0, sizeof(double), s));
  for (size_t i = 0; i < d.ns; ++i) {
    DFT_TRY(fno_set_grid(w, d.dims[3 * i], d.dims[3 * i + 1], d.dims[3 * i + 2], s));
    const long N = (long)(d.offs[i + 1] - d.offs[i]);
    const float* u = d.u + FNO_IN * d.offs[i];
    DFT_TRY(fno_forward(w, d.P, u, s));
    const float scale = 1.f / ((float)N * (float)d.ns);
    float* gout = w.g2;  // N entries of scratch
    k_fno_mse<<<std::min<unsigned>(g256(N), 256), 256, 0, s>>>(w.out, d.t + d.offs[i], N, scale, gout, d.loss); count_launch();
    // gout lives in w.g2, which the backward pass overwrites only after its first use
    DFT_CUDA_TRY(cudaMemcpyAsync(w.out, gout, sizeof(float) * N, cudaMemcpyDeviceToDevice, s));
    DFT_TRY(fno_backward(w, d.P, u, w.out, d.dP, s));
  }
  return DFTCUDA_OK;
}

}  // namespace dftcuda

using namespace dftcuda;

extern "C" int dftcuda_fno_forward(int nx, int ny, int nz, const float* u, const float* params, float* out) {
  if (!u || !params || !out) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "fno_forward: null argument");
  cudaStream_t s = nullptr;
  DFT_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamDefault));
  int st;
  {
    const long N = (long)nx * ny * nz;
    const int dims[3] = {nx, ny, nz};
    const size_t offs[2] = {0, (size_t)N};
    FnoSet d;
    FnoWork w;
    st = fno_upload(d, 1, dims, offs, u, nullptr, params, s);
    if (st == DFTCUDA_OK) st = fno_alloc(w, N, std::max(nx, std::max(ny, nz)));
    if (st == DFTCUDA_OK) st = fno_set_grid(w, nx, ny, nz, s);
    if (st == DFTCUDA_OK) st = fno_forward(w, d.P, d.u, s);
    if (st == DFTCUDA_OK) {
      cudaMemcpyAsync(out, w.out, sizeof(float) * N, is_device_pointer(out) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s);
      const cudaError_t ce = cudaStreamSynchronize(s);
      if (ce != cudaSuccess) st = fail(DFTCUDA_ERR_CUDA, cudaGetErrorString(ce));
    }
  }
  cudaStreamDestroy(s);
  return st;
}

extern "C" int dftcuda_fno_loss_grad(size_t nsamples, const int* dims, const size_t* offs, const float* u, const float* target,
                                     const float* params, double* loss, float* grad) {
  if (!nsamples || !dims || !offs || !u || !target || !params || !loss || !grad)
    return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "fno_loss_grad: null argument");
  cudaStream_t s = nullptr;
  DFT_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamDefault));
  int st;
  {
    FnoSet d;
    FnoWork w;
    st = fno_upload(d, nsamples, dims, offs, u, target, params, s);
    if (st == DFTCUDA_OK) st = fno_alloc(w, d.nmax, d.dmax);
    if (st == DFTCUDA_OK) st = fno_loss_grad(d, w, s);
    if (st == DFTCUDA_OK) {
      cudaMemcpyAsync(loss, d.loss, sizeof(double), is_device_pointer(loss) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s);
      cudaMemcpyAsync(grad, d.dP, sizeof(float) * FNO_NPARAM, is_device_pointer(grad) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s);
      const cudaError_t ce = cudaStreamSynchronize(s);
      if (ce != cudaSuccess) st = fail(DFTCUDA_ERR_CUDA, cudaGetErrorString(ce));
    }
  }
  cudaStreamDestroy(s);
  return st;
}

extern "C" int dftcuda_fno_train(size_t nsamples, const int* dims, const size_t* offs, const float* u, const float* target,
                                 float* params, size_t steps, float lr, double* loss_history) {
  if (!nsamples || !dims || !offs || !u || !target || !params)
    return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "fno_train: null argument");
  cudaStream_t s = nullptr;
  DFT_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamDefault));
  int st;
  {
    FnoSet d;
    FnoWork w;
    std::vector<double> hist(steps, 0.0);
    double* dh = nullptr;
    st = fno_upload(d, nsamples, dims, offs, u, target, params, s);
    if (st == DFTCUDA_OK) st = fno_alloc(w, d.nmax, d.dmax);
    if (st == DFTCUDA_OK && steps && dev_malloc(&dh, sizeof(double) * steps) != cudaSuccess)
      st = fail(DFTCUDA_ERR_OUT_OF_MEMORY, "fno_train: history");
    for (size_t it = 0; it < steps && st == DFTCUDA_OK; ++it) {
      st = fno_loss_grad(d, w, s);
      if (st != DFTCUDA_OK) break;
      cudaMemcpyAsync(dh + it, d.loss, sizeof(double), cudaMemcpyDeviceToDevice, s);
      k_adam<<<g256(FNO_NPARAM), 256, 0, s>>>(d.P, d.dP, d.m1, d.m2, (int)FNO_NPARAM, lr, 0.9f, 0.999f, 1e-8f, (int)it + 1);
      count_launch();
    }
    if (st == DFTCUDA_OK) {
      cudaMemcpyAsync(params, d.P, sizeof(float) * FNO_NPARAM, is_device_pointer(params) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s);
      if (steps) cudaMemcpyAsync(hist.data(), dh, sizeof(double) * steps, cudaMemcpyDeviceToHost, s);
      const cudaError_t ce = cudaStreamSynchronize(s);
      if (ce != cudaSuccess) st = fail(DFTCUDA_ERR_CUDA, cudaGetErrorString(ce));
      if (st == DFTCUDA_OK && loss_history)
        for (size_t i = 0; i < steps; ++i) loss_history[i] = hist[i];
    }
    if (dh) cudaFree(dh);
  }
  cudaStreamDestroy(s);
  return st;
}
