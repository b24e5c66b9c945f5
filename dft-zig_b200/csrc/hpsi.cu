// H|psi> for one k-point: kinetic + local potential through sphere-pruned 3D FFTs + Kleinman-Bylander
// nonlocal projectors, and the band density.  Replaces src/features/scf/apply.zig:577-1618 and
// src/features/scf/kpoint/density.zig:444-474.
//
// Local potential, three passes per column block (the reference's scatter_fft -> inverse FFT ->
// x V(r) -> forward FFT -> gather_fft, apply.zig:811-880):
//  1. k_plane_inv   one CTA per (active x-frequency plane, column): scatter that plane's plane
//                   waves into a shared-memory (z, y) plane at digit-reversed positions, inverse
//                   DIT FFT along z then y, store the plane.  Planes whose x-frequency holds no
//                   plane wave are never touched (about half the box for a 4x-ecut grid).
//  2. k_xline       one CTA per run of (z, y) lines: gather the active planes into x pencils,
//                   inverse DIT along x, multiply by V(r), forward DIF along x, keep only the active
//                   x-frequencies.
//  3. k_plane_fwd   forward DIF along y then z, gather the plane waves scaled by 1/N and add the
//                   kinetic term |k+G|^2 x_G.
// The net scaling equals the reference's (xN on scatter, 1/N in the inverse, 1/N on gather).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>

#include "kctx.cuh"

namespace dftcuda {

template <typename T>
__global__ void __launch_bounds__(512) k_plane_inv(const double2* __restrict__ x, long npw, cplx<T>* __restrict__ W,
                                                   int n_act, const int* __restrict__ plane_off,
                                                   const int* __restrict__ pw_idx, const int* __restrict__ pw_spos,
                                                   Fft1d py, Fft1d pz, int ny, int nz) {
  using C = cplx<T>;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* S = reinterpret_cast<C*>(smraw);
  const int slot = blockIdx.x;
  const long b = blockIdx.y;
  const int P = ny * nz;
  for (int i = threadIdx.x; i < P; i += blockDim.x) S[i] = mk<C>(0.0, 0.0);
  __syncthreads();
  const double2* xb = x + b * npw;
  const int j1 = plane_off[slot + 1];
  for (int j = plane_off[slot] + threadIdx.x; j < j1; j += blockDim.x) {
    const double2 c = __ldg(xb + pw_idx[j]);
    S[pw_spos[j]] = mk<C>(c.x, c.y);
  }
  __syncthreads();
  fft_lines<T, true>(S, pz, ny, 1, ny, (T)1, true);   // along z, columns are lines
  fft_lines<T, true>(S, py, 1, ny, nz, (T)1, false);  // along y, rows are lines
  C* Wp = W + (b * n_act + slot) * (long)P;
  for (int i = threadIdx.x; i < P; i += blockDim.x) Wp[i] = S[i];
}

template <typename T>
__global__ void __launch_bounds__(256) k_xline(cplx<T>* __restrict__ W, int n_act, const int* __restrict__ slot_xpos,
                                               const T* __restrict__ Vt, Fft1d px, int P, int ncols, int J,
                                               int cols_per_cta) {
  using C = cplx<T>;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int nx = px.n;
  C* tile = reinterpret_cast<C*>(smraw);                 // [nx][J]
  T* vt = reinterpret_cast<T*>(smraw + sizeof(C) * nx * J);  // [nx][J]
  const int j0 = blockIdx.x * J;
  const int nj = min(J, P - j0);
  const int c0 = blockIdx.y * cols_per_cta;
  const int c1 = min(ncols, c0 + cols_per_cta);
  for (int i = threadIdx.x; i < nx * J; i += blockDim.x) {
    const int xx = i / J, l = i - xx * J;
    vt[i] = (l < nj) ? __ldg(Vt + (long)xx * P + j0 + l) : (T)0;
  }
  for (int c = c0; c < c1; ++c) {
    for (int i = threadIdx.x; i < nx * J; i += blockDim.x) tile[i] = mk<C>(0.0, 0.0);
    __syncthreads();
    const C* Wc = W + (long)c * n_act * P + j0;
    for (int i = threadIdx.x; i < n_act * J; i += blockDim.x) {
      const int s = i / J, l = i - s * J;
      if (l < nj) tile[slot_xpos[s] * J + l] = Wc[(long)s * P + l];
    }
    __syncthreads();
    fft_lines<T, true>(tile, px, J, 1, J, (T)1, true);
    for (int i = threadIdx.x; i < nx * J; i += blockDim.x) tile[i] = cscale(tile[i], vt[i]);
    __syncthreads();
    fft_lines<T, false>(tile, px, J, 1, J, (T)-1, true);
    C* Wo = W + (long)c * n_act * P + j0;
    for (int i = threadIdx.x; i < n_act * J; i += blockDim.x) {
      const int s = i / J, l = i - s * J;
      if (l < nj) Wo[(long)s * P + l] = tile[slot_xpos[s] * J + l];
    }
    __syncthreads();
  }
}

template <typename T>
__global__ void __launch_bounds__(512) k_plane_fwd(const cplx<T>* __restrict__ W, int n_act,
                                                   const int* __restrict__ plane_off, const int* __restrict__ pw_idx,
                                                   const int* __restrict__ pw_spos, Fft1d py, Fft1d pz, int ny,
                                                   int nz, const double2* __restrict__ x, double2* __restrict__ y,
                                                   long npw, const double* __restrict__ kinetic, double invN) {
  using C = cplx<T>;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* S = reinterpret_cast<C*>(smraw);
  const int slot = blockIdx.x;
  const long b = blockIdx.y;
  const int P = ny * nz;
  const C* Wp = W + (b * n_act + slot) * (long)P;
  for (int i = threadIdx.x; i < P; i += blockDim.x) S[i] = Wp[i];
  __syncthreads();
  fft_lines<T, false>(S, py, 1, ny, nz, (T)-1, false);
  fft_lines<T, false>(S, pz, ny, 1, ny, (T)-1, true);
  const int j1 = plane_off[slot + 1];
  for (int j = plane_off[slot] + threadIdx.x; j < j1; j += blockDim.x) {
    const int g = pw_idx[j];
    const C v = S[pw_spos[j]];
    const double2 xv = __ldg(x + b * npw + g);
    const double kin = __ldg(kinetic + g);
    double2 out;
    out.x = kin * xv.x + (double)v.x * invN;
    out.y = kin * xv.y + (double)v.y * invN;
    y[b * npw + g] = out;
  }
}

// Density: inverse transform only, then rho(x, j) += sum_b w_b |psi_b|^2 / Omega over the column block.
template <typename T>
__global__ void __launch_bounds__(256) k_xline_density(const cplx<T>* __restrict__ W, int n_act,
                                                       const int* __restrict__ slot_xpos, Fft1d px, int P, int ncols,
                                                       int J, const double* __restrict__ w, double inv_vol,
                                                       double* __restrict__ rho) {
  using C = cplx<T>;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int nx = px.n;
  C* tile = reinterpret_cast<C*>(smraw);                             // [nx][J]
  double* acc = reinterpret_cast<double*>(smraw + sizeof(C) * nx * J);  // [nx][J]
  const int j0 = blockIdx.x * J;
  const int nj = min(J, P - j0);
  for (int i = threadIdx.x; i < nx * J; i += blockDim.x) acc[i] = 0.0;
  for (int c = 0; c < ncols; ++c) {
    for (int i = threadIdx.x; i < nx * J; i += blockDim.x) tile[i] = mk<C>(0.0, 0.0);
    __syncthreads();
    const C* Wc = W + (long)c * n_act * P + j0;
    for (int i = threadIdx.x; i < n_act * J; i += blockDim.x) {
      const int s = i / J, l = i - s * J;
      if (l < nj) tile[slot_xpos[s] * J + l] = Wc[(long)s * P + l];
    }
    __syncthreads();
    fft_lines<T, true>(tile, px, J, 1, J, (T)1, true);
    const double wc = __ldg(w + c) * inv_vol;
    for (int i = threadIdx.x; i < nx * J; i += blockDim.x) {
      const C v = tile[i];
      acc[i] += wc * ((double)v.x * (double)v.x + (double)v.y * (double)v.y);
    }
    __syncthreads();
  }
  // rho is x-fastest: rho[x + nx*j] with j = z*ny + y
  for (int i = threadIdx.x; i < nx * J; i += blockDim.x) {
    const int l = i / nx, xx = i - l * nx;
    if (l < nj) rho[(long)(j0 + l) * nx + xx] += acc[xx * J + l];
  }
}

// P[p][g] = phi_m(g) * exp(i G_g . tau_a) for the projectors of one atom (apply.zig:883-896, 1118-1140).
__global__ void k_build_projectors(double2* __restrict__ P, const double* __restrict__ phi, int mt, long npw,
                                   const double* __restrict__ gcart, double tx, double ty, double tz) {
  const long g = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (g >= npw) return;
  const double arg = gcart[3 * g] * tx + gcart[3 * g + 1] * ty + gcart[3 * g + 2] * tz;
  double s, c;
  sincos(arg, &s, &c);
  for (int m = 0; m < mt; ++m) {
    const double f = phi[(long)m * npw + g];
    P[(long)m * npw + g] = make_double2(f * c, f * s);
  }
}

// coef2[p][c] = sum_j D_atom[p - off][j] * coef[off + j][c]  (apply.zig:1186-1275)
__global__ void k_apply_dij(const double2* __restrict__ coef, double2* __restrict__ coef2, const double* __restrict__ D,
                            const int* __restrict__ proj_off, const int* __restrict__ proj_mt, int maxm, int nproj,
                            int ncols) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= (long)nproj * ncols) return;
  const int p = (int)(i / ncols), c = (int)(i - (long)p * ncols);
  const int off = proj_off[p], mt = proj_mt[p];
  double2 acc = make_double2(0.0, 0.0);
  for (int j = 0; j < mt; ++j) {
    const double d = D[(long)p * maxm + j];
    if (d == 0.0) continue;
    const double2 v = coef[(long)(off + j) * ncols + c];
    acc.x += d * v.x;
    acc.y += d * v.y;
  }
  coef2[(long)p * ncols + c] = acc;
}

// e[c] = Re sum_p conj(coef[p][c]) coef2[p][c] / Omega  (kpoint/density.zig:145-165)
__global__ void k_nl_energy(const double2* __restrict__ coef, const double2* __restrict__ coef2, int nproj, int ncols,
                            double inv_vol, double* __restrict__ e) {
  const int c = blockIdx.x;
  double s = 0.0;
  for (int p = threadIdx.x; p < nproj; p += blockDim.x) {
    const double2 a = coef[(long)p * ncols + c], b = coef2[(long)p * ncols + c];
    s += a.x * b.x + a.y * b.y;
  }
  __shared__ double red[256];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) e[c] = red[0] * inv_vol;
}

__global__ void k_transpose_vloc(const double* __restrict__ v, double* __restrict__ vt, float* __restrict__ vt32, int nx,
                                 int ny, int nz, double* __restrict__ vn, float* __restrict__ vn32) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const long N = (long)nx * ny * nz;
  if (i >= N) return;
  if (vn) {  // natural order for the stick-layout passes
    vn[i] = v[i];
    vn32[i] = (float)v[i];
  }
  // i = x + nx*(y + ny*z)  ->  vt[x][z][y]
  const int xx = (int)(i % nx);
  const long r = i / nx;
  const int yy = (int)(r % ny);
  const int zz = (int)(r / ny);
  const long o = (long)xx * ny * nz + (long)zz * ny + yy;
  vt[o] = v[i];
  vt32[o] = (float)v[i];
}

// ------------------------------------------------------------------------------------------

static const size_t kSmemMax = 227 * 1024;

template <typename T>
static int set_smem_attrs() {
  DFT_TRY(ensure_max_dynamic_smem((const void*)k_plane_inv<T>, (int)kSmemMax));
  DFT_TRY(ensure_max_dynamic_smem((const void*)k_plane_fwd<T>, (int)kSmemMax));
  DFT_TRY(ensure_max_dynamic_smem((const void*)k_xline<T>, (int)kSmemMax));
  DFT_TRY(ensure_max_dynamic_smem((const void*)k_xline_density<T>, (int)kSmemMax));
  return DFTCUDA_OK;
}

static int line_tile(int nx) { return nx > 64 ? 16 : 32; }

template <typename T>
static size_t box_bytes_per_col(const dftcuda_kctx* c) {
  return sizeof(cplx<T>) * (size_t)c->n_act * c->P;
}

// The local passes of this context's precision use the stick layout (local_sticks.cu).
static bool use_sticks(const dftcuda_kctx* c) {
  if (c->fft_generic || c->sticks_off) return false;
  return c->precision == DFTCUDA_PRECISION_FP64 ? c->sticks64 : c->sticks32;
}

// Workspace bytes per column of the local passes (apply = H|psi>, else the density passes, which
// keep the plane layout).
static bool use_sticks_density(const dftcuda_kctx* c) { return use_sticks(c) && kctx_sticks_density_ok(c, c->precision); }

static size_t box_col_bytes(const dftcuda_kctx* c, bool apply) {
  const size_t cs = c->precision != DFTCUDA_PRECISION_FP64 ? sizeof(float2) : sizeof(double2);
  if (apply ? use_sticks(c) : use_sticks_density(c)) return sticks_bytes_per_col(c, cs);
  return cs * (size_t)c->n_act * c->P;
}

static size_t chunk_cols(const dftcuda_kctx* c, size_t ncols, bool apply) {
  size_t ch = (size_t)std::max(1.0, c->w_budget_bytes / (double)box_col_bytes(c, apply));
  return std::min(ch, std::max<size_t>(ncols, 1));
}

static int ensure_box(dftcuda_kctx* c, size_t cols, bool apply) {
  const size_t bytes = box_col_bytes(c, apply) * cols;
  if (bytes <= c->box_bytes) return DFTCUDA_OK;
  if (c->d_box) cudaFree(c->d_box);
  c->d_box = nullptr;
  c->box_bytes = 0;
  if (dev_malloc(&c->d_box, bytes) != cudaSuccess) return fail(DFTCUDA_ERR_OUT_OF_MEMORY, "box workspace");
  c->box_bytes = bytes;
  return DFTCUDA_OK;
}

template <typename T>
static int local_block(dftcuda_kctx* c, const double2* x, double2* y, size_t ncols, cudaStream_t s) {
  DFT_TRY(set_smem_attrs<T>());
  cplx<T>* W = reinterpret_cast<cplx<T>*>(c->d_box);
  const size_t smem_plane = sizeof(cplx<T>) * (size_t)c->P;
  if (smem_plane > kSmemMax) return fail(DFTCUDA_ERR_UNSUPPORTED, "y-z plane does not fit shared memory");
  dim3 gp(c->n_act, (unsigned)ncols);
  {
    ProfScope ps(c, P_PLANE_INV, s);
    k_plane_inv<T><<<gp, 512, smem_plane, s>>>(x, (long)c->npw, W, c->n_act, c->d_plane_off, c->d_pw_idx, c->d_pw_spos,
                                               c->fy.dev, c->fz.dev, c->ny, c->nz); count_launch();
  }
  const int J = line_tile(c->nx);
  const int cpc = 4;
  dim3 gx(ceil_div(c->P, J), ceil_div(ncols, cpc));
  const size_t smem_x = (sizeof(cplx<T>) + sizeof(T)) * (size_t)c->nx * J;
  const T* vt = std::is_same<T, double>::value ? (const T*)c->d_vt : (const T*)c->d_vt32;
  {
    ProfScope ps(c, P_XLINE, s);
    k_xline<T><<<gx, 256, smem_x, s>>>(W, c->n_act, c->d_slot_xpos, vt, c->fx.dev, c->P, (int)ncols, J, cpc); count_launch();
  }
  {
    ProfScope ps(c, P_PLANE_FWD, s);
    k_plane_fwd<T><<<gp, 512, smem_plane, s>>>(W, c->n_act, c->d_plane_off, c->d_pw_idx, c->d_pw_spos, c->fy.dev,
                                               c->fz.dev, c->ny, c->nz, x, y, (long)c->npw, c->d_kinetic,
                                               1.0 / (double)c->N); count_launch();
  }
  DFT_CUDA_TRY(cudaGetLastError());
  return DFTCUDA_OK;
}

int kctx_ensure_coef(dftcuda_kctx* c, size_t cols) {
  if (c->nl.nproj == 0) return DFTCUDA_OK;
  if (cols > c->coef_cols) {
    if (c->d_coef) cudaFree(c->d_coef);
    if (c->d_coef2) cudaFree(c->d_coef2);
    c->d_coef = c->d_coef2 = nullptr;
    c->coef_cols = 0;
    const size_t b = sizeof(double2) * (size_t)c->nl.nproj * cols;
    if (dev_malloc(&c->d_coef, b) != cudaSuccess || dev_malloc(&c->d_coef2, b) != cudaSuccess)
      return fail(DFTCUDA_ERR_OUT_OF_MEMORY, "projector coefficients");
    c->coef_cols = cols;
  }
  size_t need = std::max(zgemm_workspace_elems(c->nl.nproj, (int)cols, (int)c->npw),
                         zgemm_workspace_elems((int)cols, (int)c->npw, c->nl.nproj));
  if (precision_uses_tc(c->precision)) {
    need = std::max(need, cgemm_tf32_workspace_elems(c->nl.nproj, (int)cols, (int)c->npw));
    need = std::max(need, cgemm_tf32_workspace_elems((int)cols, (int)c->npw, c->nl.nproj));
    if (!c->d_err) {
      if (dev_malloc(&c->d_err, sizeof(int)) != cudaSuccess) return fail(DFTCUDA_ERR_OUT_OF_MEMORY, "error flag");
      DFT_CUDA_TRY(cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream));
      DFT_CUDA_TRY(cudaStreamSynchronize(c->stream));
    }
  }
  // forced split counts (autotuner) need their partial sums
  need = std::max(need, (size_t)std::max(c->split_proj, 0) * c->nl.nproj * cols);
  need = std::max(need, (size_t)std::min(std::max(c->split_back, 0), std::max(1, c->nl.nproj / 32)) * cols * c->npw);
  if (need > c->gemm_ws_elems) {
    if (c->d_gemm_ws) cudaFree(c->d_gemm_ws);
    c->d_gemm_ws = nullptr;
    c->gemm_ws_elems = 0;
    if (dev_malloc(&c->d_gemm_ws, need * sizeof(double2)) != cudaSuccess) return fail(DFTCUDA_ERR_OUT_OF_MEMORY, "gemm workspace");
    c->gemm_ws_elems = need;
  }
  return DFTCUDA_OK;
}

// d_coef[p][c] = sum_g P[p][g] x[c][g]   (batch_project_coeffs, apply.zig:1143-1183)
int kctx_project(dftcuda_kctx* c, const double2* x, size_t ncols, cudaStream_t s) {
  GemmArgs g{};
  g.M = c->nl.nproj; g.N = (int)ncols; g.K = (int)c->npw;
  g.A = c->nl.P; g.lda = (long)c->npw; g.a_kc = true; g.conj_a = false;
  g.B = x; g.ldb = (long)c->npw; g.b_kc = true; g.conj_b = false;
  g.O = c->d_coef; g.ldo_r = (long)ncols; g.ldo_c = 1;
  g.alpha = 1.0; g.beta = 0.0;
  g.splits = c->split_proj;
  g.a_cache = &c->tc_ptiles_proj;
  if (precision_uses_tc(c->precision) && tc_worthwhile(g.M, g.N, g.K, c->tc_min_flops))
    return cgemm_tf32(g, s, c->d_gemm_ws, c->gemm_ws_elems, c->d_err, c->precision == DFTCUDA_PRECISION_TF32X3, &c->tc_scratch);
  return zgemm(g, s, c->d_gemm_ws, c->gemm_ws_elems);
}

static int nonlocal_block(dftcuda_kctx* c, const double2* x, double2* y, size_t ncols, cudaStream_t s) {
  {
    ProfScope ps(c, P_NL_PROJECT, s);
    DFT_TRY(kctx_project(c, x, ncols, s));
  }
  {
    ProfScope ps(c, P_NL_DIJ, s);
    const long tot = (long)c->nl.nproj * ncols;
    k_apply_dij<<<ceil_div(tot, 256), 256, 0, s>>>(c->d_coef, c->d_coef2, c->nl.D, c->nl.proj_off, c->nl.proj_mt,
                                                   c->nl.maxm, c->nl.nproj, (int)ncols); count_launch();
  }
  // y[c][g] += (1/Omega) sum_p coef2[p][c] conj(P[p][g])   (apply.zig:1278-1336)
  ProfScope ps(c, P_NL_BACK, s);
  GemmArgs g{};
  g.M = (int)ncols; g.N = (int)c->npw; g.K = c->nl.nproj;
  g.A = c->d_coef2; g.lda = (long)ncols; g.a_kc = false; g.conj_a = false;
  g.B = c->nl.P; g.ldb = (long)c->npw; g.b_kc = false; g.conj_b = true;
  g.O = y; g.ldo_r = (long)c->npw; g.ldo_c = 1;
  g.alpha = 1.0 / c->volume; g.beta = 1.0;
  g.splits = c->split_back;
  g.b_cache = &c->tc_ptiles_back;
  if (precision_uses_tc(c->precision) && tc_worthwhile(g.M, g.N, g.K, c->tc_min_flops))
    return cgemm_tf32(g, s, c->d_gemm_ws, c->gemm_ws_elems, c->d_err, c->precision == DFTCUDA_PRECISION_TF32X3, &c->tc_scratch);
  return zgemm(g, s, c->d_gemm_ws, c->gemm_ws_elems);
}

int kctx_apply_h_dev(dftcuda_kctx* c, const double2* x, double2* y, size_t ncols, cudaStream_t s) {
  if (!c->has_vloc) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "apply_h: local potential not set (dftcuda_set_vloc)");
  if (ncols == 0) return DFTCUDA_OK;
  if (c->prof.on) {
    c->prof.calls += 1;
    c->prof.columns += ncols;
  }
  const size_t ch = chunk_cols(c, ncols, true);
  DFT_TRY(ensure_box(c, ch, true));
  const bool sticks = use_sticks(c);
  c->last_layout = sticks ? 2 : ((c->precision == DFTCUDA_PRECISION_FP64 ? c->fast64 : c->fast32) && !c->fft_generic ? 1 : 0);
  for (size_t c0 = 0; c0 < ncols; c0 += ch) {
    const size_t nc = std::min(ch, ncols - c0);
    const double2* xc = x + c0 * c->npw;
    double2* yc = y + c0 * c->npw;
    if (sticks) {
      if (c->precision != DFTCUDA_PRECISION_FP64)
        DFT_TRY(local_block_sticks<float>(c, xc, yc, nc, s));
      else
        DFT_TRY(local_block_sticks<double>(c, xc, yc, nc, s));
    } else if (c->precision != DFTCUDA_PRECISION_FP64) {
      if (c->fast32 && !c->fft_generic)
        DFT_TRY(local_block4<float>(c, xc, yc, nc, s));
      else
        DFT_TRY(local_block<float>(c, xc, yc, nc, s));
    } else {
      if (c->fast64 && !c->fft_generic)
        DFT_TRY(local_block4<double>(c, xc, yc, nc, s));
      else
        DFT_TRY(local_block<double>(c, xc, yc, nc, s));
    }
  }
  if (c->nl.nproj > 0) {
    const size_t nch = std::min<size_t>(ncols, 256);
    DFT_TRY(kctx_ensure_coef(c, nch));
    for (size_t c0 = 0; c0 < ncols; c0 += nch) {
      const size_t nc = std::min(nch, ncols - c0);
      DFT_TRY(nonlocal_block(c, x + c0 * c->npw, y + c0 * c->npw, nc, s));
    }
  }
  return DFTCUDA_OK;
}

template <typename T>
static int density_block(dftcuda_kctx* c, const double2* x, size_t ncols, const double* w, double* rho, cudaStream_t s) {
  DFT_TRY(set_smem_attrs<T>());
  ProfScope ps(c, P_DENSITY, s);
  cplx<T>* W = reinterpret_cast<cplx<T>*>(c->d_box);
  const size_t smem_plane = sizeof(cplx<T>) * (size_t)c->P;
  if (smem_plane > kSmemMax) return fail(DFTCUDA_ERR_UNSUPPORTED, "y-z plane does not fit shared memory");
  dim3 gp(c->n_act, (unsigned)ncols);
  k_plane_inv<T><<<gp, 512, smem_plane, s>>>(x, (long)c->npw, W, c->n_act, c->d_plane_off, c->d_pw_idx, c->d_pw_spos,
                                             c->fy.dev, c->fz.dev, c->ny, c->nz); count_launch();
  const int J = line_tile(c->nx);
  const size_t smem_x = (sizeof(cplx<T>) + sizeof(double)) * (size_t)c->nx * J;
  k_xline_density<T><<<ceil_div(c->P, J), 256, smem_x, s>>>(W, c->n_act, c->d_slot_xpos, c->fx.dev, c->P, (int)ncols, J,
                                                            w, 1.0 / c->volume, rho); count_launch();
  DFT_CUDA_TRY(cudaGetLastError());
  return DFTCUDA_OK;
}

int kctx_density_dev(dftcuda_kctx* c, const double2* vecs, size_t nbands, const double* w_dev, double* rho_dev,
                     cudaStream_t s) {
  if (nbands == 0) return DFTCUDA_OK;
  const size_t ch = chunk_cols(c, nbands, false);
  DFT_TRY(ensure_box(c, ch, false));
  const bool sticks = use_sticks_density(c);
  for (size_t c0 = 0; c0 < nbands; c0 += ch) {
    const size_t nc = std::min(ch, nbands - c0);
    if (sticks) {
      if (c->precision != DFTCUDA_PRECISION_FP64)
        DFT_TRY(density_block_sticks<float>(c, vecs + c0 * c->npw, nc, w_dev + c0, rho_dev, s));
      else
        DFT_TRY(density_block_sticks<double>(c, vecs + c0 * c->npw, nc, w_dev + c0, rho_dev, s));
    } else if (c->precision != DFTCUDA_PRECISION_FP64) {
      if (c->fast32 && !c->fft_generic)
        DFT_TRY(density_block4<float>(c, vecs + c0 * c->npw, nc, w_dev + c0, rho_dev, s));
      else
        DFT_TRY(density_block<float>(c, vecs + c0 * c->npw, nc, w_dev + c0, rho_dev, s));
    } else {
      if (c->fast64 && !c->fft_generic)
        DFT_TRY(density_block4<double>(c, vecs + c0 * c->npw, nc, w_dev + c0, rho_dev, s));
      else
        DFT_TRY(density_block<double>(c, vecs + c0 * c->npw, nc, w_dev + c0, rho_dev, s));
    }
  }
  return DFTCUDA_OK;
}

// Turns the device error flag of the bounded waits into DFTCUDA_ERR_TIMEOUT (and clears it).
int kctx_check_error(dftcuda_kctx* c) {
  if (!c->d_err) return DFTCUDA_OK;
  int h = 0;
  DFT_CUDA_TRY(cudaMemcpyAsync(&h, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  DFT_CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (h == 0) return DFTCUDA_OK;
  DFT_CUDA_TRY(cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream));
  DFT_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return fail(DFTCUDA_ERR_TIMEOUT, "tensor-core GEMM: a bounded mbarrier wait gave up");
}

int kctx_stage(dftcuda_kctx* c, size_t cols) {
  if (cols <= c->stage_cols) return DFTCUDA_OK;
  if (c->d_x) cudaFree(c->d_x);
  if (c->d_y) cudaFree(c->d_y);
  c->d_x = c->d_y = nullptr;
  c->stage_cols = 0;
  const size_t b = sizeof(double2) * c->npw * cols;
  if (dev_malloc(&c->d_x, b) != cudaSuccess || dev_malloc(&c->d_y, b) != cudaSuccess)
    return fail(DFTCUDA_ERR_OUT_OF_MEMORY, "staging buffers");
  c->stage_cols = cols;
  return DFTCUDA_OK;
}

}  // namespace dftcuda

using namespace dftcuda;

// ------------------------------------------------------------------------------------------
// C ABI
// ------------------------------------------------------------------------------------------

static void free_nonlocal(dftcuda_kctx* c) {
  if (c->nl.P) cudaFree(c->nl.P);
  if (c->nl.D) cudaFree(c->nl.D);
  if (c->nl.proj_off) cudaFree(c->nl.proj_off);
  if (c->nl.proj_mt) cudaFree(c->nl.proj_mt);
  c->nl = NonlocalDev{};
}

extern "C" int dftcuda_kctx_destroy(dftcuda_kctx* c) {
  if (!c) return DFTCUDA_OK;
  // the context's device, whatever the caller has current; the release goes ahead even if switching
  // fails (at process exit the runtime may already be unloading)
  DeviceGuard dg(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  eig_destroy(c->eig);
  c->prof.destroy();
  free_nonlocal(c);
  void* ptrs[] = {c->d_plane_off, c->d_pw_idx, c->d_pw_spos, c->d_slot_xpos, c->d_kinetic, c->d_gcart, c->d_vt,
                  c->d_vt32, c->d_box, c->d_coef, c->d_coef2, c->d_gemm_ws, c->d_x, c->d_y, c->d_rho, c->d_w,
                  c->d_pwmap, c->d_stick_off, c->d_stick_y, c->d_slot_of_x, c->d_tw4x64, c->d_tw4x32,
                  c->d_tw4p64, c->d_tw4p32, c->d_err, c->d_mlp, c->d_vstage, c->d_st_sy, c->d_st_map, c->d_st_sox,
                  c->d_twz64, c->d_twz32, c->d_twx64, c->d_twx32, c->d_vn, c->d_vn32};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  c->fx.destroy(); c->fy.destroy(); c->fz.destroy();
  c->tc_scratch.release();
  c->tc_ptiles_proj.release();
  c->tc_ptiles_back.release();
  if (c->ev_order) cudaEventDestroy(c->ev_order);
  for (int i = 0; i < kPipeChunks; ++i) {
    if (c->ev_in[i]) cudaEventDestroy(c->ev_in[i]);
    if (c->ev_done[i]) cudaEventDestroy(c->ev_done[i]);
  }
  if (c->s_in) cudaStreamDestroy(c->s_in);
  if (c->s_out) cudaStreamDestroy(c->s_out);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return DFTCUDA_OK;
}

extern "C" int dftcuda_kctx_create(dftcuda_kctx** out, int nx, int ny, int nz, double volume, size_t n_pw,
                                   const int32_t* hkl, const double* kinetic, const double* gcart, int precision) {
  if (!out) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "kctx_create: out is null");
  *out = nullptr;
  if (nx <= 0 || ny <= 0 || nz <= 0 || !(volume > 0.0) || n_pw == 0 || !hkl || !kinetic || !gcart)
    return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "kctx_create: bad arguments");
  if (precision < DFTCUDA_PRECISION_FP64 || precision > DFTCUDA_PRECISION_TF32X3)
    return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "kctx_create: unknown precision");
  // Miller index range check, same rule as PwGridMap.init (pw_grid_map.zig:27-35).
  const int min_h = -(nx / 2), min_k = -(ny / 2), min_l = -(nz / 2);
  for (size_t i = 0; i < n_pw; ++i) {
    const int h = hkl[3 * i] - min_h, k = hkl[3 * i + 1] - min_k, l = hkl[3 * i + 2] - min_l;
    if (h < 0 || k < 0 || l < 0 || h >= nx || k >= ny || l >= nz)
      return fail(DFTCUDA_ERR_INVALID_GRID, "kctx_create: Miller index outside the FFT box");
  }
  auto* c = new dftcuda_kctx();
  c->nx = nx; c->ny = ny; c->nz = nz;
  c->N = (long)nx * ny * nz;
  c->P = ny * nz;
  c->volume = volume;
  c->npw = n_pw;
  c->precision = precision;
  int s;
  if ((s = c->fx.create(nx)) || (s = c->fy.create(ny)) || (s = c->fz.create(nz))) {
    dftcuda_kctx_destroy(c);
    return s;
  }
  if ((size_t)c->P * sizeof(double2) > kSmemMax && precision == DFTCUDA_PRECISION_FP64) {
    dftcuda_kctx_destroy(c);
    return fail(DFTCUDA_ERR_UNSUPPORTED, "kctx_create: ny*nz plane exceeds shared memory for FP64");
  }
  // A blocking stream: its work is ordered after what the caller queued on the legacy default stream
  // (torch's default stream, plain cudaMemcpy), so device inputs written there are complete when the
  // context's kernels read them; contexts' streams still run concurrently with one another.
  if (cudaGetDevice(&c->device) != cudaSuccess || cudaStreamCreateWithFlags(&c->stream, cudaStreamDefault) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_order, cudaEventDisableTiming) != cudaSuccess) {
    dftcuda_kctx_destroy(c);
    return fail(DFTCUDA_ERR_CUDA, "kctx_create: stream");
  }
  // Group plane waves by x-frequency plane.
  std::vector<int> slot_of_x(nx, -1), xs;
  std::vector<int> xpos(n_pw);
  for (size_t i = 0; i < n_pw; ++i) {
    const int x = ((hkl[3 * i] % nx) + nx) % nx;
    xpos[i] = x;
    if (slot_of_x[x] < 0) { slot_of_x[x] = 0; xs.push_back(x); }
  }
  std::sort(xs.begin(), xs.end());
  for (size_t sidx = 0; sidx < xs.size(); ++sidx) slot_of_x[xs[sidx]] = (int)sidx;
  c->n_act = (int)xs.size();
  std::vector<int> cnt(c->n_act + 1, 0);
  for (size_t i = 0; i < n_pw; ++i) cnt[slot_of_x[xpos[i]] + 1]++;
  for (int sidx = 0; sidx < c->n_act; ++sidx) cnt[sidx + 1] += cnt[sidx];
  std::vector<int> fill(cnt.begin(), cnt.end() - 1), pw_idx(n_pw), pw_spos(n_pw);
  for (size_t i = 0; i < n_pw; ++i) {
    const int sidx = slot_of_x[xpos[i]];
    const int j = fill[sidx]++;
    const int y = ((hkl[3 * i + 1] % ny) + ny) % ny, z = ((hkl[3 * i + 2] % nz) + nz) % nz;
    pw_idx[j] = (int)i;
    pw_spos[j] = c->fz.pinv[z] * ny + c->fy.pinv[y];
  }
  std::vector<int> slot_xpos(c->n_act);
  for (int sidx = 0; sidx < c->n_act; ++sidx) slot_xpos[sidx] = c->fx.pinv[xs[sidx]];
  c->h_kinetic.assign(kinetic, kinetic + n_pw);
  bool ok = dev_malloc(&c->d_plane_off, sizeof(int) * (c->n_act + 1)) == cudaSuccess &&
            dev_malloc(&c->d_pw_idx, sizeof(int) * n_pw) == cudaSuccess &&
            dev_malloc(&c->d_pw_spos, sizeof(int) * n_pw) == cudaSuccess &&
            dev_malloc(&c->d_slot_xpos, sizeof(int) * c->n_act) == cudaSuccess &&
            dev_malloc(&c->d_kinetic, sizeof(double) * n_pw) == cudaSuccess &&
            dev_malloc(&c->d_gcart, sizeof(double) * 3 * n_pw) == cudaSuccess &&
            dev_malloc(&c->d_vt, sizeof(double) * c->N) == cudaSuccess &&
            dev_malloc(&c->d_vt32, sizeof(float) * c->N) == cudaSuccess;
  if (!ok) {
    dftcuda_kctx_destroy(c);
    return fail(DFTCUDA_ERR_OUT_OF_MEMORY, "kctx_create: device tables");
  }
  // Uploads are ordered on the context's own stream (a plain cudaMemcpy from pageable memory may
  // return before its DMA lands).
  cudaStream_t st = c->stream;
  cudaMemcpyAsync(c->d_plane_off, cnt.data(), sizeof(int) * (c->n_act + 1), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(c->d_pw_idx, pw_idx.data(), sizeof(int) * n_pw, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(c->d_pw_spos, pw_spos.data(), sizeof(int) * n_pw, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(c->d_slot_xpos, slot_xpos.data(), sizeof(int) * c->n_act, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(c->d_kinetic, kinetic, sizeof(double) * n_pw, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(c->d_gcart, gcart, sizeof(double) * 3 * n_pw, cudaMemcpyHostToDevice, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) {
    dftcuda_kctx_destroy(c);
    return fail(DFTCUDA_ERR_CUDA, "kctx_create: upload");
  }
  if (const char* e = std::getenv("DFTCUDA_TC_MIN_FLOP")) c->tc_min_flops = std::atof(e);
  // The four-step register-FFT passes, unless DFTCUDA_FFT_PATH=generic asks for the stage-by-stage ones.
  const char* path = std::getenv("DFTCUDA_FFT_PATH");
  if (!(path && std::string(path) == "generic")) {
    if ((s = kctx_setup_fast_path(c, slot_of_x, xpos, hkl)) != DFTCUDA_OK ||
        (s = kctx_setup_sticks(c, slot_of_x, xpos, hkl)) != DFTCUDA_OK) {
      dftcuda_kctx_destroy(c);
      return s;
    }
  }
  *out = c;
  return DFTCUDA_OK;
}

extern "C" size_t dftcuda_kctx_npw(const dftcuda_kctx* c) { return c ? c->npw : 0; }

extern "C" int dftcuda_set_vloc(dftcuda_kctx* c, const double* v) {
  if (!c || !v) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "set_vloc: null argument");
  DeviceGuard dg(c->device);  // the context's device, whatever the caller has current
  DFT_TRY(dg.status);
  const bool dev = is_device_pointer(v);
  // A staging buffer kept in the context: cudaFree would synchronise the whole device (every other
  // k-point's stream) on each SCF iteration.
  if (!dev && !c->d_vstage && dev_malloc(&c->d_vstage, sizeof(double) * c->N) != cudaSuccess)
    return fail(DFTCUDA_ERR_OUT_OF_MEMORY, "set_vloc staging");
  if (!dev) DFT_CUDA_TRY(cudaMemcpyAsync(c->d_vstage, v, sizeof(double) * c->N, cudaMemcpyHostToDevice, c->stream));
  k_transpose_vloc<<<ceil_div(c->N, 256), 256, 0, c->stream>>>(dev ? v : c->d_vstage, c->d_vt, c->d_vt32, c->nx, c->ny, c->nz,
                                                                c->d_vn, c->d_vn32); count_launch();
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return fail(DFTCUDA_ERR_CUDA, std::string("set_vloc: ") + cudaGetErrorString(e));
  c->has_vloc = true;
  return DFTCUDA_OK;
}

extern "C" int dftcuda_set_projectors(dftcuda_kctx* c, size_t n_species, const dftcuda_species* species, size_t n_atoms,
                                      const int32_t* atom_species, const double* atom_pos) {
  if (!c) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "set_projectors: null context");
  DeviceGuard dg(c->device);  // the context's device, whatever the caller has current
  DFT_TRY(dg.status);
  cudaStreamSynchronize(c->stream);
  free_nonlocal(c);
  c->tc_ptiles_proj.release();  // the split copies of the old projector matrix
  c->tc_ptiles_back.release();
  c->natoms = 0;
  c->atom_row.clear();
  c->atom_mt.clear();
  c->atom_species.clear();
  c->atom_pos.clear();
  c->species_mt.clear();
  if (n_species == 0 || n_atoms == 0) return DFTCUDA_OK;
  if (!species || !atom_species || !atom_pos) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "set_projectors: null array");
  // Projector order follows apply.zig:1454-1482: species in order, then that species' atoms in order.
  int nproj = 0, maxm = 0;
  for (size_t s = 0; s < n_species; ++s) {
    const dftcuda_species& sp = species[s];
    size_t mt = 0;
    for (size_t b = 0; b < sp.beta_count; ++b) {
      if (sp.l_list[b] < 0) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "set_projectors: negative l");
      mt += 2 * sp.l_list[b] + 1;
    }
    if (mt != sp.m_total) return fail(DFTCUDA_ERR_INVALID_MATRIX_SIZE, "set_projectors: m_total does not match l_list");
    if (sp.m_total > 0 && !sp.phi) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "set_projectors: phi is null");
    maxm = std::max(maxm, (int)sp.m_total);
    for (size_t a = 0; a < n_atoms; ++a)
      if ((size_t)atom_species[a] == s) nproj += (int)sp.m_total;
  }
  for (size_t a = 0; a < n_atoms; ++a)
    if (atom_species[a] < 0 || (size_t)atom_species[a] >= n_species)
      return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "set_projectors: atom species index out of range");
  if (nproj == 0) return DFTCUDA_OK;
  NonlocalDev& nl = c->nl;
  nl.nproj = nproj;
  nl.maxm = maxm;
  std::vector<double> D((size_t)nproj * maxm, 0.0);
  std::vector<int> poff(nproj), pmt(nproj);
  if (dev_malloc(&nl.P, sizeof(double2) * (size_t)nproj * c->npw) != cudaSuccess) {
    free_nonlocal(c);
    return fail(DFTCUDA_ERR_OUT_OF_MEMORY, "set_projectors: projector matrix");
  }
  double* dphi = nullptr;
  c->natoms = (int)n_atoms;
  c->atom_row.assign(n_atoms, 0);
  c->atom_mt.assign(n_atoms, 0);
  c->atom_species.assign(atom_species, atom_species + n_atoms);
  c->atom_pos.assign(atom_pos, atom_pos + 3 * n_atoms);
  c->species_mt.resize(n_species);
  for (size_t s = 0; s < n_species; ++s) c->species_mt[s] = species[s].m_total;
  int p = 0;
  for (size_t s = 0; s < n_species; ++s) {
    const dftcuda_species& sp = species[s];
    const int mt = (int)sp.m_total;
    if (mt == 0) continue;
    // expanded D (radial form: same-l blocks, m-diagonal), apply.zig:1186-1226
    std::vector<int> moff(sp.beta_count);
    int acc = 0;
    for (size_t b = 0; b < sp.beta_count; ++b) { moff[b] = acc; acc += 2 * sp.l_list[b] + 1; }
    std::vector<double> dm((size_t)mt * mt, 0.0);
    for (size_t b = 0; b < sp.beta_count; ++b)
      for (size_t j = 0; j < sp.beta_count; ++j) {
        if (sp.l_list[b] != sp.l_list[j]) continue;
        const double d = sp.dij[b * sp.beta_count + j];
        for (int mi = 0; mi < 2 * sp.l_list[b] + 1; ++mi) dm[(size_t)(moff[b] + mi) * mt + moff[j] + mi] = d;
      }
    if (dev_malloc(&dphi, sizeof(double) * (size_t)mt * c->npw) != cudaSuccess) {
      free_nonlocal(c);
      return fail(DFTCUDA_ERR_OUT_OF_MEMORY, "set_projectors: phi");
    }
    cudaMemcpyAsync(dphi, sp.phi, sizeof(double) * (size_t)mt * c->npw, cudaMemcpyHostToDevice, c->stream);
    for (size_t a = 0; a < n_atoms; ++a) {
      if ((size_t)atom_species[a] != s) continue;
      c->atom_row[a] = p;
      c->atom_mt[a] = mt;
      k_build_projectors<<<ceil_div(c->npw, 256), 256, 0, c->stream>>>(nl.P + (size_t)p * c->npw, dphi, mt, (long)c->npw,
                                                                      c->d_gcart, atom_pos[3 * a], atom_pos[3 * a + 1],
                                                                      atom_pos[3 * a + 2]); count_launch();
      for (int i = 0; i < mt; ++i) {
        poff[p + i] = p;
        pmt[p + i] = mt;
        for (int j = 0; j < mt; ++j) D[(size_t)(p + i) * maxm + j] = dm[(size_t)i * mt + j];
      }
      p += mt;
    }
    cudaStreamSynchronize(c->stream);
    cudaFree(dphi);
    dphi = nullptr;
  }
  bool ok = dev_malloc(&nl.D, sizeof(double) * D.size()) == cudaSuccess &&
            dev_malloc(&nl.proj_off, sizeof(int) * nproj) == cudaSuccess &&
            dev_malloc(&nl.proj_mt, sizeof(int) * nproj) == cudaSuccess;
  if (!ok) {
    free_nonlocal(c);
    return fail(DFTCUDA_ERR_OUT_OF_MEMORY, "set_projectors: tables");
  }
  cudaMemcpyAsync(nl.D, D.data(), sizeof(double) * D.size(), cudaMemcpyHostToDevice, c->stream);
  cudaMemcpyAsync(nl.proj_off, poff.data(), sizeof(int) * nproj, cudaMemcpyHostToDevice, c->stream);
  cudaMemcpyAsync(nl.proj_mt, pmt.data(), sizeof(int) * nproj, cudaMemcpyHostToDevice, c->stream);
  DFT_CUDA_TRY(cudaStreamSynchronize(c->stream));
  DFT_CUDA_TRY(cudaGetLastError());
  return DFTCUDA_OK;
}

extern "C" int dftcuda_apply_h_batch_async(dftcuda_kctx* c, const double* x, double* y, size_t ncols, void* stream) {
  if (!c || (!x && ncols) || (!y && ncols)) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "apply_h_batch_async: null argument");
  DeviceGuard dg(c->device);  // the context's device, whatever the caller has current
  DFT_TRY(dg.status);
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  return kctx_apply_h_dev(c, (const double2*)x, (double2*)y, ncols, s);
}

// Column chunks of the host-buffer pipeline (len[0 .. returned count)).  Only the first chunk's copy
// in and the last chunk's copy out are not hidden under compute, so from 256 columns on the end
// chunks are 64 columns (one column tile of the projector GEMMs) and the middle ones multiples of 64
// (the last takes the remainder), at most kPipeChunks in all; below 256 columns, four equal chunks.
static int pipe_chunks(size_t ncols, size_t* len) {
  int k = 0;
  if (ncols < 256) {
    const size_t per = (ncols + 3) / 4;
    for (size_t c0 = 0; c0 < ncols; c0 += per) len[k++] = std::min(per, ncols - c0);
    return k;
  }
  const size_t mid = ncols - 128;
  const size_t nm = std::min<size_t>(kPipeChunks - 2, (mid + 127) / 128);
  const size_t per = ((mid + nm - 1) / nm + 63) / 64 * 64;
  len[k++] = 64;
  for (size_t left = mid; left > 0;) {
    const size_t t = std::min(per, left);
    len[k++] = t;
    left -= t;
  }
  len[k++] = 64;
  return k;
}

extern "C" int dftcuda_apply_h_batch(dftcuda_kctx* c, const double* x, double* y, size_t n, size_t ncols) {
  if (!c) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "apply_h_batch: null context");
  DeviceGuard dg(c->device);  // the context's device, whatever the caller has current
  DFT_TRY(dg.status);
  if (n != c->npw) return fail(DFTCUDA_ERR_INVALID_MATRIX_SIZE, "apply_h_batch: n != n_pw");  // apply.zig:1591
  if (ncols == 0) return DFTCUDA_OK;
  if (!x || !y) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "apply_h_batch: null buffer");
  const bool dx = is_device_pointer(x), dy = is_device_pointer(y);
  const size_t bytes = sizeof(double2) * n * ncols;
  const double2* xd = (const double2*)x;
  double2* yd = (double2*)y;
  if (!dx || !dy) DFT_TRY(kctx_stage(c, ncols));
  if (!dx && !dy && ncols >= 64) {
    // host buffers: kPipeChunks column chunks, chunk j's copy in (s_in) ahead of its compute
    // (context stream), its copy out (s_out) behind it, so the transfers hide under the compute
    // of the neighbouring chunks; every wait is an event, every stream is drained before return
    if (!c->s_in) {
      DFT_CUDA_TRY(cudaStreamCreateWithFlags(&c->s_in, cudaStreamDefault));
      DFT_CUDA_TRY(cudaStreamCreateWithFlags(&c->s_out, cudaStreamDefault));
      for (int i = 0; i < kPipeChunks; ++i) {
        DFT_CUDA_TRY(cudaEventCreateWithFlags(&c->ev_in[i], cudaEventDisableTiming));
        DFT_CUDA_TRY(cudaEventCreateWithFlags(&c->ev_done[i], cudaEventDisableTiming));
      }
    }
    size_t len[kPipeChunks];
    const int nchunks = pipe_chunks(ncols, len);
    int st = DFTCUDA_OK;
    size_t c0 = 0;
    for (int j = 0; j < nchunks && st == DFTCUDA_OK; c0 += len[j], ++j) {
      const size_t nc = len[j];
      const size_t off = c0 * n, cb = sizeof(double2) * n * nc;
      if (cudaMemcpyAsync(c->d_x + off, (const double2*)x + off, cb, cudaMemcpyHostToDevice, c->s_in) != cudaSuccess ||
          cudaEventRecord(c->ev_in[j], c->s_in) != cudaSuccess || cudaStreamWaitEvent(c->stream, c->ev_in[j], 0) != cudaSuccess) {
        st = fail(DFTCUDA_ERR_CUDA, "apply_h_batch: staging copy");
        break;
      }
      st = kctx_apply_h_dev(c, c->d_x + off, c->d_y + off, nc, c->stream);
      if (st != DFTCUDA_OK) break;
      if (cudaEventRecord(c->ev_done[j], c->stream) != cudaSuccess || cudaStreamWaitEvent(c->s_out, c->ev_done[j], 0) != cudaSuccess ||
          cudaMemcpyAsync((double2*)y + off, c->d_y + off, cb, cudaMemcpyDeviceToHost, c->s_out) != cudaSuccess)
        st = fail(DFTCUDA_ERR_CUDA, "apply_h_batch: result copy");
    }
    const cudaError_t e1 = cudaStreamSynchronize(c->s_in), e2 = cudaStreamSynchronize(c->stream), e3 = cudaStreamSynchronize(c->s_out);
    if (st != DFTCUDA_OK) return st;
    if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess) return fail(DFTCUDA_ERR_CUDA, "apply_h_batch: pipelined copies");
    DFT_TRY(kctx_check_error(c));
    return DFTCUDA_OK;
  }
  if (!dx) {
    DFT_CUDA_TRY(cudaMemcpyAsync(c->d_x, x, bytes, cudaMemcpyHostToDevice, c->stream));
    xd = c->d_x;
  }
  if (!dy) yd = c->d_y;
  DFT_TRY(kctx_apply_h_dev(c, xd, yd, ncols, c->stream));
  if (!dy) DFT_CUDA_TRY(cudaMemcpyAsync(y, yd, bytes, cudaMemcpyDeviceToHost, c->stream));
  DFT_CUDA_TRY(cudaStreamSynchronize(c->stream));
  DFT_TRY(kctx_check_error(c));
  return DFTCUDA_OK;
}

extern "C" int dftcuda_apply_h(dftcuda_kctx* c, const double* x, double* y, size_t n) {
  return dftcuda_apply_h_batch(c, x, y, n, 1);
}

extern "C" int dftcuda_nonlocal_energies(dftcuda_kctx* c, const double* psi, size_t n, size_t nbands, double* e_out) {
  if (!c) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "nonlocal_energies: null context");
  DeviceGuard dg(c->device);  // the context's device, whatever the caller has current
  DFT_TRY(dg.status);
  if (n != c->npw) return fail(DFTCUDA_ERR_INVALID_MATRIX_SIZE, "nonlocal_energies: n != n_pw");
  if (nbands == 0) return DFTCUDA_OK;
  if (!psi || !e_out) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "nonlocal_energies: null buffer");
  const bool dp = is_device_pointer(psi), de = is_device_pointer(e_out);
  if (c->nl.nproj == 0) {
    if (de) {
      DFT_CUDA_TRY(cudaMemsetAsync(e_out, 0, sizeof(double) * nbands, c->stream));
      DFT_CUDA_TRY(cudaStreamSynchronize(c->stream));
    }
    else std::memset(e_out, 0, sizeof(double) * nbands);
    return DFTCUDA_OK;
  }
  const double2* pd = (const double2*)psi;
  DFT_TRY(kctx_stage(c, nbands));
  if (!dp) {
    DFT_CUDA_TRY(cudaMemcpyAsync(c->d_x, psi, sizeof(double2) * n * nbands, cudaMemcpyHostToDevice, c->stream));
    pd = c->d_x;
  }
  double* ed = de ? e_out : (double*)c->d_y;
  const size_t nch = std::min<size_t>(nbands, 256);
  DFT_TRY(kctx_ensure_coef(c, nch));
  for (size_t c0 = 0; c0 < nbands; c0 += nch) {
    const size_t nc = std::min(nch, nbands - c0);
    DFT_TRY(kctx_project(c, pd + c0 * n, nc, c->stream));
    const long tot = (long)c->nl.nproj * nc;
    k_apply_dij<<<ceil_div(tot, 256), 256, 0, c->stream>>>(c->d_coef, c->d_coef2, c->nl.D, c->nl.proj_off, c->nl.proj_mt,
                                                          c->nl.maxm, c->nl.nproj, (int)nc); count_launch();
    k_nl_energy<<<(unsigned)nc, 256, 0, c->stream>>>(c->d_coef, c->d_coef2, c->nl.nproj, (int)nc, 1.0 / c->volume, ed + c0); count_launch();
  }
  if (!de) DFT_CUDA_TRY(cudaMemcpyAsync(e_out, ed, sizeof(double) * nbands, cudaMemcpyDeviceToHost, c->stream));
  DFT_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return DFTCUDA_OK;
}

// y[c][g] = (k + G)_d x[c][g]: the band times one Cartesian component of k + G.
__global__ void k_scale_kpg(const double2* __restrict__ x, const double* __restrict__ gcart, int d, long npw, long ncols,
                            double2* __restrict__ y) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < npw * ncols; i += (long)gridDim.x * blockDim.x) {
    const double q = gcart[3 * (i % npw) + d];
    y[i] = make_double2(q * x[i].x, q * x[i].y);
  }
}

// F[3 a + d] += scale sum_{p of atom a} sum_c w[c] Im(conj(Dp[p][c]) t[p][c]), one block per atom
// (rows row0[a] .. row0[a] + mt[a] - 1).
__global__ void k_nl_force(const double2* __restrict__ t, const double2* __restrict__ dp, const double* __restrict__ w,
                           const int* __restrict__ row0, const int* __restrict__ mt, int ncols, int d, double scale,
                           double* __restrict__ F) {
  const int a = blockIdx.x;
  const int p0 = row0[a], p1 = row0[a] + mt[a];
  double sum = 0.0;
  for (long i = threadIdx.x; i < (long)(p1 - p0) * ncols; i += blockDim.x) {
    const long idx = (long)p0 * ncols + i;
    const int c = (int)(idx % ncols);
    const double2 x = dp[idx], y = t[idx];
    sum += w[c] * (x.x * y.y - x.y * y.x);
  }
  __shared__ double red[256];
  red[threadIdx.x] = sum;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) F[3 * a + d] += scale * red[0];
}

// Nonlocal Hellmann-Feynman forces of the context's atoms (accumulate_atom_force_at_kpoint,
// forces/nonlocal_force.zig:283-341): with p = P psi (projector rows e^{+i(k+G).tau} phi), Dp = D p
// and t_d = P ((k+G)_d psi), F[a][d] = (2 / Omega) sum_b w_b Im sum_{j of atom a} conj(Dp_jb) t_jbd.
// Three more projection GEMMs than the nonlocal energy, in the context's precision.
extern "C" int dftcuda_nonlocal_forces(dftcuda_kctx* c, const double* vectors, size_t n, size_t nbands, const double* weights,
                                       double* forces) {
  if (!c) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "nonlocal_forces: null context");
  DeviceGuard dg(c->device);  // the context's device, whatever the caller has current
  DFT_TRY(dg.status);
  if (n != c->npw) return fail(DFTCUDA_ERR_INVALID_MATRIX_SIZE, "nonlocal_forces: n != n_pw");
  if (!forces || (nbands && (!vectors || !weights))) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "nonlocal_forces: null buffer");
  const int nproj = c->nl.nproj;
  const int natoms = c->natoms;
  std::vector<double> hf(3 * (size_t)natoms, 0.0);
  if (nproj == 0 || nbands == 0 || natoms == 0) {
    if (natoms > 0) {
      if (is_device_pointer(forces)) DFT_CUDA_TRY(cudaMemset(forces, 0, sizeof(double) * 3 * natoms));
      else std::memcpy(forces, hf.data(), sizeof(double) * 3 * natoms);
    }
    return DFTCUDA_OK;
  }
  cudaStream_t s = c->stream;
  const size_t nch = std::min<size_t>(nbands, 256);
  DFT_TRY(kctx_stage(c, nch));
  DFT_TRY(kctx_ensure_coef(c, nch));
  int* d_row = nullptr;
  double* d_w = nullptr;
  double* d_F = nullptr;
  auto cleanup = [&] {
    if (d_row) cudaFree(d_row);
    if (d_w) cudaFree(d_w);
    if (d_F) cudaFree(d_F);
  };
  if (dev_malloc(&d_row, sizeof(int) * 2 * (size_t)natoms) != cudaSuccess || dev_malloc(&d_w, sizeof(double) * nbands) != cudaSuccess ||
      dev_malloc(&d_F, sizeof(double) * 3 * (size_t)natoms) != cudaSuccess) {
    cleanup();
    return fail(DFTCUDA_ERR_OUT_OF_MEMORY, "nonlocal_forces: buffers");
  }
  int st = DFTCUDA_OK;
  auto run = [&]() -> int {
    DFT_CUDA_TRY(cudaMemcpyAsync(d_row, c->atom_row.data(), sizeof(int) * natoms, cudaMemcpyHostToDevice, s));
    DFT_CUDA_TRY(cudaMemcpyAsync(d_row + natoms, c->atom_mt.data(), sizeof(int) * natoms, cudaMemcpyHostToDevice, s));
    DFT_CUDA_TRY(cudaMemcpyAsync(d_w, weights, sizeof(double) * nbands, cudaMemcpyDefault, s));
    DFT_CUDA_TRY(cudaMemsetAsync(d_F, 0, sizeof(double) * 3 * natoms, s));
    const bool dv = is_device_pointer(vectors);
    for (size_t c0 = 0; c0 < nbands; c0 += nch) {
      const size_t nc = std::min(nch, nbands - c0);
      const double2* x = (const double2*)vectors + c0 * n;
      if (!dv) {
        DFT_CUDA_TRY(cudaMemcpyAsync(c->d_x, x, sizeof(double2) * n * nc, cudaMemcpyHostToDevice, s));
        x = c->d_x;
      }
      DFT_TRY(kctx_project(c, x, nc, s));
      const long tot = (long)nproj * nc;
      k_apply_dij<<<ceil_div(tot, 256), 256, 0, s>>>(c->d_coef, c->d_coef2, c->nl.D, c->nl.proj_off, c->nl.proj_mt, c->nl.maxm,
                                                   nproj, (int)nc); count_launch();
      for (int d = 0; d < 3; ++d) {
        k_scale_kpg<<<ceil_div((long)n * nc, 256), 256, 0, s>>>(x, c->d_gcart, d, (long)n, (long)nc, c->d_y); count_launch();
        DFT_TRY(kctx_project(c, c->d_y, nc, s));
        k_nl_force<<<natoms, 256, 0, s>>>(c->d_coef, c->d_coef2, d_w + c0, d_row, d_row + natoms, (int)nc, d, 2.0 / c->volume, d_F);
        count_launch();
      }
    }
    DFT_CUDA_TRY(cudaMemcpyAsync(hf.data(), d_F, sizeof(double) * 3 * natoms, cudaMemcpyDeviceToHost, s));
    DFT_CUDA_TRY(cudaStreamSynchronize(s));
    if (is_device_pointer(forces)) DFT_CUDA_TRY(cudaMemcpy(forces, hf.data(), sizeof(double) * 3 * natoms, cudaMemcpyHostToDevice));
    else std::memcpy(forces, hf.data(), sizeof(double) * 3 * natoms);
    return DFTCUDA_OK;
  };
  st = run();
  cleanup();
  return st;
}

// ---- nonlocal stress (stress/nonlocal_stress.zig:108-558, norm-conserving) -----------------------
// y = (k+G)_b x per column.
__global__ void k_scale_q(const double2* __restrict__ x, const double* __restrict__ kpg, int b, long npw, long ncols,
                          double2* __restrict__ y) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= npw * ncols) return;
  const double q = kpg[3 * (i % npw) + b];
  const double2 v = x[i];
  y[i] = make_double2(q * v.x, q * v.y);
}

// *out_u += scale sum_{p, n} w_n Re(conj(dp_pn) u_pn)   (accumulate_nonlocal_sigma_for_band), when u
// *out_t += sum_{p, n} w_n Re(conj(t_pn) dp_pn)          (compute_enl_for_band, times Omega), when t
// dp, u, t: [nproj][ncols] complex.  One block-sum per block, then an atomic add.
__global__ void k_stress_reduce(const double2* __restrict__ dp, const double2* __restrict__ u, const double2* __restrict__ t,
                                const double* __restrict__ w, long nproj, long ncols, double scale, double* __restrict__ out_u,
                                double* __restrict__ out_t) {
  __shared__ double red[2][8];
  double s0 = 0.0, s1 = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < nproj * ncols; i += (long)gridDim.x * blockDim.x) {
    const double wn = w[i % ncols];
    if (wn <= 0.0) continue;
    const double2 d = dp[i];
    if (u) {
      const double2 v = u[i];
      s0 += wn * (d.x * v.x + d.y * v.y);
    }
    if (t) {
      const double2 v = t[i];
      s1 += wn * (v.x * d.x + v.y * d.y);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    s0 += __shfl_xor_sync(0xffffffffu, s0, o);
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
  }
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
  if (lane == 0) {
    red[0][wp] = s0;
    red[1][wp] = s1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
      a += red[0][i];
      b += red[1][i];
    }
    if (u) atomicAdd(out_u, scale * a);
    if (t) atomicAdd(out_t, b);
  }
}

extern "C" int dftcuda_nonlocal_stress(dftcuda_kctx* c, const double* kpg, size_t n_species, const double* const* dphi,
                                       const double* vectors, size_t n, size_t nbands, const double* weights, double* sigma) {
  if (!c) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "nonlocal_stress: null context");
  DeviceGuard dg(c->device);  // the context's device, whatever the caller has current
  DFT_TRY(dg.status);
  if (n != c->npw) return fail(DFTCUDA_ERR_INVALID_MATRIX_SIZE, "nonlocal_stress: n != n_pw");
  if (!sigma || !kpg || (nbands && (!vectors || !weights))) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "nonlocal_stress: null buffer");
  double hs[9] = {0.0};
  const int nproj = c->nl.nproj;
  if (nproj == 0 || nbands == 0) {
    std::memcpy(sigma, hs, sizeof(hs));
    return DFTCUDA_OK;
  }
  if (n_species != c->species_mt.size() || !dphi) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "nonlocal_stress: one derivative table per species");
  for (size_t sp = 0; sp < n_species; ++sp)
    if (!dphi[sp]) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "nonlocal_stress: null derivative table");
  cudaStream_t s = c->stream;
  auto packed = [](int a, int b) { return a * 3 + b - (a * (a + 1)) / 2; };  // (a <= b) -> 0..5
  const size_t nch = std::min<size_t>(nbands, 256);
  DFT_TRY(kctx_stage(c, nch));
  DFT_TRY(kctx_ensure_coef(c, nch));
  // derivative projectors of all atoms, per direction a: DP_a[(atom, m)][G] = dphi_m,a(G) e^{i G . tau}
  double2* DP = nullptr;
  double* d_tab = nullptr;
  double* d_kpg = nullptr;
  double* d_w = nullptr;
  double* d_acc = nullptr;  // sigma_ab for a <= b (packed, 6), then sum_n f_n Omega E_nl,n
  double2* d_u = nullptr;
  auto cleanup = [&] {
    for (void* p : {(void*)DP, (void*)d_tab, (void*)d_kpg, (void*)d_w, (void*)d_acc, (void*)d_u})
      if (p) cudaFree(p);
  };
  size_t max_mt = 0;
  for (size_t mt : c->species_mt) max_mt = std::max(max_mt, mt);
  if (dev_malloc(&DP, sizeof(double2) * 3 * (size_t)nproj * n) != cudaSuccess ||
      dev_malloc(&d_tab, sizeof(double) * 3 * max_mt * n) != cudaSuccess || dev_malloc(&d_kpg, sizeof(double) * 3 * n) != cudaSuccess ||
      dev_malloc(&d_w, sizeof(double) * nbands) != cudaSuccess || dev_malloc(&d_acc, sizeof(double) * 7) != cudaSuccess ||
      dev_malloc(&d_u, sizeof(double2) * (size_t)nproj * nch) != cudaSuccess) {
    cleanup();
    return fail(DFTCUDA_ERR_OUT_OF_MEMORY, "nonlocal_stress: buffers");
  }
  auto run = [&]() -> int {
    DFT_CUDA_TRY(cudaMemcpyAsync(d_kpg, kpg, sizeof(double) * 3 * n, cudaMemcpyDefault, s));
    DFT_CUDA_TRY(cudaMemcpyAsync(d_w, weights, sizeof(double) * nbands, cudaMemcpyDefault, s));
    DFT_CUDA_TRY(cudaMemsetAsync(d_acc, 0, sizeof(double) * 7, s));
    for (size_t sp = 0; sp < n_species; ++sp) {
      const size_t mt = c->species_mt[sp];
      DFT_CUDA_TRY(cudaMemcpyAsync(d_tab, dphi[sp], sizeof(double) * 3 * mt * n, cudaMemcpyDefault, s));
      for (int a = 0; a < c->natoms; ++a) {
        if (c->atom_species[a] != (int)sp) continue;
        const double* tau = c->atom_pos.data() + 3 * a;
        for (int d = 0; d < 3; ++d) {
          k_build_projectors<<<ceil_div(n, 256), 256, 0, s>>>(DP + ((size_t)d * nproj + c->atom_row[a]) * n, d_tab + (size_t)d * mt * n,
                                                             (int)mt, (long)n, c->d_gcart, tau[0], tau[1], tau[2]);
          count_launch();
        }
      }
    }
    const bool dv = is_device_pointer(vectors);
    for (size_t c0 = 0; c0 < nbands; c0 += nch) {
      const size_t nc = std::min(nch, nbands - c0);
      const double2* x = (const double2*)vectors + c0 * n;
      if (!dv) {
        DFT_CUDA_TRY(cudaMemcpyAsync(c->d_x, x, sizeof(double2) * n * nc, cudaMemcpyHostToDevice, s));
        x = c->d_x;
      }
      DFT_TRY(kctx_project(c, x, nc, s));  // p
      const long tot = (long)nproj * nc;
      k_apply_dij<<<ceil_div(tot, 256), 256, 0, s>>>(c->d_coef, c->d_coef2, c->nl.D, c->nl.proj_off, c->nl.proj_mt, c->nl.maxm,
                                                   nproj, (int)nc); count_launch();  // Dp
      const unsigned rb = std::min<unsigned>(ceil_div(tot, 256), 1024);
      k_stress_reduce<<<rb, 256, 0, s>>>(c->d_coef2, nullptr, c->d_coef, d_w + c0, nproj, (long)nc, 0.0, nullptr, d_acc + 6);
      count_launch();
      for (int b = 0; b < 3; ++b) {
        k_scale_q<<<ceil_div((long)n * nc, 256), 256, 0, s>>>(x, d_kpg, b, (long)n, (long)nc, c->d_y); count_launch();
        for (int a = 0; a <= b; ++a) {
          GemmArgs g{};
          g.M = nproj; g.N = (int)nc; g.K = (int)n;
          g.A = DP + (size_t)a * nproj * n; g.lda = (long)n; g.a_kc = true; g.conj_a = false;
          g.B = c->d_y; g.ldb = (long)n; g.b_kc = true; g.conj_b = false;
          g.O = d_u; g.ldo_r = (long)nc; g.ldo_c = 1;
          g.alpha = 1.0; g.beta = 0.0;
          DFT_TRY(zgemm(g, s, c->d_gemm_ws, c->gemm_ws_elems));
          k_stress_reduce<<<rb, 256, 0, s>>>(c->d_coef2, d_u, nullptr, d_w + c0, nproj, (long)nc,
                                             -2.0 / (c->volume * c->volume), d_acc + packed(a, b), nullptr);
          count_launch();
        }
      }
    }
    double acc[7];
    DFT_CUDA_TRY(cudaMemcpyAsync(acc, d_acc, sizeof(acc), cudaMemcpyDeviceToHost, s));
    DFT_CUDA_TRY(cudaStreamSynchronize(s));
    // sigma_ab (a <= b, as the reference fills it) and the diagonal -sum_n f_n E_nl,n / Omega
    const double enl = acc[6] / c->volume;
    for (int a = 0; a < 3; ++a)
      for (int b = a; b < 3; ++b) hs[3 * a + b] = acc[packed(a, b)];
    for (int a = 0; a < 3; ++a) hs[4 * a] -= enl / c->volume;
    if (is_device_pointer(sigma)) DFT_CUDA_TRY(cudaMemcpy(sigma, hs, sizeof(hs), cudaMemcpyHostToDevice));
    else std::memcpy(sigma, hs, sizeof(hs));
    return DFTCUDA_OK;
  };
  const int st = run();
  cleanup();
  return st;
}

extern "C" int dftcuda_accumulate_density(dftcuda_kctx* c, const double* vectors, size_t n, size_t nbands,
                                          const double* weights, double* rho) {
  if (!c) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "accumulate_density: null context");
  DeviceGuard dg(c->device);  // the context's device, whatever the caller has current
  DFT_TRY(dg.status);
  if (n != c->npw) return fail(DFTCUDA_ERR_INVALID_MATRIX_SIZE, "accumulate_density: n != n_pw");
  if (nbands == 0) return DFTCUDA_OK;
  if (!vectors || !weights || !rho) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "accumulate_density: null buffer");
  // Keep only bands with a positive weight (kpoint/density.zig:104-107, 386-388).
  std::vector<double> hw(nbands);
  if (is_device_pointer(weights)) {
    DFT_CUDA_TRY(cudaMemcpyAsync(hw.data(), weights, sizeof(double) * nbands, cudaMemcpyDeviceToHost, c->stream));
    DFT_CUDA_TRY(cudaStreamSynchronize(c->stream));
  } else
    std::memcpy(hw.data(), weights, sizeof(double) * nbands);
  std::vector<size_t> keep;
  for (size_t b = 0; b < nbands; ++b)
    if (hw[b] > 0.0) keep.push_back(b);
  if (keep.empty()) return DFTCUDA_OK;
  const bool dv = is_device_pointer(vectors), dr = is_device_pointer(rho);
  DFT_TRY(kctx_stage(c, keep.size()));
  // Pack the kept bands contiguously into the staging buffer.
  const size_t colb = sizeof(double2) * n;
  for (size_t i = 0; i < keep.size(); ++i)
    DFT_CUDA_TRY(cudaMemcpyAsync(c->d_x + i * n, vectors + 2 * keep[i] * n, colb,
                                 dv ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, c->stream));
  std::vector<double> kw(keep.size());
  for (size_t i = 0; i < keep.size(); ++i) kw[i] = hw[keep[i]];
  if (keep.size() > c->w_cap) {
    if (c->d_w) cudaFree(c->d_w);
    if (dev_malloc(&c->d_w, sizeof(double) * keep.size()) != cudaSuccess) return fail(DFTCUDA_ERR_OUT_OF_MEMORY, "weights");
    c->w_cap = keep.size();
  }
  DFT_CUDA_TRY(cudaMemcpyAsync(c->d_w, kw.data(), sizeof(double) * kw.size(), cudaMemcpyHostToDevice, c->stream));
  double* rd = rho;
  if (!dr) {
    if (!c->d_rho && dev_malloc(&c->d_rho, sizeof(double) * c->N) != cudaSuccess)
      return fail(DFTCUDA_ERR_OUT_OF_MEMORY, "rho staging");
    DFT_CUDA_TRY(cudaMemcpyAsync(c->d_rho, rho, sizeof(double) * c->N, cudaMemcpyHostToDevice, c->stream));
    rd = c->d_rho;
  }
  DFT_TRY(kctx_density_dev(c, c->d_x, keep.size(), c->d_w, rd, c->stream));
  if (!dr) DFT_CUDA_TRY(cudaMemcpyAsync(rho, rd, sizeof(double) * c->N, cudaMemcpyDeviceToHost, c->stream));
  DFT_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return DFTCUDA_OK;
}

// ------------------------------------------------------------------------------------------
// Band density for callers that cannot allocate device memory (a framework that owns all device
// allocations through its own pool, or a loop that must not take the device-wide synchronisation an
// allocation can cause).  The scratch lives in a fixed array of the library's device image instead
// of a cudaMalloc'd buffer: the first kNoAllocMaxBands doubles hold the clamped weights, the rest
// holds the y-z planes of as many columns at a time as fit.  Nothing in it has to start at zero:
// each call writes every part of the scratch it later reads (k_plane_inv writes whole planes).
// The array keeps the last call's contents, and all calls share it, so calls that overlap on the GPU
// race.
// ------------------------------------------------------------------------------------------
namespace dftcuda {

constexpr size_t kNoAllocScratchBytes = DFTCUDA_NOALLOC_SCRATCH_BYTES;
constexpr size_t kNoAllocMaxBands = DFTCUDA_NOALLOC_MAX_BANDS;
constexpr size_t kNoAllocWeightBytes = kNoAllocMaxBands * sizeof(double);

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of g_noalloc_scratch for the current device, looked up once per device.  In host
// code the array's name is only a host-side stand-in, so kernels always receive this address.
static int noalloc_scratch(unsigned char** out) {
  static std::mutex mu;
  static void* addr[128] = {};
  int dev = 0;
  DFT_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 128) return fail(DFTCUDA_ERR_UNSUPPORTED, "accumulate_density_noalloc: device ordinal above 127");
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return fail(DFTCUDA_ERR_CUDA, std::string("accumulate_density_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    addr[dev] = p;
  }
  *out = static_cast<unsigned char*>(addr[dev]);
  return DFTCUDA_OK;
}

// w_out[b] = max(w[b], 0): a band with weight <= 0 contributes nothing (kpoint/density.zig:104-107).
__global__ void k_nonneg_weights(const double* __restrict__ w, double* __restrict__ w_out, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) w_out[i] = w[i] > 0.0 ? w[i] : 0.0;
}

template <typename T>
static int density_noalloc(dftcuda_kctx* c, const double2* x, size_t nbands, const double* w, double* rho,
                           unsigned char* scratch, cudaStream_t s) {
  DFT_TRY(set_smem_attrs<T>());
  double* ws = reinterpret_cast<double*>(scratch);
  cplx<T>* W = reinterpret_cast<cplx<T>*>(scratch + kNoAllocWeightBytes);
  const size_t per_col = sizeof(cplx<T>) * (size_t)c->n_act * c->P;
  const size_t cols = (kNoAllocScratchBytes - kNoAllocWeightBytes) / per_col;
  if (cols == 0)
    return fail(DFTCUDA_ERR_UNSUPPORTED, "accumulate_density_noalloc: one column's planes (" + std::to_string(per_col) +
                                             " bytes) exceed the fixed scratch of " + std::to_string(kNoAllocScratchBytes) + " bytes");
  const size_t smem_plane = sizeof(cplx<T>) * (size_t)c->P;
  if (smem_plane > kSmemMax)
    return fail(DFTCUDA_ERR_UNSUPPORTED, "accumulate_density_noalloc: a y-z plane (" + std::to_string(smem_plane) +
                                             " bytes) does not fit shared memory");
  k_nonneg_weights<<<ceil_div(nbands, 256), 256, 0, s>>>(w, ws, (int)nbands); count_launch();
  const int J = line_tile(c->nx);
  const size_t smem_x = (sizeof(cplx<T>) + sizeof(double)) * (size_t)c->nx * J;
  for (size_t c0 = 0; c0 < nbands; c0 += cols) {
    const size_t nc = std::min(cols, nbands - c0);
    dim3 gp(c->n_act, (unsigned)nc);
    k_plane_inv<T><<<gp, 512, smem_plane, s>>>(x + c0 * c->npw, (long)c->npw, W, c->n_act, c->d_plane_off, c->d_pw_idx,
                                               c->d_pw_spos, c->fy.dev, c->fz.dev, c->ny, c->nz); count_launch();
    k_xline_density<T><<<ceil_div(c->P, J), 256, smem_x, s>>>(W, c->n_act, c->d_slot_xpos, c->fx.dev, c->P, (int)nc, J,
                                                              ws + c0, 1.0 / c->volume, rho); count_launch();
  }
  DFT_CUDA_TRY(cudaGetLastError());
  return DFTCUDA_OK;
}

}  // namespace dftcuda

extern "C" int dftcuda_accumulate_density_noalloc(dftcuda_kctx* c, const double* vectors, size_t n, size_t nbands,
                                                  const double* weights, double* rho) {
  if (!c) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "accumulate_density_noalloc: null context");
  if (n != c->npw) return fail(DFTCUDA_ERR_INVALID_MATRIX_SIZE, "accumulate_density_noalloc: n != n_pw");
  if (nbands == 0) return DFTCUDA_OK;
  if (nbands > kNoAllocMaxBands)
    return fail(DFTCUDA_ERR_UNSUPPORTED, "accumulate_density_noalloc: nbands " + std::to_string(nbands) +
                                             " exceeds DFTCUDA_NOALLOC_MAX_BANDS (" + std::to_string(kNoAllocMaxBands) + ")");
  if (!vectors || !weights || !rho) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "accumulate_density_noalloc: null buffer");
  if (!is_device_pointer(vectors) || !is_device_pointer(weights) || !is_device_pointer(rho))
    return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "accumulate_density_noalloc: vectors, weights and rho must be device pointers");
  // Run on the context's device (the scratch address is per device), and after the work the caller
  // queued on the legacy default stream (where torch and plain CUDA code write these inputs).
  DeviceGuard dg(c->device);
  DFT_TRY(dg.status);
  unsigned char* scratch = nullptr;
  DFT_TRY(noalloc_scratch(&scratch));
  DFT_CUDA_TRY(cudaEventRecord(c->ev_order, cudaStreamLegacy));
  DFT_CUDA_TRY(cudaStreamWaitEvent(c->stream, c->ev_order, 0));
  const double2* x = reinterpret_cast<const double2*>(vectors);
  if (c->precision != DFTCUDA_PRECISION_FP64)
    DFT_TRY(density_noalloc<float>(c, x, nbands, weights, rho, scratch, c->stream));
  else
    DFT_TRY(density_noalloc<double>(c, x, nbands, weights, rho, scratch, c->stream));
  DFT_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return DFTCUDA_OK;
}
