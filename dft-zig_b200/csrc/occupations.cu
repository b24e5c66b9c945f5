// Fermi level, smearing occupations and the entropy sum of an eigenvalue table, in FP64 on the device:
// find_fermi_level_spin, smearing_occ and smearing_entropy (src/features/scf/fermi_level.zig:7-124).
//
// One CTA does the whole search.  Each trial chemical potential needs the electron count
// N(mu) = spin * sum_k w_k sum_b f((e_kb - mu) / sigma), a block reduction over the table (a few
// thousand entries at most for the configurations here), so the reference's schedule runs as written:
// the bracket [min e - pad, max e + pad] with pad = max(10 sigma, 1e-3), doubled up to 12 times
// until N(low) <= nelec <= N(high), then up to 80 bisections that stop once |N(mu) - nelec| < 1e-8.
// The table stays in shared memory when it fits, else it is re-read from global memory (L1/L2).
#include <cmath>
#include <string>
#include <vector>

#include "kctx.cuh"

namespace dftcuda {

namespace {

constexpr int kOccThreads = 512;
constexpr int kOccSmemEntries = 6000;  // eigenvalues kept in shared memory (48,000 bytes)

// smearing_occ (fermi_level.zig:7-11): Fermi-Dirac, or a step at mu when sigma <= 0.
__device__ __forceinline__ double occ_of(double e, double mu, double sigma) {
  if (sigma <= 0.0) return e <= mu ? 1.0 : 0.0;
  return 1.0 / (1.0 + exp((e - mu) / sigma));
}

// smearing_entropy (fermi_level.zig:13-19).
__device__ __forceinline__ double entropy_of(double f) {
  const double eps = 1e-12;
  if (f <= eps || f >= 1.0 - eps) return 0.0;
  return -(f * log(f) + (1.0 - f) * log(1.0 - f));
}

__device__ double block_sum(double v, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
  for (int i = 0; i < kOccThreads / 32; ++i) t += red[i];
  return t;
}

__device__ double block_min(double v, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double t = red[0];
  for (int i = 1; i < kOccThreads / 32; ++i) t = fmin(t, red[i]);
  return t;
}

struct Table {
  const double* e;      // [nk * nb], row per k-point
  const double* w;      // [nk]
  const double* s_e;    // shared copy of e (or e itself)
  int nk, nb;
  double spin;
  __device__ double weight(int i) const { return spin * w[i / nb]; }
};

__device__ double electron_count(const Table& t, double mu, double sigma, double* red) {
  double c = 0.0;
  const int n = t.nk * t.nb;
  for (int i = threadIdx.x; i < n; i += blockDim.x) c += t.weight(i) * occ_of(t.s_e[i], mu, sigma);
  return block_sum(c, red);
}

__global__ void __launch_bounds__(kOccThreads) k_fermi(const double* __restrict__ e, const double* __restrict__ w, int nk,
                                                       int nb, double nelec, double sigma, double spin,
                                                       double* __restrict__ mu_out, double* __restrict__ occ,
                                                       double* __restrict__ sums) {
  __shared__ double red[kOccThreads / 32];
  extern __shared__ double s_tab[];
  const int n = nk * nb;
  const bool in_smem = n <= kOccSmemEntries;
  if (in_smem)
    for (int i = threadIdx.x; i < n; i += blockDim.x) s_tab[i] = e[i];
  __syncthreads();
  Table t{e, w, in_smem ? s_tab : e, nk, nb, spin};
  double lo = INFINITY, hi = -INFINITY;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    lo = fmin(lo, t.s_e[i]);
    hi = fmax(hi, t.s_e[i]);
  }
  const double min_e = block_min(lo, red);
  const double max_e = -block_min(-hi, red);
  double pad = fmax(10.0 * sigma, 1e-3);
  double low = min_e - pad, high = max_e + pad;
  double c_low = electron_count(t, low, sigma, red), c_high = electron_count(t, high, sigma, red);
  for (int expand = 0; (c_low > nelec || c_high < nelec) && expand < 12; ++expand) {
    pad *= 2.0;
    low = min_e - pad;
    high = max_e + pad;
    c_low = electron_count(t, low, sigma, red);
    c_high = electron_count(t, high, sigma, red);
  }
  double left = low, right = high, mu = 0.5 * (left + right);
  bool found = false;
  for (int it = 0; it < 80; ++it) {
    const double mid = 0.5 * (left + right);
    const double c = electron_count(t, mid, sigma, red);
    if (fabs(c - nelec) < 1e-8) {
      mu = mid;
      found = true;
      break;
    }
    if (c > nelec)
      right = mid;
    else
      left = mid;
  }
  if (!found) mu = 0.5 * (left + right);
  double eb = 0.0, ent = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double ei = t.s_e[i];
    const double f = occ_of(ei, mu, sigma);
    if (occ) occ[i] = f;
    eb += t.weight(i) * f * ei;
    ent += t.weight(i) * entropy_of(f);
  }
  eb = block_sum(eb, red);
  ent = block_sum(ent, red);
  if (threadIdx.x == 0) {
    *mu_out = mu;
    if (sums) {
      sums[0] = eb;
      sums[1] = ent;
    }
  }
}

}  // namespace

}  // namespace dftcuda

using namespace dftcuda;

extern "C" int dftcuda_fermi_occupations(size_t nk, size_t nbands, const double* values, const double* kweights, double nelec,
                                         double sigma, double spin_factor, double* mu_out, double* occ, double* sums) {
  if (nk == 0 || nbands == 0) return fail(DFTCUDA_ERR_INVALID_MATRIX_SIZE, "fermi_occupations: empty eigenvalue table");
  if (!values || !kweights || !mu_out) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "fermi_occupations: null argument");
  if (nk * nbands > (size_t)1 << 26) return fail(DFTCUDA_ERR_INVALID_MATRIX_SIZE, "fermi_occupations: table too large");
  const size_t n = nk * nbands;
  cudaStream_t s = nullptr;
  // a blocking stream: ordered after the caller's work on the legacy default stream
  DFT_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamDefault));
  struct Guard {
    cudaStream_t s;
    void* p = nullptr;
    ~Guard() {
      if (p) cudaFree(p);
      cudaStreamDestroy(s);
    }
  } g{s};
  // device staging: values, weights, occupations, mu and the two sums
  const size_t bytes = sizeof(double) * (2 * n + nk + 3);
  DFT_CUDA_TRY(dev_malloc(&g.p, bytes));
  double* d_e = static_cast<double*>(g.p);
  double* d_w = d_e + n;
  double* d_occ = d_w + nk;
  double* d_res = d_occ + n;  // mu, band sum, entropy sum
  auto kind = [](const void* p, bool to_dev) {
    const bool dev = is_device_pointer(p);
    return to_dev ? (dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice) : (dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost);
  };
  DFT_CUDA_TRY(cudaMemcpyAsync(d_e, values, sizeof(double) * n, kind(values, true), s));
  DFT_CUDA_TRY(cudaMemcpyAsync(d_w, kweights, sizeof(double) * nk, kind(kweights, true), s));
  const size_t smem = n <= (size_t)kOccSmemEntries ? sizeof(double) * n : 0;
  k_fermi<<<1, kOccThreads, smem, s>>>(d_e, d_w, (int)nk, (int)nbands, nelec, sigma, spin_factor, d_res, d_occ, d_res + 1);
  count_launch();
  DFT_CUDA_TRY(cudaGetLastError());
  DFT_CUDA_TRY(cudaMemcpyAsync(mu_out, d_res, sizeof(double), kind(mu_out, false), s));
  if (occ) DFT_CUDA_TRY(cudaMemcpyAsync(occ, d_occ, sizeof(double) * n, kind(occ, false), s));
  if (sums) DFT_CUDA_TRY(cudaMemcpyAsync(sums, d_res + 1, sizeof(double) * 2, kind(sums, false), s));
  DFT_CUDA_TRY(cudaStreamSynchronize(s));
  return DFTCUDA_OK;
}
