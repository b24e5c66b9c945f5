// Host side of the 1D FFT plans: radix factorisation, twiddle and digit-reversal tables, and
// the standalone 3D FFT with FFTW-backend semantics (src/lib/fft/fftw_fft.zig:91-166).
#include <cmath>
#include <vector>

#include "kctx.cuh"

namespace dftcuda {

static std::vector<int> factorize(int n) {
  std::vector<int> rs;
  while (n % 4 == 0) { rs.push_back(4); n /= 4; }
  while (n % 2 == 0) { rs.push_back(2); n /= 2; }
  while (n % 3 == 0) { rs.push_back(3); n /= 3; }
  while (n % 5 == 0) { rs.push_back(5); n /= 5; }
  if (n != 1) rs.clear();
  return rs;
}

bool fft_len_supported(int n) {
  if (n < 1 || n > kMaxFftLen) return false;
  if (n == 1) return true;
  std::vector<int> rs = factorize(n);
  return !rs.empty() && (int)rs.size() <= kMaxStages;
}

// P(pos) for the DIT stage order r_0..r_{s-1}: position pos = p*(n/r_last) + rest holds input
// element p + r_last * P'(rest), P' the permutation of the first s-1 radices.
static std::vector<int> dit_perm(const std::vector<int>& rs) {
  std::vector<int> P(1, 0);
  int len = 1;
  for (size_t t = 0; t < rs.size(); ++t) {
    const int r = rs[t];
    std::vector<int> Q(len * r);
    for (int p = 0; p < r; ++p)
      for (int k = 0; k < len; ++k) Q[p * len + k] = p + r * P[k];
    P.swap(Q);
    len *= r;
  }
  return P;
}

int Fft1dPlan::create(int n) {
  if (!fft_len_supported(n)) return fail(DFTCUDA_ERR_UNSUPPORTED, "FFT length " + std::to_string(n) + " is not 2,3,5-smooth or exceeds 128");
  radices = (n == 1) ? std::vector<int>{} : factorize(n);
  dev.n = n;
  dev.nstages = (int)radices.size();
  std::vector<double2> tw;
  int m = 1;
  for (int t = 0; t < dev.nstages; ++t) {
    const int r = radices[t];
    const int L = m * r;
    dev.radix[t] = r;
    dev.m[t] = m;
    dev.tw_off[t] = (int)tw.size();
    for (int k = 0; k < m; ++k)
      for (int p = 1; p < r; ++p) {
        // reduce p*k modulo L before scaling so the angle keeps full precision
        const long pk = (long)p * k % L;
        const double ang = 2.0 * M_PI * (double)pk / (double)L;
        tw.push_back(make_double2(std::cos(ang), std::sin(ang)));
      }
    m = L;
  }
  if (tw.empty()) tw.push_back(make_double2(1.0, 0.0));
  std::vector<int> P = dit_perm(radices);
  pinv.assign(n, 0);
  for (int pos = 0; pos < n; ++pos) pinv[P[pos]] = pos;
  std::vector<float2> tw32(tw.size());
  for (size_t i = 0; i < tw.size(); ++i) tw32[i] = make_float2((float)tw[i].x, (float)tw[i].y);
  const size_t b64 = tw.size() * sizeof(double2), b32 = tw.size() * sizeof(float2), bp = n * sizeof(int);
  DFT_CUDA_TRY(dev_malloc(&d_buf, b64 + b32 + bp + 64));
  char* base = (char*)d_buf;
  // A pageable-host cudaMemcpy may return before its DMA lands; synchronise the device before the
  // tables are used.
  DFT_CUDA_TRY(cudaMemcpy(base, tw.data(), b64, cudaMemcpyHostToDevice));
  DFT_CUDA_TRY(cudaMemcpy(base + b64, tw32.data(), b32, cudaMemcpyHostToDevice));
  DFT_CUDA_TRY(cudaMemcpy(base + b64 + b32, pinv.data(), bp, cudaMemcpyHostToDevice));
  DFT_CUDA_TRY(cudaDeviceSynchronize());
  dev.tw64 = (const double2*)base;
  dev.tw32 = (const float2*)(base + b64);
  dev.pinv = (const int*)(base + b64 + b32);
  return DFTCUDA_OK;
}

void Fft1dPlan::destroy() {
  if (d_buf) cudaFree(d_buf);
  d_buf = nullptr;
}

// ------------------------------------------------------------------------------------------
// Standalone 3D FFT: three axis passes over the natural x-fastest box.  Each CTA stages a tile of
// `lines` pencils (consecutive along the fastest other axis, so global accesses are coalesced)
// in shared memory, permutes on load (DIT) or on store (DIF), and transforms them.
// ------------------------------------------------------------------------------------------

// Pencils along an axis of length n with element stride es; lines are indexed by (outer, inner)
// where inner runs over `ninner` consecutive addresses (stride 1) and outer over blocks of stride os.
template <bool DIT>
__global__ void k_fft_axis(double2* __restrict__ data, Fft1d p, int es, int ninner, int nouter, long os, double sg,
                           double scale) {
  extern __shared__ double2 sm[];
  const int n = p.n;
  const int lines = blockDim.y;  // pencils per CTA along the inner direction
  const int inner0 = blockIdx.x * lines;
  const int outer = blockIdx.y;
  const int nl = min(lines, ninner - inner0);
  if (nl <= 0) return;
  double2* g = data + (long)outer * os + inner0;
  // tile layout: sm[pos * lines + line]  (line fastest)
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const int nthr = blockDim.x * blockDim.y;
  for (int i = tid; i < n * lines; i += nthr) {
    const int e = i / lines, l = i - e * lines;
    double2 v = make_double2(0.0, 0.0);
    if (l < nl) v = g[(long)e * es + l];
    sm[(DIT ? p.pinv[e] : e) * lines + l] = v;
  }
  __syncthreads();
  // fft_lines uses threadIdx.x/blockDim.x; flatten by running it with a 1D view
  {
    using C = double2;
    if (DIT) {
      for (int t = 0; t < p.nstages; ++t) {
        const int r = p.radix[t], m = p.m[t], L = m * r, nb = n / r, total = nb * lines, two = p.tw_off[t];
        for (int idx = tid; idx < total; idx += nthr) {
          const int b = idx / lines, line = idx - b * lines;
          const int blk = b / m, k = b - blk * m;
          C* base = sm + (blk * L + k) * lines + line;
          const int step = m * lines;
          C x[5];
#pragma unroll
          for (int q = 0; q < 5; ++q)
            if (q < r) x[q] = base[q * step];
          if (k != 0) {
#pragma unroll
            for (int q = 1; q < 5; ++q)
              if (q < r) {
                C w = __ldg(p.tw64 + two + k * (r - 1) + (q - 1));
                w.y *= sg;
                x[q] = cmul(x[q], w);
              }
          }
          dft_small<double>(x, r, sg);
#pragma unroll
          for (int q = 0; q < 5; ++q)
            if (q < r) base[q * step] = x[q];
        }
        __syncthreads();
      }
    } else {
      for (int t = p.nstages - 1; t >= 0; --t) {
        const int r = p.radix[t], m = p.m[t], L = m * r, nb = n / r, total = nb * lines, two = p.tw_off[t];
        for (int idx = tid; idx < total; idx += nthr) {
          const int b = idx / lines, line = idx - b * lines;
          const int blk = b / m, k = b - blk * m;
          C* base = sm + (blk * L + k) * lines + line;
          const int step = m * lines;
          C x[5];
#pragma unroll
          for (int q = 0; q < 5; ++q)
            if (q < r) x[q] = base[q * step];
          dft_small<double>(x, r, sg);
          if (k != 0) {
#pragma unroll
            for (int q = 1; q < 5; ++q)
              if (q < r) {
                C w = __ldg(p.tw64 + two + k * (r - 1) + (q - 1));
                w.y *= sg;
                x[q] = cmul(x[q], w);
              }
          }
#pragma unroll
          for (int q = 0; q < 5; ++q)
            if (q < r) base[q * step] = x[q];
        }
        __syncthreads();
      }
    }
  }
  for (int i = tid; i < n * lines; i += nthr) {
    const int e = i / lines, l = i - e * lines;
    if (l < nl) {
      double2 v = sm[(DIT ? e : p.pinv[e]) * lines + l];
      g[(long)e * es + l] = cscale(v, scale);
    }
  }
}

}  // namespace dftcuda

using namespace dftcuda;

struct dftcuda_fft_plan {
  int nx, ny, nz;
  Fft1dPlan px, py, pz;
  double2* staging = nullptr;
  cudaStream_t stream = nullptr;
};

static int run_axis(dftcuda_fft_plan* /*pl*/, double2* d, const Fft1d& p, int es, int ninner, int nouter, long os, int dir,
                    double scale, cudaStream_t stream) {
  const int lines = ninner >= 16 ? 16 : ninner;
  dim3 block(16, lines);
  dim3 grid(ceil_div(ninner, lines), nouter);
  const size_t smem = (size_t)p.n * lines * sizeof(double2);
  if (dir > 0)
    k_fft_axis<true><<<grid, block, smem, stream>>>(d, p, es, ninner, nouter, os, +1.0, scale);
  else
    k_fft_axis<false><<<grid, block, smem, stream>>>(d, p, es, ninner, nouter, os, -1.0, scale);
  count_launch();
  DFT_CUDA_TRY(cudaGetLastError());
  return DFTCUDA_OK;
}

extern "C" int dftcuda_fft_plan_create(dftcuda_fft_plan** out, int nx, int ny, int nz) {
  if (!out || nx <= 0 || ny <= 0 || nz <= 0) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "fft_plan_create: bad arguments");
  *out = nullptr;
  auto* pl = new dftcuda_fft_plan();
  pl->nx = nx; pl->ny = ny; pl->nz = nz;
  int s;
  if ((s = pl->px.create(nx)) || (s = pl->py.create(ny)) || (s = pl->pz.create(nz))) {
    pl->px.destroy(); pl->py.destroy(); pl->pz.destroy();
    delete pl;
    return s;
  }
  if (cudaStreamCreateWithFlags(&pl->stream, cudaStreamDefault) != cudaSuccess) {
    delete pl;
    return fail(DFTCUDA_ERR_CUDA, "fft_plan_create: stream");
  }
  *out = pl;
  return DFTCUDA_OK;
}

extern "C" int dftcuda_fft_plan_destroy(dftcuda_fft_plan* pl) {
  if (!pl) return DFTCUDA_OK;
  pl->px.destroy(); pl->py.destroy(); pl->pz.destroy();
  if (pl->staging) cudaFree(pl->staging);
  if (pl->stream) cudaStreamDestroy(pl->stream);
  delete pl;
  return DFTCUDA_OK;
}

// The three axis passes on device data, queued on stream s (no synchronisation): z, then y (each
// over x-contiguous lines), then x; the inverse carries the 1/N.
int dftcuda::fft3d_on_stream(dftcuda_fft_plan* pl, double2* d, int direction, cudaStream_t s) {
  const long nx = pl->nx, ny = pl->ny, nz = pl->nz, N = nx * ny * nz;
  const double inv = direction > 0 ? 1.0 / (double)N : 1.0;
  DFT_TRY(run_axis(pl, d, pl->pz.dev, (int)(nx * ny), (int)nx, (int)ny, nx, direction, 1.0, s));
  DFT_TRY(run_axis(pl, d, pl->py.dev, (int)nx, (int)nx, (int)nz, nx * ny, direction, 1.0, s));
  DFT_TRY(run_axis(pl, d, pl->px.dev, 1, 1, (int)(ny * nz), nx, direction, inv, s));
  return DFTCUDA_OK;
}

extern "C" int dftcuda_fft3d(dftcuda_fft_plan* pl, double* data, int direction) {
  if (!pl || !data || (direction != 1 && direction != -1)) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "fft3d: bad arguments");
  const long nx = pl->nx, ny = pl->ny, nz = pl->nz, N = nx * ny * nz;
  const bool dev = is_device_pointer(data);
  double2* d = (double2*)data;
  if (!dev) {
    if (!pl->staging) DFT_CUDA_TRY(dev_malloc(&pl->staging, N * sizeof(double2)));
    d = pl->staging;
    DFT_CUDA_TRY(cudaMemcpyAsync(d, data, N * sizeof(double2), cudaMemcpyHostToDevice, pl->stream));
  }
  DFT_TRY(dftcuda::fft3d_on_stream(pl, d, direction, pl->stream));
  if (!dev) DFT_CUDA_TRY(cudaMemcpyAsync(data, d, N * sizeof(double2), cudaMemcpyDeviceToHost, pl->stream));
  DFT_CUDA_TRY(cudaStreamSynchronize(pl->stream));
  return DFTCUDA_OK;
}
