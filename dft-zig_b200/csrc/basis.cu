// Plane-wave basis and projector tables on the device.
//
// dftcuda_plane_wave_basis  plane_wave.generate (features/plane_wave/basis.zig:26-74): every Miller
//                           triple (h, k, l) of the box [-n, n]^3, n = ceil(sqrt(ecut) / min |b_i|) + 1,
//                           in the reference's loop order (h outer, l inner), kept when
//                           |k + G|^2 <= ecut.  The arithmetic is the reference's, term by term with
//                           round-to-nearest multiplies and adds (no contraction into FMAs), so the
//                           kept set, the order and every kinetic energy equal a host evaluation
//                           bit for bit.  Order-preserving compaction: per-block counts, one scan of
//                           the block totals, then each block writes its kept entries.
// dftcuda_projector_phi     fill_nonlocal_phi (scf/nonlocal_context.zig:524-549):
//                           phi_m(q) = 4 pi R(|q|) Y_lm(q) for m = -l..l, R from the uniform radial
//                           table by RadialTable.eval (pseudopotential/nonlocal.zig:250-300: linear
//                           interpolation, R(0) at q <= 0, the last value in the last interval, 0 at
//                           q >= g_max), Y_lm the real harmonics of nonlocal.zig:152-241 (l <= 4).
#include <cmath>
#include <map>
#include <mutex>
#include <vector>

#include "common.cuh"

namespace dftcuda {
namespace {

constexpr int kBasisThreads = 256;
constexpr int kBasisPerThread = 4;
constexpr int kBasisTile = kBasisThreads * kBasisPerThread;  // candidates per block

struct BasisArgs {
  double b[9];  // rows b1, b2, b3
  double k[3];
  double ecut;
  int n;        // box half-width
  long ncand;   // (2n + 1)^3
};

// G = (b1 h + b2 k) + b3 l and |k + G|^2 = (qx qx + qy qy) + qz qz, each operation rounded once.
__device__ __forceinline__ bool candidate(const BasisArgs& a, long c, int* hkl, double* g, double* q, double* kin) {
  const int D = 2 * a.n + 1;
  const int h = (int)(c / ((long)D * D)) - a.n;
  const int kk = (int)((c / D) % D) - a.n;
  const int l = (int)(c % D) - a.n;
  const double fh = (double)h, fk = (double)kk, fl = (double)l;
  double qq = 0.0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double gd = __dadd_rn(__dadd_rn(__dmul_rn(a.b[d], fh), __dmul_rn(a.b[3 + d], fk)), __dmul_rn(a.b[6 + d], fl));
    const double qd = __dadd_rn(a.k[d], gd);
    g[d] = gd;
    q[d] = qd;
    qq = d == 0 ? __dmul_rn(qd, qd) : __dadd_rn(qq, __dmul_rn(qd, qd));
  }
  hkl[0] = h;
  hkl[1] = kk;
  hkl[2] = l;
  *kin = qq;
  return qq <= a.ecut;
}

__global__ void __launch_bounds__(kBasisThreads) k_basis_count(BasisArgs a, int* block_count) {
  __shared__ int red[kBasisThreads / 32];
  const long base = (long)blockIdx.x * kBasisTile;
  int cnt = 0;
  for (int j = 0; j < kBasisPerThread; ++j) {
    const long c = base + (long)j * kBasisThreads + threadIdx.x;
    if (c < a.ncand) {
      int hkl[3];
      double g[3], q[3], kin;
      cnt += candidate(a, c, hkl, g, q, &kin) ? 1 : 0;
    }
  }
  for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = cnt;
  __syncthreads();
  if (threadIdx.x == 0) {
    int s = 0;
    for (int w = 0; w < kBasisThreads / 32; ++w) s += red[w];
    block_count[blockIdx.x] = s;
  }
}

// Exclusive scan of the block counts in one block (nblocks is small: a few thousand at most).
__global__ void __launch_bounds__(1024) k_basis_scan(int* block_count, int nblocks, long* total) {
  __shared__ int part[1024];
  const int per = (nblocks + 1023) / 1024;
  const int b0 = threadIdx.x * per, b1 = min(nblocks, b0 + per);
  int s = 0;
  for (int b = b0; b < b1; ++b) s += block_count[b];
  part[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    int run = 0;
    for (int t = 0; t < 1024; ++t) {
      const int v = part[t];
      part[t] = run;
      run += v;
    }
    *total = run;
  }
  __syncthreads();
  int run = part[threadIdx.x];
  for (int b = b0; b < b1; ++b) {
    const int v = block_count[b];
    block_count[b] = run;
    run += v;
  }
}

// Each block walks its candidates in reference order: for j, the 256 threads hold 256 consecutive
// candidates; a block-wide scan of their flags gives each kept candidate its output slot.
__global__ void __launch_bounds__(kBasisThreads) k_basis_write(BasisArgs a, const int* block_off, long cap, int* hkl_out,
                                                                double* g_out, double* q_out, double* kin_out) {
  __shared__ int wsum[kBasisThreads / 32];
  __shared__ int carry;
  const long base = (long)blockIdx.x * kBasisTile;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = block_off[blockIdx.x];
  __syncthreads();
  for (int j = 0; j < kBasisPerThread; ++j) {
    const long c = base + (long)j * kBasisThreads + threadIdx.x;
    int hkl[3];
    double g[3], q[3], kin = 0.0;
    const bool keep = c < a.ncand && candidate(a, c, hkl, g, q, &kin);
    const unsigned bal = __ballot_sync(0xffffffffu, keep);
    const int before = __popc(bal & ((1u << lane) - 1u));
    if (lane == 0) wsum[warp] = __popc(bal);
    __syncthreads();
    int off = carry;
    for (int w = 0; w < warp; ++w) off += wsum[w];
    const long slot = (long)off + before;
    if (keep && slot < cap) {
      hkl_out[3 * slot] = hkl[0];
      hkl_out[3 * slot + 1] = hkl[1];
      hkl_out[3 * slot + 2] = hkl[2];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        g_out[3 * slot + d] = g[d];
        q_out[3 * slot + d] = q[d];
      }
      kin_out[slot] = kin;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int s = 0;
      for (int w = 0; w < kBasisThreads / 32; ++w) s += wsum[w];
      carry += s;
    }
    __syncthreads();
  }
}

// Real spherical harmonics (nonlocal.zig:152-241); 1/sqrt(4 pi) for l = 0 at the origin, 0 otherwise.
__device__ double real_ylm(int l, int m, double x, double y, double z) {
  const double r2 = x * x + y * y + z * z;
  const double pi = 3.14159265358979323846;
  if (r2 < 1e-30) return l == 0 ? 1.0 / sqrt(4.0 * pi) : 0.0;
  const double ir = 1.0 / sqrt(r2);
  const double nx = x * ir, ny = y * ir, nz = z * ir;
  switch (l) {
    case 0: return m == 0 ? 1.0 / sqrt(4.0 * pi) : 0.0;
    case 1: {
      const double c = sqrt(3.0 / (4.0 * pi));
      return m == -1 ? c * ny : m == 0 ? c * nz : m == 1 ? c * nx : 0.0;
    }
    case 2: {
      const double c0 = sqrt(5.0 / (16.0 * pi)), c1 = sqrt(15.0 / (4.0 * pi)), c2 = sqrt(15.0 / (16.0 * pi));
      switch (m) {
        case -2: return c2 * 2.0 * nx * ny;
        case -1: return c1 * ny * nz;
        case 0: return c0 * (3.0 * nz * nz - 1.0);
        case 1: return c1 * nx * nz;
        case 2: return c2 * (nx * nx - ny * ny);
        default: return 0.0;
      }
    }
    case 3:
      switch (m) {
        case -3: return sqrt(35.0 / (32.0 * pi)) * (3.0 * nx * nx - ny * ny) * ny;
        case -2: return sqrt(105.0 / (4.0 * pi)) * nx * ny * nz;
        case -1: return sqrt(21.0 / (32.0 * pi)) * ny * (5.0 * nz * nz - 1.0);
        case 0: return sqrt(7.0 / (16.0 * pi)) * (5.0 * nz * nz * nz - 3.0 * nz);
        case 1: return sqrt(21.0 / (32.0 * pi)) * nx * (5.0 * nz * nz - 1.0);
        case 2: return sqrt(105.0 / (16.0 * pi)) * (nx * nx - ny * ny) * nz;
        case 3: return sqrt(35.0 / (32.0 * pi)) * (nx * nx - 3.0 * ny * ny) * nx;
        default: return 0.0;
      }
    case 4: {
      const double x2 = nx * nx, y2 = ny * ny, z2 = nz * nz;
      switch (m) {
        case -4: return sqrt(315.0 / (256.0 * pi)) * 4.0 * nx * ny * (x2 - y2);
        case -3: return sqrt(315.0 / (32.0 * pi)) * ny * nz * (3.0 * x2 - y2);
        case -2: return sqrt(45.0 / (64.0 * pi)) * 2.0 * nx * ny * (7.0 * z2 - 1.0);
        case -1: return sqrt(45.0 / (32.0 * pi)) * ny * nz * (7.0 * z2 - 3.0);
        case 0: return sqrt(9.0 / (256.0 * pi)) * (35.0 * z2 * z2 - 30.0 * z2 + 3.0);
        case 1: return sqrt(45.0 / (32.0 * pi)) * nx * nz * (7.0 * z2 - 3.0);
        case 2: return sqrt(45.0 / (64.0 * pi)) * (x2 - y2) * (7.0 * z2 - 1.0);
        case 3: return sqrt(315.0 / (32.0 * pi)) * nx * nz * (x2 - 3.0 * y2);
        case 4: return sqrt(315.0 / (256.0 * pi)) * (x2 * x2 - 6.0 * x2 * y2 + y2 * y2);
        default: return 0.0;
      }
    }
    default: return 0.0;
  }
}

// RadialTable.eval: linear interpolation on the uniform table of nq values over [0, gmax].
__device__ double radial_eval(const double* __restrict__ tab, int nq, double gmax, double g) {
  const double dq = gmax / (double)(nq - 1);
  if (g <= 0.0) return tab[0];
  if (g >= gmax) return 0.0;
  const double x = g / dq;
  const long i = (long)floor(x);
  const double t = x - (double)i;
  if (i + 1 >= nq) return tab[nq - 1];
  return tab[i] * (1.0 - t) + tab[i + 1] * t;
}

__global__ void k_projector_phi(int l, const double* __restrict__ tab, int nq, double gmax, const double* __restrict__ kpg, long n,
                                double* __restrict__ phi) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double x = kpg[3 * i], y = kpg[3 * i + 1], z = kpg[3 * i + 2];
  const double g = sqrt(x * x + y * y + z * z);
  const double rad = 4.0 * 3.14159265358979323846 * radial_eval(tab, nq, gmax, g);
  for (int mi = 0; mi <= 2 * l; ++mi) phi[(long)mi * n + i] = rad * real_ylm(l, mi - l, x, y, z);
}

// One stream and one growable device buffer per device, kept for the life of the process: a
// per-k-point setup calls these entry points a few times for each of hundreds of k-points, and a
// stream plus allocations per call cost more than the kernels.
struct SetupEngine {
  std::mutex mu;
  cudaStream_t s = nullptr;
  char* buf = nullptr;
  size_t cap = 0;
  int ensure(size_t bytes) {
    if (!s && cudaStreamCreateWithFlags(&s, cudaStreamDefault) != cudaSuccess) {
      s = nullptr;
      return fail(DFTCUDA_ERR_CUDA, "setup engine: stream creation failed");
    }
    if (bytes <= cap) return DFTCUDA_OK;
    cudaStreamSynchronize(s);
    if (buf) cudaFree(buf);
    buf = nullptr;
    cap = 0;
    if (dev_malloc(&buf, bytes) != cudaSuccess) return fail(DFTCUDA_ERR_OUT_OF_MEMORY, "setup engine: buffer");
    cap = bytes;
    return DFTCUDA_OK;
  }
};

SetupEngine* setup_engine() {
  static std::mutex map_mu;
  static std::map<int, SetupEngine*> engines;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  std::lock_guard<std::mutex> lock(map_mu);
  SetupEngine*& e = engines[dev];
  if (!e) e = new SetupEngine();  // lives as long as the process
  return e;
}

}  // namespace
}  // namespace dftcuda

using namespace dftcuda;

extern "C" int dftcuda_plane_wave_basis(const double* recip, double ecut_ry, const double* k_cart, size_t capacity, int32_t* hkl,
                                        double* gcart, double* kpg, double* kinetic, size_t* n_out) {
  if (!recip || !k_cart || !n_out || !(ecut_ry > 0.0))
    return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "plane_wave_basis: null argument or ecut <= 0");
  if (capacity > 0 && (!hkl || !gcart || !kpg || !kinetic))
    return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "plane_wave_basis: null output array");
  BasisArgs a{};
  double min_b = INFINITY;
  for (int r = 0; r < 3; ++r) {
    double s = 0.0;
    for (int d = 0; d < 3; ++d) {
      a.b[3 * r + d] = recip[3 * r + d];
      s += recip[3 * r + d] * recip[3 * r + d];
    }
    min_b = std::fmin(min_b, std::sqrt(s));
  }
  if (!(min_b > 0.0)) return fail(DFTCUDA_ERR_INVALID_GRID, "plane_wave_basis: degenerate reciprocal lattice");
  for (int d = 0; d < 3; ++d) a.k[d] = k_cart[d];
  a.ecut = ecut_ry;
  const double nmax = std::ceil(std::sqrt(ecut_ry) / min_b) + 1.0;
  if (nmax > 600.0) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "plane_wave_basis: Miller box above 1201^3");
  a.n = (int)nmax;
  const long D = 2L * a.n + 1;
  a.ncand = D * D * D;
  const int nblocks = (int)((a.ncand + kBasisTile - 1) / kBasisTile);
  SetupEngine* en = setup_engine();
  if (!en) return fail(DFTCUDA_ERR_CUDA, "plane_wave_basis: no device");
  std::lock_guard<std::mutex> lock(en->mu);
  // buffer: block counts, the total, then (when the outputs are host arrays) the staged basis
  const size_t off_total = ((sizeof(int) * (size_t)nblocks + 15) / 16) * 16;
  const size_t off_out = off_total + 16;
  DFT_TRY(en->ensure(off_out));
  cudaStream_t s = en->s;
  int* dcount = reinterpret_cast<int*>(en->buf);
  long* dtotal = reinterpret_cast<long*>(en->buf + off_total);
  k_basis_count<<<nblocks, kBasisThreads, 0, s>>>(a, dcount);
  count_launch();
  k_basis_scan<<<1, 1024, 0, s>>>(dcount, nblocks, dtotal);
  count_launch();
  long total = 0;
  DFT_CUDA_TRY(cudaMemcpyAsync(&total, dtotal, sizeof(long), cudaMemcpyDeviceToHost, s));
  DFT_CUDA_TRY(cudaStreamSynchronize(s));
  *n_out = (size_t)total;
  if (capacity == 0) return DFTCUDA_OK;  // size query
  if ((size_t)total > capacity) return fail(DFTCUDA_ERR_INVALID_MATRIX_SIZE, "plane_wave_basis: capacity below the basis size");
  // outputs: straight into device arrays, else through the engine's buffer
  const bool dev = is_device_pointer(hkl) && is_device_pointer(gcart) && is_device_pointer(kpg) && is_device_pointer(kinetic);
  int* oh = hkl;
  double *og = gcart, *oq = kpg, *ok = kinetic;
  const size_t nb_h = sizeof(int32_t) * 3 * total, nb_v = sizeof(double) * 3 * total, nb_k = sizeof(double) * total;
  if (!dev) {
    DFT_TRY(en->ensure(off_out + 2 * nb_v + nb_k + nb_h + 64));
    dcount = reinterpret_cast<int*>(en->buf);  // the buffer may have moved; the counts are recomputed below
    char* o = en->buf + off_out;
    og = reinterpret_cast<double*>(o);
    oq = reinterpret_cast<double*>(o + nb_v);
    ok = reinterpret_cast<double*>(o + 2 * nb_v);
    oh = reinterpret_cast<int*>(o + 2 * nb_v + nb_k);
    k_basis_count<<<nblocks, kBasisThreads, 0, s>>>(a, dcount);
    count_launch();
    k_basis_scan<<<1, 1024, 0, s>>>(dcount, nblocks, reinterpret_cast<long*>(en->buf + off_total));
    count_launch();
  }
  k_basis_write<<<nblocks, kBasisThreads, 0, s>>>(a, dcount, total, oh, og, oq, ok);
  count_launch();
  DFT_CUDA_TRY(cudaGetLastError());
  if (!dev) {
    DFT_CUDA_TRY(cudaMemcpyAsync(hkl, oh, nb_h, cudaMemcpyDeviceToHost, s));
    DFT_CUDA_TRY(cudaMemcpyAsync(gcart, og, nb_v, cudaMemcpyDeviceToHost, s));
    DFT_CUDA_TRY(cudaMemcpyAsync(kpg, oq, nb_v, cudaMemcpyDeviceToHost, s));
    DFT_CUDA_TRY(cudaMemcpyAsync(kinetic, ok, nb_k, cudaMemcpyDeviceToHost, s));
  }
  DFT_CUDA_TRY(cudaStreamSynchronize(s));
  return DFTCUDA_OK;
}

extern "C" int dftcuda_projector_phi(int l, size_t nq, double gmax, const double* table, size_t n, const double* kpg, double* phi) {
  if (l < 0 || l > 4) return fail(DFTCUDA_ERR_UNSUPPORTED, "projector_phi: l outside 0..4");
  if (nq < 2 || nq > (size_t)INT32_MAX || !(gmax > 0.0) || !table || !kpg || !phi)
    return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "projector_phi: bad arguments");
  if (n == 0) return DFTCUDA_OK;
  const size_t mt = 2 * (size_t)l + 1;
  const bool dev_in = is_device_pointer(table) && is_device_pointer(kpg);
  const bool dev_out = is_device_pointer(phi);
  SetupEngine* en = setup_engine();
  if (!en) return fail(DFTCUDA_ERR_CUDA, "projector_phi: no device");
  std::lock_guard<std::mutex> lock(en->mu);
  const size_t bt = ((sizeof(double) * nq + 15) / 16) * 16, bq = sizeof(double) * 3 * n, bp = sizeof(double) * mt * n;
  const size_t need = (dev_in ? 0 : bt + bq) + (dev_out ? 0 : bp);
  if (need) DFT_TRY(en->ensure(need));
  cudaStream_t s = en->s;
  const double* dt = table;
  const double* dq = kpg;
  double* dp = phi;
  size_t off = 0;
  if (!dev_in) {
    DFT_CUDA_TRY(cudaMemcpyAsync(en->buf, table, sizeof(double) * nq, cudaMemcpyDefault, s));
    DFT_CUDA_TRY(cudaMemcpyAsync(en->buf + bt, kpg, bq, cudaMemcpyDefault, s));
    dt = reinterpret_cast<const double*>(en->buf);
    dq = reinterpret_cast<const double*>(en->buf + bt);
    off = bt + bq;
  }
  if (!dev_out) dp = reinterpret_cast<double*>(en->buf + off);
  k_projector_phi<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(l, dt, (int)nq, gmax, dq, (long)n, dp);
  count_launch();
  DFT_CUDA_TRY(cudaGetLastError());
  if (!dev_out) DFT_CUDA_TRY(cudaMemcpyAsync(phi, dp, bp, cudaMemcpyDeviceToHost, s));
  DFT_CUDA_TRY(cudaStreamSynchronize(s));
  return DFTCUDA_OK;
}
