// Complex GEMM on the 5th-generation tensor cores (tcgen05, kind::tf32, FP32 accumulation in TMEM)
// for the mixed-precision projector contractions (apply.zig:1143-1183 projection and 1278-1336
// back-projection, with the same operand conventions as zgemm.cu):
//
//   out(r, c) = alpha * sum_k opA(A(r, k)) * opB(B(c, k)) + beta * out(r, c)     (FP64 in and out)
//
// One CTA = 4 warps computes a 128 x 64 complex tile.  Each K slice of 32 is converted from FP64 to
// TF32-representable FP32 by all 128 threads straight into the canonical K-major no-swizzle shared
// memory layout (8-row x 16-byte core matrices), real and imaginary parts in separate tiles.  One
// elected thread issues, per 8-deep K step, the four real MMAs of a complex product
//   Dr += Ar Br,  Dr += (-Ai) Bi (negate-A bit),  Di += Ar Bi,  Di += Ai Br
// into two 64-column FP32 TMEM accumulators, and commits them to the stage's mbarrier; the two-stage
// ring lets the next slice's conversion overlap the MMAs in flight.  The epilogue reads TMEM with
// tcgen05.ld (each warp its 32 lanes = 32 rows) and writes FP64 results (or split-K partials).
//
// SPLIT = true is the 3xTF32 form: each operand element x is held as hi + lo with hi = tf32(x)
// (round to nearest, cvt.rna.tf32.f32) and lo = tf32(x - hi), and every real product is taken as
// hi*hi + hi*lo + lo*hi (the lo*lo term is below FP32 rounding).  Twelve MMAs per 8-deep K step
// instead of four, two shared-memory planes per operand part; relative error ~1e-6 instead of ~1e-3.
//
// Every mbarrier wait is bounded: on timeout the CTA records an error flag, waits (bounded) for its
// outstanding MMAs, frees its TMEM and returns; the host turns the flag into DFTCUDA_ERR_TIMEOUT.
#include <algorithm>

#include "kctx.cuh"

namespace dftcuda {

constexpr int TC_M = 128, TC_N = 64, TC_K = 32;
constexpr int TC_THREADS = 128;
constexpr int TC_STAGES = 2;
constexpr int TC_A_BYTES = TC_M * TC_K * 4;  // one real plane of the A tile
constexpr int TC_B_BYTES = TC_N * TC_K * 4;
constexpr int TC_STAGE_BYTES = 2 * TC_A_BYTES + 2 * TC_B_BYTES;  // Ar, Ai, Br, Bi
__host__ __device__ constexpr int tc_stage_bytes(bool split) { return split ? 2 * TC_STAGE_BYTES : TC_STAGE_BYTES; }
__host__ __device__ constexpr int tc_smem(bool split) { return TC_STAGES * tc_stage_bytes(split) + 64; }
constexpr uint32_t TC_TMEM_COLS = 128;  // Dr (64) + Di (64)
constexpr long long TC_SPIN_LIMIT = 1LL << 26;

// Byte offset of element (row, k) in a K-major no-swizzle tile with TC_K columns.
__device__ __forceinline__ uint32_t tc_off(int row, int k) {
  return (uint32_t)((row >> 3) * (TC_K / 4) * 128 + (k >> 2) * 128 + (row & 7) * 16 + (k & 3) * 4);
}

__device__ __forceinline__ uint64_t tc_desc(uint32_t smem_addr) {
  // start address >> 4 | LBO (128 B, the K-adjacent core matrix) | SBO (row-group stride) | version 1 (sm100)
  const uint64_t lbo = 128 >> 4, sbo = ((TC_K / 4) * 128) >> 4;
  return (uint64_t)((smem_addr >> 4) & 0x3FFF) | (lbo << 16) | (sbo << 32) | (1ULL << 46);
}

__device__ __forceinline__ uint32_t tc_idesc(bool neg_a) {
  // D = F32 (bits 4-5 = 1), A = B = TF32 (2), both K-major, N >> 3 at bit 17, M >> 4 at bit 24
  return (1u << 4) | (2u << 7) | (2u << 10) | ((neg_a ? 1u : 0u) << 13) | ((uint32_t)(TC_N >> 3) << 17) |
         ((uint32_t)(TC_M >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, bool accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum ? 1 : 0));
}

__device__ __forceinline__ void tc_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(mbar));
}

// Bounded wait for the completion of the phase with the given parity.  Returns false on timeout.
__device__ __forceinline__ bool tc_wait(uint32_t mbar, uint32_t parity) {
  for (long long i = 0; i < TC_SPIN_LIMIT; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ float tf32_rna(float x) {
  uint32_t u;
  asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(u) : "f"(x));
  return __uint_as_float(u);
}

template <bool AKC, bool BKC, bool CJA, bool CJB, bool SPLIT>
__global__ void __launch_bounds__(TC_THREADS) k_cgemm_tf32(int M, int N, int K, const double2* __restrict__ A, long lda,
                                                           const double2* __restrict__ B, long ldb,
                                                           double2* __restrict__ O, long ldo_r, long ldo_c,
                                                           double alpha, double beta, int kps,
                                                           double2* __restrict__ part, int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char tsm[];
  unsigned char* stages = tsm;
  constexpr int SB = tc_stage_bytes(SPLIT);
  uint64_t* mbar = reinterpret_cast<uint64_t*>(tsm + TC_STAGES * SB);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mbar + TC_STAGES);
  __shared__ int s_abort;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int r0 = blockIdx.y * TC_M, c0 = blockIdx.x * TC_N;
  const int kbeg = blockIdx.z * kps;
  const int kend = min(K, kbeg + kps);
  const int ntiles = kend > kbeg ? (kend - kbeg + TC_K - 1) / TC_K : 0;
  const uint32_t smem_base = (uint32_t)__cvta_generic_to_shared(stages);
  const uint32_t mbar_base = (uint32_t)__cvta_generic_to_shared(mbar);

  if (tid == 0) {
    s_abort = 0;
    for (int s = 0; s < TC_STAGES; ++s)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(mbar_base + 8 * s));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
  }
  if (warp == 0) {
    const uint32_t slot = (uint32_t)__cvta_generic_to_shared(tmem_slot);
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(slot), "r"(TC_TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  const uint32_t tmem = *tmem_slot;
  const uint32_t d_re = tmem, d_im = tmem + TC_N;

  for (int t = 0; t < ntiles; ++t) {
    const int s = t % TC_STAGES;
    if (t >= TC_STAGES) {
      // the MMAs that last read this stage must be done before it is overwritten
      if (!tc_wait(mbar_base + 8 * s, (uint32_t)((t / TC_STAGES - 1) & 1))) {
        if (lane == 0) atomicExch(err, 1);
        s_abort = 1;
      }
    }
    __syncthreads();
    if (s_abort) break;
    // stage layout: Ar, Ai, Br, Bi (hi parts), then for SPLIT Ar, Ai, Br, Bi lo parts
    unsigned char* st = stages + s * SB;
    float* Ar = reinterpret_cast<float*>(st);
    float* Ai = reinterpret_cast<float*>(st + TC_A_BYTES);
    float* Br = reinterpret_cast<float*>(st + 2 * TC_A_BYTES);
    float* Bi = reinterpret_cast<float*>(st + 2 * TC_A_BYTES + TC_B_BYTES);
    float* ArL = reinterpret_cast<float*>(st + TC_STAGE_BYTES);
    float* AiL = reinterpret_cast<float*>(st + TC_STAGE_BYTES + TC_A_BYTES);
    float* BrL = reinterpret_cast<float*>(st + TC_STAGE_BYTES + 2 * TC_A_BYTES);
    float* BiL = reinterpret_cast<float*>(st + TC_STAGE_BYTES + 2 * TC_A_BYTES + TC_B_BYTES);
    const int k0 = kbeg + t * TC_K;
    // one 8 x 4 core matrix per warp instruction: lane = (row in core, k in core)
    const int rr = lane & 7, ee = lane >> 3;
    for (int cm = warp; cm < (TC_M / 8) * (TC_K / 4); cm += TC_THREADS / 32) {
      const int g = cm / (TC_K / 4), h = cm % (TC_K / 4);
      const int r = g * 8 + rr, k = h * 4 + ee;
      const int gr = r0 + r, gk = k0 + k;
      double2 v = make_double2(0.0, 0.0);
      if (gr < M && gk < kend) v = AKC ? __ldg(A + (long)gr * lda + gk) : __ldg(A + (long)gk * lda + gr);
      const uint32_t o = tc_off(r, k) >> 2;
      const double vi = CJA ? -v.y : v.y;
      if (SPLIT) {
        const float hr = tf32_rna((float)v.x), hi = tf32_rna((float)vi);
        Ar[o] = hr;
        Ai[o] = hi;
        ArL[o] = tf32_rna((float)(v.x - (double)hr));
        AiL[o] = tf32_rna((float)(vi - (double)hi));
      } else {
        Ar[o] = (float)v.x;
        Ai[o] = (float)vi;
      }
    }
    for (int cm = warp; cm < (TC_N / 8) * (TC_K / 4); cm += TC_THREADS / 32) {
      const int g = cm / (TC_K / 4), h = cm % (TC_K / 4);
      const int c = g * 8 + rr, k = h * 4 + ee;
      const int gc = c0 + c, gk = k0 + k;
      double2 v = make_double2(0.0, 0.0);
      if (gc < N && gk < kend) v = BKC ? __ldg(B + (long)gc * ldb + gk) : __ldg(B + (long)gk * ldb + gc);
      const uint32_t o = tc_off(c, k) >> 2;
      const double vi = CJB ? -v.y : v.y;
      if (SPLIT) {
        const float hr = tf32_rna((float)v.x), hi = tf32_rna((float)vi);
        Br[o] = hr;
        Bi[o] = hi;
        BrL[o] = tf32_rna((float)(v.x - (double)hr));
        BiL[o] = tf32_rna((float)(vi - (double)hi));
      } else {
        Br[o] = (float)v.x;
        Bi[o] = (float)vi;
      }
    }
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
      const uint32_t sa = smem_base + s * SB;
      const uint32_t sar = sa, sai = sa + TC_A_BYTES, sbr = sa + 2 * TC_A_BYTES, sbi = sbr + TC_B_BYTES;
      const uint32_t lo = TC_STAGE_BYTES;  // offset of the lo planes
      const uint32_t id_pos = tc_idesc(false), id_neg = tc_idesc(true);
#pragma unroll
      for (int kk = 0; kk < TC_K / 8; ++kk) {
        const uint32_t koff = kk * 256;  // two 128-byte core matrices per 8-deep step
        const bool acc = (t > 0) || (kk > 0);
        if (SPLIT) {
          // cross terms first (smaller), then hi*hi
          tc_mma(d_re, tc_desc(sar + koff), tc_desc(sbr + lo + koff), id_pos, acc);
          tc_mma(d_re, tc_desc(sar + lo + koff), tc_desc(sbr + koff), id_pos, true);
          tc_mma(d_re, tc_desc(sai + koff), tc_desc(sbi + lo + koff), id_neg, true);
          tc_mma(d_re, tc_desc(sai + lo + koff), tc_desc(sbi + koff), id_neg, true);
          tc_mma(d_re, tc_desc(sar + koff), tc_desc(sbr + koff), id_pos, true);
          tc_mma(d_re, tc_desc(sai + koff), tc_desc(sbi + koff), id_neg, true);
          tc_mma(d_im, tc_desc(sar + koff), tc_desc(sbi + lo + koff), id_pos, acc);
          tc_mma(d_im, tc_desc(sar + lo + koff), tc_desc(sbi + koff), id_pos, true);
          tc_mma(d_im, tc_desc(sai + koff), tc_desc(sbr + lo + koff), id_pos, true);
          tc_mma(d_im, tc_desc(sai + lo + koff), tc_desc(sbr + koff), id_pos, true);
          tc_mma(d_im, tc_desc(sar + koff), tc_desc(sbi + koff), id_pos, true);
          tc_mma(d_im, tc_desc(sai + koff), tc_desc(sbr + koff), id_pos, true);
        } else {
          tc_mma(d_re, tc_desc(sar + koff), tc_desc(sbr + koff), id_pos, acc);
          tc_mma(d_re, tc_desc(sai + koff), tc_desc(sbi + koff), id_neg, true);
          tc_mma(d_im, tc_desc(sar + koff), tc_desc(sbi + koff), id_pos, acc);
          tc_mma(d_im, tc_desc(sai + koff), tc_desc(sbr + koff), id_pos, true);
        }
      }
      tc_commit(mbar_base + 8 * s);
    }
  }

  // all MMAs done: wait for the last commit of each stage in use
  bool ok = !s_abort;
  if (ntiles > 0) {
    const int last = ntiles - 1;
    if (!tc_wait(mbar_base + 8 * (last % TC_STAGES), (uint32_t)((last / TC_STAGES) & 1))) {
      ok = false;
      if (lane == 0) atomicExch(err, 1);
    }
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  const int r = r0 + warp * 32 + lane;
  if (ok && !s_abort) {
#pragma unroll 1
    for (int ch = 0; ch < TC_N / 16; ++ch) {
      uint32_t vr[16], vi[16];
      const uint32_t lane_addr = ((uint32_t)(warp * 32) << 16);
      if (ntiles > 0) {
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
            : "=r"(vr[0]), "=r"(vr[1]), "=r"(vr[2]), "=r"(vr[3]), "=r"(vr[4]), "=r"(vr[5]), "=r"(vr[6]), "=r"(vr[7]),
              "=r"(vr[8]), "=r"(vr[9]), "=r"(vr[10]), "=r"(vr[11]), "=r"(vr[12]), "=r"(vr[13]), "=r"(vr[14]), "=r"(vr[15])
            : "r"(d_re + lane_addr + ch * 16));
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
            : "=r"(vi[0]), "=r"(vi[1]), "=r"(vi[2]), "=r"(vi[3]), "=r"(vi[4]), "=r"(vi[5]), "=r"(vi[6]), "=r"(vi[7]),
              "=r"(vi[8]), "=r"(vi[9]), "=r"(vi[10]), "=r"(vi[11]), "=r"(vi[12]), "=r"(vi[13]), "=r"(vi[14]), "=r"(vi[15])
            : "r"(d_im + lane_addr + ch * 16));
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
      } else {
#pragma unroll
        for (int j = 0; j < 16; ++j) vr[j] = vi[j] = 0u;
      }
      if (r < M) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int c = c0 + ch * 16 + j;
          if (c >= N) continue;
          const double re = (double)__uint_as_float(vr[j]), im = (double)__uint_as_float(vi[j]);
          if (part) {
            part[((long)blockIdx.z * M + r) * N + c] = make_double2(re, im);
          } else {
            double2* o = O + (long)r * ldo_r + (long)c * ldo_c;
            double2 v = make_double2(alpha * re, alpha * im);
            if (beta != 0.0) {
              const double2 old = *o;
              v.x += beta * old.x;
              v.y += beta * old.y;
            }
            *o = v;
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TC_TMEM_COLS));
}

__global__ void k_cgemm_reduce(int M, int N, int splits, const double2* __restrict__ part, double2* __restrict__ O,
                               long ldo_r, long ldo_c, double alpha, double beta) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= (long)M * N) return;
  const int r = (int)(i / N), c = (int)(i - (long)r * N);
  double2 s = make_double2(0.0, 0.0);
  for (int z = 0; z < splits; ++z) {
    const double2 v = part[(long)z * M * N + i];
    s.x += v.x;
    s.y += v.y;
  }
  double2* o = O + (long)r * ldo_r + (long)c * ldo_c;
  double2 v = make_double2(alpha * s.x, alpha * s.y);
  if (beta != 0.0) {
    const double2 old = *o;
    v.x += beta * old.x;
    v.y += beta * old.y;
  }
  *o = v;
}

static int tc_splits(int M, int N, int K) {
  const long tiles = (long)ceil_div(M, TC_M) * ceil_div(N, TC_N);
  const long wave = 148;  // one 98 KB CTA per SM... two fit: keep the split count modest
  if (tiles >= wave || K < 8 * TC_K) return 1;
  const long maxs = std::max<long>(1, K / (TC_K * 16));
  return (int)std::max<long>(1, std::min<long>(maxs, (wave + tiles - 1) / tiles));
}

size_t cgemm_tf32_workspace_elems(int M, int N, int K) {
  const int s = tc_splits(M, N, K);
  return s > 1 ? (size_t)s * M * N : 0;
}

template <bool AKC, bool BKC, bool CJA, bool CJB, bool SPLIT>
static void tc_launch(const GemmArgs& g, dim3 grid, int kps, double2* part, int* err, cudaStream_t s) {
  static int attr_dev = -1;
  int dev = 0;
  cudaGetDevice(&dev);
  if (attr_dev != dev) {
    cudaFuncSetAttribute(k_cgemm_tf32<AKC, BKC, CJA, CJB, SPLIT>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc_smem(SPLIT));
    attr_dev = dev;
  }
  k_cgemm_tf32<AKC, BKC, CJA, CJB, SPLIT><<<grid, TC_THREADS, tc_smem(SPLIT), s>>>(
      g.M, g.N, g.K, g.A, g.lda, g.B, g.ldb, g.O, g.ldo_r, g.ldo_c, g.alpha, g.beta, kps, part, err);
  count_launch();
}

template <bool SPLIT>
static int tc_dispatch(const GemmArgs& g, dim3 grid, int kps, double2* part, int* err_dev, cudaStream_t s) {
  const int key = (g.a_kc ? 8 : 0) | (g.b_kc ? 4 : 0) | (g.conj_a ? 2 : 0) | (g.conj_b ? 1 : 0);
  switch (key) {
    case 12: tc_launch<true, true, false, false, SPLIT>(g, grid, kps, part, err_dev, s); break;   // projection
    case 1: tc_launch<false, false, false, true, SPLIT>(g, grid, kps, part, err_dev, s); break;   // back-projection
    case 14: tc_launch<true, true, true, false, SPLIT>(g, grid, kps, part, err_dev, s); break;    // Gram V^H W
    case 4: tc_launch<false, true, false, false, SPLIT>(g, grid, kps, part, err_dev, s); break;
    case 8: tc_launch<true, false, false, false, SPLIT>(g, grid, kps, part, err_dev, s); break;   // V C
    case 0: tc_launch<false, false, false, false, SPLIT>(g, grid, kps, part, err_dev, s); break;
    default: return fail(DFTCUDA_ERR_UNSUPPORTED, "cgemm_tf32: operand layout not instantiated");
  }
  return DFTCUDA_OK;
}

int cgemm_tf32(const GemmArgs& g, cudaStream_t s, double2* ws, size_t ws_elems, int* err_dev, bool split) {
  if (g.M <= 0 || g.N <= 0) return DFTCUDA_OK;
  if (g.K <= 0) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "cgemm_tf32: K must be positive");
  int splits = g.splits > 0 ? std::min(g.splits, std::max(1, g.K / 32)) : tc_splits(g.M, g.N, g.K);
  if (splits > 1 && (size_t)splits * g.M * g.N > ws_elems) splits = 1;
  int kps = (g.K + splits - 1) / splits;
  kps = ((kps + TC_K - 1) / TC_K) * TC_K;
  splits = (g.K + kps - 1) / kps;
  dim3 grid(ceil_div(g.N, TC_N), ceil_div(g.M, TC_M), splits);
  double2* part = splits > 1 ? ws : nullptr;
  DFT_TRY(split ? tc_dispatch<true>(g, grid, kps, part, err_dev, s) : tc_dispatch<false>(g, grid, kps, part, err_dev, s));
  if (part) {
    const long tot = (long)g.M * g.N;
    k_cgemm_reduce<<<ceil_div(tot, 256), 256, 0, s>>>(g.M, g.N, splits, part, g.O, g.ldo_r, g.ldo_c, g.alpha, g.beta); count_launch();
  }
  DFT_CUDA_TRY(cudaGetLastError());
  return DFTCUDA_OK;
}

}  // namespace dftcuda
