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
#include <cstdlib>
#include <string>

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

// ---- pipelined variant -----------------------------------------------------------------------------
// The same contraction with the operand traffic decoupled from the conversion: 8 warps per CTA;
// each 16-deep K slice of A (128 rows) and B (64 rows) streams into a two-slot FP64 staging ring
// with cp.async (zero-fill outside the matrix), so the loads of slices t+1 and t+2 are in flight
// while slice t is converted into the TF32 core-matrix ring and the MMAs of slice t-1 run.
constexpr int T2_K = 16;
constexpr int T2_THREADS = 256;
constexpr int T2_A64 = TC_M * T2_K;  // complex elements of one A slice
constexpr int T2_B64 = TC_N * T2_K;
constexpr int T2_STAGE64 = (T2_A64 + T2_B64) * 16;       // bytes of one FP64 staging slot
constexpr int T2_APL = TC_M * T2_K * 4, T2_BPL = TC_N * T2_K * 4;  // one TF32 plane
constexpr int T2_STAGE32 = 2 * T2_APL + 2 * T2_BPL;       // Ar, Ai, Br, Bi
__host__ __device__ constexpr int t2_stage32(bool split) { return split ? 2 * T2_STAGE32 : T2_STAGE32; }
__host__ __device__ constexpr int t2_smem(bool split) { return 2 * T2_STAGE64 + 2 * t2_stage32(split) + 64; }

__device__ __forceinline__ uint32_t t2_off(int row, int k) {
  return (uint32_t)((row >> 3) * (T2_K / 4) * 128 + (k >> 2) * 128 + (row & 7) * 16 + (k & 3) * 4);
}
__device__ __forceinline__ uint64_t t2_desc(uint32_t smem_addr) {
  const uint64_t lbo = 128 >> 4, sbo = ((T2_K / 4) * 128) >> 4;
  return (uint64_t)((smem_addr >> 4) & 0x3FFF) | (lbo << 16) | (sbo << 32) | (1ULL << 46);
}
__device__ __forceinline__ void t2_cp16(uint32_t sdst, const void* gsrc, bool pred) {
  const int sz = pred ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sdst), "l"(gsrc), "r"(sz) : "memory");
}

// Staging index e of a slice equals the linear index of its element: K-contiguous operands are
// staged [row][k], the others [k][row], so consecutive threads copy consecutive addresses.
template <bool KC, int ROWS>
__device__ __forceinline__ void t2_issue(const double2* __restrict__ X, long ldx, int nrows, int r0, int k0, int kend,
                                         uint32_t sbase, int tid) {
#pragma unroll
  for (int i = 0; i < ROWS * T2_K / T2_THREADS; ++i) {
    const int e = tid + i * T2_THREADS;
    const int r = KC ? e / T2_K : e % ROWS, k = KC ? e % T2_K : e / ROWS;
    const int gr = r0 + r, gk = k0 + k;
    const bool ok = gr < nrows && gk < kend;
    const double2* src = ok ? (KC ? X + (long)gr * ldx + gk : X + (long)gk * ldx + gr) : X;
    t2_cp16(sbase + (uint32_t)e * 16, src, ok);
  }
}

// One warp converts one 8-row x 4-k core matrix per step: its 32 lanes cover the core matrix's 32
// words, so the TF32 stores never conflict; the lane order within the core matrix follows the
// staging layout (rows fastest for [k][row] staging), so the FP64 staging reads stay sequential.
template <bool KC, int ROWS, bool CJ, bool SPLIT>
__device__ __forceinline__ void t2_convert(const double2* __restrict__ st, float* re, float* im, float* reL, float* imL, int tid) {
  const int warp = tid >> 5, lane = tid & 31;
  const int rr = KC ? (lane >> 2) : (lane & 7), kk = KC ? (lane & 3) : (lane >> 3);
  constexpr int NCM = (ROWS / 8) * (T2_K / 4);
#pragma unroll
  for (int i = 0; i < NCM / (T2_THREADS / 32); ++i) {
    const int cm = warp + i * (T2_THREADS / 32);
    const int r = (cm / (T2_K / 4)) * 8 + rr, k = (cm % (T2_K / 4)) * 4 + kk;
    const double2 v = st[KC ? r * T2_K + k : k * ROWS + r];
    const uint32_t o = t2_off(r, k) >> 2;
    const double vi = CJ ? -v.y : v.y;
    if (SPLIT) {
      const float hr = tf32_rna((float)v.x), hi = tf32_rna((float)vi);
      re[o] = hr;
      im[o] = hi;
      reL[o] = tf32_rna((float)(v.x - (double)hr));
      imL[o] = tf32_rna((float)(vi - (double)hi));
    } else {
      re[o] = (float)v.x;
      im[o] = (float)vi;
    }
  }
}

template <bool AKC, bool BKC, bool CJA, bool CJB, bool SPLIT>
__global__ void __launch_bounds__(T2_THREADS) k_cgemm_tc2(int M, int N, int K, const double2* __restrict__ A, long lda,
                                                          const double2* __restrict__ B, long ldb,
                                                          double2* __restrict__ O, long ldo_r, long ldo_c,
                                                          double alpha, double beta, int kps,
                                                          double2* __restrict__ part, int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char tsm2[];
  constexpr int S32 = t2_stage32(SPLIT);
  unsigned char* st64 = tsm2;
  unsigned char* st32 = tsm2 + 2 * T2_STAGE64;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(st32 + 2 * S32);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mbar + 2);
  __shared__ int s_abort;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int r0 = blockIdx.y * TC_M, c0 = blockIdx.x * TC_N;
  const int kbeg = blockIdx.z * kps;
  const int kend = min(K, kbeg + kps);
  const int ntiles = kend > kbeg ? (kend - kbeg + T2_K - 1) / T2_K : 0;
  const uint32_t s64_base = (uint32_t)__cvta_generic_to_shared(st64);
  const uint32_t s32_base = (uint32_t)__cvta_generic_to_shared(st32);
  const uint32_t mbar_base = (uint32_t)__cvta_generic_to_shared(mbar);
  if (tid == 0) {
    s_abort = 0;
    for (int q = 0; q < 2; ++q) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(mbar_base + 8 * q));
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
  // prologue: slices 0 and 1 in flight
  for (int q = 0; q < 2; ++q) {
    if (q < ntiles) {
      const int k0 = kbeg + q * T2_K;
      const uint32_t sb = s64_base + q * T2_STAGE64;
      t2_issue<AKC, TC_M>(A, lda, M, r0, k0, kend, sb, tid);
      t2_issue<BKC, TC_N>(B, ldb, N, c0, k0, kend, sb + T2_A64 * 16, tid);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  }
  int t_stop = ntiles;  // slices whose MMAs were issued: [0, t_stop)
  for (int t = 0; t < ntiles; ++t) {
    const int q = t & 1;
    asm volatile("cp.async.wait_group 1;\n" ::: "memory");
    if (t >= 2) {
      // the MMAs that last read this TF32 slot must be done before it is overwritten
      if (!tc_wait(mbar_base + 8 * q, (uint32_t)((t / 2 - 1) & 1))) {
        if (lane == 0) atomicExch(err, 1);
        s_abort = 1;
      }
    }
    __syncthreads();
    if (s_abort) {
      t_stop = t;
      break;
    }
    const double2* sa = reinterpret_cast<const double2*>(st64 + q * T2_STAGE64);
    unsigned char* s3 = st32 + q * S32;
    float* Ar = reinterpret_cast<float*>(s3);
    float* Ai = reinterpret_cast<float*>(s3 + T2_APL);
    float* Br = reinterpret_cast<float*>(s3 + 2 * T2_APL);
    float* Bi = reinterpret_cast<float*>(s3 + 2 * T2_APL + T2_BPL);
    float* ArL = reinterpret_cast<float*>(s3 + T2_STAGE32);
    float* AiL = reinterpret_cast<float*>(s3 + T2_STAGE32 + T2_APL);
    float* BrL = reinterpret_cast<float*>(s3 + T2_STAGE32 + 2 * T2_APL);
    float* BiL = reinterpret_cast<float*>(s3 + T2_STAGE32 + 2 * T2_APL + T2_BPL);
    t2_convert<AKC, TC_M, CJA, SPLIT>(sa, Ar, Ai, ArL, AiL, tid);
    t2_convert<BKC, TC_N, CJB, SPLIT>(sa + T2_A64, Br, Bi, BrL, BiL, tid);
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    // the staging slot is free again: slice t+2 streams into it
    if (t + 2 < ntiles) {
      const int k0 = kbeg + (t + 2) * T2_K;
      const uint32_t sb = s64_base + q * T2_STAGE64;
      t2_issue<AKC, TC_M>(A, lda, M, r0, k0, kend, sb, tid);
      t2_issue<BKC, TC_N>(B, ldb, N, c0, k0, kend, sb + T2_A64 * 16, tid);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
      const uint32_t sa3 = s32_base + q * S32;
      const uint32_t sar = sa3, sai = sa3 + T2_APL, sbr = sa3 + 2 * T2_APL, sbi = sbr + T2_BPL;
      const uint32_t lo = T2_STAGE32;
      const uint32_t id_pos = tc_idesc(false), id_neg = tc_idesc(true);
#pragma unroll
      for (int kk = 0; kk < T2_K / 8; ++kk) {
        const uint32_t koff = kk * 256;
        const bool acc = (t > 0) || (kk > 0);
        if (SPLIT) {
          tc_mma(d_re, t2_desc(sar + koff), t2_desc(sbr + lo + koff), id_pos, acc);
          tc_mma(d_re, t2_desc(sar + lo + koff), t2_desc(sbr + koff), id_pos, true);
          tc_mma(d_re, t2_desc(sai + koff), t2_desc(sbi + lo + koff), id_neg, true);
          tc_mma(d_re, t2_desc(sai + lo + koff), t2_desc(sbi + koff), id_neg, true);
          tc_mma(d_re, t2_desc(sar + koff), t2_desc(sbr + koff), id_pos, true);
          tc_mma(d_re, t2_desc(sai + koff), t2_desc(sbi + koff), id_neg, true);
          tc_mma(d_im, t2_desc(sar + koff), t2_desc(sbi + lo + koff), id_pos, acc);
          tc_mma(d_im, t2_desc(sar + lo + koff), t2_desc(sbi + koff), id_pos, true);
          tc_mma(d_im, t2_desc(sai + koff), t2_desc(sbr + lo + koff), id_pos, true);
          tc_mma(d_im, t2_desc(sai + lo + koff), t2_desc(sbr + koff), id_pos, true);
          tc_mma(d_im, t2_desc(sar + koff), t2_desc(sbi + koff), id_pos, true);
          tc_mma(d_im, t2_desc(sai + koff), t2_desc(sbr + koff), id_pos, true);
        } else {
          tc_mma(d_re, t2_desc(sar + koff), t2_desc(sbr + koff), id_pos, acc);
          tc_mma(d_re, t2_desc(sai + koff), t2_desc(sbi + koff), id_neg, true);
          tc_mma(d_im, t2_desc(sar + koff), t2_desc(sbi + koff), id_pos, acc);
          tc_mma(d_im, t2_desc(sai + koff), t2_desc(sbr + koff), id_pos, true);
        }
      }
      tc_commit(mbar_base + 8 * q);
    }
  }
  // drain every copy this thread issued (also on the abort path)
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  bool ok = !s_abort;
  if (t_stop > 0) {
    // the last commit tracks every MMA issued before it (bounded wait, also after an abort, so the
    // TMEM is not freed under running MMAs)
    const int last = t_stop - 1;
    if (!tc_wait(mbar_base + 8 * (last & 1), (uint32_t)((last / 2) & 1))) {
      ok = false;
      if (lane == 0) atomicExch(err, 1);
    }
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  if (ok && !s_abort) {
    // warps 0-3 columns 0-31, warps 4-7 columns 32-63; each warp its 32 TMEM lanes = rows
    const int quarter = warp & 3, half = warp >> 2;
    const int r = r0 + quarter * 32 + lane;
#pragma unroll 1
    for (int ch = 0; ch < 2; ++ch) {
      const int cbase = half * 32 + ch * 16;
      uint32_t vr[16], vi[16];
      const uint32_t lane_addr = ((uint32_t)(quarter * 32) << 16);
      if (ntiles > 0) {
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
            : "=r"(vr[0]), "=r"(vr[1]), "=r"(vr[2]), "=r"(vr[3]), "=r"(vr[4]), "=r"(vr[5]), "=r"(vr[6]), "=r"(vr[7]),
              "=r"(vr[8]), "=r"(vr[9]), "=r"(vr[10]), "=r"(vr[11]), "=r"(vr[12]), "=r"(vr[13]), "=r"(vr[14]), "=r"(vr[15])
            : "r"(d_re + lane_addr + cbase));
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
            : "=r"(vi[0]), "=r"(vi[1]), "=r"(vi[2]), "=r"(vi[3]), "=r"(vi[4]), "=r"(vi[5]), "=r"(vi[6]), "=r"(vi[7]),
              "=r"(vi[8]), "=r"(vi[9]), "=r"(vi[10]), "=r"(vi[11]), "=r"(vi[12]), "=r"(vi[13]), "=r"(vi[14]), "=r"(vi[15])
            : "r"(d_im + lane_addr + cbase));
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
      } else {
#pragma unroll
        for (int j = 0; j < 16; ++j) vr[j] = vi[j] = 0u;
      }
      if (r < M) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int c = c0 + cbase + j;
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
  if (M < TC_M && N > M) std::swap(M, N);  // the transposed problem cgemm_tf32 runs
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

template <bool AKC, bool BKC, bool CJA, bool CJB, bool SPLIT>
static void tc2_launch(const GemmArgs& g, dim3 grid, int kps, double2* part, int* err, cudaStream_t s) {
  static int attr_dev = -1;
  int dev = 0;
  cudaGetDevice(&dev);
  if (attr_dev != dev) {
    cudaFuncSetAttribute(k_cgemm_tc2<AKC, BKC, CJA, CJB, SPLIT>, cudaFuncAttributeMaxDynamicSharedMemorySize, t2_smem(SPLIT));
    attr_dev = dev;
  }
  k_cgemm_tc2<AKC, BKC, CJA, CJB, SPLIT><<<grid, T2_THREADS, t2_smem(SPLIT), s>>>(
      g.M, g.N, g.K, g.A, g.lda, g.B, g.ldb, g.O, g.ldo_r, g.ldo_c, g.alpha, g.beta, kps, part, err);
  count_launch();
}

// DFTCUDA_TC=v1 selects the first (synchronous-load) kernel for A/B measurements.
static bool tc_v1() {
  static const bool v = [] {
    const char* e = std::getenv("DFTCUDA_TC");
    return e && std::string(e) == "v1";
  }();
  return v;
}

template <bool AKC, bool BKC, bool CJA, bool CJB, bool SPLIT>
static void tc_any(const GemmArgs& g, dim3 grid, int kps, double2* part, int* err, cudaStream_t s) {
  if (tc_v1()) tc_launch<AKC, BKC, CJA, CJB, SPLIT>(g, grid, kps, part, err, s);
  else tc2_launch<AKC, BKC, CJA, CJB, SPLIT>(g, grid, kps, part, err, s);
}

template <bool SPLIT>
static int tc_dispatch(const GemmArgs& g, dim3 grid, int kps, double2* part, int* err_dev, cudaStream_t s) {
  const int key = (g.a_kc ? 8 : 0) | (g.b_kc ? 4 : 0) | (g.conj_a ? 2 : 0) | (g.conj_b ? 1 : 0);
  switch (key) {
    case 12: tc_any<true, true, false, false, SPLIT>(g, grid, kps, part, err_dev, s); break;   // projection
    case 1: tc_any<false, false, false, true, SPLIT>(g, grid, kps, part, err_dev, s); break;   // back-projection
    case 14: tc_any<true, true, true, false, SPLIT>(g, grid, kps, part, err_dev, s); break;    // Gram V^H W
    case 4: tc_any<false, true, false, false, SPLIT>(g, grid, kps, part, err_dev, s); break;
    case 8: tc_any<true, false, false, false, SPLIT>(g, grid, kps, part, err_dev, s); break;   // V C
    case 0: tc_any<false, false, false, false, SPLIT>(g, grid, kps, part, err_dev, s); break;
    case 2: tc_any<false, false, true, false, SPLIT>(g, grid, kps, part, err_dev, s); break;    // back-projection, transposed
    case 13: tc_any<true, true, false, true, SPLIT>(g, grid, kps, part, err_dev, s); break;    // Gram, transposed
    default: return fail(DFTCUDA_ERR_UNSUPPORTED, "cgemm_tf32: operand layout not instantiated");
  }
  return DFTCUDA_OK;
}

int cgemm_tf32(const GemmArgs& g0, cudaStream_t s, double2* ws, size_t ws_elems, int* err_dev, bool split) {
  if (g0.M <= 0 || g0.N <= 0) return DFTCUDA_OK;
  // out(r, c) = sum_k A(r, k) B(c, k) is also out^T(c, r) = sum_k B(c, k) A(r, k): with fewer rows
  // than one 128-row MMA tile and more columns, compute the transpose so the wide dimension fills
  // the MMA's M (the back-projection: rows = bands, columns = plane waves).
  GemmArgs g = g0;
  if (g0.M < TC_M && g0.N > g0.M) {
    g.M = g0.N; g.N = g0.M;
    g.A = g0.B; g.lda = g0.ldb; g.a_kc = g0.b_kc; g.conj_a = g0.conj_b;
    g.B = g0.A; g.ldb = g0.lda; g.b_kc = g0.a_kc; g.conj_b = g0.conj_a;
    g.ldo_r = g0.ldo_c; g.ldo_c = g0.ldo_r;
  }
  if (g.K <= 0) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "cgemm_tf32: K must be positive");
  int splits = g.splits > 0 ? std::min(g.splits, std::max(1, g.K / 32)) : tc_splits(g.M, g.N, g.K);
  if (splits > 1 && (size_t)splits * g.M * g.N > ws_elems) splits = 1;
  int kps = (g.K + splits - 1) / splits;
  kps = ((kps + TC_K - 1) / TC_K) * TC_K;  // a multiple of both kernels' K slice
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
