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

// ---- k_cgemm_tc3: warp-specialised 128 x 256 tiles ---------------------------------------------
// For products whose both output dimensions reach 128 (Rayleigh-Ritz Gram matrices, subspace
// rotations): a 256-column tile gives every converted operand element four times the MMA work of
// the 64-column tiles above.  Warps 0-7 are converters: each thread owns three of the slot's 768
// core-matrix rows (A: 16 row groups x 2 k groups x 8 rows, B: 32 x 2 x 8), copies their FP64
// elements with cp.async one K step ahead into its own part of a shared-memory staging area, waits
// for the TF32 slot to be free, writes the TF32 planes (hi and lo parts for 3xTF32) into the ring
// as 16-byte vectors and arrives on the slot's "full" mbarrier.  Lane 0 of warp 8 waits for full slots and
// issues one 8-deep K step per slot (12 MMAs for 3xTF32, 4 otherwise) of 128 x 256 x 8, committing
// each slot back to its "empty" mbarrier.  TMEM holds the two 256-column FP32 accumulators (all 512
// columns; the shared-memory footprint keeps one CTA per SM).  Waits are bounded; a timeout sets the
// error flag and every role winds down: each converter thread waits for its own staging copies
// (cp.async.wait_all) before it leaves, and one final commit is waited for so that no MMA is in
// flight when the TMEM is freed.
constexpr int T3_N = 256;
constexpr int T3_K = 8;
constexpr int T3_CONV_WARPS = 8;
constexpr int T3_THREADS = 32 * (T3_CONV_WARPS + 1);
constexpr int T3_APL = TC_M * T3_K * 4;  // one TF32 plane of the A slot (4 KB)
constexpr int T3_BPL = T3_N * T3_K * 4;  // one TF32 plane of the B slot (8 KB)
constexpr int T3_SLOT = 2 * T3_APL + 2 * T3_BPL;  // Ar, Ai, Br, Bi
constexpr int T3_ACM = (TC_M / 8) * (T3_K / 4);   // 32 core matrices of A per slot
constexpr uint32_t T3_TMEM_COLS = 512;
__host__ __device__ constexpr int t3_slot(bool split) { return split ? 2 * T3_SLOT : T3_SLOT; }
__host__ __device__ constexpr int t3_stages(bool split) { return split ? 3 : 6; }
// FP64 staging: each converter thread's 12 elements of a K step, element-major (element e of
// thread t at e * 4 KB + t * 16 B, so consecutive lanes touch consecutive 16 bytes), T3_D steps
// deep: the cp.async copies of step t + T3_D are in flight while step t converts.  One step of
// lead covers the load latency (a K step takes ~2 us); the shared memory goes to a 3-slot TF32 ring
// instead (measured: 5 % faster than 2 staging and 2 ring slots).
constexpr int T3_D = 1;
constexpr int T3_STG = 12 * T3_CONV_WARPS * 32 * 16;  // 48 KB
__host__ __device__ constexpr int t3_smem(bool split) {
  return t3_stages(split) * t3_slot(split) + T3_D * T3_STG + 256;  // + barriers, TMEM slot
}

// Byte offset of (row, k) in a slot plane: core matrices of 8 rows x 4 k (128 B), the two k groups
// of a row group adjacent (LBO 128 B), row groups 256 B apart (SBO).
__device__ __forceinline__ uint32_t t3_off(int row, int k) {
  return (uint32_t)((row >> 3) * 256 + (k >> 2) * 128 + (row & 7) * 16 + (k & 3) * 4);
}
__device__ __forceinline__ uint64_t t3_desc(uint32_t smem_addr) {
  const uint64_t lbo = 128 >> 4, sbo = 256 >> 4;
  return (uint64_t)((smem_addr >> 4) & 0x3FFF) | (lbo << 16) | (sbo << 32) | (1ULL << 46);
}
__device__ __forceinline__ uint32_t t3_idesc(bool neg_a) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((neg_a ? 1u : 0u) << 13) | ((uint32_t)(T3_N >> 3) << 17) |
         ((uint32_t)(TC_M >> 4) << 24);
}

// One core-matrix row (4 consecutive k of one row) of an operand: hi parts (and lo parts for 3xTF32)
// of its real and imaginary planes, stored as 16-byte vectors.  The split is taken in FP32: x is
// rounded to FP32, hi = tf32(x) (round to nearest), lo = tf32(x - hi).
template <bool CJ, bool SPLIT>
__device__ __forceinline__ void t3_store_row(unsigned char* plane0, int plane_bytes, int slot_lo, uint32_t off,
                                             const double2* v) {
  float hr[4], hi[4], lr[4], li[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const float fr = (float)v[j].x, fi = CJ ? -(float)v[j].y : (float)v[j].y;
    if (SPLIT) {
      hr[j] = tf32_rna(fr);
      hi[j] = tf32_rna(fi);
      lr[j] = tf32_rna(fr - hr[j]);
      li[j] = tf32_rna(fi - hi[j]);
    } else {
      hr[j] = fr;
      hi[j] = fi;
    }
  }
  *reinterpret_cast<float4*>(plane0 + off) = make_float4(hr[0], hr[1], hr[2], hr[3]);
  *reinterpret_cast<float4*>(plane0 + plane_bytes + off) = make_float4(hi[0], hi[1], hi[2], hi[3]);
  if (SPLIT) {
    *reinterpret_cast<float4*>(plane0 + slot_lo + off) = make_float4(lr[0], lr[1], lr[2], lr[3]);
    *reinterpret_cast<float4*>(plane0 + slot_lo + plane_bytes + off) = make_float4(li[0], li[1], li[2], li[3]);
  }
}

__device__ __forceinline__ void t3_arrive(uint32_t mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(mbar) : "memory");
}

// The tensor cores' FP32 accumulation is not round-to-nearest: its error grows with the number of
// accumulation steps (measured on 3xTF32 products: ~1e-5 relative after 1000 terms, ~1e-4 after
// 120000).  So the FP32 accumulators only ever hold T3_CHUNK K steps (2048 terms): at each chunk
// end the converter warps drain TMEM into FP64 sums kept in the destination (the output tile, or the
// split's partial block), and the MMA warp starts the next chunk afresh once the drain is done.
constexpr int T3_CHUNK = 256;  // default chunk, in K steps of 8

// Drain of the TMEM accumulators into the FP64 destination by one converter warp (TMEM lanes
// 32 (warp % 4) .. = rows, columns 128 (warp / 4) .. + 127).  first: this split's first chunk (the
// destination starts as beta * out, or as the partial block).
__device__ __forceinline__ void t3_drain(uint32_t d_re, uint32_t d_im, int warp, int lane, bool have, bool first, int M,
                                         int N, int r0, int c0, double2* __restrict__ O, long ldo_r, long ldo_c,
                                         double alpha, double beta, double2* __restrict__ part, int z) {
  const int quarter = warp & 3, half = warp >> 2;
  const int r = r0 + quarter * 32 + lane;
  const uint32_t lane_addr = ((uint32_t)(quarter * 32) << 16);
#pragma unroll 1
  for (int ch = 0; ch < 16; ++ch) {
    const int cbase = half * 128 + ch * 8;
    if (c0 + cbase >= N) break;
    uint32_t vr[8], vi[8];
    if (have) {
      asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
                   : "=r"(vr[0]), "=r"(vr[1]), "=r"(vr[2]), "=r"(vr[3]), "=r"(vr[4]), "=r"(vr[5]), "=r"(vr[6]), "=r"(vr[7])
                   : "r"(d_re + lane_addr + cbase));
      asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
                   : "=r"(vi[0]), "=r"(vi[1]), "=r"(vi[2]), "=r"(vi[3]), "=r"(vi[4]), "=r"(vi[5]), "=r"(vi[6]), "=r"(vi[7])
                   : "r"(d_im + lane_addr + cbase));
      asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
    } else {
#pragma unroll
      for (int j = 0; j < 8; ++j) vr[j] = vi[j] = 0u;
    }
    if (r < M) {
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int c = c0 + cbase + j;
        if (c >= N) continue;
        const double re = (double)__uint_as_float(vr[j]), im = (double)__uint_as_float(vi[j]);
        if (part) {
          double2* o = part + ((long)z * N + c) * M + r;  // column-major partials
          double2 v = make_double2(re, im);
          if (!first) {
            const double2 old = *o;
            v.x += old.x;
            v.y += old.y;
          }
          *o = v;
        } else {
          double2* o = O + (long)r * ldo_r + (long)c * ldo_c;
          double2 v = make_double2(alpha * re, alpha * im);
          const double2 old = (first && beta == 0.0) ? make_double2(0.0, 0.0) : *o;
          const double b = first ? beta : 1.0;
          v.x += b * old.x;
          v.y += b * old.y;
          *o = v;
        }
      }
    }
  }
}

template <bool AKC, bool BKC, bool CJA, bool CJB, bool SPLIT>
__global__ void __launch_bounds__(T3_THREADS, 1) k_cgemm_tc3(int M, int N, int K, const double2* __restrict__ A, long lda,
                                                             const double2* __restrict__ B, long ldb,
                                                             double2* __restrict__ O, long ldo_r, long ldo_c,
                                                             double alpha, double beta, int kps,
                                                             double2* __restrict__ part, int* __restrict__ err,
                                                             int chunk) {
  extern __shared__ __align__(1024) unsigned char tsm3[];
  constexpr int NS = t3_stages(SPLIT);
  constexpr int SL = t3_slot(SPLIT);
  // barriers: full[NS] (converters -> MMA), empty[NS] (MMA -> converters), chunk_done (MMA ->
  // converters: a chunk's MMAs are complete), drained (converters -> MMA: TMEM read out), fin (all
  // MMAs complete)
  uint64_t* mbar = reinterpret_cast<uint64_t*>(tsm3 + NS * SL + T3_D * T3_STG);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mbar + 2 * NS + 3);
  __shared__ volatile int s_abort;
  __shared__ int s_issued;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int r0 = blockIdx.y * TC_M, c0 = blockIdx.x * T3_N;
  const int kbeg = blockIdx.z * kps;
  const int kend = min(K, kbeg + kps);
  const int ntiles = kend > kbeg ? (kend - kbeg + T3_K - 1) / T3_K : 0;
  const int nchunks = (ntiles + chunk - 1) / chunk;
  const uint32_t ring = (uint32_t)__cvta_generic_to_shared(tsm3);
  const uint32_t mb = (uint32_t)__cvta_generic_to_shared(mbar);
  const uint32_t mb_chunk = mb + 16 * NS, mb_drained = mb_chunk + 8, mb_fin = mb_chunk + 16;
  if (tid == 0) {
    s_abort = 0;
    for (int q = 0; q < NS; ++q) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(mb + 8 * q), "r"(T3_CONV_WARPS));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(mb + 8 * (NS + q)));
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(mb_chunk));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(mb_drained), "r"(T3_CONV_WARPS));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(mb_fin));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
  }
  if (warp == T3_CONV_WARPS) {
    const uint32_t slot = (uint32_t)__cvta_generic_to_shared(tmem_slot);
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(slot), "r"(T3_TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  const uint32_t tmem = *tmem_slot;
  const uint32_t d_re = tmem, d_im = tmem + T3_N;
  if (warp < T3_CONV_WARPS) {
    // ---- converters (and, at chunk ends, the drain) ----
    // Thread t owns three core-matrix rows per slot: unit t of A and units t, t + 256 of B, a unit
    // being (row group, k group, row in group) with the row fastest, so 8 consecutive lanes fill one
    // 128-byte core matrix (conflict-free 16-byte stores) and read consecutive rows (coalesced
    // when rows are contiguous) or one 64-byte run each (K-contiguous storage).
    const double2* up[3];
    long ustep[3];
    bool uok[3];
    uint32_t uoff[3];
#pragma unroll
    for (int u = 0; u < 3; ++u) {
      const int unit = tid + u * T3_CONV_WARPS * 32;
      const int cm = unit >> 3, r8 = unit & 7;
      const bool isA = cm < T3_ACM;
      const int cc = isA ? cm : cm - T3_ACM;
      const int rg = cc >> 1, kg = cc & 1;
      const int row = (isA ? r0 : c0) + rg * 8 + r8;
      const bool kc = isA ? AKC : BKC;
      const long ld = isA ? lda : ldb;
      uok[u] = row < (isA ? M : N);
      const double2* X = isA ? A : B;
      up[u] = kc ? X + (long)(uok[u] ? row : 0) * ld + kbeg + kg * 4 : X + (long)(kbeg + kg * 4) * ld + (uok[u] ? row : 0);
      ustep[u] = kc ? 1 : ld;  // between consecutive k
      uoff[u] = (uint32_t)(rg * 256 + kg * 128 + r8 * 16);
    }
    double2 cur[12];
    const uint32_t stg = (uint32_t)__cvta_generic_to_shared(tsm3 + NS * SL) + (uint32_t)tid * 16;
    const double2* stg_own = reinterpret_cast<const double2*>(tsm3 + NS * SL) + tid;
    // cp.async copies of K step t into staging slot t % T3_D (zero-filled outside the matrix;
    // pointers advance by 8 k per step, the k bound only matters on the last step); one commit group
    auto issue_step = [&](int t) {
      if (t < ntiles) {
        const int kk0 = kbeg + t * T3_K;
        const bool full = kk0 + T3_K <= kend;
        const uint32_t sb = stg + (uint32_t)((t % T3_D) * T3_STG);
#pragma unroll
        for (int u = 0; u < 3; ++u) {
          const int kgu = (int)((uoff[u] >> 7) & 1);
          const double2* p = up[u] + (long)t * T3_K * ustep[u];
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const bool ok = uok[u] && (full || kk0 + kgu * 4 + j < kend);
            // a predicated-off copy reads nothing (zero fill); its source is the operand's base
            t2_cp16(sb + (uint32_t)((u * 4 + j) * 4096), ok ? (const void*)(p + (long)j * ustep[u]) : (const void*)(u == 0 ? A : B), ok);
          }
        }
      }
      asm volatile("cp.async.commit_group;\n" ::: "memory");
    };
    int drained = 0;  // chunks drained so far
    // wait for chunk `drained` to finish, drain it, release the accumulators; false on abort
    auto drain_next = [&]() -> bool {
      int ok = 1;
      if (lane == 0) ok = tc_wait(mb_chunk, (uint32_t)(drained & 1)) ? 1 : 0;
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) {
        if (lane == 0) atomicExch(err, 1);
        s_abort = 1;
        return false;
      }
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
      t3_drain(d_re, d_im, warp, lane, true, drained == 0, M, N, r0, c0, O, ldo_r, ldo_c, alpha, beta, part, blockIdx.z);
      asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
      __syncwarp();
      if (lane == 0) t3_arrive(mb_drained);
      ++drained;
      return true;
    };
#pragma unroll
    for (int d = 0; d < T3_D; ++d) issue_step(d);
    for (int t = 0; t < ntiles; ++t) {
      const int q = t % NS;
      // the slot's previous stage t - NS opens a new chunk: its MMAs wait for the previous chunk's
      // drain, so drain it before waiting for the slot (before the next loads, to keep registers low)
      if (t >= NS && (t - NS) % chunk == 0 && (t - NS) / chunk > drained) {
        if (!__shfl_sync(0xffffffffu, s_abort, 0)) drain_next();
      }
      // this thread's copies of step t have landed (the T3_D - 1 younger groups may be pending);
      // the thread reads only what it copied itself, so no block barrier is needed
      asm volatile("cp.async.wait_group %0;\n" ::"n"(T3_D - 1) : "memory");
#pragma unroll
      for (int e = 0; e < 12; ++e) cur[e] = stg_own[(t % T3_D) * (T3_STG / 16) + e * 256];
      issue_step(t + T3_D);
      if (t >= NS) {
        int ok = 1;
        if (lane == 0) ok = tc_wait(mb + 8 * (NS + q), (uint32_t)((t / NS - 1) & 1)) ? 1 : 0;
        ok = __shfl_sync(0xffffffffu, ok, 0);
        if (!ok) {
          if (lane == 0) atomicExch(err, 1);
          s_abort = 1;
        }
      }
      if (__shfl_sync(0xffffffffu, s_abort, 0)) break;  // one read per warp: the warp leaves together
      unsigned char* slot = tsm3 + q * SL;
      t3_store_row<CJA, SPLIT>(slot, T3_APL, T3_SLOT, uoff[0], cur);
      t3_store_row<CJB, SPLIT>(slot + 2 * T3_APL, T3_BPL, T3_SLOT, uoff[1], cur + 4);
      t3_store_row<CJB, SPLIT>(slot + 2 * T3_APL, T3_BPL, T3_SLOT, uoff[2], cur + 8);
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      __syncwarp();
      if (lane == 0) t3_arrive(mb + 8 * q);
    }
    // every copy this thread issued has landed before the CTA goes on (also after an abort)
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    // the chunks not drained inside the loop, the last one included
    while (drained < nchunks && !__shfl_sync(0xffffffffu, s_abort, 0)) {
      if (!drain_next()) break;
    }
  } else if (lane == 0) {
    // ---- MMA issuer ----
    const uint32_t id_pos = t3_idesc(false), id_neg = t3_idesc(true);
    int issued = 0;
    for (int t = 0; t < ntiles; ++t) {
      const int q = t % NS;
      const int tc = t % chunk;
      if (tc == 0 && t > 0) {
        // the accumulators are reused once the previous chunk is drained
        if (!tc_wait(mb_drained, (uint32_t)((t / chunk - 1) & 1))) {
          atomicExch(err, 1);
          s_abort = 1;
        }
      }
      if (!s_abort && !tc_wait(mb + 8 * q, (uint32_t)((t / NS) & 1))) {
        atomicExch(err, 1);
        s_abort = 1;
      }
      if (s_abort) break;
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
      const uint32_t sar = ring + q * SL, sai = sar + T3_APL, sbr = sar + 2 * T3_APL, sbi = sbr + T3_BPL;
      const uint32_t lo = T3_SLOT;
      const bool acc = tc > 0;
      if (SPLIT) {
        tc_mma(d_re, t3_desc(sar), t3_desc(sbr + lo), id_pos, acc);
        tc_mma(d_re, t3_desc(sar + lo), t3_desc(sbr), id_pos, true);
        tc_mma(d_re, t3_desc(sai), t3_desc(sbi + lo), id_neg, true);
        tc_mma(d_re, t3_desc(sai + lo), t3_desc(sbi), id_neg, true);
        tc_mma(d_re, t3_desc(sar), t3_desc(sbr), id_pos, true);
        tc_mma(d_re, t3_desc(sai), t3_desc(sbi), id_neg, true);
        tc_mma(d_im, t3_desc(sar), t3_desc(sbi + lo), id_pos, acc);
        tc_mma(d_im, t3_desc(sar + lo), t3_desc(sbi), id_pos, true);
        tc_mma(d_im, t3_desc(sai), t3_desc(sbr + lo), id_pos, true);
        tc_mma(d_im, t3_desc(sai + lo), t3_desc(sbr), id_pos, true);
        tc_mma(d_im, t3_desc(sar), t3_desc(sbi), id_pos, true);
        tc_mma(d_im, t3_desc(sai), t3_desc(sbr), id_pos, true);
      } else {
        tc_mma(d_re, t3_desc(sar), t3_desc(sbr), id_pos, acc);
        tc_mma(d_re, t3_desc(sai), t3_desc(sbi), id_neg, true);
        tc_mma(d_im, t3_desc(sar), t3_desc(sbi), id_pos, acc);
        tc_mma(d_im, t3_desc(sai), t3_desc(sbr), id_pos, true);
      }
      tc_commit(mb + 8 * (NS + q));
      ++issued;
      // chunk end: the chunk barrier tracks every MMA issued so far
      if (tc == chunk - 1 || t == ntiles - 1) tc_commit(mb_chunk);
    }
    // no MMA may be in flight when the TMEM is freed, also after an abort: one more commit, on a
    // barrier of its own, tracks them all (bounded wait)
    if (issued > 0) {
      tc_commit(mb_fin);
      if (!tc_wait(mb_fin, 0u)) {
        atomicExch(err, 1);
        s_abort = 1;
      }
    }
    s_issued = issued;
  }
  __syncwarp();  // the MMA warp's lanes reconverge before the block barrier
  __syncthreads();
  bool ok = !s_abort;
  if (ok && ntiles == 0 && warp < T3_CONV_WARPS) {
    // an empty K range: the destination still receives its (zero) contribution
    t3_drain(d_re, d_im, warp, lane, false, true, M, N, r0, c0, O, ldo_r, ldo_c, alpha, beta, part, blockIdx.z);
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  if (warp == T3_CONV_WARPS) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(T3_TMEM_COLS));
}

// ---- k_cgemm_tc4: the 128 x 256 kernel on pre-split operands -----------------------------------
// The converter warps of k_cgemm_tc3 bound it (a TF32 product runs nearly as slowly as the 3xTF32
// one).  Here every operand is split once, by k_tf32_tiles, into the MMA's own shared-memory image:
// for each 8-deep K step and each plane (real hi, imaginary hi, then for 3xTF32 real lo, imaginary
// lo) the operand's 8-row groups, 256 bytes each (two 8 x 4 core matrices, the layout of t3_off), one
// after another.  A slot plane of a 128-row (256-row) tile is then one contiguous 4 KB (8 KB) block
// of global memory, fetched by one bulk copy (cp.async.bulk) that completes on the slot's mbarrier.
// Rows are padded to a multiple of 256 and K to a multiple of 8 with zeros, so no copy needs a bound.
// Warp 8 lane 0 issues the copies, warp 9 lane 0 the MMAs, warps 0-7 drain the accumulators (the
// same chunked FP64 drains as k_cgemm_tc3).  Every wait is bounded; on a timeout each role winds down
// and the producer waits (bounded) for the copies it issued before the CTA exits.
constexpr int T4_THREADS = 32 * (T3_CONV_WARPS + 2);
constexpr int T4_PRODUCER = T3_CONV_WARPS, T4_MMA = T3_CONV_WARPS + 1;
__host__ __device__ constexpr int t4_planes(bool split) { return split ? 4 : 2; }
__host__ __device__ constexpr int t4_slot(bool split) { return t4_planes(split) * (T3_APL + T3_BPL); }
__host__ __device__ constexpr int t4_stages(bool split) { return split ? 4 : 8; }
__host__ __device__ constexpr int t4_smem(bool split) { return t4_stages(split) * t4_slot(split) + 256; }

// Split of one operand into TF32 tiles: out[((ks * planes + p) * RG + rg) * 64 + w] (32-bit words),
// rg = row / 8, the word of (row, k) within its 256-byte group at t3_off(row % 8, k % 8) / 4.
// X(r, k) = X[r * ld + k] when kc, else X[k * ld + r]; conj conjugates.  hi = tf32(x) and
// lo = tf32(x - hi), the difference taken in FP64.  One thread per (row, 4-k group).
template <bool SPLIT>
__global__ void k_tf32_tiles(const double2* __restrict__ X, long ld, bool kc, bool conj, int R, int K, int RG, int KS,
                             float* __restrict__ out) {
  constexpr int NP = t4_planes(SPLIT);
  const long u = blockIdx.x * (long)blockDim.x + threadIdx.x;  // unit = ((ks * 2 + kg) * RG + rg) * 8 + r8
  const long nunits = (long)KS * 2 * RG * 8;
  if (u >= nunits) return;
  const int r8 = (int)(u & 7);
  const long v = u >> 3;
  const int rg = (int)(v % RG);
  const long w = v / RG;
  const int kg = (int)(w & 1), ks = (int)(w >> 1);
  const int row = rg * 8 + r8, k0 = ks * 8 + kg * 4;
  float hr[4], hi[4], lr[4], li[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    double2 x = make_double2(0.0, 0.0);
    if (row < R && k0 + j < K) x = kc ? X[(long)row * ld + k0 + j] : X[(long)(k0 + j) * ld + row];
    const double xr = x.x, xi = conj ? -x.y : x.y;
    hr[j] = tf32_rna((float)xr);
    hi[j] = tf32_rna((float)xi);
    lr[j] = SPLIT ? tf32_rna((float)(xr - (double)hr[j])) : 0.f;
    li[j] = SPLIT ? tf32_rna((float)(xi - (double)hi[j])) : 0.f;
  }
  const long base = (((long)ks * NP) * RG + rg) * 64 + (kg * 128 + r8 * 16) / 4;  // words
  const long pstride = (long)RG * 64;
  *reinterpret_cast<float4*>(out + base) = make_float4(hr[0], hr[1], hr[2], hr[3]);
  *reinterpret_cast<float4*>(out + base + pstride) = make_float4(hi[0], hi[1], hi[2], hi[3]);
  if (SPLIT) {
    *reinterpret_cast<float4*>(out + base + 2 * pstride) = make_float4(lr[0], lr[1], lr[2], lr[3]);
    *reinterpret_cast<float4*>(out + base + 3 * pstride) = make_float4(li[0], li[1], li[2], li[3]);
  }
}

__device__ __forceinline__ void t4_bulk(uint32_t dst, const void* src, uint32_t bytes, uint32_t mbar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(dst), "l"(src),
               "r"(bytes), "r"(mbar)
               : "memory");
}
__device__ __forceinline__ void t4_expect(uint32_t mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(mbar), "r"(bytes) : "memory");
}

template <bool SPLIT>
__global__ void __launch_bounds__(T4_THREADS, 1) k_cgemm_tc4(int M, int N, const float* __restrict__ At, int RGA,
                                                             const float* __restrict__ Bt, int RGB, int KS,
                                                             double2* __restrict__ O, long ldo_r, long ldo_c, double alpha,
                                                             double beta, int kps, double2* __restrict__ part,
                                                             int* __restrict__ err, int chunk) {
  extern __shared__ __align__(1024) unsigned char tsm4[];
  constexpr int NS = t4_stages(SPLIT);
  constexpr int SL = t4_slot(SPLIT);
  constexpr int NP = t4_planes(SPLIT);
  uint64_t* mbar = reinterpret_cast<uint64_t*>(tsm4 + NS * SL);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mbar + 2 * NS + 3);
  __shared__ volatile int s_abort;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int r0 = blockIdx.y * TC_M, c0 = blockIdx.x * T3_N;
  const int kbeg = blockIdx.z * kps;  // in K steps of 8
  const int kend = min(KS, kbeg + kps);
  const int ntiles = max(0, kend - kbeg);
  const int nchunks = (ntiles + chunk - 1) / chunk;
  const uint32_t ring = (uint32_t)__cvta_generic_to_shared(tsm4);
  const uint32_t mb = (uint32_t)__cvta_generic_to_shared(mbar);
  const uint32_t mb_chunk = mb + 16 * NS, mb_drained = mb_chunk + 8, mb_fin = mb_chunk + 16;
  if (tid == 0) {
    s_abort = 0;
    for (int q = 0; q < NS; ++q) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(mb + 8 * q));         // full: the producer's expect_tx
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(mb + 8 * (NS + q)));  // empty: the MMA commit
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(mb_chunk));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(mb_drained), "r"(T3_CONV_WARPS));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(mb_fin));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
  }
  if (warp == T4_MMA) {
    const uint32_t slot = (uint32_t)__cvta_generic_to_shared(tmem_slot);
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(slot), "r"(T3_TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  const uint32_t tmem = *tmem_slot;
  const uint32_t d_re = tmem, d_im = tmem + T3_N;
  if (warp < T3_CONV_WARPS) {
    // ---- drains ----
    for (int ch = 0; ch < nchunks; ++ch) {
      int ok = 1;
      if (lane == 0) ok = tc_wait(mb_chunk, (uint32_t)(ch & 1)) ? 1 : 0;
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) {
        if (lane == 0) atomicExch(err, 1);
        s_abort = 1;
      }
      if (__shfl_sync(0xffffffffu, s_abort, 0)) break;
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
      t3_drain(d_re, d_im, warp, lane, true, ch == 0, M, N, r0, c0, O, ldo_r, ldo_c, alpha, beta, part, blockIdx.z);
      asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
      __syncwarp();
      if (lane == 0) t3_arrive(mb_drained);
    }
  } else if (warp == T4_PRODUCER) {
    // ---- bulk copies ----
    if (lane == 0) {
      const long a_plane = (long)RGA * 64, b_plane = (long)RGB * 64;  // words per plane of a K step
      const float* a0 = At + (long)(r0 / 8) * 64;
      const float* b0 = Bt + (long)(c0 / 8) * 64;
      int issued = 0;
      for (int t = 0; t < ntiles; ++t) {
        const int q = t % NS;
        if (t >= NS && !tc_wait(mb + 8 * (NS + q), (uint32_t)((t / NS - 1) & 1))) {
          atomicExch(err, 1);
          s_abort = 1;
        }
        if (s_abort) break;
        const uint32_t full = mb + 8 * q;
        t4_expect(full, (uint32_t)SL);
        const uint32_t dst = ring + q * SL;
        const long ks = kbeg + t;
#pragma unroll
        for (int p = 0; p < NP; ++p) {
          t4_bulk(dst + p * T3_APL, a0 + (ks * NP + p) * a_plane, T3_APL, full);
          t4_bulk(dst + NP * T3_APL + p * T3_BPL, b0 + (ks * NP + p) * b_plane, T3_BPL, full);
        }
        ++issued;
      }
      // no copy may be in flight when the CTA exits: wait for the last full phase of every slot used
      for (int t = max(0, issued - NS); t < issued; ++t) {
        if (!tc_wait(mb + 8 * (t % NS), (uint32_t)((t / NS) & 1))) atomicExch(err, 1);
      }
    }
  } else if (lane == 0) {
    // ---- MMA issuer ----
    const uint32_t id_pos = t3_idesc(false), id_neg = t3_idesc(true);
    int issued = 0;
    for (int t = 0; t < ntiles; ++t) {
      const int q = t % NS;
      const int tc = t % chunk;
      if (tc == 0 && t > 0) {
        if (!tc_wait(mb_drained, (uint32_t)((t / chunk - 1) & 1))) {
          atomicExch(err, 1);
          s_abort = 1;
        }
      }
      if (!s_abort && !tc_wait(mb + 8 * q, (uint32_t)((t / NS) & 1))) {
        atomicExch(err, 1);
        s_abort = 1;
      }
      if (s_abort) break;
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
      // slot image: A planes (hi re, hi im[, lo re, lo im]) then the B planes in the same order
      const uint32_t sa = ring + q * SL, sb = sa + NP * T3_APL;
      const uint32_t sar = sa, sai = sa + T3_APL, sbr = sb, sbi = sb + T3_BPL;
      const bool acc = tc > 0;
      if (SPLIT) {
        const uint32_t arl = sa + 2 * T3_APL, ail = sa + 3 * T3_APL, brl = sb + 2 * T3_BPL, bil = sb + 3 * T3_BPL;
        tc_mma(d_re, t3_desc(sar), t3_desc(brl), id_pos, acc);
        tc_mma(d_re, t3_desc(arl), t3_desc(sbr), id_pos, true);
        tc_mma(d_re, t3_desc(sai), t3_desc(bil), id_neg, true);
        tc_mma(d_re, t3_desc(ail), t3_desc(sbi), id_neg, true);
        tc_mma(d_re, t3_desc(sar), t3_desc(sbr), id_pos, true);
        tc_mma(d_re, t3_desc(sai), t3_desc(sbi), id_neg, true);
        tc_mma(d_im, t3_desc(sar), t3_desc(bil), id_pos, acc);
        tc_mma(d_im, t3_desc(arl), t3_desc(sbi), id_pos, true);
        tc_mma(d_im, t3_desc(sai), t3_desc(brl), id_pos, true);
        tc_mma(d_im, t3_desc(ail), t3_desc(sbr), id_pos, true);
        tc_mma(d_im, t3_desc(sar), t3_desc(sbi), id_pos, true);
        tc_mma(d_im, t3_desc(sai), t3_desc(sbr), id_pos, true);
      } else {
        tc_mma(d_re, t3_desc(sar), t3_desc(sbr), id_pos, acc);
        tc_mma(d_re, t3_desc(sai), t3_desc(sbi), id_neg, true);
        tc_mma(d_im, t3_desc(sar), t3_desc(sbi), id_pos, acc);
        tc_mma(d_im, t3_desc(sai), t3_desc(sbr), id_pos, true);
      }
      tc_commit(mb + 8 * (NS + q));
      ++issued;
      if (tc == chunk - 1 || t == ntiles - 1) tc_commit(mb_chunk);
    }
    if (issued > 0) {
      tc_commit(mb_fin);
      if (!tc_wait(mb_fin, 0u)) {
        atomicExch(err, 1);
        s_abort = 1;
      }
    }
  }
  __syncwarp();
  __syncthreads();
  if (!s_abort && ntiles == 0 && warp < T3_CONV_WARPS)
    t3_drain(d_re, d_im, warp, lane, false, true, M, N, r0, c0, O, ldo_r, ldo_c, alpha, beta, part, blockIdx.z);
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  if (warp == T4_MMA) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(T3_TMEM_COLS));
}

// Sum of the column-major split-K partials of k_cgemm_tc3 into the output.
__global__ void k_cgemm_reduce_cm(int M, int N, int splits, const double2* __restrict__ part, double2* __restrict__ O,
                                  long ldo_r, long ldo_c, double alpha, double beta) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= (long)M * N) return;
  const int c = (int)(i / M), r = (int)(i - (long)c * M);
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

// Split-K of the 128 x 256 kernel (one CTA per SM): the fewest splits whose CTAs fill at least 85 %
// of their waves on 148 SMs and three quarters of one wave, else the best wave fill; at least 512 K
// per split.
static int t3_splits(int M, int N, int K) {
  const long tiles = (long)ceil_div(M, TC_M) * ceil_div(N, T3_N);
  const long wave = 148;
  if (tiles >= wave || K < 1024) return 1;
  const long maxs = std::max<long>(1, std::min<long>(K / 512, 64));
  long best = 1;
  double best_eff = 0.0;
  for (long sp = 1; sp <= maxs; ++sp) {
    const long ctas = tiles * sp;
    const double eff = (double)ctas / (double)(((ctas + wave - 1) / wave) * wave);
    if (eff >= 0.85 && ctas * 4 >= wave * 3) return (int)sp;
    const double score = eff * std::min(1.0, (double)ctas / wave);
    if (score > best_eff + 1e-9) {
      best_eff = score;
      best = sp;
    }
  }
  return (int)best;
}

// DFTCUDA_TC=v1 / v2 select the earlier 128 x 64 kernels for every shape (A/B measurements).
static int tc_variant() {
  static const int v = [] {
    const char* e = std::getenv("DFTCUDA_TC");
    if (e && std::string(e) == "v1") return 1;
    if (e && std::string(e) == "v2") return 2;
    return 3;
  }();
  return v;
}

// Accumulation chunk of the wide kernel in K steps (DFTCUDA_TC_CHUNK overrides, for measurements).
static int t3_chunk() {
  static const int c = [] {
    const char* e = std::getenv("DFTCUDA_TC_CHUNK");
    const int v = e ? std::atoi(e) : 0;
    return v >= 1 ? v : T3_CHUNK;
  }();
  return c;
}

struct TcPlan {
  GemmArgs g;      // the problem as run (possibly transposed)
  bool wide;       // k_cgemm_tc3 (128 x 256 tiles) rather than the 128 x 64 kernels
  int splits;      // heuristic split-K count before the workspace clamp
};

// out(r, c) = sum_k A(r, k) B(c, k) is also out^T(c, r) = sum_k B(c, k) A(r, k).  With both output
// dimensions at 128 or more the wide kernel runs, oriented so consecutive tile rows are consecutive
// output addresses (coalesced FP64 stores).  Otherwise, with fewer rows than one 128-row MMA tile
// and more columns, the transpose runs so the wide dimension fills the MMA's M (the
// back-projection: rows = bands, columns = plane waves).
static TcPlan tc_plan(const GemmArgs& g0) {
  auto transposed = [](const GemmArgs& a) {
    GemmArgs g = a;
    g.M = a.N; g.N = a.M;
    g.A = a.B; g.lda = a.ldb; g.a_kc = a.b_kc; g.conj_a = a.conj_b;
    g.B = a.A; g.ldb = a.lda; g.b_kc = a.a_kc; g.conj_b = a.conj_a;
    g.ldo_r = a.ldo_c; g.ldo_c = a.ldo_r;
    g.a_cache = a.b_cache; g.b_cache = a.a_cache;
    return g;
  };
  TcPlan p{g0, false, 1};
  if (tc_variant() == 3 && g0.M >= TC_M && g0.N >= TC_M) {
    p.wide = true;
    if (g0.ldo_c == 1 && g0.ldo_r != 1) p.g = transposed(g0);
    p.splits = t3_splits(p.g.M, p.g.N, p.g.K);
    return p;
  }
  if (g0.M < TC_M && g0.N > g0.M) p.g = transposed(g0);
  p.splits = tc_splits(p.g.M, p.g.N, p.g.K);
  return p;
}

size_t tc4_operand_bytes(int R, int K, bool split) {
  const size_t KS = ((size_t)K + 7) / 8, RG = ((size_t)R + 255) / 256 * 32;
  return KS * t4_planes(split) * RG * 256;
}

size_t cgemm_tf32_workspace_elems(int M, int N, int K) {
  GemmArgs g{};
  g.M = M; g.N = N; g.K = K; g.ldo_r = 1; g.ldo_c = M;
  size_t need = 0;
  for (int o = 0; o < 2; ++o) {  // either output orientation
    if (o == 1) { g.ldo_r = N; g.ldo_c = 1; }
    const TcPlan p = tc_plan(g);
    if (p.splits > 1) need = std::max(need, (size_t)p.splits * M * N);
  }
  return need;
}

template <bool AKC, bool BKC, bool CJA, bool CJB, bool SPLIT>
static void tc_launch(const GemmArgs& g, dim3 grid, int kps, double2* part, int* err, cudaStream_t s) {
  ensure_max_dynamic_smem((const void*)k_cgemm_tf32<AKC, BKC, CJA, CJB, SPLIT>, tc_smem(SPLIT));
  k_cgemm_tf32<AKC, BKC, CJA, CJB, SPLIT><<<grid, TC_THREADS, tc_smem(SPLIT), s>>>(
      g.M, g.N, g.K, g.A, g.lda, g.B, g.ldb, g.O, g.ldo_r, g.ldo_c, g.alpha, g.beta, kps, part, err);
  count_launch();
}

template <bool AKC, bool BKC, bool CJA, bool CJB, bool SPLIT>
static void tc2_launch(const GemmArgs& g, dim3 grid, int kps, double2* part, int* err, cudaStream_t s) {
  ensure_max_dynamic_smem((const void*)k_cgemm_tc2<AKC, BKC, CJA, CJB, SPLIT>, t2_smem(SPLIT));
  k_cgemm_tc2<AKC, BKC, CJA, CJB, SPLIT><<<grid, T2_THREADS, t2_smem(SPLIT), s>>>(
      g.M, g.N, g.K, g.A, g.lda, g.B, g.ldb, g.O, g.ldo_r, g.ldo_c, g.alpha, g.beta, kps, part, err);
  count_launch();
}

template <bool AKC, bool BKC, bool CJA, bool CJB, bool SPLIT>
static void tc3_launch(const GemmArgs& g, dim3 grid, int kps, double2* part, int* err, cudaStream_t s) {
  ensure_max_dynamic_smem((const void*)k_cgemm_tc3<AKC, BKC, CJA, CJB, SPLIT>, t3_smem(SPLIT));
  k_cgemm_tc3<AKC, BKC, CJA, CJB, SPLIT><<<grid, T3_THREADS, t3_smem(SPLIT), s>>>(
      g.M, g.N, g.K, g.A, g.lda, g.B, g.ldb, g.O, g.ldo_r, g.ldo_c, g.alpha, g.beta, kps, part, err, t3_chunk());
  count_launch();
}

template <bool AKC, bool BKC, bool CJA, bool CJB, bool SPLIT>
static void tc_any(const GemmArgs& g, bool wide, dim3 grid, int kps, double2* part, int* err, cudaStream_t s) {
  if (wide) tc3_launch<AKC, BKC, CJA, CJB, SPLIT>(g, grid, kps, part, err, s);
  else if (tc_variant() == 1) tc_launch<AKC, BKC, CJA, CJB, SPLIT>(g, grid, kps, part, err, s);
  else tc2_launch<AKC, BKC, CJA, CJB, SPLIT>(g, grid, kps, part, err, s);
}

template <bool SPLIT>
static int tc_dispatch(const GemmArgs& g, bool wide, dim3 grid, int kps, double2* part, int* err_dev, cudaStream_t s) {
  const int key = (g.a_kc ? 8 : 0) | (g.b_kc ? 4 : 0) | (g.conj_a ? 2 : 0) | (g.conj_b ? 1 : 0);
  switch (key) {
    case 12: tc_any<true, true, false, false, SPLIT>(g, wide, grid, kps, part, err_dev, s); break;   // projection
    case 1: tc_any<false, false, false, true, SPLIT>(g, wide, grid, kps, part, err_dev, s); break;   // back-projection
    case 14: tc_any<true, true, true, false, SPLIT>(g, wide, grid, kps, part, err_dev, s); break;    // Gram V^H W
    case 4: tc_any<false, true, false, false, SPLIT>(g, wide, grid, kps, part, err_dev, s); break;   // V C, transposed
    case 8: tc_any<true, false, false, false, SPLIT>(g, wide, grid, kps, part, err_dev, s); break;   // V C
    case 0: tc_any<false, false, false, false, SPLIT>(g, wide, grid, kps, part, err_dev, s); break;
    case 2: tc_any<false, false, true, false, SPLIT>(g, wide, grid, kps, part, err_dev, s); break;    // back-projection, transposed
    case 13: tc_any<true, true, false, true, SPLIT>(g, wide, grid, kps, part, err_dev, s); break;    // Gram, transposed
    default: return fail(DFTCUDA_ERR_UNSUPPORTED, "cgemm_tf32: operand layout not instantiated");
  }
  return DFTCUDA_OK;
}

// DFTCUDA_TC=v3 keeps the wide products on k_cgemm_tc3 (operands converted inside the GEMM) for A/B
// measurements; otherwise, with a scratch buffer, they run on pre-split operands (k_cgemm_tc4).
static bool tc4_enabled() {
  static const bool v = [] {
    const char* e = std::getenv("DFTCUDA_TC");
    return !(e && (std::string(e) == "v1" || std::string(e) == "v2" || std::string(e) == "v3"));
  }();
  return v;
}

static int tc4_run(const GemmArgs& g, cudaStream_t s, double2* ws, size_t ws_elems, int* err_dev, bool split, TcScratch* scratch) {
  const int np = t4_planes(split);
  const int RGA = (int)(((size_t)g.M + 255) / 256 * 32), RGB = (int)(((size_t)g.N + 255) / 256 * 32);
  const int KS = (g.K + 7) / 8;
  const size_t a_bytes = (size_t)KS * np * RGA * 256, b_bytes = (size_t)KS * np * RGB * 256;
  // an operand goes to its cache (split once while the cache holds it) or to the per-call scratch
  auto key_of = [&](const double2* X, long ld, bool kc, bool cj, int R) {
    unsigned long long h = (unsigned long long)(uintptr_t)X;
    for (unsigned long long v : {(unsigned long long)ld, (unsigned long long)kc, (unsigned long long)cj, (unsigned long long)R,
                                 (unsigned long long)g.K, (unsigned long long)split})
      h = h * 1000003ULL ^ v;
    return h;
  };
  DFT_TRY(scratch->ensure((g.a_cache ? 0 : a_bytes) + (g.b_cache ? 0 : b_bytes)));
  unsigned char* sp = static_cast<unsigned char*>(scratch->p);
  auto place = [&](TcScratch* cache, size_t bytes, const double2* X, long ld, bool kc, bool cj, int R, int RG,
                   float** out) -> int {
    bool convert = true;
    if (cache) {
      const unsigned long long key = key_of(X, ld, kc, cj, R);
      if (cache->valid && cache->key == key && cache->bytes >= bytes) convert = false;
      else {
        cache->valid = false;
        DFT_TRY(cache->ensure(bytes));
        cache->key = key;
        cache->valid = true;
      }
      *out = reinterpret_cast<float*>(cache->p);
    } else {
      *out = reinterpret_cast<float*>(sp);
      sp += bytes;
    }
    if (convert) {
      const long units = (long)KS * 2 * RG * 8;
      if (split) k_tf32_tiles<true><<<ceil_div(units, 256), 256, 0, s>>>(X, ld, kc, cj, R, g.K, RG, KS, *out);
      else k_tf32_tiles<false><<<ceil_div(units, 256), 256, 0, s>>>(X, ld, kc, cj, R, g.K, RG, KS, *out);
      count_launch();
    }
    return DFTCUDA_OK;
  };
  float *At = nullptr, *Bt = nullptr;
  DFT_TRY(place(g.a_cache, a_bytes, g.A, g.lda, g.a_kc, g.conj_a, g.M, RGA, &At));
  DFT_TRY(place(g.b_cache, b_bytes, g.B, g.ldb, g.b_kc, g.conj_b, g.N, RGB, &Bt));
  int splits = g.splits > 0 ? std::min(g.splits, std::max(1, KS / 4)) : t3_splits(g.M, g.N, g.K);
  if (splits > 1) splits = (int)std::max<size_t>(1, std::min<size_t>(splits, ws_elems / ((size_t)g.M * g.N)));
  const int kps = (KS + splits - 1) / splits;  // K steps per split
  splits = (KS + kps - 1) / kps;
  const dim3 grid(ceil_div(g.N, T3_N), ceil_div(g.M, TC_M), splits);
  double2* part = splits > 1 ? ws : nullptr;
  if (split) {
    DFT_TRY(ensure_max_dynamic_smem((const void*)k_cgemm_tc4<true>, t4_smem(true)));
    k_cgemm_tc4<true><<<grid, T4_THREADS, t4_smem(true), s>>>(g.M, g.N, At, RGA, Bt, RGB, KS, g.O, g.ldo_r, g.ldo_c, g.alpha, g.beta,
                                                              kps, part, err_dev, t3_chunk());
  } else {
    DFT_TRY(ensure_max_dynamic_smem((const void*)k_cgemm_tc4<false>, t4_smem(false)));
    k_cgemm_tc4<false><<<grid, T4_THREADS, t4_smem(false), s>>>(g.M, g.N, At, RGA, Bt, RGB, KS, g.O, g.ldo_r, g.ldo_c, g.alpha, g.beta,
                                                                kps, part, err_dev, t3_chunk());
  }
  count_launch();
  if (part) {
    const long tot = (long)g.M * g.N;
    k_cgemm_reduce_cm<<<ceil_div(tot, 256), 256, 0, s>>>(g.M, g.N, splits, part, g.O, g.ldo_r, g.ldo_c, g.alpha, g.beta);
    count_launch();
  }
  DFT_CUDA_TRY(cudaGetLastError());
  return DFTCUDA_OK;
}

int TcScratch::ensure(size_t need) {
  if (need <= bytes) return DFTCUDA_OK;
  if (p) cudaFree(p);
  p = nullptr;
  bytes = 0;
  valid = false;
  if (dev_malloc(&p, need) != cudaSuccess) return fail(DFTCUDA_ERR_OUT_OF_MEMORY, "tensor-core operand tiles");
  bytes = need;
  return DFTCUDA_OK;
}

void TcScratch::release() {
  if (p) cudaFree(p);
  p = nullptr;
  bytes = 0;
  valid = false;
}

int cgemm_tf32(const GemmArgs& g0, cudaStream_t s, double2* ws, size_t ws_elems, int* err_dev, bool split, TcScratch* scratch) {
  if (g0.M <= 0 || g0.N <= 0) return DFTCUDA_OK;
  if (g0.K <= 0) return fail(DFTCUDA_ERR_INVALID_ARGUMENT, "cgemm_tf32: K must be positive");
  const TcPlan p = tc_plan(g0);
  const GemmArgs& g = p.g;
  if (p.wide && scratch && tc4_enabled()) return tc4_run(g, s, ws, ws_elems, err_dev, split, scratch);
  int splits = g.splits > 0 ? std::min(g.splits, std::max(1, g.K / 32)) : p.splits;
  if (splits > 1) splits = (int)std::max<size_t>(1, std::min<size_t>(splits, ws_elems / ((size_t)g.M * g.N)));  // what fits the workspace
  int kps = (g.K + splits - 1) / splits;
  kps = ((kps + TC_K - 1) / TC_K) * TC_K;  // a multiple of every kernel's K slice
  splits = (g.K + kps - 1) / kps;
  const dim3 grid(ceil_div(g.N, p.wide ? T3_N : TC_N), ceil_div(g.M, TC_M), splits);
  double2* part = splits > 1 ? ws : nullptr;
  DFT_TRY(split ? tc_dispatch<true>(g, p.wide, grid, kps, part, err_dev, s)
                : tc_dispatch<false>(g, p.wide, grid, kps, part, err_dev, s));
  if (part) {
    const long tot = (long)g.M * g.N;
    if (p.wide) {
      k_cgemm_reduce_cm<<<ceil_div(tot, 256), 256, 0, s>>>(g.M, g.N, splits, part, g.O, g.ldo_r, g.ldo_c, g.alpha, g.beta);
    } else {
      k_cgemm_reduce<<<ceil_div(tot, 256), 256, 0, s>>>(g.M, g.N, splits, part, g.O, g.ldo_r, g.ldo_c, g.alpha, g.beta);
    }
    count_launch();
  }
  DFT_CUDA_TRY(cudaGetLastError());
  return DFTCUDA_OK;
}

}  // namespace dftcuda
