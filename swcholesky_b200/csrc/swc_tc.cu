// Trailing SYRK/GEMM step of the mixed (split-TF32) factorization on the 5th-generation
// tensor cores: tcgen05.mma kind::tf32, operands in shared memory, accumulator in TMEM.
//
// A 64x64 tile update C = A B^T by one 64-column block (A = rows r0.. of the block, B = rows
// c0..) is computed from the split mirror ({hi, lo} TF32 pairs): viewed as 128-row
// operands A' (row 2i = hi of row i, row 2i+1 = lo) and B', one 128x128x64 TF32 product
// D' = A' B'^T holds every partial product, and C(i, j) = sum of the 2x2 block
// D'(2i..2i+1, 2j..2j+1) = hi*hi' + hi*lo' + lo*hi' + lo*lo' (FP32 accumulation, about
// 2^-22 relative error, the accuracy of the split representation).  The tile's FP64 value
// is then updated in place: tile -= C, lower triangle only.
//
// Per CTA (128 threads, grid-stride over the step's tiles): warp 0 allocates 128 TMEM
// columns once; per tile every thread stages its share of A' and B' (cp.async, 4 bytes per
// TF32 value) into the K-major canonical layout without swizzle (core matrices of 8 rows x
// 16 bytes; 8-row groups SBO apart, 4-column groups LBO apart), one thread issues the 8
// MMAs (K = 8 each) and commits them to an mbarrier, every warp reads its 32 TMEM lanes
// (tcgen05.ld 32x32b) and folds the 2x2 blocks with one shuffle.  The wait on the
// mbarrier is bounded; on a timeout the CTA records it in status[3] and stops.
#include <cuda_runtime.h>

#include <cstdint>

#include "swc_engine.h"

namespace swc {

namespace {

constexpr int TCT = 128;                        // threads
constexpr int TC_K = TB;                        // K of one step: one column block
constexpr int TC_LBO = 128;                     // bytes between 4-column groups (K)
constexpr int TC_SBO = (TC_K / 4) * TC_LBO;     // bytes between 8-row groups (M)
constexpr int TC_OPB = (2 * TB / 8) * TC_SBO;   // bytes per 128-row operand
constexpr int TC_SMEM = 2 * TC_OPB;             // A' and B'
constexpr int TC_COLS = 128;                    // TMEM columns (D' is 128 x 128 FP32)
// instruction descriptor: D F32, A and B TF32, both K-major, N = 128, M = 128
constexpr uint32_t TC_IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((128u >> 3) << 17) |
                              ((128u >> 4) << 24);
constexpr long long TC_SPIN = 1LL << 24;

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// shared-memory matrix descriptor: start, LBO, SBO (16-byte units), version 1, no swizzle
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((TC_LBO >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((TC_SBO >> 4) & 0x3FFF) << 32) | ((uint64_t)1 << 46);
}

__device__ __forceinline__ void cp_async4(uint32_t dst, const void *src, bool pred) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(dst), "l"(src),
               "r"(pred ? 4 : 0));
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase) {
  uint32_t done = 0;
  for (long long it = 0; it < TC_SPIN && !done; ++it)
    asm volatile(
        "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(phase)
        : "memory");
  return done != 0;
}

__global__ void __launch_bounds__(TCT) k_syrk_step_tc(DevSym S, const int4 *tasks, int count,
                                                      int step) {
  extern __shared__ __align__(128) unsigned char sm[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tbase;
  __shared__ int failed;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  unsigned char *As = sm, *Bs = sm + TC_OPB;
  const uint32_t bar = smem_addr(&mbar);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_addr(&tbase)),
                 "r"(TC_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid == 0) {
    failed = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = tbase;
  uint32_t phase = 0;
  for (int t = blockIdx.x; t < count; t += gridDim.x) {
    const int4 tk = tasks[t];
    const int s = tk.x, r0 = tk.y, c0 = tk.z;
    const int w = S.super[s + 1] - S.super[s];
    const int m = (int)(S.rowptr[s + 1] - S.rowptr[s]);
    const int k0 = step * TB;
    const int nrow = min(TB, m - r0), ncol = min(TB, w - c0);
    const float2 *Lf = S.Lf + S.xptr[s];
    // stage A' and B': value (row i, column k, piece p) -> row' 2i + p.  A warp fills one
    // core matrix (8 rows' x 4 columns = 32 words) per copy: lane = (piece, row, column) so
    // the 32 shared-memory words are distinct banks and the global reads are 4 runs of 32 B
    {
      const int p = lane & 1, ii = (lane >> 1) & 3, kk = lane >> 3;
      const uint32_t in_core = (uint32_t)(2 * ii + p) * 16 + (uint32_t)kk * 4;
      for (int cm = warp; cm < (2 * TB / 8) * (TC_K / 4); cm += TCT / 32) {
        const int gm = cm >> 4, gk = cm & 15;   // 8-row' group, 4-column group
        const int i = 4 * gm + ii, k = 4 * gk + kk;
        const uint32_t off = (uint32_t)gm * TC_SBO + (uint32_t)gk * TC_LBO + in_core;
        const size_t col = (size_t)(k0 + k) * m;
        cp_async4(smem_addr(As + off), i < nrow ? (const float *)(Lf + col + r0 + i) + p : (const float *)Lf, i < nrow);
        cp_async4(smem_addr(Bs + off), i < ncol ? (const float *)(Lf + col + c0 + i) + p : (const float *)Lf, i < ncol);
      }
    }
    asm volatile("cp.async.commit_group;\n" ::);
    asm volatile("cp.async.wait_group 0;\n" ::);
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    if (tid == 0) {
#pragma unroll
      for (int g = 0; g < TC_K / 8; ++g) {
        const uint64_t da = tc_desc(smem_addr(As + g * 2 * TC_LBO));
        const uint64_t db = tc_desc(smem_addr(Bs + g * 2 * TC_LBO));
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(
                tmem),
            "l"(da), "l"(db), "r"(TC_IDESC), "r"(g > 0 ? 1u : 0u), "r"(0), "r"(0), "r"(0), "r"(0));
      }
      asm volatile(
          "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar)
          : "memory");
    }
    if (!mbar_wait(bar, phase)) {
      atomicExch(&S.status[3], 1);
      failed = 1;
    }
    phase ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    // epilogue: warp w reads rows' 32w.. (tile rows i = 16w + lane/2); the two lanes of a
    // row pair fold their halves and update alternate columns of the FP64 tile
    double *P = S.L + S.xptr[s];
    const int i = 16 * warp + (lane >> 1);
#pragma unroll 1
    for (int cc = 0; cc < 2 * TB; cc += 32) {
      uint32_t r[32];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
          "%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
            "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
            "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
            "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
            "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
            "=r"(r[31])
          : "r"(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)cc));
      asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
      float v[16];
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        v[q] = __uint_as_float(r[2 * q]) + __uint_as_float(r[2 * q + 1]);
        v[q] += __shfl_xor_sync(0xffffffffu, v[q], 1);
      }
      // lane parity picks the columns: j = cc/2 + q for q of that parity
      double old[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int j = cc / 2 + 2 * u + (lane & 1);
        old[u] = (i < nrow && j < ncol && r0 + i >= c0 + j) ? P[(size_t)(c0 + j) * m + r0 + i] : 0.0;
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int j = cc / 2 + 2 * u + (lane & 1);
        const float cv = (lane & 1) ? v[2 * u + 1] : v[2 * u];
        if (i < nrow && j < ncol && r0 + i >= c0 + j)
          P[(size_t)(c0 + j) * m + r0 + i] = old[u] - (double)cv;
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();   // shared operands and TMEM free for the next tile
    if (failed) break;
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  }
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TC_COLS));
}

}  // namespace

bool tc_configure(std::string &err) {
  cudaError_t e = cudaFuncSetAttribute(k_syrk_step_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       TC_SMEM);
  if (e != cudaSuccess) {
    err = std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e);
    return false;
  }
  return true;
}

int syrk_tc_ctas(int count) {
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_syrk_step_tc, TCT, TC_SMEM) !=
          cudaSuccess || per < 1)
    per = 1;
  // two per SM: the CTAs stay resident for the whole step, and the next diagonal block's
  // kernel (concurrent, on the second stream) must still find room on every SM
  per = per > 2 ? 2 : per;
  return count < sms * per ? count : sms * per;
}

void launch_syrk_step_tc(const DevSym &S, const int4 *tasks, int count, int ctas, int step,
                         cudaStream_t st) {
  if (count > 0) k_syrk_step_tc<<<ctas, TCT, TC_SMEM, st>>>(S, tasks, count, step);
}

}  // namespace swc
