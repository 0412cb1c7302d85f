// Split-TF32 Schur updates of the tiled class on the 5th-generation tensor cores.
//
// The reference forms every update of a target supernode from a descendant as a dense
// SYRK + GEMM into a contribution buffer and scatters it through relative indices
// (cholesky/sw_parallel_PB_Cholesky_05.c:299-378).  Here a 64x64 tile of a target panel
// owns its updates: for every (tile, descendant) pair the descendant's rows that fall in
// the tile are GATHERED by the tensor memory accelerator straight into the tile's own row
// and column positions, so the product lands in the tile's coordinates and no scatter is
// needed; the tile leaves the chip once, after all its descendants.  The same kernel runs
// the trailing SYRK/GEMM steps of the blocked dense factorization of wide supernodes (a
// "pair" whose descendant is the supernode itself and whose K range is one 64-column block).
//
// Operands: the split mirror of L in K-major form.  Every value x of supernode d (md rows,
// wd columns, pitch wp = wd rounded up to 4) is stored as hi = tf32(x) in row r of the hi
// plane and lo = tf32(x - hi) in row md + r of the lo plane (rows of wp floats).  One 2D
// tensor map per supernode covers both planes ({wd, 2 md}, 128-byte swizzle); a
// cp.async.bulk.tensor ... tile::gather4 load copies four rows of 32 values (any four
// row coordinates: a row outside the map, used for tile rows no descendant row feeds,
// reads zeros) into one half of a 1024-byte swizzle atom.  A stage holds the 128-row
// operands A' and B' of one 32-column K chunk: atom a holds tile rows 4a..4a+3, hi pieces
// in its first 512 bytes and lo pieces in its second.
//
// Product: one tcgen05.mma kind::tf32 with M = N = 128 and K = 8 multiplies A' by B'^T, so
// the accumulator D' (128 x 128 FP32 in TMEM) holds all four piece products of every
// (row, column) pair: C(i, j) = hi hi' + hi lo' + lo hi' + lo lo', about 2^-22 relative
// error (the accuracy of the split); the four entries are folded in the epilogue.
//
// Roles (192 threads, one CTA per SM, persistent over the tile list):
//   warp 4   producer: per K chunk, waits for a free stage, arms its "full" mbarrier with
//            the stage's byte count and issues 64 gather4 loads (two per lane);
//   warp 5   MMA issuer (one thread): per chunk, waits for the stage, issues 4 MMAs into
//            one of two TMEM accumulators and commits the stage back to the producer;
//            after a group of descendants (at least 8 chunks, or the tile's last) commits
//            the accumulator to the epilogue and switches to the other one;
//   warps 0-3 epilogue (TMEM lane quarter = warp): per group, reads the accumulator,
//            folds the pieces, adds it in FP64 to the tile held in registers (seeded with
//            minus the tile's FP64 values), releases the accumulator; stores the tile
//            once per tile.  The next tile's FP64 values load while the MMAs of its first
//            group run.
// Every wait is bounded; a wait that runs out sets status[3] and an abort flag that stops
// the other roles; the kernel then waits (bounded) for its copies and MMAs in flight,
// frees its TMEM and returns.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "swc_engine.h"

namespace swc {

namespace {

// threads: 4 epilogue warps, the producer warp(s), the MMA warp
constexpr int ut_threads(bool tma) { return 32 * (tma ? 6 : 9); }
constexpr int UT_STAGES = 4;
constexpr int UT_KCHUNK = 32;                       // K columns per stage (128 bytes of TF32)
constexpr int UT_OPB = 16 * 1024;                   // bytes of one 128-row operand chunk
constexpr int UT_STAGE_BYTES = 2 * UT_OPB;          // A' and B'
constexpr int UT_SMEM = UT_STAGES * UT_STAGE_BYTES + 1024;   // + alignment slack
constexpr int UT_TMEM_COLS = 256;                   // two 128-column FP32 accumulators
constexpr int UT_GROUP_CHUNKS = 8;                  // chunks of one FP32 accumulation group
constexpr unsigned long long UT_WAIT_NS = 2000000000ULL;   // a pipeline wait gives up after 2 s
// instruction descriptor: D F32, A and B TF32, both K-major, N = 128, M = 128
constexpr uint32_t UT_IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((128u >> 3) << 17) |
                              ((128u >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor, K-major operand with the 128-byte swizzle: 8-row groups
// 1024 bytes apart (SBO), leading offset 16 bytes (unused by this layout), version 1.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
  return t;
}

// Bounded wait for the phase of the given parity; false when it ran out (after UT_WAIT_NS,
// recorded in status[3] and the abort flag) or another role aborted.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int *abort_flag,
                                          int *status) {
  if (mbar_try(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (long long it = 1;; ++it) {
    if (mbar_try(bar, parity)) return true;
    if ((it & 63) == 0) {
      if (*abort_flag) return false;
      if (global_ns() - t0 > UT_WAIT_NS) {
        *abort_flag = 1;
        atomicExch(&status[3], 1);
        return false;
      }
    }
  }
}

// The same wait done by lane 0 of a warp for the whole warp (a warp-uniform result, so the
// .sync.aligned instructions after it see every lane).
__device__ __forceinline__ bool mbar_wait_warp(uint32_t bar, uint32_t parity,
                                               volatile int *abort_flag, int *status) {
  int ok = 1;
  if ((threadIdx.x & 31) == 0) ok = mbar_wait(bar, parity, abort_flag, status);
  ok = __shfl_sync(0xffffffffu, ok, 0);
  __syncwarp();
  return ok != 0;
}

// Bounded wait used while shutting down (ignores the abort flag).
__device__ __forceinline__ void mbar_drain(uint32_t bar, uint32_t parity, int *status) {
  const unsigned long long t0 = global_ns();
  for (long long it = 0;; ++it) {
    if (mbar_try(bar, parity)) return;
    if ((it & 63) == 63 && global_ns() - t0 > UT_WAIT_NS) break;
  }
  atomicExch(&status[3], 1);
}

__device__ __forceinline__ void tma_gather4(uint32_t dst, const CUtensorMap *map, uint32_t bar,
                                            int x, int y0, int y1, int y2, int y3) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];\n" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y0), "r"(y1), "r"(y2), "r"(y3), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem, uint64_t adesc, uint64_t bdesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
      "l"(adesc), "l"(bdesc), "r"(UT_IDESC), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}
__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar)
      : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t addr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(addr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int q = 0; q < 32; ++q) v[q] = __uint_as_float(r[q]);
}

// K chunks of a pair, and whether the accumulation group closes after it.
__device__ __forceinline__ int pair_chunks(const TcPair &pr) {
  return ((pr.kk >> 16) + UT_KCHUNK - 1) / UT_KCHUNK;
}

// Row coordinate of tile row i of the pair's operand (mask, first source row s0) in the
// map of a supernode with md rows: plane p (0 hi, 1 lo), or a row outside the map (zeros)
// when no source row feeds it.
__device__ __forceinline__ int gather_row(uint64_t mask, int s0, int i, int p, int md) {
  if (!((mask >> i) & 1ull)) return 2 * md;
  const int rank = __popcll(mask & ((1ull << i) - 1ull));
  return p * md + s0 + rank;
}

// 16-byte copy global -> shared with zero fill beyond `bytes` (0..16) of the source.
__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, int bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(bytes)
               : "memory");
}

// TMA = true: one producer warp stages with tile::gather4 loads; false: four producer warps
// stage with 16-byte cp.async copies into the same swizzled layout and hand each stage to
// the MMA warp through its mbarrier after a proxy fence.
template <bool TMA>
__global__ void __launch_bounds__(ut_threads(TMA), 1)
    k_update_tc(DevSym S, const CUtensorMap *__restrict__ maps, const int4 *__restrict__ tasks,
                const int *__restrict__ task_end, const TcPair *__restrict__ pairs, int count) {
  constexpr int NPROD = TMA ? 1 : 4;          // producer warps: 4 .. 3 + NPROD
  constexpr int MMA_WARP = 4 + NPROD;
  extern __shared__ unsigned char ut_dyn[];
  __shared__ __align__(8) uint64_t full_bar[UT_STAGES], empty_bar[UT_STAGES];
  __shared__ __align__(8) uint64_t accf_bar[2], acce_bar[2], done_bar;
  __shared__ uint32_t tmem_base;
  __shared__ volatile int abort_flag;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // 1024-byte aligned stages (the swizzle atoms must be)
  const uint32_t sbase = (smem_u32(ut_dyn) + 1023u) & ~1023u;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(&tmem_base)),
                 "r"(UT_TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid == 32 * MMA_WARP) {
    for (int s = 0; s < UT_STAGES; ++s) {
      mbar_init(smem_u32(&full_bar[s]), TMA ? 1 : NPROD);
      mbar_init(smem_u32(&empty_bar[s]), 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(smem_u32(&accf_bar[b]), 1);
      mbar_init(smem_u32(&acce_bar[b]), 4);
    }
    mbar_init(smem_u32(&done_bar), 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = tmem_base;

  if (!TMA && warp >= 4 && warp < 4 + NPROD) {
    // ------------------------- producers (cp.async) ------------------------
    // warp pw fills rows' 32 pw .. 32 pw + 31 of A' and B': per instruction four rows' of
    // 128 bytes (lane = row' (lane / 8), 16-byte chunk lane % 8), swizzled as the MMA reads
    // them; a chunk completes two chunks later (wait_group 2), then proxy fence and arrival.
    const int pw = warp - 4;
    int stage = 0;
    uint32_t phase = 0;
    int pend[2] = {-1, -1};   // stages issued one and two chunks ago
    bool ok = true;
    const float *mir = reinterpret_cast<const float *>(S.Lf);
    const int c = lane & 7;
    for (int t = blockIdx.x; t < count && ok; t += gridDim.x) {
      const int p_end = task_end[t];
      for (int q = tasks[t].w; q < p_end && ok; ++q) {
        const TcPair pr = pairs[q];
        const int wd = S.super[pr.d + 1] - S.super[pr.d], wp = (wd + 3) & ~3;
        const int md = (int)(S.rowptr[pr.d + 1] - S.rowptr[pr.d]);
        const float *base = mir + S.xk[pr.d];
        const int k0 = pr.kk & 0xffff, kend = k0 + (pr.kk >> 16);
        for (int k = k0; k < kend; k += UT_KCHUNK) {
          if (!mbar_wait_warp(smem_u32(&empty_bar[stage]), phase ^ 1u, &abort_flag, S.status)) {
            ok = false;
            break;
          }
          const uint32_t sa = sbase + stage * UT_STAGE_BYTES;
          const int kk = k + 4 * c;
          const int bytes = kend - kk >= 4 ? 16 : (kend > kk ? 4 * (kend - kk) : 0);
#pragma unroll 4
          for (int j = 0; j < 8; ++j) {
            const int R = 32 * pw + 4 * j + (lane >> 3);
            const int a = R >> 3, u = R & 7, p = u >> 2, i = 4 * a + (u & 3);
            const uint32_t off = (uint32_t)(a * 1024 + u * 128 + ((c ^ u) << 4));
            const int ya = gather_row(pr.rmask, pr.a0, i, p, md);
            const int yb = gather_row(pr.cmask, pr.b0, i, p, md);
            const bool va = ya < 2 * md && bytes > 0, vb = yb < 2 * md && bytes > 0;
            cp_async16(sa + off, va ? base + (size_t)ya * wp + kk : base, va ? bytes : 0);
            cp_async16(sa + UT_OPB + off, vb ? base + (size_t)yb * wp + kk : base, vb ? bytes : 0);
          }
          asm volatile("cp.async.commit_group;\n" ::: "memory");
          if (pend[1] >= 0) {   // the chunk issued two chunks ago has landed: hand it over
            asm volatile("cp.async.wait_group 2;\n" ::: "memory");
            asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&full_bar[pend[1]]));
          }
          pend[1] = pend[0];
          pend[0] = stage;
          if (++stage == UT_STAGES) { stage = 0; phase ^= 1u; }
        }
      }
    }
    // the last chunks (and, after an abort, every copy in flight) land before leaving
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncwarp();
    if (lane == 0)
      for (int k = 1; k >= 0; --k)
        if (pend[k] >= 0) mbar_arrive(smem_u32(&full_bar[pend[k]]));
  } else if (TMA && warp == 4) {
    // --------------------------- producer (TMA) ---------------------------
    int stage = 0;
    uint32_t phase = 0;
    int armed[UT_STAGES];
#pragma unroll
    for (int s = 0; s < UT_STAGES; ++s) armed[s] = 0;
    const int a = lane >> 1, p = lane & 1;   // this lane's swizzle atom and piece
    bool ok = true;
    for (int t = blockIdx.x; t < count && ok; t += gridDim.x) {
      const int p_end = task_end[t];
      for (int q = tasks[t].w; q < p_end && ok; ++q) {
        const TcPair pr = pairs[q];
        const int md = (int)(S.rowptr[pr.d + 1] - S.rowptr[pr.d]);
        const CUtensorMap *map = maps + pr.d;
        int ya[4], yb[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          ya[r] = gather_row(pr.rmask, pr.a0, 4 * a + r, p, md);
          yb[r] = gather_row(pr.cmask, pr.b0, 4 * a + r, p, md);
        }
        const int k0 = pr.kk & 0xffff, kend = k0 + (pr.kk >> 16);
        for (int k = k0; k < kend; k += UT_KCHUNK) {
          if (!mbar_wait_warp(smem_u32(&empty_bar[stage]), phase ^ 1u, &abort_flag, S.status)) {
            ok = false;
            break;
          }
          const uint32_t fb = smem_u32(&full_bar[stage]);
          if (lane == 0) mbar_arrive_tx(fb, UT_STAGE_BYTES);
          armed[stage] += 1;
          __syncwarp();
          const uint32_t dst = sbase + stage * UT_STAGE_BYTES + a * 1024 + p * 512;
          tma_gather4(dst, map, fb, k, ya[0], ya[1], ya[2], ya[3]);
          tma_gather4(dst + UT_OPB, map, fb, k, yb[0], yb[1], yb[2], yb[3]);
          if (++stage == UT_STAGES) { stage = 0; phase ^= 1u; }
        }
      }
    }
    // copies in flight complete before the CTA leaves
    if (lane == 0)
      for (int s = 0; s < UT_STAGES; ++s)
        if (armed[s] > 0) mbar_drain(smem_u32(&full_bar[s]), (uint32_t)(armed[s] - 1) & 1u, S.status);
  } else if (warp == MMA_WARP) {
    // ------------------------------ MMA issuer ----------------------------
    if (lane == 0) {
      int stage = 0, buf = 0;
      uint32_t phase = 0, accphase[2] = {0, 0};
      bool ok = true;
      for (int t = blockIdx.x; t < count && ok; t += gridDim.x) {
        const int p_end = task_end[t];
        int gchunks = 0;
        for (int q = tasks[t].w; q < p_end && ok; ++q) {
          const int nch = pair_chunks(pairs[q]);
          const bool open = gchunks == 0;
          if (open) {   // the epilogue has drained this accumulator
            if (!mbar_wait(smem_u32(&acce_bar[buf]), accphase[buf] ^ 1u, &abort_flag, S.status)) {
              ok = false;
              break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
          }
          const uint32_t dt = tmem + (uint32_t)buf * 128u;
          for (int c = 0; c < nch; ++c) {
            if (!mbar_wait(smem_u32(&full_bar[stage]), phase, &abort_flag, S.status)) {
              ok = false;
              break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const uint32_t sa = sbase + stage * UT_STAGE_BYTES, sb = sa + UT_OPB;
#pragma unroll
            for (int kk = 0; kk < UT_KCHUNK / 8; ++kk)
              mma_tf32(dt, sw128_desc(sa + 32 * kk), sw128_desc(sb + 32 * kk),
                       (open && c == 0 && kk == 0) ? 0u : 1u);
            mma_commit(smem_u32(&empty_bar[stage]));   // stage free once these MMAs are done
            if (++stage == UT_STAGES) { stage = 0; phase ^= 1u; }
          }
          if (!ok) break;
          gchunks += nch;
          if (gchunks >= UT_GROUP_CHUNKS || q + 1 == p_end) {
            mma_commit(smem_u32(&accf_bar[buf]));      // group done: to the epilogue
            accphase[buf] ^= 1u;
            buf ^= 1;
            gchunks = 0;
          }
        }
      }
      // every MMA issued has completed before TMEM is freed
      mma_commit(smem_u32(&done_bar));
      mbar_drain(smem_u32(&done_bar), 0u, S.status);
    }
    __syncwarp();
  } else {
    // ------------------------------ epilogue ------------------------------
    // thread tid owns TMEM lane tid: row' tid = atom a, piece p, tile row i = 4a + r
    const int a = tid >> 3, p = (tid >> 2) & 1, i = 4 * a + (tid & 3);
    int buf = 0;
    uint32_t accphase[2] = {0, 0};
    bool ok = true;
    for (int t = blockIdx.x; t < count && ok; t += gridDim.x) {
      const int4 tk = tasks[t];
      const int s = tk.x, r0 = tk.y, c0 = tk.z;
      const int p_end = task_end[t];
      const int w = S.super[s + 1] - S.super[s];
      const int m = (int)(S.rowptr[s + 1] - S.rowptr[s]);
      const int nrow = min(TB, m - r0), ncol = min(TB, w - c0);
      double *P = S.L + S.xptr[s];
      // my 32 entries of the tile: row i, columns 4b + 2p + e; seeded with minus the tile
      double acc[16][2];
#pragma unroll
      for (int b = 0; b < 16; ++b)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int j = 4 * b + 2 * p + e;
          acc[b][e] = (i < nrow && j < ncol && r0 + i >= c0 + j)
                          ? -P[(size_t)(c0 + j) * m + r0 + i] : 0.0;
        }
      int gchunks = 0;
      for (int q = tk.w; q < p_end; ++q) {
        gchunks += pair_chunks(pairs[q]);
        if (!(gchunks >= UT_GROUP_CHUNKS || q + 1 == p_end)) continue;
        gchunks = 0;
        if (!mbar_wait_warp(smem_u32(&accf_bar[buf]), accphase[buf], &abort_flag, S.status)) {
          ok = false;
          break;
        }
        accphase[buf] ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        const uint32_t ta = tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)buf * 128u;
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) {
          float v[32];
          tmem_ld32(ta + 32u * cc, v);
#pragma unroll
          for (int bb = 0; bb < 4; ++bb) {
            float f[4];
#pragma unroll
            for (int c = 0; c < 4; ++c) {
              f[c] = v[8 * bb + c] + v[8 * bb + 4 + c];          // hi' + lo' of column 4b + c
              f[c] += __shfl_xor_sync(0xffffffffu, f[c], 4);   // + the other piece of row i
            }
            const int b = 4 * cc + bb;
            acc[b][0] += (double)(p ? f[2] : f[0]);
            acc[b][1] += (double)(p ? f[3] : f[1]);
          }
        }
        asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
        __syncwarp();
        if (lane == 0) mbar_arrive(smem_u32(&acce_bar[buf]));
        buf ^= 1;
      }
      if (!ok) break;
#pragma unroll
      for (int b = 0; b < 16; ++b)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int j = 4 * b + 2 * p + e;
          if (i < nrow && j < ncol && r0 + i >= c0 + j) P[(size_t)(c0 + j) * m + r0 + i] = -acc[b][e];
        }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem),
                 "r"(UT_TMEM_COLS));
}

using EncodeTiled = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                 const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                 const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                 CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_fn() {
  static EncodeTiled fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiled>(p);
  }
  return fn;
}

}  // namespace

bool update_tc_configure(std::string &err) {
  cudaError_t e = cudaFuncSetAttribute(k_update_tc<true>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, UT_SMEM);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_update_tc<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             UT_SMEM);
  if (e != cudaSuccess) {
    err = std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e);
    return false;
  }
  return true;
}

int64_t kmirror_layout(const std::vector<int> &super, const std::vector<int64_t> &rowptr,
                       std::vector<int64_t> &xk) {
  const int ns = (int)super.size() - 1;
  xk.resize(ns);
  int64_t off = 0;
  for (int d = 0; d < ns; ++d) {
    const int64_t w = super[d + 1] - super[d], m = rowptr[d + 1] - rowptr[d];
    xk[d] = off;
    off += 2 * m * ((w + 3) & ~3LL);
  }
  return off;
}

bool build_tensor_maps(const std::vector<int> &super, const std::vector<int64_t> &rowptr,
                       const std::vector<int64_t> &xk, float *Lk, void *maps_host,
                       std::string &err) {
  EncodeTiled enc = encode_fn();
  if (!enc) {
    err = "cuTensorMapEncodeTiled is not available from the driver";
    return false;
  }
  CUtensorMap *maps = static_cast<CUtensorMap *>(maps_host);
  const int ns = (int)super.size() - 1;
  for (int d = 0; d < ns; ++d) {
    const uint64_t w = super[d + 1] - super[d], m = rowptr[d + 1] - rowptr[d];
    const uint64_t wp = (w + 3) & ~3ULL;
    const cuuint64_t dims[2] = {w, 2 * m};
    const cuuint64_t strides[1] = {wp * sizeof(float)};
    const cuuint32_t box[2] = {UT_KCHUNK, 1};
    const cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(&maps[d], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, Lk + xk[d], dims, strides, box,
                     estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
      err = "cuTensorMapEncodeTiled failed for supernode " + std::to_string(d) + " (code " +
            std::to_string((int)r) + ")";
      return false;
    }
  }
  return true;
}

size_t tensor_map_bytes() { return sizeof(CUtensorMap); }

int update_tc_ctas(int count) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return count < sms ? count : sms;
}

void launch_update_tc(const DevSym &S, const void *maps, const int4 *tasks, const int *task_end,
                      const TcPair *pairs, int count, bool tma, cudaStream_t st) {
  if (count <= 0) return;
  if (tma)
    k_update_tc<true><<<update_tc_ctas(count), ut_threads(true), UT_SMEM, st>>>(
        S, static_cast<const CUtensorMap *>(maps), tasks, task_end, pairs, count);
  else
    k_update_tc<false><<<update_tc_ctas(count), ut_threads(false), UT_SMEM, st>>>(
        S, static_cast<const CUtensorMap *>(maps), tasks, task_end, pairs, count);
}

}  // namespace swc
