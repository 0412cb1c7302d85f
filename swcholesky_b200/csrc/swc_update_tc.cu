// Split-precision Schur updates of the tiled class on the 5th-generation tensor cores.
//
// The reference forms every update of a target supernode from a descendant as a dense
// SYRK + GEMM into a contribution buffer and scatters it through relative indices
// (cholesky/sw_parallel_PB_Cholesky_05.c:299-378).  Here a 64x64 tile of a target panel
// owns its updates: for every (tile, descendant) pair the descendant's rows that fall in
// the tile are gathered straight into the tile's own row and column positions in shared
// memory, so the product lands in the tile's coordinates and no scatter is needed; the tile
// leaves the chip once, after all its descendants.  The same kernel runs the trailing
// SYRK/GEMM steps of the blocked dense factorization of wide supernodes (a "pair" whose
// descendant is the supernode itself and whose K range is one or more 64-column blocks).
//
// Operands: the split mirror of L in K-major form, supernode d (md rows, wd columns) at
// (float *)Lf + xk[d] (128-byte aligned); xk[nsuper] names the format:
//   0  split-TF32: hi = tf32(x) in row r of the hi plane, lo = tf32(x - hi) in row md + r
//      of the lo plane; rows of wd rounded up to 32 floats (128 bytes);
//   1  BF16x3: hi = bf16(x), mid = bf16(x - hi), lo = bf16(x - hi - mid) in rows r, md + r,
//      2 md + r of three planes; rows of wd rounded up to 64 bfloat16 values.
// A 32-column K chunk of a row is then one aligned 128-byte (or 64-byte) run of memory.
// A stage holds one 32-column K chunk of the 128-row operands, each in the canonical K-major
// layout the MMA reads with a swizzle (128-byte rows, 128-byte swizzle for TF32; 64-byte
// rows, 64-byte swizzle for BF16): atom a (8 rows) holds tile rows 4a..4a+3 twice, one piece
// in its first four rows and another in its last four.  A tile row that no descendant row
// feeds is zero-filled.
//
// Products (one CTA, M = N = 128, accumulators in TMEM, FP32):
//   split-TF32: operands A' = [hi; lo] and B' = [hi; lo]; one kind::tf32 MMA per 8 columns of
//     K gives every piece product: C(i, j) = hi hi' + hi lo' + lo hi' + lo lo' (about 2^-22
//     relative error, the accuracy of the split);
//   BF16x3: operands A1 = [hi; mid], A2 = [lo; hi] (and B1, B2 alike); per 16 columns of K one
//     kind::f16 MMA accumulates D1 = A1 B1^T and one D2 = A2 B2^T; the epilogue takes all of
//     D1 and the lo hi' and hi lo' blocks of D2: the six piece products down to the third
//     order (the split-bfloat16 method of Henry, Tang and Heinecke, ARITH 2019), about 2^-24
//     relative error.
// The pieces are folded in the epilogue (one shuffle: the two rows of a tile row's pieces
// are lanes t and t ^ 4).
//
// Staging (per K chunk, 32 KB):
//   cp.async  four producer warps copy 16 bytes per lane, a warp instruction covering 512
//             contiguous shared-memory bytes (four 128-byte or eight 64-byte rows) and 128-
//             or 64-byte runs of global memory; each thread's copies arrive on the stage's
//             mbarrier when they land (cp.async.mbarrier.arrive.noinc), and the MMA thread
//             fences the async proxy after its wait;
//   TMA       (split-TF32, plan 6) one producer warp issues 64 cp.async.bulk.tensor.2d ...
//             tile::gather4 loads (four rows of 32 values each, into one half of a swizzle
//             atom) from one 2D tensor map per supernode ({wd, 2 md}, 128-byte swizzle, zero
//             fill outside); measured slower than the cp.async path on this workload.
//
// Roles (one CTA per SM, persistent over the launch's tile list):
//   warps 0-3  epilogue (TMEM lane quarter = warp): per group of descendants (at least 8
//              chunks, or the tile's last), reads the accumulator(s), folds the pieces, adds
//              them in FP64 to the tile held in registers (seeded with minus the tile's FP64
//              values), releases the accumulator; stores the tile once per tile.  The next
//              tile's values load while the MMAs of its first group run;
//   producers  as above;
//   MMA warp   one thread: per chunk waits for the stage, issues the MMAs into one of two
//              accumulator sets and commits the stage back to the producers
//              (tcgen05.commit); at the end of a group commits the accumulators to the
//              epilogue and switches sets.
// Every mbarrier wait is bounded (2 s of %globaltimer): a wait that runs out sets status[3]
// and an abort flag that stops the other roles; the kernel then waits (bounded) for its
// copies and MMAs in flight, frees its TMEM and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "swc_engine.h"

namespace swc {

namespace {

// variants of the kernel
constexpr int V_TF32 = UT_VARIANT_TF32;           // split-TF32, cp.async staging
constexpr int V_TF32_TMA = UT_VARIANT_TF32_TMA;   // split-TF32, TMA gather4 staging
constexpr int V_BF16 = UT_VARIANT_BF16;           // BF16x3, cp.async staging

constexpr int UT_MAX_STAGES = 6;
constexpr int UT_KCHUNK = 32;                       // K columns per stage
constexpr int UT_STAGE_BYTES = 32 * 1024;           // the operand chunks of one stage
// dynamic shared memory of a launch with `stages` stages (+ alignment slack)
constexpr int ut_smem(int stages) { return stages * UT_STAGE_BYTES + 1024; }
constexpr int UT_GROUP_CHUNKS = 8;                  // chunks of one FP32 accumulation group
constexpr unsigned long long UT_WAIT_NS = 2000000000ULL;   // a pipeline wait gives up after 2 s

// Per-variant constants: element bytes, row bytes of an operand chunk (= its swizzle span),
// operands per stage, bytes of one operand chunk, TMEM columns (two accumulator sets),
// producer warps, threads, instruction descriptor (D F32, K-major A and B, N = M = 128;
// A/B format TF32 = 2 or BF16 = 1), descriptor layout type (SWIZZLE_128B = 2, _64B = 4).
template <int V>
struct Ut {
  static constexpr bool BF16 = V == V_BF16;
  static constexpr int ELEM = BF16 ? 2 : 4;
  static constexpr int ROW = UT_KCHUNK * ELEM;               // 128 (TF32) or 64 (BF16)
  static constexpr int ATOM = 8 * ROW;                       // bytes of an 8-row atom
  static constexpr int NOPS = BF16 ? 4 : 2;                  // A1, A2, B1, B2 / A', B'
  static constexpr int OPB = 128 * ROW;                      // bytes of one operand chunk
  static constexpr int TMEM_COLS = BF16 ? 512 : 256;
  static constexpr int NPROD = V == V_TF32_TMA ? 1 : 4;
  static constexpr int THREADS = 32 * (5 + NPROD);
  static constexpr int FMT = BF16 ? 1 : 2;
  static constexpr uint32_t IDESC = (1u << 4) | ((uint32_t)FMT << 7) | ((uint32_t)FMT << 10) |
                                    ((128u >> 3) << 17) | ((128u >> 4) << 24);
  static constexpr uint64_t LAYOUT = BF16 ? 4 : 2;
  static_assert(NOPS * OPB == UT_STAGE_BYTES, "a stage holds the operand chunks");
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor of a K-major swizzled operand: 8-row groups `sbo` bytes
// apart, leading offset 16 bytes (unused by the swizzled K-major layouts), version 1.
__device__ __forceinline__ uint64_t sw_desc(uint32_t saddr, uint32_t sbo, uint64_t layout) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)1 << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | ((uint64_t)1 << 46) | (layout << 61);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
// One bounded try: the thread sleeps until the phase completes or about 20 us pass, so
// waiting warps do not take issue slots from the producers.
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2, %3;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity), "r"(20000)
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

// Arrival on the mbarrier once every cp.async this thread issued so far has landed (the
// barrier's count includes this arrival: no increment).
__device__ __forceinline__ void cp_async_arrive(uint32_t bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];\n" ::"r"(bar) : "memory");
}

// 16-byte copy global -> shared with zero fill beyond `bytes` (0..16) of the source.
__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, int bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(bytes)
               : "memory");
}

template <int V>
__device__ __forceinline__ void mma_issue(uint32_t tmem, uint64_t adesc, uint64_t bdesc,
                                          uint32_t accumulate) {
  if (Ut<V>::BF16)
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(
            tmem),
        "l"(adesc), "l"(bdesc), "r"(Ut<V>::IDESC), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
  else
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(
            tmem),
        "l"(adesc), "l"(bdesc), "r"(Ut<V>::IDESC), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
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

// K chunks of a pair.
__device__ __forceinline__ int pair_chunks(const TcPair &pr) {
  return ((pr.kk >> 16) + UT_KCHUNK - 1) / UT_KCHUNK;
}

// Row of the source supernode (md rows) that feeds tile row i of the pair's operand (mask,
// first source row s0), in plane p of the mirror, or -1 when no source row feeds it.
__device__ __forceinline__ int source_row(uint64_t mask, int s0, int i, int p, int md) {
  if (!((mask >> i) & 1ull)) return -1;
  return p * md + s0 + __popcll(mask & ((1ull << i) - 1ull));
}

// Mirror plane of piece slot p (0: first four rows of an atom, 1: last four) of operand o.
template <int V>
__device__ __forceinline__ int operand_plane(int o, int p) {
  if (!Ut<V>::BF16) return p;                    // A', B': hi, lo
  return (o & 1) == 0 ? p : (p == 0 ? 2 : 0);    // A1, B1: hi, mid;  A2, B2: lo, hi
}

template <int V>
__global__ void __launch_bounds__(Ut<V>::THREADS, 1)
    k_update_tc(DevSym S, const CUtensorMap *__restrict__ maps, const int4 *__restrict__ tasks,
                const int *__restrict__ task_end, const TcPair *__restrict__ pairs, int count,
                int nst) {
  using T = Ut<V>;
  constexpr int MMA_WARP = 4 + T::NPROD;
  extern __shared__ unsigned char ut_dyn[];
  __shared__ __align__(8) uint64_t full_bar[UT_MAX_STAGES], empty_bar[UT_MAX_STAGES];
  __shared__ __align__(8) uint64_t accf_bar[2], acce_bar[2], done_bar;
  __shared__ uint32_t tmem_base;
  __shared__ volatile int abort_flag;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // 1024-byte aligned stages (the swizzle atoms must be)
  const uint32_t sbase = (smem_u32(ut_dyn) + 1023u) & ~1023u;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(&tmem_base)),
                 "r"(T::TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid == 32 * MMA_WARP) {
    for (int s = 0; s < nst; ++s) {
      // cp.async staging: one hardware arrival per producer thread; TMA: the arming thread
      mbar_init(smem_u32(&full_bar[s]), V == V_TF32_TMA ? 1 : 32 * T::NPROD);
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

  if (V != V_TF32_TMA && warp >= 4 && warp < 4 + T::NPROD) {
    // ------------------------- producers (cp.async) ------------------------
    // warp pw fills rows' 32 pw .. 32 pw + 31 of every operand chunk; an instruction covers
    // RPI rows' of T::ROW bytes (lane: row' RPI j + lane / CPR, 16-byte column chunk
    // lane % CPR), written where the swizzled K-major layout puts them.  The lane's NSLOT
    // shared-memory slots are fixed for the kernel and its source rows for a pair, so a
    // chunk costs one add and one copy per slot.  Each thread's copies arrive on the stage's
    // mbarrier when they land (cp.async.mbarrier.arrive.noinc), so up to nst chunks are in
    // flight.
    constexpr int CPR = T::ROW / 16, RPI = 32 / CPR, JS = 32 / RPI, NSLOT = T::NOPS * JS;
    const int pw = warp - 4, cc = lane % CPR, rsub = lane / CPR;
    uint32_t soff[NSLOT];   // shared-memory offset of each slot within a stage
#pragma unroll
    for (int o = 0; o < T::NOPS; ++o)
#pragma unroll
      for (int j = 0; j < JS; ++j) {
        const int R = 32 * pw + RPI * j + rsub, a = R >> 3, u = R & 7;
        const int swz = T::BF16 ? (u >> 1) : u;
        soff[o * JS + j] = (uint32_t)(o * T::OPB + a * T::ATOM + u * T::ROW + ((cc ^ swz) << 4));
      }
    int stage = 0;
    uint32_t phase = 0;
    bool ok = true;
    const unsigned char *mir = reinterpret_cast<const unsigned char *>(S.Lf);
    for (int t = blockIdx.x; t < count && ok; t += gridDim.x) {
      const int p_end = task_end[t];
      for (int q = tasks[t].w; q < p_end && ok; ++q) {
        const TcPair pr = pairs[q];
        const int wd = S.super[pr.d + 1] - S.super[pr.d];
        const int pitch = T::BF16 ? kmirror_pitch_bf16(wd) : kmirror_pitch_tf32(wd);
        const int md = (int)(S.rowptr[pr.d + 1] - S.rowptr[pr.d]);
        const unsigned char *base = mir + 4 * S.xk[pr.d];
        // each slot's source row (plane row * pitch elements from base), null: zeros
        const unsigned char *src[NSLOT];
#pragma unroll
        for (int o = 0; o < T::NOPS; ++o)
#pragma unroll
          for (int j = 0; j < JS; ++j) {
            const bool isA = o < T::NOPS / 2;
            const int R = 32 * pw + RPI * j + rsub, u = R & 7;
            const int y = source_row(isA ? pr.rmask : pr.cmask, isA ? pr.a0 : pr.b0,
                                     4 * (R >> 3) + (u & 3), operand_plane<V>(o, u >> 2), md);
            src[o * JS + j] = y >= 0 ? base + (size_t)y * pitch * T::ELEM : nullptr;
          }
        const int k0 = pr.kk & 0xffff, kend = k0 + (pr.kk >> 16);
        for (int k = k0; k < kend; k += UT_KCHUNK) {
          if (!mbar_wait_warp(smem_u32(&empty_bar[stage]), phase ^ 1u, &abort_flag, S.status)) {
            ok = false;
            break;
          }
          const uint32_t sa = sbase + stage * UT_STAGE_BYTES;
          const int kk = k + cc * (16 / T::ELEM);
          const int left = (kend - kk) * T::ELEM;
          const int bytes = left >= 16 ? 16 : (left > 0 ? left : 0);
          const size_t kb = (size_t)kk * T::ELEM;
#pragma unroll
          for (int e = 0; e < NSLOT; ++e)
            cp_async16(sa + soff[e], src[e] ? src[e] + kb : base, src[e] ? bytes : 0);
          cp_async_arrive(smem_u32(&full_bar[stage]));
          if (++stage == nst) { stage = 0; phase ^= 1u; }
        }
      }
    }
    // every copy in flight lands before the CTA leaves
    asm volatile("cp.async.wait_all;\n" ::: "memory");
  } else if (V == V_TF32_TMA && warp == 4) {
    // --------------------------- producer (TMA) ---------------------------
    int stage = 0;
    uint32_t phase = 0;
    int armed[UT_MAX_STAGES];
#pragma unroll
    for (int s = 0; s < UT_MAX_STAGES; ++s) armed[s] = 0;
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
        for (int r = 0; r < 4; ++r) {   // a row outside the map (2 md) reads zeros
          ya[r] = source_row(pr.rmask, pr.a0, 4 * a + r, p, md);
          yb[r] = source_row(pr.cmask, pr.b0, 4 * a + r, p, md);
          if (ya[r] < 0) ya[r] = 2 * md;
          if (yb[r] < 0) yb[r] = 2 * md;
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
          const uint32_t dst = sbase + stage * UT_STAGE_BYTES + a * T::ATOM + p * (T::ATOM / 2);
          tma_gather4(dst, map, fb, k, ya[0], ya[1], ya[2], ya[3]);
          tma_gather4(dst + T::OPB, map, fb, k, yb[0], yb[1], yb[2], yb[3]);
          if (++stage == nst) { stage = 0; phase ^= 1u; }
        }
      }
    }
    // copies in flight complete before the CTA leaves
    if (lane == 0)
      for (int s = 0; s < nst; ++s)
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
          if (open) {   // the epilogue has drained this accumulator set
            if (!mbar_wait(smem_u32(&acce_bar[buf]), accphase[buf] ^ 1u, &abort_flag, S.status)) {
              ok = false;
              break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
          }
          const uint32_t dt = tmem + (uint32_t)buf * (T::TMEM_COLS / 2);
          for (int c = 0; c < nch; ++c) {
            if (!mbar_wait(smem_u32(&full_bar[stage]), phase, &abort_flag, S.status)) {
              ok = false;
              break;
            }
            // the stage's bytes (written by cp.async in the generic proxy, or by TMA) are
            // read by the MMAs through the async proxy
            asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const uint32_t sa = sbase + stage * UT_STAGE_BYTES;
            if (T::BF16) {
              // 16 columns of K per MMA: D1 += A1 B1^T, D2 += A2 B2^T
#pragma unroll
              for (int kk = 0; kk < UT_KCHUNK / 16; ++kk) {
                const uint32_t acc = (open && c == 0 && kk == 0) ? 0u : 1u;
                mma_issue<V>(dt, sw_desc(sa + 32 * kk, T::ATOM, T::LAYOUT),
                             sw_desc(sa + 2 * T::OPB + 32 * kk, T::ATOM, T::LAYOUT), acc);
                mma_issue<V>(dt + 128, sw_desc(sa + T::OPB + 32 * kk, T::ATOM, T::LAYOUT),
                             sw_desc(sa + 3 * T::OPB + 32 * kk, T::ATOM, T::LAYOUT), acc);
              }
            } else {
              // 8 columns of K per MMA: D += A' B'^T
#pragma unroll
              for (int kk = 0; kk < UT_KCHUNK / 8; ++kk)
                mma_issue<V>(dt, sw_desc(sa + 32 * kk, T::ATOM, T::LAYOUT),
                             sw_desc(sa + T::OPB + 32 * kk, T::ATOM, T::LAYOUT),
                             (open && c == 0 && kk == 0) ? 0u : 1u);
            }
            mma_commit(smem_u32(&empty_bar[stage]));   // stage free once these MMAs are done
            if (++stage == nst) { stage = 0; phase ^= 1u; }
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
  } else if (warp < 4) {
    // ------------------------------ epilogue ------------------------------
    // thread tid owns TMEM lane tid: row' tid = atom a, piece slot p, tile row i = 4a + r;
    // lanes tid and tid ^ 4 hold the two slots of the same tile row
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
        const uint32_t ta = tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)buf * (T::TMEM_COLS / 2);
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) {
          float v[32], v2[32];
          tmem_ld32(ta + 32u * cc, v);
          if (T::BF16) tmem_ld32(ta + 128u + 32u * cc, v2);
#pragma unroll
          for (int bb = 0; bb < 4; ++bb) {
            float f[4];
#pragma unroll
            for (int c = 0; c < 4; ++c) {
              // column 4b + c: both pieces of the column from D (D1) ...
              f[c] = v[8 * bb + c] + v[8 * bb + 4 + c];
              // ... and, for BF16x3, D2's lo hi' (slot 0 rows, slot 1 columns) or hi lo'
              if (T::BF16) f[c] += p == 0 ? v2[8 * bb + 4 + c] : v2[8 * bb + c];
              f[c] += __shfl_xor_sync(0xffffffffu, f[c], 4);   // + the other slot of row i
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
                 "r"(T::TMEM_COLS));
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

template <int V>
void launch_variant(const DevSym &S, const void *maps, const int4 *tasks, const int *task_end,
                    const TcPair *pairs, int count, int nst, cudaStream_t st) {
  k_update_tc<V><<<update_tc_ctas(count), Ut<V>::THREADS, ut_smem(nst), st>>>(
      S, static_cast<const CUtensorMap *>(maps), tasks, task_end, pairs, count, nst);
}

}  // namespace

bool update_tc_configure(std::string &err) {
  const int smem = ut_smem(UT_MAX_STAGES);
  cudaError_t e = cudaFuncSetAttribute(k_update_tc<V_TF32>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_update_tc<V_TF32_TMA>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_update_tc<V_BF16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             smem);
  if (e != cudaSuccess) {
    err = std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e);
    return false;
  }
  return true;
}

int64_t kmirror_layout(const std::vector<int> &super, const std::vector<int64_t> &rowptr,
                       std::vector<int64_t> &xk) {
  const int ns = (int)super.size() - 1;
  xk.resize(ns + 1);
  int64_t off = 0;
  for (int d = 0; d < ns; ++d) {
    const int64_t w = super[d + 1] - super[d], m = rowptr[d + 1] - rowptr[d];
    // floats: two TF32 planes or three bfloat16 planes (rows of 128-byte multiples); the
    // larger, so every supernode starts on a 128-byte boundary
    const int64_t tf32 = 2 * m * kmirror_pitch_tf32((int)w);
    const int64_t bf16 = (3 * m * kmirror_pitch_bf16((int)w) + 1) / 2;
    xk[d] = off;
    off += ((tf32 > bf16 ? tf32 : bf16) + 31) & ~31LL;
  }
  xk[ns] = 0;   // the format entry, set per mode
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
    const uint64_t wp = (uint64_t)kmirror_pitch_tf32((int)w);
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
                      const TcPair *pairs, int count, int variant, bool shared_sm,
                      cudaStream_t st) {
  if (count <= 0) return;
  // alone on the GPU: 6 stages (193 KB); next to the diagonal-block kernel: 4 (129 KB)
  const int nst = shared_sm ? 4 : UT_MAX_STAGES;
  if (variant == UT_VARIANT_BF16)
    launch_variant<V_BF16>(S, maps, tasks, task_end, pairs, count, nst, st);
  else if (variant == UT_VARIANT_TF32_TMA)
    launch_variant<V_TF32_TMA>(S, maps, tasks, task_end, pairs, count, nst, st);
  else
    launch_variant<V_TF32>(S, maps, tasks, task_end, pairs, count, nst, st);
}

}  // namespace swc
