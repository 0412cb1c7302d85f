// Right-looking split-TF32 Schur updates of the tiled class on the 5th-generation tensor
// cores, scattered into the targets with FP64 atomic adds.
//
// The reference forms the update of every target supernode by every descendant d as a dense
// SYRK/GEMM of d's rows below the target's first column into a contribution buffer, then
// adds it to the target through relative indices (cholesky/sw_parallel_PB_Cholesky_05.c:
// 299-378).  Here, in the split-TF32 mode, d's whole contribution is formed at once, as soon
// as d is factored: C = B B^T with B the rows of d (below its own columns) whose column
// index falls in a tiled-class supernode onwards, a dense product of 128x128 tiles over K =
// the width of d, and each entry of the lower triangle of C is added to its target entry of
// L (the supernode s owning C's column, at the target's row of C's row) by one FP64 atomic
// add.  Operands are plain 2D tiles of d's K-major split mirror (no gather), so every tile
// is a full 128x128x(width) product; the only padding is the diagonal tiles' upper halves and
// the ragged last tiles.  Concurrent contributions to one target entry are summed by the
// atomics in an unspecified order (results reproduce to rounding, not bit for bit); the FP64
// mode keeps the deterministic tile-owner kernels.
//
// Split-TF32 products: x = hi + lo with hi = tf32(x) and lo = tf32(x - hi) (the mirror's two
// planes); per 8 columns of K three kind::tf32 MMAs (M = N = 128) accumulate
// hi hi' + lo hi' + hi lo' in one FP32 accumulator in TMEM (the lo lo' term, below 2^-22 of
// the product, is dropped).
//
// Roles (608 threads, one CTA per SM, persistent over the launch's tile list, tile t handled
// by CTA t mod gridDim.x):
//   warps 0-15 epilogue: warp w owns tile rows 32 (w % 4) .. + 31 (its TMEM lane quarter) and
//              columns 32 (w / 4) .. + 31; reads its 32 FP32 values, releases the
//              accumulator, then adds minus each lower-triangle entry to L at the address the
//              tile's scatter table gives (shared memory only); sixteen warps keep enough
//              atomic adds in flight;
//   warp 16    TMA producer (one thread): per 32-column K chunk, four 2D tiled loads (A hi,
//              A lo, B hi, B lo; 128 rows x 128 bytes each, 128-byte swizzle) into a stage,
//              two for a diagonal tile (B = A);
//   warp 17    MMA issuer (one thread): twelve MMAs per stage into one of two accumulators,
//              tcgen05.commit frees the stage and, after the tile's last chunk, hands the
//              accumulator to the epilogue;
//   warp 18    table warp: builds the next tile's scatter table in shared memory (two
//              tables in a ring): the target base and run slot of every column and, per
//              run, the target position of every tile row, loaded as independent reads so
//              the epilogue meets no chain of dependent global loads.
// Every mbarrier wait is bounded (2 s of %globaltimer): a wait that runs out sets status[3]
// and an abort flag that stops the other roles; the kernel then waits (bounded) for its loads
// and MMAs in flight, frees its TMEM and returns.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdint>
#include <string>
#include <vector>

#include "swc_engine.h"

namespace swc {

namespace {

constexpr int SC_KCHUNK = 32;                 // K columns per stage
constexpr int SC_MAX_STAGES = 4;
constexpr int SC_EPI_WARPS = 16;              // epilogue: (row quarter, 32-column group)
constexpr int SC_PRODUCER = 16, SC_MMA = 17, SC_TABLE = 18;   // warps of the other roles
constexpr int SC_THREADS = 32 * 19;
constexpr int SC_TMEM_COLS = 256;             // two 128-column FP32 accumulators
constexpr unsigned long long SC_WAIT_NS = 2000000000ULL;
// The two split formats (the mirror's format entry): per format the planes of a value, the
// bytes of a 32-column row chunk (= its swizzle span: 128-byte swizzle for TF32, 64-byte for
// bfloat16), the stages of the ring, the MMA kind's operand format and the products per K
// step (TF32: K = 8, hi hi' + lo hi' + hi lo'; BF16x3: K = 16, the six products down to the
// third order).  A stage holds the A planes, then the B planes, each 128 rows x ROW bytes.
template <bool BF16>
struct Sc {
  static constexpr int PLANES = BF16 ? 3 : 2;
  static constexpr int ROW = SC_KCHUNK * (BF16 ? 2 : 4);
  static constexpr int OP = 128 * ROW;
  static constexpr int STAGE = 2 * PLANES * OP;
  static constexpr int STAGES = BF16 ? 4 : 3;
  static constexpr int SBO = 8 * ROW;                 // bytes between 8-row groups
  static constexpr uint64_t LAYOUT = BF16 ? 4 : 2;    // SWIZZLE_64B / SWIZZLE_128B
  static constexpr uint32_t FMT = BF16 ? 1 : 2;       // BF16 / TF32 operands
  static constexpr int KSTEP = BF16 ? 16 : 8;         // K of one MMA
};
constexpr int SC_SMEM = 3 * 4 * 128 * 128 + 1024;   // either format: 192 KB of stages + slack
static_assert(Sc<false>::STAGES * Sc<false>::STAGE + 1024 <= SC_SMEM, "TF32 ring fits");
static_assert(Sc<true>::STAGES * Sc<true>::STAGE + 1024 <= SC_SMEM, "BF16x3 ring fits");

// Instruction descriptor: D F32 (bit 4), A and B format at bits 7 and 10 (TF32 2, BF16 1),
// K-major, N >> 3 at bit 17, M >> 4 at bit 24; M = 128, N = 128 or 64.
__host__ __device__ constexpr uint32_t sc_idesc(uint32_t fmt, uint32_t n) {
  return (1u << 4) | (fmt << 7) | (fmt << 10) | ((n >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// K-major swizzled operand: 8-row groups sbo bytes apart, leading offset 16 (unused by the
// swizzled K-major layouts), version 1, the layout type of the swizzle.
__device__ __forceinline__ uint64_t sw_desc(uint32_t saddr, uint32_t sbo, uint64_t layout) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)1 << 16) | ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) |
         ((uint64_t)1 << 46) | (layout << 61);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
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
// Bounded wait for the phase of the given parity; false when it ran out (recorded in
// status[3] and the abort flag) or another role aborted.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int *abort_flag,
                                          int *status) {
  if (mbar_try(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (long long it = 1;; ++it) {
    if (mbar_try(bar, parity)) return true;
    if ((it & 63) == 0) {
      if (*abort_flag) return false;
      if (global_ns() - t0 > SC_WAIT_NS) {
        *abort_flag = 1;
        atomicExch(&status[3], 1);
        return false;
      }
    }
  }
}
// Lane 0 waits for the warp (a warp-uniform result).
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
    if ((it & 63) == 63 && global_ns() - t0 > SC_WAIT_NS) break;
  }
  atomicExch(&status[3], 1);
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, uint32_t bar,
                                            int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];\n" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

template <bool BF16>
__device__ __forceinline__ void mma_split(uint32_t tmem, uint64_t adesc, uint64_t bdesc,
                                          uint32_t idesc, uint32_t accumulate) {
  if (BF16)
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(
            tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
  else
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(
            tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}
__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar)
      : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t addr, float *v) {
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

// Scatter table of one tile, built by the table warp ahead of the epilogue: per column the
// target's first entry in L (-1: no tiled target) and its run slot (a run: consecutive
// columns with one target supernode); per slot the offset of the run's relative indices and
// its first column; for the first SC_RUNS slots the target position of every tile row.
constexpr int SC_RUNS = 16;
struct ScTable {
  int64_t base[128];
  int slot[128];
  int ro[128];
  int rj[SC_RUNS];
  int pos[SC_RUNS][128];
  int md, i0, j0, nslots;
};

template <bool BF16>
__global__ void __launch_bounds__(SC_THREADS, 1)
    k_scatter_tc(DevSym S, const CUtensorMap *__restrict__ maps, const ScTile *__restrict__ tiles,
                 int count, ScatterCols C) {
  using F = Sc<BF16>;
  constexpr int NP = F::PLANES;
  extern __shared__ unsigned char sc_dyn[];
  __shared__ __align__(8) uint64_t full_bar[SC_MAX_STAGES], empty_bar[SC_MAX_STAGES];
  __shared__ __align__(8) uint64_t accf_bar[2], acce_bar[2], tblf_bar[2], tble_bar[2], done_bar;
  __shared__ __align__(16) ScTable tbl[2];
  __shared__ uint32_t tmem_base;
  __shared__ volatile int abort_flag;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t sbase = (smem_u32(sc_dyn) + 1023u) & ~1023u;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(&tmem_base)),
                 "r"(SC_TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid == 32 * SC_MMA) {
    for (int s = 0; s < F::STAGES; ++s) {
      mbar_init(smem_u32(&full_bar[s]), 1);
      mbar_init(smem_u32(&empty_bar[s]), 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(smem_u32(&accf_bar[b]), 1);
      mbar_init(smem_u32(&acce_bar[b]), SC_EPI_WARPS);
      mbar_init(smem_u32(&tblf_bar[b]), 32);
      mbar_init(smem_u32(&tble_bar[b]), SC_EPI_WARPS);
    }
    mbar_init(smem_u32(&done_bar), 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = tmem_base;

  if (warp == SC_PRODUCER) {
    // ------------------------------ TMA producer ------------------------------
    if (lane == 0) {
      int stage = 0, armed[SC_MAX_STAGES];
      uint32_t phase = 0;
      for (int s = 0; s < SC_MAX_STAGES; ++s) armed[s] = 0;
      bool ok = true;
      const int ns = S.nsuper;
      for (int t = blockIdx.x; t < count && ok; t += gridDim.x) {
        const ScTile tl = tiles[t];
        // maps: plane p of supernode d at [(box * NP + p) * nsuper + d], box 0: 128 rows,
        // box 1: 64 rows (B of a tile of at most 64 columns)
        const bool narrow = tl.ncol <= 64;
        const CUtensorMap *amap = maps + tl.d, *bmap = maps + (narrow ? NP : 0) * ns + tl.d;
        const bool diag = tl.i0 == tl.j0;   // B = the first ncol rows of A
        const uint32_t bytes = NP * F::OP + (diag ? 0 : NP * (narrow ? F::OP / 2 : F::OP));
        for (int kc = 0; kc < tl.nk; ++kc) {
          if (!mbar_wait(smem_u32(&empty_bar[stage]), phase ^ 1u, &abort_flag, S.status)) {
            ok = false;
            break;
          }
          const uint32_t fb = smem_u32(&full_bar[stage]);
          const uint32_t sa = sbase + stage * F::STAGE;
          mbar_arrive_tx(fb, bytes);
          armed[stage] += 1;
          const int x = tl.k0 + kc * SC_KCHUNK;
#pragma unroll
          for (int p = 0; p < NP; ++p) {
            tma_load_2d(sa + p * F::OP, amap + p * ns, fb, x, tl.i0);
            if (!diag) tma_load_2d(sa + (NP + p) * F::OP, bmap + p * ns, fb, x, tl.j0);
          }
          if (++stage == F::STAGES) { stage = 0; phase ^= 1u; }
        }
      }
      // loads in flight land before the CTA leaves
      for (int s = 0; s < F::STAGES; ++s)
        if (armed[s] > 0) mbar_drain(smem_u32(&full_bar[s]), (uint32_t)(armed[s] - 1) & 1u, S.status);
    }
    __syncwarp();
  } else if (warp == SC_MMA) {
    // ------------------------------- MMA issuer -------------------------------
    if (lane == 0) {
      int stage = 0, buf = 0;
      uint32_t phase = 0, accphase[2] = {0, 0};
      bool ok = true;
      for (int t = blockIdx.x; t < count && ok; t += gridDim.x) {
        const int i0 = tiles[t].i0, j0 = tiles[t].j0, nk = tiles[t].nk;
        const bool diag = i0 == j0;
        const uint32_t idesc = sc_idesc(F::FMT, tiles[t].ncol <= 64 ? 64u : 128u);
        if (!mbar_wait(smem_u32(&acce_bar[buf]), accphase[buf] ^ 1u, &abort_flag, S.status)) break;
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        const uint32_t dt = tmem + (uint32_t)buf * 128u;
        for (int kc = 0; kc < nk; ++kc) {
          if (!mbar_wait(smem_u32(&full_bar[stage]), phase, &abort_flag, S.status)) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
          // plane p of A at a[p], of B at b[p] (B = A for a diagonal tile)
          const uint32_t a0 = sbase + stage * F::STAGE;
          uint32_t a[NP], b[NP];
#pragma unroll
          for (int p = 0; p < NP; ++p) {
            a[p] = a0 + p * F::OP;
            b[p] = diag ? a[p] : a0 + (NP + p) * F::OP;
          }
#pragma unroll
          for (int kk = 0; kk < SC_KCHUNK / F::KSTEP; ++kk) {
            const uint32_t o = 32u * kk;   // one MMA's K = 32 bytes along the swizzled row
            auto mma = [&](int pa, int pb, uint32_t acc) {
              mma_split<BF16>(dt, sw_desc(a[pa] + o, F::SBO, F::LAYOUT),
                              sw_desc(b[pb] + o, F::SBO, F::LAYOUT), idesc, acc);
            };
            mma(0, 0, (kc | kk) != 0);   // hi hi'
            if (BF16) {                  // planes hi, mid, lo
              mma(0, 1, 1u);
              mma(1, 0, 1u);
              mma(1, 1, 1u);
              mma(0, 2, 1u);
              mma(2, 0, 1u);
            } else {                     // planes hi, lo
              mma(1, 0, 1u);
              mma(0, 1, 1u);
            }
          }
          mma_commit(smem_u32(&empty_bar[stage]));   // the stage is free once these are done
          if (++stage == F::STAGES) { stage = 0; phase ^= 1u; }
        }
        if (!ok) break;
        mma_commit(smem_u32(&accf_bar[buf]));          // the tile's product: to the epilogue
        accphase[buf] ^= 1u;
        buf ^= 1;
      }
      // every MMA issued has completed before TMEM is freed
      mma_commit(smem_u32(&done_bar));
      mbar_drain(smem_u32(&done_bar), 0u, S.status);
    }
    __syncwarp();
  } else if (warp == SC_TABLE) {
    // ------------------------------- table warp -------------------------------
    // lane: columns 4 lane .. 4 lane + 3 of the tile, rows lane + 32 k
    int b = 0;
    uint32_t tph[2] = {0, 0};
    for (int t = blockIdx.x; t < count; t += gridDim.x) {
      if (!mbar_wait_warp(smem_u32(&tble_bar[b]), tph[b] ^ 1u, &abort_flag, S.status)) break;
      const ScTile tl = tiles[t];
      const int md = tl.md;
      const int64_t co = tl.co;
      ScTable &T = tbl[b];
      if (tl.dense) {
        // d's own columns j0 .. j0 + ncol - 1, one run, row i at position i
        const int wdd = S.super[tl.d + 1] - S.super[tl.d];
        const int64_t xp = S.xptr[tl.d];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int c = 4 * lane + q, j = tl.j0 + c;
          const int64_t cbv = (c < tl.ncol && j < wdd) ? xp + (int64_t)j * md : -1;
          T.base[c] = cbv;
          T.slot[c] = cbv >= 0 ? 0 : -1;
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) T.pos[0][lane + 32 * k] = tl.i0 + lane + 32 * k;
        if (lane == 0) {
          T.ro[0] = 0;
          T.rj[0] = tl.j0;
          T.md = md;
          T.i0 = tl.i0;
          T.j0 = tl.j0;
          T.nslots = 1;
        }
        __syncwarp();
        mbar_arrive(smem_u32(&tblf_bar[b]));
        tph[b] ^= 1u;
        b ^= 1;
        continue;
      }
      int64_t cb[4];
      int ro[4], fl[4], nf = 0;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int j = tl.j0 + 4 * lane + q;
        cb[q] = j < md ? C.base[co + j] : -1;
        ro[q] = j < md ? C.rel[co + j] : 0;
      }
      // a run starts at a tiled column whose predecessor is untiled or has another run
      int64_t pcb = __shfl_up_sync(0xffffffffu, cb[3], 1);
      const int pro = __shfl_up_sync(0xffffffffu, ro[3], 1);
      if (lane == 0) pcb = -1;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int64_t prevb = q ? cb[q - 1] : pcb;
        const int prevr = q ? ro[q - 1] : pro;
        fl[q] = cb[q] >= 0 && (prevb < 0 || prevr != ro[q]);
        nf += fl[q];
      }
      int incl = nf;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
      }
      int sl = incl - nf;   // runs started before my first column
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int c = 4 * lane + q;
        sl += fl[q];
        T.base[c] = cb[q];
        T.slot[c] = cb[q] >= 0 ? sl - 1 : -1;
        if (fl[q]) {
          T.ro[sl - 1] = ro[q];
          if (sl - 1 < SC_RUNS) T.rj[sl - 1] = tl.j0 + c;
        }
      }
      const int nslots = __shfl_sync(0xffffffffu, incl, 31);
      if (lane == 0) {
        T.md = md;
        T.i0 = tl.i0;
        T.j0 = tl.j0;
        T.nslots = nslots;
      }
      __syncwarp();
      // target positions of the tile rows for the first SC_RUNS runs (rows before a run's
      // first column have no position in its target and are not read)
      const int ns = min(nslots, SC_RUNS);
      for (int s0 = 0; s0 < ns; s0 += 4) {
        int pv[4][4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int s = s0 + u;
          const int rro = s < ns ? T.ro[s] : 0, rj = s < ns ? T.rj[s] : INT_MAX;
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            const int i = tl.i0 + lane + 32 * k;
            pv[u][k] = (i < md && i >= rj) ? C.relidx[rro + i] : 0;
          }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
          if (s0 + u < ns)
#pragma unroll
            for (int k = 0; k < 4; ++k) T.pos[s0 + u][lane + 32 * k] = pv[u][k];
      }
      __syncwarp();
      mbar_arrive(smem_u32(&tblf_bar[b]));   // every lane: its writes are released
      tph[b] ^= 1u;
      b ^= 1;
    }
  } else if (warp < SC_EPI_WARPS) {
    // -------------------------------- epilogue --------------------------------
    // warp w: tile rows 32 (w % 4) + lane (its TMEM lane quarter), columns 32 (w / 4) ..
    const int rt = 32 * (warp & 3) + lane, c0 = 32 * (warp >> 2);
    int buf = 0, b = 0;
    uint32_t accphase[2] = {0, 0}, tph[2] = {0, 0};
    for (int t = blockIdx.x; t < count; t += gridDim.x) {
      if (!mbar_wait_warp(smem_u32(&tblf_bar[b]), tph[b], &abort_flag, S.status)) break;
      if (!mbar_wait_warp(smem_u32(&accf_bar[buf]), accphase[buf], &abort_flag, S.status)) break;
      accphase[buf] ^= 1u;
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      float v[32];
      tmem_ld32(tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)buf * 128u + (uint32_t)c0, v);
      asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(&acce_bar[buf]));
      buf ^= 1;
      // row i of d: add minus C(i, j) for every column j <= i whose target is tiled
      const ScTable &T = tbl[b];
      const int i = T.i0 + rt;
      if (i < T.md) {
        const int jn = min(32, i - T.j0 - c0 + 1);   // columns j = j0 + c0 + q with j <= i
#pragma unroll
        for (int q = 0; q < 32; ++q) {
          if (q < jn) {
            const int sl = T.slot[c0 + q];
            if (sl >= 0) {
              const int pos = sl < SC_RUNS ? T.pos[sl][rt] : C.relidx[T.ro[sl] + i];
              atomicAdd(S.L + T.base[c0 + q] + pos, -(double)v[q]);
            }
          }
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(&tble_bar[b]));
      tph[b] ^= 1u;
      b ^= 1;
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem),
                 "r"(SC_TMEM_COLS));
}

// Small contributions in FP64: CTA = one descendant d from row c0 (r = md - c0 <= 128 rows);
// its rows c0.. are staged column by column in shared memory (V[k][row], rows padded to a
// multiple of 32, at most SC_SMALL_ELEMS values); thread t owns row i = c0 + t and adds
// minus sum_k L(i, k) L(j, k) to the target entry of every column j <= i with a tiled target.
__global__ void __launch_bounds__(128) k_scatter_small(DevSym S, const int2 *__restrict__ tasks,
                                                       ScatterCols C) {
  __shared__ double V[SC_SMALL_ELEMS];
  __shared__ int64_t cbase[128];
  __shared__ int crel[128];
  const int d = tasks[blockIdx.x].x, c0 = tasks[blockIdx.x].y;
  const int wd = S.super[d + 1] - S.super[d];
  const int md = (int)(S.rowptr[d + 1] - S.rowptr[d]);
  const int r = md - c0, R = (r + 31) & ~31;
  const double *Ld = S.L + S.xptr[d];
  const int64_t co = C.coff[d];
  for (int e = threadIdx.x; e < wd * R; e += blockDim.x) {
    const int k = e / R, q = e - k * R;
    V[e] = q < r ? Ld[(size_t)k * md + c0 + q] : 0.0;
  }
  for (int q = threadIdx.x; q < r; q += blockDim.x) {
    cbase[q] = C.base[co + c0 + q];
    crel[q] = C.rel[co + c0 + q];
  }
  __syncthreads();
  const int t = threadIdx.x;
  if (t >= r) return;
  const int i = c0 + t;
  int cur = INT_MIN, pos = 0;
  for (int q = 0; q <= t; ++q) {
    const int64_t b = cbase[q];
    if (b < 0) continue;
    double acc = 0.0;
    for (int k = 0; k < wd; ++k) acc = fma(V[k * R + t], V[k * R + q], acc);
    const int ro = crel[q];
    if (ro != cur) {
      cur = ro;
      pos = C.relidx[ro + i];
    }
    atomicAdd(S.L + b + pos, -acc);
  }
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

bool scatter_tc_configure(std::string &err) {
  cudaError_t e = cudaFuncSetAttribute(k_scatter_tc<false>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, SC_SMEM);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_scatter_tc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             SC_SMEM);
  if (e != cudaSuccess) {
    err = std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e);
    return false;
  }
  return true;
}

size_t scatter_maps_count(int nsuper, bool bf16) { return (size_t)2 * (bf16 ? 3 : 2) * nsuper; }

bool build_scatter_maps(const std::vector<int> &super, const std::vector<int64_t> &rowptr,
                        const std::vector<int64_t> &xk, const std::vector<char> &used, float *Lk,
                        bool bf16, void *maps_host, std::string &err) {
  EncodeTiled enc = encode_fn();
  if (!enc) {
    err = "cuTensorMapEncodeTiled is not available from the driver";
    return false;
  }
  CUtensorMap *maps = static_cast<CUtensorMap *>(maps_host);
  const int ns = (int)super.size() - 1, np = bf16 ? 3 : 2, esz = bf16 ? 2 : 4;
  for (int box = 0; box < 2; ++box)
    for (int d = 0; d < ns; ++d) {
      if (!(used[d] & (box == 0 ? 1 : 2))) continue;
      const uint64_t w = super[d + 1] - super[d], m = rowptr[d + 1] - rowptr[d];
      const uint64_t wp = (uint64_t)(bf16 ? kmirror_pitch_bf16((int)w) : kmirror_pitch_tf32((int)w));
      const cuuint64_t dims[2] = {w, m};
      const cuuint64_t strides[1] = {wp * esz};
      const cuuint32_t boxdim[2] = {SC_KCHUNK, (cuuint32_t)(box == 0 ? 128 : 64)};
      const cuuint32_t estr[2] = {1, 1};
      // planes hi, (mid,) lo of m rows each (rows outside a plane read zeros)
      unsigned char *base = reinterpret_cast<unsigned char *>(Lk + xk[d]);
      for (int p = 0; p < np; ++p) {
        CUresult r = enc(&maps[(size_t)(box * np + p) * ns + d],
                         bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                         2, base + (size_t)p * m * wp * esz, dims, strides, boxdim, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE,
                         bf16 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_128B,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) {
          err = "cuTensorMapEncodeTiled failed for supernode " + std::to_string(d) + " (code " +
                std::to_string((int)r) + ")";
          return false;
        }
      }
    }
  return true;
}

void launch_scatter_tc(const DevSym &S, const void *maps, const ScTile *tiles, int count,
                       const ScatterCols &C, int reserve, bool bf16, cudaStream_t st) {
  if (count <= 0) return;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int ctas = std::max(1, std::min(count, sms - reserve));
  const CUtensorMap *m = static_cast<const CUtensorMap *>(maps);
  if (bf16)
    k_scatter_tc<true><<<ctas, SC_THREADS, SC_SMEM, st>>>(S, m, tiles, count, C);
  else
    k_scatter_tc<false><<<ctas, SC_THREADS, SC_SMEM, st>>>(S, m, tiles, count, C);
}

void launch_scatter_small(const DevSym &S, const int2 *tasks, int count, const ScatterCols &C,
                          cudaStream_t st) {
  if (count <= 0) return;
  k_scatter_small<<<count, 128, 0, st>>>(S, tasks, C);
}

}  // namespace swc
