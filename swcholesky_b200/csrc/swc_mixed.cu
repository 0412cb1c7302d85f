// BF16x3 Schur updates (SWC_MODE_MIXED_BF16X3): the SYRK/GEMM updates of the tiled class
// (the bulk of the flops) computed as split-bfloat16 products on the tensor cores, with FP32
// accumulation inside one descendant's product and FP64 accumulation across descendants.
//
// Every finished panel (small-class supernodes, TRSM'd tiles of the tiled class) also
// writes a split copy of itself (the "mirror", same indexing as L): each value x as three
// bfloat16 pieces hi = bf16(x), mid = bf16(x - hi), lo = bf16(x - hi - mid), so the
// tensor-core kernel loads fragments without any conversion.  A product sums the six piece
// products whose order is at most two pieces below the leading one (the split-bfloat16
// method of Henry, Tang and Heinecke, ARITH 2019), about 2^-24 relative error -- the
// FP32-class accuracy that FP64 iterative refinement then removes.  POTRF, TRSM, the
// diagonal tiles and the small supernodes stay FP64.  (The split-TF32 mode runs its updates
// on tcgen05: swc_update_tc.cu.)
#include <cuda_runtime.h>

#include <cstdint>

#include "swc_engine.h"

namespace swc {

namespace {

constexpr int MXT = 128;            // threads (4 warps, 2x2 warp grid of 32x32 sub-tiles)
constexpr int KF = 16;              // k-chunk (2 steps of k8, 1 of k16)
constexpr int LDF = TB + 4;         // padded row of a staged k-slice ({hi, lo} pairs):
                                    // 64-bit fragment loads conflict-free
constexpr int STAGEF = 2 * KF * LDF;
static_assert(MXT == 2 * TB, "staging pattern: two threads per tile row");

__device__ __forceinline__ int lbound_m(const int *a, int len, int key) {
  int lo = 0, hi = len;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (a[mid] < key) lo = mid + 1; else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ void cp_async8f(float2 *smem, const float2 *gmem, bool pred) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  const int sz = pred ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }


// Accumulator of one warp's 32x32 sub-tile: 2 x 4 MMA tiles of 16x8, fragment layout of
// m16n8k8: c0 (g, 2t), c1 (g, 2t+1), c2 (g+8, 2t), c3 (g+8, 2t+1), g = lane/4, t = lane%4.
struct Acc32 {
  float v[2][4][4];
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e) v[i][j][e] = 0.0f;
  }
};
__device__ __forceinline__ int mx_row(int i, int e) {
  return ((threadIdx.x >> 5) >> 1) * 32 + 16 * i + ((threadIdx.x & 31) >> 2) + ((e & 2) ? 8 : 0);
}
__device__ __forceinline__ int mx_col(int j, int e) {
  return ((threadIdx.x >> 5) & 1) * 32 + 8 * j + 2 * (threadIdx.x & 3) + (e & 1);
}

// Stages one k-chunk of both operands (gathered rows; -1 = zero row) from the mirror.
// Thread t always copies tile row t % 64 at chunk offsets t / 64, t / 64 + 2, ...; its
// source rows (ra, rb) are looked up once per product, so a copy costs one pointer step.
__device__ __forceinline__ void load_chunk_f(const float2 *__restrict__ Lf, int ld, int ra, int rb,
                                             int K, int k0, float2 *st) {
  const int i = threadIdx.x & (TB - 1), kq = threadIdx.x >> 6;
  float2 *As = st + kq * LDF + i, *Bs = st + KF * LDF + kq * LDF + i;
  const float2 *pa = Lf + (size_t)(k0 + kq) * ld + (ra >= 0 ? ra : 0);
  const float2 *pb = Lf + (size_t)(k0 + kq) * ld + (rb >= 0 ? rb : 0);
  const size_t step = (size_t)2 * ld;
#pragma unroll
  for (int it = 0; it < KF / 2; ++it) {
    const bool kin = k0 + kq + 2 * it < K;
    cp_async8f(As + 2 * it * LDF, kin && ra >= 0 ? pa : Lf, kin && ra >= 0);
    cp_async8f(Bs + 2 * it * LDF, kin && rb >= 0 ? pb : Lf, kin && rb >= 0);
    pa += step;
    pb += step;
  }
  cp_commit();
}

__device__ __forceinline__ void mma_bf16(float (&c)[4], const unsigned (&a)[4], const unsigned (&b)[2]) {
  asm("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Two BF16x3 elements (bits: x = hi | mid << 16, y = lo) -> one register of component p for
// the MMA, the element with the lower k index in the low half.
__device__ __forceinline__ unsigned pack_bf16(uint2 e0, uint2 e1, int p) {
  return p == 0 ? ((e0.x & 0xffffu) | (e1.x << 16))
       : p == 1 ? ((e0.x >> 16) | (e1.x & 0xffff0000u))
                : ((e0.y & 0xffffu) | (e1.y << 16));
}

// One staged k-chunk, BF16x3: elements are three bfloat16 pieces {hi, mid, lo} (x = hi + mid
// + lo to about 24 bits); per k16 step the six partial products whose order is at most
// two pieces below the leading one (lo*hi', mid*mid', hi*lo', mid*hi', hi*mid', hi*hi',
// small terms first), FP32 accumulation.  Fragment layout of m16n8k16 .bf16: A regs
// {(g, 2t..2t+1), (g+8, 2t..), (g, 2t+8..), (g+8, 2t+8..)}, B regs {(2t..2t+1, g),
// (2t+8..2t+9, g)}, g = lane/4, t = lane%4.
__device__ __forceinline__ void chunk_bf16(const float2 *Asf, const float2 *Bsf, int wr, int wc,
                                           int g, int t, unsigned rmask, unsigned cmask,
                                           Acc32 &acc) {
  const uint2 *As = reinterpret_cast<const uint2 *>(Asf), *Bs = reinterpret_cast<const uint2 *>(Bsf);
#pragma unroll
  for (int k16 = 0; k16 < KF; k16 += 16) {
    unsigned a[3][2][4], b[3][4][2];
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int r = wr + 16 * i + g;
      const int k0 = k16 + 2 * t;
      const uint2 e00 = As[k0 * LDF + r], e01 = As[(k0 + 1) * LDF + r];
      const uint2 e10 = As[k0 * LDF + r + 8], e11 = As[(k0 + 1) * LDF + r + 8];
      const uint2 e20 = As[(k0 + 8) * LDF + r], e21 = As[(k0 + 9) * LDF + r];
      const uint2 e30 = As[(k0 + 8) * LDF + r + 8], e31 = As[(k0 + 9) * LDF + r + 8];
#pragma unroll
      for (int p = 0; p < 3; ++p) {
        a[p][i][0] = pack_bf16(e00, e01, p);
        a[p][i][1] = pack_bf16(e10, e11, p);
        a[p][i][2] = pack_bf16(e20, e21, p);
        a[p][i][3] = pack_bf16(e30, e31, p);
      }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int n = wc + 8 * j + g;
      const int k0 = k16 + 2 * t;
      const uint2 f00 = Bs[k0 * LDF + n], f01 = Bs[(k0 + 1) * LDF + n];
      const uint2 f10 = Bs[(k0 + 8) * LDF + n], f11 = Bs[(k0 + 9) * LDF + n];
#pragma unroll
      for (int p = 0; p < 3; ++p) {
        b[p][j][0] = pack_bf16(f00, f01, p);
        b[p][j][1] = pack_bf16(f10, f11, p);
      }
    }
    constexpr int PA[6] = {2, 1, 0, 1, 0, 0}, PB[6] = {0, 1, 2, 0, 1, 0};
#pragma unroll
    for (int q = 0; q < 6; ++q)
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
          if (((rmask >> i) & (cmask >> j)) & 1u) mma_bf16(acc.v[i][j], a[PA[q]][i], b[PB[q]][j]);
  }
}

// acc += A B^T over K columns from the BF16x3 mirror, with A / B rows gathered through
// ia / ib.  rmask / cmask: this warp's non-empty 16-row and 8-column groups.
__device__ __forceinline__ void split_product(const float2 *__restrict__ Lf, int ld, const int *ia,
                                              const int *ib, int K, float2 *stages, Acc32 &acc) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wr = (warp >> 1) * 32, wc = (warp & 1) * 32;
  const int g = lane >> 2, t = lane & 3;
  const int nchunks = (K + KF - 1) / KF;
  __syncthreads();
  unsigned rmask = 0, cmask = 0;
#pragma unroll
  for (int i = 0; i < 2; ++i)
    if (__any_sync(0xffffffffu, ia[wr + 16 * i + (lane & 15)] >= 0)) rmask |= 1u << i;
#pragma unroll
  for (int j = 0; j < 4; ++j)
    if (__any_sync(0xffffffffu, ib[wc + 8 * j + (lane & 7)] >= 0)) cmask |= 1u << j;
  const int ra = ia[threadIdx.x & (TB - 1)], rb = ib[threadIdx.x & (TB - 1)];
  load_chunk_f(Lf, ld, ra, rb, K, 0, stages);
  for (int c = 0; c < nchunks; ++c) {
    if (c + 1 < nchunks) {
      load_chunk_f(Lf, ld, ra, rb, K, (c + 1) * KF, stages + ((c + 1) & 1) * STAGEF);
      cp_wait<1>();
    } else {
      cp_wait<0>();
    }
    __syncthreads();
    const float2 *As = stages + (c & 1) * STAGEF, *Bs = As + KF * LDF;
    if (rmask && cmask) chunk_bf16(As, Bs, wr, wc, g, t, rmask, cmask, acc);
    __syncthreads();
  }
}

// Mixed-precision tile-owner update (same tasks and pair lists as the FP64 kernel).
constexpr int UPDM_SMEM = 2 * STAGEF * 8 + 3 * TB * 4;

__global__ void __launch_bounds__(MXT, 4) k_update_tiles_mx(DevSym S, const int4 *tasks,
                                                           const int *task_end,
                                                           const int4 *pairs, int count) {
  extern __shared__ float2 dynf[];
  float2 *stages = dynf;
  int *trow = reinterpret_cast<int *>(dynf + 2 * STAGEF);
  int *ia = trow + TB, *ib = ia + TB;
  const int4 tk = tasks[blockIdx.x];
  const int s = tk.x, r0 = tk.y, c0 = tk.z;
  const int p_begin = tk.w, p_end = task_end[blockIdx.x];
  const int tid = threadIdx.x;
  const int f = S.super[s];
  const int w = S.super[s + 1] - f;
  const int64_t rb = S.rowptr[s];
  const int m = (int)(S.rowptr[s + 1] - rb);
  const int nrow = min(TB, m - r0), ncol = min(TB, w - c0);
  const int gc_lo = f + c0;
  for (int i = tid; i < nrow; i += MXT) trow[i] = S.Ls[rb + r0 + i];
  double acc64[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc64[i][j][e] = 0.0;
  for (int q = p_begin; q < p_end; ++q) {
    const int4 pr = pairs[q];
    const int d = pr.x, a0 = pr.y, b0 = pr.z;
    const int na = pr.w & 0xffff, nb = pr.w >> 16;
    const int wd = S.super[d + 1] - S.super[d];
    const int64_t rbd = S.rowptr[d];
    const int md = (int)(S.rowptr[d + 1] - rbd);
    const int *Lsd = S.Ls + rbd;
    __syncthreads();
    if (tid < TB) { ia[tid] = -1; ib[tid] = -1; }
    __syncthreads();
    if (tid < na) {
      const int key = Lsd[a0 + tid];
      const int pos = lbound_m(trow, nrow, key);
      if (pos < nrow && trow[pos] == key) ia[pos] = a0 + tid;
      else atomicExch(&S.status[1], 1);
    } else if (tid >= TB && tid < TB + nb) {
      const int cc = Lsd[b0 + tid - TB] - gc_lo;
      if (cc >= 0 && cc < ncol) ib[cc] = b0 + tid - TB;
      else atomicExch(&S.status[1], 1);
    }
    Acc32 acc;
    acc.zero();
    split_product(S.Lf + S.xptr[d], md, ia, ib, wd, stages, acc);
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e) acc64[i][j][e] += (double)acc.v[i][j][e];
  }
  double *P = S.L + S.xptr[s];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int r = mx_row(i, e), c = mx_col(j, e);
        if (r < nrow && c < ncol && r0 + r >= c0 + c)
          P[(size_t)(c0 + c) * m + r0 + r] -= acc64[i][j][e];
      }
}

}  // namespace

bool mixed_configure(std::string &err) {
  cudaError_t e = cudaFuncSetAttribute(k_update_tiles_mx,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, UPDM_SMEM);
  if (e != cudaSuccess) {
    err = std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e);
    return false;
  }
  return true;
}

void launch_update_tiles_mx(const DevSym &S, const int4 *tasks, const int *task_end,
                            const int4 *pairs, int count, cudaStream_t st) {
  if (count <= 0) return;
  k_update_tiles_mx<<<count, MXT, UPDM_SMEM, st>>>(S, tasks, task_end, pairs, count);
}

}  // namespace swc
