// FP64 kernels of the supernodal numeric factorization.
//
// The work of the reference executor (cholesky/sw_parallel_PB_Cholesky_05.c:209-484) is
// split by supernode size class:
//
//   k_factor_small   one CTA factors one supernode whose panel fits in shared memory:
//                    assembly of A (.c:211-224), every update from its prune set with the
//                    relative-index scatter fused in (.c:254-378), then POTRF and TRSM on
//                    the panel (.c:419-484).  Many such CTAs run per level.
//   k_assemble       copies A's columns into the panels of the tiled class.
//   k_update_tiles   tile-owner left-looking update: each CTA owns a 64x64 tile of a
//                    target panel and accumulates, in shared memory, the contribution of
//                    every descendant in the prune set (the SYRK/GEMM of .c:299-359 limited
//                    to the tile, scattered through relative indices, .c:364-378); the tile
//                    is written once.  Deterministic: no atomics, fixed update order.
//   k_diag_step,     blocked right-looking dense factorization of a wide supernode by
//   k_trsm_step,     64-column blocks: per block, POTRF of the diagonal block (and its
//   k_syrk_step      inverse), the TRSM of the tiles below it as a DMMA product with that
//                    inverse, and the trailing SYRK/GEMM update; the next diagonal block's
//                    update and POTRF run concurrently with that trailing update.
//
// All arithmetic is FP64; tiles are 64x64 with 256 threads, each thread holding a 4x4
// register micro-tile.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdint>

#include "swc_engine.h"

namespace swc {

namespace {

constexpr int NT = 256;
constexpr int KC = 16;

__device__ __forceinline__ int lbound(const int *a, int len, int key) {
  int lo = 0, hi = len;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (a[mid] < key) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// {hi, lo} split of x for the tensor-core mirror: hi = tf32(x), lo = tf32(x - hi).
__device__ __forceinline__ float2 split_tf32(double x) {
  const float xf = (float)x;
  unsigned hi, lo;
  asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(hi) : "f"(xf));
  asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(lo) : "f"(xf - __uint_as_float(hi)));
  return make_float2(__uint_as_float(hi), __uint_as_float(lo));
}

// Three bfloat16 pieces of x: hi = bf16(x), mid = bf16(x - hi), lo = bf16(x - hi - mid)
// (the remainders are exact in FP64).
struct Bf16x3 {
  unsigned short hi, mid, lo;
};
__device__ __forceinline__ Bf16x3 split_bf16x3(double x) {
  const __nv_bfloat16 hi = __float2bfloat16_rn((float)x);
  const double r1 = x - (double)__bfloat162float(hi);
  const __nv_bfloat16 mid = __float2bfloat16_rn((float)r1);
  const double r2 = r1 - (double)__bfloat162float(mid);
  const __nv_bfloat16 lo = __float2bfloat16_rn((float)r2);
  return Bf16x3{__bfloat16_as_ushort(hi), __bfloat16_as_ushort(mid), __bfloat16_as_ushort(lo)};
}

// The mirror entries of value x of row r, column c of supernode s (m rows, w columns), in
// the K-major split mirror at (float *)Lf + xk[s], format xk[nsuper]: 0, hi / lo TF32
// planes; 1, hi / mid / lo bfloat16 planes (row pitch kmirror_pitch_tf32 / _bf16 (w)).
__device__ __forceinline__ void store_mirror(const DevSym &S, int s, int m, int w, int r, int c,
                                             double x) {
  float *base = reinterpret_cast<float *>(S.Lf) + S.xk[s];
  if (S.xk[S.nsuper] == 0) {
    const int wp = kmirror_pitch_tf32(w);
    const float2 v = split_tf32(x);
    base[(size_t)r * wp + c] = v.x;
    base[((size_t)m + r) * wp + c] = v.y;
  } else {
    const int wq = kmirror_pitch_bf16(w);
    unsigned short *b = reinterpret_cast<unsigned short *>(base);
    const Bf16x3 v = split_bf16x3(x);
    b[(size_t)r * wq + c] = v.hi;
    b[((size_t)m + r) * wq + c] = v.mid;
    b[((size_t)2 * m + r) * wq + c] = v.lo;
  }
}

// The whole m x w panel P (column-major, ld m) of supernode s into the mirror; threads
// t, t + nt, ... (consecutive threads write consecutive mirror entries of a row).
__device__ __forceinline__ void store_mirror_panel(const DevSym &S, int s, int m, int w,
                                                   const double *P, int t, int nt) {
  float *base = reinterpret_cast<float *>(S.Lf) + S.xk[s];
  if (S.xk[S.nsuper] == 0) {
    const int wp = kmirror_pitch_tf32(w);
    float *hi = base, *lo = hi + (size_t)m * wp;
    for (int e = t; e < m * w; e += nt) {
      const int r = e / w, c = e - r * w;
      const float2 v = split_tf32(P[(size_t)c * m + r]);
      hi[(size_t)r * wp + c] = v.x;
      lo[(size_t)r * wp + c] = v.y;
    }
  } else {
    const int wq = kmirror_pitch_bf16(w);
    unsigned short *hi = reinterpret_cast<unsigned short *>(base);
    unsigned short *mid = hi + (size_t)m * wq, *lo = mid + (size_t)m * wq;
    for (int e = t; e < m * w; e += nt) {
      const int r = e / w, c = e - r * w;
      const Bf16x3 v = split_bf16x3(P[(size_t)c * m + r]);
      hi[(size_t)r * wq + c] = v.hi;
      mid[(size_t)r * wq + c] = v.mid;
      lo[(size_t)r * wq + c] = v.lo;
    }
  }
}

// An nr x nc block of the panel (rows r0.., columns c0..), staged in shared memory as
// X[c * ld + r], into the mirror: consecutive threads write consecutive columns of a mirror
// row (the rows are K-major), so every warp store is one contiguous piece of a plane.
__device__ __forceinline__ void store_mirror_block(const DevSym &S, int s, int m, int w, int r0,
                                                   int c0, int nr, int nc, const double *X,
                                                   int ld, int t, int nt) {
  float *base = reinterpret_cast<float *>(S.Lf) + S.xk[s];
  if (S.xk[S.nsuper] == 0) {
    const int wp = kmirror_pitch_tf32(w);
    float *hi = base, *lo = hi + (size_t)m * wp;
    for (int e = t; e < TB * TB; e += nt) {
      const int r = e >> 6, c = e & (TB - 1);
      if (r >= nr || c >= nc) continue;
      const float2 v = split_tf32(X[c * ld + r]);
      hi[(size_t)(r0 + r) * wp + c0 + c] = v.x;
      lo[(size_t)(r0 + r) * wp + c0 + c] = v.y;
    }
  } else {
    const int wq = kmirror_pitch_bf16(w);
    unsigned short *hi = reinterpret_cast<unsigned short *>(base);
    unsigned short *mid = hi + (size_t)m * wq, *lo = mid + (size_t)m * wq;
    for (int e = t; e < TB * TB; e += nt) {
      const int r = e >> 6, c = e & (TB - 1);
      if (r >= nr || c >= nc) continue;
      const Bf16x3 v = split_bf16x3(X[c * ld + r]);
      hi[(size_t)(r0 + r) * wq + c0 + c] = v.hi;
      mid[(size_t)(r0 + r) * wq + c0 + c] = v.mid;
      lo[(size_t)(r0 + r) * wq + c0 + c] = v.lo;
    }
  }
}

// The same for one warp, out of line (keeps the warp-per-supernode kernel's registers).
__device__ __noinline__ void store_mirror_panel_warp(const DevSym &S, int s, int m, int w,
                                                     const double *P) {
  store_mirror_panel(S, s, m, w, P, threadIdx.x & 31, 32);
}

__device__ __forceinline__ void flag_structure_error(const DevSym &S) {
  atomicExch(&S.status[1], 1);
}

// Update of a small panel P (m rows, column-major) by descendant d: rows lb.. of d's panel
// (Ld points at row lb; md = d's rows, wd = its width, nr rows from lb, the first n1 of them
// inside the target's columns).  The rows go through the shared slab (capacity slab_cap
// doubles) a column chunk at a time, then P[rel[a]][rel[b]] -= sum_k X[b][k] X[a][k] for
// a < n1, b >= a, from shared memory.  The first chunk is already in the slab (staged from
// registers loaded ahead, see prefetch_chunk); later chunks load here.  Threads t, t + nt,
// ...; the barrier is the thread group's (block or warp).
template <bool WARP>
__device__ __forceinline__ void small_update(const double *Ld, int md, int wd, int n1, int nr,
                                             const int *rel, double *P, int m, double *slab,
                                             int slab_cap, int t, int nt) {
  const int kch = max(1, min(wd, slab_cap / nr));
  for (int k0 = 0; k0 < wd; k0 += kch) {
    const int kc = min(kch, wd - k0);
    if (k0 > 0)
      for (int e = t; e < nr * kc; e += nt) {
        const int kk = e / nr, i = e - kk * nr;
        slab[e] = Ld[(size_t)(k0 + kk) * md + i];
      }
    if (WARP) __syncwarp(); else __syncthreads();
    const int total = n1 * nr;
    for (int idx = t; idx < total; idx += nt) {
      const int a = idx / nr, b = idx - a * nr;
      if (b < a) continue;
      const int ra = rel[a], rbi = rel[b];
      if (ra < 0 || rbi < 0) continue;
      double acc = 0.0;
      for (int kk = 0; kk < kc; ++kk) acc = fma(slab[kk * nr + b], slab[kk * nr + a], acc);
      P[(size_t)ra * m + rbi] -= acc;
    }
    if (WARP) __syncwarp(); else __syncthreads();
  }
}

// Loads the first slab chunk of update-list entry q into registers (element e = t + i nt of
// the chunk in pf[i]), so the loads are in flight while the previous entry is applied.
template <int PF>
__device__ __forceinline__ void prefetch_chunk(const DevSym &S, const int2 *lbub, int q,
                                               int slab_cap, int t, int nt, double (&pf)[PF]) {
  const int d = S.upd[q];
  const int wd = S.super[d + 1] - S.super[d];
  const int md = (int)(S.rowptr[d + 1] - S.rowptr[d]);
  const int lb = lbub[q].x, nr = md - lb;
  const int cnt = nr > 0 ? nr * max(1, min(wd, slab_cap / nr)) : 0;
  const double *Ld = S.L + S.xptr[d] + lb;
#pragma unroll
  for (int i = 0; i < PF; ++i) {
    const int e = t + i * nt;
    pf[i] = 0.0;
    if (e < cnt) {
      const int kk = e / nr;
      pf[i] = Ld[(size_t)kk * md + (e - kk * nr)];
    }
  }
}

// Updates of panel P from every descendant of s's update list, in order, each descendant's
// first chunk loaded while the previous one is applied.
template <bool WARP, int PF>
__device__ __forceinline__ void small_updates(const DevSym &S, const int2 *lbub, int s, int f,
                                              int w, int m, const int *rows, int *rel, double *P,
                                              double *slab, int slab_cap, int t, int nt) {
  const int q0 = S.upd_ptr[s], q1 = S.upd_ptr[s + 1];
  double pf[PF];
  if (q0 < q1) prefetch_chunk<PF>(S, lbub, q0, slab_cap, t, nt, pf);
  for (int q = q0; q < q1; ++q) {
    const int d = S.upd[q];
    const int wd = S.super[d + 1] - S.super[d];
    const int64_t rbd = S.rowptr[d];
    const int md = (int)(S.rowptr[d + 1] - rbd);
    const int *Lsd = S.Ls + rbd;
    const int2 lu = lbub[q];   // d's rows at or below f, and below f + w (host-computed)
    const int lb = lu.x, ub = lu.y;
    const int nr = md - lb;    // nSupRs
    const int n1 = ub - lb;    // ndrow1
    const bool skip = n1 <= 0 || nr > m;
    if (!skip) {
      for (int i = t; i < nr; i += nt) {
        const int key = Lsd[lb + i];
        int pos = lbound(rows, m, key);
        if (pos >= m || rows[pos] != key) { flag_structure_error(S); pos = -1; }
        rel[i] = pos;
      }
      const int cnt = nr * max(1, min(wd, slab_cap / nr));
#pragma unroll
      for (int i = 0; i < PF; ++i)
        if (t + i * nt < cnt) slab[t + i * nt] = pf[i];
    } else if (nr > m && t == 0) {
      flag_structure_error(S);
    }
    if (q + 1 < q1) prefetch_chunk<PF>(S, lbub, q + 1, slab_cap, t, nt, pf);
    if (skip) continue;
    small_update<WARP>(S.L + S.xptr[d] + lb, md, wd, n1, nr, rel, P, m, slab, slab_cap, t, nt);
  }
}

// ---------------------------------------------------------------------------------------
// Whole factorization of one small supernode s by the calling CTA (all NT threads).
__device__ __noinline__ void factor_small_body(const DevSym &S, const int2 *lbub, int s,
                                               double *smem) {
  const int tid = threadIdx.x;
  const int f = S.super[s];
  const int w = S.super[s + 1] - f;
  const int64_t rb = S.rowptr[s];
  const int m = (int)(S.rowptr[s + 1] - rb);
  double *P = smem;                 // m x w, column-major, ld = m
  int *rows = (int *)(P + (size_t)m * w);
  int *rel = rows + m;

  for (int i = tid; i < m; i += NT) rows[i] = S.Ls[rb + i];
  for (int i = tid; i < m * w; i += NT) P[i] = 0.0;
  __syncthreads();

  // assembly: one warp per column of A
  const int lane = tid & 31, warp = tid >> 5;
  for (int j = warp; j < w; j += NT / 32) {
    for (int p = S.Ap[f + j] + lane; p < S.Ap[f + j + 1]; p += 32) {
      int i = S.Ai[p];
      int pos = lbound(rows, m, i);
      if (pos < m && rows[pos] == i) P[(size_t)j * m + pos] = S.Ax[p];
      else flag_structure_error(S);
    }
  }
  __syncthreads();

  // updates from every descendant in the prune set, in order
  small_updates<false, SMALL_SLAB / NT>(S, lbub, s, f, w, m, rows, rel, P,
                                        reinterpret_cast<double *>(rel + m) + w, SMALL_SLAB,
                                        tid, NT);

  // POTRF of the w x w diagonal block by warp 0 alone (warp barriers only; lanes own rows
  // lane and lane + 32), keeping the pivots' reciprocals in rd; then every thread solves
  // its rows below the block against it (row i of L21 = A21(i, :) L11^{-T}), two block
  // barriers in all instead of two per column.
  double *rd = reinterpret_cast<double *>(rel + m);   // w doubles (8-byte aligned slot)
  if (warp == 0) {
    for (int j = 0; j < w; ++j) {
      const double piv = P[(size_t)j * m + j];
      const double inv = rsqrt(piv);
      if (lane == 0) {
        rd[j] = inv;
        if (!(piv > 0.0)) atomicMin(&S.status[0], f + j + 1);
      }
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int r = lane + 32 * h;
        if (r >= j && r < w) P[(size_t)j * m + r] = (r == j) ? piv * inv : P[(size_t)j * m + r] * inv;
      }
      __syncwarp();
      for (int c = j + 1; c < w; ++c) {
        const double lcj = P[(size_t)j * m + c];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int r = lane + 32 * h;
          if (r >= c && r < w) P[(size_t)c * m + r] = fma(-P[(size_t)j * m + r], lcj, P[(size_t)c * m + r]);
        }
      }
      __syncwarp();
    }
  }
  __syncthreads();
  for (int i = w + tid; i < m; i += NT) {
    for (int j = 0; j < w; ++j) {
      double acc = P[(size_t)j * m + i];
      for (int k = 0; k < j; ++k) acc = fma(-P[(size_t)k * m + i], P[(size_t)k * m + j], acc);
      P[(size_t)j * m + i] = acc * rd[j];
    }
  }
  __syncthreads();
  double *dst = S.L + S.xptr[s];
  for (int i = tid; i < m * w; i += NT) dst[i] = P[i];
  if (S.Lf)   // mixed-precision factorization: split mirror for the Schur updates
    store_mirror_panel(S, s, m, w, P, tid, NT);
}

// One CTA per small supernode of a level.
__global__ void __launch_bounds__(NT) k_factor_small(DevSym S, const int2 *lbub, const int *list,
                                                     int count) {
  extern __shared__ double smem[];
  factor_small_body(S, lbub, list[blockIdx.x], smem);
}

// The small supernodes of the bottom of the tree (a set closed under descendants) in ONE
// persistent launch: CTAs take supernodes from a device work queue in level order
// (order[0 .. count)), wait until every descendant in the supernode's update list is
// finished (acquire on its done flag), factor it and publish its own flag (release).  A
// CTA only waits for supernodes taken from the queue before its own, which were taken by
// CTAs already running and waiting on even earlier ones, so the walk always progresses,
// whatever the number of resident CTAs.  qctr[0] is the queue head, qctr[1 + s] the done
// flag of supernode s; both are zeroed before every launch.  A wait gives up after the
// poll budget in status[4] and records the timeout in status[3].

__device__ __forceinline__ int ld_acquire_k(const int *p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];\n" : "=r"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ void st_release_k(int *p, int v) {
  asm volatile("st.release.gpu.global.s32 [%0], %1;\n" ::"l"(p), "r"(v));
}

__global__ void __launch_bounds__(NT) k_factor_small_persist(DevSym S, const int2 *lbub,
                                                              const int *order, int count,
                                                              int *qctr) {
  extern __shared__ double smem[];
  __shared__ int item;
  int *done = qctr + 1;
  for (;;) {
    if (threadIdx.x == 0) item = atomicAdd(qctr, 1);
    __syncthreads();
    const int idx = item;
    if (idx >= count) break;
    const int s = order[idx];
    if (threadIdx.x < 32) {   // warp 0 waits for the update sources, one lane per source
      bool timed_out = false;
      const long long budget = wait_budget(S.status);
      for (int q = S.upd_ptr[s] + threadIdx.x; q < S.upd_ptr[s + 1] && !timed_out; q += 32) {
        const int *flag = done + S.upd[q];
        long long it = 0;
        while (ld_acquire_k(flag) == 0) {
          if (++it > budget) {
            atomicExch(&S.status[3], 1);
            timed_out = true;
            break;
          }
          __nanosleep(64);
        }
      }
    }
    __syncthreads();
    factor_small_body(S, lbub, s, smem);
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      st_release_k(done + s, 1);
    }
  }
}

// ---------------------------------------------------------------------------------------
// Assembly of A into tiled-class panels: one warp per (supernode, column).
__global__ void k_assemble(DevSym S, const int2 *tasks, int count) {
  const int wg = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (wg >= count) return;
  const int s = tasks[wg].x, j = tasks[wg].y;
  const int f = S.super[s];
  const int64_t rb = S.rowptr[s];
  const int m = (int)(S.rowptr[s + 1] - rb);
  const int *rows = S.Ls + rb;
  double *col = S.L + S.xptr[s] + (size_t)(j - f) * m;
  for (int p = S.Ap[j] + lane; p < S.Ap[j + 1]; p += 32) {
    int i = S.Ai[p];
    int pos = lbound(rows, m, i);
    if (pos < m && rows[pos] == i) col[pos] = S.Ax[p];
    else flag_structure_error(S);
  }
}

// ---------------------------------------------------------------------------------------
// 64x64 FP64 tile product on the tensor cores (DMMA, mma.sync m8n8k4 .f64):
//   C[i][j] = sum_k A[i][k] * B[j][k],  A = rows [0,na) of a column-major panel (lda),
//                                       B = rows [0,nb) of a column-major panel (ldb).
// 128 threads = 4 warps in a 2x2 grid, each warp a 32x32 sub-tile of 4x4 MMA tiles.
// Operands stream through shared memory in k-chunks of KC columns with a two-stage
// cp.async pipeline; rows beyond na / nb and columns beyond K are zero-filled.
// Fragment layout of m8n8k4 .f64: A[lane/4][lane%4], B[k = lane%4][n = lane/4],
// C[lane/4][2*(lane%4) + e].
constexpr int MT = 128;               // threads of the tensor-core tile kernels
constexpr int LDS = TB + 4;           // padded row of a staged k-slice: 64-bit fragment loads conflict-free
constexpr int STAGE = 2 * KC * LDS;   // doubles per pipeline stage (A and B slices)
static_assert(MT == 2 * TB, "staging pattern: two threads per tile row");

__device__ __forceinline__ void cp_async8(double *smem, const double *gmem, bool pred) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  const int sz = pred ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ void dmma(double (&c)[2], double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c[0]), "+d"(c[1])
               : "d"(a), "d"(b));
}

struct TileAcc {
  double v[4][4][2];
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) v[i][j][0] = v[i][j][1] = 0.0;
  }
};

// Thread t copies tile row t % 64 at chunk offsets t / 64, t / 64 + 2, ... (one pointer
// step per copy).
__device__ __forceinline__ void load_chunk(const double *__restrict__ Pa, int lda, int na,
                                           const double *__restrict__ Pb, int ldb, int nb,
                                           int K, int k0, double *st) {
  const int i = threadIdx.x & (TB - 1), kq = threadIdx.x >> 6;
  double *As = st + kq * LDS + i, *Bs = st + KC * LDS + kq * LDS + i;
  const double *pa = Pa + (size_t)(k0 + kq) * lda + i, *pb = Pb + (size_t)(k0 + kq) * ldb + i;
  const bool ina = i < na, inb = i < nb;
#pragma unroll
  for (int it = 0; it < KC / 2; ++it) {
    const bool kin = k0 + kq + 2 * it < K;
    cp_async8(As + 2 * it * LDS, kin && ina ? pa : Pa, kin && ina);
    cp_async8(Bs + 2 * it * LDS, kin && inb ? pb : Pb, kin && inb);
    pa += (size_t)2 * lda;
    pb += (size_t)2 * ldb;
  }
  cp_async_commit();
}

__device__ __forceinline__ void dmma_tile_product(const double *__restrict__ Pa, int lda, int na,
                                                  const double *__restrict__ Pb, int ldb, int nb,
                                                  int K, double *stages, TileAcc &acc) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wr = (warp >> 1) * 32, wc = (warp & 1) * 32;
  const int kq = lane & 3, g = lane >> 2;
  const int nchunks = (K + KC - 1) / KC;
  __syncthreads();   // stages free (previous users done)
  load_chunk(Pa, lda, na, Pb, ldb, nb, K, 0, stages);
  for (int c = 0; c < nchunks; ++c) {
    if (c + 1 < nchunks) {
      load_chunk(Pa, lda, na, Pb, ldb, nb, K, (c + 1) * KC, stages + ((c + 1) & 1) * STAGE);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const double *As = stages + (c & 1) * STAGE, *Bs = As + KC * LDS;
#pragma unroll
    for (int k4 = 0; k4 < KC; k4 += 4) {
      double a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[(k4 + kq) * LDS + wr + 8 * i + g];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[(k4 + kq) * LDS + wc + 8 * j + g];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma(acc.v[i][j], a[i], b[j]);
    }
    __syncthreads();
  }
}

// Gathered variant: operand rows are picked through index maps, ia[i] / ib[j] = row of the
// source panel that feeds tile row i / column j, or -1 for a zero row.  Lets one
// accumulator collect the contributions of several descendants in the target's own
// coordinates, with no scatter.
__device__ __forceinline__ void load_chunk_gather(const double *__restrict__ Ld, int ld, int ra,
                                                  int rb, int K, int k0, double *st) {
  const int i = threadIdx.x & (TB - 1), kq = threadIdx.x >> 6;
  double *As = st + kq * LDS + i, *Bs = st + KC * LDS + kq * LDS + i;
  const double *pa = Ld + (size_t)(k0 + kq) * ld + (ra >= 0 ? ra : 0);
  const double *pb = Ld + (size_t)(k0 + kq) * ld + (rb >= 0 ? rb : 0);
#pragma unroll
  for (int it = 0; it < KC / 2; ++it) {
    const bool kin = k0 + kq + 2 * it < K;
    cp_async8(As + 2 * it * LDS, kin && ra >= 0 ? pa : Ld, kin && ra >= 0);
    cp_async8(Bs + 2 * it * LDS, kin && rb >= 0 ? pb : Ld, kin && rb >= 0);
    pa += (size_t)2 * ld;
    pb += (size_t)2 * ld;
  }
  cp_async_commit();
}

__device__ __forceinline__ void dmma_tile_product_gather(const double *__restrict__ Ld, int ld,
                                                         const int *ia, const int *ib, int K,
                                                         double *stages, TileAcc &acc) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wr = (warp >> 1) * 32, wc = (warp & 1) * 32;
  const int kq = lane & 3, g = lane >> 2;
  const int nchunks = (K + KC - 1) / KC;
  __syncthreads();
  // 8x8 MMA tiles whose gathered rows (or columns) are all empty contribute nothing: skip
  // them (warp-uniform masks over this warp's 4 row groups and 4 column groups)
  unsigned rmask = 0, cmask = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    if (__any_sync(0xffffffffu, ia[wr + 8 * i + (lane & 7)] >= 0)) rmask |= 1u << i;
    if (__any_sync(0xffffffffu, ib[wc + 8 * i + (lane & 7)] >= 0)) cmask |= 1u << i;
  }
  const int ra = ia[threadIdx.x & (TB - 1)], rb = ib[threadIdx.x & (TB - 1)];
  load_chunk_gather(Ld, ld, ra, rb, K, 0, stages);
  for (int c = 0; c < nchunks; ++c) {
    if (c + 1 < nchunks) {
      load_chunk_gather(Ld, ld, ra, rb, K, (c + 1) * KC, stages + ((c + 1) & 1) * STAGE);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const double *As = stages + (c & 1) * STAGE, *Bs = As + KC * LDS;
    if (rmask && cmask) {
#pragma unroll
      for (int k4 = 0; k4 < KC; k4 += 4) {
        double a[4], b[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = As[(k4 + kq) * LDS + wr + 8 * i + g];
#pragma unroll
        for (int j = 0; j < 4; ++j) b[j] = Bs[(k4 + kq) * LDS + wc + 8 * j + g];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j)
            if (((rmask >> i) & (cmask >> j)) & 1u) dmma(acc.v[i][j], a[i], b[j]);
      }
    }
    __syncthreads();
  }
}

// Sign flip through the integer pipe (FP64 arithmetic outside the tensor cores is slow).
__device__ __forceinline__ double neg(double x) {
  return __longlong_as_double(__double_as_longlong(x) ^ (long long)0x8000000000000000ULL);
}

// Position of accumulator element (i, j, e) of this thread inside the 64x64 tile.
__device__ __forceinline__ int acc_row(int i) {
  return ((threadIdx.x >> 5) >> 1) * 32 + 8 * i + ((threadIdx.x & 31) >> 2);
}
__device__ __forceinline__ int acc_col(int j, int e) {
  return ((threadIdx.x >> 5) & 1) * 32 + 8 * j + 2 * (threadIdx.x & 3) + e;
}

// Tile-owner update of the tiled class.  task = (s, r0, c0, first pair); the tile covers
// panel rows [r0, r0+64) and columns [c0, c0+64) of supernode s.  Its pair list holds
// exactly the descendants that touch it: pair = (d, a0, b0, na | nb << 16) where rows
// a0..a0+na-1 of d's row list fall in the tile's rows and b0..b0+nb-1 in its columns.
// The accumulator starts as minus the tile, collects every pair's product in the tile's
// own coordinates (rows gathered through index maps), and minus it is stored back:
// tile - sum_d L_d L_d^T without any scalar FP64 operation.
constexpr int UPD_SMEM = 2 * STAGE * 8 + 4 * TB * 4;

__global__ void __launch_bounds__(MT, 4) k_update_tiles(DevSym S, const int4 *tasks,
                                                     const int *task_end, const int4 *pairs,
                                                     int count) {
  extern __shared__ double dyn[];
  double *stages = dyn;
  int *trow = reinterpret_cast<int *>(dyn + 2 * STAGE);
  int *ia = trow + TB, *ib = ia + TB;
  const int4 t = tasks[blockIdx.x];
  const int s = t.x, r0 = t.y, c0 = t.z;
  const int p_begin = t.w, p_end = task_end[blockIdx.x];
  const int tid = threadIdx.x;
  const int f = S.super[s];
  const int w = S.super[s + 1] - f;
  const int64_t rb = S.rowptr[s];
  const int m = (int)(S.rowptr[s + 1] - rb);
  const int nrow = min(TB, m - r0), ncol = min(TB, w - c0);
  const int gc_lo = f + c0;
  double *P = S.L + S.xptr[s];
  for (int i = tid; i < nrow; i += MT) trow[i] = S.Ls[rb + r0 + i];
  TileAcc acc;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int r = acc_row(i);
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int c = acc_col(j, e);
        acc.v[i][j][e] = (r < nrow && c < ncol && r0 + r >= c0 + c)
                             ? neg(P[(size_t)(c0 + c) * m + r0 + r]) : 0.0;
      }
  }
  for (int q = p_begin; q < p_end; ++q) {
    const int4 pr = pairs[q];
    const int d = pr.x, a0 = pr.y, b0 = pr.z;
    const int na = pr.w & 0xffff, nb = pr.w >> 16;
    const int wd = S.super[d + 1] - S.super[d];
    const int64_t rbd = S.rowptr[d];
    const int md = (int)(S.rowptr[d + 1] - rbd);
    const int *Lsd = S.Ls + rbd;
    __syncthreads();   // trow ready; the previous pair is done with ia / ib
    if (tid < TB) { ia[tid] = -1; ib[tid] = -1; }
    __syncthreads();
    if (tid < na) {
      const int key = Lsd[a0 + tid];
      const int pos = lbound(trow, nrow, key);
      if (pos < nrow && trow[pos] == key) ia[pos] = a0 + tid;
      else flag_structure_error(S);
    } else if (tid >= TB && tid < TB + nb) {
      const int cc = Lsd[b0 + tid - TB] - gc_lo;
      if (cc >= 0 && cc < ncol) ib[cc] = b0 + tid - TB;
      else flag_structure_error(S);
    }
    const double *Ld = S.L + S.xptr[d];
    dmma_tile_product_gather(Ld, md, ia, ib, wd, stages, acc);
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int r = acc_row(i);
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int c = acc_col(j, e);
        if (r < nrow && c < ncol && r0 + r >= c0 + c)
          P[(size_t)(c0 + c) * m + r0 + r] = neg(acc.v[i][j][e]);
      }
  }
}

// ---------------------------------------------------------------------------------------
// Dense factorization of a tiled-class panel, blocked by 64 columns (right-looking):
//   step j:  TRSM of the tiles below diagonal block j (k_trsm_step), then, concurrently,
//            the trailing SYRK/GEMM update of the column blocks after j (k_syrk_step in
//            FP64, dense tiles of the split scatter kernel in the mixed modes; it leaves out
//            the next diagonal tile) and, for diagonal block j+1, its update by block j,
//            POTRF and inverse (k_diag_step), so every diagonal block is factored before the
//            next step's TRSM reads it.  In the mixed modes the trailing update is launched
//            in two parts: column block j+1 (read by the next TRSM) on the chain's stream,
//            the grouped updates of the later column blocks on a stream of their own.
//   block 0 is factored by k_diag_step with step 0.

// ---- one 64x64 diagonal block: POTRF and its inverse, blocked by 8 ----------------------
// Every 8x8 block product runs on the tensor cores (DMMA); scalar FP64 work is limited to
// the 8x8 diagonal pieces, done by one warp with shuffles.  D is a [column][row] shared
// array with leading dimension DLD; E (the inverse, lower triangular) holds only its 36
// lower 8x8 blocks, packed: block (bi, bk), bi >= bk, at (bi (bi + 1) / 2 + bk) * 64, each
// block column-major.  128 threads (4 warps).
// DLD = 68: the 8x8 DMMA operand loads (lane 4g + kq reads row g, column kq of a block)
// hit 16 different bank pairs per half warp (68 = 4 mod 16); 65 gave four-way conflicts.
constexpr int DLD = TB + 4;
constexpr int E_ELEMS = 36 * 64;

__device__ __forceinline__ int eix(int r, int c) {
  const int bi = r >> 3, bk = c >> 3;
  return ((bi * (bi + 1) / 2 + bk) << 6) + ((c & 7) << 3) + (r & 7);
}

// c += A_blk * B_blk^T for 8x8 blocks of [column][row] arrays: A_blk = rows ar0..ar0+7,
// columns ak0..ak0+7 of Am; B_blk = rows bn0..bn0+7, columns bk0..bk0+7 of Bm.
__device__ __forceinline__ void mma8_abt(double (&c)[2], const double *Am, int ar0, int ak0,
                                         const double *Bm, int bn0, int bk0, bool negate_a) {
  const int lane = threadIdx.x & 31, g = lane >> 2, kq = lane & 3;
#pragma unroll
  for (int t = 0; t < 2; ++t) {
    const double a = Am[(ak0 + 4 * t + kq) * DLD + ar0 + g];
    const double b = Bm[(bk0 + 4 * t + kq) * DLD + bn0 + g];
    dmma(c, negate_a ? neg(a) : a, b);
  }
}

__device__ __forceinline__ void load8(double (&c)[2], const double *X, int r0, int c0) {
  const int lane = threadIdx.x & 31, g = lane >> 2, kq = lane & 3;
  c[0] = X[(c0 + 2 * kq) * DLD + r0 + g];
  c[1] = X[(c0 + 2 * kq + 1) * DLD + r0 + g];
}
__device__ __forceinline__ void store8(const double (&c)[2], double *X, int r0, int c0, bool lower_only) {
  const int lane = threadIdx.x & 31, g = lane >> 2, kq = lane & 3;
#pragma unroll
  for (int e = 0; e < 2; ++e)
    if (!lower_only || g >= 2 * kq + e) X[(c0 + 2 * kq + e) * DLD + r0 + g] = c[e];
}

// Warp-level Cholesky of the 8x8 diagonal block kb of D and its inverse into E (same
// position).  Every lane factors the whole block in registers (broadcast loads of its 36
// entries), so the chain of pivots is one reciprocal square root, one product and one
// FMA per column with no shuffle on it; lane j < 8 then forms column j of the inverse by
// forward substitution.
__device__ void potrf8_inv8(double *D, double *E, int kb, const DevSym &S, int gcol0, int bw,
                            bool report) {
  const int lane = threadIdx.x & 31, k0 = 8 * kb;
  double a[8][8];
#pragma unroll
  for (int j = 0; j < 8; ++j)
#pragma unroll
    for (int i = j; i < 8; ++i) a[i][j] = D[(k0 + j) * DLD + k0 + i];
  double rinv[8];
  int bad = 8;   // first column with a pivot <= 0 or NaN (reported after the chain)
  double inv = rsqrt(a[0][0]);
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const double piv = a[j][j];
    if (!(piv > 0.0) && j < bad) bad = j;
    rinv[j] = inv;
    a[j][j] = piv * inv;
    // the chain first: the next pivot and its reciprocal square root, issued before the
    // rest of the column's update, which runs under its latency
    if (j + 1 < 8) {
      a[j + 1][j] *= inv;
      a[j + 1][j + 1] = fma(-a[j + 1][j], a[j + 1][j], a[j + 1][j + 1]);
    }
    const double inv_next = (j + 1 < 8) ? rsqrt(a[j + 1][j + 1]) : 0.0;
#pragma unroll
    for (int i = j + 2; i < 8; ++i) a[i][j] *= inv;
#pragma unroll
    for (int k = j + 1; k < 8; ++k)
#pragma unroll
      for (int i = k; i < 8; ++i)
        if (!(k == j + 1 && i == j + 1)) a[i][k] = fma(-a[i][j], a[k][j], a[i][k]);
    inv = inv_next;
  }
  if (report && lane == 0 && bad < 8 && k0 + bad < bw) atomicMin(&S.status[0], gcol0 + k0 + bad + 1);
  // every lane stores the same 36 values (one write per address; no lane-dependent index
  // into a[][], which would move the array to local memory)
#pragma unroll
  for (int j = 0; j < 8; ++j)
#pragma unroll
    for (int i = j; i < 8; ++i) D[(k0 + j) * DLD + k0 + i] = a[i][j];
  // lane j < 8: column j of the inverse, 1/L(i,i) = rinv[i]
  const int j = lane & 7;
  double t[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    double sacc = 0.0;
#pragma unroll
    for (int k = 0; k < i; ++k)
      if (k >= j) sacc = fma(a[i][k], t[k], sacc);
    t[i] = (i < j) ? 0.0 : ((i == j) ? rinv[i] : -sacc * rinv[i]);
  }
  if (lane < 8) {
#pragma unroll
    for (int i = 0; i < 8; ++i) E[eix(k0 + i, k0 + j)] = t[i];
  }
  __syncwarp();
}

// D: bw x bw lower block padded to a multiple of 8 with identity.  Factors it in place
// (right-looking over 8-column blocks) and leaves the inverses of its 8x8 diagonal blocks
// in E.  Look-ahead: in the trailing update of step kb, warp 0 updates diagonal block kb+1
// first and factors it while the other NW - 1 warps update the other blocks, so each step
// costs one panel phase and one trailing phase (two barriers).  NW warps (32 NW threads).
template <int NW>
__device__ void potrf64_blocked(double *D, double *E, int bw, const DevSym &S, int gcol0) {
  const int warp = threadIdx.x >> 5;
  const int nbk = (bw + 7) >> 3;
  if (warp == 0) potrf8_inv8(D, E, 0, S, gcol0, bw, true);
  __syncthreads();
  for (int kb = 0; kb < nbk; ++kb) {
    // panel below: X_ib = B_ib * T_kk^T (warp 0 gets ib = kb + 1)
    for (int ib = kb + 1 + warp; ib < nbk; ib += NW) {
      double c[2] = {0.0, 0.0};
      const int lane = threadIdx.x & 31, g = lane >> 2, kq = lane & 3;
#pragma unroll
      for (int t = 0; t < 2; ++t)   // X_ib = B_ib T_kk^T
        dmma(c, D[(8 * kb + 4 * t + kq) * DLD + 8 * ib + g], E[eix(8 * kb + g, 8 * kb + 4 * t + kq)]);
      __syncwarp();
      store8(c, D, 8 * ib, 8 * kb, false);
    }
    __syncthreads();
    if (kb + 1 >= nbk) break;
    // trailing update D_ib,jb -= X_ib X_jb^T for kb < jb <= ib
    if (warp == 0) {
      const int nb = kb + 1;
      double c[2];
      load8(c, D, 8 * nb, 8 * nb);
      mma8_abt(c, D, 8 * nb, 8 * kb, D, 8 * nb, 8 * kb, true);
      store8(c, D, 8 * nb, 8 * nb, true);
      __syncwarp();
      potrf8_inv8(D, E, nb, S, gcol0, bw, true);
    } else if ((warp & 3) != 0) {
      // blocks (ib, jb), kb < jb <= ib < nbk, except (kb+1, kb+1), in column order; the
      // warps that do not share warp 0's scheduler (warp % 4 != 0: NU of them, rank u) take
      // the blocks u, u + NU, .. and run them interleaved (independent DMMA chains: their
      // latency, not their issue, bounds a short chain); warp 0's chain of pivots keeps its
      // scheduler to itself
      constexpr int NU = NW - NW / 4;
      constexpr int MAXT = (27 + NU - 1) / NU;
      const int u = warp - 1 - (warp >> 2);
      const int nrem = nbk - kb - 1;                       // block rows/columns left
      const int ntot = nrem * (nrem + 1) / 2 - 1;
      double c[MAXT][2];
      int bi[MAXT], bj[MAXT];
#pragma unroll
      for (int t = 0; t < MAXT; ++t) {
        int idx = u + NU * t;
        if (idx >= ntot) idx = -1;  // an unused slot: block (kb+1, kb+1), nothing stored
        idx += 1;                   // skip (kb+1, kb+1), the first block of the order
        int jj = 0;
        while (idx >= nrem - jj) { idx -= nrem - jj; ++jj; }
        bj[t] = 8 * (kb + 1 + jj);
        bi[t] = bj[t] + 8 * idx;
        load8(c[t], D, bi[t], bj[t]);
      }
#pragma unroll
      for (int t = 0; t < MAXT; ++t)
        if (u + NU * t < ntot) mma8_abt(c[t], D, bi[t], 8 * kb, D, bj[t], 8 * kb, true);
#pragma unroll
      for (int t = 0; t < MAXT; ++t)
        if (u + NU * t < ntot) store8(c[t], D, bi[t], bj[t], bi[t] == bj[t]);
    }
    __syncthreads();
  }
}

// Inverse of the factored block: off-diagonal 8x8 blocks T_ik = -T_ii sum_{j=k}^{i-1}
// L_ij T_jk, one column block per warp (E holds T_kk on entry; W: 64 doubles per warp).
template <int NW>
__device__ void trtri64_blocked(const double *D, double *E, double *W, int bw) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, kq = lane & 3;
  const int nbk = (bw + 7) >> 3;
  double *Ww = W + warp * 64;
  for (int k = warp; k < nbk; k += NW) {
    for (int i = k + 1; i < nbk; ++i) {
      double sacc[2] = {0.0, 0.0};
      for (int j = k; j < i; ++j)   // sacc += L_ij T_jk
#pragma unroll
        for (int t = 0; t < 2; ++t)
          dmma(sacc, D[(8 * j + 4 * t + kq) * DLD + 8 * i + g], E[eix(8 * j + 4 * t + kq, 8 * k + g)]);
      // S (C layout) -> W[col * 8 + row], read back as the B operand of T_ii * S
      Ww[(2 * kq) * 8 + g] = sacc[0];
      Ww[(2 * kq + 1) * 8 + g] = sacc[1];
      __syncwarp();
      double c[2] = {0.0, 0.0};
#pragma unroll
      for (int t = 0; t < 2; ++t) {
        const double a = neg(E[eix(8 * i + g, 8 * i + 4 * t + kq)]);
        const double b = Ww[g * 8 + 4 * t + kq];
        dmma(c, a, b);
      }
#pragma unroll
      for (int e = 0; e < 2; ++e) E[eix(8 * i + g, 8 * k + 2 * kq + e)] = c[e];
      __syncwarp();
    }
  }
  __syncthreads();
}

// Factor diagonal block c0/64 of supernode s in place (lower triangle only) and store its
// inverse (T(r, c) at dinv[c * 64 + r]) for the TRSM of the rows below it and for the
// chained triangular solves.  upd (optional): the diagonal tile's value, negated, as left in
// a tile accumulator by syrk_tile_acc (its update by the previous column block), so the
// updated block never leaves the chip before its factorization; when the block is narrower
// than 64 the tile's remaining rows are panel rows below it and go to L.
// NW warps (upd needs NW = 4: the tile accumulator's layout), diag_smem(NW) bytes of
// dynamic shared memory: E, W (NW x 64), then D.
constexpr int diag_smem(int nw) { return (E_ELEMS + nw * 64 + TB * DLD) * 8; }
constexpr int diag_prev_smem(int nw) { return diag_smem(nw) + TB * DLD * 8; }   // + X
constexpr int DIAG_SMEM = diag_smem(4);
constexpr int DIAG_NW = 8;   // warps of the per-step diagonal-block kernel

// PREV: the block still misses its update by column block c0/64 - 1 (the rows just above it
// solved by the previous TRSM launch): it is applied here, on the tile in shared memory,
// before the factorization (and to the panel rows below a narrower last block, in L).
template <int NW, bool PREV = false>
__device__ void factor_diag_block(const DevSym &S, int s, int c0, double *smem,
                                  const TileAcc *upd) {
  constexpr int NTH = 32 * NW;
  double *E = smem, *W = smem + E_ELEMS, *D = W + NW * 64;
  const int tid = threadIdx.x;
  const int f = S.super[s];
  const int w = S.super[s + 1] - f;
  const int m = (int)(S.rowptr[s + 1] - S.rowptr[s]);
  double *P = S.L + S.xptr[s];
  const int bw = min(TB, w - c0);
  __syncthreads();
  // the tile and, with PREV, X = rows c0.. of column block c0/64 - 1 (64 wide, [column][row]
  // after D): eight loads of each in flight per thread before the shared stores
  double *Xs = D + TB * DLD;
  const int nr = min(TB, m - c0);
  for (int e0 = tid; e0 < TB * TB; e0 += 8 * NTH) {
    double v[8], xv[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int e = e0 + q * NTH, c = e >> 6, r = e & (TB - 1);
      if (c < bw && r < bw) v[q] = (!upd && r >= c) ? P[(size_t)(c0 + c) * m + c0 + r] : 0.0;
      else v[q] = (r == c) ? 1.0 : 0.0;
      if (PREV) xv[q] = r < nr ? P[(size_t)(c0 - TB + c) * m + c0 + r] : 0.0;
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int e = e0 + q * NTH;
      D[(e >> 6) * DLD + (e & (TB - 1))] = v[q];
      if (PREV) Xs[(e >> 6) * DLD + (e & (TB - 1))] = xv[q];
    }
  }
  for (int e = tid; e < E_ELEMS; e += blockDim.x) E[e] = 0.0;
  if (PREV) {
    __syncthreads();
    // tile -= X X^T over the lower 8x8 blocks (DMMA), block columns of the diagonal block
    // only.  Blocks in column order (column bj holds 8 - bj of them); warp w takes blocks
    // w, w + NW, .. and runs their DMMA chains interleaved (independent accumulators).
    constexpr int MAXB = (36 + NW - 1) / NW;
    const int warp = tid >> 5, lane = tid & 31, g = lane >> 2, qq = lane & 3;
    const int nbj = (bw + 7) / 8, nblk = 8 * nbj - nbj * (nbj - 1) / 2;
    double acc[MAXB][2];
    int ar[MAXB], br[MAXB];
#pragma unroll
    for (int q = 0; q < MAXB; ++q) {
      acc[q][0] = acc[q][1] = 0.0;
      int blk = warp + NW * q, bj = 0;
      if (blk >= nblk) blk = 0;   // unused slot: a valid block, its result dropped below
      while (blk >= 8 - bj) { blk -= 8 - bj; ++bj; }
      ar[q] = 8 * (bj + blk);
      br[q] = 8 * bj;
    }
#pragma unroll
    for (int k0 = 0; k0 < TB; k0 += 8)
#pragma unroll
      for (int q = 0; q < MAXB; ++q)
        if (warp + NW * q < nblk) mma8_abt(acc[q], Xs, ar[q], k0, Xs, br[q], k0, false);
#pragma unroll
    for (int q = 0; q < MAXB; ++q) {
      if (warp + NW * q >= nblk) continue;
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int r = ar[q] + g, c = br[q] + 2 * qq + e;
        if (c >= bw) continue;
        if (r < bw) {
          if (r >= c) D[c * DLD + r] -= acc[q][e];
        } else if (c0 + r < m) {   // a partial last block: panel rows below it, in L
          P[(size_t)(c0 + c) * m + c0 + r] -= acc[q][e];
        }
      }
    }
  }
  if (upd) {
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int r = acc_row(i);
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int c = acc_col(j, e);
          if (r < bw && c < bw && r >= c) D[c * DLD + r] = neg(upd->v[i][j][e]);
          // a partial last block: the tile's rows below the block are panel rows
          else if (r >= bw && c < bw && c0 + r < m) P[(size_t)(c0 + c) * m + c0 + r] = neg(upd->v[i][j][e]);
        }
    }
  }
  __syncthreads();
  potrf64_blocked<NW>(D, E, bw, S, f + c0);
  for (int e = tid; e < TB * TB; e += blockDim.x) {
    const int c = e >> 6, r = e & (TB - 1);
    if (c < bw && r < bw && r >= c) P[(size_t)(c0 + c) * m + c0 + r] = D[c * DLD + r];
  }
  {   // the inverse serves the TRSM of the rows below and the chained triangular solves
    trtri64_blocked<NW>(D, E, W, bw);
    double *T = S.dinv + ((size_t)S.dinv_off[s] + c0 / TB) * (TB * TB);
    for (int e = tid; e < TB * TB; e += blockDim.x) {
      const int c = e >> 6, r = e & (TB - 1);
      T[e] = (c < bw && r < bw && r >= c) ? E[eix(r, c)] : 0.0;
    }
  }
}

// Trailing SYRK/GEMM update of one 64x64 tile of a tiled-class panel by column blocks
// kblk .. kblk + nblk - 1: tile(r0, c0) -= L[r0:, blocks] L[c0:, blocks]^T.  The
// accumulator is seeded with minus the tile, so the tensor cores produce -(C - A B^T).
__device__ void syrk_tile_acc(const DevSym &S, int s, int r0, int c0, int kblk, double *stages,
                              TileAcc &acc, int nblk = 1) {
  const int f = S.super[s];
  const int w = S.super[s + 1] - f;
  const int m = (int)(S.rowptr[s + 1] - S.rowptr[s]);
  const double *P = S.L + S.xptr[s];
  const int k0 = kblk * TB;
  const int bk = min(nblk * TB, w - k0);
  const int nrow = min(TB, m - r0), ncol = min(TB, w - c0);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int r = acc_row(i);
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int c = acc_col(j, e);
        acc.v[i][j][e] = (r < nrow && c < ncol && r0 + r >= c0 + c)
                             ? neg(P[(size_t)(c0 + c) * m + r0 + r]) : 0.0;
      }
  }
  dmma_tile_product(P + (size_t)k0 * m + r0, m, nrow, P + (size_t)k0 * m + c0, m, ncol, bk,
                    stages, acc);
}

// ... stored back negated.
__device__ void syrk_tile(const DevSym &S, int s, int r0, int c0, int kblk, double *stages,
                          int nblk = 1) {
  const int f = S.super[s];
  const int w = S.super[s + 1] - f;
  const int m = (int)(S.rowptr[s + 1] - S.rowptr[s]);
  double *P = S.L + S.xptr[s];
  const int nrow = min(TB, m - r0), ncol = min(TB, w - c0);
  TileAcc acc;
  syrk_tile_acc(S, s, r0, c0, kblk, stages, acc, nblk);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int r = acc_row(i);
    if (r >= nrow) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int c = acc_col(j, e);
        if (c < ncol && r0 + r >= c0 + c) P[(size_t)(c0 + c) * m + r0 + r] = neg(acc.v[i][j][e]);
      }
  }
}

// Dataflow plan: one task brings diagonal block `step` up to date (its update by column
// block step-1, which the trailing-update tasks of that step leave out) and factors it.
__device__ void diag_task(const DevSym &S, int s, int step, double *smem) {
  const int c0 = step * TB;
  if (step > 0) {
    TileAcc acc;
    syrk_tile_acc(S, s, c0, c0, step - 1, smem, acc);
    factor_diag_block<4>(S, s, c0, smem, &acc);
  } else {
    factor_diag_block<4>(S, s, c0, smem, nullptr);
  }
}

// Per-step launches: one CTA per supernode of the list factors diagonal block `step`, after
// applying its update by column block step-1 (the last one it misses).
__global__ void __launch_bounds__(DIAG_NW * 32) k_diag_step(DevSym S, const int *list, int count,
                                                           int step) {
  extern __shared__ double dyn[];
  if (step > 0)
    factor_diag_block<DIAG_NW, true>(S, list[blockIdx.x], step * TB, dyn, nullptr);
  else
    factor_diag_block<DIAG_NW, false>(S, list[blockIdx.x], 0, dyn, nullptr);
}

// task = (s, r0): B = L[r0:r0+64, blk] := B * L_blk^{-T} = B * T^T with T = L_blk^{-1},
// stored by the CTA that factored the block (T(r, c) at T[c * 64 + r]), as one DMMA tile
// product.
__device__ void trsm_task(const DevSym &S, int s, int r0, int step, double *dyn) {
  const int f = S.super[s];
  const int w = S.super[s + 1] - f;
  const int m = (int)(S.rowptr[s + 1] - S.rowptr[s]);
  double *P = S.L + S.xptr[s];
  const int c0 = step * TB;
  const int bw = min(TB, w - c0);
  const int nr = min(TB, m - r0);
  const double *T = S.dinv + ((size_t)S.dinv_off[s] + step) * (TB * TB);
  TileAcc acc;
  acc.zero();
  // X[r][c] = sum_k B[r][k] T(c, k); operand element (row c, column k) = T[k * 64 + c]
  dmma_tile_product(P + (size_t)c0 * m + r0, m, nr, T, TB, bw, bw, dyn, acc);
  // through shared memory (the staging area), so the stores of L (column-major) and of
  // the mirror (K-major rows) are both contiguous per warp
  constexpr int XLD = TB + 1;
  static_assert(TB * XLD <= 2 * STAGE, "result tile fits the staging area");
  __syncthreads();   // every warp is done with the stages
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e) dyn[acc_col(j, e) * XLD + acc_row(i)] = acc.v[i][j][e];
  __syncthreads();
  for (int e = threadIdx.x; e < TB * TB; e += blockDim.x) {
    const int c = e >> 6, r = e & (TB - 1);
    if (r < nr && c < bw) P[(size_t)(c0 + c) * m + r0 + r] = dyn[c * XLD + r];
  }
  if (S.Lf) store_mirror_block(S, s, m, w, r0, c0, nr, bw, dyn, XLD, threadIdx.x, blockDim.x);
}

// TRSM tiles of step `step`, one product each; the next diagonal block's update by this
// column block is applied by the diagonal-block kernel that factors it (on the tile in its
// shared memory), so every TRSM task of the chain's launch takes one product.
__global__ void __launch_bounds__(MT, 4) k_trsm_step(DevSym S, const int2 *tasks, int count,
                                                  int step) {
  extern __shared__ double dyn[];
  trsm_task(S, tasks[blockIdx.x].x, tasks[blockIdx.x].y, step, dyn);
}

// Trailing update of a step: task = (s, r0, c0, product index) with c0 >= (step+1)*64,
// r0 >= c0; the product names the column blocks applied (the step's block, or a group of
// blocks ending with it).  The diagonal tile of the next block is updated by the TRSM
// launch of the step and factored by k_diag_step, which runs concurrently.
constexpr int SYRK_SMEM = 2 * STAGE * 8;

__global__ void __launch_bounds__(MT) k_syrk_step(DevSym S, const int4 *tasks, const TcPair *prod,
                                                  int count) {
  extern __shared__ double dyn[];
  const int4 t = tasks[blockIdx.x];
  const int kk = prod[t.w].kk;   // the task's column blocks: first = k0 / 64, then kcnt columns
  syrk_tile(S, t.x, t.y, t.z, (kk & 0xffff) / TB, dyn, ((kk >> 16) + TB - 1) / TB);
}

// ---------------------------------------------------------------------------------------
// The same dense factorization as ONE persistent dataflow launch per wave: every diagonal
// block, TRSM tile and trailing-update tile of the wave's tiled-class panels is a task,
// task = (s, r0, c0, kind | step << 2 | first << 17) with kind 0: diagonal block `step`
// (its update by block step-1, POTRF, inverse; r0 = c0 = step * 64), 1: TRSM of rows r0..
// of block `step`, 2: update of tile (r0, c0) by the column blocks first .. step in one
// product (updates far from the diagonal are grouped: fewer, longer products).  Tile
// (I, J) of a panel (64-row block I, 64-column block J; I >= J) has a version counter
// ver[toff[s] + J * mb + I] (mb = row blocks of s): the number of column blocks applied
// to it, plus one once it is final (factored or solved).  A task waits (acquire, bounded
// spin) for the versions it reads, runs, and publishes its tile's new version (release):
//   diagonal block J:  ver(J, J) >= J - 1 and ver(J, J-1) >= J;       sets ver(J, J) = J + 1
//   TRSM (r0, J):      ver(J, J) >= J + 1, ver(I, J) >= J for the row blocks I != J it
//                      covers;                                         sets ver(I, J) = J + 1
//   update (I, C; F..J): ver(I, C) >= F, ver(I, J) >= J + 1, ver(C, J) >= J + 1 (a final
//                      tile (I, J) implies final tiles (I, F..J-1));   sets ver(I, C) = J + 1
// (the TRSM of a partial last block spans two row blocks and feeds nothing in the panel;
// a diagonal tile C gets update tasks for blocks 0 .. C-2, its diagonal task applies C-1).
// The list is in a topological order (decreasing length of the longest chain of tasks
// that depends on each task), so a CTA only waits for tasks taken before its own and the
// walk progresses whatever the number of resident CTAs.  A wait gives up after
// poll budget in status[4] (or when another one has) and records the timeout in status[3].
constexpr int DENSE_SMEM = DIAG_SMEM > SYRK_SMEM ? DIAG_SMEM : SYRK_SMEM;
static_assert(DENSE_SMEM >= 2 * STAGE * 8, "the TRSM stages fit");

__device__ __forceinline__ bool dense_wait(const int *p, int need, int *status) {
  long long it = 0;
  const long long budget = wait_budget(status);
  while (ld_acquire_k(p) < need) {
    if ((++it & 31) == 0 && *(volatile int *)&status[3]) return false;
    if (it > budget) {
      atomicExch(&status[3], 1);
      return false;
    }
    __nanosleep(32);
  }
  return true;
}

__global__ void __launch_bounds__(MT, 4) k_dense_persist(DevSym S, const int4 *tasks, int count,
                                                         const int *toff, int *ver, int *qhead) {
  extern __shared__ double dyn[];
  __shared__ int item, ok;
  for (;;) {
    if (threadIdx.x == 0) item = atomicAdd(qhead, 1);
    __syncthreads();
    const int idx = item;
    if (idx >= count) break;
    const int4 t = tasks[idx];
    const int s = t.x, kind = t.w & 3, step = (t.w >> 2) & 0x7fff, first = t.w >> 17;
    const int w = S.super[s + 1] - S.super[s];
    const int m = (int)(S.rowptr[s + 1] - S.rowptr[s]);
    const int mb = (m + TB - 1) / TB;
    int *V = ver + toff[s];
    if (threadIdx.x == 0) {
      bool good = true;
      if (kind == 0) {
        if (step > 0)
          good = dense_wait(V + step * mb + step, step - 1, S.status) &&
                 dense_wait(V + (step - 1) * mb + step, step, S.status);
      } else if (kind == 1) {
        const int nr = min(TB, m - t.y);
        good = dense_wait(V + step * mb + step, step + 1, S.status);
        for (int I = t.y / TB; I <= (t.y + nr - 1) / TB && good; ++I)
          if (I != step) good = dense_wait(V + step * mb + I, step, S.status);
      } else {
        const int I = t.y / TB, C = t.z / TB;
        good = dense_wait(V + C * mb + I, first, S.status) &&
               dense_wait(V + step * mb + I, step + 1, S.status) &&
               dense_wait(V + step * mb + C, step + 1, S.status);
      }
      ok = good;
    }
    __syncthreads();
    if (!ok) break;
    if (kind == 0) diag_task(S, s, step, dyn);
    else if (kind == 1) trsm_task(S, s, t.y, step, dyn);
    else syrk_tile(S, s, t.y, t.z, first, dyn, step - first + 1);
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      if (kind == 0) st_release_k(V + step * mb + step, step + 1);
      else if (kind == 2) st_release_k(V + (t.z / TB) * mb + t.y / TB, step + 1);
      else if (t.y % TB == 0 && w - step * TB >= TB) st_release_k(V + step * mb + t.y / TB, step + 1);
    }
  }
}

__global__ void k_init_status(int *status) {
  status[0] = INT_MAX;
  status[1] = 0;
  status[3] = 0;
}


// ---------------------------------------------------------------------------------------
// Tiny supernodes (panel at most TINY_ELEMS doubles, at most TINY_M rows): one WARP per
// supernode, TW warps per CTA, each with its own shared-memory slice.  The bottom of the
// tree (a set closed under descendants) is walked in ONE persistent launch: warps take
// supernodes from their own device queue in level order, wait for the descendants in the
// update list, factor with warp-synchronous code (no block barriers) and publish their done
// flag, as the CTA walk below does at CTA granularity.
constexpr int TW = 4;
constexpr int TINY_SLICE = (TINY_ELEMS * 8 + TINY_SLAB * 8 + 2 * TINY_M * 4 + 15) / 16 * 16;   // bytes per warp
constexpr int TINY_SMEM = TW * TINY_SLICE;

__device__ void factor_tiny_body(const DevSym &S, const int2 *lbub, int s, double *P, int *rows,
                                 int *rel, double *slab) {
  const int lane = threadIdx.x & 31;
  const int f = S.super[s];
  const int w = S.super[s + 1] - f;
  const int64_t rb = S.rowptr[s];
  const int m = (int)(S.rowptr[s + 1] - rb);
  for (int i = lane; i < m; i += 32) rows[i] = S.Ls[rb + i];
  for (int i = lane; i < m * w; i += 32) P[i] = 0.0;
  __syncwarp();
  // assembly of A's columns
  for (int j = 0; j < w; ++j)
    for (int p = S.Ap[f + j] + lane; p < S.Ap[f + j + 1]; p += 32) {
      const int i = S.Ai[p];
      const int pos = lbound(rows, m, i);
      if (pos < m && rows[pos] == i) P[(size_t)j * m + pos] = S.Ax[p];
      else flag_structure_error(S);
    }
  __syncwarp();
  // updates from the descendants of the update list, in order
  small_updates<true, TINY_SLAB / 32>(S, lbub, s, f, w, m, rows, rel, P, slab, TINY_SLAB, lane, 32);
  // right-looking POTRF + TRSM of the m x w panel, lanes along the rows
  for (int j = 0; j < w; ++j) {
    const double piv = P[(size_t)j * m + j];
    const double inv = rsqrt(piv), dsq = piv * inv;
    if (lane == 0 && !(piv > 0.0)) atomicMin(&S.status[0], f + j + 1);
    __syncwarp();
    for (int i = j + lane; i < m; i += 32) P[(size_t)j * m + i] = (i == j) ? dsq : P[(size_t)j * m + i] * inv;
    __syncwarp();
    for (int c = j + 1; c < w; ++c) {
      const double lcj = P[(size_t)j * m + c];
      for (int i = c + lane; i < m; i += 32)
        P[(size_t)c * m + i] = fma(-P[(size_t)j * m + i], lcj, P[(size_t)c * m + i]);
    }
    __syncwarp();
  }
  double *dst = S.L + S.xptr[s];
  for (int i = lane; i < m * w; i += 32) dst[i] = P[i];
  if (S.Lf) store_mirror_panel_warp(S, s, m, w, P);
}

// qctr[1 + s]: done flags (shared with the CTA walk); qhead: this walk's queue head.
__global__ void __launch_bounds__(TW * 32) k_factor_tiny_persist(DevSym S, const int2 *lbub,
                                                                 const int *order,
                                                                 int count, int *qctr,
                                                                 int *qhead) {
  extern __shared__ double smem_t[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  unsigned char *slice = reinterpret_cast<unsigned char *>(smem_t) + (size_t)warp * TINY_SLICE;
  double *P = reinterpret_cast<double *>(slice);
  double *slab = reinterpret_cast<double *>(slice + TINY_ELEMS * 8);
  int *rows = reinterpret_cast<int *>(slice + (TINY_ELEMS + TINY_SLAB) * 8);
  int *rel = rows + TINY_M;
  int *done = qctr + 1;
  for (;;) {
    int idx = 0;
    if (lane == 0) idx = atomicAdd(qhead, 1);
    idx = __shfl_sync(0xffffffffu, idx, 0);
    if (idx >= count) break;
    const int s = order[idx];
    bool timed_out = false;
    const long long budget = wait_budget(S.status);
    for (int q = S.upd_ptr[s] + lane; q < S.upd_ptr[s + 1] && !timed_out; q += 32) {
      const int *flag = done + S.upd[q];
      long long it = 0;
      while (ld_acquire_k(flag) == 0) {
        if (++it > budget) {
          atomicExch(&S.status[3], 1);
          timed_out = true;
          break;
        }
        __nanosleep(64);
      }
    }
    __syncwarp();
    factor_tiny_body(S, lbub, s, P, rows, rel, slab);
    __syncwarp();
    if (lane == 0) {
      __threadfence();
      st_release_k(done + s, 1);
    }
  }
}

}  // namespace

bool kernels_configure(std::string &err) {
  cudaError_t e = cudaFuncSetAttribute(k_factor_small, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       200 * 1024);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_factor_small_persist, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             200 * 1024);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_factor_tiny_persist, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             TINY_SMEM);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_update_tiles, cudaFuncAttributeMaxDynamicSharedMemorySize, UPD_SMEM);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_trsm_step, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * STAGE * 8);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_diag_step, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             diag_prev_smem(DIAG_NW));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_syrk_step, cudaFuncAttributeMaxDynamicSharedMemorySize, SYRK_SMEM);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_dense_persist, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             DENSE_SMEM);
  if (e != cudaSuccess) {
    err = std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e);
    return false;
  }
  return true;
}

void launch_factor_small(const DevSym &S, const int2 *lbub, const int *list, int count, int smem,
                         cudaStream_t st) {
  if (count > 0) k_factor_small<<<count, NT, smem, st>>>(S, lbub, list, count);
}
int persist_ctas(int smem, int count) {
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_factor_small_persist, NT, smem) !=
          cudaSuccess || per < 1)
    per = 1;
  return std::max(1, std::min(count, sms * per));
}
int tiny_ctas(int count) {
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_factor_tiny_persist, TW * 32,
                                                    TINY_SMEM) != cudaSuccess || per < 1)
    per = 1;
  return std::max(1, std::min((count + TW - 1) / TW, sms * per));
}
void launch_factor_tiny_persist(const DevSym &S, const int2 *lbub, const int *order, int count,
                                int ctas, int *qctr, int *qhead, cudaStream_t st) {
  if (count > 0)
    k_factor_tiny_persist<<<ctas, TW * 32, TINY_SMEM, st>>>(S, lbub, order, count, qctr, qhead);
}
void launch_factor_small_persist(const DevSym &S, const int2 *lbub, const int *order, int count,
                                 int smem, int ctas, int *qctr, cudaStream_t st) {
  if (count > 0) k_factor_small_persist<<<ctas, NT, smem, st>>>(S, lbub, order, count, qctr);
}
void launch_assemble(const DevSym &S, const int2 *tasks, int count, cudaStream_t st) {
  if (count > 0) k_assemble<<<(count * 32 + NT - 1) / NT, NT, 0, st>>>(S, tasks, count);
}
void launch_update_tiles(const DevSym &S, const int4 *tasks, const int *task_end,
                         const int4 *pairs, int count, cudaStream_t st) {
  if (count > 0) k_update_tiles<<<count, MT, UPD_SMEM, st>>>(S, tasks, task_end, pairs, count);
}
void launch_diag_step(const DevSym &S, const int *list, int count, int step, cudaStream_t st) {
  if (count > 0)
    k_diag_step<<<count, DIAG_NW * 32, diag_prev_smem(DIAG_NW), st>>>(S, list, count, step);
}
void launch_trsm_step(const DevSym &S, const int2 *tasks, int count, int step, cudaStream_t st) {
  if (count > 0) k_trsm_step<<<count, MT, 2 * STAGE * 8, st>>>(S, tasks, count, step);
}
void launch_syrk_step(const DevSym &S, const int4 *tasks, const TcPair *prod, int count,
                      cudaStream_t st) {
  if (count > 0) k_syrk_step<<<count, MT, SYRK_SMEM, st>>>(S, tasks, prod, count);
}
int dense_ctas(int count) {
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_dense_persist, MT, DENSE_SMEM) !=
          cudaSuccess || per < 1)
    per = 1;
  return std::max(1, std::min(count, sms * per));
}
void launch_dense_persist(const DevSym &S, const int4 *tasks, int count, int ctas, const int *toff,
                          int *ver, int *qhead, cudaStream_t st) {
  if (count > 0)
    k_dense_persist<<<ctas, MT, DENSE_SMEM, st>>>(S, tasks, count, toff, ver, qhead);
}
void launch_init_status(int *status, cudaStream_t st) { k_init_status<<<1, 1, 0, st>>>(status); }

}  // namespace swc
