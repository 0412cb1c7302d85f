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
//   k_potrf_first,   blocked right-looking dense factorization of a wide supernode by
//   k_trsm_step,     64-column blocks: POTRF of diagonal block 0, then per block the TRSM
//   k_syrk_step      of the tiles below the diagonal block and the trailing SYRK/GEMM
//                    update, whose diagonal-tile CTA also factors the next diagonal block.
//
// All arithmetic is FP64; tiles are 64x64 with 256 threads, each thread holding a 4x4
// register micro-tile.
#include <cuda_runtime.h>

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

__device__ __forceinline__ void flag_structure_error(const DevSym &S) {
  atomicExch(&S.status[1], 1);
}

// ---------------------------------------------------------------------------------------
// One CTA per small supernode.
__global__ void __launch_bounds__(NT) k_factor_small(DevSym S, const int *list, int count) {
  extern __shared__ double smem[];
  const int s = list[blockIdx.x];
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
  for (int q = S.upd_ptr[s]; q < S.upd_ptr[s + 1]; ++q) {
    const int d = S.upd[q];
    const int fd = S.super[d];
    const int wd = S.super[d + 1] - fd;
    const int64_t rbd = S.rowptr[d];
    const int md = (int)(S.rowptr[d + 1] - rbd);
    const int *Lsd = S.Ls + rbd;
    const int lb = wd + lbound(Lsd + wd, md - wd, f);
    const int ub = wd + lbound(Lsd + wd, md - wd, f + w);
    const int nr = md - lb;   // nSupRs
    const int n1 = ub - lb;   // ndrow1
    if (n1 <= 0 || nr > m) {
      if (nr > m) flag_structure_error(S);
      continue;
    }
    for (int i = tid; i < nr; i += NT) {
      int key = Lsd[lb + i];
      int pos = lbound(rows, m, key);
      if (pos >= m || rows[pos] != key) { flag_structure_error(S); pos = -1; }
      rel[i] = pos;
    }
    __syncthreads();
    const double *Ld = S.L + S.xptr[d];
    const int total = n1 * nr;
    for (int idx = tid; idx < total; idx += NT) {
      const int a = idx / nr, b = idx - a * nr;
      if (b < a) continue;
      const int ra = rel[a], rbi = rel[b];
      if (ra < 0 || rbi < 0) continue;
      double acc = 0.0;
      const double *pa = Ld + lb + a, *pb = Ld + lb + b;
      for (int k = 0; k < wd; ++k) acc += pb[(size_t)k * md] * pa[(size_t)k * md];
      P[(size_t)ra * m + rbi] -= acc;
    }
    __syncthreads();
  }

  // POTRF + TRSM on the tall panel: unblocked right-looking Cholesky of m x w
  for (int j = 0; j < w; ++j) {
    const double djj = P[(size_t)j * m + j];
    if (!(djj > 0.0) && tid == 0) atomicMin(&S.status[0], f + j + 1);
    const double dsq = sqrt(djj);
    __syncthreads();
    for (int i = j + tid; i < m; i += NT)
      P[(size_t)j * m + i] = (i == j) ? dsq : P[(size_t)j * m + i] / dsq;
    __syncthreads();
    const int ncol = w - j - 1;
    for (int idx = tid; idx < ncol * m; idx += NT) {
      const int cc = j + 1 + idx / m;
      const int i = idx - (cc - j - 1) * m;
      if (i >= cc) P[(size_t)cc * m + i] -= P[(size_t)j * m + i] * P[(size_t)j * m + cc];
    }
    __syncthreads();
  }
  double *dst = S.L + S.xptr[s];
  for (int i = tid; i < m * w; i += NT) dst[i] = P[i];
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
// Register-tiled 64x64 FP64 product of two row blocks over K columns:
//   acc[i][j] += sum_k A[ty+16i, k] * B[tx+16j, k]
// A rows come from a column-major panel (ld), starting at row a0, na valid rows; same for B.
__device__ __forceinline__ void tile_product(const double *__restrict__ Pa, int lda, int na,
                                             const double *__restrict__ Pb, int ldb, int nb,
                                             int K, double (*As)[TB], double (*Bs)[TB],
                                             double acc[4][4]) {
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;
  for (int k0 = 0; k0 < K; k0 += KC) {
    __syncthreads();
    for (int e = tid; e < KC * TB; e += NT) {
      const int k = e / TB, i = e - k * TB;
      const bool kin = (k0 + k) < K;
      As[k][i] = (kin && i < na) ? Pa[(size_t)(k0 + k) * lda + i] : 0.0;
      Bs[k][i] = (kin && i < nb) ? Pb[(size_t)(k0 + k) * ldb + i] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < KC; ++k) {
      double a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[k][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[k][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
  }
}

// Tile-owner update of the tiled class.  task = (s, r0, c0): the tile covers panel rows
// [r0, r0+64) and columns [c0, c0+64) of supernode s.
constexpr int UPD_SMEM = (2 * KC * TB + TB * (TB + 1)) * 8 + 3 * TB * 4;

__global__ void __launch_bounds__(NT) k_update_tiles(DevSym S, const int4 *tasks, int count) {
  extern __shared__ double dyn[];
  double(*As)[TB] = reinterpret_cast<double(*)[TB]>(dyn);
  double(*Bs)[TB] = reinterpret_cast<double(*)[TB]>(dyn + KC * TB);
  double(*Acc)[TB + 1] = reinterpret_cast<double(*)[TB + 1]>(dyn + 2 * KC * TB);  // [col][row]
  int *trow = reinterpret_cast<int *>(dyn + 2 * KC * TB + TB * (TB + 1));
  int *relr = trow + TB, *relc = relr + TB;
  const int4 t = tasks[blockIdx.x];
  const int s = t.x, r0 = t.y, c0 = t.z;
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;
  const int f = S.super[s];
  const int w = S.super[s + 1] - f;
  const int64_t rb = S.rowptr[s];
  const int m = (int)(S.rowptr[s + 1] - rb);
  const int nrow = min(TB, m - r0), ncol = min(TB, w - c0);
  for (int i = tid; i < nrow; i += NT) trow[i] = S.Ls[rb + r0 + i];
  for (int e = tid; e < TB * (TB + 1); e += NT) (&Acc[0][0])[e] = 0.0;
  __syncthreads();
  const int gr_lo = trow[0], gr_hi = trow[nrow - 1];
  const int gc_lo = f + c0, gc_hi = f + c0 + ncol - 1;

  for (int q = S.upd_ptr[s]; q < S.upd_ptr[s + 1]; ++q) {
    const int d = S.upd[q];
    const int wd = S.super[d + 1] - S.super[d];
    const int64_t rbd = S.rowptr[d];
    const int md = (int)(S.rowptr[d + 1] - rbd);
    const int *Lsd = S.Ls + rbd;
    const int a0 = lbound(Lsd, md, gr_lo), a1 = lbound(Lsd, md, gr_hi + 1);
    const int b0 = lbound(Lsd, md, gc_lo), b1 = lbound(Lsd, md, gc_hi + 1);
    if (a0 >= a1 || b0 >= b1) continue;   // uniform across the CTA
    int na = a1 - a0, nb = b1 - b0;
    if (na > TB || nb > TB) { flag_structure_error(S); continue; }
    if (tid < na) {
      const int key = Lsd[a0 + tid];
      int pos = lbound(trow, nrow, key);
      if (pos >= nrow || trow[pos] != key) { flag_structure_error(S); pos = -1; }
      relr[tid] = pos;
    } else if (tid >= TB && tid < TB + nb) {
      relc[tid - TB] = Lsd[b0 + tid - TB] - gc_lo;
    }
    double acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
    const double *Ld = S.L + S.xptr[d];
    tile_product(Ld + a0, md, na, Ld + b0, md, nb, wd, As, Bs, acc);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int r = ty + 16 * i;
      if (r >= na) continue;
      const int rr = relr[r];
      if (rr < 0) continue;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int c = tx + 16 * j;
        if (c < nb) Acc[relc[c]][rr] += acc[i][j];
      }
    }
    __syncthreads();
  }
  double *P = S.L + S.xptr[s];
  for (int e = tid; e < TB * TB; e += NT) {
    const int c = e / TB, r = e - c * TB;
    if (r < nrow && c < ncol && trow[r] >= gc_lo + c)
      P[(size_t)(c0 + c) * m + r0 + r] -= Acc[c][r];
  }
}

// ---------------------------------------------------------------------------------------
// Dense factorization of a tiled-class panel, blocked by 64 columns (right-looking):
//   step j:  TRSM of the tiles below diagonal block j against the factored block,
//            then the trailing SYRK/GEMM update of the column blocks after j; the CTA that
//            owns diagonal tile j+1 factors it (POTRF) right after its update, so every
//            diagonal block is factored before the next step's TRSM reads it.
//   block 0 is factored by k_potrf_first.

// In-place lower Cholesky of the bw x bw block D (shared memory, [column][row]); the
// first non-positive pivot's global column + 1 goes to status[0] when `report`.
__device__ void potrf_smem(double (*D)[TB + 1], int bw, const DevSym &S, int gcol0, bool report) {
  const int tid = threadIdx.x;
  for (int j = 0; j < bw; ++j) {
    const double djj = D[j][j];
    const double dsq = sqrt(djj);
    if (report && tid == 0 && !(djj > 0.0)) atomicMin(&S.status[0], gcol0 + j + 1);
    __syncthreads();
    if (tid >= j && tid < bw) D[j][tid] = (tid == j) ? dsq : D[j][tid] / dsq;
    __syncthreads();
    const int nc = bw - j - 1;
    for (int e = tid; e < nc * bw; e += NT) {
      const int c = j + 1 + e / bw, r = e - (c - j - 1) * bw;
      if (r >= c) D[c][r] -= D[j][r] * D[j][c];
    }
    __syncthreads();
  }
}

// Factor diagonal block `c0/64` of supernode s in place (lower triangle only).
__device__ void factor_diag_block(const DevSym &S, int s, int c0, double (*D)[TB + 1]) {
  const int tid = threadIdx.x;
  const int f = S.super[s];
  const int w = S.super[s + 1] - f;
  const int m = (int)(S.rowptr[s + 1] - S.rowptr[s]);
  double *P = S.L + S.xptr[s];
  const int bw = min(TB, w - c0);
  __syncthreads();
  for (int e = tid; e < bw * bw; e += NT) {
    const int c = e / bw, r = e - c * bw;
    D[c][r] = (r >= c) ? P[(size_t)(c0 + c) * m + c0 + r] : 0.0;
  }
  __syncthreads();
  potrf_smem(D, bw, S, f + c0, true);
  for (int e = tid; e < bw * bw; e += NT) {
    const int c = e / bw, r = e - c * bw;
    if (r >= c) P[(size_t)(c0 + c) * m + c0 + r] = D[c][r];
  }
}

constexpr int PANEL_SMEM = 2 * TB * (TB + 1) * 8;

// One CTA per supernode of the list: factor diagonal block 0.
__global__ void __launch_bounds__(NT) k_potrf_first(DevSym S, const int *list, int count) {
  __shared__ double D[TB][TB + 1];
  factor_diag_block(S, list[blockIdx.x], 0, D);
}

// task = (s, r0): B = L[r0:r0+64, blk] := B * L_blk^{-T}, L_blk already factored.
__global__ void __launch_bounds__(NT) k_trsm_step(DevSym S, const int2 *tasks, int count,
                                                  int step) {
  extern __shared__ double dyn[];
  double(*D)[TB + 1] = reinterpret_cast<double(*)[TB + 1]>(dyn);   // [column][row]
  double(*B)[TB + 1] = reinterpret_cast<double(*)[TB + 1]>(dyn + TB * (TB + 1));
  const int s = tasks[blockIdx.x].x, r0 = tasks[blockIdx.x].y;
  const int tid = threadIdx.x;
  const int f = S.super[s];
  const int w = S.super[s + 1] - f;
  const int m = (int)(S.rowptr[s + 1] - S.rowptr[s]);
  double *P = S.L + S.xptr[s];
  const int c0 = step * TB;
  const int bw = min(TB, w - c0);
  const int nr = min(TB, m - r0);
  for (int e = tid; e < bw * bw; e += NT) {
    const int c = e / bw, r = e - c * bw;
    D[c][r] = (r >= c) ? P[(size_t)(c0 + c) * m + c0 + r] : 0.0;
  }
  for (int e = tid; e < nr * bw; e += NT) {
    const int c = e / nr, r = e - c * nr;
    B[c][r] = P[(size_t)(c0 + c) * m + r0 + r];
  }
  __syncthreads();
  // X D^T = B, column by column
  for (int c = 0; c < bw; ++c) {
    if (tid < nr) B[c][tid] = B[c][tid] / D[c][c];
    __syncthreads();
    const int nc = bw - c - 1;
    for (int e = tid; e < nr * nc; e += NT) {
      const int c2 = c + 1 + e / nr, r = e - (c2 - c - 1) * nr;
      B[c2][r] -= B[c][r] * D[c][c2];
    }
    __syncthreads();
  }
  for (int e = tid; e < nr * bw; e += NT) {
    const int c = e / nr, r = e - c * nr;
    P[(size_t)(c0 + c) * m + r0 + r] = B[c][r];
  }
}

// Trailing update of step `step`: task = (s, r0, c0) with c0 >= (step+1)*64, r0 >= c0:
// tile(r0, c0) -= L[r0:, blk] * L[c0:, blk]^T over the step's column block.  The CTA
// holding tile (c0, c0) with c0 == (step+1)*64 then factors that diagonal block.
__global__ void __launch_bounds__(NT) k_syrk_step(DevSym S, const int4 *tasks, int count,
                                                  int step) {
  __shared__ double buf[TB * (TB + 1)];
  double(*As)[TB] = reinterpret_cast<double(*)[TB]>(buf);
  double(*Bs)[TB] = reinterpret_cast<double(*)[TB]>(buf + KC * TB);
  const int4 t = tasks[blockIdx.x];
  const int s = t.x, r0 = t.y, c0 = t.z;
  const int tid = threadIdx.x;
  const int tx = tid & 15, ty = tid >> 4;
  const int f = S.super[s];
  const int w = S.super[s + 1] - f;
  const int m = (int)(S.rowptr[s + 1] - S.rowptr[s]);
  double *P = S.L + S.xptr[s];
  const int k0 = step * TB;
  const int bk = min(TB, w - k0);
  const int nrow = min(TB, m - r0), ncol = min(TB, w - c0);
  double acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
  tile_product(P + (size_t)k0 * m + r0, m, nrow, P + (size_t)k0 * m + c0, m, ncol, bk, As,
               Bs, acc);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int r = ty + 16 * i;
    if (r >= nrow) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int c = tx + 16 * j;
      if (c < ncol && r0 + r >= c0 + c) P[(size_t)(c0 + c) * m + r0 + r] -= acc[i][j];
    }
  }
  if (r0 == c0 && c0 == k0 + TB) {
    // writes above are visible to the whole CTA after the barrier inside factor_diag_block
    factor_diag_block(S, s, c0, reinterpret_cast<double(*)[TB + 1]>(buf));
  }
}

__global__ void k_init_status(int *status) {
  status[0] = INT_MAX;
  status[1] = 0;
}

}  // namespace

bool kernels_configure(std::string &err) {
  cudaError_t e = cudaFuncSetAttribute(k_factor_small, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       200 * 1024);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_update_tiles, cudaFuncAttributeMaxDynamicSharedMemorySize, UPD_SMEM);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_trsm_step, cudaFuncAttributeMaxDynamicSharedMemorySize, PANEL_SMEM);
  if (e != cudaSuccess) {
    err = std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e);
    return false;
  }
  return true;
}

void launch_factor_small(const DevSym &S, const int *list, int count, int smem, cudaStream_t st) {
  if (count > 0) k_factor_small<<<count, NT, smem, st>>>(S, list, count);
}
void launch_assemble(const DevSym &S, const int2 *tasks, int count, cudaStream_t st) {
  if (count > 0) k_assemble<<<(count * 32 + NT - 1) / NT, NT, 0, st>>>(S, tasks, count);
}
void launch_update_tiles(const DevSym &S, const int4 *tasks, int count, cudaStream_t st) {
  if (count > 0) k_update_tiles<<<count, NT, UPD_SMEM, st>>>(S, tasks, count);
}
void launch_potrf_first(const DevSym &S, const int *list, int count, cudaStream_t st) {
  if (count > 0) k_potrf_first<<<count, NT, 0, st>>>(S, list, count);
}
void launch_trsm_step(const DevSym &S, const int2 *tasks, int count, int step, cudaStream_t st) {
  if (count > 0) k_trsm_step<<<count, NT, PANEL_SMEM, st>>>(S, tasks, count, step);
}
void launch_syrk_step(const DevSym &S, const int4 *tasks, int count, int step, cudaStream_t st) {
  if (count > 0) k_syrk_step<<<count, NT, 0, st>>>(S, tasks, count, step);
}
void launch_init_status(int *status, cudaStream_t st) { k_init_status<<<1, 1, 0, st>>>(status); }

}  // namespace swc
