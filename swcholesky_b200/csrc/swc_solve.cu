// Supernodal triangular solves, sparse matrix-vector product and vector kernels for
// iterative refinement.  No reference counterpart for the backward solve; the forward
// solve follows the reference's layout-compatible blockedLsolve
// (triangularSolve/Triangular_BCSC.h:14-48) in gather (left-looking) form, so every
// supernode of a level runs in parallel with no atomics and a fixed summation order.
#include <cuda_runtime.h>

#include <cstdint>

#include "swc_engine.h"

namespace swc {

namespace {

constexpr int ST = 256;   // threads of the solve kernels
constexpr int SB = 32;    // column block of the dense triangular solves (one warp)

// Forward solve, level by level (leaves first), in two kernels per level:
//   k_fwd_diag    y[cols of s] := L_ss^{-1} (y[cols of s] - sum of the contributions the
//                 descendants stored for those columns), one CTA per supernode; column j's
//                 contributions are listed in cidx[cptr[j] .. cptr[j+1]) (one entry per
//                 off-diagonal row of L equal to j, in increasing supernode order), so
//                 every column sums its own list with no barrier.
//   k_fwd_contrib c_s = L_s[rows below the diagonal block, :] y[cols of s], one CTA per
//                 32-row slab: the off-diagonal GEMV of every supernode runs in parallel.
// c_s lives at contrib + rowptr[s] - super[s] (one entry per off-diagonal row).
__global__ void __launch_bounds__(ST) k_fwd_diag(DevSym S, const int *list, double *y,
                                                 const double *contrib, const int *cptr,
                                                 const int *cidx, int n, int nrhs,
                                                 int64_t cstride) {
  extern __shared__ double v[];
  __shared__ double blk[SB * (SB + 1)];
  const int s = list[blockIdx.x];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int f = S.super[s], w = S.super[s + 1] - f;
  const int m = (int)(S.rowptr[s + 1] - S.rowptr[s]);
  const double *Ls_s = S.L + S.xptr[s];
  for (int rhs = 0; rhs < nrhs; ++rhs) {
    double *yr = y + (size_t)rhs * n;
    const double *cr = contrib + (size_t)rhs * cstride;
    __syncthreads();
    // column j of s receives the contributions listed for it (descendant order)
    for (int i = tid; i < w; i += ST) {
      double acc = yr[f + i];
      for (int q = cptr[f + i]; q < cptr[f + i + 1]; ++q) acc -= cr[cidx[q]];
      v[i] = acc;
    }
    __syncthreads();
    // dense lower solve with the diagonal block, blocked by SB columns; each SB x SB block
    // and the reciprocals of its diagonal are staged first, so the serial chain of warp 0
    // reads only shared memory
    for (int j0 = 0; j0 < w; j0 += SB) {
      const int jb = min(SB, w - j0);
      for (int e = tid; e < jb * jb; e += ST) {
        const int j = e / jb, i = e - j * jb;
        blk[j * (SB + 1) + i] = Ls_s[(size_t)(j0 + j) * m + j0 + i];
      }
      __syncthreads();
      if (warp == 0) {
        const double rdl = (lane < jb) ? 1.0 / blk[lane * (SB + 1) + lane] : 0.0;
        double x = (lane < jb) ? v[j0 + lane] : 0.0;
        for (int j = 0; j < jb; ++j) {
          if (lane == j) x *= rdl;
          const double xj = __shfl_sync(0xffffffffu, x, j);
          if (lane > j && lane < jb) x = fma(-blk[j * (SB + 1) + lane], xj, x);
        }
        if (lane < jb) v[j0 + lane] = x;
      }
      __syncthreads();
      for (int i = j0 + jb + tid; i < w; i += ST) {
        double acc = v[i];
        for (int j = 0; j < jb; ++j) acc = fma(-Ls_s[(size_t)(j0 + j) * m + i], v[j0 + j], acc);
        v[i] = acc;
      }
      __syncthreads();
    }
    for (int i = tid; i < w; i += ST) yr[f + i] = v[i];
  }
}

// Contribution tasks.  Very wide supernodes (w > SOLVE_CONTRIB_BIG_W; few of them, each a
// long row of work): task = (s, r0), 32 rows, one CTA of 32 warps, warp q summing the
// columns k = q (mod 32) with four loads in flight, so a level of one or two such
// supernodes still spreads over the GPU.  Wide supernodes (w > SOLVE_NARROW_W): task = (s, r0), rows
// r0 .. r0 + SOLVE_CONTRIB_WIDE_ROWS - 1 of the off-diagonal block (r0 >= w), one CTA of CW
// warps: warp q sums the columns k = q (mod CW), lane l the rows r0 + l + 32 t (t < 4), with
// four columns unrolled (sixteen loads in flight per lane, each warp load 32 consecutive
// rows of a column), and the CW partial sums meet in shared memory in a fixed order.
// Narrow supernodes: task = (s, r0), 32 rows, one warp (lane = row, all w columns), CW per
// CTA after the nwide wide tasks.
constexpr int CR = SOLVE_CONTRIB_ROWS, CRW = SOLVE_CONTRIB_WIDE_ROWS, CW = 8, CT = 32 * CW;
constexpr int CTB = 1024, CQB = CTB / CR;
__global__ void __launch_bounds__(CTB) k_fwd_contrib_big(DevSym S, const int2 *tasks,
                                                        const double *y, double *contrib, int n,
                                                        int nrhs, int64_t cstride) {
  __shared__ double part[CQB][CR];
  const int s = tasks[blockIdx.x].x, r0 = tasks[blockIdx.x].y;
  const int f = S.super[s], w = S.super[s + 1] - f;
  const int64_t rb = S.rowptr[s];
  const int m = (int)(S.rowptr[s + 1] - rb);
  const double *Ls_s = S.L + S.xptr[s];
  const int r = threadIdx.x & (CR - 1), q = threadIdx.x / CR;
  const int a = r0 + r;
  for (int rhs = 0; rhs < nrhs; ++rhs) {
    const double *yr = y + (size_t)rhs * n + f;
    double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0, acc3 = 0.0;
    if (a < m) {
      const double *col = Ls_s + a;
      int k = q;
      for (; k + 3 * CQB < w; k += 4 * CQB) {
        acc0 = fma(col[(size_t)k * m], yr[k], acc0);
        acc1 = fma(col[(size_t)(k + CQB) * m], yr[k + CQB], acc1);
        acc2 = fma(col[(size_t)(k + 2 * CQB) * m], yr[k + 2 * CQB], acc2);
        acc3 = fma(col[(size_t)(k + 3 * CQB) * m], yr[k + 3 * CQB], acc3);
      }
      for (; k < w; k += CQB) acc0 = fma(col[(size_t)k * m], yr[k], acc0);
    }
    part[q][r] = (acc0 + acc1) + (acc2 + acc3);
    __syncthreads();
    if (q == 0 && a < m) {
      double t = 0.0;
#pragma unroll
      for (int g = 0; g < CQB; ++g) t += part[g][r];
      contrib[(size_t)rhs * cstride + (rb - f) + (a - w)] = t;
    }
    __syncthreads();
  }
}

static_assert(CR == 32 && CRW == 4 * CR, "a lane covers four rows of a wide task");
__device__ void fwd_contrib_narrow(const DevSym &S, int2 task, const double *y, double *contrib,
                                   int n, int nrhs, int64_t cstride) {
  const int s = task.x, r0 = task.y, lane = threadIdx.x & 31;
  const int f = S.super[s], w = S.super[s + 1] - f;
  const int64_t rb = S.rowptr[s];
  const int m = (int)(S.rowptr[s + 1] - rb);
  const int a = r0 + lane;
  if (a >= m) return;
  const double *col = S.L + S.xptr[s] + a;
  for (int rhs = 0; rhs < nrhs; ++rhs) {
    const double *yr = y + (size_t)rhs * n + f;
    double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0, acc3 = 0.0;
    int k = 0;
    for (; k + 3 < w; k += 4) {
      acc0 = fma(col[(size_t)k * m], yr[k], acc0);
      acc1 = fma(col[(size_t)(k + 1) * m], yr[k + 1], acc1);
      acc2 = fma(col[(size_t)(k + 2) * m], yr[k + 2], acc2);
      acc3 = fma(col[(size_t)(k + 3) * m], yr[k + 3], acc3);
    }
    for (; k < w; ++k) acc0 = fma(col[(size_t)k * m], yr[k], acc0);
    contrib[(size_t)rhs * cstride + (rb - f) + (a - w)] = (acc0 + acc1) + (acc2 + acc3);
  }
}

__global__ void __launch_bounds__(CT) k_fwd_contrib(DevSym S, const int2 *tasks, int count,
                                                    int nwide, const double *y, double *contrib,
                                                    int n, int nrhs, int64_t cstride) {
  __shared__ double part[CW][CRW];
  if ((int)blockIdx.x >= nwide) {
    const int t = nwide + ((int)blockIdx.x - nwide) * CW + (int)(threadIdx.x >> 5);
    if (t < count) fwd_contrib_narrow(S, tasks[t], y, contrib, n, nrhs, cstride);
    return;
  }
  const int s = tasks[blockIdx.x].x, r0 = tasks[blockIdx.x].y;
  const int f = S.super[s], w = S.super[s + 1] - f;
  const int64_t rb = S.rowptr[s];
  const int m = (int)(S.rowptr[s + 1] - rb);
  const double *Ls_s = S.L + S.xptr[s];
  const int lane = threadIdx.x & 31, q = threadIdx.x >> 5;
  // rows of this lane (rows past the panel read row r0 and are dropped)
  int ra[4];
  bool in[4];
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    ra[t] = r0 + lane + 32 * t;
    in[t] = ra[t] < m;
    if (!in[t]) ra[t] = r0;
  }
  for (int rhs = 0; rhs < nrhs; ++rhs) {
    const double *yr = y + (size_t)rhs * n + f;
    double acc[4][2];
#pragma unroll
    for (int t = 0; t < 4; ++t) acc[t][0] = acc[t][1] = 0.0;
    int k = q;
    for (; k + 3 * CW < w; k += 4 * CW) {
      const double y0 = yr[k], y1 = yr[k + CW], y2 = yr[k + 2 * CW], y3 = yr[k + 3 * CW];
      const double *c0 = Ls_s + (size_t)k * m, *c1 = c0 + (size_t)CW * m;
      const double *c2 = c1 + (size_t)CW * m, *c3 = c2 + (size_t)CW * m;
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        acc[t][0] = fma(c0[ra[t]], y0, acc[t][0]);
        acc[t][1] = fma(c1[ra[t]], y1, acc[t][1]);
        acc[t][0] = fma(c2[ra[t]], y2, acc[t][0]);
        acc[t][1] = fma(c3[ra[t]], y3, acc[t][1]);
      }
    }
    for (; k < w; k += CW) {
      const double yk = yr[k];
      const double *ck = Ls_s + (size_t)k * m;
#pragma unroll
      for (int t = 0; t < 4; ++t) acc[t][0] = fma(ck[ra[t]], yk, acc[t][0]);
    }
#pragma unroll
    for (int t = 0; t < 4; ++t) part[q][lane + 32 * t] = acc[t][0] + acc[t][1];
    __syncthreads();
    if (threadIdx.x < CRW) {
      const int a = r0 + (int)threadIdx.x;
      if (a < m) {
        double t = 0.0;
#pragma unroll
        for (int g = 0; g < CW; ++g) t += part[g][threadIdx.x];
        contrib[(size_t)rhs * cstride + (rb - f) + (a - w)] = t;
      }
    }
    __syncthreads();
  }
}

// Backward solve, level by level (root first):
//   k_bwd_gather  x[f + j] := x[f + j] - sum_{a >= w} L(a, j) x[rows[a]] for the columns
//                 j0..j0+15 of s (one warp per column, eight loads in flight per lane);
//                 the rows below are columns of ancestors, already solved.
//   k_bwd_diag    x[cols of s] := L_ss^{-T} x[cols of s], one CTA per supernode.
constexpr int GCH = 2048;       // gathered rows staged per chunk
constexpr int GT = 32 * SOLVE_GATHER_COLS;   // one warp per column of the task
__global__ void __launch_bounds__(GT) k_bwd_gather(DevSym S, const int2 *tasks, double *x,
                                                   int n, int nrhs) {
  __shared__ double xg[GCH];
  const int s = tasks[blockIdx.x].x, j0 = tasks[blockIdx.x].y;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int f = S.super[s], w = S.super[s + 1] - f;
  const int64_t rb = S.rowptr[s];
  const int m = (int)(S.rowptr[s + 1] - rb);
  const int *rows = S.Ls + rb;
  const double *Ls_s = S.L + S.xptr[s];
  const int j = j0 + warp;
  const bool own = j < w;
  // every column of this CTA reads the same x[rows[a]]: gather them once per chunk
  for (int rhs = 0; rhs < nrhs; ++rhs) {
    double *xr = x + (size_t)rhs * n;
    double acc[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) acc[u] = 0.0;
    for (int a0 = w; a0 < m; a0 += GCH) {
      const int len = min(GCH, m - a0);
      __syncthreads();
      for (int i = threadIdx.x; i < len; i += GT) xg[i] = xr[rows[a0 + i]];
      __syncthreads();
      if (own) {
        const double *col = Ls_s + (size_t)j * m + a0;
        int i = lane;
        for (; i + 7 * 32 < len; i += 8 * 32)
#pragma unroll
          for (int u = 0; u < 8; ++u) acc[u] = fma(col[i + 32 * u], xg[i + 32 * u], acc[u]);
        for (; i < len; i += 32) acc[0] = fma(col[i], xg[i], acc[0]);
      }
    }
    double t = ((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (lane == 0 && own) xr[f + j] -= t;
    __syncthreads();   // these columns are written before the next right-hand side gathers
  }
}

// ---- small supernodes (w <= SOLVE_WARP_W, at most SOLVE_WARP_ROWS rows below the diagonal
// block), one warp each, lane = column of the supernode.  Forward: the contributions the
// descendants stored for its columns, the lower solve with the diagonal block (shuffles),
// then its own contributions to the rows below (lane = row); backward: the gather from the
// ancestors' solved values (lane = column, walking the rows below), then the transposed
// solve.  Level by level like the CTA kernels; a CTA holds WPC independent warps.
constexpr int WPC = ST / 32;

__global__ void __launch_bounds__(ST) k_fwd_warp(DevSym S, const int *list, int count,
                                                 double *y, double *contrib, const int *cptr,
                                                 const int *cidx, int n, int nrhs,
                                                 int64_t cstride) {
  const int t = blockIdx.x * WPC + (threadIdx.x >> 5);
  if (t >= count) return;
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int s = list[t];
  const int f = S.super[s], w = S.super[s + 1] - f;
  const int64_t rb = S.rowptr[s];
  const int m = (int)(S.rowptr[s + 1] - rb);
  const double *Ls_s = S.L + S.xptr[s];
  for (int rhs = 0; rhs < nrhs; ++rhs) {
    double *yr = y + (size_t)rhs * n;
    double *cr = contrib + (size_t)rhs * cstride;
    double v = 0.0;
    if (lane < w) {
      v = yr[f + lane];
      for (int q = cptr[f + lane]; q < cptr[f + lane + 1]; ++q) v -= cr[cidx[q]];
    }
    // L_ss y = v
#pragma unroll 4
    for (int j = 0; j < w; ++j) {
      const double ljj = Ls_s[(size_t)j * m + j];
      const double lij = (lane > j && lane < w) ? Ls_s[(size_t)j * m + lane] : 0.0;
      if (lane == j) v = v / ljj;
      const double yj = __shfl_sync(FULL, v, j);
      if (lane > j) v = fma(-lij, yj, v);
    }
    if (lane < w) yr[f + lane] = v;
    // contributions of the rows below: c[a] = sum_j L(a, j) y_j
    for (int a0 = w; a0 < m; a0 += 32) {
      const int a = a0 + lane;
      double acc = 0.0;
#pragma unroll 4
      for (int j = 0; j < w; ++j) {
        const double yj = __shfl_sync(FULL, v, j);
        if (a < m) acc = fma(Ls_s[(size_t)j * m + a], yj, acc);
      }
      if (a < m) cr[(rb - f) + (a - w)] = acc;
    }
  }
}

__global__ void __launch_bounds__(ST) k_bwd_warp(DevSym S, const int *list, int count, double *x,
                                                 int n, int nrhs) {
  const int t = blockIdx.x * WPC + (threadIdx.x >> 5);
  if (t >= count) return;
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int s = list[t];
  const int f = S.super[s], w = S.super[s + 1] - f;
  const int64_t rb = S.rowptr[s];
  const int m = (int)(S.rowptr[s + 1] - rb);
  const int *rows = S.Ls + rb;
  const double *Ls_s = S.L + S.xptr[s];
  for (int rhs = 0; rhs < nrhs; ++rhs) {
    double *xr = x + (size_t)rhs * n;
    double v = 0.0;
    if (lane < w) {
      // x_i - sum_{a >= w} L(a, i) x[rows[a]]
      const double *col = Ls_s + (size_t)lane * m;
      double a0 = 0.0, a1 = 0.0;
      int a = w;
      for (; a + 1 < m; a += 2) {
        a0 = fma(col[a], xr[rows[a]], a0);
        a1 = fma(col[a + 1], xr[rows[a + 1]], a1);
      }
      if (a < m) a0 = fma(col[a], xr[rows[a]], a0);
      v = xr[f + lane] - (a0 + a1);
    }
    // L_ss^T x = v
#pragma unroll 4
    for (int j = w - 1; j >= 0; --j) {
      const double ljj = Ls_s[(size_t)j * m + j];
      const double lji = lane < j ? Ls_s[(size_t)lane * m + j] : 0.0;
      if (lane == j) v = v / ljj;
      const double xj = __shfl_sync(FULL, v, j);
      if (lane < j) v = fma(-lji, xj, v);
    }
    if (lane < w) xr[f + lane] = v;
  }
}

__global__ void __launch_bounds__(ST) k_bwd_diag(DevSym S, const int *list, double *x, int n,
                                                 int nrhs) {
  extern __shared__ double v[];
  __shared__ double blk[SB * (SB + 1)];
  const int s = list[blockIdx.x];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int f = S.super[s], w = S.super[s + 1] - f;
  const int m = (int)(S.rowptr[s + 1] - S.rowptr[s]);
  const double *Ls_s = S.L + S.xptr[s];
  for (int rhs = 0; rhs < nrhs; ++rhs) {
    double *xr = x + (size_t)rhs * n;
    __syncthreads();
    for (int i = tid; i < w; i += ST) v[i] = xr[f + i];
    __syncthreads();
    for (int j1 = w; j1 > 0; j1 -= SB) {
      const int j0 = max(0, j1 - SB), jb = j1 - j0;
      // v[j0..j1) -= sum_{i >= j1} L(i, j) v[i]
      for (int j = j0 + warp; j < j1; j += ST / 32) {
        double acc = 0.0;
        for (int i = j1 + lane; i < w; i += 32) acc = fma(Ls_s[(size_t)j * m + i], v[i], acc);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) v[j] -= acc;
      }
      for (int e = tid; e < jb * jb; e += ST) {
        const int j = e / jb, i = e - j * jb;
        blk[j * (SB + 1) + i] = Ls_s[(size_t)(j0 + j) * m + j0 + i];
      }
      __syncthreads();
      if (warp == 0) {
        const double rdl = (lane < jb) ? 1.0 / blk[lane * (SB + 1) + lane] : 0.0;
        double xv = (lane < jb) ? v[j0 + lane] : 0.0;
        for (int jj = jb - 1; jj >= 0; --jj) {
          if (lane == jj) xv *= rdl;
          const double xj = __shfl_sync(0xffffffffu, xv, jj);
          if (lane < jj) xv = fma(-blk[lane * (SB + 1) + jj], xj, xv);
        }
        if (lane < jb) v[j0 + lane] = xv;
      }
      __syncthreads();
    }
    for (int i = tid; i < w; i += ST) xr[f + i] = v[i];
  }
}

// Per-block counters of the chained solves: each of a block's eight warps adds 1 (release)
// once its rows of the block's solution are in global memory, so the solution of pass e
// (the e-th chain launch that includes the block since the counters were cleared) is
// complete when the counter reaches 8e.  Waits are
// bounded: after the poll budget in status[4] a waiter records a timeout in status[2] and
// stops waiting.
constexpr int CHAIN_WARPS = ST / 32;
__device__ __forceinline__ int ld_acquire(const int *p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];\n" : "=r"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ void red_release_add(int *p, int v) {
  asm volatile("red.release.gpu.global.add.s32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}

// Lane u < nf polls the counter at flag + dir * u (no sleep between polls: a hop between
// clusters is on the chain's critical path) until the first one has reached `target`;
// returns how many consecutive counters from the first have reached it (1 .. nf), or 0
// after a timeout (its own, or one another block recorded).  A batch is never held back
// by a block that is not finished yet.
__device__ int warp_wait_prefix(const int *flag, int dir, int nf, int target, int *status) {
  const long long budget = wait_budget(status);
  long long it = 0;
  const int lane = threadIdx.x & 31;
  bool mine = lane < nf && ld_acquire(flag + dir * lane) >= target;
  int n = 0;
  for (;;) {
    const unsigned done = __ballot_sync(0xffffffffu, mine);
    n = min(nf, __ffs(~done) - 1);
    if (n > 0) break;
    if (++it > budget || ((it & 31) == 0 && *(volatile int *)&status[2])) {
      if (lane == 0) atomicExch(&status[2], 1);
      break;
    }
    if (lane < nf && !mine) mine = ld_acquire(flag + dir * lane) >= target;
  }
  __syncwarp();   // the lanes' later loads are ordered after the polling lanes' acquires
  return n;
}

template <int N>
__device__ __forceinline__ void stage_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }
// an empty cp.async group (keeps one group per ring step)
__device__ __forceinline__ void stage_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp8(double *dst, const double *src, bool in) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(
                   (unsigned)__cvta_generic_to_shared(dst)),
               "l"(src), "r"(in ? 8 : 0));
}

// ---- chained dense solves with the diagonal block of a tiled-class supernode -----------
// One CTA per 64-row block k of the diagonal block; block k consumes the solved blocks
// c < k (forward) or c > k (backward) as they arrive and applies its own block through the
// stored inverse T_k of the 64x64 diagonal block.  All CTAs of a chain are resident
// together (a few hundred at most) and only wait on CTAs with a lower blockIdx, which the
// hardware dispatches first.
//
// Warp w owns rows 8w .. 8w + 7 of the block's right-hand side v: it stages its eight rows
// of each predecessor's panel block in its own shared-memory ring (cp.async, NS slots,
// NS - 1 blocks ahead), holds them and its rows of T_k in registers, and lane
// l multiplies columns l and l + 32; a butterfly of shuffles sums the eight rows across
// the lanes (row 8w + (l >> 2) in every lane of quad l >> 2).  No block barrier until the
// last predecessor is applied; then one barrier hands v to every warp for x_k = T_k v.
// The step that waits for a predecessor's solution therefore only reads it, sixteen FMAs
// and nine shuffles.
// Ring depth: CHAIN_NS_BIG for launches that fit the GPU at one CTA per SM (long chains:
// deep prefetch), CHAIN_NS_SMALL (two CTAs per SM) for levels of many short chains.
constexpr int CHAIN_NS_BIG = 5, CHAIN_NS_SMALL = 2;
constexpr int LW = TB + 1;                      // padded row of a staged block
constexpr int CHAIN_SLOT = 8 * LW;              // one warp's eight rows
// Predecessors outside the cluster come from global memory in batches of up to CHAIN_XB
// finished blocks: their counters are polled together and their solutions loaded together
// (a lane keeps the two elements it multiplies, in its warp's batch buffer), so a batch
// costs two memory round trips instead of two per block.
constexpr int CHAIN_XB = 8;
// dynamic shared memory: the ring, then each warp's batch buffer (forward: x_c(8w .. 8w+7)
// of up to eight blocks; backward: whole x_c of up to CHAIN_XB blocks)
constexpr int CHAIN_XW_FWD = TB, CHAIN_XW_BWD = CHAIN_XB * TB;
constexpr int chain_smem(int ns, int xw) { return (ns * CHAIN_SLOT + xw) * CHAIN_WARPS * 8; }

// Chains launch in thread-block clusters of CHAIN_CL consecutive tasks.  A block publishes its
// solution through global memory and its counter (for the blocks of later clusters and the
// next level's kernels) and also writes it straight into the shared memory of the later blocks
// of its supernode in its own cluster (distributed shared memory) with st.async, whose
// transaction bytes complete the receiver's mbarrier of that sender slot: a hop inside a
// cluster neither goes through L2 nor waits for a release fence.  Slot j of a block
// receives the solution of cluster rank j (64 doubles, 512 transaction bytes, armed at
// set-up).  Every CTA of a cluster (tail padding included) passes a cluster barrier after
// the mbarrier set-up and another before it exits, so no block leaves while a remote
// write to it may be in flight.
constexpr int CHAIN_CL = 8;
struct ChainCluster {
  double yin[CHAIN_CL][TB];
  unsigned long long bar[CHAIN_CL];
};

__device__ __forceinline__ uint32_t chain_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;\n" : "=r"(r));
  return r;
}
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;\n" ::
                   : "memory");
}
__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
// address of the same shared-memory location in the CTA of cluster rank `rank`
__device__ __forceinline__ uint32_t cluster_addr(const void *p, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;\n" : "=r"(r) : "r"(smem_addr(p)), "r"(rank));
  return r;
}
__device__ __forceinline__ void chain_cluster_init(ChainCluster &cc) {
  if (threadIdx.x == 0) {
    for (int j = 0; j < CHAIN_CL; ++j) {
      const uint32_t b = smem_addr(&cc.bar[j]);
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(b) : "memory");
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(b), "r"(TB * 8)
                   : "memory");
    }
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  cluster_sync_all();
}
// Lane l (holding element `row` of this block's solution when (l & 3) == 0; every lane of
// quad l >> 2 holds it) sends it to the later ranks me+1 .. last of its cluster, the four
// lanes of a quad to different ranks.
__device__ __forceinline__ void chain_send(ChainCluster &cc, int me, int last, int row, double val) {
  for (int q = me + 1 + (threadIdx.x & 3); q <= last; q += 4)
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.f64 [%0], %1, [%2];\n" ::"r"(
                     cluster_addr(&cc.yin[me][row], q)),
                 "d"(val), "r"(cluster_addr(&cc.bar[me], q))
                 : "memory");
}
// Every lane waits (bounded) for slot j's 512 bytes; false after a timeout (its own, or
// one another block recorded) in any lane.
__device__ bool warp_chain_recv(ChainCluster &cc, int j, int *status) {
  const uint32_t b = smem_addr(&cc.bar[j]);
  const long long budget = wait_budget(status);
  long long it = 0;
  int ok = 1;
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 P1, [%1], 0;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(done)
        : "r"(b)
        : "memory");
    if (done) break;
    if (++it > budget || ((it & 31) == 0 && *(volatile int *)&status[2])) {
      atomicExch(&status[2], 1);
      ok = 0;
      break;
    }
  }
  return __all_sync(0xffffffffu, ok) != 0;
}

// Sum over the lanes of a[i] (this lane's part of row 8w + i): the total of row
// 8w + ((lane >> 2) & 7), in every lane of the quad.
__device__ __forceinline__ double warp_rows8(double (&a)[8], int lane) {
  const unsigned F = 0xffffffffu;
  const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const double o = __shfl_xor_sync(F, b4 ? a[i] : a[i + 4], 16);
    a[i] = (b4 ? a[i + 4] : a[i]) + o;
  }
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const double o = __shfl_xor_sync(F, b3 ? a[i] : a[i + 2], 8);
    a[i] = (b3 ? a[i + 2] : a[i]) + o;
  }
  {
    const double o = __shfl_xor_sync(F, b2 ? a[0] : a[1], 4);
    a[0] = (b2 ? a[1] : a[0]) + o;
  }
  a[0] += __shfl_xor_sync(F, a[0], 2);
  a[0] += __shfl_xor_sync(F, a[0], 1);
  return a[0];
}

// task = (s, k); forward: y[f + 64k ..] := T_k (y[...] - contributions - sum_{c<k} L_kc x_c)
// (tasks of a supernode consecutive, in increasing k; CTAs from `count` on are padding).
// Warp w takes columns 8w .. 8w + 7 of every L_kc (eight contiguous 512-byte column pieces
// of the panel, staged by the warp alone) and keeps its partial sums of all 64 rows (rows
// l and l + 32 in lane l); the eight warps' partial sums meet once, after the last
// predecessor, and x_k = T_k v is then formed with warp w owning rows 8w .. 8w + 7.
template <int NS>
__global__ void __launch_bounds__(ST, NS == CHAIN_NS_SMALL ? 2 : 1) k_fwd_chain(DevSym S, const int2 *tasks, int count,
                                                     double *y, const double *contrib,
                                                     const int *cptr, const int *cidx, int *flags,
                                                     int epoch, int n, int64_t cstride) {
  extern __shared__ double csm[];
  __shared__ double vs[TB], part[CHAIN_WARPS][TB];
  __shared__ ChainCluster cc;
  chain_cluster_init(cc);
  const int me = (int)chain_rank();
  if ((int)blockIdx.x < count) {
    const int s = tasks[blockIdx.x].x, k = tasks[blockIdx.x].y;
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5, w8 = wp * 8;
    const int row = w8 + ((lane >> 2) & 7);   // the row of x_k this lane's sums belong to
    const int f = S.super[s], w = S.super[s + 1] - f;
    const int m = (int)(S.rowptr[s + 1] - S.rowptr[s]);
    const double *P = S.L + S.xptr[s];
    const int r0 = k * TB, bw = min(TB, w - r0);
    const int nb = (w + TB - 1) / TB;
    const int base = S.dinv_off[s];
    const double *T = S.dinv + ((size_t)base + k) * (TB * TB);   // T(r, c) at T[c * 64 + r]
    // predecessors c >= cfirst are in this cluster (rank me - (k - c)); the later ranks of
    // the same supernode receive this block's solution
    const int cfirst = k - me, last = me + min(nb - 1 - k, CHAIN_CL - 1 - me);
    double *ring = csm + wp * CHAIN_SLOT;   // slot j at ring + j * CHAIN_WARPS * CHAIN_SLOT
    double *xw = csm + NS * CHAIN_WARPS * CHAIN_SLOT + wp * CHAIN_XW_FWD;
    // this warp's columns of L_kc: element (r, 8w + q) = P[(64c + 8w + q) m + r0 + r] at
    // [q * LW + r] (a warp instruction copies 32 consecutive rows of one column)
    auto stage = [&](int c) {
      if (c < k) {
        double *d = ring + (c % NS) * CHAIN_WARPS * CHAIN_SLOT;
        const double *src = P + (size_t)(c * TB + w8) * m + r0;
#pragma unroll 4
        for (int t = 0; t < 16; ++t) {
          const int e = lane + 32 * t, q = e >> 6, r = e & (TB - 1);
          const bool in = r < bw;
          cp8(d + q * LW + r, in ? src + (size_t)q * m + r : src, in);
        }
      }
      stage_commit();
    };
    for (int c = 0; c < NS - 1; ++c) stage(c);
    double tr[8][2];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      tr[i][0] = T[(size_t)lane * TB + w8 + i];
      tr[i][1] = T[(size_t)(lane + 32) * TB + w8 + i];
    }
    // right-hand side minus the descendants' contributions (read after the last barrier)
    if (threadIdx.x < TB) {
      double v = 0.0;
      if ((int)threadIdx.x < bw) {
        const int j = f + r0 + threadIdx.x;
        v = y[j];
        for (int qq = cptr[j]; qq < cptr[j + 1]; ++qq) v -= contrib[cidx[qq]];
      }
      vs[threadIdx.x] = v;
    }
    double acc0 = 0.0, acc1 = 0.0;   // rows lane, lane + 32 over this warp's columns
    bool ok = true;
    int xb0 = 0, nbt = 0;            // the batch in xw: blocks xb0 .. xb0 + nbt - 1
    for (int c = 0; c < k; ++c) {
      stage(c + NS - 1);                 // into the slot freed by step c - 1
      stage_wait<NS - 1>();              // block c has landed (this lane's copies)
      __syncwarp();
      const double *Lc = ring + (c % NS) * CHAIN_WARPS * CHAIN_SLOT;
      double lr[8][2];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        lr[q][0] = Lc[q * LW + lane];
        lr[q][1] = Lc[q * LW + lane + 32];
      }
      __syncwarp();                      // the slot is refilled at step c + 1
      const double *xc;                  // x_c(8w + q) at xc[q]
      if (c >= cfirst) {   // from the cluster
        const int j = me - (k - c);
        if (!warp_chain_recv(cc, j, S.status)) { ok = false; break; }
        xc = &cc.yin[j][w8];
      } else {             // from global memory, a batch of finished blocks at a time
        if (c >= xb0 + nbt) {
          xb0 = c;
          nbt = warp_wait_prefix(&flags[base + c], 1, min(CHAIN_XB, cfirst - c), CHAIN_WARPS * epoch,
                                 S.status);
          if (nbt == 0) { ok = false; break; }
          // x_{c+u}(8w + q) into xw[u * 8 + q], lane = u * 8 + q (two rounds of four blocks)
          const int q = lane & 7, u = lane >> 3;
          const double a0 = u < nbt ? __ldcg(&y[f + (c + u) * TB + w8 + q]) : 0.0;
          const double a1 = u + 4 < nbt ? __ldcg(&y[f + (c + u + 4) * TB + w8 + q]) : 0.0;
          xw[lane] = a0;
          xw[lane + 32] = a1;
          __syncwarp();
        }
        xc = xw + (c - xb0) * 8;
      }
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const double xq = xc[q];
        acc0 = fma(lr[q][0], xq, acc0);
        acc1 = fma(lr[q][1], xq, acc1);
      }
      __syncwarp();                      // xw is rewritten by the next batch
    }
    stage_wait<0>();
    part[wp][lane] = acc0;
    part[wp][lane + 32] = acc1;
    ok = __syncthreads_and(ok) != 0;
    if (ok) {
      // v(j) for j = lane, lane + 32; then x_k = T_k v
      double x0 = vs[lane], x1 = vs[lane + 32];
#pragma unroll
      for (int g = 0; g < CHAIN_WARPS; ++g) {
        x0 -= part[g][lane];
        x1 -= part[g][lane + 32];
      }
      double a[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) a[i] = fma(tr[i][1], x1, tr[i][0] * x0);
      const double xk = warp_rows8(a, lane);
      // the cluster's later blocks first, then global memory and the counter
      chain_send(cc, me, last, row, row < bw ? xk : 0.0);
      if ((lane & 3) == 0 && row < bw) y[f + r0 + row] = xk;
      __syncwarp();
      if (lane == 0) red_release_add(&flags[base + k], 1);
    }
  }
  cluster_sync_all();
}

// task = (s, k) in decreasing k; backward: x[f + 64k ..] := T_k^T (x[...] - sum_{c>k} L_ck^T x_c)
// (tasks of a supernode consecutive, in decreasing k; CTAs from `count` on are padding)
template <int NS>
__global__ void __launch_bounds__(ST, NS == CHAIN_NS_SMALL ? 2 : 1) k_bwd_chain(DevSym S, const int2 *tasks, int count,
                                                  double *x, int *flags, int epoch) {
  extern __shared__ double csm[];
  __shared__ double vs[TB];
  __shared__ ChainCluster cc;
  chain_cluster_init(cc);
  const int me = (int)chain_rank();
  if ((int)blockIdx.x < count) {
    const int s = tasks[blockIdx.x].x, k = tasks[blockIdx.x].y;
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5, w8 = wp * 8;
    const int row = w8 + ((lane >> 2) & 7);
    const int f = S.super[s], w = S.super[s + 1] - f;
    const int m = (int)(S.rowptr[s + 1] - S.rowptr[s]);
    const double *P = S.L + S.xptr[s];
    const int r0 = k * TB, bw = min(TB, w - r0);
    const int nb = (w + TB - 1) / TB;
    const int base = S.dinv_off[s];
    const double *T = S.dinv + ((size_t)base + k) * (TB * TB);   // T(r, c) at T[c * 64 + r]
    // successors c <= clast are in this cluster (rank me - (c - k)); the later ranks (lower
    // k) of the same supernode receive this block's solution
    const int clast = k + me, last = me + min(k, CHAIN_CL - 1 - me);
    double *ring = csm + wp * CHAIN_SLOT;
    double *xw = csm + NS * CHAIN_WARPS * CHAIN_SLOT + wp * CHAIN_XW_BWD;
    // successor step t = nb - 1 - c (c = nb - 1 first); this warp's columns of block (c, k):
    // element (i, rr) = P[(r0 + w8 + i) m + 64c + rr] at [i * LW + rr]
    auto stage = [&](int t) {
      const int c = nb - 1 - t;
      if (c > k) {
        double *d = ring + (t % NS) * CHAIN_WARPS * CHAIN_SLOT;
        const int cw = min(TB, w - c * TB);
        const double *src = P + (size_t)(r0 + w8) * m + c * TB;
#pragma unroll 4
        for (int u = 0; u < 16; ++u) {
          const int e = lane + 32 * u, i = e >> 6, rr = e & 63;
          const bool in = w8 + i < bw && rr < cw;
          cp8(d + i * LW + rr, in ? src + (size_t)i * m + rr : src, in);
        }
      }
      stage_commit();
    };
    for (int t = 0; t < NS - 1; ++t) stage(t);
    double tr[8][2];   // T(rr, w8 + i) for rr = lane, lane + 32
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      tr[i][0] = T[(size_t)(w8 + i) * TB + lane];
      tr[i][1] = T[(size_t)(w8 + i) * TB + lane + 32];
    }
    double v = (row < bw) ? x[f + r0 + row] : 0.0;
    bool ok = true;
    int xb0 = nb, nbt = 0;               // the batch in xw: blocks xb0, .., xb0 - nbt + 1
    for (int c = nb - 1; c > k; --c) {
      const int t = nb - 1 - c;
      stage(t + NS - 1);
      stage_wait<NS - 1>();              // block (c, k) has landed (this lane's copies)
      __syncwarp();
      const double *Lc = ring + (t % NS) * CHAIN_WARPS * CHAIN_SLOT;
      double lr[8][2];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        lr[i][0] = Lc[i * LW + lane];
        lr[i][1] = Lc[i * LW + lane + 32];
      }
      __syncwarp();
      double x0, x1;
      if (c <= clast) {   // from the cluster
        const int j = me - (c - k);
        if (!warp_chain_recv(cc, j, S.status)) { ok = false; break; }
        x0 = cc.yin[j][lane];
        x1 = cc.yin[j][lane + 32];
      } else {            // from global memory, a batch of blocks c, c - 1, .. at a time
        if (c <= xb0 - nbt) {
          xb0 = c;                         // blocks c, c - 1, .., c - nbt + 1
          nbt = warp_wait_prefix(&flags[base + c], -1, min(CHAIN_XB, c - clast), CHAIN_WARPS * epoch,
                                 S.status);
          if (nbt == 0) { ok = false; break; }
          double t2[CHAIN_XB][2];
#pragma unroll
          for (int u = 0; u < CHAIN_XB; ++u)
            if (u < nbt) {
              const int cu = c - u, cwu = min(TB, w - cu * TB);
              t2[u][0] = lane < cwu ? __ldcg(&x[f + cu * TB + lane]) : 0.0;
              t2[u][1] = lane + 32 < cwu ? __ldcg(&x[f + cu * TB + lane + 32]) : 0.0;
            }
#pragma unroll
          for (int u = 0; u < CHAIN_XB; ++u)
            if (u < nbt) {
              xw[u * TB + lane] = t2[u][0];
              xw[u * TB + lane + 32] = t2[u][1];
            }
        }
        x0 = xw[(xb0 - c) * TB + lane];   // written by this lane
        x1 = xw[(xb0 - c) * TB + lane + 32];
      }
      double a[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) a[i] = fma(lr[i][1], x1, lr[i][0] * x0);
      v -= warp_rows8(a, lane);
    }
    stage_wait<0>();
    if ((lane & 3) == 0) vs[row] = v;
    ok = __syncthreads_and(ok) != 0;
    if (ok) {
      // x_k[i] = sum_rr T(rr, i) v[rr]
      const double x0 = vs[lane], x1 = vs[lane + 32];
      double a[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) a[i] = fma(tr[i][1], x1, tr[i][0] * x0);
      const double xk = warp_rows8(a, lane);
      chain_send(cc, me, last, row, row < bw ? xk : 0.0);
      if ((lane & 3) == 0 && row < bw) x[f + r0 + row] = xk;
      __syncwarp();
      if (lane == 0) red_release_add(&flags[base + k], 1);
    }
  }
  cluster_sync_all();
}

// y = A x for the symmetric matrix held as full CSR (both triangles), nrhs vectors.
__global__ void __launch_bounds__(256) k_spmv(int n, const int *rp, const int *ci,
                                              const double *val, const double *x, double *y,
                                              int nrhs) {
  // eight lanes per row (rows of a stencil matrix hold 7 to 81 entries: a warp per row
  // left most lanes idle), 32 rows per CTA; the eight partial sums meet by shuffles
  const int row = blockIdx.x * 32 + (int)(threadIdx.x >> 3);
  const int sub = threadIdx.x & 7;
  const bool ok = row < n;
  const int p0 = ok ? rp[row] : 0, p1 = ok ? rp[row + 1] : 0;
  for (int r = 0; r < nrhs; ++r) {
    const double *xr = x + (size_t)r * n;
    double acc = 0.0;
    for (int p = p0 + sub; p < p1; p += 8) acc = fma(val[p], xr[ci[p]], acc);
    acc += __shfl_xor_sync(0xffffffffu, acc, 4);
    acc += __shfl_xor_sync(0xffffffffu, acc, 2);
    acc += __shfl_xor_sync(0xffffffffu, acc, 1);
    if (ok && sub == 0) y[(size_t)r * n + row] = acc;
  }
}

// out[i] = sum_j |A(i, j)| (rows of the full CSR)
__global__ void k_rowabs(int n, const int *rp, const double *val, double *out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double acc = 0.0;
  for (int p = rp[i]; p < rp[i + 1]; ++p) acc += fabs(val[p]);
  out[i] = acc;
}

// full-CSR values from the lower-CSC values through the precomputed map
__global__ void k_gather_vals(int nnz, const int *map, const double *ax, double *val) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nnz) val[i] = ax[map[i]];
}

// r = b - r (r holds A x on entry)
__global__ void k_residual(size_t len, const double *b, double *r) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < len) r[i] = b[i] - r[i];
}

// p = z + beta p
__global__ void k_xpby(size_t len, const double *z, double beta, double *p) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < len) p[i] = fma(beta, p[i], z[i]);
}

__global__ void k_axpy(size_t len, double a, const double *x, double *y) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < len) y[i] = fma(a, x[i], y[i]);
}

// per-vector max |x| and sum x*y for nrhs vectors of length n (out[2*r], out[2*r+1]),
// deterministic: NORM_BLOCKS fixed slices per vector, then one CTA per vector sums the
// slices in order.
constexpr int NORM_BLOCKS = 128;
__global__ void k_norms_part(int n, const double *x, const double *y, double *part) {
  __shared__ double smax[ST], sdot[ST];
  const int r = blockIdx.y, b = blockIdx.x;
  const double *xr = x + (size_t)r * n, *yr = y ? y + (size_t)r * n : nullptr;
  const int per = (n + NORM_BLOCKS - 1) / NORM_BLOCKS;
  const int lo = b * per, hi = min(n, lo + per);
  double mx = 0.0, dt = 0.0;
  for (int i = lo + threadIdx.x; i < hi; i += ST) {
    mx = fmax(mx, fabs(xr[i]));
    if (yr) dt = fma(xr[i], yr[i], dt);
  }
  smax[threadIdx.x] = mx;
  sdot[threadIdx.x] = dt;
  __syncthreads();
  for (int o = ST / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      smax[threadIdx.x] = fmax(smax[threadIdx.x], smax[threadIdx.x + o]);
      sdot[threadIdx.x] += sdot[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * ((size_t)r * NORM_BLOCKS + b)] = smax[0];
    part[2 * ((size_t)r * NORM_BLOCKS + b) + 1] = sdot[0];
  }
}
__global__ void k_norms_final(const double *part, double *out) {
  __shared__ double smax[NORM_BLOCKS], sdot[NORM_BLOCKS];
  const int r = blockIdx.x, t = threadIdx.x;
  smax[t] = part[2 * ((size_t)r * NORM_BLOCKS + t)];
  sdot[t] = part[2 * ((size_t)r * NORM_BLOCKS + t) + 1];
  __syncthreads();
  for (int o = NORM_BLOCKS / 2; o > 0; o >>= 1) {
    if (t < o) {
      smax[t] = fmax(smax[t], smax[t + o]);
      sdot[t] += sdot[t + o];
    }
    __syncthreads();
  }
  if (t == 0) {
    out[2 * r] = smax[0];
    out[2 * r + 1] = sdot[0];
  }
}

}  // namespace

// the chains' grids: whole clusters of CHAIN_CL CTAs; launches that fit the SMs at one CTA
// each take the deep ring
static int g_num_sms = 148;
static int chain_grid(int count) { return (count + CHAIN_CL - 1) / CHAIN_CL * CHAIN_CL; }

bool solve_configure(int max_w, std::string &err) {
  size_t smem = sizeof(double) * (size_t)(max_w > 0 ? max_w : 1);
  if (smem > 220 * 1024) {
    err = "supernode too wide for the shared-memory triangular solve";
    return false;
  }
  cudaError_t e = cudaFuncSetAttribute(k_fwd_diag, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_fwd_chain<CHAIN_NS_BIG>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             chain_smem(CHAIN_NS_BIG, CHAIN_XW_FWD));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_fwd_chain<CHAIN_NS_SMALL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             chain_smem(CHAIN_NS_SMALL, CHAIN_XW_FWD));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_bwd_chain<CHAIN_NS_BIG>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             chain_smem(CHAIN_NS_BIG, CHAIN_XW_BWD));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_bwd_chain<CHAIN_NS_SMALL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             chain_smem(CHAIN_NS_SMALL, CHAIN_XW_BWD));
  if (e == cudaSuccess) {
    int dev = 0;
    e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
  }
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_bwd_diag, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) {
    err = std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e);
    return false;
  }
  return true;
}

void launch_fwd_diag(const DevSym &S, const int *list, int count, int smem, double *y,
                     const double *contrib, const int *cptr, const int *cidx, int n, int nrhs,
                     int64_t cstride, cudaStream_t st) {
  if (count > 0)
    k_fwd_diag<<<count, ST, smem, st>>>(S, list, y, contrib, cptr, cidx, n, nrhs, cstride);
}
void launch_fwd_contrib(const DevSym &S, const int2 *tasks, int count, int nbig, int nwide,
                        const double *y, double *contrib, int n, int nrhs, int64_t cstride,
                        cudaStream_t st) {
  if (nbig > 0) k_fwd_contrib_big<<<nbig, CTB, 0, st>>>(S, tasks, y, contrib, n, nrhs, cstride);
  tasks += nbig;
  count -= nbig;
  const int blocks = nwide + (count - nwide + CW - 1) / CW;
  if (count > 0)
    k_fwd_contrib<<<blocks, CT, 0, st>>>(S, tasks, count, nwide, y, contrib, n, nrhs, cstride);
}
void launch_fwd_warp(const DevSym &S, const int *list, int count, double *y, double *contrib,
                     const int *cptr, const int *cidx, int n, int nrhs, int64_t cstride,
                     cudaStream_t st) {
  if (count > 0)
    k_fwd_warp<<<(count + WPC - 1) / WPC, ST, 0, st>>>(S, list, count, y, contrib, cptr, cidx, n,
                                                       nrhs, cstride);
}
void launch_bwd_warp(const DevSym &S, const int *list, int count, double *x, int n, int nrhs,
                     cudaStream_t st) {
  if (count > 0) k_bwd_warp<<<(count + WPC - 1) / WPC, ST, 0, st>>>(S, list, count, x, n, nrhs);
}
void launch_bwd_gather(const DevSym &S, const int2 *tasks, int count, double *x, int n, int nrhs,
                       cudaStream_t st) {
  if (count > 0) k_bwd_gather<<<count, GT, 0, st>>>(S, tasks, x, n, nrhs);
}
void launch_bwd_diag(const DevSym &S, const int *list, int count, int smem, double *x, int n,
                     int nrhs, cudaStream_t st) {
  if (count > 0) k_bwd_diag<<<count, ST, smem, st>>>(S, list, x, n, nrhs);
}
// the chains' launch configuration: a grid of whole clusters of CHAIN_CL CTAs
static cudaLaunchConfig_t chain_config(int count, int smem, cudaStream_t st,
                                       cudaLaunchAttribute *at) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)chain_grid(count));
  cfg.blockDim = dim3(ST);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = CHAIN_CL;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cfg;
}
void launch_fwd_chain(const DevSym &S, const int2 *tasks, int count, double *y,
                      const double *contrib, const int *cptr, const int *cidx, int *flags,
                      int epoch, int n, int64_t cstride, cudaStream_t st) {
  if (count <= 0) return;
  cudaLaunchAttribute at[1];
  if (chain_grid(count) <= g_num_sms) {
    const cudaLaunchConfig_t cfg = chain_config(count, chain_smem(CHAIN_NS_BIG, CHAIN_XW_FWD), st, at);
    cudaLaunchKernelEx(&cfg, k_fwd_chain<CHAIN_NS_BIG>, S, tasks, count, y, contrib, cptr, cidx,
                       flags, epoch, n, cstride);
  } else {
    const cudaLaunchConfig_t cfg = chain_config(count, chain_smem(CHAIN_NS_SMALL, CHAIN_XW_FWD), st, at);
    cudaLaunchKernelEx(&cfg, k_fwd_chain<CHAIN_NS_SMALL>, S, tasks, count, y, contrib, cptr, cidx,
                       flags, epoch, n, cstride);
  }
}
void launch_bwd_chain(const DevSym &S, const int2 *tasks, int count, double *x, int *flags,
                      int epoch, cudaStream_t st) {
  if (count <= 0) return;
  cudaLaunchAttribute at[1];
  if (chain_grid(count) <= g_num_sms) {
    const cudaLaunchConfig_t cfg = chain_config(count, chain_smem(CHAIN_NS_BIG, CHAIN_XW_BWD), st, at);
    cudaLaunchKernelEx(&cfg, k_bwd_chain<CHAIN_NS_BIG>, S, tasks, count, x, flags, epoch);
  } else {
    const cudaLaunchConfig_t cfg = chain_config(count, chain_smem(CHAIN_NS_SMALL, CHAIN_XW_BWD), st, at);
    cudaLaunchKernelEx(&cfg, k_bwd_chain<CHAIN_NS_SMALL>, S, tasks, count, x, flags, epoch);
  }
}
void launch_spmv(int n, const int *rp, const int *ci, const double *val, const double *x,
                 double *y, int nrhs, cudaStream_t st) {
  k_spmv<<<(n + 31) / 32, 256, 0, st>>>(n, rp, ci, val, x, y, nrhs);
}
void launch_gather_vals(int nnz, const int *map, const double *ax, double *val, cudaStream_t st) {
  if (nnz > 0) k_gather_vals<<<(nnz + 255) / 256, 256, 0, st>>>(nnz, map, ax, val);
}
void launch_rowabs(int n, const int *rp, const double *val, double *out, cudaStream_t st) {
  k_rowabs<<<(n + 255) / 256, 256, 0, st>>>(n, rp, val, out);
}
void launch_residual(size_t len, const double *b, double *r, cudaStream_t st) {
  if (len) k_residual<<<(unsigned)((len + 255) / 256), 256, 0, st>>>(len, b, r);
}
void launch_xpby(size_t len, const double *z, double beta, double *p, cudaStream_t st) {
  if (len) k_xpby<<<(unsigned)((len + 255) / 256), 256, 0, st>>>(len, z, beta, p);
}
void launch_axpy(size_t len, double a, const double *x, double *y, cudaStream_t st) {
  if (len) k_axpy<<<(unsigned)((len + 255) / 256), 256, 0, st>>>(len, a, x, y);
}
void launch_norms(int n, int nrhs, const double *x, const double *y, double *out, double *part,
                  cudaStream_t st) {
  k_norms_part<<<dim3(NORM_BLOCKS, nrhs), ST, 0, st>>>(n, x, y, part);
  k_norms_final<<<nrhs, NORM_BLOCKS, 0, st>>>(part, out);
}
int norm_scratch_doubles(int nrhs) { return 2 * NORM_BLOCKS * nrhs; }

}  // namespace swc
