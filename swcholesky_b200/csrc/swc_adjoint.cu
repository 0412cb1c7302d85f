// Adjoint of the supernodal factorization: gradients with respect to the stored nonzeros of
// A (the lower triangle of P A P^T, symmetric storage: a stored off-diagonal value stands
// for both A_ij and A_ji).
//
// log det A.  d log det A = tr(A^{-1} dA), so the gradient is A^{-1} on the pattern of A,
// times 2 off the diagonal.  A^{-1} is computed on the whole pattern of L (the selected
// inverse Z) by a reverse sweep over the elimination tree, root to leaves, that retraces the
// factorization's POTRF / TRSM / SYRK steps backwards.  Per column block K of a supernode
// (at most 64 columns; a wide supernode is a chain of such blocks) with the rows R of L
// below it:
//     U    = L_RK L_KK^{-1}                  recomputed from L (the factorization stores no
//                                            intermediate panels)
//     Z_RK = -Z_RR U                         Z_RR: symmetric, gathered from the ancestors
//     Z_KK = L_KK^{-T} L_KK^{-1} - U^T Z_RK
// (Takahashi, Fagan and Chin, 1973; the supernodal form of the reverse-mode Cholesky of
// Murray, "Differentiation of the Cholesky decomposition", 2016).  Z_RR is inside the
// ancestors' stored pattern: for rows i >= j of R, row i belongs to the row list of the
// supernode holding column j (row lists are closed under the elimination).  Its entries are
// located through position tables built once per structure: for every off-diagonal row run
// of a supernode that falls into one ancestor (a "segment"), the positions of the
// supernode's later rows in that ancestor's row list.
//
// Functions of x = A^{-1} b.  With lam = A^{-1} (df/dx):
//     df/dA_ij = -(lam_i x_j + lam_j x_i)  (i != j),   -lam_i x_i  (i == j).
//
// The reference has no adjoint; this is a new capability of the library.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <string>
#include <type_traits>
#include <vector>

#include "swc_engine.h"

namespace swc {

namespace {

constexpr int AT = 256;       // threads of the tile kernels (4x4 register micro-tiles)
constexpr int AKC = 16;       // rows of R per gathered chunk
constexpr int ALD = TB + 1;   // padded row of a 64-wide shared tile
constexpr int64_t OWN = INT64_MIN;  // location code: the row belongs to the unit's own supernode

struct AdjDev {
  const int4 *units;         // (supernode J, first column offset c0, width w, off = c0 + w)
  const int64_t *tinv_off;   // per unit: offset of its w x w inverse in tinv
  const int2 *tasks;         // (unit, x0): 64-row block of R starting at R index x0
  const int *rowseg;         // per Ls position of an off-diagonal row: its segment
  const int *seg_t;          // segment: first off-diagonal row index inside its supernode
  const int *seg_S;          //          ancestor supernode holding the segment's columns
  const int64_t *seg_tbl;    //          offset of its position list in tbl
  const int *tbl;            // positions in the ancestor's row list
  double *Z;                 // selected inverse, same layout as L
  double *U;                 // L_RK L_KK^{-1}, same layout as L
  double *tinv;              // L_KK^{-1} per unit, column-major w x w
  double *P;                 // per task of the current wave: U(X,:)^T (Z_RR U)(X,:), 64 x 64
};

__device__ __forceinline__ int lbound_a(const int *a, int len, int key) {
  int lo = 0, hi = len;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (a[mid] < key) lo = mid + 1; else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ int nrows_of(const DevSym &S, int s) {
  return (int)(S.rowptr[s + 1] - S.rowptr[s]);
}

// L_KK^{-1} of every unit (one CTA of 64 threads per unit; thread c forms column c by
// forward substitution, all threads walking the rows in lock step).
constexpr int TINV_SMEM = 2 * TB * ALD * 8 + TB * 8;
__global__ void __launch_bounds__(TB) k_adj_tinv(DevSym S, AdjDev A) {
  extern __shared__ double sm[];
  double *T = sm, *X = sm + TB * ALD, *rd = X + TB * ALD;
  const int4 u = A.units[blockIdx.x];
  const int J = u.x, c0 = u.y, w = u.z;
  const int ns = nrows_of(S, J);
  const double *Lb = S.L + S.xptr[J] + (size_t)c0 * ns + c0;
  const int c = threadIdx.x;
  for (int idx = c; idx < w * w; idx += TB) {
    const int col = idx / w, row = idx - col * w;
    T[row * ALD + col] = row >= col ? Lb[(size_t)col * ns + row] : 0.0;
  }
  __syncthreads();
  if (c < w) rd[c] = 1.0 / T[c * ALD + c];
  __syncthreads();
  if (c < w) {
    for (int i = 0; i < w; ++i) {
      double acc = (i == c) ? 1.0 : 0.0;
      for (int k = c; k < i; ++k) acc -= T[i * ALD + k] * X[k * ALD + c];
      X[i * ALD + c] = i >= c ? acc * rd[i] : 0.0;
    }
  }
  __syncthreads();
  double *out = A.tinv + A.tinv_off[blockIdx.x];
  for (int idx = c; idx < w * w; idx += TB) {
    const int col = idx / w, row = idx - col * w;
    out[idx] = X[row * ALD + col];
  }
}

// U(X, :) = L_RK(X, :) L_KK^{-1} for one 64-row block X of R.
constexpr int U_SMEM = 2 * TB * ALD * 8;
__global__ void __launch_bounds__(AT) k_adj_u(DevSym S, AdjDev A, const int2 *tasks) {
  extern __shared__ double sm[];
  double *Lx = sm, *Ti = sm + TB * ALD;
  const int2 tk = tasks[blockIdx.x];
  const int4 u = A.units[tk.x];
  const int J = u.x, c0 = u.y, w = u.z, off = u.w;
  const int ns = nrows_of(S, J);
  const int m = ns - off, x0 = tk.y;
  const int nrow = min(TB, m - x0);
  const size_t base = S.xptr[J] + (size_t)c0 * ns + off + x0;
  const double *ti = A.tinv + A.tinv_off[tk.x];
  for (int idx = threadIdx.x; idx < TB * TB; idx += AT) {
    const int col = idx >> 6, row = idx & (TB - 1);
    Lx[row * ALD + col] = (row < nrow && col < w) ? S.L[base + (size_t)col * ns + row] : 0.0;
    Ti[row * ALD + col] = (row < w && col < w) ? ti[col * w + row] : 0.0;
  }
  __syncthreads();
  const int r0 = (threadIdx.x >> 4) * 4, cc0 = (threadIdx.x & 15) * 4;
  double acc[4][4] = {};
  for (int k = 0; k < w; ++k) {
    double a[4], b[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) a[i] = Lx[(r0 + i) * ALD + k];
#pragma unroll
    for (int j = 0; j < 4; ++j) b[j] = Ti[k * ALD + cc0 + j];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (r0 + i < nrow && cc0 + j < w) A.U[base + (size_t)(cc0 + j) * ns + r0 + i] = acc[i][j];
}

// Location of column j of Z_RR (j: index into R = rows off.. of J's row list, as the
// smaller index of a lower-triangle entry): the column's base offset in Z and the code that
// turns the row index i into a position (OWN: position off + i in J's list; else an offset
// into tbl).
__device__ __forceinline__ void locate(const DevSym &S, const AdjDev &A, int J, int off, int own,
                                       int ns, int j, int64_t &cb, int64_t &to) {
  if (j < own) {
    cb = S.xptr[J] + (int64_t)(off + j) * ns;
    to = OWN;
  } else {
    const int64_t q = S.rowptr[J] + off + j;
    const int sg = A.rowseg[q];
    const int Sa = A.seg_S[sg];
    cb = S.xptr[Sa] + (int64_t)(S.Ls[q] - S.super[Sa]) * nrows_of(S, Sa);
    to = A.seg_tbl[sg] - A.seg_t[sg] - own;
  }
}

// Z_RK(X, :) = -(Z_RR U)(X, :) for one 64-row block X of R, and the block's share of
// U^T Z_RR U (for Z_KK), written to the wave's P scratch.
constexpr int ZRK_SMEM = 2 * TB * 8 + 2 * AKC * 8 + TB * (AKC + 1) * 8 + AKC * ALD * 8 +
                         2 * TB * ALD * 8;
__global__ void __launch_bounds__(AT) k_adj_zrk(DevSym S, AdjDev A, const int2 *tasks) {
  extern __shared__ double sm[];
  int64_t *xcb = reinterpret_cast<int64_t *>(sm), *xto = xcb + TB;
  int64_t *bcb = xto + TB, *bto = bcb + AKC;
  double *zt = reinterpret_cast<double *>(bto + AKC);   // [x][b], ld AKC + 1
  double *uc = zt + TB * (AKC + 1);                      // [b][c], ld ALD
  double *ys = uc + AKC * ALD, *ux = ys + TB * ALD;      // [x][c], ld ALD
  const int2 tk = tasks[blockIdx.x];
  const int4 u = A.units[tk.x];
  const int J = u.x, c0 = u.y, w = u.z, off = u.w;
  const int ns = nrows_of(S, J);
  const int wJ = S.super[J + 1] - S.super[J];
  const int own = wJ - off;
  const int m = ns - off, x0 = tk.y;
  const int nrow = min(TB, m - x0);
  const size_t ubase = S.xptr[J] + (size_t)c0 * ns + off;   // + col * ns + R index
  const int tid = threadIdx.x;
  if (tid < TB && tid < nrow) locate(S, A, J, off, own, ns, x0 + tid, xcb[tid], xto[tid]);
  const int r0 = (tid >> 4) * 4, cc0 = (tid & 15) * 4;
  double acc[4][4] = {};
  for (int b0 = 0; b0 < m; b0 += AKC) {
    __syncthreads();
    if (tid < AKC && b0 + tid < m) locate(S, A, J, off, own, ns, b0 + tid, bcb[tid], bto[tid]);
    for (int idx = tid; idx < AKC * TB; idx += AT) {
      const int b = idx >> 6, c = idx & (TB - 1);
      uc[b * ALD + c] = (b0 + b < m && c < w) ? A.U[ubase + (size_t)c * ns + b0 + b] : 0.0;
    }
    __syncthreads();
    for (int idx = tid; idx < AKC * TB; idx += AT) {
      const int b = idx >> 6, x = idx & (TB - 1);
      const int ix = x0 + x, ib = b0 + b;
      double v = 0.0;
      if (x < nrow && ib < m) {
        int64_t cb, to;
        int i;
        if (ix >= ib) { cb = bcb[b]; to = bto[b]; i = ix; }
        else { cb = xcb[x]; to = xto[x]; i = ib; }
        const int64_t pos = (to == OWN) ? (int64_t)(off + i) : (int64_t)A.tbl[to + i];
        v = A.Z[cb + pos];
      }
      zt[x * (AKC + 1) + b] = v;
    }
    __syncthreads();
#pragma unroll
    for (int b = 0; b < AKC; ++b) {
      double a[4], bb[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = zt[(r0 + i) * (AKC + 1) + b];
#pragma unroll
      for (int j = 0; j < 4; ++j) bb[j] = uc[b * ALD + cc0 + j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], bb[j], acc[i][j]);
    }
  }
  // Z_RK(X, :) = -Y; stage Y and U(X, :) for the Z_KK share
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int r = r0 + i, c = cc0 + j;
      const bool ok = r < nrow && c < w;
      if (ok) A.Z[ubase + (size_t)c * ns + x0 + r] = -acc[i][j];
      ys[r * ALD + c] = ok ? acc[i][j] : 0.0;
    }
  for (int idx = tid; idx < TB * TB; idx += AT) {
    const int c = idx >> 6, r = idx & (TB - 1);
    ux[r * ALD + c] = (r < nrow && c < w) ? A.U[ubase + (size_t)c * ns + x0 + r] : 0.0;
  }
  __syncthreads();
  double p[4][4] = {};
  for (int r = 0; r < nrow; ++r) {
    double a[4], bb[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) a[i] = ux[r * ALD + r0 + i];
#pragma unroll
    for (int j = 0; j < 4; ++j) bb[j] = ys[r * ALD + cc0 + j];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) p[i][j] = fma(a[i], bb[j], p[i][j]);
  }
  double *P = A.P + (size_t)blockIdx.x * TB * TB;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) P[(size_t)(cc0 + j) * TB + r0 + i] = p[i][j];
}

// Z_KK = L_KK^{-T} L_KK^{-1} + sum over the unit's row blocks of U^T Z_RR U (lower part).
constexpr int ZKK_SMEM = TB * ALD * 8;
__global__ void __launch_bounds__(AT) k_adj_zkk(DevSym S, AdjDev A, const int *wave_units,
                                                const int *ut_begin, const int *ut_end,
                                                int task_base) {
  extern __shared__ double sm[];
  double *Ti = sm;
  const int ui = wave_units[blockIdx.x];
  const int4 u = A.units[ui];
  const int J = u.x, c0 = u.y, w = u.z;
  const int ns = nrows_of(S, J);
  const double *ti = A.tinv + A.tinv_off[ui];
  for (int idx = threadIdx.x; idx < TB * TB; idx += AT) {
    const int col = idx >> 6, row = idx & (TB - 1);
    Ti[row * ALD + col] = (row < w && col < w) ? ti[col * w + row] : 0.0;
  }
  __syncthreads();
  const int r0 = (threadIdx.x >> 4) * 4, cc0 = (threadIdx.x & 15) * 4;
  double acc[4][4] = {};
  for (int k = 0; k < w; ++k) {
    double a[4], b[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) a[i] = Ti[k * ALD + r0 + i];
#pragma unroll
    for (int j = 0; j < 4; ++j) b[j] = Ti[k * ALD + cc0 + j];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
  }
  for (int t = ut_begin[ui]; t < ut_end[ui]; ++t) {
    const double *P = A.P + (size_t)(t - task_base) * TB * TB;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[i][j] += P[(size_t)(cc0 + j) * TB + r0 + i];
  }
  double *Zb = A.Z + S.xptr[J] + (size_t)c0 * ns + c0;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int r = r0 + i, c = cc0 + j;
      if (r < w && c < w && r >= c) Zb[(size_t)c * ns + r] = acc[i][j];
    }
}

// Supernode holding column j.
__device__ __forceinline__ int snode_of(const DevSym &S, int j) {
  int lo = 0, hi = S.nsuper;   // last s with super[s] <= j
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (S.super[mid] <= j) lo = mid; else hi = mid;
  }
  return lo;
}

// Partial sums of log L_jj (fixed grid, fixed order: deterministic).
constexpr int LD_BLOCKS = 256;
__global__ void __launch_bounds__(256) k_logdet(DevSym S, double *partial) {
  __shared__ double red[256];
  double acc = 0.0;
  for (int j = blockIdx.x * 256 + threadIdx.x; j < S.n; j += LD_BLOCKS * 256) {
    const int s = snode_of(S, j);
    const int c = j - S.super[s];
    acc += log(S.L[S.xptr[s] + (size_t)c * nrows_of(S, s) + c]);
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

// grad[p] = d log det A / d Ax[p] = Z_ij (2 - delta_ij); one warp per column.
__global__ void k_logdet_grad(DevSym S, const double *Z, double *grad) {
  const int j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (j >= S.n) return;
  const int s = snode_of(S, j);
  const int64_t rb = S.rowptr[s];
  const int m = (int)(S.rowptr[s + 1] - rb);
  const double *col = Z + S.xptr[s] + (size_t)(j - S.super[s]) * m;
  for (int p = S.Ap[j] + lane; p < S.Ap[j + 1]; p += 32) {
    const int i = S.Ai[p];
    const int pos = lbound_a(S.Ls + rb, m, i);
    grad[p] = (pos < m && S.Ls[rb + pos] == i) ? col[pos] * (i == j ? 1.0 : 2.0) : 0.0;
    if (!(pos < m && S.Ls[rb + pos] == i)) atomicExch(&S.status[1], 1);
  }
}

// grad[p] = -(lam_i x_j + lam_j x_i) for i != j, -lam_i x_i on the diagonal.
__global__ void k_solve_grad(DevSym S, const double *x, const double *lam, double *grad) {
  const int j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (j >= S.n) return;
  const double xj = x[j], lj = lam[j];
  for (int p = S.Ap[j] + lane; p < S.Ap[j + 1]; p += 32) {
    const int i = S.Ai[p];
    grad[p] = (i == j) ? -lam[i] * xj : -(lam[i] * xj + lj * x[i]);
  }
}

}  // namespace

// ---------------------------------------------------------------------------------------

struct AdjointPlan {
  bool ready = false;
  std::vector<int4> units;
  std::vector<int64_t> tinv_off;
  std::vector<int> wave_unit_off, wave_units;   // units of wave v (root side first)
  std::vector<int> wave_task_off;
  std::vector<int2> tasks;                      // grouped by wave
  std::vector<int> ut_begin, ut_end;            // per unit: its tasks
  int max_wave_tasks = 0;
  std::vector<int> rowseg, seg_t, seg_S, tbl;
  std::vector<int64_t> seg_tbl;
};

bool Engine::prepare_adjoint(std::string &err) {
  if (adj_ && adj_->ready) return true;
  if (!adj_) adj_.reset(new AdjointPlan);
  AdjointPlan &AP = *adj_;
  const std::vector<int> &super = hsym_.super;
  const std::vector<int64_t> &rowptr = hsym_.rowptr;
  const int ns_ = nsuper_;
  std::vector<int> col2sup(n_);
  for (int s = 0; s < ns_; ++s)
    for (int j = super[s]; j < super[s + 1]; ++j) col2sup[j] = s;
  // segments and position tables
  AP.rowseg.assign(h_Ls_.size(), -1);
  for (int J = 0; J < ns_; ++J) {
    const int wJ = super[J + 1] - super[J];
    const int64_t rb = rowptr[J], re = rowptr[J + 1];
    int64_t q = rb + wJ;
    while (q < re) {
      const int Sa = col2sup[h_Ls_[q]];
      int64_t qe = q;
      while (qe < re && col2sup[h_Ls_[qe]] == Sa) ++qe;
      const int sg = (int)AP.seg_t.size();
      AP.seg_t.push_back((int)(q - rb - wJ));
      AP.seg_S.push_back(Sa);
      AP.seg_tbl.push_back((int64_t)AP.tbl.size());
      const int *ls = h_Ls_.data() + rowptr[Sa];
      const int lsn = (int)(rowptr[Sa + 1] - rowptr[Sa]);
      int pos = 0;
      for (int64_t t = q; t < re; ++t) {
        pos = (int)(std::lower_bound(ls + pos, ls + lsn, h_Ls_[t]) - ls);
        if (pos >= lsn || ls[pos] != h_Ls_[t]) {
          err = "adjoint: row list not closed under the elimination (invalid structure)";
          return false;
        }
        AP.tbl.push_back(pos);
      }
      for (int64_t t = q; t < qe; ++t) AP.rowseg[t] = sg;
      q = qe;
    }
  }
  // units (64-column blocks) and their levels, root side first
  std::vector<int> ufirst(ns_ + 1, 0);
  for (int J = 0; J < ns_; ++J) ufirst[J + 1] = ufirst[J] + (super[J + 1] - super[J] + TB - 1) / TB;
  const int nunits = ufirst[ns_];
  AP.units.resize(nunits);
  AP.tinv_off.assign(nunits + 1, 0);
  std::vector<int> ulev(nunits), top(ns_);
  int nlev = 0;
  for (int J = ns_ - 1; J >= 0; --J) {
    const int wJ = super[J + 1] - super[J];
    const int64_t m = rowptr[J + 1] - rowptr[J];
    const int nb = ufirst[J + 1] - ufirst[J];
    int t = 0;
    if (m > wJ) {
      const int p = col2sup[h_Ls_[rowptr[J] + wJ]];
      t = top[p] + (ufirst[p + 1] - ufirst[p]);   // one past the parent's last unit level
    }
    top[J] = t;
    for (int b = 0; b < nb; ++b) {
      const int c0 = b * TB, w = std::min(TB, wJ - c0);
      const int u = ufirst[J] + b;
      AP.units[u] = make_int4(J, c0, w, c0 + w);
      ulev[u] = t + (nb - 1 - b);
      nlev = std::max(nlev, ulev[u] + 1);
    }
  }
  for (int u = 0; u < nunits; ++u)
    AP.tinv_off[u + 1] = AP.tinv_off[u] + (int64_t)AP.units[u].z * AP.units[u].z;
  std::vector<std::vector<int>> bylev(nlev);
  for (int u = 0; u < nunits; ++u) bylev[ulev[u]].push_back(u);
  AP.ut_begin.assign(nunits, 0);
  AP.ut_end.assign(nunits, 0);
  AP.wave_unit_off.clear();
  AP.wave_units.clear();
  AP.wave_task_off.clear();
  AP.tasks.clear();
  AP.max_wave_tasks = 0;
  for (int l = 0; l < nlev; ++l) {
    AP.wave_unit_off.push_back((int)AP.wave_units.size());
    AP.wave_task_off.push_back((int)AP.tasks.size());
    for (int u : bylev[l]) {
      AP.wave_units.push_back(u);
      const int J = AP.units[u].x;
      const int m = (int)(rowptr[J + 1] - rowptr[J]) - AP.units[u].w;
      AP.ut_begin[u] = (int)AP.tasks.size();
      for (int x0 = 0; x0 < m; x0 += TB) AP.tasks.push_back(make_int2(u, x0));
      AP.ut_end[u] = (int)AP.tasks.size();
    }
    AP.max_wave_tasks = std::max(AP.max_wave_tasks, (int)AP.tasks.size() - AP.wave_task_off.back());
  }
  AP.wave_unit_off.push_back((int)AP.wave_units.size());
  AP.wave_task_off.push_back((int)AP.tasks.size());
  // device copies and scratch
  cudaStream_t st = stream_;
  cudaError_t e = cudaSuccess;
  auto up = [&](auto *&dst, const auto &v) {
    using T = typename std::remove_reference<decltype(v[0])>::type;
    if (e != cudaSuccess) return;
    e = cudaMalloc(&dst, sizeof(T) * std::max<size_t>(v.size(), 1));
    if (e == cudaSuccess && !v.empty())
      e = cudaMemcpyAsync(dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, st);
  };
  up(d_adj_units_, AP.units);
  up(d_adj_tinv_off_, AP.tinv_off);
  up(d_adj_tasks_, AP.tasks);
  up(d_adj_wave_units_, AP.wave_units);
  up(d_adj_ut_begin_, AP.ut_begin);
  up(d_adj_ut_end_, AP.ut_end);
  up(d_adj_rowseg_, AP.rowseg);
  up(d_adj_seg_t_, AP.seg_t);
  up(d_adj_seg_S_, AP.seg_S);
  up(d_adj_seg_tbl_, AP.seg_tbl);
  up(d_adj_tbl_, AP.tbl);
  if (e == cudaSuccess) e = cudaMalloc(&d_adj_Z_, sizeof(double) * std::max<int64_t>(xsize_, 1));
  if (e == cudaSuccess) e = cudaMalloc(&d_adj_U_, sizeof(double) * std::max<int64_t>(xsize_, 1));
  if (e == cudaSuccess)
    e = cudaMalloc(&d_adj_tinv_, sizeof(double) * std::max<int64_t>(AP.tinv_off[nunits], 1));
  if (e == cudaSuccess)
    e = cudaMalloc(&d_adj_P_, sizeof(double) * TB * TB * std::max(AP.max_wave_tasks, 1));
  if (e == cudaSuccess) e = cudaMalloc(&d_adj_partial_, sizeof(double) * LD_BLOCKS);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_adj_tinv, cudaFuncAttributeMaxDynamicSharedMemorySize, TINV_SMEM);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_adj_u, cudaFuncAttributeMaxDynamicSharedMemorySize, U_SMEM);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_adj_zrk, cudaFuncAttributeMaxDynamicSharedMemorySize, ZRK_SMEM);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_adj_zkk, cudaFuncAttributeMaxDynamicSharedMemorySize, ZKK_SMEM);
  if (e != cudaSuccess) {
    err = std::string("adjoint setup: ") + cudaGetErrorString(e);
    return false;
  }
  AP.ready = true;
  return true;
}

void Engine::release_adjoint() {
  void *bufs[] = {d_adj_units_, d_adj_tinv_off_, d_adj_tasks_, d_adj_wave_units_, d_adj_ut_begin_,
                  d_adj_ut_end_, d_adj_rowseg_, d_adj_seg_t_, d_adj_seg_S_, d_adj_seg_tbl_,
                  d_adj_tbl_, d_adj_Z_, d_adj_U_, d_adj_tinv_, d_adj_P_, d_adj_partial_};
  for (void *p : bufs)
    if (p) cudaFree(p);
  d_adj_units_ = nullptr;
  d_adj_tinv_off_ = nullptr;
  d_adj_tasks_ = nullptr;
  d_adj_wave_units_ = d_adj_ut_begin_ = d_adj_ut_end_ = d_adj_rowseg_ = nullptr;
  d_adj_seg_t_ = d_adj_seg_S_ = d_adj_tbl_ = nullptr;
  d_adj_seg_tbl_ = nullptr;
  d_adj_Z_ = d_adj_U_ = d_adj_tinv_ = d_adj_P_ = d_adj_partial_ = nullptr;
  adj_.reset();
}

bool Engine::logdet(double *out, std::string &err) {
  cudaSetDevice(device_);
  if (!prepare_adjoint(err)) return false;
  k_logdet<<<LD_BLOCKS, 256, 0, stream_>>>(sym_, d_adj_partial_);
  double part[LD_BLOCKS];
  cudaError_t e = cudaMemcpyAsync(part, d_adj_partial_, sizeof(part), cudaMemcpyDeviceToHost, stream_);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
  if (e != cudaSuccess) {
    err = std::string("logdet: ") + cudaGetErrorString(e);
    return false;
  }
  double s = 0.0;
  for (int i = 0; i < LD_BLOCKS; ++i) s += part[i];
  *out = 2.0 * s;
  return true;
}

bool Engine::selected_inverse(std::string &err) {
  cudaSetDevice(device_);
  if (!prepare_adjoint(err)) return false;
  const AdjointPlan &AP = *adj_;
  AdjDev A;
  A.units = d_adj_units_;
  A.tinv_off = d_adj_tinv_off_;
  A.tasks = d_adj_tasks_;
  A.rowseg = d_adj_rowseg_;
  A.seg_t = d_adj_seg_t_;
  A.seg_S = d_adj_seg_S_;
  A.seg_tbl = d_adj_seg_tbl_;
  A.tbl = d_adj_tbl_;
  A.Z = d_adj_Z_;
  A.U = d_adj_U_;
  A.tinv = d_adj_tinv_;
  A.P = d_adj_P_;
  cudaStream_t st = stream_;
  cudaMemsetAsync(d_adj_Z_, 0, sizeof(double) * xsize_, st);
  const int nunits = (int)AP.units.size();
  if (nunits > 0) k_adj_tinv<<<nunits, TB, TINV_SMEM, st>>>(sym_, A);
  const int nw = (int)AP.wave_unit_off.size() - 1;
  for (int v = 0; v < nw; ++v) {
    const int t0 = AP.wave_task_off[v], nt = AP.wave_task_off[v + 1] - t0;
    const int u0 = AP.wave_unit_off[v], nu = AP.wave_unit_off[v + 1] - u0;
    if (nt > 0) {
      k_adj_u<<<nt, AT, U_SMEM, st>>>(sym_, A, d_adj_tasks_ + t0);
      k_adj_zrk<<<nt, AT, ZRK_SMEM, st>>>(sym_, A, d_adj_tasks_ + t0);
    }
    if (nu > 0)
      k_adj_zkk<<<nu, AT, ZKK_SMEM, st>>>(sym_, A, d_adj_wave_units_ + u0, d_adj_ut_begin_,
                                          d_adj_ut_end_, t0);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    err = std::string("adjoint sweep: ") + cudaGetErrorString(e);
    return false;
  }
  return true;
}

bool Engine::logdet_grad(double *grad, std::string &err) {
  if (!selected_inverse(err)) return false;
  cudaStream_t st = stream_;
  cudaMemsetAsync(d_status_ + 1, 0, sizeof(int), st);
  const int blocks = (int)(((int64_t)n_ * 32 + 255) / 256);
  k_logdet_grad<<<blocks, 256, 0, st>>>(sym_, d_adj_Z_, grad);
  int flag = 0;
  cudaError_t e = cudaMemcpyAsync(&flag, d_status_ + 1, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    err = std::string("logdet gradient: ") + cudaGetErrorString(e);
    return false;
  }
  if (flag) {
    err = "logdet gradient: a nonzero of A is outside the pattern of L";
    return false;
  }
  return true;
}

bool Engine::solve_grad(const double *x, const double *lam, double *grad, std::string &err) {
  cudaSetDevice(device_);
  const int blocks = (int)(((int64_t)n_ * 32 + 255) / 256);
  k_solve_grad<<<blocks, 256, 0, stream_>>>(sym_, x, lam, grad);
  cudaError_t e = cudaStreamSynchronize(stream_);
  if (e != cudaSuccess) {
    err = std::string("solve gradient: ") + cudaGetErrorString(e);
    return false;
  }
  return true;
}

}  // namespace swc
