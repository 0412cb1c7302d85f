// Engine: validates and uploads the symbolic structure, derives the level schedule and
// the task lists of every kernel, and runs the factorization on one CUDA stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstring>

#include "swc_engine.h"

namespace swc {

namespace {

template <typename T>
bool upload(T *&dst, const T *src, size_t count, cudaStream_t st, std::string &err) {
  if (dst) { cudaFree(dst); dst = nullptr; }
  size_t bytes = sizeof(T) * std::max<size_t>(count, 1);
  cudaError_t e = cudaMalloc(&dst, bytes);
  if (e == cudaSuccess && count) e = cudaMemcpyAsync(dst, src, sizeof(T) * count, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) {
    err = std::string("device upload: ") + cudaGetErrorString(e);
    return false;
  }
  return true;
}

bool small_class(int w, int64_t m) {
  return w <= SMALL_MAX_W && m <= SMALL_MAX_M && (int64_t)w * m <= SMALL_MAX_ELEMS;
}

}  // namespace

Engine::Engine(int device) : device_(device) {
  cudaSetDevice(device_);
  cudaStreamCreateWithFlags(&own_stream_, cudaStreamNonBlocking);
  stream_ = own_stream_;
  cudaMallocHost(&h_status_, 2 * sizeof(int));
}

Engine::~Engine() {
  release();
  if (h_status_) cudaFreeHost(h_status_);
  if (own_stream_) cudaStreamDestroy(own_stream_);
}

void Engine::release() {
  void *ptrs[] = {d_super_, d_Ls_, d_Ap_, d_Ai_, d_rowptr_, d_xptr_, d_upd_ptr_, d_upd_,
                  d_Ax_, dL_, d_status_, d_small_, d_big_, d_asm_, d_panel_, d_upd_tasks_,
                  d_syrk_};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  d_super_ = d_Ls_ = d_Ap_ = d_Ai_ = nullptr;
  d_rowptr_ = d_xptr_ = nullptr;
  d_upd_ptr_ = d_upd_ = nullptr;
  d_Ax_ = dL_ = nullptr;
  d_status_ = d_small_ = d_big_ = nullptr;
  d_asm_ = d_panel_ = nullptr;
  d_upd_tasks_ = d_syrk_ = nullptr;
}

bool Engine::analyze(int n, const int *c, const int *r, const int64_t *lC, const int *Ls,
                     const int64_t *Li_ptr, const int *blockSet, int supNo,
                     const int *prunePtr, const int *pruneSet, std::string &err) {
  cudaSetDevice(device_);
  if (!kernels_configure(err)) return false;
  // ---- host-side validation of the symbolic arrays (no device work on bad input) ----
  if (n <= 0 || supNo <= 0 || !c || !r || !lC || !Ls || !Li_ptr || !blockSet || !prunePtr ||
      !pruneSet) {
    err = "null or empty symbolic input";
    return false;
  }
  if (blockSet[0] != 0 || blockSet[supNo] != n) {
    err = "blockSet must start at 0 and end at n";
    return false;
  }
  std::vector<int> super(blockSet, blockSet + supNo + 1);
  std::vector<int64_t> rowptr(supNo + 1), xptr(supNo);
  for (int s = 0; s < supNo; ++s) {
    int f = super[s], l = super[s + 1];
    if (l <= f) { err = "blockSet must be strictly increasing"; return false; }
    int64_t m = Li_ptr[l] - Li_ptr[f];
    if (m < l - f) { err = "supernode has fewer rows than columns"; return false; }
    for (int j = f; j < l; ++j) {
      if (Li_ptr[j] != Li_ptr[f] || lC[j + 1] - lC[j] != m) {
        err = "Li_ptr / lC are not a supernodal layout";
        return false;
      }
    }
    rowptr[s] = Li_ptr[f];
    xptr[s] = lC[f];
    for (int64_t q = Li_ptr[f]; q < Li_ptr[l]; ++q) {
      int64_t k = q - Li_ptr[f];
      if (Ls[q] < 0 || Ls[q] >= n || (k < l - f && Ls[q] != f + k) ||
          (k > 0 && Ls[q] <= Ls[q - 1])) {
        err = "row list of a supernode is not sorted / does not start with its columns";
        return false;
      }
    }
  }
  rowptr[supNo] = Li_ptr[n];
  int64_t nls = Li_ptr[n];
  int64_t xsize = lC[n];
  int64_t nnz = c[n];
  for (int j = 0; j < n; ++j)
    if (c[j + 1] < c[j]) { err = "column pointers of A not monotone"; return false; }
  for (int s = 0; s <= supNo; ++s)
    if (s < supNo && prunePtr[s + 1] < prunePtr[s]) { err = "prunePtr not monotone"; return false; }
  int nprune = prunePtr[supNo];
  for (int q = 0; q < nprune; ++q)
    if (pruneSet[q] < 0 || pruneSet[q] >= supNo) { err = "pruneSet entry out of range"; return false; }
  for (int s = 0; s < supNo; ++s)
    for (int q = prunePtr[s]; q < prunePtr[s + 1]; ++q)
      if (pruneSet[q] >= s) { err = "prune set holds a non-descendant"; return false; }

  // ---- supernodal etree and levels ----
  std::vector<int> col2sup(n);
  for (int s = 0; s < supNo; ++s)
    for (int j = super[s]; j < super[s + 1]; ++j) col2sup[j] = s;
  std::vector<int> level(supNo, 0);
  int nlev = 0;
  for (int s = 0; s < supNo; ++s) {
    int w = super[s + 1] - super[s];
    int64_t m = rowptr[s + 1] - rowptr[s];
    nlev = std::max(nlev, level[s] + 1);
    if (m > w) {
      int p = col2sup[Ls[rowptr[s] + w]];
      level[p] = std::max(level[p], level[s] + 1);
    }
  }
  // every update source must sit on an earlier level than its target
  for (int s = 0; s < supNo; ++s)
    for (int q = prunePtr[s]; q < prunePtr[s + 1]; ++q)
      if (level[pruneSet[q]] >= level[s]) { err = "prune set is not consistent with the etree"; return false; }

  // ---- plan ----
  Plan P;
  P.waves.resize(nlev);
  std::vector<std::vector<int>> by_level(nlev);
  for (int s = 0; s < supNo; ++s) by_level[level[s]].push_back(s);
  int launches = 2;
  for (int lv = 0; lv < nlev; ++lv) {
    Wave &W = P.waves[lv];
    W.small_off = (int)P.small_list.size();
    W.asm_off = (int)P.asm_tasks.size();
    W.upd_off = (int)P.upd_tasks.size();
    std::vector<int> big;
    for (int s : by_level[lv]) {
      int w = super[s + 1] - super[s];
      int64_t m = rowptr[s + 1] - rowptr[s];
      if (small_class(w, m)) {
        P.small_list.push_back(s);
        W.small_smem = std::max<int>(W.small_smem, (int)(8 * m * w + 8 * m));
      } else {
        big.push_back(s);
      }
    }
    W.small_cnt = (int)P.small_list.size() - W.small_off;
    W.big_off = (int)P.big_list.size();
    W.big_cnt = (int)big.size();
    P.big_list.insert(P.big_list.end(), big.begin(), big.end());
    int maxnb = 0;
    for (int s : big) {
      int f = super[s], w = super[s + 1] - f;
      int m = (int)(rowptr[s + 1] - rowptr[s]);
      for (int j = f; j < f + w; ++j) P.asm_tasks.push_back(make_int2(s, j));
      if (prunePtr[s + 1] > prunePtr[s]) {
        for (int c0 = 0; c0 < w; c0 += TB)
          for (int r0 = 0; r0 < m; r0 += TB)
            if (r0 + TB - 1 >= c0) P.upd_tasks.push_back(make_int4(s, r0, c0, 0));
      }
      maxnb = std::max(maxnb, (w + TB - 1) / TB);
    }
    W.asm_cnt = (int)P.asm_tasks.size() - W.asm_off;
    W.upd_cnt = (int)P.upd_tasks.size() - W.upd_off;
    for (int j = 0; j < maxnb; ++j) {
      W.panel_off.push_back((int)P.panel_tasks.size());
      W.syrk_off.push_back((int)P.syrk_tasks.size());
      for (int s : big) {
        int w = super[s + 1] - super[s];
        int m = (int)(rowptr[s + 1] - rowptr[s]);
        int c0 = j * TB;
        if (c0 >= w) continue;
        int bw = std::min(TB, w - c0);
        for (int r0 = c0 + bw; r0 < m; r0 += TB) P.panel_tasks.push_back(make_int2(s, r0));
        for (int cc = c0 + TB; cc < w; cc += TB)
          for (int r0 = cc; r0 < m; r0 += TB) P.syrk_tasks.push_back(make_int4(s, r0, cc, 0));
      }
      W.panel_cnt.push_back((int)P.panel_tasks.size() - W.panel_off.back());
      W.syrk_cnt.push_back((int)P.syrk_tasks.size() - W.syrk_off.back());
    }
    launches += (W.small_cnt > 0) + (W.asm_cnt > 0) + (W.upd_cnt > 0) + (W.big_cnt > 0);
    for (int j = 0; j < maxnb; ++j) launches += (W.panel_cnt[j] > 0) + (W.syrk_cnt[j] > 0);
  }
  P.launches = launches;

  // ---- algorithmic work per kernel class (one factorization) ----
  {
    KernelStats &K = P.work;
    auto upd_flops = [&](int s, int64_t lo_row, int64_t hi_row, int64_t lo_col, int64_t hi_col,
                         double &bytes) {
      // sum over the prune set of 2 * (rows of d in [lo_row,hi_row]) * (rows of d in
      // [lo_col,hi_col]) * width(d)
      double fl = 0;
      for (int q = prunePtr[s]; q < prunePtr[s + 1]; ++q) {
        int d = pruneSet[q];
        const int *b = Ls + rowptr[d], *e = Ls + rowptr[d + 1];
        int64_t na = std::lower_bound(b, e, (int)hi_row + 1) - std::lower_bound(b, e, (int)lo_row);
        int64_t nb = std::lower_bound(b, e, (int)hi_col + 1) - std::lower_bound(b, e, (int)lo_col);
        int wd = super[d + 1] - super[d];
        if (na > 0 && nb > 0) {
          fl += 2.0 * na * nb * wd;
          bytes += 8.0 * (na + nb) * wd;
        }
      }
      return fl;
    };
    for (int s : P.small_list) {
      int f = super[s], w = super[s + 1] - f;
      int64_t m = rowptr[s + 1] - rowptr[s];
      double fl = 0, by = 0;
      for (int q = prunePtr[s]; q < prunePtr[s + 1]; ++q) {
        int d = pruneSet[q];
        const int *b = Ls + rowptr[d], *e = Ls + rowptr[d + 1];
        int64_t lb = std::lower_bound(b, e, f) - b, ub = std::lower_bound(b, e, f + w) - b;
        int64_t nr = (e - b) - lb, n1 = ub - lb;
        int wd = super[d + 1] - super[d];
        fl += 2.0 * (n1 * nr - n1 * (n1 - 1) / 2) * wd;
        by += 8.0 * nr * wd;
      }
      fl += (double)w * w * w / 3.0 + (double)(m - w) * w * w;
      by += 16.0 * m * w + 12.0 * (c[f + w] - c[f]);
      K.flops[K_SMALL] += fl;
      K.bytes[K_SMALL] += by;
    }
    for (const int4 &t : P.upd_tasks) {
      int s = t.x, f = super[s], w = super[s + 1] - f;
      int64_t m = rowptr[s + 1] - rowptr[s];
      int nrow = (int)std::min<int64_t>(TB, m - t.y), ncol = std::min(TB, w - t.z);
      const int *rows = Ls + rowptr[s];
      double by = 16.0 * nrow * ncol;
      K.flops[K_UPDATE] += upd_flops(s, rows[t.y], rows[t.y + nrow - 1], f + t.z, f + t.z + ncol - 1, by);
      K.bytes[K_UPDATE] += by;
    }
    for (const int4 &t : P.syrk_tasks) {
      int s = t.x, w = super[s + 1] - super[s];
      int64_t m = rowptr[s + 1] - rowptr[s];
      int nrow = (int)std::min<int64_t>(TB, m - t.y), ncol = std::min(TB, w - t.z);
      K.flops[K_SYRK] += 2.0 * nrow * ncol * TB;
      K.bytes[K_SYRK] += 8.0 * (2.0 * nrow * ncol + (nrow + ncol) * TB);
    }
    // dense factorization of the tiled class: POTRF + TRSM per column block
    for (int lv = 0; lv < nlev; ++lv)
      for (int s : by_level[lv]) {
        int w = super[s + 1] - super[s];
        int64_t m = rowptr[s + 1] - rowptr[s];
        if (small_class(w, m)) continue;
        for (int c0 = 0; c0 < w; c0 += TB) {
          int bw = std::min(TB, w - c0);
          K.flops[K_PANEL] += (double)bw * bw * bw / 3.0 + (double)(m - c0 - bw) * bw * bw;
          K.bytes[K_PANEL] += 16.0 * (m - c0) * bw;
        }
        K.bytes[K_ASSEMBLE] += 12.0 * (c[super[s + 1]] - c[super[s]]) + 8.0 * m * w;
      }
  }

  // ---- upload ----
  release();
  cudaStream_t st = stream_;
  std::vector<int64_t> rp(rowptr);
  bool ok = upload(d_super_, super.data(), super.size(), st, err) &&
            upload(d_rowptr_, rp.data(), rp.size(), st, err) &&
            upload(d_Ls_, Ls, (size_t)nls, st, err) &&
            upload(d_xptr_, xptr.data(), xptr.size(), st, err) &&
            upload(d_Ap_, c, (size_t)n + 1, st, err) &&
            upload(d_Ai_, r, (size_t)nnz, st, err) &&
            upload(d_upd_ptr_, prunePtr, (size_t)supNo + 1, st, err) &&
            upload(d_upd_, pruneSet, (size_t)nprune, st, err) &&
            upload(d_small_, P.small_list.data(), P.small_list.size(), st, err) &&
            upload(d_big_, P.big_list.data(), P.big_list.size(), st, err) &&
            upload(d_asm_, P.asm_tasks.data(), P.asm_tasks.size(), st, err) &&
            upload(d_upd_tasks_, P.upd_tasks.data(), P.upd_tasks.size(), st, err) &&
            upload(d_panel_, P.panel_tasks.data(), P.panel_tasks.size(), st, err) &&
            upload(d_syrk_, P.syrk_tasks.data(), P.syrk_tasks.size(), st, err);
  if (!ok) return false;
  cudaError_t e = cudaMalloc(&d_Ax_, sizeof(double) * std::max<int64_t>(nnz, 1));
  if (e == cudaSuccess) e = cudaMalloc(&dL_, sizeof(double) * std::max<int64_t>(xsize, 1));
  if (e == cudaSuccess) e = cudaMalloc(&d_status_, 2 * sizeof(int));
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    err = std::string("device allocation: ") + cudaGetErrorString(e);
    return false;
  }
  n_ = n;
  nsuper_ = supNo;
  xsize_ = xsize;
  nnz_ = nnz;
  plan_ = std::move(P);
  sym_.n = n;
  sym_.nsuper = supNo;
  sym_.super = d_super_;
  sym_.rowptr = d_rowptr_;
  sym_.Ls = d_Ls_;
  sym_.xptr = d_xptr_;
  sym_.Ap = d_Ap_;
  sym_.Ai = d_Ai_;
  sym_.Ax = d_Ax_;
  sym_.upd_ptr = d_upd_ptr_;
  sym_.upd = d_upd_;
  sym_.L = dL_;
  sym_.status = d_status_;
  return true;
}

void Engine::launch_all(std::vector<std::pair<int, cudaEvent_t>> *prof) {
  cudaStream_t st = stream_;
  // With profiling on, every launch is preceded by an event and followed by one.
  auto mark = [&](int kind, int count) {
    if (!prof || count <= 0) return;
    cudaEvent_t ev;
    cudaEventCreate(&ev);
    cudaEventRecord(ev, st);
    prof->emplace_back(kind, ev);
  };
  mark(K_MEMSET, 1);
  cudaMemsetAsync(dL_, 0, sizeof(double) * xsize_, st);
  launch_init_status(d_status_, st);
  mark(-1, 1);
  for (const Wave &W : plan_.waves) {
    mark(K_SMALL, W.small_cnt);
    launch_factor_small(sym_, d_small_ + W.small_off, W.small_cnt, W.small_smem, st);
    mark(-1, W.small_cnt);
    mark(K_ASSEMBLE, W.asm_cnt);
    launch_assemble(sym_, d_asm_ + W.asm_off, W.asm_cnt, st);
    mark(-1, W.asm_cnt);
    mark(K_UPDATE, W.upd_cnt);
    launch_update_tiles(sym_, d_upd_tasks_ + W.upd_off, W.upd_cnt, st);
    mark(-1, W.upd_cnt);
    mark(K_PANEL, W.big_cnt);
    launch_potrf_first(sym_, d_big_ + W.big_off, W.big_cnt, st);
    mark(-1, W.big_cnt);
    for (size_t j = 0; j < W.panel_off.size(); ++j) {
      mark(K_PANEL, W.panel_cnt[j]);
      launch_trsm_step(sym_, d_panel_ + W.panel_off[j], W.panel_cnt[j], (int)j, st);
      mark(-1, W.panel_cnt[j]);
      mark(K_SYRK, W.syrk_cnt[j]);
      launch_syrk_step(sym_, d_syrk_ + W.syrk_off[j], W.syrk_cnt[j], (int)j, st);
      mark(-1, W.syrk_cnt[j]);
    }
  }
}

int Engine::factor(const double *values, bool values_on_device, int *info, std::string &err) {
  if (!dL_) { err = "factor before analyze"; return -1; }
  cudaSetDevice(device_);
  cudaStream_t st = stream_;
  cudaError_t e;
  if (values_on_device) {
    sym_.Ax = values;
    e = cudaSuccess;
  } else {
    sym_.Ax = d_Ax_;
    e = cudaMemcpyAsync(d_Ax_, values, sizeof(double) * nnz_, cudaMemcpyHostToDevice, st);
  }
  if (e != cudaSuccess) { err = std::string("values upload: ") + cudaGetErrorString(e); return -1; }
  h2d_bytes_ = values_on_device ? 0 : (int64_t)sizeof(double) * nnz_;
  launch_all();
  return finish(info, err);
}

int Engine::factor_profiled(const double *values, bool values_on_device, int *info,
                            KernelStats &out, std::string &err) {
  if (!dL_) { err = "factor before analyze"; return -1; }
  cudaSetDevice(device_);
  cudaStream_t st = stream_;
  cudaError_t e = cudaSuccess;
  if (values_on_device) {
    sym_.Ax = values;
  } else {
    sym_.Ax = d_Ax_;
    e = cudaMemcpyAsync(d_Ax_, values, sizeof(double) * nnz_, cudaMemcpyHostToDevice, st);
  }
  if (e != cudaSuccess) { err = std::string("values upload: ") + cudaGetErrorString(e); return -1; }
  std::vector<std::pair<int, cudaEvent_t>> prof;
  launch_all(&prof);
  int rc = finish(info, err);
  out = plan_.work;
  for (int k = 0; k < K_NKINDS; ++k) { out.launches[k] = 0; out.ms[k] = 0; }
  for (size_t i = 0; i + 1 < prof.size(); i += 2) {
    float ms = 0;
    cudaEventElapsedTime(&ms, prof[i].second, prof[i + 1].second);
    int k = prof[i].first;
    out.launches[k] += 1;
    out.ms[k] += ms;
  }
  for (auto &pe : prof) cudaEventDestroy(pe.second);
  return rc;
}

int Engine::finish(int *info, std::string &err) {
  cudaStream_t st = stream_;
  cudaError_t e = cudaMemcpyAsync(h_status_, d_status_, 2 * sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) { err = std::string("factor: ") + cudaGetErrorString(e); return -1; }
  if (h_status_[1]) { err = "symbolic structure inconsistent with the matrix pattern"; return -2; }
  if (h_status_[0] != INT_MAX) {
    if (info) *info = h_status_[0];
    err = "matrix is not positive definite";
    return 1;
  }
  if (info) *info = 0;
  return 0;
}

bool Engine::download(double *lValues, bool to_device, std::string &err) {
  if (!dL_) { err = "download before factor"; return false; }
  cudaSetDevice(device_);
  cudaError_t e = cudaMemcpyAsync(lValues, dL_, sizeof(double) * xsize_,
                                  to_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                                  stream_);
  d2h_bytes_ = to_device ? 0 : (int64_t)sizeof(double) * xsize_;
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
  if (e != cudaSuccess) { err = std::string("download: ") + cudaGetErrorString(e); return false; }
  return true;
}

}  // namespace swc
