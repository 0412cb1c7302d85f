// C ABI of libswchol_b200 (declared in include/swcholesky_b200.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/swcholesky_b200.h"
#include "swc_engine.h"

#include "swc_handle.h"

namespace {

thread_local std::string g_err;
int g_last_info = 0;
std::mutex g_default_mu;
swc_handle *g_default = nullptr;

int fail(int code, const std::string &msg) {
  g_err = msg;
  return code;
}

// Status of a failed solve: SWC_TIMEOUT when a bounded wait ran out, else a CUDA error.
int solve_code(const std::string &err) {
  return err.rfind("timeout:", 0) == 0 ? SWC_TIMEOUT : SWC_CUDA_ERROR;
}

std::vector<int64_t> to_i64(const size_t *p, int count) {
  std::vector<int64_t> v(count);
  for (int i = 0; i < count; ++i) v[i] = (int64_t)p[i];
  return v;
}

}  // namespace

namespace swc {
void set_last_error(const std::string &msg) { g_err = msg; }
}  // namespace swc

namespace {
// Runs fn on device copies of host right-hand sides (and copies x back) when needed; the
// copies go through the handle's staging buffer (allocated once, grown on demand).
template <typename F>
int with_device_vectors(swc_handle_t h, const double *b, double *x, int nrhs, int on_device, F fn) {
  if (on_device) return fn(b, x);
  const size_t len = (size_t)h->eng->n() * nrhs;
  std::string err;
  double *stage = h->eng->staging(2 * len, err);
  if (!stage) return fail(SWC_CUDA_ERROR, err);
  double *db = stage, *dx = stage + len;
  cudaStream_t st = h->eng->stream();
  if (cudaMemcpyAsync(db, b, sizeof(double) * len, cudaMemcpyHostToDevice, st) != cudaSuccess)
    return fail(SWC_CUDA_ERROR, "copy of the right-hand sides to the device failed");
  int rc = fn(db, dx);
  if (rc == SWC_OK &&
      (cudaMemcpyAsync(x, dx, sizeof(double) * len, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
       cudaStreamSynchronize(st) != cudaSuccess))
    rc = fail(SWC_CUDA_ERROR, "copy of the solution to the host failed");
  return rc;
}
}  // namespace

extern "C" {

const char *swc_last_error(void) { return g_err.c_str(); }
int swc_last_info(void) { return g_last_info; }

int swc_create(swc_handle_t *handle, int device) {
  if (!handle) return fail(SWC_INVALID_INPUT, "null handle pointer");
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0)
    return fail(SWC_CUDA_ERROR, std::string("no CUDA device: ") + cudaGetErrorString(e));
  if (device < 0 || device >= ndev) return fail(SWC_INVALID_INPUT, "device out of range");
  swc_handle *h = new swc_handle;
  h->device = device;
  h->eng.reset(new swc::Engine(device));
  *handle = h;
  return SWC_OK;
}

int swc_destroy(swc_handle_t handle) {
  delete handle;
  return SWC_OK;
}

int swc_set_stream(swc_handle_t h, void *stream) {
  if (!h) return fail(SWC_INVALID_INPUT, "null handle");
  h->eng->set_stream((cudaStream_t)stream);
  return SWC_OK;
}

int swc_set_plan(swc_handle_t h, int plan) {
  if (!h) return fail(SWC_INVALID_INPUT, "null handle");
  if (plan < 0 || plan >= swc::num_plans()) return fail(SWC_INVALID_INPUT, "unknown plan");
  h->plan = plan;
  return SWC_OK;
}

void *swc_get_stream(swc_handle_t h) { return h ? (void *)h->eng->stream() : nullptr; }

int swc_set_wait_budget(swc_handle_t h, long long polls) {
  if (!h) return fail(SWC_INVALID_INPUT, "null handle");
  std::string err;
  if (!h->eng->set_wait_budget(polls, err)) return fail(SWC_CUDA_ERROR, err);
  return SWC_OK;
}

int swc_analyze(swc_handle_t h, int n, const int *c, const int *r, const size_t *lC,
                const int *Ls, const size_t *Li_ptr, const int *blockSet, int supNo,
                const int *prunePtr, const int *pruneSet, int nLevels, const int *levelPtr,
                const int *parPtr, const int *partition) {
  if (!h) return fail(SWC_INVALID_INPUT, "null handle");
  if (n <= 0 || !lC || !Li_ptr) return fail(SWC_INVALID_INPUT, "null or empty symbolic input");
  // The H-level schedule, when given, must cover every supernode exactly once.
  if (levelPtr && parPtr && partition && nLevels > 0) {
    int nparts = levelPtr[nLevels];
    if (levelPtr[0] != 0 || nparts < 0 || parPtr[0] != 0 || parPtr[nparts] != supNo)
      return fail(SWC_INVALID_INPUT, "H-level schedule does not cover the supernodes");
    std::vector<char> seen(supNo, 0);
    for (int k = 0; k < supNo; ++k) {
      int s = partition[k];
      if (s < 0 || s >= supNo || seen[s]) return fail(SWC_INVALID_INPUT, "partition is not a permutation");
      seen[s] = 1;
    }
  }
  std::vector<int64_t> lc = to_i64(lC, n + 1), lip = to_i64(Li_ptr, n + 1);
  std::string err;
  h->analyzed = false;
  h->factored = false;
  h->batch.reset();
  h->eng->set_tuning(swc::plan_candidate(h->plan));
  if (!h->eng->analyze(n, c, r, lc.data(), Ls, lip.data(), blockSet, supNo, prunePtr, pruneSet, err))
    return fail(err.rfind("device", 0) == 0 ? SWC_CUDA_ERROR : SWC_INVALID_INPUT, err);
  h->analyzed = true;
  return SWC_OK;
}

int swc_factor(swc_handle_t h, const double *values, int values_on_device, int mode, int *info) {
  if (!h) return fail(SWC_INVALID_INPUT, "null handle");
  if (!h->analyzed) return fail(SWC_NOT_READY, "factor before analyze");
  if (mode != SWC_MODE_FP64 && mode != SWC_MODE_MIXED_TF32X3 && mode != SWC_MODE_MIXED_BF16X3)
    return fail(SWC_INVALID_INPUT, "unknown factorization mode");
  if (!values) return fail(SWC_INVALID_INPUT, "null values");
  std::string err;
  int lin = 0;
  int rc = h->eng->factor(values, values_on_device != 0, &lin, err, mode);
  if (info) *info = lin;
  if (rc == 0) {
    h->factored = true;
    return SWC_OK;
  }
  h->factored = false;
  if (rc == 1) return fail(SWC_NOT_SPD, err);
  if (rc == -2) return fail(SWC_STRUCTURE_ERROR, err);
  if (rc == -3) return fail(SWC_TIMEOUT, err);
  return fail(SWC_CUDA_ERROR, err);
}

int swc_get_L(swc_handle_t h, double *lValues, int to_device) {
  if (!h) return fail(SWC_INVALID_INPUT, "null handle");
  if (!h->analyzed) return fail(SWC_NOT_READY, "no factor");
  std::string err;
  if (!h->eng->download(lValues, to_device != 0, err)) return fail(SWC_CUDA_ERROR, err);
  return SWC_OK;
}

const double *swc_device_L(swc_handle_t h) { return h ? h->eng->device_L() : nullptr; }


int swc_solve(swc_handle_t h, const double *b, double *x, int nrhs, int on_device) {
  if (!h) return fail(SWC_INVALID_INPUT, "null handle");
  if (!h->factored) return fail(SWC_NOT_READY, "solve before a successful factor");
  if (!b || !x || nrhs <= 0) return fail(SWC_INVALID_INPUT, "bad solve arguments");
  return with_device_vectors(h, b, x, nrhs, on_device, [&](const double *db, double *dx) {
    std::string err;
    if (!h->eng->solve(db, dx, nrhs, err)) return fail(solve_code(err), err);
    return SWC_OK;
  });
}

int swc_refine(swc_handle_t h, const double *b, double *x, int nrhs, int on_device, double tol,
               int maxit, double *berr, int *iterations, int *method) {
  if (!h) return fail(SWC_INVALID_INPUT, "null handle");
  if (!h->factored) return fail(SWC_NOT_READY, "refine before a successful factor");
  if (!b || !x || nrhs <= 0 || maxit < 0) return fail(SWC_INVALID_INPUT, "bad refine arguments");
  return with_device_vectors(h, b, x, nrhs, on_device, [&](const double *db, double *dx) {
    std::string err;
    swc::RefineInfo info;
    if (!h->eng->refine(db, dx, nrhs, tol, maxit, info, err)) return fail(solve_code(err), err);
    if (berr) for (int k = 0; k < nrhs; ++k) berr[k] = info.berr[k];
    if (iterations) *iterations = info.iterations;
    if (method) *method = info.method;
    return SWC_OK;
  });
}

int swc_logdet(swc_handle_t h, double *logdet) {
  if (!h || !logdet) return fail(SWC_INVALID_INPUT, "null argument");
  if (!h->factored) return fail(SWC_NOT_READY, "logdet before a successful factor");
  std::string err;
  if (!h->eng->logdet(logdet, err)) return fail(SWC_CUDA_ERROR, err);
  return SWC_OK;
}

int swc_logdet_grad(swc_handle_t h, double *grad, int on_device) {
  if (!h || !grad) return fail(SWC_INVALID_INPUT, "null argument");
  if (!h->factored) return fail(SWC_NOT_READY, "logdet gradient before a successful factor");
  std::string err;
  const size_t bytes = sizeof(double) * (size_t)h->eng->nnz();
  double *dg = grad;
  if (!on_device && cudaMalloc(&dg, std::max<size_t>(bytes, 8)) != cudaSuccess)
    return fail(SWC_CUDA_ERROR, "gradient buffer");
  int rc = SWC_OK;
  if (!h->eng->logdet_grad(dg, err)) rc = fail(SWC_CUDA_ERROR, err);
  else if (!on_device && cudaMemcpy(grad, dg, bytes, cudaMemcpyDeviceToHost) != cudaSuccess)
    rc = fail(SWC_CUDA_ERROR, "copy of the gradient to the host failed");
  if (!on_device) cudaFree(dg);
  return rc;
}

int swc_solve_grad(swc_handle_t h, const double *x, const double *lam, double *grad,
                   int on_device) {
  if (!h || !x || !lam || !grad) return fail(SWC_INVALID_INPUT, "null argument");
  if (!h->analyzed) return fail(SWC_NOT_READY, "solve gradient before analyze");
  std::string err;
  const size_t gbytes = sizeof(double) * (size_t)h->eng->nnz();
  const size_t vbytes = sizeof(double) * (size_t)h->eng->n();
  if (on_device) {
    if (!h->eng->solve_grad(x, lam, grad, err)) return fail(SWC_CUDA_ERROR, err);
    return SWC_OK;
  }
  double *dx = nullptr, *dl = nullptr, *dg = nullptr;
  cudaError_t e = cudaMalloc(&dx, vbytes);
  if (e == cudaSuccess) e = cudaMalloc(&dl, vbytes);
  if (e == cudaSuccess) e = cudaMalloc(&dg, std::max<size_t>(gbytes, 8));
  if (e == cudaSuccess) e = cudaMemcpy(dx, x, vbytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dl, lam, vbytes, cudaMemcpyHostToDevice);
  int rc = SWC_OK;
  if (e != cudaSuccess) rc = fail(SWC_CUDA_ERROR, std::string("solve gradient buffers: ") + cudaGetErrorString(e));
  else if (!h->eng->solve_grad(dx, dl, dg, err)) rc = fail(SWC_CUDA_ERROR, err);
  else if (cudaMemcpy(grad, dg, gbytes, cudaMemcpyDeviceToHost) != cudaSuccess)
    rc = fail(SWC_CUDA_ERROR, "copy of the gradient to the host failed");
  if (dx) cudaFree(dx);
  if (dl) cudaFree(dl);
  if (dg) cudaFree(dg);
  return rc;
}

int swc_batch_analyze(swc_handle_t h, int nmat, const int *n, const int *c, const int *r) {
  if (!h) return fail(SWC_INVALID_INPUT, "null handle");
  std::string err;
  h->analyzed = false;
  h->factored = false;
  std::unique_ptr<swc::BatchState> b(new swc::BatchState);
  if (!b->set(nmat, n, c, r, err)) return fail(SWC_INVALID_INPUT, err);
  if (!b->analyze(*h->eng, 0, swc::plan_candidate(h->plan), err))
    return fail(err.rfind("device", 0) == 0 ? SWC_CUDA_ERROR : SWC_INVALID_INPUT, err);
  h->batch = std::move(b);
  h->analyzed = true;
  return SWC_OK;
}

int swc_batch_autotune(swc_handle_t h, const double *values, int values_on_device, int mode,
                       const char *cache_path, int *choice, double *best_ms) {
  if (!h) return fail(SWC_INVALID_INPUT, "null handle");
  if (!h->batch || !h->analyzed) return fail(SWC_NOT_READY, "autotune before swc_batch_analyze");
  if (mode != SWC_MODE_FP64 && mode != SWC_MODE_MIXED_TF32X3 && mode != SWC_MODE_MIXED_BF16X3)
    return fail(SWC_INVALID_INPUT, "unknown factorization mode");
  if (!values) return fail(SWC_INVALID_INPUT, "null values");
  const size_t bytes = sizeof(double) * h->batch->cp[h->batch->N];
  const double *dv = values;
  double *tmp = nullptr;
  if (!values_on_device) {
    if (cudaMalloc(&tmp, std::max<size_t>(bytes, 8)) != cudaSuccess ||
        cudaMemcpy(tmp, values, bytes, cudaMemcpyHostToDevice) != cudaSuccess) {
      if (tmp) cudaFree(tmp);
      return fail(SWC_CUDA_ERROR, "autotune: values upload failed");
    }
    dv = tmp;
  }
  std::string err;
  h->factored = false;
  const bool ok = h->batch->autotune(*h->eng, dv, mode, cache_path, 3,
                                     choice, best_ms, err);
  if (tmp) cudaFree(tmp);
  if (!ok) {
    h->analyzed = false;
    return fail(err.find("not positive definite") != std::string::npos ? SWC_NOT_SPD : SWC_CUDA_ERROR, err);
  }
  h->analyzed = true;
  return SWC_OK;
}

int swc_batch_berr(swc_handle_t h, const double *b, const double *x, int on_device, double *berr) {
  if (!h || !b || !x || !berr) return fail(SWC_INVALID_INPUT, "null argument");
  if (!h->batch) return fail(SWC_NOT_READY, "swc_batch_berr without swc_batch_analyze");
  if (!h->factored) return fail(SWC_NOT_READY, "swc_batch_berr before a successful factor");
  std::string err;
  const size_t bytes = sizeof(double) * (size_t)h->batch->N;
  const double *db = b, *dx = x;
  double *tb = nullptr, *tx = nullptr;
  if (!on_device) {
    cudaError_t e = cudaMalloc(&tb, bytes);
    if (e == cudaSuccess) e = cudaMalloc(&tx, bytes);
    if (e == cudaSuccess) e = cudaMemcpy(tb, b, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(tx, x, bytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      if (tb) cudaFree(tb);
      if (tx) cudaFree(tx);
      return fail(SWC_CUDA_ERROR, std::string("batch berr buffers: ") + cudaGetErrorString(e));
    }
    db = tb;
    dx = tx;
  }
  const bool ok = h->eng->segment_berr(h->batch->d_seg, h->batch->nmat, db, dx, berr, err);
  if (tb) cudaFree(tb);
  if (tx) cudaFree(tx);
  return ok ? SWC_OK : fail(SWC_CUDA_ERROR, err);
}

int swc_supernodes(int n, const int *c, const int *r, const int *nrelax, const double *zrelax,
                   int max_width, int *blockSet, int *supNo) {
  if (!c || !r || !blockSet || !supNo) return fail(SWC_INVALID_INPUT, "null argument");
  static const int kNrelax[3] = {4, 16, 48};
  static const double kZrelax[3] = {0.8, 0.1, 0.05};
  std::vector<int> super;
  std::string err;
  if (!swc::supernode_partition(n, c, r, nrelax ? nrelax : kNrelax, zrelax ? zrelax : kZrelax,
                                max_width, super, err))
    return fail(SWC_INVALID_INPUT, err);
  std::copy(super.begin(), super.end(), blockSet);
  *supNo = (int)super.size() - 1;
  return SWC_OK;
}

int swc_sizes(swc_handle_t h, long long *sizes) {
  if (!h || !sizes) return fail(SWC_INVALID_INPUT, "null argument");
  sizes[0] = h->eng->n();
  sizes[1] = h->eng->nsuper();
  sizes[2] = h->eng->xsize();
  sizes[3] = h->eng->launches_per_factor();
  sizes[4] = h->eng->h2d_bytes();
  sizes[5] = h->eng->d2h_bytes();
  return SWC_OK;
}

int swc_profile(swc_handle_t h, const double *values, int values_on_device, int mode, int *info,
                int *launches, double *ms, double *flops, double *bytes) {
  if (!h) return fail(SWC_INVALID_INPUT, "null handle");
  if (!h->analyzed) return fail(SWC_NOT_READY, "profile before analyze");
  if (!values) return fail(SWC_INVALID_INPUT, "null values");
  swc::KernelStats ks;
  std::string err;
  int lin = 0;
  int rc = h->eng->factor_profiled(values, values_on_device != 0, &lin, ks, err,
                                   mode);
  h->factored = (rc == 0);
  if (info) *info = lin;
  for (int k = 0; k < swc::K_NKINDS; ++k) {
    if (launches) launches[k] = ks.launches[k];
    if (ms) ms[k] = ks.ms[k];
    if (flops) flops[k] = ks.flops[k];
    if (bytes) bytes[k] = ks.bytes[k];
  }
  if (rc == 0) return SWC_OK;
  if (rc == 1) return fail(SWC_NOT_SPD, err);
  if (rc == -2) return fail(SWC_STRUCTURE_ERROR, err);
  return fail(SWC_CUDA_ERROR, err);
}

int sw_cholesky_left_par_05(int n, int *c, int *r, double *values, size_t *lC, int *Ls,
                            size_t *Li_ptr, double *lValues, int *blockSet, int supNo,
                            double *timing, int *prunePtr, int *pruneSet, int nLevels,
                            int *levelPtr, int *levelSet, int nPar, int *parPtr,
                            int *partition, int chunk, int threads, int super_max,
                            int col_max, double *nodCost) {
  (void)timing; (void)levelSet; (void)nPar; (void)chunk; (void)threads;
  (void)super_max; (void)col_max; (void)nodCost;
  std::lock_guard<std::mutex> lock(g_default_mu);
  g_last_info = 0;
  if (!g_default) {
    int dev = 0;
    cudaGetDevice(&dev);
    swc_handle_t h = nullptr;
    if (swc_create(&h, dev) != SWC_OK) return 0;
    g_default = h;
  }
  if (swc_analyze(g_default, n, c, r, lC, Ls, Li_ptr, blockSet, supNo, prunePtr, pruneSet,
                  nLevels, levelPtr, parPtr, partition) != SWC_OK)
    return 0;
  int info = 0;
  int rc = swc_factor(g_default, values, 0, SWC_MODE_FP64, &info);
  g_last_info = info;
  if (rc != SWC_OK && rc != SWC_NOT_SPD) return 0;
  if (swc_get_L(g_default, lValues, 0) != SWC_OK) return 0;
  return rc == SWC_OK ? 1 : 0;
}

int swc_plan_stats(int n, const int *c, const int *r, const size_t *lC, const int *Ls,
                   const size_t *Li_ptr, const int *blockSet, int supNo, const int *prunePtr,
                   const int *pruneSet, int plan, double *stats) {
  if (n <= 0 || !lC || !Li_ptr || !stats) return fail(SWC_INVALID_INPUT, "null or empty input");
  if (plan < 0 || plan >= swc::num_plans()) return fail(SWC_INVALID_INPUT, "unknown plan");
  std::vector<int64_t> lc = to_i64(lC, n + 1), lip = to_i64(Li_ptr, n + 1);
  swc::HostSym H;
  swc::Plan P;
  std::string err;
  if (!swc::build_plan(n, c, r, lc.data(), Ls, lip.data(), blockSet, supNo, prunePtr, pruneSet,
                       H, P, err, swc::plan_candidate(plan)))
    return fail(SWC_INVALID_INPUT, err);
  if (!swc::check_scatter_plan(n, Ls, H, P, swc::plan_candidate(plan), err))
    return fail(SWC_INVALID_INPUT, err);
  swc::SolvePlan SP;
  swc::build_solve_plan(n, Ls, H, SP);
  if (!swc::check_solve_plan(n, Ls, H, SP, err)) return fail(SWC_INVALID_INPUT, err);
  stats[0] = (double)P.waves.size();
  stats[1] = (double)P.launches;
  stats[2] = (double)P.small_list.size();
  stats[3] = (double)P.big_list.size();
  stats[4] = (double)P.upd_tasks.size();
  stats[5] = (double)P.upd_pairs.size();
  stats[6] = (double)P.panel_tasks.size();
  stats[7] = (double)P.syrk_tasks.size();
  for (int k = 0; k < swc::K_NKINDS; ++k) {
    stats[8 + k] = P.work.flops[k];
    stats[8 + swc::K_NKINDS + k] = P.work.bytes[k];
  }
  return SWC_OK;
}

int swc_layout_sizes(int n, const int *c, const int *r, const int *blockSet, int supNo,
                     long long *sizes) {
  swc::Layout L;
  std::string err;
  if (!sizes) return fail(SWC_INVALID_INPUT, "null sizes");
  if (!swc::build_layout(n, c, r, blockSet, supNo, L, err)) return fail(SWC_INVALID_INPUT, err);
  sizes[0] = (long long)L.Ls.size();
  sizes[1] = (long long)L.pruneSet.size();
  sizes[2] = (long long)L.xsize;
  sizes[3] = (long long)(L.levelPtr.size() - 1);
  return SWC_OK;
}

int swc_layout(int n, const int *c, const int *r, const int *blockSet, int supNo,
               size_t *lC, int *Ls, size_t *Li_ptr, int *sparent, int *prunePtr,
               int *pruneSet, int *levelPtr, int *parPtr, int *partition) {
  swc::Layout L;
  std::string err;
  if (!swc::build_layout(n, c, r, blockSet, supNo, L, err)) return fail(SWC_INVALID_INPUT, err);
  if (lC) for (int j = 0; j <= n; ++j) lC[j] = (size_t)L.lC[j];
  if (Li_ptr) for (int j = 0; j <= n; ++j) Li_ptr[j] = (size_t)L.Li_ptr[j];
  if (Ls) std::memcpy(Ls, L.Ls.data(), sizeof(int) * L.Ls.size());
  if (sparent) std::memcpy(sparent, L.sparent.data(), sizeof(int) * supNo);
  if (prunePtr) std::memcpy(prunePtr, L.prunePtr.data(), sizeof(int) * (supNo + 1));
  if (pruneSet) std::memcpy(pruneSet, L.pruneSet.data(), sizeof(int) * L.pruneSet.size());
  if (levelPtr) std::memcpy(levelPtr, L.levelPtr.data(), sizeof(int) * L.levelPtr.size());
  if (parPtr) std::memcpy(parPtr, L.parPtr.data(), sizeof(int) * L.parPtr.size());
  if (partition) std::memcpy(partition, L.partition.data(), sizeof(int) * L.partition.size());
  return SWC_OK;
}

// ---- input files and ordering (host only) --------------------------------------------

int swc_read_mtx(const char *path, int *n, int **colptr, int **rowind, double **values) {
  if (!path || !n || !colptr || !rowind || !values) return fail(SWC_INVALID_INPUT, "null argument");
  swc::MtxLower M;
  std::string err;
  if (!swc::read_matrix_market(path, M, err)) return fail(SWC_INVALID_INPUT, err);
  const size_t nnz = M.rowind.size();
  int *c = static_cast<int *>(std::malloc(sizeof(int) * ((size_t)M.n + 1)));
  int *r = static_cast<int *>(std::malloc(sizeof(int) * std::max<size_t>(nnz, 1)));
  double *v = static_cast<double *>(std::malloc(sizeof(double) * std::max<size_t>(nnz, 1)));
  if (!c || !r || !v) {
    std::free(c);
    std::free(r);
    std::free(v);
    return fail(SWC_INVALID_INPUT, "out of host memory");
  }
  std::memcpy(c, M.colptr.data(), sizeof(int) * ((size_t)M.n + 1));
  std::memcpy(r, M.rowind.data(), sizeof(int) * nnz);
  std::memcpy(v, M.values.data(), sizeof(double) * nnz);
  *n = M.n;
  *colptr = c;
  *rowind = r;
  *values = v;
  return SWC_OK;
}

void swc_free(void *p) { std::free(p); }

int swc_write_mtx(const char *path, int n, const int *c, const int *r, const double *values) {
  if (!path) return fail(SWC_INVALID_INPUT, "null path");
  std::string err;
  if (!swc::write_matrix_market(path, n, c, r, values, err)) return fail(SWC_INVALID_INPUT, err);
  return SWC_OK;
}

int swc_read_perm(const char *path, int n, size_t *perm) {
  if (!path || !perm) return fail(SWC_INVALID_INPUT, "null argument");
  std::vector<int64_t> p;
  std::string err;
  if (!swc::read_perm_file(path, n, p, err)) return fail(SWC_INVALID_INPUT, err);
  for (int k = 0; k < n; ++k) perm[k] = (size_t)p[k];
  return SWC_OK;
}

int swc_write_perm(const char *path, int n, const size_t *perm) {
  if (!path || !perm) return fail(SWC_INVALID_INPUT, "null argument");
  std::vector<int64_t> p(n > 0 ? n : 0);
  for (int k = 0; k < n; ++k) p[k] = perm[k] > (size_t)INT32_MAX ? -1 : (int64_t)perm[k];
  std::string err;
  if (!swc::write_perm_file(path, n, p.data(), err)) return fail(SWC_INVALID_INPUT, err);
  return SWC_OK;
}

int swc_order_nd(int n, const int *c, const int *r, int leaf, size_t *perm) {
  if (!perm) return fail(SWC_INVALID_INPUT, "null perm");
  swc::NdOptions opt;
  if (leaf > 0) opt.leaf = leaf;
  std::vector<int64_t> p;
  std::string err;
  if (!swc::nested_dissection_order(n, c, r, opt, p, err)) return fail(SWC_INVALID_INPUT, err);
  for (int k = 0; k < n; ++k) perm[k] = (size_t)p[k];
  return SWC_OK;
}

}  // extern "C"
