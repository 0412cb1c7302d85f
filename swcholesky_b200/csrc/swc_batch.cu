// Batched factorization of many independent SPD matrices of uneven size.
//
// The matrices (each already ordered, lower CSC) become one block-diagonal matrix whose
// elimination tree is a forest: one supernode partition and one layout for all of them,
// so every kernel of the engine -- the persistent small-supernode walk, the per-level
// tile updates and dense steps -- serves all matrices at once, and the whole batch is one
// CUDA graph replay.  Nothing couples the matrices numerically: each supernode, update and
// tile belongs to exactly one of them.
//
// The autotuner picks the supernode grouping (relaxation of the partition) and the plan's
// size classes (small-class limits, persistent-walk shared-memory cap) by timing the
// factorization of the batch itself: first the partition candidates with the default plan,
// then plan candidates on the best partition.  Results are cached per structure and mode
// in a text file (one line per key: hash, partition index, plan index, milliseconds).
//
// The reference has no batched path; this is a new capability of the library.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "swc_batch.h"

namespace swc {

namespace {

// Per matrix (one CTA): max |b - A x|, max |x|, max row sum of |A| over its rows.
__global__ void __launch_bounds__(256) k_segment_norms(const int64_t *seg, const int *rp,
                                                       const int *ci, const double *val,
                                                       const double *b, const double *x,
                                                       double *out) {
  __shared__ double red[3][256];
  const int k = blockIdx.x;
  double mr = 0.0, mx = 0.0, ma = 0.0;
  for (int64_t i = seg[k] + threadIdx.x; i < seg[k + 1]; i += 256) {
    double acc = b[i], ra = 0.0;
    for (int p = rp[i]; p < rp[i + 1]; ++p) {
      acc -= val[p] * x[ci[p]];
      ra += fabs(val[p]);
    }
    mr = fmax(mr, fabs(acc));
    mx = fmax(mx, fabs(x[i]));
    ma = fmax(ma, ra);
  }
  red[0][threadIdx.x] = mr;
  red[1][threadIdx.x] = mx;
  red[2][threadIdx.x] = ma;
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if (threadIdx.x < h)
      for (int q = 0; q < 3; ++q) red[q][threadIdx.x] = fmax(red[q][threadIdx.x], red[q][threadIdx.x + h]);
    __syncthreads();
  }
  if (threadIdx.x < 3) out[3 * k + threadIdx.x] = red[threadIdx.x][0];
}

uint64_t fnv1a(uint64_t h, const void *data, size_t bytes) {
  const unsigned char *p = static_cast<const unsigned char *>(data);
  for (size_t i = 0; i < bytes; ++i) {
    h ^= p[i];
    h *= 1099511628211ULL;
  }
  return h;
}

}  // namespace

bool Engine::segment_berr(const int64_t *d_seg, int nseg, const double *b, const double *x,
                          double *berr, std::string &err) {
  cudaSetDevice(device_);
  double *d_out = nullptr;
  cudaError_t e = cudaMalloc(&d_out, sizeof(double) * 3 * std::max(nseg, 1));
  std::vector<double> h(3 * (size_t)std::max(nseg, 1));
  if (e == cudaSuccess && nseg > 0) {
    k_segment_norms<<<nseg, 256, 0, stream_>>>(d_seg, d_csr_rp_, d_csr_ci_, d_csr_val_, b, x, d_out);
    e = cudaMemcpyAsync(h.data(), d_out, sizeof(double) * 3 * nseg, cudaMemcpyDeviceToHost, stream_);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
  if (d_out) cudaFree(d_out);
  if (e != cudaSuccess) {
    err = std::string("segment backward error: ") + cudaGetErrorString(e);
    return false;
  }
  for (int k = 0; k < nseg; ++k) {
    const double den = h[3 * k + 2] * h[3 * k + 1];
    berr[k] = den > 0.0 ? h[3 * k] / den : (h[3 * k] > 0.0 ? INFINITY : 0.0);
  }
  return true;
}

const PartitionParams kPartitions[] = {
    {{4, 16, 48}, {0.8, 0.1, 0.05}, 1 << 30},   // the reference's relaxation
    {{0, 0, 0}, {0.0, 0.0, 0.0}, 1 << 30},      // exact supernodes (no explicit zeros)
    {{8, 32, 64}, {0.8, 0.2, 0.1}, 1 << 30},    // coarser grouping
};
const int kNumPartitions = sizeof(kPartitions) / sizeof(kPartitions[0]);

Tuning plan_candidate(int k) {
  Tuning t;
  switch (k) {
    case 0: break;                                       // defaults: persistent <= 24 KB
    case 1: t.persist_max_smem = 100 * 1024; break;      // bigger supernodes in the walk
    case 2: t.persist = 0; break;                        // level-by-level launches only
    case 3:                                              // fewer tiled supernodes
      t.small_max_elems = SMALL_MAX_ELEMS;
      t.small_max_m = SMALL_MAX_M;
      t.persist_max_smem = 48 * 1024;
      break;
    case 4: t.dense_dataflow = 1; break;                 // dense steps as one dataflow launch
    case 5: t.syrk_fp64 = 1; break;                      // mixed modes: FP64 SYRK steps
    case 6: t.scatter = 0; t.tc_tma = 1; break;          // mixed: tile-owner updates (TMA for TF32)
    case 7: t.scatter = 0; break;                        // mixed: tile-owner, cp.async
    case 8: t.scatter_kmax = 256; break;                 // mixed: K cut into 256-column tiles
    case 9: t.scatter_kmax = 128; break;                 // mixed: 128-column tiles
    default: break;
  }
  return t;
}
const int kNumPlans = 10;
int num_plans() { return kNumPlans; }

bool BatchState::set(int nm, const int *n, const int *c, const int *r, std::string &err) {
  if (nm <= 0 || !n || !c || !r) {
    err = "invalid batch arguments";
    return false;
  }
  nmat = nm;
  col_off.assign(nmat + 1, 0);
  std::vector<int64_t> cptr_off(nmat + 1, 0);
  for (int k = 0; k < nmat; ++k) {
    if (n[k] <= 0) {
      err = "every matrix needs n > 0";
      return false;
    }
    col_off[k + 1] = col_off[k] + n[k];
    cptr_off[k + 1] = cptr_off[k] + n[k] + 1;
  }
  if (col_off[nmat] > INT32_MAX) {
    err = "batch too large (total columns exceed 2^31)";
    return false;
  }
  N = (int)col_off[nmat];
  cp.assign((size_t)N + 1, 0);
  int64_t nz = 0;
  for (int k = 0; k < nmat; ++k) {
    const int *ck = c + cptr_off[k];
    if (ck[0] != 0) {
      err = "each matrix's column pointers must start at 0";
      return false;
    }
    for (int j = 0; j < n[k]; ++j) {
      if (ck[j + 1] < ck[j]) {
        err = "column pointers must be non-decreasing";
        return false;
      }
      cp[col_off[k] + j] = (int)nz + ck[j];
    }
    nz += ck[n[k]];
    if (nz > INT32_MAX) {
      err = "batch too large (nonzeros exceed 2^31)";
      return false;
    }
  }
  cp[N] = (int)nz;
  ri.resize(nz);
  for (int k = 0; k < nmat; ++k) {
    const int *ck = c + cptr_off[k];
    const int64_t base = cp[col_off[k]];
    for (int64_t p = 0; p < ck[n[k]]; ++p) {
      const int i = r[base + p];
      if (i < 0 || i >= n[k]) {
        err = "row index out of range in matrix " + std::to_string(k);
        return false;
      }
      ri[base + p] = i + (int)col_off[k];
    }
  }
  uint64_t h = 1469598103934665603ULL;
  h = fnv1a(h, &N, sizeof(N));
  h = fnv1a(h, col_off.data(), col_off.size() * sizeof(int64_t));
  h = fnv1a(h, cp.data(), cp.size() * sizeof(int));
  h = fnv1a(h, ri.data(), ri.size() * sizeof(int));
  key = h;
  return true;
}

bool BatchState::analyze(Engine &eng, int part, const Tuning &t, std::string &err) {
  const PartitionParams &pp = kPartitions[part];
  std::vector<int> super;
  if (!supernode_partition(N, cp.data(), ri.data(), pp.nrelax, pp.zrelax, pp.max_width, super,
                           err))
    return false;
  Layout lay;
  if (!build_layout(N, cp.data(), ri.data(), super.data(), (int)super.size() - 1, lay, err))
    return false;
  eng.set_tuning(t);
  if (!eng.analyze(N, cp.data(), ri.data(), lay.lC.data(), lay.Ls.data(), lay.Li_ptr.data(),
                   super.data(), (int)super.size() - 1, lay.prunePtr.data(), lay.pruneSet.data(),
                   err))
    return false;
  partition = part;
  plan = t;
  if (d_seg) cudaFree(d_seg);
  d_seg = nullptr;
  cudaError_t e = cudaMalloc(&d_seg, sizeof(int64_t) * (nmat + 1));
  if (e == cudaSuccess)
    e = cudaMemcpy(d_seg, col_off.data(), sizeof(int64_t) * (nmat + 1), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    err = std::string("batch offsets: ") + cudaGetErrorString(e);
    return false;
  }
  return true;
}

BatchState::~BatchState() {
  if (d_seg) cudaFree(d_seg);
}

namespace {

bool cache_lookup(const std::string &path, uint64_t key, int mode, int &part, int &plan,
                  double &ms) {
  FILE *f = fopen(path.c_str(), "r");
  if (!f) return false;
  unsigned long long k;
  int md, pa, pl;
  double t;
  bool found = false;
  while (fscanf(f, "%llx %d %d %d %lf", &k, &md, &pa, &pl, &t) == 5)
    if (k == key && md == mode && pa >= 0 && pa < kNumPartitions && pl >= 0 && pl < kNumPlans) {
      part = pa;
      plan = pl;
      ms = t;
      found = true;
    }
  fclose(f);
  return found;
}

void cache_store(const std::string &path, uint64_t key, int mode, int part, int plan, double ms) {
  FILE *f = fopen(path.c_str(), "a");
  if (!f) return;
  fprintf(f, "%llx %d %d %d %.6f\n", (unsigned long long)key, mode, part, plan, ms);
  fclose(f);
}

}  // namespace

bool BatchState::autotune(Engine &eng, const double *d_values, int mixed, const char *cache_path,
                          int reps, int *choice, double *best_ms, std::string &err) {
  const int mode = mixed;
  int bp = 0, bl = 0;
  double best = DBL_MAX;
  if (cache_path && cache_lookup(cache_path, key, mode, bp, bl, best)) {
    if (!analyze(eng, bp, plan_candidate(bl), err)) return false;
    if (choice) { choice[0] = bp; choice[1] = bl; }
    if (best_ms) *best_ms = best;
    return true;
  }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  auto measure = [&](int part, int plan_k, double &ms) -> bool {
    if (!analyze(eng, part, plan_candidate(plan_k), err)) return false;
    int info = 0;
    if (eng.factor(d_values, true, &info, err, mixed) != 0) return false;   // warm-up + graph
    cudaEventRecord(e0, eng.stream());
    for (int i = 0; i < reps; ++i)
      if (eng.factor(d_values, true, &info, err, mixed) != 0) return false;
    cudaEventRecord(e1, eng.stream());
    cudaEventSynchronize(e1);
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    ms = t / reps;
    return true;
  };
  bool ok = true;
  // stage 1: partition, default plan
  for (int p = 0; p < kNumPartitions && ok; ++p) {
    double ms;
    ok = measure(p, 0, ms);
    if (ok && ms < best) { best = ms; bp = p; bl = 0; }
  }
  // stage 2: plan, best partition (only the plans that change something in this mode:
  // 5 to 7 apply to the mixed modes, 6 differs from 7 in the split-TF32 mode only)
  for (int k = 1; k < kNumPlans && ok; ++k) {
    if ((k >= 5 && mode == 0) || (k == 6 && mode != 1)) continue;
    double ms;
    ok = measure(bp, k, ms);
    if (ok && ms < best) { best = ms; bl = k; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (!ok) return false;
  if (!analyze(eng, bp, plan_candidate(bl), err)) return false;
  if (cache_path) cache_store(cache_path, key, mode, bp, bl, best);
  if (choice) { choice[0] = bp; choice[1] = bl; }
  if (best_ms) *best_ms = best;
  return true;
}

}  // namespace swc
