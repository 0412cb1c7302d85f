// The numeric-factorization engine: device-resident symbolic data, the execution plan
// derived from it, and the launch sequence of the FP64 supernodal factorization.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "swc_internal.h"

namespace swc {

// Device view of one analysed matrix, passed by value to every kernel.
struct DevSym {
  int n, nsuper;
  const int *super;       // nsuper+1: first column of each supernode
  const int64_t *rowptr;  // nsuper+1: start of each supernode's row list in Ls
  const int *Ls;          // row lists
  const int64_t *xptr;    // nsuper: offset of each supernode's values in L
  const int *Ap;          // lower CSC of P A P^T
  const int *Ai;
  const double *Ax;
  const int *upd_ptr;     // update lists (prune sets)
  const int *upd;
  double *L;              // supernodal values (the reference's lValues)
  int *status;            // [0] = smallest failing column + 1 (INT_MAX if none),
                          // [1] = structure error flag
};

// One level of the schedule (supernodes whose descendants all belong to earlier levels).
struct Wave {
  int small_off = 0, small_cnt = 0;
  int small_smem = 0;
  int asm_off = 0, asm_cnt = 0;    // (supernode, column) tasks of the tiled class
  int upd_off = 0, upd_cnt = 0;    // (supernode, row tile, column tile) update tasks
  int big_off = 0, big_cnt = 0;    // tiled-class supernodes (block 0 POTRF)
  std::vector<int> panel_off, panel_cnt;  // per column block step: TRSM tiles
  std::vector<int> syrk_off, syrk_cnt;
};

// Kernel classes, for per-kernel timing (profiled factorization) and flop accounting.
enum KernelKind { K_MEMSET = 0, K_SMALL, K_ASSEMBLE, K_UPDATE, K_PANEL, K_SYRK, K_NKINDS };

struct KernelStats {
  int launches[K_NKINDS] = {0};
  double ms[K_NKINDS] = {0};
  double flops[K_NKINDS] = {0};   // algorithmic flops of one factorization
  double bytes[K_NKINDS] = {0};   // algorithmic DRAM bytes of one factorization
};

struct Plan {
  std::vector<Wave> waves;
  std::vector<int> small_list;
  std::vector<int> big_list;
  std::vector<int2> asm_tasks;
  std::vector<int4> upd_tasks;
  std::vector<int2> panel_tasks;
  std::vector<int4> syrk_tasks;
  int launches = 0;  // kernel launches per factorization
  KernelStats work;  // algorithmic flops/bytes per kernel class
};


class Engine {
 public:
  explicit Engine(int device);
  ~Engine();
  bool analyze(int n, const int *c, const int *r, const int64_t *lC, const int *Ls,
               const int64_t *Li_ptr, const int *blockSet, int supNo, const int *prunePtr,
               const int *pruneSet, std::string &err);
  // values: the A2 values (host or device).  Returns 0 on success, 1 if not SPD
  // (*info = failing column + 1), <0 on errors.
  int factor(const double *values, bool values_on_device, int *info, std::string &err);
  // The same factorization with a CUDA event pair around every launch; fills per-class
  // launch counts and device milliseconds (no other difference).
  int factor_profiled(const double *values, bool values_on_device, int *info,
                      KernelStats &out, std::string &err);
  int64_t h2d_bytes() const { return h2d_bytes_; }
  int64_t d2h_bytes() const { return d2h_bytes_; }
  bool download(double *lValues, bool to_device, std::string &err);
  cudaStream_t stream() const { return stream_; }
  void set_stream(cudaStream_t s) { stream_ = s ? s : own_stream_; }
  int64_t xsize() const { return xsize_; }
  int n() const { return n_; }
  int nsuper() const { return nsuper_; }
  const Plan &plan() const { return plan_; }
  double *device_L() const { return dL_; }
  int launches_per_factor() const { return plan_.launches; }

 private:
  void release();
  void launch_all(std::vector<std::pair<int, cudaEvent_t>> *prof = nullptr);
  int finish(int *info, std::string &err);
  int64_t h2d_bytes_ = 0, d2h_bytes_ = 0;
  int device_ = 0;
  cudaStream_t stream_ = nullptr;
  cudaStream_t own_stream_ = nullptr;
  int n_ = 0, nsuper_ = 0;
  int64_t xsize_ = 0, nnz_ = 0;
  // device buffers
  int *d_super_ = nullptr, *d_Ls_ = nullptr, *d_Ap_ = nullptr, *d_Ai_ = nullptr;
  int64_t *d_rowptr_ = nullptr, *d_xptr_ = nullptr;
  int *d_upd_ptr_ = nullptr, *d_upd_ = nullptr;
  double *d_Ax_ = nullptr, *dL_ = nullptr;
  int *d_status_ = nullptr, *h_status_ = nullptr;
  int *d_small_ = nullptr, *d_big_ = nullptr;
  int2 *d_asm_ = nullptr, *d_panel_ = nullptr;
  int4 *d_upd_tasks_ = nullptr, *d_syrk_ = nullptr;
  Plan plan_;
  DevSym sym_{};
};

// kernel launch wrappers (swc_kernels.cu)
void launch_factor_small(const DevSym &S, const int *list, int count, int smem, cudaStream_t st);
void launch_assemble(const DevSym &S, const int2 *tasks, int count, cudaStream_t st);
void launch_update_tiles(const DevSym &S, const int4 *tasks, int count, cudaStream_t st);
void launch_potrf_first(const DevSym &S, const int *list, int count, cudaStream_t st);
void launch_trsm_step(const DevSym &S, const int2 *tasks, int count, int step, cudaStream_t st);
void launch_syrk_step(const DevSym &S, const int4 *tasks, int count, int step, cudaStream_t st);
void launch_init_status(int *status, cudaStream_t st);
bool kernels_configure(std::string &err);

}  // namespace swc
