// Helpers shared by the C entry-point files.
#pragma once

#include <cuda_runtime.h>

#include <chrono>
#include <vector>

#include "../../include/bksp.h"
#include "../../include/bksp_gpu.h"
#include "runtime.h"
#include "spai.h"

// Device-resident operator handle of bksp_gpu.h.
struct bksp_gpu_matrix {
  bk::DevCsr A;
  bk::DevCsr At;
  bool has_t = false;
  int flags = 0;
  int device = 0;
  // Jacobi preconditioner M = diag(A)^-1 as a one-entry-per-row CSR (FP32).
  bk::DevCsr jacobi;
  bool has_jacobi = false;
  bool diag_ok = false;       // every diagonal entry present and non-zero
  bk::SpaiSlots spai;         // learned-preconditioner slot map / features
};

namespace bk {

extern thread_local bksp_gpu_stats* g_stats;

bool is_symmetric(const dspmat* A);
int check_matrix(const dspmat* A);
double* upload_vec(const double* h, int n, long long cols, cudaStream_t st);
void download_vec(double* h, const double* d, int n, long long cols,
                  cudaStream_t st);
void upload_operator(const dspmat* A, bool expand, bool want_fp32, DevCsr& out,
                     cudaStream_t st);
int hist_cap_for(int max_iter);

// Device + wall timing of one call, reported into the recorded stats.
struct Timer {
  cudaStream_t st;
  cudaEvent_t e0, e1;
  std::chrono::steady_clock::time_point t0;
  explicit Timer(cudaStream_t s);
  ~Timer();
  void begin_solve();
  void end_solve();
  void report(int ret, const SolveState* ss, int hist_len);
};

}  // namespace bk
