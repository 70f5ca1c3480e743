// Learned SPAI preconditioner (host side): model handle, per-operator slot
// map and features, inference into M values on A's pattern, training.
#pragma once

#include <vector>

#include "runtime.h"
#include "spai_api.h"

struct bksp_gpu_matrix;

struct bksp_gpu_spai_model {
  float* w = nullptr;      // kSpaiParams parameters (device)
  float* am = nullptr;     // Adam first moments
  float* av = nullptr;     // Adam second moments
  float* grad = nullptr;   // last gradient
  double* loss = nullptr;  // last loss (device scalar)
  int step = 0;
  int device = 0;
};

namespace bk {

// Per-operator data of the learned preconditioner, owned by the matrix
// handle: slot of every row entry (near-to-far diagonal order), features.
struct SpaiSlots {
  bool ok = false;           // the operator has <= 3 negative and <= 4
                             // positive diagonal offsets, incl. the diagonal
  int* slot_entry = nullptr; // n x kSlots CSR indices (-1: absent), device
  float* feat = nullptr;     // n x kSlots features, device (lazy)
  float* dinv = nullptr;     // n, device (lazy)
  void release(cudaStream_t st);
};

// Slot map of an uploaded, scanned operator (built on the GPU); leaves
// s.ok false when the operator is not stencil-like.
void spai_build_slots(const DevCsr& A, SpaiSlots& s, cudaStream_t st);
// Scratch floats spai_apply needs: M's CSR values (nnz + 8, padded to 64)
// then, when A has a diagonal form, M's diagonal form, then (symmetric)
// the predicted values before symmetrisation.
long long spai_scratch_floats(const bksp_gpu_matrix* m, bool symmetric = false);
// M (FP32 values in mvals, spai_scratch_floats floats) on A's pattern from
// the model; returns a view sharing A's index arrays and row masks (never
// released).  symmetric: M = (M_pred + M_pred^T) / 2, for CG, whose
// preconditioner must be symmetric.
DevCsr spai_apply(bksp_gpu_spai_model* model, bksp_gpu_matrix* m,
                  float* mvals, cudaStream_t st, bool symmetric = false);

}  // namespace bk
