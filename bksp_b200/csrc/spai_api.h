// Learned SPAI preconditioner: constants and kernel launches shared by
// spai_kernels.cu (device) and spai.cpp (host).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "kernel_api.h"

namespace bk {

constexpr int kSlots = 8;        // stencil slots per row (MLP inputs / outputs)
constexpr int kCenterSlot = 3;   // the diagonal's slot
constexpr int kHidden = 64;      // two hidden layers of this width
constexpr int kSpaiParams = kHidden * kSlots + kHidden + kHidden * kHidden +
                            kHidden + kSlots * kHidden + kSlots;   // 5256

// slot_entry[i * kSlots + sl[q]] = index of row i's first entry with column
// offset so[q] (q < ns), -1 where the row has none.
void launch_spai_slot_map(int n, const int* rowptr, const int* col,
                          const int* so, const int* sl, int ns, int* slot_entry,
                          cudaStream_t st);
void launch_spai_features(int n, const int* rowptr, const double* val,
                          const int* slot_entry, float* feat, float* dinv,
                          cudaStream_t st);
// out = (M + M^T) / 2 on M's (symmetric) pattern, CSR values in and out.
void launch_spai_symmetrize(int n, const int* rowptr, const int* col,
                            const float* in, float* out, cudaStream_t st);
void launch_spai_infer(int n, const float* w, const float* feat,
                       const float* dinv, const int* slot_entry, float* mval,
                       cudaStream_t st);
int spai_grad_blocks(int n);
void launch_spai_grad(int n, const float* w, const float* feat,
                      const float* dinv, const int* slot_entry, const int* col,
                      const float* Z, const float* AZ, int probes,
                      long long ldz, float scale, float* gpart, float* lpart,
                      cudaStream_t st);
void launch_spai_reduce_adam(int nblk, const float* gpart, const float* lpart,
                             float* grad, double* loss, float loss_scale,
                             float* w, float* am, float* av, int step, float lr,
                             cudaStream_t st);
void launch_spai_probes(int n, int probes, long long ldz, uint32_t seed,
                        float* Z, cudaStream_t st);

}  // namespace bk
