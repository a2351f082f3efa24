// Read-only view of a prepared PPE handle for other solvers of this library
// (the network-preconditioned flexible CG).  Internal; not part of the C ABI.
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>

#include "../../include/tpf.h"

namespace tpf {

struct PpeView {
  int ndim;
  int n0, n1, n2;   // nodes per axis (n2 = 1 in 2-D)
  int N0, N1, N2;   // cells per axis (N2 = 0 in 2-D)
  int ndof, pin;
  const double* s[3];     // symmetric face couplings of S = -W L (upper face of each node)
  const double* dinvS;    // 1 / diag(S), pin -> 1
  const double* dv[3];    // control-volume widths per axis
  bool prepared;
};

int ppe_view(tpf_ppe* h, PpeView* v);
int ppe_options(tpf_ppe* h, tpf_ppe_options* o);

// U-Net internals used by the learned solver (unet.cu)
int unet_dims(const tpf_unet* n, int* H, int* W, int* max_batch);
__nv_bfloat16* unet_input(tpf_unet* n);
const float* unet_output(tpf_unet* n);
int unet_forward_packed(tpf_unet* n, int B, cudaStream_t s);
int unet_prepare_weights(tpf_unet* n, cudaStream_t s);
int unet_check(tpf_unet* n, cudaStream_t s);

}  // namespace tpf
