// Tensor-core trailing updates of the large fronts of the FP32 factor
// (factor_tc.cu).  Host-side launchers; the kernels are sm_100a only.
#pragma once

#include <cuda_runtime.h>

namespace psipm {

// Status bit a tensor-core kernel ORs into *err when a wait on the tensor
// core's completion barrier ran out.  The factor passes its fail word, whose
// bit 0 marks a failed pivot; the host tells the two apart.
constexpr int kTcErrWait = 1 << 20;

// F[i, j] -= sum_{k < kb} F[i, k0 + k] F[j, k0 + k] for k0 + kb <= j <= i < r,
// j < jend; F column-major r x r (the lower triangle is used).  `passes` is 3
// (3xTF32: hi*hi + hi*lo + lo*hi, FP32-level products) or 1 (plain TF32).
// Throws psipm::Failure on a launch error.
void syrk_update_tc(float* F, int r, int k0, int kb, int jend, int passes, int* err, cudaStream_t st);

// Dynamic shared memory the update needs (for occupancy planning and tests).
size_t syrk_update_tc_smem();

}  // namespace psipm
