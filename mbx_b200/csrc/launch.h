// Host-side declarations of the generated per-evaluator launchers
// (gen/<name>_kernels.cu).  Internal to the library; the C ABI is in
// include/mbx_b200.h.
#pragma once
#include <cuda_runtime.h>

struct HolderArgs;

#define MBX_DECLARE_EVALUATOR(name)                                                                   \
    int mbx_set_coef_##name(const double* a, int from_device, cudaStream_t s);                        \
    int mbx_launch_##name(const HolderArgs& A, int mode, int grid, int block, cudaStream_t s);        \
    int mbx_launch_dcoef_##name(const HolderArgs& A, const double* w, double* out, int grid, int block, \
                                cudaStream_t s);

MBX_DECLARE_EVALUATOR(mbpol2b)
MBX_DECLARE_EVALUATOR(mbpol3b)
MBX_DECLARE_EVALUATOR(ch4h2o2b)
MBX_DECLARE_EVALUATOR(ch4ch42b)
MBX_DECLARE_EVALUATOR(ch4h2o3b)
