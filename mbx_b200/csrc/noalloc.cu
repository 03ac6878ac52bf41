// mbx_evaluate_noalloc: the evaluator entry point for callers that cannot
// allocate device memory.
//
// Some callers run where cudaMalloc is off limits: inside a host callback or
// an allocator-free real-time loop, under a memory pool that must not grow, or
// from a plugin that owns no CUDA context state of its own.  mbx_evaluate
// stages its work counter, its energy/virial accumulators and (when the caller
// does not want them) the per-n-mer energies in buffers the context allocates.
// This variant takes only caller-owned inputs and outputs and keeps its
// scratch in one file-scope device array, sized for at most
// MBX_NOALLOC_MAX_NMERS n-mers; every GPU that loads the library holds that
// array (about 2 MiB) until the process exits.
//
// The scratch holds the evaluation kernel's work counter and the switched
// energy of every n-mer; the total energy is then summed over those per-n-mer
// energies in a fixed order by one block, so it is the same bit for bit from
// call to call (the atomics-based total of mbx_evaluate is not).
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "../../include/mbx_b200.h"
#include "device_state.h"
#include "holder_kernel.cuh"

#define MBX_NOALLOC_HEAD 32   // doubles reserved in front of the per-n-mer energies (slot 0: work counter)

// File-scope scratch.  In host code this name is only a stand-in for the
// symbol; the device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) double mbx_noalloc_scratch[MBX_NOALLOC_HEAD + MBX_NOALLOC_MAX_NMERS];

int mbx_launch_mbpol2b_g(const HolderArgs& A, int grid, int block, cudaStream_t s);
int mbx_launch_mbpol3b_g(const HolderArgs& A, int grid, int block, cudaStream_t s);
int mbx_launch_ch4h2o2b_g(const HolderArgs& A, int grid, int block, cudaStream_t s);
int mbx_launch_ch4h2o3b_g(const HolderArgs& A, int grid, int block, cudaStream_t s);
int mbx_launch_mbpol2b_e(const HolderArgs& A, int grid, int block, cudaStream_t s);
int mbx_launch_mbpol3b_e(const HolderArgs& A, int grid, int block, cudaStream_t s);
int mbx_launch_ch4h2o2b_e(const HolderArgs& A, int grid, int block, cudaStream_t s);
int mbx_launch_ch4h2o3b_e(const HolderArgs& A, int grid, int block, cudaStream_t s);

namespace {

struct NoallocEval {
    const char* name;
    int nreal;
    int (*launch)(const HolderArgs&, int, int, cudaStream_t);         // energy + gradient
    int (*launch_e)(const HolderArgs&, int, int, cudaStream_t);       // energy only (grad == NULL)
};

const NoallocEval kEvals[] = {
    {"mbpol2b", 6, mbx_launch_mbpol2b_g, mbx_launch_mbpol2b_e},
    {"mbpol3b", 9, mbx_launch_mbpol3b_g, mbx_launch_mbpol3b_e},
    {"ch4h2o2b", 8, mbx_launch_ch4h2o2b_g, mbx_launch_ch4h2o2b_e},
    {"ch4h2o3b", 11, mbx_launch_ch4h2o3b_g, mbx_launch_ch4h2o3b_e},
};

// Device address of the scratch array, looked up once per device with that
// device current.
constexpr int kMaxDevices = 64;
double* g_scratch[kMaxDevices] = {nullptr};
std::mutex g_scratch_mu;

int scratch_for(int dev, double** out) {
    if (dev < 0 || dev >= kMaxDevices) return MBX_EINVAL;
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, mbx_noalloc_scratch);
        if (e != cudaSuccess || !p) return MBX_ECUDA;
        g_scratch[dev] = static_cast<double*>(p);
    }
    *out = g_scratch[dev];
    return MBX_OK;
}

// Fixed-order sum of e[0..n): each thread adds a contiguous slice in order,
// then a shared-memory tree in a fixed pattern.  Writes result[0].
__global__ void __launch_bounds__(1024) k_fixed_order_sum(const double* __restrict__ e, long n,
                                                          double* __restrict__ result) {
    __shared__ double part[1024];
    const long per = (n + blockDim.x - 1) / blockDim.x;
    const long b = threadIdx.x * per;
    const long end = b + per < n ? b + per : n;
    double s = 0.0;
    for (long i = b; i < end; ++i) s += e[i];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) result[0] = part[0];
}

}  // namespace

// Declared in include/mbx_b200.h.
extern "C" int mbx_evaluate_noalloc(const char* evaluator, long n, const double* xyz, double* grad, double* e_per,
                                    double* result, void* stream) {
    if (!evaluator || n < 0 || (n > 0 && !xyz) || !result) return MBX_EINVAL;
    if (n > MBX_NOALLOC_MAX_NMERS) return MBX_EINVAL;
    const NoallocEval* E = nullptr;
    for (const auto& x : kEvals)
        if (!strcmp(x.name, evaluator)) E = &x;
    if (!E) return MBX_ENOTSUP;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return MBX_ENODEV;
    // the models' fitted coefficients in the kernels' constant banks: loaded
    // by the first call on a device that no context has loaded them on
    // (constant-memory copies only, no allocation)
    int rc = mbx_device_constants(dev);
    if (rc) return rc;
    double* scratch = nullptr;
    rc = scratch_for(dev, &scratch);
    if (rc) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // the array keeps the previous call's contents: the counter must restart
    // at zero and the result is accumulated from zero
    if (cudaMemsetAsync(scratch, 0, MBX_NOALLOC_HEAD * sizeof(double), s) != cudaSuccess) return MBX_ECUDA;
    if (cudaMemsetAsync(result, 0, 7 * sizeof(double), s) != cudaSuccess) return MBX_ECUDA;
    double* eper = e_per ? e_per : scratch + MBX_NOALLOC_HEAD;
    if (n > 0) {
        HolderArgs A;
        memset(&A, 0, sizeof(A));
        A.n = n;
        A.aos = 1;
        A.xyz = xyz;
        A.grad = grad;
        A.out = result;
        A.e_per = eper;
        A.counter = reinterpret_cast<int*>(scratch);
        if ((grad ? E->launch : E->launch_e)(A, 1, 128, s) != 0) return MBX_ECUDA;
        k_fixed_order_sum<<<1, 1024, 0, s>>>(eper, n, result);
        if (cudaGetLastError() != cudaSuccess) return MBX_ECUDA;
    }
    return MBX_OK;
}
