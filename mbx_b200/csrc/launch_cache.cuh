// Per-device launch facts of one kernel, looked up once per device.
//
// A kernel's dynamic-shared-memory limit (cudaFuncSetAttribute) and its
// occupancy belong to the device that is current when they are set or asked
// for, so they are cached per device: the first launch on each device sets
// the attribute and reads the SM count and the resident blocks per SM with
// that device current.  std::call_once makes the first launches from several
// host threads safe.
#pragma once
#include <cuda_runtime.h>

#include <mutex>

#define MBX_MAX_DEVICES 64

struct LaunchCache {
    std::once_flag once[MBX_MAX_DEVICES];
    int sms[MBX_MAX_DEVICES] = {0};
    int bps[MBX_MAX_DEVICES] = {0};
    int err[MBX_MAX_DEVICES] = {0};
};

// smem_attr: dynamic shared memory the kernel may use at most (0: leave the
// attribute alone); block / smem_occ: the launch shape whose resident blocks
// per SM are wanted (block 0: not needed).  Returns a cudaError_t value.
template <class K>
int launch_facts(LaunchCache& lc, K kern, int block, int smem_attr, int smem_occ, int* sms, int* bps) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return (int)e;
    if (dev < 0 || dev >= MBX_MAX_DEVICES) return (int)cudaErrorInvalidDevice;
    std::call_once(lc.once[dev], [&] {
        int s = 0, b = 1;
        cudaError_t r = cudaDeviceGetAttribute(&s, cudaDevAttrMultiProcessorCount, dev);
        if (r == cudaSuccess && smem_attr > 0)
            r = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_attr);
        if (r == cudaSuccess && block > 0) r = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kern, block, smem_occ);
        lc.sms[dev] = s;
        lc.bps[dev] = b < 1 ? 1 : b;
        lc.err[dev] = (int)r;
    });
    *sms = lc.sms[dev];
    *bps = lc.bps[dev];
    return lc.err[dev];
}
