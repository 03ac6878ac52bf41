// Library state kept once per device and shared by every context on it.
//
// * The fitted coefficients of the straight-line kernels live in their
//   __constant__ banks, which exist once per device.  They are loaded with
//   the models' fitted values the first time anything runs on a device
//   (mbx_device_constants); that step copies to constant memory only and
//   allocates nothing, so the allocation-free entry point can take it too.
// * The term tables of all evaluators (one embedded binary) and a copy of
//   every evaluator's coefficients in global memory, read by the
//   table-driven kernels, are uploaded on the first context creation on a
//   device (mbx_device_tables; allocates once per device, freed at exit).
//
// mbx_set_coefficients changes the coefficients of an evaluator on its
// context's device, for every context there: the coefficients are per device,
// not per context.  It takes the device-state lock and waits for the device to
// be idle before it writes, so that no kernel in flight on another stream
// reads half-updated values.
#pragma once
#include <cuda_runtime.h>

#include <mutex>

struct DeviceTables {
    const unsigned char* blob = nullptr;   // device copy of the term-table binary
    double* coef = nullptr;                // every evaluator's coefficients, at coef_off[evaluator]
};

// Loads the fitted coefficients into the constant banks of device dev (once).
// Returns an MBX_* code.
int mbx_device_constants(int dev);
// Term tables and global-memory coefficients of device dev (uploaded once).
int mbx_device_tables(int dev, DeviceTables* out);
// Offset of an evaluator's coefficients in DeviceTables::coef.
long mbx_coef_offset(int evaluator);
// The lock that serialises coefficient changes and first-time set-up.
std::mutex& mbx_device_mutex();
