// The HIP runtime calls of SELF's memory layer, served by the CUDA runtime.
//
// SELF's Fortran allocates and moves every device array through hipfort's
// bind(c) interfaces (src/SELF_Memory.f90:11-12 `USE hipfort`; GPUAvailable
// :336-350 calls hipGetDeviceCount; the hfReal_rN/hfInt32_rN Alloc, Free,
// UpdateDevice and UpdateHost routines call hipMalloc, hipFree and hipMemcpy,
// e.g. :362, :767-777, :988-1033; src/SELF_Mesh.f90:2043-2050 picks the rank's
// GPU with hipGetDeviceCount and hipSetDevice).  Those interfaces bind the C
// symbols of the HIP runtime.  Exporting the same five symbols from
// libselfgpu lets the Fortran memory layer run unchanged on a machine with
// only CUDA: link hipfort's interface modules against this library instead
// of the HIP runtime (never both in one process).
//
// Argument conventions are hipfort's: hipMalloc(void** ptr, size_t bytes),
// hipMemcpy(void* dst, const void* src, size_t bytes, int kind) with
// hipMemcpyKind values 0..4 (host-to-host, host-to-device, device-to-host,
// device-to-device, default; the same numbering as cudaMemcpyKind),
// hipFree(void*), hipGetDeviceCount(int*), hipSetDevice(int).  The return
// value is hipError_t: 0 on success; the CUDA runtime's error codes that HIP
// shares (1 invalid value, 2 out of memory, 100 no device, 101 invalid
// device) pass through, any other failure is reported as 999 (unknown).
// Like the HIP runtime, hipMemcpy is synchronous with respect to the host
// and ordered on the legacy default stream, so it also orders with the
// engine's default (blocking) stream.
#include <cuda_runtime.h>

#include <cstddef>

#include "selfgpu_internal.h"

namespace {

int hip_status(cudaError_t e) {
  // a failed call leaves its code as the runtime's last error; clear it so
  // that a later, unrelated cudaGetLastError() does not report it again
  if (e != cudaSuccess) cudaGetLastError();
  switch (e) {
    case cudaSuccess: return 0;
    case cudaErrorInvalidValue: return 1;
    case cudaErrorMemoryAllocation: return 2;
    case cudaErrorNoDevice: return 100;
    case cudaErrorInvalidDevice: return 101;
    default: return 999;
  }
}

}  // namespace

extern "C" {

int hipMalloc(void** ptr, size_t sizeBytes) {
  if (ptr == nullptr) return hip_status(cudaErrorInvalidValue);
  *ptr = nullptr;
  if (sizeBytes == 0) return 0;  // HIP returns success and a null pointer for a zero-byte request
  return hip_status(cudaMalloc(ptr, sizeBytes));
}

int hipFree(void* ptr) { return hip_status(cudaFree(ptr)); }

int hipMemcpy(void* dst, const void* src, size_t sizeBytes, int kind) {
  if (kind < 0 || kind > 4) return hip_status(cudaErrorInvalidValue);
  if (sizeBytes == 0) return 0;
  return hip_status(cudaMemcpy(dst, src, sizeBytes, static_cast<cudaMemcpyKind>(kind)));
}

int hipGetDeviceCount(int* count) {
  if (count == nullptr) return hip_status(cudaErrorInvalidValue);
  cudaError_t e = cudaGetDeviceCount(count);
  if (e != cudaSuccess) *count = 0;
  return hip_status(e);
}

int hipSetDevice(int deviceId) { return hip_status(cudaSetDevice(deviceId)); }

}  // extern "C"
