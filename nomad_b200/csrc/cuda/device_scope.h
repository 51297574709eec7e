// Device selection for the library's entry points.
#pragma once
#include <cuda_runtime.h>

// Makes a device current for the rest of an entry point's scope and gives the calling thread its
// previous current device back on every return path, so the library never leaves a caller on a
// device other than the one it called with.
struct NomadDeviceScope {
  int prev = -1;
  cudaError_t err = cudaSuccess;
  explicit NomadDeviceScope(int device) {
    if (cudaGetDevice(&prev) != cudaSuccess) {
      cudaGetLastError();
      prev = -1;
    }
    if (prev != device) err = cudaSetDevice(device);
    if (err != cudaSuccess) prev = -1;
  }
  ~NomadDeviceScope() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
  NomadDeviceScope(const NomadDeviceScope &) = delete;
  NomadDeviceScope &operator=(const NomadDeviceScope &) = delete;
};
