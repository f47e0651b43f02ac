// Helpers shared by the C-ABI translation units.
#pragma once
#include <cuda_runtime.h>

#include <string>

namespace naja {

// Records `msg` as this thread's last error and returns `code`.
int fail(int code, const std::string& msg);

// True for device or managed memory, false for host memory of any kind.
bool is_device_ptr(const void* p);

// Makes `device` current for the scope, restoring the previous device.
class DeviceGuard {
 public:
  explicit DeviceGuard(int device);
  ~DeviceGuard();
  bool ok() const { return ok_; }

 private:
  int prev_ = 0;
  bool ok_ = true;
  bool switched_ = false;
};

// Stream-ordered scratch allocation freed at scope exit.
struct DeviceBuffer {
  void* ptr = nullptr;
  size_t bytes = 0;
  cudaStream_t stream = nullptr;
  DeviceBuffer() = default;
  DeviceBuffer(const DeviceBuffer&) = delete;
  DeviceBuffer& operator=(const DeviceBuffer&) = delete;
  ~DeviceBuffer();
  int alloc(size_t nbytes, cudaStream_t s);
};

// Device view of `n` bytes at `p`: `p` itself when it is device memory,
// else a copy staged into `buf` on stream `s`.
int device_view(const void* p, size_t n, cudaStream_t s, DeviceBuffer& buf, const void** out);

}  // namespace naja
