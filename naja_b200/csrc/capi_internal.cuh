// Helpers shared by the C-ABI translation units.
#pragma once
#include <cuda_runtime.h>

#include <initializer_list>
#include <string>

struct naja_polytope;

namespace naja {

// Device the polytope lives on (capi.cu).
int polytope_device(const naja_polytope* P);

// Records `msg` as this thread's last error and returns `code`.
int fail(int code, const std::string& msg);

// Where `p` lives: 0 host memory of any kind (or null), 1 device memory of
// the current device or managed memory, -1 device memory of another device.
int ptr_location(const void* p);

// True for device or managed memory, false for host memory of any kind.
bool is_device_ptr(const void* p);

// NAJA_ERR_INVALID_ARGUMENT (message names `fn` and the argument's position
// in `ptrs`) when a pointer is plain device memory of a device other than the
// current one: kernels of this call would fault on it unless peer access
// happened to be enabled.  Null pointers and host memory pass.
int require_local(const char* fn, std::initializer_list<const void*> ptrs);

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

// Tensor-core backmap pieces (backmap_tc.cu), shared by naja_backmap,
// naja_backmap_noalloc and the sampling pipeline.  Modes NAJA_BACKMAP_BF16X3
// and NAJA_BACKMAP_TF32X3; every pointer is device memory.
//
// Bytes of one split operand (the hi or the lo half) of `rows` rows of d
// values: rows x (d rounded up to 64) elements of 2 (BF16) or 4 (TF32) bytes,
// rounded up to 1 KiB.
size_t backmap_tc_operand_bytes(long long rows, int d, int mode);
// T (n x d column-major, ldt) -> its split halves Th, Tl.
int backmap_tc_split_T(int n, int d, const double* T, int ldt, void* Th, void* Tl, int mode, cudaStream_t stream);
// Splits Y (N rows of d values, y_dtype) into Yh, Yl and launches the GEMM
// V = Y T^T + shift against the split T; a bounded wait that expires sets
// err[0..3].  Asynchronous: nothing is read back.
int backmap_tc_enqueue(int n, int d, long long N, const void* Y, int y_dtype, const void* Th, const void* Tl, void* Yh,
                       void* Yl, const double* shift, void* V, int v_dtype, int mode, int* err, cudaStream_t stream);
// Synchronises `stream` and turns a set error word into NAJA_ERR_DEVICE.
int backmap_tc_read_error(const int* err, cudaStream_t stream, const char* who);
// FP64 SIMT backmap launch (backmap.cu), asynchronous, device pointers.
int backmap_fp64_enqueue(int n, int d, long long N, const double* T, int ldt, const double* shift, const void* Y,
                         int y_dtype, void* V, int v_dtype, cudaStream_t stream);
// Allocating and allocation-free one-shot forms (synchronise `stream`).
int backmap_tc(int n, int d, long long N, const double* T, int ldt, const double* shift, const void* Y, int y_dtype,
               void* V, int v_dtype, int mode, cudaStream_t stream);
int backmap_tc_noalloc(int n, int d, long long N, const double* T, int ldt, const double* shift, const void* Y,
                       int y_dtype, void* V, int v_dtype, int mode, cudaStream_t stream);

}  // namespace naja
