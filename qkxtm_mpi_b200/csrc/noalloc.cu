// noalloc.cu -- the allocation-free variant of the reCdotXdagY reduction.
//
// Some callers cannot allocate device memory: code that runs with a fixed
// device-memory budget that another allocator (a framework's caching pool, a
// job that reserved the whole GPU up front) already owns, or that must not
// call into the allocator at all on its path.  Such a caller cannot create a
// qkx_ctx (that allocates work fields), so this entry point takes only the
// caller's own device fields and keeps its scratch -- the per-block partial
// sums and the final sum -- in a fixed array compiled into this library.
//
// That array lives in device memory on every GPU that loads the library,
// from load until process exit.  Its size caps the input: at most
// QKX_NOALLOC_MAX_SITES sites (larger inputs are rejected before any launch).
// Every call on a device shares the one array: each call writes all the
// partials it later reads, so nothing has to be cleared, but calls whose GPU
// work overlaps (different streams, or different host threads) race on it.
#include <stdint.h>

#include <mutex>

#include "blas.cuh"
#include "qkx_b200.h"
#include "qkx_ctx.cuh"

namespace {

constexpr int NA_NT = 256;           // threads per block
constexpr int NA_PER_THREAD = 8;     // complex numbers per thread
constexpr size_t NA_PER_BLOCK = (size_t)NA_NT * NA_PER_THREAD;
constexpr size_t NA_MAX_BLOCKS = 65536;
constexpr int NA_MAX_DEVICES = 64;

// [0, NA_MAX_BLOCKS): partial sums, one per block; [NA_MAX_BLOCKS]: the result
static __device__ __align__(256) double g_noalloc_scratch[NA_MAX_BLOCKS + 1];

// the array's device address per device, looked up once; a cudaDeviceReset of a
// device invalidates it, so a process that resets a device must not call again
std::mutex g_na_mu;
double* g_na_ptr[NA_MAX_DEVICES] = {};

// Re sum conj(x) y over this block's range of complex numbers
__global__ void __launch_bounds__(NA_NT) k_na_partials(const double2* __restrict__ x, const double2* __restrict__ y,
                                                       size_t n, double* __restrict__ part) {
  const size_t base = (size_t)blockIdx.x * NA_PER_BLOCK;
  double acc = 0.0;
#pragma unroll
  for (int k = 0; k < NA_PER_THREAD; k++) {
    const size_t i = base + (size_t)k * NA_NT + threadIdx.x;
    if (i < n) {
      const double2 a = x[i], b = y[i];
      acc += a.x * b.x + a.y * b.y;
    }
  }
  const double s = qkx::block_sum<NA_NT>(acc);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// the partials summed in a fixed order into part[NA_MAX_BLOCKS]
__global__ void __launch_bounds__(1024) k_na_final(double* __restrict__ part, int nblocks) {
  double acc = 0.0;
  for (int i = threadIdx.x; i < nblocks; i += 1024) acc += part[i];
  const double s = qkx::block_sum<1024>(acc);
  if (threadIdx.x == 0) part[NA_MAX_BLOCKS] = s;
}

// A field pointer the kernel may read: 16-byte aligned (the kernel reads double2)
// and device or managed memory that the current device `dev` can address.
// Host memory, registered or not, is refused: reading it from the kernel would
// fault the GPU or read across PCIe.  cudaPointerGetAttributes allocates nothing.
bool na_field_ok(const void* p, int dev, const char* name) {
  if (((uintptr_t)p & 15u) != 0) {
    qkx::set_error("invalid argument: %s is not 16-byte aligned", name);
    return false;
  }
  cudaPointerAttributes a{};
  const cudaError_t e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) {
    cudaGetLastError();  // the query records its (non-sticky) error; clear it
    qkx::set_error("invalid argument: %s is not a CUDA pointer (%s)", name, cudaGetErrorString(e));
    return false;
  }
  if (a.type == cudaMemoryTypeManaged) return true;
  if (a.type != cudaMemoryTypeDevice) {
    qkx::set_error("invalid argument: %s is not device memory", name);
    return false;
  }
  if (a.device != dev) {
    qkx::set_error("invalid argument: %s lives on device %d, the current device is %d", name, a.device, dev);
    return false;
  }
  return true;
}

}  // namespace

extern "C" int qkx_reCdotXdagY_noalloc(const double* x_dev, const double* y_dev, size_t n_sites, double* result,
                                       void* stream) {
  if (!x_dev || !y_dev || !result) {
    qkx::set_error("invalid argument: NULL pointer");
    return QKX_ERR_INVALID;
  }
  if (n_sites > QKX_NOALLOC_MAX_SITES) {
    qkx::set_error("invalid argument: %zu sites exceed the %llu-site limit of the allocation-free dot product",
                   n_sites, (unsigned long long)QKX_NOALLOC_MAX_SITES);
    return QKX_ERR_INVALID;
  }
  if (n_sites == 0) {
    *result = 0.0;
    return QKX_OK;
  }
  int dev = 0;
  QKX_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= NA_MAX_DEVICES) {
    qkx::set_error("device index %d above %d", dev, NA_MAX_DEVICES - 1);
    return QKX_ERR_INVALID;
  }
  if (!na_field_ok(x_dev, dev, "x") || !na_field_ok(y_dev, dev, "y")) return QKX_ERR_INVALID;
  cudaStream_t st = (cudaStream_t)stream;
  {
    // the result is read back with a synchronizing copy, which a capturing stream cannot do
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    QKX_CUDA(cudaStreamIsCapturing(st, &cs));
    if (cs != cudaStreamCaptureStatusNone) {
      qkx::set_error("invalid argument: the stream is capturing; this call synchronizes and cannot be captured");
      return QKX_ERR_INVALID;
    }
  }
  double* scratch = nullptr;
  {
    // first call on this device: look up the device address of the array
    std::lock_guard<std::mutex> lock(g_na_mu);
    if (!g_na_ptr[dev]) {
      double* p = nullptr;
      cudaError_t e = cudaGetSymbolAddress((void**)&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p) {
        qkx::set_error("cudaGetSymbolAddress of the scratch array failed: %s", cudaGetErrorString(e));
        return QKX_ERR_CUDA;
      }
      g_na_ptr[dev] = p;
    }
    scratch = g_na_ptr[dev];
  }
  const size_t n = 12 * n_sites;  // complex numbers
  const int nblocks = (int)((n + NA_PER_BLOCK - 1) / NA_PER_BLOCK);
  k_na_partials<<<nblocks, NA_NT, 0, st>>>((const double2*)x_dev, (const double2*)y_dev, n, scratch);
  k_na_final<<<1, 1024, 0, st>>>(scratch, nblocks);
  QKX_CUDA(cudaGetLastError());
  QKX_CUDA(cudaMemcpyAsync(result, scratch + NA_MAX_BLOCKS, sizeof(double), cudaMemcpyDeviceToHost, st));
  QKX_CUDA(cudaStreamSynchronize(st));
  return QKX_OK;
}
