// charming_jacobi2d_sweeps_noalloc: Jacobi sweeps of one grid that allocate
// no device memory.
//
// Who needs it: code that runs where allocating is not allowed or not
// possible, e.g. a host that hands this library device buffers from its own
// pool or arena and forbids allocations outside it, a caller inside a
// region where cudaMalloc would synchronise the device, or a process whose
// memory is already fully reserved. charming_jacobi2d_create/run allocate
// the chare grids, staging buffers and the scheduler's inboxes; this entry
// point needs only the caller's input and output grids plus a fixed scratch
// array that is part of the library image.
//
// Scratch: g_noalloc_scratch below, 16 MiB, one per GPU that loads the
// library, held until the process exits. It holds the second (ping-pong)
// grid. Every call overwrites the part it uses before reading it, so
// nothing in it has to start at zero. All calls share it: calls that
// overlap on the GPU (from several host threads, or on several streams)
// race on it and must be serialised by the caller.
//
// The arithmetic is the chares' (jac::stencil), so the result equals the
// grid that charming_jacobi2d_run produces for the same input, bit for bit.
#include "jacobi_sweep.cuh"
#include "../host.cuh"

#include <mutex>

namespace {

constexpr size_t NOALLOC_SCRATCH_BYTES = 16u << 20;
constexpr int NOALLOC_MAX_DEVICES = 64;

// Device-side scratch; in host code this name is only a host stand-in for
// the symbol, never a device address (see scratch_on_current_device).
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

std::mutex g_scratch_mu;
void* g_scratch_ptr[NOALLOC_MAX_DEVICES];  // device address of the scratch, per device
int g_sm_count[NOALLOC_MAX_DEVICES];       // multiprocessors of each device

// Resolves the scratch's device address and the device's multiprocessor
// count on the current device, once per device (the first call on a device
// does this).
int scratch_on_current_device(void** out, int* sms) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return charm_host::cuda_fail(e, "jacobi2d noalloc: cudaGetDevice");
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) {
    charm_host::set_error_text("jacobi2d noalloc: device ordinal out of range");
    return CHARMING_ERR_CONFIG;
  }
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return charm_host::cuda_fail(e, "jacobi2d noalloc: cudaGetSymbolAddress");
    int n = 0;
    e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return charm_host::cuda_fail(e, "jacobi2d noalloc: cudaDeviceGetAttribute");
    g_sm_count[dev] = n > 0 ? n : 1;
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  *sms = g_sm_count[dev];
  return CHARMING_OK;
}

// One sweep src -> dst over the interior of a row-major (ny+2) x (nx+2)
// grid; the boundary ring of dst is already in place.
template <typename T>
__global__ void __launch_bounds__(256) noalloc_sweep_kernel(const T* __restrict__ src,
    T* __restrict__ dst, int nx, int ny) {
  const long long W = nx + 2;
  const long long n = (long long)nx * ny;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    long long r = i / nx + 1, c = i % nx + 1;
    const T* m = src + r * W + c;
    dst[r * W + c] = jac::stencil(m[0], m[-1], m[1], m[-W], m[W]);
  }
}

template <typename T>
int run_sweeps(int nx, int ny, int sweeps, const T* in, T* out, T* scratch, int sms) {
  const size_t bytes = ((size_t)nx + 2) * ((size_t)ny + 2) * sizeof(T);
  // Both buffers start as the input (boundary ring included); the first
  // source is picked so that the last sweep writes `out`.
  cudaError_t e = cudaMemcpyAsync(out, in, bytes, cudaMemcpyDeviceToDevice, 0);
  if (e == cudaSuccess) e = cudaMemcpyAsync(scratch, in, bytes, cudaMemcpyDeviceToDevice, 0);
  T* a = (sweeps % 2 == 0) ? out : scratch;
  T* b = (a == out) ? scratch : out;
  const long long pts = (long long)nx * ny;
  const int blocks = (int)std::min<long long>((pts + 255) / 256, (long long)sms * 8);
  for (int s = 0; s < sweeps && e == cudaSuccess; s++) {
    noalloc_sweep_kernel<T><<<blocks, 256, 0, 0>>>(a, b, nx, ny);
    e = cudaGetLastError();
    T* t = a;
    a = b;
    b = t;
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(0);
  if (e != cudaSuccess) return charm_host::cuda_fail(e, "jacobi2d noalloc sweeps");
  return CHARMING_OK;
}

}  // namespace

extern "C" int charming_jacobi2d_sweeps_noalloc(int dtype, int nx, int ny, int sweeps,
    const void* dev_in, void* dev_out) {
  if (dtype != CHARMING_F64 && dtype != CHARMING_F32) {
    charm_host::set_error_text("jacobi2d noalloc: dtype must be CHARMING_F64 or CHARMING_F32");
    return CHARMING_ERR_CONFIG;
  }
  if (nx < 1 || ny < 1 || sweeps < 0 || !dev_in || !dev_out) {
    charm_host::set_error_text("jacobi2d noalloc: bad arguments");
    return CHARMING_ERR_CONFIG;
  }
  const size_t esz = dtype == CHARMING_F64 ? 8 : 4;
  // A misaligned element pointer would fault in the kernel's loads.
  if (reinterpret_cast<uintptr_t>(dev_in) % esz || reinterpret_cast<uintptr_t>(dev_out) % esz) {
    charm_host::set_error_text("jacobi2d noalloc: dev_in and dev_out must be aligned to the element size");
    return CHARMING_ERR_CONFIG;
  }
  const unsigned long long cells = ((unsigned long long)nx + 2) * ((unsigned long long)ny + 2);
  if (cells > NOALLOC_SCRATCH_BYTES / esz) {
    charm_host::set_error_text(
        "jacobi2d noalloc: grid larger than the 16 MiB scratch ((nx+2)*(ny+2)*element size must "
        "be <= 16 MiB)");
    return CHARMING_ERR_CONFIG;
  }
  const char* i0 = static_cast<const char*>(dev_in);
  const char* o0 = static_cast<const char*>(dev_out);
  const size_t bytes = cells * esz;
  if (i0 < o0 + bytes && o0 < i0 + bytes) {
    charm_host::set_error_text("jacobi2d noalloc: input and output grids overlap");
    return CHARMING_ERR_CONFIG;
  }
  void* scratch = nullptr;
  int sms = 1;
  int rc = scratch_on_current_device(&scratch, &sms);
  if (rc) return rc;
  if (dtype == CHARMING_F64)
    return run_sweeps<double>(nx, ny, sweeps, static_cast<const double*>(dev_in),
                              static_cast<double*>(dev_out), static_cast<double*>(scratch), sms);
  return run_sweeps<float>(nx, ny, sweeps, static_cast<const float*>(dev_in),
                           static_cast<float*>(dev_out), static_cast<float*>(scratch), sms);
}
