// Sweep throughput without the messages: n_blocks thread blocks (the
// runtime's PE shape: its threads, its dynamic shared memory) each run
// `passes` passes over their own pitched chare block, with the chare code's
// sweep functions and the chare layout (depth ghost rows and columns, row 0
// at depth-1 rows into the buffer). All four sides are taken as the domain
// boundary and no halos move, so only the sweep is timed. For measuring and
// profiling the sweep kernels; the results are not checked here (the chare
// runs are, against the oracle).
//   variant 0: multi-sweep pass, phase-split items (depth >= 2)
//           1: multi-sweep pass, single-loop items (depth >= 2)
//           2: one sweep per pass, direct strip walker (depth 1)
#include "suite.cuh"
#include "jacobi_sweep.cuh"
#ifndef CHARMING_HOST_EMULATION
#include "../host.cuh"

namespace {

template <typename T>
__global__ void __launch_bounds__(charm::rt::MAX_THREADS, 1) sweep_bench_kernel(char* base,
    size_t block_bytes, size_t buf_bytes, int pitch, int w, int h, int depth, int passes, int variant) {
  char* mine = base + (size_t)blockIdx.x * block_bytes;
  T* buf[2] = {reinterpret_cast<T*>(mine) + (size_t)(depth - 1) * pitch,
               reinterpret_cast<T*>(mine + buf_bytes) + (size_t)(depth - 1) * pitch};
  for (int p = 0; p < passes; p++) {
    jac::block_view<T> in{buf[p & 1], pitch}, out{buf[(p + 1) & 1], pitch};
    __syncthreads();
    if (variant == 2) jac::sweep_direct<T, false>(in, out, w, h);
    else jac::sweep_deep<T, false>(in, out, w, h, depth, 15, variant == 0);
    __syncthreads();
  }
}

}  // namespace

extern "C" int charming_sweep_bench(int dtype, int w, int h, int depth, int passes, int n_blocks,
    int variant, double* ms) {
  int rc = charm_host::ensure_init();
  if (rc) return rc;
  if ((dtype != CHARMING_F64 && dtype != CHARMING_F32) || w < 1 || h < 1 || passes < 1 ||
      n_blocks < 1 || variant < 0 || variant > 2 || !ms || depth < 1 || depth > jac::DEPTH_MAX ||
      (variant == 2) != (depth == 1))
    return CHARMING_ERR_CONFIG;
  const charming_info& inf = charm_host::info();
  if (n_blocks > inf.n_pes) return CHARMING_ERR_CONFIG;  // one resident block per PE slot
  const int esz = dtype == CHARMING_F64 ? 8 : 4;
  const int off = 128 / esz, vec = 16 / esz, align_el = 128 / esz;
  const int pitch = (off + w + depth + 2 * vec + align_el - 1) / align_el * align_el;
  const size_t buf_bytes = ((size_t)pitch * (h + 2 * depth) * esz + 255) / 256 * 256;
  const size_t block_bytes = 2 * buf_bytes;
  char* d = nullptr;
  cudaError_t e = cudaMalloc(&d, block_bytes * n_blocks);
  if (e != cudaSuccess) return charm_host::cuda_fail(e, "sweep bench blocks");
  e = cudaMemset(d, 0, block_bytes * n_blocks);
  const void* fn = dtype == CHARMING_F64 ? (const void*)sweep_bench_kernel<double>
                                         : (const void*)sweep_bench_kernel<float>;
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, inf.smem_bytes_per_pe);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  void* args[] = {&d, (void*)&block_bytes, (void*)&buf_bytes, (void*)&pitch, &w, &h, &depth, &passes, &variant};
  size_t bb = block_bytes, fb = buf_bytes;
  int pt = pitch;
  args[1] = &bb;
  args[2] = &fb;
  args[3] = &pt;
  cudaStream_t s = charm_host::stream();
  if (e == cudaSuccess) e = cudaEventRecord(e0, s);
  if (e == cudaSuccess)
    e = cudaLaunchKernel(fn, dim3(n_blocks), dim3(inf.threads_per_pe), args, (size_t)inf.smem_bytes_per_pe, s);
  if (e == cudaSuccess) e = cudaEventRecord(e1, s);
  if (e == cudaSuccess) e = cudaEventSynchronize(e1);
  float f = 0.f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&f, e0, e1);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(d);
  if (e != cudaSuccess) return charm_host::cuda_fail(e, "sweep bench");
  *ms = f;
  return CHARMING_OK;
}
#endif
