// charm::main of libcharming_b200.so and helpers shared by the programs.
#include "suite.cuh"
#ifndef CHARMING_HOST_EMULATION  // the CPU check of the runtime has no CUDA API
#include "../host.cuh"
#endif

__constant__ suite::app_params g_app;

namespace {
__shared__ unsigned long long s_red_u64[32];
__shared__ double s_red_f64[32];
}

__device__ void charm::main(int argc, char** argv, size_t* argvs, int pe) {
  // In GPU-level mode every block runs each entry method: only programs
  // written against pe_thread()/pe_threads()/pe_sync() can run there.
  if (charm::is_gpu_level() && g_app.id != suite::APP_DECOMP1D && g_app.id != suite::APP_NONE) {
    if (charm::pe_thread() == 0) charm::rt::set_error(CHARMING_ERR_CONFIG, g_app.id, 1);
    return;
  }
  // Over several processes only the message programs run: the others keep
  // their grids and logs in one process's memory.
  if (charm::rt::c_rt.n_procs > 1 && g_app.id != suite::APP_HELLO && g_app.id != suite::APP_REFNUM &&
      g_app.id != suite::APP_PINGPONG && g_app.id != suite::APP_FANOUT && g_app.id != suite::APP_NONE) {
    if (threadIdx.x == 0) charm::rt::set_error(CHARMING_ERR_CONFIG, g_app.id, 2);
    return;
  }
  switch (g_app.id) {
    case suite::APP_HELLO: suite::hello_main(pe); break;
    case suite::APP_REFNUM: suite::refnum_main(pe); break;
    case suite::APP_PINGPONG: suite::pingpong_main(pe); break;
    case suite::APP_FANOUT: suite::fanout_main(pe); break;
    case suite::APP_JACOBI2D: suite::jacobi2d_main(pe); break;
    case suite::APP_JACOBI1D: suite::jacobi1d_main(pe); break;
    case suite::APP_SERVE: suite::serve_main(pe); break;
    case suite::APP_ASYNC_WAIT: suite::async_wait_main(pe); break;
    case suite::APP_USER_HEAP: suite::user_heap_main(pe); break;
    case suite::APP_DECOMP1D: suite::decomp1d_main(pe); break;
    default:
      if (charm::pe_thread() == 0 && pe == 0) charm::end();
      break;
  }
}

__device__ unsigned long long suite::block_sum_u64(unsigned long long v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = (blockDim.x + 31) >> 5;
  __syncthreads();
  if (l == 0) s_red_u64[w] = v;
  __syncthreads();
  unsigned long long r = 0;
  for (int i = 0; i < nw; i++) r += s_red_u64[i];
  __syncthreads();
  return r;
}

__device__ double suite::block_sum_f64(double v) {
  // Fixed tree: butterfly within each warp, then warps in index order.
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = (blockDim.x + 31) >> 5;
  __syncthreads();
  if (l == 0) s_red_f64[w] = v;
  __syncthreads();
  double r = 0.0;
  for (int i = 0; i < nw; i++) r += s_red_f64[i];
  __syncthreads();
  return r;
}

__device__ unsigned long long suite::checksum_block(const void* data, unsigned long long n) {
  const unsigned char* b = reinterpret_cast<const unsigned char*>(data);
  unsigned long long nw = (n + 7) / 8, acc = 0;
  bool aligned = (reinterpret_cast<uintptr_t>(b) & 7) == 0;
  for (unsigned long long i = threadIdx.x; i < nw; i += blockDim.x) {
    unsigned long long w = 0;
    if (aligned && 8 * i + 8 <= n) {
      w = reinterpret_cast<const unsigned long long*>(b)[i];
    } else {
      for (int k = 0; k < 8; k++) {
        unsigned long long j = 8 * i + k;
        if (j < n) w |= (unsigned long long)b[j] << (8 * k);
      }
    }
    acc += checksum_word(w, i);
  }
  return block_sum_u64(acc) ^ n;
}

__device__ unsigned long long suite::checksum_warp(const void* data, unsigned long long n) {
  const unsigned char* b = reinterpret_cast<const unsigned char*>(data);
  const unsigned long long nw = (n + 7) / 8;
  const bool aligned = (reinterpret_cast<uintptr_t>(b) & 7) == 0;
  unsigned long long acc = 0;
  const unsigned stride = blockDim.x < 32 ? blockDim.x : 32;  // blocks under a warp (host checks)
  for (unsigned long long i = threadIdx.x & 31; i < nw; i += stride) {
    unsigned long long w = 0;
    if (aligned && 8 * i + 8 <= n) {
      w = reinterpret_cast<const unsigned long long*>(b)[i];
    } else {
      for (int k = 0; k < 8; k++) {
        const unsigned long long j = 8 * i + k;
        if (j < n) w |= (unsigned long long)b[j] << (8 * k);
      }
    }
    acc += checksum_word(w, i);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  return acc ^ n;
}

#ifndef CHARMING_HOST_EMULATION
int suite_run(const suite::app_params& p) {
  int rc = charm_host::ensure_init();
  if (rc) return rc;
  cudaError_t e = cudaMemcpyToSymbol(g_app, &p, sizeof(p));
  if (e != cudaSuccess) return charm_host::cuda_fail(e, "program parameters");
  char name[] = "charming_b200";
  char* argv[] = {name, nullptr};
  return charm_host::run_scheduler(1, argv);
}
#endif
