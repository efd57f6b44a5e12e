// Built-in programs of libcharming_b200.so. The library's charm::main runs
// the program selected by g_app.id; each program's C ABI entry point fills
// g_app and starts one scheduler run.
#pragma once

#include <charming.h>
#include "../rt.cuh"

namespace suite {

enum app_id : int {
  APP_NONE = 0,
  APP_HELLO = 1,
  APP_REFNUM = 2,
  APP_PINGPONG = 3,
  APP_FANOUT = 4,
  APP_JACOBI2D = 5,
  APP_JACOBI1D = 6,
  APP_SERVE = 7,
  APP_ASYNC_WAIT = 8,
  APP_USER_HEAP = 9,
  APP_DECOMP1D = 10,
};

struct app_params {
  int id;
  int pad;
  long long a[16];
  double d[8];
  void* p[16];
};

// Seeded generators shared with the oracle (oracle/msgmodel.py restates
// them): SplitMix64 finaliser, and the word stream used for payloads.
__host__ __device__ inline unsigned long long mix64(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
__host__ __device__ inline unsigned long long gen_word(unsigned long long seed,
    unsigned long long stream, unsigned long long j) {
  return mix64(seed ^ (stream * 0xD1B54A32D192ED03ULL) ^ (j * 0x9E3779B97F4A7C15ULL));
}

// Position-dependent 64-bit checksum of n bytes, computable in parallel:
// sum over little-endian words w_i (zero-padded) of mix64(w_i ^ (i+1)*K),
// xor n. Block-collective; returns the same value on every thread.
__device__ unsigned long long checksum_block(const void* data, unsigned long long n);
__host__ __device__ inline unsigned long long checksum_word(unsigned long long w,
    unsigned long long i) {
  return mix64(w ^ ((i + 1) * 0xA0761D6478BD642FULL));
}

// The same checksum computed by the 32 lanes of the calling warp alone (for
// small payloads: no block barrier); every lane gets the result.
__device__ unsigned long long checksum_warp(const void* data, unsigned long long n);

// Block-wide sum of one u64 per thread (every thread gets the result).
__device__ unsigned long long block_sum_u64(unsigned long long v);
// Block-wide deterministic FP64 sum: fixed reduction tree for a given
// blockDim, so the result is bit-reproducible run to run.
__device__ double block_sum_f64(double v);

}  // namespace suite

// Parameters of the current run (written by the host before each launch;
// constant memory, so reads stay cached whatever the chares' loads do).
extern __constant__ suite::app_params g_app;

// Program entry points (called from charm::main on every PE, all threads).
namespace suite {
__device__ void hello_main(int pe);
__device__ void refnum_main(int pe);
__device__ void pingpong_main(int pe);
__device__ void fanout_main(int pe);
__device__ void jacobi2d_main(int pe);
__device__ void jacobi1d_main(int pe);
__device__ void serve_main(int pe);
__device__ void async_wait_main(int pe);
__device__ void user_heap_main(int pe);
__device__ void decomp1d_main(int pe);
}  // namespace suite

// Host helper: copy params to g_app and run the scheduler once.
int suite_run(const suite::app_params& p);
