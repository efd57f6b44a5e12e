// Host-compilation shim for the Jacobi chare code (TEST INFRASTRUCTURE).
//
// Lets g++ compile charming_b200/csrc/apps/jacobi2d.cu for the CPU, so that
// the exact C++ of the chare state machine, halo pack/unpack and direct
// sweep can run under AddressSanitizer. Each emulated PE is one host thread
// and its PE block has a single thread (blockDim.x == 1, threadIdx.x == 0):
// block-level barriers become no-ops and block-static __shared__ variables
// become thread_local. The TMA pipeline is excluded
// (CHARMING_HOST_EMULATION); tests/emu/jacobi_emu.cpp provides the runtime.
#pragma once

#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <algorithm>

#define CHARMING_HOST_EMULATION 1
#define __device__
#define __host__
#define __global__
#define __forceinline__ inline
#define __constant__
#define __shared__ thread_local
#define __launch_bounds__(...)
#define __restrict__

struct emu_dim3 {
  unsigned x, y, z;
};
extern thread_local emu_dim3 threadIdx;
extern thread_local emu_dim3 blockIdx;
extern emu_dim3 blockDim;
extern emu_dim3 gridDim;

inline void __syncthreads() {}
inline void __syncwarp(unsigned = 0xffffffffu) {}
inline void __threadfence() { std::atomic_thread_fence(std::memory_order_seq_cst); }
inline void __nanosleep(unsigned) {}
inline bool __isLocal(const void*) { return true; }
inline bool __all_sync(unsigned, bool p) { return p; }
template <typename T> inline T __shfl_xor_sync(unsigned, T v, int) { return v; }
template <typename T> inline T __shfl_up_sync(unsigned, T v, int) { return v; }
template <typename T> inline T __shfl_down_sync(unsigned, T v, int) { return v; }
inline long long clock64() { return 0; }

template <typename T> inline T atomicAdd(T* p, T v) { return __atomic_fetch_add(p, v, __ATOMIC_SEQ_CST); }
template <typename T> inline T atomicAdd_block(T* p, T v) { return atomicAdd(p, v); }
template <typename T> inline T atomicExch(T* p, T v) { return __atomic_exchange_n(p, v, __ATOMIC_SEQ_CST); }
template <typename T> inline T atomicCAS(T* p, T c, T v) {
  __atomic_compare_exchange_n(p, &c, v, false, __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST);
  return c;
}
template <typename T> inline T atomicMin(T* p, T v) {
  T old = *p;
  if (v < old) *p = v;
  return old;
}

inline double __dadd_rn(double a, double b) { return a + b; }
inline double __dsub_rn(double a, double b) { return a - b; }
inline double __dmul_rn(double a, double b) { return a * b; }
inline double __ddiv_rn(double a, double b) { return a / b; }
inline float __fadd_rn(float a, float b) { return a + b; }
inline float __double2float_rn(double a) { return (float)a; }

struct alignas(16) double2 { double x, y; };
struct alignas(16) float4 { float x, y, z, w; };
struct alignas(16) uint4 { unsigned x, y, z, w; };
inline double2 make_double2(double a, double b) { return double2{a, b}; }
inline float4 make_float4(float a, float b, float c, float d) { return float4{a, b, c, d}; }

using std::min;
using std::max;
inline size_t __cvta_generic_to_shared(const void* p) { return (size_t)p; }
