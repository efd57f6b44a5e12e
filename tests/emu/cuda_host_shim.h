// Host-compilation shim for the Jacobi chare code (TEST INFRASTRUCTURE).
//
// Lets g++ compile charming_b200/csrc/apps/jacobi2d.cu for the CPU, so that
// the exact C++ of the chare state machine, halo pack/unpack and both
// sweeps runs on host threads (tests/emu/jacobi_emu.cpp provides the
// runtime). Two builds:
//
//   default  one host thread per PE, blockDim.x == 1; block-static
//            __shared__ variables become thread_local (one per PE). Built
//            with AddressSanitizer: catches out-of-bounds accesses of the
//            chare logic across many PEs and message orders. Direct sweep.
//   EMU_MT   one PE whose block has blockDim.x host threads; __shared__
//            variables are plain statics shared by the block, and
//            __syncthreads() is a real barrier that checks every thread
//            arrives at the same call site (a barrier reached from
//            different places aborts the run). Warp-level calls run the
//            32 threads of a warp in lockstep, and the TMA sweep runs on a
//            model of mbarriers and asynchronous bulk copies. Built with
//            ThreadSanitizer: catches thread-0-writes / other-threads-read
//            races that a one-thread block cannot show.
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
#define __noinline__
#define __constant__
#ifdef EMU_MT
#define __shared__ static
#else
#define __shared__ thread_local
#endif
#define __launch_bounds__(...)
#define __restrict__

struct emu_dim3 {
  unsigned x, y, z;
};
extern thread_local emu_dim3 threadIdx;
extern thread_local emu_dim3 blockIdx;
extern emu_dim3 blockDim;
extern emu_dim3 gridDim;

// Block barrier of the calling PE; `file`/`line` identify the call site.
void emu_sync(const char* file, int line);
#define __syncthreads() emu_sync(__FILE__, __LINE__)

#ifdef EMU_MT
// Warps of 32 host threads in lockstep at every warp-level call; the TMA
// sweep runs on modelled mbarriers and bulk copies (jacobi_emu.cpp).
#define CHARMING_HOST_EMULATION_TMA 1
void emu_syncwarp(const char* file, int line);
#define __syncwarp(...) emu_syncwarp(__FILE__, __LINE__)
bool emu_all_sync(bool p);
bool emu_any_sync(bool p);
unsigned emu_match_any(long long v);
inline unsigned __match_any_sync(unsigned, long long v) { return emu_match_any(v); }
inline unsigned __match_any_sync(unsigned, int v) { return emu_match_any(v); }
void emu_shfl(void* v, unsigned bytes, int mode, int arg);  // mode 0 up, 1 down, 2 xor, 3 index
inline bool __all_sync(unsigned, bool p) { return emu_all_sync(p); }
inline bool __any_sync(unsigned, bool p) { return emu_any_sync(p); }
template <typename T> inline T __shfl_up_sync(unsigned, T v, int d) {
  emu_shfl(&v, sizeof(T), 0, d);
  return v;
}
template <typename T> inline T __shfl_down_sync(unsigned, T v, int d) {
  emu_shfl(&v, sizeof(T), 1, d);
  return v;
}
template <typename T> inline T __shfl_xor_sync(unsigned, T v, int m) {
  emu_shfl(&v, sizeof(T), 2, m);
  return v;
}
template <typename T> inline T __shfl_sync(unsigned, T v, int src) {
  emu_shfl(&v, sizeof(T), 3, src);
  return v;
}
#else
inline unsigned __match_any_sync(unsigned, long long) { return 1u; }
inline unsigned __match_any_sync(unsigned, int) { return 1u; }
inline void __syncwarp(unsigned = 0xffffffffu) {}
inline bool __all_sync(unsigned, bool p) { return p; }
inline bool __any_sync(unsigned, bool p) { return p; }
// one thread per block: the partner lane of a butterfly does not exist and
// contributes nothing
template <typename T> inline T __shfl_xor_sync(unsigned, T v, int o) { return o ? T(0) : v; }
template <typename T> inline T __shfl_up_sync(unsigned, T v, int) { return v; }
template <typename T> inline T __shfl_down_sync(unsigned, T v, int) { return v; }
template <typename T> inline T __shfl_sync(unsigned, T v, int) { return v; }
#endif
inline void __threadfence() { std::atomic_thread_fence(std::memory_order_seq_cst); }
inline void __threadfence_system() { std::atomic_thread_fence(std::memory_order_seq_cst); }
inline void __nanosleep(unsigned) {}
inline bool __isLocal(const void*) { return true; }
inline int __ffs(unsigned x) { return x ? __builtin_ffs((int)x) : 0; }
inline int __popc(unsigned x) { return __builtin_popcount(x); }
inline long long clock64() { return 0; }

template <typename T> inline T atomicAdd(T* p, T v) { return __atomic_fetch_add(p, v, __ATOMIC_SEQ_CST); }
template <typename T> inline T atomicAdd_block(T* p, T v) { return atomicAdd(p, v); }
template <typename T> inline T atomicExch(T* p, T v) { return __atomic_exchange_n(p, v, __ATOMIC_SEQ_CST); }
template <typename T> inline T atomicCAS(T* p, T c, T v) {
  __atomic_compare_exchange_n(p, &c, v, false, __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST);
  return c;
}
template <typename T> inline T atomicExch_block(T* p, T v) { return atomicExch(p, v); }
// system scope (other GPUs): the same C++ atomics; in the two-process check
// they act on memory both processes map
template <typename T> inline T atomicAdd_system(T* p, T v) { return atomicAdd(p, v); }
template <typename T> inline T atomicExch_system(T* p, T v) { return atomicExch(p, v); }
template <typename T> inline T atomicCAS_system(T* p, T c, T v) { return atomicCAS(p, c, v); }
template <typename T> inline T atomicCAS_block(T* p, T c, T v) { return atomicCAS(p, c, v); }
inline void __threadfence_block() { std::atomic_thread_fence(std::memory_order_seq_cst); }
template <typename T> inline T atomicMax(T* p, T v) {
  T old = __atomic_load_n(p, __ATOMIC_SEQ_CST);
  while (v > old && !__atomic_compare_exchange_n(p, &old, v, false, __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST)) {
  }
  return old;
}
template <typename T> inline T atomicMin(T* p, T v) {
  T old = __atomic_load_n(p, __ATOMIC_SEQ_CST);
  while (v < old && !__atomic_compare_exchange_n(p, &old, v, false, __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST)) {
  }
  return old;
}

inline double __dadd_rn(double a, double b) { return a + b; }
inline double __dsub_rn(double a, double b) { return a - b; }
inline double __dmul_rn(double a, double b) { return a * b; }
inline double __ddiv_rn(double a, double b) { return a / b; }
inline float __fadd_rn(float a, float b) { return a + b; }
inline float __fmul_rn(float a, float b) { return a * b; }
inline float __fmaf_rn(float a, float b, float c) { return std::fma(a, b, c); }
inline float __double2float_rn(double a) { return (float)a; }

struct alignas(16) double2 { double x, y; };
struct alignas(16) float4 { float x, y, z, w; };
struct alignas(16) uint4 { unsigned x, y, z, w; };
inline double2 make_double2(double a, double b) { return double2{a, b}; }
inline float4 make_float4(float a, float b, float c, float d) { return float4{a, b, c, d}; }

using std::min;
using std::max;
inline size_t __cvta_generic_to_shared(const void* p) { return (size_t)p; }

// Stand-in for the scheduler's dynamic shared memory: one per PE thread for
// the runtime check (EMU_RT), referenced but unused by the chare checks.
#ifdef EMU_RT
extern thread_local uint64_t* s_mem_of_pe;  // set by each PE thread
#define s_mem s_mem_of_pe
// whether p lies in the calling PE block's stand-in shared memory
bool emu_is_shared(const void* p);
inline bool __isShared(const void* p) { return emu_is_shared(p); }
#else
extern uint64_t s_mem[];
#endif
