// charming-b200: block- and grid-strided memory helpers for device code.
//
// Names and signatures follow the reference's include/kernel.h:6-204 so user
// code keeps compiling. nvshmem_memcpy_block/grid keep their names for that
// reason only: nothing here uses NVSHMEM. The copies move 16-byte vectors
// whenever source and destination share their alignment modulo 16, with a
// scalar head and tail (the reference falls back to 8/4/2/1-byte loops as
// soon as either pointer is misaligned, include/kernel.h:30-116).
#ifndef _KERNEL_H_
#define _KERNEL_H_

#include <stdint.h>
#include <stddef.h>

namespace charm {

__device__ __forceinline__ void memset_kernel_block(void* addr, int val, size_t size) {
  for (size_t i = threadIdx.x; i < size; i += blockDim.x) {
    ((char*)addr)[i] = (char)val;
  }
}

__device__ __forceinline__ void memset_kernel_grid(void* addr, int val, size_t size) {
  for (size_t i = (size_t)blockDim.x * blockIdx.x + threadIdx.x; i < size;
       i += (size_t)gridDim.x * blockDim.x) {
    ((char*)addr)[i] = (char)val;
  }
}

__device__ __forceinline__ void memcpy_kernel_block(void* dst, void* src, size_t size) {
  for (size_t i = threadIdx.x; i < size; i += blockDim.x) {
    ((char*)dst)[i] = ((char*)src)[i];
  }
}

__device__ __forceinline__ void memcpy_kernel_grid(void* dst, void* src, size_t size) {
  for (size_t i = (size_t)blockDim.x * blockIdx.x + threadIdx.x; i < size;
       i += (size_t)gridDim.x * blockDim.x) {
    ((char*)dst)[i] = ((char*)src)[i];
  }
}

// Cooperative copy by `nthr` threads where this thread is `tid`.
// 16-byte vectors when (dst - src) % 16 == 0, else 8/4/1-byte words.
__device__ __forceinline__ void copy_cooperative(void* __restrict__ dst,
    const void* __restrict__ src, size_t len, size_t tid, size_t nthr) {
  char* d = (char*)dst;
  const char* s = (const char*)src;
  if ((((uintptr_t)d ^ (uintptr_t)s) & 15) == 0) {
    size_t head = (16 - ((uintptr_t)d & 15)) & 15;
    if (head > len) head = len;
    for (size_t i = tid; i < head; i += nthr) d[i] = s[i];
    d += head; s += head; len -= head;
    size_t nvec = len >> 4;
    uint4* dv = (uint4*)d;
    const uint4* sv = (const uint4*)s;
    size_t i = tid;
    // Four independent 16-byte loads in flight per thread.
    for (; i + 3 * nthr < nvec; i += 4 * nthr) {
      uint4 a = sv[i], b = sv[i + nthr], c = sv[i + 2 * nthr], e = sv[i + 3 * nthr];
      dv[i] = a; dv[i + nthr] = b; dv[i + 2 * nthr] = c; dv[i + 3 * nthr] = e;
    }
    for (; i < nvec; i += nthr) dv[i] = sv[i];
    d += nvec << 4; s += nvec << 4; len -= nvec << 4;
    for (size_t k = tid; k < len; k += nthr) d[k] = s[k];
  } else if ((((uintptr_t)d ^ (uintptr_t)s) & 7) == 0) {
    size_t head = (8 - ((uintptr_t)d & 7)) & 7;
    if (head > len) head = len;
    for (size_t i = tid; i < head; i += nthr) d[i] = s[i];
    d += head; s += head; len -= head;
    size_t nw = len >> 3;
    for (size_t i = tid; i < nw; i += nthr) ((uint64_t*)d)[i] = ((const uint64_t*)s)[i];
    d += nw << 3; s += nw << 3; len -= nw << 3;
    for (size_t k = tid; k < len; k += nthr) d[k] = s[k];
  } else if ((((uintptr_t)d ^ (uintptr_t)s) & 3) == 0) {
    size_t head = (4 - ((uintptr_t)d & 3)) & 3;
    if (head > len) head = len;
    for (size_t i = tid; i < head; i += nthr) d[i] = s[i];
    d += head; s += head; len -= head;
    size_t nw = len >> 2;
    for (size_t i = tid; i < nw; i += nthr) ((uint32_t*)d)[i] = ((const uint32_t*)s)[i];
    d += nw << 2; s += nw << 2; len -= nw << 2;
    for (size_t k = tid; k < len; k += nthr) d[k] = s[k];
  } else {
    for (size_t i = tid; i < len; i += nthr) d[i] = s[i];
  }
}

__device__ inline void nvshmem_memcpy_block(void* __restrict__ dst,
    const void* __restrict__ src, size_t len) {
  copy_cooperative(dst, src, len, threadIdx.x, blockDim.x);
}

__device__ inline void nvshmem_memcpy_grid(void* __restrict__ dst,
    const void* __restrict__ src, size_t len) {
  copy_cooperative(dst, src, len, (size_t)blockDim.x * blockIdx.x + threadIdx.x,
      (size_t)gridDim.x * blockDim.x);
}

} // namespace charm

#endif // _KERNEL_H_
