// charming-b200: runtime constants and print macros shared by the device API.
//
// Source-compatible with the reference's include/common.h (print macros at
// include/common.h:7-13, topology constants at :15-34). The reference's
// SM-level shared-memory slot table (s_idx, :37-51) and the PE/CE rank maths
// (:53-85) are internal to its NVSHMEM transport; this runtime has no CE, so a
// PE is simply a thread block and those helpers are not part of the API.
#ifndef _COMMON_H_
#define _COMMON_H_

#include <stdio.h>
#include <stdint.h>
#include <stddef.h>
#include <new>  // placement new in device code

// Scheduling mode. By default one PE per thread block (the reference's
// -DSM_LEVEL build), and examples that branch on SM_LEVEL pick that branch.
// A program compiled with -DCHARMING_GPU_LEVEL takes its GPU-level branch
// (the reference's default build: GID over the whole grid, BARRIER_LOCAL =
// charm::barrier_local()), and the weak symbol below asks the library's
// process main for GPU-level mode, in which all blocks form one PE.
#ifdef CHARMING_GPU_LEVEL
extern "C" __attribute__((weak)) const int charming_program_gpu_level = 1;
#elif !defined(SM_LEVEL)
#define SM_LEVEL 1
#endif

namespace charm {
// Comparisons of chare_proxy<C>::async_wait, with the values of the
// NVSHMEM_CMP_* constants the reference passes there.
enum : int { CMP_EQ = 0, CMP_NE = 1, CMP_GT = 2, CMP_LE = 3, CMP_LT = 4, CMP_GE = 5 };
}  // namespace charm

// Print functions (include/common.h:7-13 of the reference)
#define PINFO(...) printf("[INFO] " __VA_ARGS__)
#define PERROR(...) printf("[ERROR] " __VA_ARGS__)
#ifdef DEBUG
#define PDEBUG(...) printf("[DEBUG] " __VA_ARGS__)
#else
#define PDEBUG(...) do {} while (0)
#endif

// Execution-environment constants, written by the host before the scheduler
// launch (reference: src/charming.cu:172-187). One GPU: c_my_dev = 0,
// c_n_devs = c_n_nodes = 1, c_n_pes = number of PE thread blocks.
extern __constant__ int c_n_sms;
extern __constant__ int c_my_dev;
extern __constant__ int c_my_dev_node;
extern __constant__ int c_n_devs;
extern __constant__ int c_n_devs_node;
extern __constant__ int c_n_nodes;
extern __constant__ int c_n_pes;
extern __constant__ int c_n_pes_node;

// Dynamic shared memory of the scheduler kernel. The runtime keeps its
// per-PE state at the front; charm::smem_scratch() hands out the rest.
#ifndef CHARMING_HOST_EMULATION  // the CPU check of app code has no PE block memory
extern __shared__ uint64_t s_mem[];
#endif

#endif // _COMMON_H_
