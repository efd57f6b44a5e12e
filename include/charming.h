// charming-b200: the user-facing device API.
//
// Same names and signatures as the reference's include/charming.h:11-35.
// A program defines charm::main (device, run once per PE thread block with
// all of its threads) and, optionally, charm::main_host (host, run before the
// launch); it links against libcharming.a, which owns the process main().
#ifndef _CHARMING_H_
#define _CHARMING_H_

#include "chare.h"
#include "message.h"
#include "kernel.h"

namespace charm {

// Main function executed on the host before the scheduler launch. Optional:
// the library declares it weak, so programs without one still link (the
// reference calls it unconditionally, src/charming.cu:73).
void main_host(int argc, char** argv);

// Main function executed on all PEs, with all threads of each PE block.
__device__ void main(int argc, char** argv, size_t* argvs, int pe);

// Runtime functions that can be called by the user.
// end(): the first call from any thread of any PE stops every PE after its
// current entry method; messages still in flight are dropped (reference:
// src/charming.cu:265-267, src/sched/scheduler.cu:60-66, :123-153).
__device__ void end();
// abort(): stops the calling PE only (src/charming.cu:270-277).
__device__ void abort();

__device__ int my_pe();
__device__ int n_pes();
__device__ int my_pe_node();
__device__ int n_pes_node();
__device__ int n_nodes();

// Barriers over all PE blocks (block-collective).
__device__ void barrier();
__device__ void barrier_local();

__device__ int device_atoi(const char* str, int strlen);

// Memory of the calling PE for the program's own use (reference
// include/charming.h:33-34, GPU-level mode only there; here on every PE).
// malloc_user returns `size` bytes (16-byte aligned) of the PE's heap region
// in device memory, readable and writable by every PE of the GPU, and sets
// `offset` to the block's offset in that region; nullptr when the region has
// no room. free_user(size, offset) returns the block; space comes back in
// allocation order once the older blocks are freed too. Single-threaded;
// blocks live until free_user or the end of the run. The region's size per
// PE is CHARMING_USER_HEAP_BYTES (default 1 MiB).
__device__ void* malloc_user(size_t size, size_t& offset);
__device__ void free_user(size_t size, size_t offset);

// ---- Extensions of this runtime (not in the reference) -------------------
// Dynamic shared memory left for entry methods after the runtime's own
// per-PE state; 16-byte aligned. *bytes receives its size.
__device__ void* smem_scratch(size_t* bytes);
// Nanoseconds from the GPU global timer (%globaltimer).
__device__ uint64_t now_ns();
// SM the calling thread runs on (%smid; reference src/util/util.cu:3-7).
__device__ unsigned int smid();

// The threads of the calling PE, for code that runs in both modes: in
// SM-level mode (the default) a PE is one thread block, in GPU-level mode
// (charming_config::gpu_level, or a program compiled with
// -DCHARMING_GPU_LEVEL) every block of the launch. pe_thread() is the
// reference examples' GID (threadIdx.x, or the grid-wide thread index),
// pe_threads() their GROUP_SIZE, pe_sync() their BARRIER_LOCAL
// (__syncthreads, or a barrier over all blocks).
__device__ int pe_thread();
__device__ int pe_threads();
__device__ void pe_sync();
__device__ bool is_gpu_level();

} // namespace charm

#endif // _CHARMING_H_
