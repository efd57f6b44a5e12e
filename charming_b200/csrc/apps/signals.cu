// Programs that exercise async_wait and the per-PE user heap.
//
// async_wait chain (reference: chare_proxy::async_wait, include/chare.h:
// 214-239, and the scheduler's check, src/comm/get/get.cu:1172-1202): chare
// i registers a wait on its two signal words (both >= 1); the chare before
// it in the chain sets them when it wakes. The host sets chare 0's words.
// With `broken` set, nobody signals the last chare, whose wait then never
// completes: the run ends at the idle timeout with an error status.
//
// User heap (reference: malloc_user / free_user, src/comm/get/get.cu:
// 1348-1362): every chare takes rounds of blocks of seeded sizes from its
// PE's heap, fills them with a seeded pattern, checks them and frees them in
// a scrambled order. Once every chare has done so (chare 0 counts), each
// hands one block to the next chare, on another PE, which checks the
// pattern there and acknowledges, and the owner frees it. (A block that
// stays allocated holds back the space of every later one, as in the
// reference, so the hand-off comes after the rounds.)
#include "suite.cuh"
#ifndef CHARMING_HOST_EMULATION  // the CPU check of the runtime has no CUDA API
#include "../host.cuh"
#endif

namespace {

// ---- async_wait chain ------------------------------------------------------
// g_app: a[0] n chares, a[1] broken; p[0] signal words (u64[2n]), p[1] wake
// order (int[n]), p[2] wake counter (u64).
struct WaitChare : charm::chare {
  __device__ WaitChare() {}
};
__shared__ charm::chare_proxy<WaitChare>* wait_proxy;

enum : int { EP_W_START = 0, EP_W_WOKEN = 1 };

__device__ void w_start(WaitChare& c, void* arg) {
  if (threadIdx.x == 0) {
    uint64_t* sig = reinterpret_cast<uint64_t*>(g_app.p[0]) + 2 * (size_t)c.i;
    wait_proxy->async_wait(sig, 2, charm::CMP_GE, 1, c.i, EP_W_WOKEN);
  }
  __syncthreads();
}

__device__ void w_woken(WaitChare& c, void* arg) {
  using namespace charm::rt;
  __shared__ int s_last;
  if (threadIdx.x == 0) {
    const int n = (int)g_app.a[0];
    const bool broken = g_app.a[1] != 0;
    unsigned long long pos = atomicAdd(reinterpret_cast<unsigned long long*>(g_app.p[2]), 1ULL);
    reinterpret_cast<int*>(g_app.p[1])[c.i] = (int)pos;
    s_last = c.i == n - 1;
    const int next = c.i + 1;
    if (next < n && !(broken && next == n - 1)) {
      unsigned long long* sig = reinterpret_cast<unsigned long long*>(g_app.p[0]) + 2 * (size_t)next;
      st_release_u64(sig, 1);
      st_release_u64(sig + 1, 1);
    }
  }
  __syncthreads();
  if (s_last) charm::end();
}

// ---- user heap -------------------------------------------------------------
// g_app: a[0] n chares, a[1] blocks per round (<= 16), a[2] rounds, a[3] seed;
// p[0] counters (u64[8]): 0 blocks taken, 1 pattern errors, 2 allocation
// failures, 3 blocks checked on another PE, 4 blocks freed, 5 chares done,
// 6 bytes taken.
struct HeapChare : charm::chare {
  int ready;  // chare 0: chares done with their rounds
  __device__ HeapChare() : ready(0) {}
};
__shared__ charm::chare_proxy<HeapChare>* heap_proxy;

enum : int { EP_H_START = 0, EP_H_CHECK = 1, EP_H_ACK = 2, EP_H_READY = 3, EP_H_NOTE = 4 };
constexpr int HEAP_BLOCKS_MAX = 16;

struct heap_note {  // message: a block to check on another PE
  unsigned long long ptr;
  unsigned long long bytes;
  unsigned long long stream;
  unsigned long long offset;
  int owner;
  int pad[3];
};

__device__ __forceinline__ unsigned long long* heap_ctr() {
  return reinterpret_cast<unsigned long long*>(g_app.p[0]);
}

__device__ unsigned long long heap_block_bytes(int chare, int round, int k) {
  return 48 + 16 * (unsigned long long)((chare * 31 + round * 7 + k * 13) % 61);
}

// All threads: fills `bytes` at p with the pattern of `stream`.
__device__ void heap_fill(unsigned char* p, unsigned long long bytes, unsigned long long stream) {
  const unsigned long long seed = (unsigned long long)g_app.a[3];
  for (unsigned long long j = threadIdx.x; j < bytes / 8; j += blockDim.x)
    reinterpret_cast<unsigned long long*>(p)[j] = suite::gen_word(seed, stream, j);
}

// All threads: words of the block that differ from the pattern.
__device__ unsigned long long heap_check(const unsigned char* p, unsigned long long bytes,
    unsigned long long stream) {
  const unsigned long long seed = (unsigned long long)g_app.a[3];
  unsigned long long bad = 0;
  for (unsigned long long j = threadIdx.x; j < bytes / 8; j += blockDim.x)
    bad += reinterpret_cast<const unsigned long long*>(p)[j] != suite::gen_word(seed, stream, j);
  return suite::block_sum_u64(bad);
}

// All threads: counts one chare as finished; the last ends the run.
__device__ void heap_chare_done() {
  __shared__ int s_end;
  if (threadIdx.x == 0)
    s_end = atomicAdd(&heap_ctr()[5], 1ULL) + 1 == (unsigned long long)g_app.a[0];
  __syncthreads();
  if (s_end) charm::end();
}

__device__ void h_start(HeapChare& c, void* arg) {
  const int B = (int)g_app.a[1], R = (int)g_app.a[2];
  __shared__ unsigned char* s_ptr[HEAP_BLOCKS_MAX];
  __shared__ size_t s_off[HEAP_BLOCKS_MAX];
  unsigned long long bad = 0, taken = 0, failed = 0, freed = 0, bytes = 0;
  for (int r = 0; r < R; r++) {
    if (threadIdx.x == 0) {
      for (int k = 0; k < B; k++) {
        size_t off = 0;
        s_ptr[k] = reinterpret_cast<unsigned char*>(charm::malloc_user(heap_block_bytes(c.i, r, k), off));
        s_off[k] = off;
        if (s_ptr[k]) {
          taken++;
          bytes += heap_block_bytes(c.i, r, k);
        } else {
          failed++;
        }
      }
    }
    __syncthreads();
    for (int k = 0; k < B; k++) {
      if (!s_ptr[k]) continue;
      heap_fill(s_ptr[k], heap_block_bytes(c.i, r, k), ((unsigned long long)c.i << 32) | (unsigned)(r * B + k));
    }
    __syncthreads();
    for (int k = 0; k < B; k++) {
      if (!s_ptr[k]) continue;
      bad += heap_check(s_ptr[k], heap_block_bytes(c.i, r, k), ((unsigned long long)c.i << 32) | (unsigned)(r * B + k));
    }
    if (threadIdx.x == 0) {
      for (int j = 0; j < B; j++) {  // newest first in odd rounds, rotated in even ones
        const int k = (r & 1) ? B - 1 - j : (j + r / 2) % B;
        if (s_ptr[k]) {
          charm::free_user(heap_block_bytes(c.i, r, k), s_off[k]);
          freed++;
        }
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    atomicAdd(&heap_ctr()[0], taken);
    atomicAdd(&heap_ctr()[1], bad);
    atomicAdd(&heap_ctr()[2], failed);
    atomicAdd(&heap_ctr()[4], freed);
    atomicAdd(&heap_ctr()[6], bytes);
  }
  __syncthreads();
  heap_proxy->invoke(0, EP_H_READY);
}

__device__ void h_ready(HeapChare& c, void* arg) {
  if (threadIdx.x == 0) c.ready++;
  __syncthreads();
  if (c.ready == c.n) heap_proxy->invoke_all(EP_H_NOTE);
}

// One block for the next chare to check.
__device__ void h_note(HeapChare& c, void* arg) {
  const int n = (int)g_app.a[0];
  __shared__ heap_note s_note;
  if (threadIdx.x == 0) {
    const unsigned long long bytes = 1024;
    size_t off = 0;
    unsigned char* p = reinterpret_cast<unsigned char*>(charm::malloc_user(bytes, off));
    s_note.ptr = reinterpret_cast<unsigned long long>(p);
    s_note.bytes = bytes;
    s_note.stream = 0xB10C0000ULL + (unsigned long long)c.i;
    s_note.offset = off;
    s_note.owner = c.i;
    atomicAdd(&heap_ctr()[p ? 0 : 2], 1ULL);
  }
  __syncthreads();
  unsigned char* p = reinterpret_cast<unsigned char*>(s_note.ptr);
  if (p) heap_fill(p, s_note.bytes, s_note.stream);
  __syncthreads();
  heap_note m = s_note;
  __syncthreads();
  if (p) {
    heap_proxy->invoke((c.i + 1) % n, EP_H_CHECK, &m, sizeof(m));
  } else {
    heap_chare_done();
  }
}

__device__ void h_check(HeapChare& c, void* arg) {
  const heap_note* m = reinterpret_cast<const heap_note*>(arg);
  const unsigned long long bad =
      heap_check(reinterpret_cast<const unsigned char*>(m->ptr), m->bytes, m->stream);
  heap_note back = *m;
  if (threadIdx.x == 0) {
    atomicAdd(&heap_ctr()[1], bad);
    atomicAdd(&heap_ctr()[3], 1ULL);
  }
  __syncthreads();
  heap_proxy->invoke(back.owner, EP_H_ACK, &back, sizeof(back));
}

__device__ void h_ack(HeapChare& c, void* arg) {
  if (threadIdx.x == 0) {
    const heap_note* m = reinterpret_cast<const heap_note*>(arg);
    charm::free_user(m->bytes, (size_t)m->offset);
    atomicAdd(&heap_ctr()[4], 1ULL);
  }
  __syncthreads();
  heap_chare_done();
}

}  // namespace

__device__ void suite::async_wait_main(int pe) {
  if (threadIdx.x == 0) {
    wait_proxy = new charm::chare_proxy<WaitChare>();
    wait_proxy->add_entry_method<&w_start>();
    wait_proxy->add_entry_method<&w_woken>();
    wait_proxy->create((int)g_app.a[0]);
  }
  __syncthreads();
  for (int i = wait_proxy->start_idx; i <= wait_proxy->end_idx && wait_proxy->n_local > 0; i++)
    wait_proxy->invoke(i, EP_W_START);
}

__device__ void suite::user_heap_main(int pe) {
  if (threadIdx.x == 0) {
    heap_proxy = new charm::chare_proxy<HeapChare>();
    heap_proxy->add_entry_method<&h_start>();
    heap_proxy->add_entry_method<&h_check>();
    heap_proxy->add_entry_method<&h_ack>();
    heap_proxy->add_entry_method<&h_ready>();
    heap_proxy->add_entry_method<&h_note>();
    heap_proxy->create((int)g_app.a[0]);
  }
  __syncthreads();
  for (int i = heap_proxy->start_idx; i <= heap_proxy->end_idx && heap_proxy->n_local > 0; i++)
    heap_proxy->invoke(i, EP_H_START);
}

#ifndef CHARMING_HOST_EMULATION
extern "C" int charming_async_wait_chain(int n_chares, int broken, int* order, int n_order) {
  int rc = charm_host::ensure_init();
  if (rc) return rc;
  if (n_chares < 1 || !order || n_order < n_chares) return CHARMING_ERR_CONFIG;
  unsigned long long* d = nullptr;
  const size_t words = 2 * (size_t)n_chares + 1 + ((size_t)n_chares + 1) / 2;
  cudaError_t e = cudaMalloc(&d, 8 * words);
  if (e != cudaSuccess) return charm_host::cuda_fail(e, "async_wait chain buffers");
  cudaMemset(d, 0, 8 * words);
  int* d_order = reinterpret_cast<int*>(d + 2 * (size_t)n_chares + 1);
  cudaMemset(d_order, 0xff, sizeof(int) * n_chares);
  const unsigned long long one[2] = {1, 1};
  cudaMemcpy(d, one, sizeof(one), cudaMemcpyHostToDevice);  // chare 0 may start
  suite::app_params p{};
  p.id = suite::APP_ASYNC_WAIT;
  p.a[0] = n_chares;
  p.a[1] = broken;
  p.p[0] = d;
  p.p[1] = d_order;
  p.p[2] = d + 2 * (size_t)n_chares;
  rc = suite_run(p);
  cudaMemcpy(order, d_order, sizeof(int) * n_chares, cudaMemcpyDeviceToHost);
  cudaFree(d);
  return rc;
}

extern "C" int charming_user_heap_check(int n_chares, int blocks_per_round, int rounds, uint64_t seed,
    uint64_t* counters) {
  int rc = charm_host::ensure_init();
  if (rc) return rc;
  if (n_chares < 2 || blocks_per_round < 1 || blocks_per_round > HEAP_BLOCKS_MAX || rounds < 0 ||
      !counters)
    return CHARMING_ERR_CONFIG;
  unsigned long long* d = nullptr;
  cudaError_t e = cudaMalloc(&d, 64);
  if (e != cudaSuccess) return charm_host::cuda_fail(e, "user heap counters");
  cudaMemset(d, 0, 64);
  suite::app_params p{};
  p.id = suite::APP_USER_HEAP;
  p.a[0] = n_chares;
  p.a[1] = blocks_per_round;
  p.a[2] = rounds;
  p.a[3] = (long long)seed;
  p.p[0] = d;
  rc = suite_run(p);
  cudaMemcpy(counters, d, 7 * sizeof(uint64_t), cudaMemcpyDeviceToHost);
  cudaFree(d);
  return rc;
}
#endif
