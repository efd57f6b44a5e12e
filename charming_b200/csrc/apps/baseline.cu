// SM-to-SM pingpong floors: what one message hop costs on this GPU without
// the runtime, to set the runtime's pingpong latency against.
//
// Two thread blocks, forced onto different SMs (each takes more than half of
// an SM's shared memory), bounce a counter n times; block 0 times the round
// trips (%globaltimer and clock64) and reports the one-way time. Modes:
//   0 flag:      thread 0 stores the counter with st.release.gpu, the peer's
//                thread 0 polls it with ld.acquire.gpu (the floor: one store
//                and one load through L2 per hop)
//   1 relaxed:   polls with ld.relaxed.gpu and takes one fence.acq_rel.gpu on
//                a hit (polling without invalidating L1 each time)
//   2 block:     mode 0 plus what any block-collective dispatch adds: a block
//                barrier after the receive and one before the send
//   3 reference: the reference's raw baseline (examples/baseline/
//                baseline.cu:14-138): LOCAL_MAX = 4 slots per (sender,
//                receiver) pair, the sender's block scans its slots at the
//                receiver for a free one and atomicCAS-es a token in, the
//                receiver's block scans all 4 * n_sms slots of its row
//                (atomicMin_block for the lowest occupied), then clears it
//                with atomicCAS; __threadfence and volatile loads as there.
// Every wait is bounded: a wait that runs out sets *err and both blocks stop.
#include "suite.cuh"
#ifndef CHARMING_HOST_EMULATION
#include "../host.cuh"
#endif
#include <climits>

namespace {

using namespace charm::rt;

constexpr int BL_LOCAL_MAX = 4;                       // slots per pair (reference baseline.cu:5)
constexpr unsigned long long BL_WAIT_NS = 2000000000ull;  // any single wait: 2 s at most

struct alignas(128) bl_line {
  unsigned long long v;
  unsigned long long pad[15];
};

// Thread 0: waits until *w == want; false when the wait ran out or the peer
// failed (then *err is set).
template <int MODE>
__device__ bool bl_wait(const unsigned long long* w, unsigned long long want, volatile int* err) {
  const unsigned long long t0 = globaltimer();
  unsigned spins = 0;
  while (true) {
    const unsigned long long v = MODE == 1 ? ld_relaxed_u64(w) : ld_acquire_u64(w);
    if (v == want) {
      if (MODE == 1) fence_acq_rel_gpu();
      return true;
    }
    if ((++spins & 1023) == 0 && (*err || globaltimer() - t0 > BL_WAIT_NS)) {
      *err = 1;
      return false;
    }
  }
}

// Block-collective (reference find_free): a free slot among the sender's
// LOCAL_MAX at the receiver, or -1 (on every thread) when the wait ran out.
__device__ int bl_find_free(volatile unsigned long long* slots, volatile int* err) {
  __shared__ volatile int idx;
  __shared__ int state;  // 0 searching, 1 found, 2 stop
  if (threadIdx.x == 0) state = 0;
  const unsigned long long t0 = globaltimer();
  while (true) {
    if (threadIdx.x == 0) idx = INT_MAX;
    __syncthreads();
    for (int i = threadIdx.x; i < BL_LOCAL_MAX; i += blockDim.x) {
      if (slots[i] == 0) atomicMin_block((int*)&idx, i);
      __threadfence();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      if (idx != INT_MAX) state = 1;
      else if (*err || globaltimer() - t0 > BL_WAIT_NS) {
        *err = 1;
        state = 2;
      }
    }
    __syncthreads();
    const int st = state, found = idx;
    __syncthreads();
    if (st) return st == 1 ? found : -1;
  }
}

// Block-collective (reference find_msg + recv): waits for the lowest
// occupied slot of the receiver's row, takes it and clears it. False (on
// every thread) when the wait ran out.
__device__ bool bl_recv(volatile unsigned long long* row, int n, volatile int* err) {
  __shared__ volatile int idx;
  __shared__ int state;
  if (threadIdx.x == 0) state = 0;
  const unsigned long long t0 = globaltimer();
  while (true) {
    if (threadIdx.x == 0) idx = INT_MAX;
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      if (row[i] != 0) atomicMin_block((int*)&idx, i);
      __threadfence();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      if (idx != INT_MAX) {
        const unsigned long long env = row[idx];
        __threadfence();
        atomicCAS((unsigned long long*)&row[idx], env, 0ULL);
        state = 1;
      } else if (*err || globaltimer() - t0 > BL_WAIT_NS) {
        *err = 1;
        state = 2;
      }
    }
    __syncthreads();
    const int st = state;
    __syncthreads();
    if (st) return st == 1;
  }
}

__global__ void __launch_bounds__(512, 1) sm_pingpong_kernel(int mode, int iters, int warmup,
    bl_line* flags, unsigned long long* slots, int n_slot_sms, unsigned long long* out, int* err_word) {
  const int me = blockIdx.x;
  if (me > 1) return;
  volatile int* err = err_word;
  if (threadIdx.x == 0) reinterpret_cast<unsigned int*>(out + 2)[me] = charm::smid();
  unsigned long long t0 = 0, c0 = 0;
  const int total = warmup + iters;
  if (mode == 3) {
    // the receiver's row holds LOCAL_MAX slots per sender SM
    const int n = BL_LOCAL_MAX * n_slot_sms;
    volatile unsigned long long* my_row = slots + (size_t)me * n;
    volatile unsigned long long* to_peer = slots + (size_t)(1 - me) * n + BL_LOCAL_MAX * me;
    for (int i = 0; i < total; i++) {
      if (i == warmup && me == 0 && threadIdx.x == 0) {
        t0 = globaltimer();
        c0 = clock64();
      }
      bool ok = true;
      if (me == 1) ok = bl_recv(my_row, n, err);
      if (ok) {
        const int f = bl_find_free(to_peer, err);
        if (f < 0) ok = false;
        else if (threadIdx.x == 0) atomicCAS((unsigned long long*)&to_peer[f], 0ULL, 1ULL);
      }
      if (ok && me == 0) ok = bl_recv(my_row, n, err);
      if (!ok) break;  // uniform: the helpers return the same value on every thread
    }
  } else if (mode == 2) {
    __shared__ int s_ok;
    unsigned long long* mine = &flags[me].v;
    unsigned long long* peer = &flags[1 - me].v;
    for (int i = 0; i < total; i++) {
      __syncthreads();
      if (threadIdx.x == 0) {
        if (i == warmup && me == 0) {
          t0 = globaltimer();
          c0 = clock64();
        }
        const unsigned long long k = (unsigned long long)i + 1;
        bool ok = true;
        if (me == 0) {
          st_release_u64(peer, k);
          ok = bl_wait<0>(mine, k, err);
        } else {
          ok = bl_wait<0>(mine, k, err);
          if (ok) st_release_u64(peer, k);
        }
        s_ok = ok;
      }
      __syncthreads();
      if (!s_ok) break;
    }
  } else if (threadIdx.x == 0) {
    unsigned long long* mine = &flags[me].v;
    unsigned long long* peer = &flags[1 - me].v;
    for (int i = 0; i < total; i++) {
      if (i == warmup && me == 0) {
        t0 = globaltimer();
        c0 = clock64();
      }
      const unsigned long long k = (unsigned long long)i + 1;
      bool ok = true;
      if (me == 0) {
        st_release_u64(peer, k);
        ok = mode == 1 ? bl_wait<1>(mine, k, err) : bl_wait<0>(mine, k, err);
      } else {
        ok = mode == 1 ? bl_wait<1>(mine, k, err) : bl_wait<0>(mine, k, err);
        if (ok) st_release_u64(peer, k);
      }
      if (!ok) break;
    }
  }
  if (me == 0 && threadIdx.x == 0) {
    out[0] = globaltimer() - t0;
    out[1] = (unsigned long long)(clock64() - (long long)c0);
  }
}

}  // namespace

#ifndef CHARMING_HOST_EMULATION
extern "C" int charming_sm_pingpong(int mode, int round_trips, double* oneway_ns, double* oneway_cycles,
    int* sm_pair) {
  int rc = charm_host::ensure_init();
  if (rc) return rc;
  if (mode < 0 || mode > 3 || round_trips < 1 || !oneway_ns || !oneway_cycles) return CHARMING_ERR_CONFIG;
  const int n_sms = charm_host::info().n_sms;
  const size_t flag_bytes = 2 * sizeof(bl_line);
  const size_t slot_bytes = 2 * (size_t)BL_LOCAL_MAX * n_sms * sizeof(unsigned long long);
  char* d = nullptr;
  cudaError_t e = cudaMalloc(&d, flag_bytes + slot_bytes + 64);
  if (e != cudaSuccess) return charm_host::cuda_fail(e, "sm pingpong buffers");
  cudaMemset(d, 0, flag_bytes + slot_bytes + 64);
  bl_line* flags = reinterpret_cast<bl_line*>(d);
  unsigned long long* slots = reinterpret_cast<unsigned long long*>(d + flag_bytes);
  unsigned long long* out = reinterpret_cast<unsigned long long*>(d + flag_bytes + slot_bytes);
  int* err = reinterpret_cast<int*>(out + 4);
  // more than half of an SM's shared memory per block: the two blocks sit
  // on different SMs
  cudaDeviceProp prop;
  e = cudaGetDeviceProperties(&prop, 0);
  int smem = (int)(prop.sharedMemPerMultiprocessor / 2 + 1024);
  if (smem > (int)prop.sharedMemPerBlockOptin) smem = (int)prop.sharedMemPerBlockOptin;
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute((const void*)sm_pingpong_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  int warmup = round_trips / 10 + 10;
  int n_slot_sms = n_sms;
  void* args[] = {&mode, &round_trips, &warmup, &flags, &slots, &n_slot_sms, &out, &err};
  if (e == cudaSuccess)
    e = cudaLaunchCooperativeKernel((const void*)sm_pingpong_kernel, dim3(2), dim3(512), args, (size_t)smem, 0);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  unsigned long long h[4] = {0, 0, 0, 0};
  int herr = 0;
  if (e == cudaSuccess) e = cudaMemcpy(h, out, sizeof(h), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(&herr, err, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return charm_host::cuda_fail(e, "sm pingpong");
  if (herr) {
    charm_host::set_error_text("sm pingpong: a wait ran out");
    return CHARMING_ERR_DEADLINE;
  }
  *oneway_ns = (double)h[0] / (2.0 * round_trips);
  *oneway_cycles = (double)h[1] / (2.0 * round_trips);
  if (sm_pair) {
    const unsigned int* sm = reinterpret_cast<const unsigned int*>(&h[2]);
    sm_pair[0] = (int)sm[0];
    sm_pair[1] = (int)sm[1];
  }
  return CHARMING_OK;
}
#endif
