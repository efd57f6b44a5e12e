// Hello chain and refnum scenario as built-in programs with result logs.
//
// Hello: the scenario of examples/hello/hello.cu:6-52 (2 * n_pes chares,
// chare 0 receives 0, each chare forwards value + 1 to the next, the last
// calls end()); out[i] records what chare i received.
// Refnum: the scenario of examples/refnum/refnum.cu:6-53 (chare 1 starts at
// refnum 1, chare 0 sends refnum 1 then refnum 0, chare 1 sets its refnum to
// 0 on delivery). The reference never terminates; here chare 1 calls end()
// after its second delivery. out records the delivered refnums in order.
#include "suite.cuh"
#ifndef CHARMING_HOST_EMULATION  // the CPU check of the runtime has no CUDA API
#include "../host.cuh"
#endif

namespace {

struct HelloChare : charm::chare {
  __device__ HelloChare() {}
};
struct RefChare : charm::chare {
  int received;
  __device__ RefChare() : received(0) {}
};

__shared__ charm::chare_proxy<HelloChare>* hello_proxy;
__shared__ charm::chare_proxy<RefChare>* ref_proxy;

__device__ void hello_greet(HelloChare& c, void* arg) {
  __shared__ int value;
  if (threadIdx.x == 0) {
    value = *reinterpret_cast<int*>(arg);
    reinterpret_cast<int*>(g_app.p[0])[c.i] = value;
  }
  __syncthreads();
  if (c.i == c.n - 1) {
    charm::end();
  } else {
    int next = value + 1;
    hello_proxy->invoke(c.i + 1, 0, &next, sizeof(int));
  }
}

// g_app.a[0] == 0: refnum 1 then refnum 0 (the reference's order);
// g_app.a[0] == 1: refnum 0 first, which chare 1 must stash until it has
// delivered refnum 1 and moved its own refnum to 0.
__device__ void ref_send(RefChare& c, void* arg) {
  int first = g_app.a[0] ? 0 : 1;
  int r = first;
  ref_proxy->invoke(1, 1, &r, sizeof(int), first);
  r = 1 - first;
  ref_proxy->invoke(1, 1, &r, sizeof(int), 1 - first);
}

__device__ void ref_recv(RefChare& c, void* arg) {
  if (threadIdx.x == 0) {
    int* out = reinterpret_cast<int*>(g_app.p[0]);
    out[c.received] = *reinterpret_cast<int*>(arg);
    c.received++;
    ref_proxy->set_refnum(1, 0);
  }
  __syncthreads();
  if (c.received == 2) charm::end();
}

}  // namespace

__device__ void suite::hello_main(int pe) {
  if (threadIdx.x == 0) {
    hello_proxy = new charm::chare_proxy<HelloChare>();
    hello_proxy->add_entry_method<&hello_greet>();
    hello_proxy->create(charm::n_pes() * 2);
  }
  __syncthreads();
  charm::barrier();
  if (pe == 0) {
    int zero = 0;
    hello_proxy->invoke(0, 0, &zero, sizeof(int));
  }
}

__device__ void suite::refnum_main(int pe) {
  if (threadIdx.x == 0) {
    ref_proxy = new charm::chare_proxy<RefChare>();
    ref_proxy->add_entry_method<&ref_send>();
    ref_proxy->add_entry_method<&ref_recv>();
    int n = charm::n_pes();
    int* block_map = new int[n];
    for (int i = 0; i < n; i++) block_map[i] = 0;
    block_map[0] += 1;
    block_map[n / 2] += 1;
    ref_proxy->create(2, block_map);
    delete[] block_map;
    if (pe == 0) ref_proxy->set_refnum(0, 0);
    if (pe == n / 2) ref_proxy->set_refnum(1, 1);
  }
  __syncthreads();
  charm::barrier();
  if (pe == 0) ref_proxy->invoke(0, 0, nullptr, 0, 0);
}

#ifndef CHARMING_HOST_EMULATION
extern "C" int charming_hello(int* out, int n_out, int* n_chares) {
  int rc = charm_host::ensure_init();
  if (rc) return rc;
  int n = 2 * charm_host::info().n_pes;
  if (n_chares) *n_chares = n;
  if (out == nullptr || n_out < n) return CHARMING_ERR_CONFIG;
  int* d = nullptr;
  cudaError_t e = cudaMalloc(&d, sizeof(int) * n);
  if (e != cudaSuccess) return charm_host::cuda_fail(e, "hello log");
  cudaMemset(d, 0xff, sizeof(int) * n);
  suite::app_params p{};
  p.id = suite::APP_HELLO;
  p.p[0] = d;
  rc = suite_run(p);
  cudaMemcpy(out, d, sizeof(int) * n, cudaMemcpyDeviceToHost);
  cudaFree(d);
  return rc;
}

static int refnum_run(int* out, int n_out, int* n_delivered, int reversed) {
  int rc = charm_host::ensure_init();
  if (rc) return rc;
  if (out == nullptr || n_out < 2) return CHARMING_ERR_CONFIG;
  int* d = nullptr;
  cudaError_t e = cudaMalloc(&d, sizeof(int) * 4);
  if (e != cudaSuccess) return charm_host::cuda_fail(e, "refnum log");
  cudaMemset(d, 0xff, sizeof(int) * 4);
  suite::app_params p{};
  p.id = suite::APP_REFNUM;
  p.a[0] = reversed;
  p.p[0] = d;
  rc = suite_run(p);
  int h[4];
  cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
  cudaFree(d);
  int cnt = 0;
  for (int i = 0; i < 2; i++) {
    out[i] = h[i];
    if (h[i] != -1) cnt++;
  }
  if (n_delivered) *n_delivered = cnt;
  return rc;
}

extern "C" int charming_refnum(int* out, int n_out, int* n_delivered) {
  return refnum_run(out, n_out, n_delivered, 0);
}

// Same scenario with the two sends swapped, so that the refnum-0 message
// reaches chare 1 first and goes through the stash.
extern "C" int charming_refnum_reversed(int* out, int n_out, int* n_delivered) {
  return refnum_run(out, n_out, n_delivered, 1);
}
#endif
