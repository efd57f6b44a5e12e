// Compile-and-link check of the device API forms of the reference's headers
// that the built-in programs do not use (TEST INFRASTRUCTURE): the const
// message invoke overloads (reference include/chare.h:257-262), malloc_user
// / free_user (include/charming.h:33-34) and async_wait
// (include/chare.h:214-239). Built against include/ and linked with
// libcharming.a by tests/test_boundary_cpu.py; never run.
#include <charming.h>

struct Block : charm::chare {
  int x;
  __device__ Block() : x(0) {}
};

__shared__ charm::chare_proxy<Block>* proxy;
__device__ uint64_t signals[2];

__device__ void on_msg(Block& b, void* arg) {
  charm::message msg;
  if (proxy->alloc_msg(msg, (b.i + 1) % b.n, 64)) {
    const charm::message& cm = msg;
    proxy->invoke((b.i + 1) % b.n, 0, cm);  // const message&
  }
  charm::message msg2;
  if (proxy->alloc_msg(msg2, (b.i + 1) % b.n, 64)) {
    proxy->invoke((b.i + 1) % b.n, 0, static_cast<const charm::message&>(msg2), (size_t)32);
  }
  if (threadIdx.x == 0) {
    size_t off = 0;
    void* p = charm::malloc_user(256, off);
    if (p) charm::free_user(256, off);
    proxy->async_wait(signals, 2, charm::CMP_GE, 1, b.i, 1);
  }
  __syncthreads();
}

__device__ void on_signal(Block& b, void* arg) { charm::end(); }

__device__ void charm::main(int argc, char** argv, size_t* argvs, int pe) {
  if (threadIdx.x == 0) {
    proxy = new charm::chare_proxy<Block>();
    proxy->add_entry_method<&on_msg>();
    proxy->add_entry_method<&on_signal>();
    proxy->create(charm::n_pes());
  }
  __syncthreads();
  if (pe == 0) proxy->invoke(0, 0);
}
