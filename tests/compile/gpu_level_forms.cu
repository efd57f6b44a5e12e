// GPU-level program forms (compiled with -DCHARMING_GPU_LEVEL): the
// reference examples' #ifndef SM_LEVEL branch (GID over the grid,
// BARRIER_LOCAL = charm::barrier_local(), __device__ proxy and data
// pointers, `new` from GID 0) and the mode-independent pe_thread() /
// pe_threads() / pe_sync(). Two chares on the one PE pass a counter and a
// 1024-int array back and forth; every entry method adds 1 to each array
// element with all threads of the grid, and GID 0 checks the sums.
#include <charming.h>

#ifdef SM_LEVEL
#error "a GPU-level program must not see SM_LEVEL"
#endif
#define GID (blockDim.x * blockIdx.x + threadIdx.x)
#define BARRIER_LOCAL charm::barrier_local()

constexpr int N = 1024, ROUNDS = 6;

struct Cell : charm::chare {
  int hits;
  __device__ Cell() : hits(0) {}
};
__device__ charm::chare_proxy<Cell>* cells;
__device__ int* data;
__device__ int* bad;

__device__ void on_msg(Cell& c, void* arg) {
  const int round = *static_cast<const int*>(arg);
  if (GID == 0) c.hits++;
  for (int i = charm::pe_thread(); i < N; i += charm::pe_threads()) {
    if (data[i] != round) atomicAdd(bad, 1);
    data[i] = round + 1;
  }
  charm::pe_sync();
  if (round + 1 < ROUNDS) {
    int next = round + 1;
    cells->invoke(1 - c.i, 0, &next, sizeof(int));
  } else if (GID == 0) {
    printf("gpu-level forms: pe %d of %d, rounds %d, hits %d, bad %d\n", charm::my_pe(), charm::n_pes(), round + 1,
           c.hits, *bad);
    charm::end();
  }
}

__device__ void charm::main(int argc, char** argv, size_t* argvs, int pe) {
  if (GID == 0) {
    cells = new charm::chare_proxy<Cell>();
    cells->add_entry_method<&on_msg>();
    cells->create(2);
    data = new int[N];
    bad = new int;
    *bad = 0;
  }
  BARRIER_LOCAL;
  for (int i = charm::pe_thread(); i < N; i += charm::pe_threads()) data[i] = 0;
  charm::barrier();
  if (pe == 0 && charm::is_gpu_level()) {
    int first = 0;
    cells->invoke(0, 0, &first, sizeof(int));
  }
}
