// GPU-level program forms (compiled with -DCHARMING_GPU_LEVEL): the
// reference examples' #ifndef SM_LEVEL branch (GID over the grid,
// BARRIER_LOCAL = charm::barrier_local(), a __device__ proxy pointer) and
// the mode-independent pe_thread() / pe_threads() / pe_sync().
#include <charming.h>

#ifdef SM_LEVEL
#error "a GPU-level program must not see SM_LEVEL"
#endif
#define GID (blockDim.x * blockIdx.x + threadIdx.x)
#define BARRIER_LOCAL charm::barrier_local()

struct Cell : charm::chare {
  int hits;
  __device__ Cell() : hits(0) {}
};
__device__ charm::chare_proxy<Cell>* cells;
__device__ int* data;

__device__ void on_msg(Cell& c, void* arg) {
  if (GID == 0) c.hits++;
  BARRIER_LOCAL;
  for (int i = charm::pe_thread(); i < 1024; i += charm::pe_threads()) data[i] += 1;
  charm::pe_sync();
  if (c.hits < 3) cells->invoke(c.i, 0, data, 64);
  else if (charm::pe_thread() == 0) charm::end();
}

__device__ void charm::main(int argc, char** argv, size_t* argvs, int pe) {
  if (GID == 0) {
    cells = new charm::chare_proxy<Cell>();
    cells->add_entry_method<&on_msg>();
    cells->create(2);
    data = new int[1024];
  }
  BARRIER_LOCAL;
  charm::barrier();
  if (pe == 0 && charm::is_gpu_level()) cells->invoke(0, 0);
}
