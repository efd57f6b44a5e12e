#include "suite.cuh"
__device__ void suite::serve_main(int pe) { if (threadIdx.x == 0 && pe == 0) charm::end(); }
