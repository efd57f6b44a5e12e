#include "suite.cuh"
#include "../host.cuh"
__device__ void suite::serve_main(int pe) { if (threadIdx.x == 0 && pe == 0) charm::end(); }
extern "C" {
int charming_serve_start(const charming_serve_config*, void**) { return CHARMING_ERR_CONFIG; }
int charming_serve_submit(void*, const charming_jacobi_problem*, uint64_t) { return CHARMING_ERR_CONFIG; }
int charming_serve_poll(void*, charming_serve_completion*, int, int*) { return CHARMING_ERR_CONFIG; }
int charming_serve_fetch(void*, uint64_t, void*) { return CHARMING_ERR_CONFIG; }
int charming_serve_release(void*, uint64_t) { return CHARMING_ERR_CONFIG; }
int charming_serve_stop(void*, charming_serve_stats*) { return CHARMING_ERR_CONFIG; }
}
