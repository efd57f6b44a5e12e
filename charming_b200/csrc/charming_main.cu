// Process main() of libcharming.a: programs that define charm::main (and
// optionally charm::main_host) link against the library and get this entry
// point, as with the reference (src/charming.cu:50-263).
//
// Environment overrides: CHARMING_GPU_LEVEL (1: GPU-level mode), CHARMING_PES_PER_SM, CHARMING_RING_BYTES,
// CHARMING_DEADLINE_S, CHARMING_IDLE_TIMEOUT_S, CHARMING_HEAP_BYTES,
// CHARMING_QUIET (suppress the [INFO] lines).
// Several GPUs, one process each (the reference's multi-GPU launch through
// MPI or NVSHMEM's launcher): WORLD_SIZE > 1, RANK, LOCAL_RANK (the GPU;
// default RANK), as torchrun sets them, and CHARMING_RDV_DIR, an empty
// directory all ranks see, for the bootstrap. CHARMING_VIRTUAL_DEVS=n (one
// process): this GPU's PEs form n GPUs in one launch.
#include <cstdio>
#include <cstdlib>
#include <memory>
#include "../../include/charming_c.h"
#include "rendezvous.h"

namespace charm {
// Weak: programs without a host main still link (the reference requires one).
__attribute__((weak)) void main_host(int argc, char** argv);
}

// Defined (weak) by programs compiled with -DCHARMING_GPU_LEVEL (common.h).
extern "C" {
extern const int charming_program_gpu_level __attribute__((weak));
}

static unsigned long long env_u64(const char* name, unsigned long long dflt) {
  const char* s = getenv(name);
  return s ? strtoull(s, nullptr, 0) : dflt;
}

int main(int argc, char** argv) {
  if (charm::main_host) charm::main_host(argc, argv);

  charming_config cfg;
  charming_default_config(&cfg);
  cfg.pes_per_sm = (int)env_u64("CHARMING_PES_PER_SM", (unsigned long long)cfg.pes_per_sm);
  cfg.ring_bytes = env_u64("CHARMING_RING_BYTES", cfg.ring_bytes);
  cfg.heap_bytes = env_u64("CHARMING_HEAP_BYTES", cfg.heap_bytes);
  cfg.gpu_level = &charming_program_gpu_level != nullptr ? charming_program_gpu_level : 0;
  cfg.gpu_level = (int)env_u64("CHARMING_GPU_LEVEL", (unsigned long long)cfg.gpu_level);
  bool quiet = getenv("CHARMING_QUIET") != nullptr;

  charming_devices devs{};
  devs.world = (int)env_u64("WORLD_SIZE", 1);
  devs.rank = (int)env_u64("RANK", 0);
  devs.virtual_devs = (int)env_u64("CHARMING_VIRTUAL_DEVS", 1);
  std::unique_ptr<charm_host::file_rendezvous> rdv;
  if (devs.world > 1) {
    const char* dir = getenv("CHARMING_RDV_DIR");
    if (!dir) {
      fprintf(stderr, "[ERROR] WORLD_SIZE > 1 needs CHARMING_RDV_DIR (an empty directory all ranks see)\n");
      return CHARMING_ERR_CONFIG;
    }
    rdv.reset(new charm_host::file_rendezvous(dir, devs.rank, devs.world));
    devs.allgather = &charm_host::file_rendezvous::allgather_cb;
    devs.barrier = &charm_host::file_rendezvous::barrier_cb;
    devs.ctx = rdv.get();
    cfg.device = (int)env_u64("LOCAL_RANK", (unsigned long long)devs.rank);
  }
  cfg.verbose = (quiet || devs.rank != 0) ? 0 : 1;

  int rc = charming_init_devices(&cfg, &devs);
  if (rc != CHARMING_OK) {
    fprintf(stderr, "[ERROR] charming_init: %s (%s)\n", charming_status_string(rc),
        charming_last_error());
    return rc;
  }
  rc = charming_run(argc, argv);
  charming_stats st;
  charming_last_stats(&st);
  if (rc != CHARMING_OK) {
    fprintf(stderr, "[ERROR] run ended with status %d: %s (pe %d, info %d %d) %s\n", rc,
        charming_status_string(rc), st.err_pe, st.err_info0, st.err_info1, charming_last_error());
  }
  if (!quiet && devs.rank == 0) {
    printf("[INFO] Exiting CharminG: %llu messages delivered, %.3f ms\n",
        (unsigned long long)st.delivered, st.kernel_ms);
  }
  fflush(stdout);
  charming_fini();
  return rc;
}
