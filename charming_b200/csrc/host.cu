// Host runtime: device setup, buffer allocation, the scheduler launch and the
// core C ABI (charming_init / run / fini / stats).
//
// Replaces the reference's process main (src/charming.cu:50-263) and
// comm_init_host / comm_fini_host (src/comm/get/get.cu:69-169): no NVSHMEM or
// MPI bootstrap, plain cudaMalloc'd HBM for the inbox rings, and a
// cooperative launch so that every PE block is resident. Over several GPUs
// (one process each), every GPU's inbox side is one allocation exported with
// CUDA IPC and mapped by the others; the host's allgather and barrier
// (charming_devices) exchange the handles and order the runs.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <string>
#include "host.cuh"

__global__ void charming_scheduler_kernel(int argc, char** argv, size_t* argvs);
__global__ void charming_reset_kernel();

using namespace charm::rt;

namespace {

struct HostRuntime {
  bool inited = false;
  charming_config cfg{};
  charming_info inf{};
  cudaDeviceProp prop{};
  device_state ds{};
  std::vector<void*> dev_allocs;
  int* h_stop = nullptr;
  int* d_stop = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  charming_stats last{};
  char* d_args = nullptr;
  size_t d_args_cap = 0;
  int n_local = 0;                  // PE slots of this launch (1 in GPU-level mode)
  int rank = 0, world = 1, vdevs = 1;
  charming_devices devs{};          // the host collectives (world > 1)
  std::vector<void*> ipc_opened;    // peers' inbox regions mapped here
  std::vector<int*> launch_ctrl;    // control words of this launch's GPUs
};

HostRuntime g;
std::string g_err;

template <typename T>
int dev_alloc(T** p, size_t bytes, const char* what) {
  void* q = nullptr;
  cudaError_t e = cudaMalloc(&q, bytes);
  if (e != cudaSuccess) return charm_host::cuda_fail(e, what);
  e = cudaMemset(q, 0, bytes);
  if (e != cudaSuccess) {
    cudaFree(q);
    return charm_host::cuda_fail(e, what);
  }
  g.dev_allocs.push_back(q);
  g.inf.device_bytes += bytes;
  *p = reinterpret_cast<T*>(q);
  return CHARMING_OK;
}

bool is_pow2(uint64_t v) { return v && !(v & (v - 1)); }

// One GPU's inbox side in one allocation (what another GPU maps): tails,
// heads, control words, progress stamps, then flags and rings on 2 MiB
// boundaries.
struct inbox_layout {
  size_t tail, head, ctrl, progress, flags, ring, bytes;
};
inbox_layout inbox_layout_for(int pes, const device_state& ds) {
  auto up = [](size_t v, size_t a) { return (v + a - 1) / a * a; };
  inbox_layout L{};
  size_t o = 0;
  L.tail = o;
  o = up(o + sizeof(line_u64) * (size_t)pes, 4096);
  L.head = o;
  o = up(o + sizeof(line_u64) * (size_t)pes, 4096);
  L.ctrl = o;
  o = up(o + sizeof(int) * CTRL_WORDS, 4096);
  L.progress = o;
  o = up(o + 8ull * (size_t)pes, 2u << 20);
  L.flags = o;
  o = up(o + 8ull * ds.ring_cells * (size_t)pes, 2u << 20);
  L.ring = o;
  o = up(o + ds.ring_stride * (size_t)pes, 2u << 20);
  L.bytes = o;
  return L;
}
dev_inbox carve_inbox(unsigned char* base, const inbox_layout& L) {
  dev_inbox d{};
  d.tail = reinterpret_cast<line_u64*>(base + L.tail);
  d.head = reinterpret_cast<line_u64*>(base + L.head);
  d.ctrl = reinterpret_cast<int*>(base + L.ctrl);
  d.progress = reinterpret_cast<unsigned long long*>(base + L.progress);
  d.flags = reinterpret_cast<unsigned long long*>(base + L.flags);
  d.ring = base + L.ring;
  return d;
}

// What each rank tells the others at init.
struct peer_record {
  cudaIpcMemHandle_t handle;
  uint64_t region_bytes, ring_bytes, max_msg;
  int32_t pes, rank;
};

int host_barrier() {
  if (g.world <= 1) return CHARMING_OK;
  if (g.devs.barrier(g.devs.ctx) != 0) {
    g_err = "host barrier failed";
    return CHARMING_ERR_CONFIG;
  }
  return CHARMING_OK;
}

double env_double(const char* name, double dflt) {
  const char* s = getenv(name);
  return s ? atof(s) : dflt;
}

}  // namespace

namespace charm_host {

int cuda_fail(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return CHARMING_OK;
  g_err = std::string(what) + ": " + cudaGetErrorString(e);
  return CHARMING_ERR_CUDA;
}
void set_error_text(const std::string& s) { g_err = s; }
bool initialised() { return g.inited; }
cudaStream_t stream() { return g.stream; }
const charming_info& info() { return g.inf; }
int n_procs() { return g.world; }

int ensure_init() {
  if (g.inited) return CHARMING_OK;
  charming_config cfg;
  charming_default_config(&cfg);
  return charming_init(&cfg);
}

int set_deadline(double seconds) {
  if (!g.inited) return CHARMING_ERR_NOT_INIT;
  g.ds.deadline_ns = (unsigned long long)((seconds > 0 ? seconds : g.cfg.deadline_s) * 1e9);
  return cuda_fail(cudaMemcpyToSymbol(c_rt, &g.ds, sizeof(g.ds)), "run deadline");
}

void request_stop(int value) {
  if (g.h_stop) {
    *reinterpret_cast<volatile int*>(g.h_stop) = value;
  }
}

int enqueue_scheduler(cudaStream_t s) {
  if (!g.inited) return CHARMING_ERR_NOT_INIT;
  if (g.world > 1) {  // runs over several processes need the host barriers of run_scheduler
    g_err = "stream-ordered runs are single-process";
    return CHARMING_ERR_CONFIG;
  }
  int nb = (g.n_local + 255) / 256;
  charming_reset_kernel<<<nb, 256, 0, s>>>();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "reset kernel launch");
  int argc = 0;
  char** argv = nullptr;
  size_t* argvs = nullptr;
  void* args[] = {&argc, &argv, &argvs};
  cudaLaunchConfig_t lc{};
  lc.gridDim = dim3(g.inf.n_blocks);
  lc.blockDim = dim3(g.inf.threads_per_pe);
  lc.dynamicSmemBytes = g.inf.smem_bytes_per_pe;
  lc.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  lc.attrs = attr;
  lc.numAttrs = 1;
  e = cudaLaunchKernelExC(&lc, (const void*)charming_scheduler_kernel, args);
  if (e != cudaSuccess) return cuda_fail(e, "scheduler launch");
  return CHARMING_OK;
}

__global__ void charming_status_latch_kernel(const int* ctrl, int* latch) {
  if (latch[0] == 0 && ctrl[CTRL_STATUS] != 0) {
    latch[0] = ctrl[CTRL_STATUS];
    latch[1] = ctrl[CTRL_ERR_PE];
    latch[2] = ctrl[CTRL_ERR_I0];
    latch[3] = ctrl[CTRL_ERR_I1];
  }
}

int enqueue_status_latch(int* latch, cudaStream_t s) {
  if (!g.inited) return CHARMING_ERR_NOT_INIT;
  charming_status_latch_kernel<<<1, 1, 0, s>>>(g.ds.ctrl, latch);
  return cuda_fail(cudaGetLastError(), "status latch");
}

int collect_run(double kernel_ms) {
  // the first error any of this launch's GPUs recorded
  int ctrl_h[CTRL_WORDS];
  cudaError_t e = cudaSuccess;
  for (size_t d = 0; d < g.launch_ctrl.size(); d++) {
    e = cudaMemcpy(ctrl_h, g.launch_ctrl[d], sizeof(ctrl_h), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "read status");
    if (ctrl_h[CTRL_STATUS] != 0) break;
  }
  const int n_local = g.n_local;
  std::vector<unsigned long long> st((size_t)n_local * N_STATS), tm((size_t)n_local * 3);
  e = cudaMemcpy(st.data(), g.ds.pe_stats, st.size() * 8, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(tm.data(), g.ds.pe_times, tm.size() * 8, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "read stats");
  charming_stats s{};
  unsigned long long tmin = ~0ULL, tmax = 0, main_max = 0;
  for (int p = 0; p < n_local; p++) {
    const unsigned long long* t = &tm[3 * (size_t)p];
    if (t[1] > t[0] && t[1] - t[0] > main_max) main_max = t[1] - t[0];
    const unsigned long long* q = &st[(size_t)p * N_STATS];
    s.delivered += q[ST_DELIVERED];
    s.sent += q[ST_SENT];
    s.stashed += q[ST_STASHED];
    s.revived += q[ST_REVIVED];
    s.bytes_sent += q[ST_BYTES_SENT];
    s.idle_polls += q[ST_IDLE_POLLS];
    s.space_waits += q[ST_SPACE_WAITS];
    s.deferred += q[ST_DEFERRED];
    s.batched += q[ST_BATCHED];
    if (t[1] && t[1] < tmin) tmin = t[1];
    if (t[2] > tmax) tmax = t[2];
  }
  s.loop_ms = (tmax > tmin && tmin != ~0ULL) ? (tmax - tmin) * 1e-6 : 0.0;
  double idle = 0;
  for (int p = 0; p < n_local; p++) idle += (double)st[(size_t)p * N_STATS + ST_IDLE_CYC];
  s.idle_ms = (n_local && g.prop.clockRate > 0) ? idle / n_local / (double)g.prop.clockRate : 0.0;
  double em = 0;
  for (int p = 0; p < n_local; p++) em += (double)st[(size_t)p * N_STATS + ST_EM_CYC];
  s.em_ms = (n_local && g.prop.clockRate > 0) ? em / n_local / (double)g.prop.clockRate : 0.0;
  double tk = 0, sp = 0;
  for (int p = 0; p < n_local; p++) {
    tk += (double)st[(size_t)p * N_STATS + ST_TICKET_NS];
    sp += (double)st[(size_t)p * N_STATS + ST_SPACE_NS];
  }
  s.ticket_ms = n_local ? tk / n_local * 1e-6 : 0.0;
  s.space_ms = n_local ? sp / n_local * 1e-6 : 0.0;
  s.main_ms = main_max * 1e-6;
  s.kernel_ms = kernel_ms;
  s.status = ctrl_h[CTRL_STATUS];
  s.err_pe = ctrl_h[CTRL_ERR_PE];
  s.err_info0 = ctrl_h[CTRL_ERR_I0];
  s.err_info1 = ctrl_h[CTRL_ERR_I1];
  g.last = s;
  return s.status;
}

int run_scheduler(int argc, char** argv) {
  if (!g.inited) return CHARMING_ERR_NOT_INIT;
  // Arguments into device memory (reference: managed memory,
  // src/charming.cu:146-169).
  size_t total = (size_t)argc * (sizeof(char*) + sizeof(size_t)) + 16;
  for (int i = 0; i < argc; i++) total += strlen(argv[i]) + 1;
  if (total > g.d_args_cap) {
    if (g.d_args) cudaFree(g.d_args);
    g.d_args = nullptr;
    size_t cap = total < 4096 ? 4096 : total * 2;
    cudaError_t e = cudaMalloc(&g.d_args, cap);
    if (e != cudaSuccess) return cuda_fail(e, "argv buffer");
    g.d_args_cap = cap;
  }
  std::vector<char> blob(total, 0);
  char** h_argv = reinterpret_cast<char**>(blob.data());
  size_t* h_argvs = reinterpret_cast<size_t*>(blob.data() + (size_t)argc * sizeof(char*));
  size_t off = (size_t)argc * (sizeof(char*) + sizeof(size_t));
  for (int i = 0; i < argc; i++) {
    size_t n = strlen(argv[i]);
    memcpy(blob.data() + off, argv[i], n + 1);
    h_argv[i] = g.d_args + off;
    h_argvs[i] = n;
    off += n + 1;
  }
  cudaError_t e = cudaMemcpyAsync(g.d_args, blob.data(), total, cudaMemcpyHostToDevice, g.stream);
  if (e != cudaSuccess) return cuda_fail(e, "argv copy");
  *reinterpret_cast<volatile int*>(g.h_stop) = 0;

  // Several processes: the previous run has ended on every GPU (the barrier
  // at the end of run_scheduler); every GPU resets before any launches.
  int nb = (g.n_local + 255) / 256;
  charming_reset_kernel<<<nb, 256, 0, g.stream>>>();
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "reset kernel launch");
  if (g.world > 1) {
    e = cudaStreamSynchronize(g.stream);
    if (e != cudaSuccess) return cuda_fail(e, "reset");
    if (int rc = host_barrier()) return rc;
  }

  char** d_argv = reinterpret_cast<char**>(g.d_args);
  size_t* d_argvs = reinterpret_cast<size_t*>(g.d_args + (size_t)argc * sizeof(char*));
  void* args[] = {&argc, &d_argv, &d_argvs};
  cudaEventRecord(g.ev0, g.stream);
  e = cudaLaunchCooperativeKernel((const void*)charming_scheduler_kernel, dim3(g.inf.n_blocks),
      dim3(g.inf.threads_per_pe), args, (size_t)g.inf.smem_bytes_per_pe, g.stream);
  if (e != cudaSuccess) return cuda_fail(e, "scheduler launch");
  cudaEventRecord(g.ev1, g.stream);
  e = cudaStreamSynchronize(g.stream);
  if (e != cudaSuccess) return cuda_fail(e, "scheduler run");
  // every launch has ended: nothing writes this GPU's control words any more
  if (int rc = host_barrier()) return rc;
  float ms = 0.f;
  cudaEventElapsedTime(&ms, g.ev0, g.ev1);
  return collect_run(ms);
}

}  // namespace charm_host

using namespace charm_host;

extern "C" {

void charming_default_config(charming_config* cfg) {
  memset(cfg, 0, sizeof(*cfg));
  cfg->device = 0;
  cfg->pes_per_sm = 1;
  cfg->threads_per_pe = 512;
  cfg->n_pes = 0;
  cfg->ring_bytes = 4ull << 20;
  cfg->max_msg_bytes = (1ull << 20) + 64;
  cfg->stash_bytes = 4ull << 20;
  cfg->stash_entries = 4096;
  cfg->heap_bytes = 1ull << 30;
  cfg->stack_bytes = 8192;
  cfg->deadline_s = env_double("CHARMING_DEADLINE_S", 120.0);
  cfg->idle_timeout_s = env_double("CHARMING_IDLE_TIMEOUT_S", 10.0);
  cfg->free_chares_at_exit = 1;
  cfg->verbose = 0;
}

int charming_init(const charming_config* cfg_in) { return charming_init_devices(cfg_in, nullptr); }

int charming_init_devices(const charming_config* cfg_in, const charming_devices* devs) {
  if (g.inited) return CHARMING_OK;
  charming_config cfg = *cfg_in;
  charming_devices dv{};
  dv.world = 1;
  dv.virtual_devs = 1;
  if (devs) dv = *devs;
  if (dv.world < 1) dv.world = 1;
  if (dv.virtual_devs < 1) dv.virtual_devs = 1;
  const int n_devs = dv.world > 1 ? dv.world : dv.virtual_devs;
#ifndef CHARMING_MULTI_GPU
  if (n_devs > 1) {
    set_error_text("this build is single-GPU: several GPUs need the multi-GPU build "
                   "(libcharming_b200_multi.so, libcharming_multi.a)");
    return CHARMING_ERR_CONFIG;
  }
#endif
  if (n_devs > MAX_DEVS || dv.rank < 0 || dv.rank >= dv.world || (dv.world > 1 && dv.virtual_devs > 1) ||
      (dv.world > 1 && (!dv.allgather || !dv.barrier)) || (n_devs > 1 && cfg.gpu_level)) {
    set_error_text("invalid charming_devices (at most 8 GPUs, SM-level mode, collectives for world > 1)");
    return CHARMING_ERR_CONFIG;
  }
  g.inf = charming_info{};
  cudaError_t e = cudaSetDevice(cfg.device);
  if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
  e = cudaGetDeviceProperties(&g.prop, cfg.device);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDeviceProperties");
  if (!g.prop.cooperativeLaunch) {
    set_error_text("device does not support cooperative launch");
    return CHARMING_ERR_CONFIG;
  }
  if (cfg.pes_per_sm < 1 || cfg.pes_per_sm > 4 || cfg.threads_per_pe < 32 ||
      cfg.threads_per_pe > MAX_THREADS || (cfg.threads_per_pe % 32) ||
      !is_pow2(cfg.ring_bytes) || cfg.ring_bytes < 4096 ||
      cfg.max_msg_bytes < 64 || cfg.max_msg_bytes > cfg.ring_bytes / 2 ||
      cfg.stash_entries < 16 || cfg.stash_bytes < cfg.max_msg_bytes ||
      cfg.deadline_s <= 0) {
    set_error_text("invalid charming_config");
    return CHARMING_ERR_CONFIG;
  }
  int n_sms = g.prop.multiProcessorCount;
  // GPU-level mode: the blocks (n_pes of them, by default one per SM slot)
  // form one PE
  const int n_blocks = cfg.n_pes > 0 ? cfg.n_pes : n_sms * cfg.pes_per_sm;
  if (n_blocks % dv.virtual_devs) {
    set_error_text("PE blocks must split evenly into the virtual GPUs");
    return CHARMING_ERR_CONFIG;
  }
  // Several GPUs: P PEs per GPU (all of this launch's blocks per process, or
  // an equal share of them per virtual GPU), numbered globally.
  const int pes_per_dev = dv.world > 1 ? n_blocks : n_blocks / dv.virtual_devs;
  const int n_pes = cfg.gpu_level ? 1 : pes_per_dev * n_devs;
  const int n_local = cfg.gpu_level ? 1 : n_blocks;  // this launch's PE slots
  const int dev0 = dv.world > 1 ? dv.rank : 0;        // its first GPU

  // Device limits (reference: src/charming.cu:197-203).
  // The heap size is fixed once a kernel of the context has run (a second
  // charming_init in the same process): keep it when it is large enough.
  size_t heap_now = 0;
  e = cudaDeviceGetLimit(&heap_now, cudaLimitMallocHeapSize);
  if (e != cudaSuccess) return cuda_fail(e, "heap limit query");
  if (heap_now != cfg.heap_bytes) {
    e = cudaDeviceSetLimit(cudaLimitMallocHeapSize, cfg.heap_bytes);
    if (e != cudaSuccess && heap_now >= cfg.heap_bytes) {
      (void)cudaGetLastError();
      e = cudaSuccess;
    }
    if (e != cudaSuccess) return cuda_fail(e, "heap limit");
  }
  size_t stack_now = 0;
  e = cudaDeviceGetLimit(&stack_now, cudaLimitStackSize);
  if (e != cudaSuccess) return cuda_fail(e, "stack limit query");
  if (stack_now != cfg.stack_bytes) {
    e = cudaDeviceSetLimit(cudaLimitStackSize, cfg.stack_bytes);
    if (e != cudaSuccess && stack_now >= cfg.stack_bytes) {
      (void)cudaGetLastError();
      e = cudaSuccess;
    }
    if (e != cudaSuccess) return cuda_fail(e, "stack limit");
  }
  size_t stack_eff = 0;
  e = cudaDeviceGetLimit(&stack_eff, cudaLimitStackSize);
  if (e != cudaSuccess) return cuda_fail(e, "stack limit query");

  cudaFuncAttributes fa;
  e = cudaFuncGetAttributes(&fa, (const void*)charming_scheduler_kernel);
  if (e != cudaSuccess) return cuda_fail(e, "scheduler attributes");
  int smem_state = (int)((sizeof(pe_state) + 8ull * n_pes + 127) / 128 * 128);
  // on-chip object arena (chare objects, proxies, their tables); the device
  // arena and heap take what does not fit
  int smem_arena = cfg.pes_per_sm > 1 ? (16 << 10) : (32 << 10);
  if (const char* ev = getenv("CHARMING_SMEM_ARENA_BYTES")) smem_arena = (int)strtol(ev, nullptr, 10) / 128 * 128;
  long per_block = (long)g.prop.sharedMemPerBlockOptin - (long)fa.sharedSizeBytes;
  long per_sm = (long)g.prop.sharedMemPerMultiprocessor / cfg.pes_per_sm -
                (long)fa.sharedSizeBytes - (long)g.prop.reservedSharedMemPerBlock;
  long smem_total = per_block < per_sm ? per_block : per_sm;
  // A cap leaves the rest of the SM's 256 KB of L1/shared storage to the L1
  // cache (local memory and global loads). 96 KiB holds the runtime state,
  // the object arena and the deep pass's cp.async rings of 16 warps (64 KiB),
  // and the L1 it frees made the headline launch 4 % faster (the halo copies
  // and the spills hit it). CHARMING_SMEM_PER_PE sets another cap (0: none).
  long cap = 96 << 10;
  if (const char* ev = getenv("CHARMING_SMEM_PER_PE")) cap = strtol(ev, nullptr, 10);
  if (cap > 0 && cap < smem_total) smem_total = cap;
  smem_total = smem_total / 128 * 128;
  if (smem_arena > smem_total / 4) smem_arena = (int)(smem_total / 4) / 128 * 128;
  if (smem_total < smem_state + smem_arena + 1024) {
    set_error_text("not enough shared memory per PE");
    return CHARMING_ERR_CONFIG;
  }
  e = cudaFuncSetAttribute((const void*)charming_scheduler_kernel,
      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_total);
  if (e != cudaSuccess) return cuda_fail(e, "smem attribute");
  int per_sm_blocks = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_blocks,
      (const void*)charming_scheduler_kernel, cfg.threads_per_pe, (size_t)smem_total);
  if (e != cudaSuccess) return cuda_fail(e, "occupancy");
  if ((long)per_sm_blocks * n_sms < n_blocks) {
    char buf[256];
    snprintf(buf, sizeof(buf), "%d PE blocks cannot be co-resident (%d blocks/SM x %d SMs)",
        n_blocks, per_sm_blocks, n_sms);
    set_error_text(buf);
    return CHARMING_ERR_CONFIG;
  }

  g.cfg = cfg;
  g.n_local = n_local;
  g.rank = dv.rank;
  g.world = dv.world;
  g.vdevs = dv.virtual_devs;
  g.devs = dv;
  g.launch_ctrl.clear();
  g.ipc_opened.clear();
  g.inf.n_pes = n_pes;
  g.inf.n_devs = n_devs;
  g.inf.my_dev = dev0;
  g.inf.n_blocks = n_blocks;
  g.inf.gpu_level = cfg.gpu_level ? 1 : 0;
  g.inf.n_sms = n_sms;
  g.inf.threads_per_pe = cfg.threads_per_pe;
  g.inf.smem_bytes_per_pe = (int)smem_total;
  g.inf.smem_scratch_bytes = (int)smem_total - smem_state - smem_arena;
  g.inf.regs_per_thread = fa.numRegs;
  g.inf.stack_bytes = (uint64_t)stack_eff;
  g.inf.local_bytes = (uint64_t)fa.localSizeBytes;
  g.inf.ring_bytes = cfg.ring_bytes;
  g.inf.max_msg_bytes = (cfg.max_msg_bytes + 15) / 16 * 16;

  device_state& ds = g.ds;
  ds = device_state{};
  ds.n_pes = n_pes;
  ds.threads = cfg.threads_per_pe;
  ds.ring_cells = cfg.ring_bytes / CELL;
  ds.max_msg = (cfg.max_msg_bytes + 15) / 16 * 16;
  ds.ring_stride = cfg.ring_bytes + (ds.max_msg + CELL - 1) / CELL * CELL + 128;
  ds.stash_bytes = (cfg.stash_bytes + 127) / 128 * 128;
  ds.stash_entries = cfg.stash_entries;
  ds.smem_state_bytes = smem_state;
  ds.smem_arena_bytes = smem_arena;
  ds.smem_total = (unsigned long long)smem_total;
  ds.deadline_ns = (unsigned long long)(cfg.deadline_s * 1e9);
  ds.idle_timeout_ns = (unsigned long long)(cfg.idle_timeout_s * 1e9);
  ds.free_chares_at_exit = cfg.free_chares_at_exit;
  ds.gpu_level = cfg.gpu_level ? 1 : 0;
  // pause between the inbox polls of a PE idle for 32 polls
  // (CHARMING_IDLE_SLEEP_NS; 0 polls without pausing)
  ds.idle_sleep_ns = 2000;
  if (const char* ev = getenv("CHARMING_IDLE_SLEEP_NS")) ds.idle_sleep_ns = (unsigned)strtoul(ev, nullptr, 10);
  ds.n_blocks = n_blocks;
  ds.n_devs = n_devs;
  ds.pes_per_dev = cfg.gpu_level ? 1 : pes_per_dev;
  ds.pe0 = dev0 * ds.pes_per_dev;
  ds.n_procs = dv.world;

  int rc;
  // The inbox side: one region per GPU of this launch (one, or one per
  // virtual GPU); with several processes, the others' regions mapped here.
  const inbox_layout L = inbox_layout_for(cfg.gpu_level ? 1 : pes_per_dev, ds);
  const int launch_devs = dv.world > 1 ? 1 : dv.virtual_devs;
  unsigned char* own_region = nullptr;
  for (int k = 0; k < launch_devs; k++) {
    unsigned char* base = nullptr;
    if ((rc = dev_alloc(&base, L.bytes, "inbox region"))) return rc;
    if (k == 0) own_region = base;
    ds.dev[dev0 + k] = carve_inbox(base, L);
    g.launch_ctrl.push_back(ds.dev[dev0 + k].ctrl);
  }
  ds.tail = ds.dev[dev0].tail;
  ds.head = ds.dev[dev0].head;
  ds.flags = ds.dev[dev0].flags;
  ds.ring = ds.dev[dev0].ring;
  ds.ctrl = ds.dev[dev0].ctrl;
  ds.progress = ds.dev[dev0].progress;
  if (dv.world > 1) {
    peer_record mine{};
    e = cudaIpcGetMemHandle(&mine.handle, own_region);
    if (e != cudaSuccess) return cuda_fail(e, "export the inbox region");
    mine.region_bytes = L.bytes;
    mine.ring_bytes = cfg.ring_bytes;
    mine.max_msg = ds.max_msg;
    mine.pes = pes_per_dev;
    mine.rank = dv.rank;
    std::vector<peer_record> all((size_t)dv.world);
    if (dv.allgather(dv.ctx, &mine, all.data(), sizeof(peer_record)) != 0) {
      set_error_text("host allgather failed");
      return CHARMING_ERR_CONFIG;
    }
    for (int r = 0; r < dv.world; r++) {
      const peer_record& q = all[(size_t)r];
      if (q.rank != r || q.pes != mine.pes || q.region_bytes != mine.region_bytes ||
          q.ring_bytes != mine.ring_bytes || q.max_msg != mine.max_msg) {
        set_error_text("ranks disagree on PEs per GPU, ring or message sizes");
        return CHARMING_ERR_CONFIG;
      }
      if (r == dv.rank) continue;
      void* peer = nullptr;
      e = cudaIpcOpenMemHandle(&peer, q.handle, cudaIpcMemLazyEnablePeerAccess);
      if (e != cudaSuccess) return cuda_fail(e, "map a peer GPU's inbox region");
      g.ipc_opened.push_back(peer);
      ds.dev[r] = carve_inbox(static_cast<unsigned char*>(peer), L);
    }
  }
  if ((rc = dev_alloc(&ds.stash_keys, sizeof(stash_key) * (size_t)ds.stash_entries * n_local, "stash keys"))) return rc;
  if ((rc = dev_alloc(&ds.stash_data, ds.stash_bytes * n_local, "stash arena"))) return rc;
  if ((rc = dev_alloc(&ds.proxy_tables, sizeof(charm::chare_proxy_table) * n_local, "proxy tables"))) return rc;
  if ((rc = dev_alloc(&ds.pe_stats, 8ull * N_STATS * n_local, "stats"))) return rc;
  if ((rc = dev_alloc(&ds.pe_times, 24ull * n_local, "times"))) return rc;
  if (ds.gpu_level && (rc = dev_alloc(&ds.gl, sizeof(group_state), "group state"))) return rc;
  // per-PE arena for proxy tables and chare objects (reset every run; the
  // device heap takes over when a PE needs more)
  ds.arena_bytes = 256ull << 10;
  if (const char* ev = getenv("CHARMING_ARENA_BYTES")) ds.arena_bytes = strtoull(ev, nullptr, 10);
  ds.arena = nullptr;
  if (ds.arena_bytes && (rc = dev_alloc(&ds.arena, ds.arena_bytes * n_local, "arena"))) return rc;
  // per-PE outbox for sends deferred while their destination ring is full:
  // room for a few of the largest messages
  ds.outbox_bytes = 2 * ds.max_msg + (1ull << 20);
  if (const char* ev = getenv("CHARMING_OUTBOX_BYTES")) ds.outbox_bytes = strtoull(ev, nullptr, 10);
  ds.outbox_bytes = (ds.outbox_bytes + 127) / 128 * 128;
  ds.outbox_stride = ds.outbox_bytes + (ds.max_msg + OB_HDR + 127) / 128 * 128;
  ds.outbox = nullptr;
  if (ds.outbox_bytes && (rc = dev_alloc(&ds.outbox, ds.outbox_stride * n_local, "outbox"))) return rc;
  // malloc_user heap per PE
  ds.user_heap_bytes = 1ull << 20;
  if (const char* ev = getenv("CHARMING_USER_HEAP_BYTES")) ds.user_heap_bytes = strtoull(ev, nullptr, 10);
  ds.user_heap_bytes = (ds.user_heap_bytes + 127) / 128 * 128;
  ds.user_blocks_max = 1024;
  ds.user_heap = nullptr;
  ds.user_blocks = nullptr;
  if (ds.user_heap_bytes) {
    if ((rc = dev_alloc(&ds.user_heap, ds.user_heap_bytes * n_local, "user heap"))) return rc;
    if ((rc = dev_alloc(&ds.user_blocks, sizeof(user_block) * (size_t)ds.user_blocks_max * n_local,
                        "user heap blocks")))
      return rc;
  }
  e = cudaHostAlloc(&g.h_stop, 64, cudaHostAllocMapped);
  if (e != cudaSuccess) return cuda_fail(e, "host stop word");
  *g.h_stop = 0;
  e = cudaHostGetDevicePointer(&g.d_stop, g.h_stop, 0);
  if (e != cudaSuccess) return cuda_fail(e, "host stop pointer");
  ds.host_stop = g.d_stop;

  // one NVSwitch domain: every GPU of the run is on this node
  int one = 1;
  e = cudaMemcpyToSymbol(c_n_sms, &n_sms, sizeof(int));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_my_dev, &dev0, sizeof(int));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_my_dev_node, &dev0, sizeof(int));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_n_devs, &n_devs, sizeof(int));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_n_devs_node, &n_devs, sizeof(int));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_n_nodes, &one, sizeof(int));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_n_pes, &n_pes, sizeof(int));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_n_pes_node, &n_pes, sizeof(int));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_rt, &ds, sizeof(ds));
  if (e != cudaSuccess) return cuda_fail(e, "constants");
  e = cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&g.ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&g.ev1);
  if (e != cudaSuccess) return cuda_fail(e, "stream/events");
  e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return cuda_fail(e, "init sync");
  g.inited = true;
  if (cfg.verbose) {
    PINFO("Initiating CharminG (B200 runtime)\n");
    if (ds.gpu_level)
      PINFO("GPU-level mode: 1 PE of %d blocks x %d threads, SMs: %d, regs/thread: %d\n", n_blocks,
          cfg.threads_per_pe, n_sms, fa.numRegs);
    else if (n_devs > 1)
      PINFO("PEs: %d on %d GPUs (%d per GPU, %s; this process: GPU %d), threads per PE: %d, regs/thread: %d\n",
          n_pes, n_devs, pes_per_dev, dv.world > 1 ? "one process each" : "virtual, one launch", dev0,
          cfg.threads_per_pe, fa.numRegs);
    else
      PINFO("PEs: %d (%d per SM), SMs: %d, threads per PE: %d, regs/thread: %d\n", n_pes,
          cfg.pes_per_sm, n_sms, cfg.threads_per_pe, fa.numRegs);
    PINFO("Dynamic smem per PE: %ld B (scratch %d B), ring %llu B per PE\n", smem_total,
        g.inf.smem_scratch_bytes, (unsigned long long)cfg.ring_bytes);
  }
  return CHARMING_OK;
}

int charming_run(int argc, char** argv) { return run_scheduler(argc, argv); }

// Stream-ordered timer over any number of runs: CUDA events recorded on the
// runtime's stream, so host time between runs counts as idle device time.
static cudaEvent_t g_timer0 = nullptr, g_timer1 = nullptr;

int charming_timer_start(void) {
  if (!g.inited) return CHARMING_ERR_NOT_INIT;
  cudaError_t e = cudaSuccess;
  if (!g_timer0) e = cudaEventCreate(&g_timer0);
  if (e == cudaSuccess && !g_timer1) e = cudaEventCreate(&g_timer1);
  if (e == cudaSuccess) e = cudaEventRecord(g_timer0, g.stream);
  return cuda_fail(e, "timer start");
}

int charming_timer_stop(double* ms) {
  if (!g.inited || !g_timer0) return CHARMING_ERR_NOT_INIT;
  cudaError_t e = cudaEventRecord(g_timer1, g.stream);
  if (e == cudaSuccess) e = cudaEventSynchronize(g_timer1);
  float f = 0.f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&f, g_timer0, g_timer1);
  if (ms) *ms = f;
  return cuda_fail(e, "timer stop");
}

int charming_fini(void) {
  if (!g.inited) return CHARMING_OK;
  cudaDeviceSynchronize();
  if (g.world > 1) {
    // unmap the peers' regions once no GPU runs; free this one once every
    // peer has unmapped it
    (void)host_barrier();
    for (void* p : g.ipc_opened) cudaIpcCloseMemHandle(p);
    (void)host_barrier();
  }
  g.ipc_opened.clear();
  g.launch_ctrl.clear();
  g.world = 1;
  for (void* p : g.dev_allocs) cudaFree(p);
  g.dev_allocs.clear();
  if (g.d_args) cudaFree(g.d_args);
  g.d_args = nullptr;
  g.d_args_cap = 0;
  if (g.h_stop) cudaFreeHost(g.h_stop);
  g.h_stop = nullptr;
  if (g.ev0) cudaEventDestroy(g.ev0);
  if (g.ev1) cudaEventDestroy(g.ev1);
  if (g.stream) cudaStreamDestroy(g.stream);
  g.ev0 = g.ev1 = nullptr;
  g.stream = nullptr;
  g.inited = false;
  return CHARMING_OK;
}

int charming_get_info(charming_info* out) {
  if (!g.inited) return CHARMING_ERR_NOT_INIT;
  *out = g.inf;
  return CHARMING_OK;
}

int charming_last_stats(charming_stats* out) {
  *out = g.last;
  return CHARMING_OK;
}

const char* charming_status_string(int code) {
  switch (code) {
    case CHARMING_OK: return "ok";
    case CHARMING_ERR_RING_FULL: return "inbox ring full (no space within the wait limit)";
    case CHARMING_ERR_STASH_FULL: return "refnum stash full";
    case CHARMING_ERR_BAD_TARGET: return "invalid chare array, index or entry method";
    case CHARMING_ERR_BARRIER_TIMEOUT: return "barrier timeout";
    case CHARMING_ERR_IDLE_TIMEOUT: return "idle timeout (nothing delivered; missing end()?)";
    case CHARMING_ERR_DEADLINE: return "run deadline exceeded";
    case CHARMING_ERR_BAD_MSG: return "malformed message";
    case CHARMING_ERR_MSG_TOO_LARGE: return "message larger than max_msg_bytes";
    case CHARMING_ERR_HOST_STOP: return "stopped by host";
    case CHARMING_ERR_TOO_MANY_TYPES: return "too many chare types on a PE";
    case CHARMING_ERR_TOO_MANY_EMS: return "too many entry methods";
    case CHARMING_ERR_PIPELINE: return "bulk-copy pipeline wait ran out";
    case CHARMING_ERR_LAUNCH: return "scheduler launch failed";
    case CHARMING_ERR_CONFIG: return "invalid configuration";
    case CHARMING_ERR_CUDA: return "CUDA error";
    case CHARMING_ERR_NOT_INIT: return "runtime not initialised";
    case CHARMING_ERR_NO_MEMORY: return "out of memory";
    case CHARMING_ERR_APP: return "program reported a failure";
    case CHARMING_ERR_TOO_MANY_WAITS: return "too many pending async_waits on a chare array";
    default: return "unknown status";
  }
}

const char* charming_last_error(void) { return g_err.c_str(); }

}  // extern "C"
