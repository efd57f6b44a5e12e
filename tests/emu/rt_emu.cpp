// CPU check of the runtime itself (TEST INFRASTRUCTURE ONLY).
//
// Compiles charming_b200/csrc/runtime.cu (scheduler loop, inbox rings and
// flags, stash and revive, termination, grid barrier) and the message
// programs of apps/basic.cu and apps/msgbench.cu for the host, and runs the
// scheduler kernel with one host thread per PE block (blockDim.x == 1), the
// PTX acquire/release helpers mapped onto C++ atomics. Built under
// AddressSanitizer and, separately, ThreadSanitizer; small inbox rings make
// tickets wrap many times.
//
// usage: rt_emu fanout n_pes ring_bytes n_chares msgs payload seed mode
//        rt_emu hello n_pes ring_bytes
//        rt_emu refnum n_pes ring_bytes reversed
// The EMU_MT build (rt_emu_mt) runs one PE block of RT_EMU_THREADS threads
// (barriers checked per call site, warps in lockstep) under ThreadSanitizer.
// prints a status line; for fanout also the delivery log (8 u32 per record)
// as hex lines "L w0 ... w7".
#include "cuda_host_shim.h"
#include "../../charming_b200/csrc/rt.cuh"
#include "../../charming_b200/csrc/apps/suite.cuh"

#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

thread_local emu_dim3 threadIdx{0, 0, 0};
thread_local emu_dim3 blockIdx{0, 0, 0};
emu_dim3 blockDim{1, 1, 1};
emu_dim3 gridDim{1, 1, 1};
constexpr size_t SMEM_BYTES = 1 << 16;
thread_local uint64_t* s_mem_of_pe = nullptr;

__global__ void charming_scheduler_kernel(int argc, char** argv, size_t* argvs);
__global__ void charming_reset_kernel();
extern suite::app_params g_app;

#ifndef EMU_MT
void emu_sync(const char*, int) {}  // one thread per block
#else
// One PE block of blockDim.x threads: a barrier that checks every thread
// arrives from the same call site, and warps of 32 in lockstep.
namespace {
struct SiteBarrier {
  std::mutex m;
  std::condition_variable cv;
  int n = 1, count = 0;
  unsigned long long gen = 0;
  const char* file = nullptr;
  int line = 0;
  void sync(const char* f, int l) {
    std::unique_lock<std::mutex> lk(m);
    if (count == 0) {
      file = f;
      line = l;
    } else if (l != line || strcmp(f, file) != 0) {
      fprintf(stderr, "barrier divergence: thread %u at %s:%d, others at %s:%d\n", threadIdx.x, f, l,
              file, line);
      fflush(stderr);
      _exit(3);
    }
    if (++count == n) {
      count = 0;
      gen++;
      cv.notify_all();
    } else {
      unsigned long long g = gen;
      cv.wait(lk, [&] { return gen != g; });
    }
  }
};
SiteBarrier g_block;
struct Warp {
  SiteBarrier bar;
  unsigned char slot[32][8];
  bool flag[32];
};
std::vector<Warp*> g_warps;
Warp& my_warp() { return *g_warps[threadIdx.x / 32]; }
}  // namespace
void emu_sync(const char* file, int line) { g_block.sync(file, line); }
void emu_syncwarp(const char* file, int line) { my_warp().bar.sync(file, line); }
bool emu_all_sync(bool p) {
  Warp& w = my_warp();
  w.flag[threadIdx.x & 31] = p;
  w.bar.sync("all_sync", 0);
  bool r = true;
  for (int i = 0; i < 32; i++) r = r && w.flag[i];
  w.bar.sync("all_sync", 1);
  return r;
}
bool emu_any_sync(bool p) {
  Warp& w = my_warp();
  w.flag[threadIdx.x & 31] = p;
  w.bar.sync("any_sync", 0);
  bool r = false;
  for (int i = 0; i < 32; i++) r = r || w.flag[i];
  w.bar.sync("any_sync", 1);
  return r;
}
void emu_shfl(void* v, unsigned bytes, int mode, int arg) {
  Warp& w = my_warp();
  int lane = (int)(threadIdx.x & 31);
  memcpy(w.slot[lane], v, bytes);
  w.bar.sync("shfl", 0);
  int src = lane;
  if (mode == 0 && lane - arg >= 0) src = lane - arg;
  if (mode == 1 && lane + arg < 32) src = lane + arg;
  if (mode == 2) src = lane ^ arg;
  if (mode == 3) src = arg & 31;
  memcpy(v, w.slot[src], bytes);
  w.bar.sync("shfl", 1);
}
#endif

unsigned long long charm::rt::globaltimer() {
  return (unsigned long long)std::chrono::duration_cast<std::chrono::nanoseconds>(
             std::chrono::steady_clock::now().time_since_epoch()).count();
}

// programs of the library that this check does not run
__device__ void suite::jacobi2d_main(int) { charm::end(); }
__device__ void suite::jacobi1d_main(int) { charm::end(); }
__device__ void suite::serve_main(int) { charm::end(); }

namespace {

template <typename T>
T* zalloc(size_t n) {
  T* p = static_cast<T*>(aligned_alloc(256, (n * sizeof(T) + 255) / 256 * 256));
  memset(p, 0, (n * sizeof(T) + 255) / 256 * 256);
  return p;
}

// The parts of charming_init that build the device state.
void init_runtime(int n_pes, size_t ring_bytes) {
  using namespace charm::rt;
  device_state ds{};
  ds.n_pes = n_pes;
  ds.threads = 1;
  ds.ring_cells = ring_bytes / CELL;
  ds.max_msg = 4096 + 64;
  ds.ring_stride = ds.ring_cells * CELL + ds.max_msg;
  ds.stash_bytes = 4 << 20;
  ds.stash_entries = 4096;
  ds.smem_state_bytes = (int)((sizeof(pe_state) + 8ull * n_pes + 127) / 128 * 128);
  ds.smem_total = SMEM_BYTES;
  ds.deadline_ns = 60ull * 1000000000ull;
  ds.idle_timeout_ns = 5ull * 1000000000ull;
  ds.tail = zalloc<line_u64>(n_pes);
  ds.head = zalloc<line_u64>(n_pes);
  ds.flags = zalloc<unsigned long long>(ds.ring_cells * n_pes);
  ds.ring = zalloc<unsigned char>(ds.ring_stride * n_pes);
  ds.stash_keys = zalloc<stash_key>((size_t)ds.stash_entries * n_pes);
  ds.stash_data = zalloc<unsigned char>(ds.stash_bytes * n_pes);
  ds.proxy_tables = zalloc<charm::chare_proxy_table>(n_pes);
  ds.ctrl = zalloc<int>(CTRL_WORDS);
  ds.progress = zalloc<unsigned long long>(n_pes);
  ds.pe_stats = zalloc<unsigned long long>((size_t)N_STATS * n_pes);
  ds.pe_times = zalloc<unsigned long long>(3 * (size_t)n_pes);
  ds.host_stop = nullptr;
  ds.free_chares_at_exit = 1;
  ds.arena_bytes = 64 << 10;
  ds.arena = zalloc<unsigned char>(ds.arena_bytes * n_pes);
  c_rt = ds;
  c_n_pes = c_n_pes_node = c_n_sms = n_pes;
  c_n_nodes = c_n_devs = c_n_devs_node = 1;
}

int run_scheduler(int n_pes, int threads) {
  blockIdx = emu_dim3{0, 0, 0};
  gridDim = emu_dim3{1, 1, 1};
  blockDim = emu_dim3{1, 1, 1};
  charming_reset_kernel();
  gridDim = emu_dim3{(unsigned)n_pes, 1, 1};
  blockDim = emu_dim3{(unsigned)threads, 1, 1};
#ifdef EMU_MT
  g_block.n = threads;
  for (auto* w : g_warps) delete w;
  g_warps.clear();
  for (int k = 0; k < (threads + 31) / 32; k++) {
    g_warps.push_back(new Warp());
    g_warps.back()->bar.n = 32;
  }
#endif
  std::vector<std::vector<uint64_t>> block_mem(n_pes, std::vector<uint64_t>(SMEM_BYTES / 8 + 16));
  std::vector<std::thread> th;
  for (int p = 0; p < n_pes; p++) {
    for (int t = 0; t < threads; t++) {
      uint64_t* mem = reinterpret_cast<uint64_t*>(
          (reinterpret_cast<uintptr_t>(block_mem[p].data()) + 127) & ~uintptr_t(127));
      th.emplace_back([p, t, mem] {
        s_mem_of_pe = mem;
        threadIdx = emu_dim3{(unsigned)t, 0, 0};
        blockIdx = emu_dim3{(unsigned)p, 0, 0};
        charming_scheduler_kernel(0, nullptr, nullptr);
      });
    }
  }
  for (auto& t : th) t.join();
  return charm::rt::c_rt.ctrl[charm::rt::CTRL_STATUS];
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 4) {
    fprintf(stderr, "usage: %s fanout|hello|refnum n_pes ring_bytes ...\n", argv[0]);
    return 2;
  }
  std::string app = argv[1];
  int n_pes = atoi(argv[2]);
  int threads = 1;
  if (const char* t = getenv("RT_EMU_THREADS")) threads = atoi(t);
#ifdef EMU_MT
  if (n_pes != 1) {
    fprintf(stderr, "the threaded build runs one PE block\n");
    return 2;
  }
#else
  if (threads != 1) return 2;
#endif
  size_t ring_bytes = strtoull(argv[3], nullptr, 10);
  init_runtime(n_pes, ring_bytes);
  g_app = suite::app_params{};
  if (app == "fanout") {
    if (argc < 9) return 2;
    int n = atoi(argv[4]), msgs = atoi(argv[5]), payload = atoi(argv[6]);
    unsigned long long seed = strtoull(argv[7], nullptr, 0);
    int mode = atoi(argv[8]);
    int reps = argc >= 10 ? atoi(argv[9]) : 1;
    size_t total = (size_t)n * msgs;
    std::vector<unsigned int> log(8 * total + 8);
    std::vector<unsigned long long> ctr(8);
    std::vector<int> expected(total);
    int status = 0;
    for (int rep = 0; rep < reps && status == 0; rep++) {  // runs in a row: rings keep their tickets
      std::fill(ctr.begin(), ctr.end(), 0ull);
      std::fill(expected.begin(), expected.end(), 0);
      g_app.id = suite::APP_FANOUT;
      g_app.a[0] = n;
      g_app.a[1] = msgs;
      g_app.a[2] = payload;
      g_app.a[3] = (long long)seed;
      g_app.a[4] = mode;
      g_app.a[5] = (long long)total;
      g_app.p[0] = log.data();
      g_app.p[1] = ctr.data();
      g_app.p[2] = expected.data();
      status = run_scheduler(n_pes, threads);
    }
    printf("status=%d delivered=%llu\n", status, (unsigned long long)ctr[1]);
    unsigned long long nrec = std::min<unsigned long long>(ctr[0], total);
    for (unsigned long long r = 0; r < nrec; r++) {
      printf("L");
      for (int k = 0; k < 8; k++) printf(" %08x", log[8 * r + k]);
      printf("\n");
    }
    return status;
  }
  if (app == "hello" || app == "refnum") {
    std::vector<int> out(4 * n_pes + 16, -1);
    g_app.id = app == "hello" ? suite::APP_HELLO : suite::APP_REFNUM;
    g_app.a[0] = (app == "refnum" && argc >= 5) ? atoi(argv[4]) : 0;
    g_app.p[0] = out.data();
    int status = run_scheduler(n_pes, threads);
    printf("status=%d out=", status);
    for (int v : out) printf("%d,", v);
    printf("\n");
    return status;
  }
  return 2;
}
