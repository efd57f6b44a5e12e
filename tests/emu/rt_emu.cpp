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
// Several GPUs: RT_EMU_VDEVS=n splits the PE blocks into n GPUs in one
// process (each GPU's inbox side its own allocation); RT_EMU_WORLD=w,
// RT_EMU_RANK=r and RT_EMU_DIR=<empty directory> run w processes, one GPU
// each, whose inbox sides are files every process maps shared (in the role
// of CUDA IPC), bootstrapped by the process main's file rendezvous.
// usage (n_pes: PE blocks; with RT_EMU_GPU_LEVEL set they form one PE):
//        rt_emu fanout n_pes ring_bytes n_chares msgs payload seed mode
//        rt_emu hello n_pes ring_bytes
//        rt_emu refnum n_pes ring_bytes reversed
//        rt_emu serve n_pes ring_bytes n_requests seed workers_per_pe
//               max_inflight chare_side dtype(0 f64, 1 f32)
// serve runs the Jacobi2d solve server (apps/jacobi2d.cu in serving mode,
// admission by apps/serve_host.h) with a host thread in the role of the
// request loop: seeded requests of mixed sizes arrive while others run,
// each result is compared bit for bit with the serial oracle.
// The EMU_MT build (rt_emu_mt) runs one PE block of RT_EMU_THREADS threads
// (barriers checked per call site, warps in lockstep) under ThreadSanitizer.
// prints a status line; for fanout also the delivery log (8 u32 per record)
// as hex lines "L w0 ... w7".
#include "cuda_host_shim.h"
#include "../../charming_b200/csrc/rt.cuh"
#include "../../charming_b200/csrc/apps/suite.cuh"
#include "../../charming_b200/csrc/apps/jacobi_types.cuh"
#include "../../charming_b200/csrc/apps/jacobi_sweep.cuh"
#include "../../charming_b200/csrc/apps/serve_host.h"
#include "../../charming_b200/csrc/apps/decomp1d.h"
#include "../../charming_b200/csrc/rendezvous.h"

#include <fcntl.h>
#include <memory>
#include <sys/mman.h>

#include <atomic>
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
bool emu_is_shared(const void* p) {
  const unsigned char* b = reinterpret_cast<const unsigned char*>(s_mem_of_pe);
  const unsigned char* q = static_cast<const unsigned char*>(p);
  return b && q >= b && q < b + SMEM_BYTES;
}

__global__ void charming_scheduler_kernel(int argc, char** argv, size_t* argvs);
__global__ void charming_reset_kernel();
extern suite::app_params g_app;

#ifndef EMU_MT
void emu_sync(const char*, int) {}  // one thread per block
#else
// One PE block of blockDim.x threads: a barrier that checks every thread
// arrives from the same call site, and warps of 32 in lockstep.
namespace {
// Arrivals are counted under a mutex (which also checks the call site);
// waiters spin on the generation word and yield the core, which costs far
// less than a condition-variable wake-up of every thread per barrier (a
// PE block of 64 host threads passes several barriers per message).
struct SiteBarrier {
  std::mutex m;
  int n = 1, count = 0;
  std::atomic<unsigned long long> gen{0};
  const char* file = nullptr;
  int line = 0;
  void sync(const char* f, int l) {
    const unsigned long long g = gen.load(std::memory_order_acquire);
    {
      std::lock_guard<std::mutex> lk(m);
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
        gen.store(g + 1, std::memory_order_release);
        return;
      }
    }
    while (gen.load(std::memory_order_acquire) == g) std::this_thread::yield();
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
unsigned emu_match_any(long long v) {
  Warp& w = my_warp();
  const int lane = (int)(threadIdx.x & 31);
  static_assert(sizeof(w.slot[0]) >= sizeof(long long), "slot");
  memcpy(w.slot[lane], &v, sizeof(v));
  w.bar.sync("match_any", 0);
  unsigned m = 0;
  for (int i = 0; i < 32; i++) {
    long long o;
    memcpy(&o, w.slot[i], sizeof(o));
    if (o == v) m |= 1u << i;
  }
  w.bar.sync("match_any", 1);
  return m;
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

#ifdef EMU_MT
// The bulk-copy sweep is not used by these programs (pipeline = 0); its
// mbarrier model lives in jacobi_emu.cpp.
namespace jac {
[[noreturn]] static void no_tma() {
  fprintf(stderr, "bulk-copy sweep not modelled in rt_emu\n");
  _exit(4);
}
void mbar_init(unsigned long long*, unsigned) { no_tma(); }
void mbar_inval(unsigned long long*) { no_tma(); }
void mbar_expect_tx(unsigned long long*, unsigned) { no_tma(); }
void mbar_arrive(unsigned long long*) { no_tma(); }
bool mbar_test_wait(unsigned long long*, unsigned) { no_tma(); }
bool mbar_try_wait(unsigned long long*, unsigned) { no_tma(); }
void bulk_g2s(void*, const void*, unsigned, unsigned long long*) { no_tma(); }
}  // namespace jac
#endif

unsigned long long charm::rt::globaltimer() {
  return (unsigned long long)std::chrono::duration_cast<std::chrono::nanoseconds>(
             std::chrono::steady_clock::now().time_since_epoch()).count();
}

extern "C" int oracle_jacobi2d_f64(double* grid, int nx, int ny, int sweeps);
// apps/msgbench.cu: host plan of the fan-out (delivery counts, log offsets)
int fanout_plan(int n, int msgs, unsigned long long seed, std::vector<int>& expected,
    std::vector<unsigned long long>& off);
extern "C" int oracle_jacobi2d_f32(float* grid, int nx, int ny, int sweeps, int threads);

// programs of the library that this check does not run
__device__ void suite::jacobi1d_main(int) { charm::end(); }
__device__ void suite::serve_main(int) { charm::end(); }

namespace {

template <typename T>
T* zalloc(size_t n) {
  T* p = static_cast<T*>(aligned_alloc(256, (n * sizeof(T) + 255) / 256 * 256));
  memset(p, 0, (n * sizeof(T) + 255) / 256 * 256);
  return p;
}

int env_int(const char* name, int dflt) {
  const char* v = getenv(name);
  return v ? atoi(v) : dflt;
}

// Several processes: this one's rank and the rendezvous.
int g_rank = 0, g_world = 1;
std::unique_ptr<charm_host::file_rendezvous> g_rdv;

// One GPU's inbox side for pes PEs, carved from base (bytes: inbox_bytes).
size_t inbox_bytes(int pes, const charm::rt::device_state& ds) {
  using namespace charm::rt;
  return 2 * sizeof(line_u64) * pes + 4 * CTRL_WORDS + 8ull * pes + 8ull * ds.ring_cells * pes +
         ds.ring_stride * pes + 4096;
}
charm::rt::dev_inbox carve(unsigned char* base, int pes, const charm::rt::device_state& ds) {
  using namespace charm::rt;
  dev_inbox d{};
  size_t o = 0;
  auto take = [&](size_t n) {
    unsigned char* p = base + o;
    o = (o + n + 255) / 256 * 256;
    return p;
  };
  d.tail = reinterpret_cast<line_u64*>(take(sizeof(line_u64) * pes));
  d.head = reinterpret_cast<line_u64*>(take(sizeof(line_u64) * pes));
  d.ctrl = reinterpret_cast<int*>(take(4 * CTRL_WORDS));
  d.progress = reinterpret_cast<unsigned long long*>(take(8ull * pes));
  d.flags = reinterpret_cast<unsigned long long*>(take(8ull * ds.ring_cells * pes));
  d.ring = take(ds.ring_stride * pes);
  return d;
}

// A file of `bytes` in the shared directory, mapped shared.
unsigned char* map_file(const std::string& path, size_t bytes, bool create) {
  const int fd = open(path.c_str(), create ? (O_RDWR | O_CREAT | O_EXCL) : O_RDWR, 0600);
  if (fd < 0 || (create && ftruncate(fd, (off_t)bytes) != 0)) {
    fprintf(stderr, "cannot %s %s\n", create ? "create" : "open", path.c_str());
    _exit(5);
  }
  void* p = mmap(nullptr, bytes, PROT_READ | PROT_WRITE, MAP_SHARED, fd, 0);
  close(fd);
  if (p == MAP_FAILED) {
    fprintf(stderr, "cannot map %s\n", path.c_str());
    _exit(5);
  }
  return static_cast<unsigned char*>(p);
}

// The parts of charming_init that build the device state. GPU-level mode
// (RT_EMU_GPU_LEVEL set): the n_blocks blocks form one PE.
void init_runtime(int n_blocks, size_t ring_bytes, bool gpu_level) {
  using namespace charm::rt;
  device_state ds{};
  const int vdevs = env_int("RT_EMU_VDEVS", 1);
  g_world = env_int("RT_EMU_WORLD", 1);
  g_rank = env_int("RT_EMU_RANK", 0);
  const int n_devs = g_world > 1 ? g_world : vdevs;
  const int pes_per_dev = g_world > 1 ? n_blocks : n_blocks / vdevs;
  const int n_pes = gpu_level ? 1 : pes_per_dev * n_devs;
  const int n_local = gpu_level ? 1 : n_blocks;
  ds.n_pes = n_pes;
  ds.n_blocks = n_blocks;
  ds.gpu_level = gpu_level ? 1 : 0;
  ds.gl = gpu_level ? zalloc<group_state>(1) : nullptr;
  ds.threads = 1;
  ds.ring_cells = ring_bytes / CELL;
  ds.max_msg = 4096 + 64;
  ds.ring_stride = ds.ring_cells * CELL + ds.max_msg;
  ds.stash_bytes = 4 << 20;
  ds.stash_entries = 4096;
  ds.smem_state_bytes = (int)((sizeof(pe_state) + 8ull * n_pes + 127) / 128 * 128);
  ds.smem_total = SMEM_BYTES;
  ds.smem_arena_bytes = 8 << 10;
  // The run deadline guards against a hung emulation. A PE block of many
  // host threads is slow (every block barrier is a rendezvous of all of
  // them), so its runs get proportionally longer.
  ds.deadline_ns = 60ull * 1000000000ull;
  if (const char* t = getenv("RT_EMU_THREADS")) {
    const int th = atoi(t);
    if (th > 16) ds.deadline_ns = ds.deadline_ns / 16 * (unsigned long long)th;
  }
  ds.idle_timeout_ns = 5ull * 1000000000ull;
  // the inbox side of each GPU (virtual ones: one allocation each; several
  // processes: this one's own file, then the others' files mapped)
  ds.n_devs = n_devs;
  ds.pes_per_dev = gpu_level ? 1 : pes_per_dev;
  ds.n_procs = g_world;
  ds.pe0 = g_world > 1 ? g_rank * pes_per_dev : 0;
  const int P = gpu_level ? 1 : pes_per_dev;
  const size_t ib = inbox_bytes(P, ds);
  if (g_world > 1) {
    const char* dir = getenv("RT_EMU_DIR");
    if (!dir) _exit(5);
    g_rdv.reset(new charm_host::file_rendezvous(dir, g_rank, g_world, 60.0));
    const std::string own = std::string(dir) + "/inbox." + std::to_string(g_rank);
    ds.dev[g_rank] = carve(map_file(own, ib, true), P, ds);
    if (g_rdv->barrier() != 0) _exit(6);  // every file exists at its size
    for (int r = 0; r < g_world; r++)
      if (r != g_rank)
        ds.dev[r] = carve(map_file(std::string(dir) + "/inbox." + std::to_string(r), ib, false), P, ds);
  } else {
    for (int d = 0; d < vdevs; d++) ds.dev[d] = carve(zalloc<unsigned char>(ib), P, ds);
  }
  const int dev0 = g_world > 1 ? g_rank : 0;
  ds.tail = ds.dev[dev0].tail;
  ds.head = ds.dev[dev0].head;
  ds.flags = ds.dev[dev0].flags;
  ds.ring = ds.dev[dev0].ring;
  ds.ctrl = ds.dev[dev0].ctrl;
  ds.progress = ds.dev[dev0].progress;
  ds.stash_keys = zalloc<stash_key>((size_t)ds.stash_entries * n_local);
  ds.stash_data = zalloc<unsigned char>(ds.stash_bytes * n_local);
  ds.proxy_tables = zalloc<charm::chare_proxy_table>(n_local);
  ds.pe_stats = zalloc<unsigned long long>((size_t)N_STATS * n_local);
  ds.pe_times = zalloc<unsigned long long>(3 * (size_t)n_local);
  ds.host_stop = nullptr;
  ds.free_chares_at_exit = 1;
  ds.arena_bytes = 64 << 10;
  ds.arena = zalloc<unsigned char>(ds.arena_bytes * n_local);
  ds.outbox_bytes = 2 * ds.max_msg + (64 << 10);
  ds.outbox_stride = ds.outbox_bytes + (ds.max_msg + OB_HDR + 127) / 128 * 128;
  ds.outbox = zalloc<unsigned char>(ds.outbox_stride * n_local);
  ds.user_heap_bytes = 64 << 10;
  ds.user_blocks_max = 64;
  ds.user_heap = zalloc<unsigned char>(ds.user_heap_bytes * n_local);
  ds.user_blocks = zalloc<user_block>((size_t)ds.user_blocks_max * n_local);
  c_rt = ds;
  c_n_pes = c_n_pes_node = n_pes;
  c_n_sms = n_blocks;
  c_n_nodes = 1;
  c_n_devs = c_n_devs_node = n_devs;
  c_my_dev = c_my_dev_node = dev0;
}

unsigned long long g_deferred = 0;  // sends moved to an outbox in the last run
unsigned long long g_batched = 0;   // deliveries in batches of warp-level entry methods

int run_scheduler(int n_pes, int threads) {
  blockIdx = emu_dim3{0, 0, 0};
  gridDim = emu_dim3{1, 1, 1};
  blockDim = emu_dim3{1, 1, 1};
  charming_reset_kernel();
  // several processes: every GPU resets before any runs
  if (g_rdv && g_rdv->barrier() != 0) _exit(6);
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
  // every process's run has ended: nothing writes this one's words any more
  if (g_rdv && g_rdv->barrier() != 0) _exit(6);
  g_deferred = g_batched = 0;
  const int n_local = charm::rt::c_rt.gpu_level ? 1 : n_pes;
  for (int p = 0; p < n_local; p++) {
    g_deferred += charm::rt::c_rt.pe_stats[(size_t)p * charm::rt::N_STATS + charm::rt::ST_DEFERRED];
    g_batched += charm::rt::c_rt.pe_stats[(size_t)p * charm::rt::N_STATS + charm::rt::ST_BATCHED];
  }
  // the first error any of this process's GPUs recorded
  const int* ctl = charm::rt::c_rt.ctrl;
  const int launch_devs = g_world > 1 ? 1 : charm::rt::c_rt.n_devs;
  for (int d = 0; d < launch_devs && ctl[charm::rt::CTRL_STATUS] == 0; d++)
    ctl = charm::rt::c_rt.dev[(g_world > 1 ? g_rank : 0) + d].ctrl;
  if (ctl[charm::rt::CTRL_STATUS])
    fprintf(stderr, "run status %d: pe %d info %d %d\n", ctl[charm::rt::CTRL_STATUS], ctl[charm::rt::CTRL_ERR_PE],
            ctl[charm::rt::CTRL_ERR_I0], ctl[charm::rt::CTRL_ERR_I1]);
  return ctl[charm::rt::CTRL_STATUS];
}

// ---- serving ---------------------------------------------------------------
struct EmuServe : jserve::sink {
  int Q = 0;
  std::vector<jac::serve_req> req;
  std::vector<jac::chare_desc> stage_d;
  std::vector<jac::prob_desc> stage_p;
  unsigned long long ticket = 0;
  void stage_desc(int w, const jac::chare_desc& d) override { stage_d[w] = d; }
  void stage_prob(int s, const jac::prob_desc& p) override { stage_p[s] = p; }
  void post(int slot, int root, unsigned gen) override {
    jac::serve_req* r = &req[ticket % Q];
    r->slot = slot;
    r->root = root;
    r->gen = gen;
    __atomic_store_n(&r->seq, ticket + 1, __ATOMIC_RELEASE);
    ticket++;
  }
};

double wall_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

template <typename T>
int serve_run(int n_pes, int threads, int n_req, unsigned long long seed, int wpp, int max_inflight, int side) {
  const int n_workers = n_pes * wpp;
  const int OFF = jac::traits<T>::OFF, VEC = jac::traits<T>::VEC;
  std::vector<unsigned char> slab_mem((8u << 20) + 256);
  uintptr_t slab = (reinterpret_cast<uintptr_t>(slab_mem.data()) + 255) & ~uintptr_t(255);
  jserve::params P;
  P.n_pes = n_pes;
  P.workers_per_pe = wpp;
  P.max_inflight = max_inflight;
  P.budget = 8u << 20;
  P.chare_side = side;
  P.esz = sizeof(T);
  P.off = OFF;
  P.vec = VEC;
  jserve::server_state st;
  st.init(P, slab);
  EmuServe sk;
  sk.Q = max_inflight;
  sk.req.assign(max_inflight, jac::serve_req{});
  sk.stage_d.assign(n_workers, jac::chare_desc{});
  sk.stage_p.assign(max_inflight, jac::prob_desc{});
  std::vector<jac::serve_comp> comp(max_inflight);
  std::vector<jac::chare_desc> desc(n_workers);
  std::vector<jac::prob_desc> probs(n_workers);
  std::vector<unsigned long long> ctr(16, 0);
  std::vector<unsigned> done(max_inflight, 0);
  std::vector<int> bm(n_pes, wpp), sm(n_pes, 0), fin(n_workers, 0), ctl(32, 0);
  sm[0] = 1;
  std::vector<unsigned long long> pe_ns(8 * (size_t)n_pes, 0);
  g_app = suite::app_params{};
  g_app.id = suite::APP_JACOBI2D;
  g_app.a[0] = n_workers;
  g_app.a[2] = sizeof(T) == 8 ? CHARMING_F64 : CHARMING_F32;
  g_app.a[6] = 1;
  g_app.a[7] = max_inflight;
  g_app.a[8] = max_inflight;
  g_app.p[0] = desc.data();
  g_app.p[1] = probs.data();
  g_app.p[4] = fin.data();
  g_app.p[5] = bm.data();
  g_app.p[6] = pe_ns.data();
  g_app.p[7] = sk.req.data();
  g_app.p[8] = sk.stage_d.data();
  g_app.p[9] = sk.stage_p.data();
  g_app.p[10] = comp.data();
  g_app.p[11] = ctr.data();
  g_app.p[12] = done.data();
  g_app.p[13] = ctl.data();
  g_app.p[14] = sm.data();

  // seeded requests: sizes that make 1 to ~12 chares, sweep caps, with and
  // without residual checks and early stops
  struct Req {
    charming_jacobi_problem q;
    double at;
  };
  std::vector<Req> reqs(std::max(n_req, 0));
  unsigned long long z = seed;
  auto rnd = [&]() { return suite::mix64(z++); };
  double t = 0;
  for (int i = 0; i < n_req; i++) {
    charming_jacobi_problem q{};
    q.nx = 3 + (int)(rnd() % 45);
    q.ny = 3 + (int)(rnd() % 45);
    q.max_sweeps = (int)(rnd() % 41);
    int k = (int)(rnd() % 3);
    q.check_every = k == 0 ? 0 : (k == 1 ? 5 : 3);
    q.tol = (q.check_every && (rnd() & 1)) ? 0.3 : 0.0;
    for (int e = 0; e < 4; e++) q.bc[e] = (double)(rnd() >> 11) * (1.0 / 9007199254740992.0);
    reqs[i] = Req{q, t};
    t += (double)(rnd() % 2000) * 1e-6;
  }

  if (n_req < 0) {  // a server nobody stops must still end at its deadline
    charm::rt::c_rt.deadline_ns = 1000000000ull;
    int st0 = run_scheduler(n_pes, threads);
    printf("status=%d (deadline)\n", st0);
    return st0 == CHARMING_ERR_DEADLINE ? 0 : 1;
  }
  int status = 0;
  std::atomic<bool> ended{false};
  std::thread sched([&] {
    status = run_scheduler(n_pes, threads);
    ended = true;
  });
  const double t0 = wall_s();
  int next = 0, completed = 0, bad = 0;
  unsigned long long comp_next = 0;
  const double host_limit_s = 2e-9 * (double)charm::rt::c_rt.deadline_ns;
  while (completed < n_req && wall_s() - t0 < host_limit_s && !ended) {
    const double now = wall_s() - t0;
    while (next < n_req && reqs[next].at <= now) {
      if (st.submit(reqs[next].q, (uint64_t)next, now) != CHARMING_OK) {
        printf("S tag=%d refused: %s\n", next, st.err.c_str());
        completed++;  // refused at submission (too large for this pool)
      }
      next++;
    }
    if (st.admit(sk, now) < 0) {
      printf("admit failed: %s\n", st.err.c_str());
      bad++;
      break;
    }
    bool any = false;
    while (true) {
      jac::serve_comp* r = &comp[comp_next % max_inflight];
      if (__atomic_load_n(&r->seq, __ATOMIC_ACQUIRE) != comp_next + 1) break;
      jac::serve_comp c = *r;
      comp_next++;
      any = true;
      jserve::admitted* a = st.complete(c, now);
      if (!a) {
        printf("completion of no request: slot %d gen %u\n", c.slot, c.gen);
        bad++;
        continue;
      }
      const charming_jacobi_problem& q = a->prob;
      const size_t W = q.nx + 2;
      std::vector<T> got((size_t)(q.ny + 2) * W, (T)0), ref((size_t)(q.ny + 2) * W, (T)0);
      for (size_t y = 0; y < (size_t)q.ny + 2; y++)
        for (size_t x = 0; x < W; x++) {
          double v = 0.0;
          if (y == 0) v = q.bc[0];
          else if (y == (size_t)q.ny + 1) v = q.bc[1];
          else if (x == 0) v = q.bc[2];
          else if (x == W - 1) v = q.bc[3];
          ref[y * W + x] = (T)v;
          got[y * W + x] = (T)v;
        }
      for (const jac::chare_desc& d : a->chares) {
        const T* b = reinterpret_cast<const T*>(d.buf[c.final_buf]);
        for (int r2 = 1; r2 <= d.h; r2++)
          for (int c2 = 1; c2 <= d.w; c2++)
            got[(size_t)(d.y0 + r2) * W + d.x0 + c2] = b[(size_t)r2 * d.pitch + OFF - 1 + c2];
      }
      if (sizeof(T) == 8) oracle_jacobi2d_f64(reinterpret_cast<double*>(ref.data()), q.nx, q.ny, c.sweeps);
      else oracle_jacobi2d_f32(reinterpret_cast<float*>(ref.data()), q.nx, q.ny, c.sweeps, 1);
      bool same = memcmp(got.data(), ref.data(), got.size() * sizeof(T)) == 0;
      bool sweeps_ok = q.tol > 0 ? c.sweeps <= q.max_sweeps : c.sweeps == q.max_sweeps;
      printf("R tag=%llu nx=%d ny=%d chares=%zu max=%d K=%d tol=%g sweeps=%d checks=%d gen=%u same=%d\n",
             (unsigned long long)a->tag, q.nx, q.ny, a->chares.size(), q.max_sweeps, q.check_every, q.tol,
             c.sweeps, c.checks, c.gen, same ? 1 : 0);
      if (!same || !sweeps_ok) bad++;
      st.release(a->tag);
      completed++;
    }
    if (!any) std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
  __atomic_store_n(&ctl[0], 1, __ATOMIC_RELEASE);
  sched.join();
  printf("status=%d completed=%d of %d bad=%d peak_inflight=%d peak_bytes=%llu\n", status, completed, n_req,
         bad, st.peak_inflight, (unsigned long long)st.mem.peak());
  return (status == 0 && completed == n_req && bad == 0) ? 0 : 1;
}

}  // namespace

int main(int argc, char** argv) {
  setvbuf(stdout, nullptr, _IOLBF, 0);
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
  init_runtime(n_pes, ring_bytes, getenv("RT_EMU_GPU_LEVEL") != nullptr);
  g_app = suite::app_params{};
  if (app == "fanout") {
    if (argc < 9) return 2;
    int n = atoi(argv[4]), msgs = atoi(argv[5]), payload = atoi(argv[6]);
    unsigned long long seed = strtoull(argv[7], nullptr, 0);
    int mode = atoi(argv[8]);
    int reps = argc >= 10 ? atoi(argv[9]) : 1;
    // argv[10] = 1: a program that never ends (one chare more counted as
    // receiving than receive anything): the idle timeout stops every GPU
    const int never_ends = argc >= 11 ? atoi(argv[10]) : 0;
    size_t total = (size_t)n * msgs;
    std::vector<unsigned int> log(8 * total + 8);
    std::vector<unsigned long long> ctr(8), off;
    std::vector<int> expected;
    const int active = fanout_plan(n, msgs, seed, expected, off);
    int status = 0;
    for (int rep = 0; rep < reps && status == 0; rep++) {  // runs in a row: rings keep their tickets
      std::fill(ctr.begin(), ctr.end(), 0ull);
      std::fill(log.begin(), log.end(), 0u);
      g_app.id = suite::APP_FANOUT;
      g_app.a[0] = n;
      g_app.a[1] = msgs;
      g_app.a[2] = payload;
      g_app.a[3] = (long long)seed;
      g_app.a[4] = mode;
      g_app.a[5] = (long long)total;
      g_app.a[6] = active + never_ends;
      g_app.a[7] = charm::rt::c_rt.n_procs > 1 ? 1 : 0;
      g_app.p[0] = log.data();
      g_app.p[1] = ctr.data();
      g_app.p[2] = expected.data();
      g_app.p[3] = off.data();
      status = run_scheduler(n_pes, threads);
    }
    const int* ectl = charm::rt::c_rt.ctrl;
    printf("status=%d chares_done=%llu deferred=%llu err_pe=%d batched=%llu\n", status, (unsigned long long)ctr[1],
           g_deferred, status ? ectl[charm::rt::CTRL_ERR_PE] : -1, g_batched);
    unsigned long long nrec = total;
    for (unsigned long long r = 0; r < nrec; r++) {
      printf("L");
      for (int k = 0; k < 8; k++) printf(" %08x", log[8 * r + k]);
      printf("\n");
    }
    return never_ends ? 0 : status;
  }
  if (app == "serve") {
    if (argc < 10) return 2;
    int n_req = atoi(argv[4]);
    unsigned long long seed = strtoull(argv[5], nullptr, 0);
    int wpp = atoi(argv[6]), max_inflight = atoi(argv[7]), side = atoi(argv[8]), dt = atoi(argv[9]);
    return dt == 0 ? serve_run<double>(n_pes, threads, n_req, seed, wpp, max_inflight, side)
                   : serve_run<float>(n_pes, threads, n_req, seed, wpp, max_inflight, side);
  }
  if (app == "await") {  // rt_emu await n_pes ring_bytes n_chares broken
    if (argc < 6) return 2;
    int n = atoi(argv[4]), broken = atoi(argv[5]);
    std::vector<unsigned long long> sig(2 * (size_t)n + 2, 0), ctr(2, 0);
    std::vector<int> order(n, -1);
    sig[0] = sig[1] = 1;
    g_app.id = suite::APP_ASYNC_WAIT;
    g_app.a[0] = n;
    g_app.a[1] = broken;
    g_app.p[0] = sig.data();
    g_app.p[1] = order.data();
    g_app.p[2] = ctr.data();
    if (broken) charm::rt::c_rt.idle_timeout_ns = 1000000000ull;
    int status = run_scheduler(n_pes, threads);
    printf("status=%d order=", status);
    for (int v : order) printf("%d,", v);
    printf("\n");
    return 0;
  }
  if (app == "decomp1d") {  // rt_emu decomp1d n_pes ring_bytes n_chares nx ny iters mode
    if (argc < 9) return 2;
    const int n = atoi(argv[4]), nx = atoi(argv[5]), ny = atoi(argv[6]), iters = atoi(argv[7]),
              mode = atoi(argv[8]);
    std::vector<d1_desc> descs;
    std::vector<int> g0;
    std::vector<float> bc;
    if (!decomp1d_plan(n, ny, descs, g0, bc)) return 2;
    const size_t cnt = (size_t)nx * ((ny - 2) / n + 3);
    // exactly the chares' buffers: a read past the last one is an ASan error
    float* base = zalloc<float>(cnt * 2 * n);
    for (int c = 0; c < n; c++)
      for (int r = 1; r <= descs[c].chunk; r++)
        for (int b = 0; b < 2; b++) {
          base[((size_t)c * 2 + b) * cnt + (size_t)r * nx] = bc[g0[c] + r - 1];
          base[((size_t)c * 2 + b) * cnt + (size_t)r * nx + nx - 1] = bc[g0[c] + r - 1];
        }
    std::vector<unsigned long long> sig(2 * (size_t)n + 8, 0);
    g_app.id = suite::APP_DECOMP1D;
    g_app.a[0] = n;
    g_app.a[1] = nx;
    g_app.a[2] = iters;
    g_app.a[3] = mode;
    g_app.a[4] = (long long)cnt;
    g_app.p[0] = base;
    g_app.p[1] = descs.data();
    g_app.p[2] = sig.data();
    g_app.p[3] = sig.data() + 2 * (size_t)n;
    int status = run_scheduler(n_pes, threads);
    printf("status=%d\n", status);
    for (int c = 0; c < n; c++)
      for (int r = 1; r <= descs[c].chunk; r++) {
        printf("G");
        for (int x = 0; x < nx; x++) {
          const float v = base[((size_t)c * 2 + (iters & 1)) * cnt + (size_t)r * nx + x];
          unsigned u;
          memcpy(&u, &v, 4);
          printf(" %08x", u);
        }
        printf("\n");
      }
    return 0;
  }
  if (app == "userheap") {  // rt_emu userheap n_pes ring_bytes n_chares blocks rounds seed
    if (argc < 8) return 2;
    std::vector<unsigned long long> ctr(8, 0);
    g_app.id = suite::APP_USER_HEAP;
    g_app.a[0] = atoi(argv[4]);
    g_app.a[1] = atoi(argv[5]);
    g_app.a[2] = atoi(argv[6]);
    g_app.a[3] = (long long)strtoull(argv[7], nullptr, 0);
    g_app.p[0] = ctr.data();
    int status = run_scheduler(n_pes, threads);
    printf("status=%d taken=%llu bad=%llu failed=%llu checked=%llu freed=%llu done=%llu bytes=%llu\n", status,
           ctr[0], ctr[1], ctr[2], ctr[3], ctr[4], ctr[5], ctr[6]);
    return 0;
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
