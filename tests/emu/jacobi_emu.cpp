// CPU check of the Jacobi2d chare code (TEST INFRASTRUCTURE ONLY).
//
// Compiles charming_b200/csrc/apps/jacobi2d.cu for the host (see
// cuda_host_shim.h) and runs it on an in-process stand-in for the device
// runtime with the same block-collective contract: every thread of a PE
// block runs the scheduler loop, thread 0 picks the next message, all
// threads run the entry method, sends are collective (thread 0 enqueues
// thread 0's buffer). Per-PE FIFO inboxes, the refnum stash with
// revive-in-arrival-order, end() as a global flag. The final grid is
// compared bit for bit with the serial oracle (oracle/jacobi_oracle.c).
//
// usage: jacobi_emu nx ny px py max_sweeps check_every tol dtype(0 f64|1 f32)
//                   n_pes halo_mode [bc_top bc_bottom bc_left bc_right] [seed]
//                   [threads_per_pe] [pipeline 0|1] [tile_w] [depth] [balance]
// (the EMU_MT build takes n_pes == 1 and threads_per_pe >= 1, a multiple of
// 32 with pipeline 1; the default build takes threads_per_pe == 1)
// prints: status=<code> sweeps=<n> res0=<x> res_last=<x> exact=<0|1>
#include "cuda_host_shim.h"
#include <charming.h>
#include "../../charming_b200/csrc/apps/suite.cuh"
#include "../../charming_b200/csrc/apps/jacobi_types.cuh"
#include "../../charming_b200/csrc/apps/jacobi_sweep.cuh"
#include "../../charming_b200/csrc/apps/jacobi_layout.h"

#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

extern "C" int oracle_jacobi2d_f64(double* grid, int nx, int ny, int sweeps);
extern "C" int oracle_jacobi2d_f32(float* grid, int nx, int ny, int sweeps, int threads);

thread_local emu_dim3 threadIdx{0, 0, 0};
thread_local emu_dim3 blockIdx{0, 0, 0};
emu_dim3 blockDim{1, 1, 1};
emu_dim3 gridDim{1, 1, 1};
int c_n_sms, c_my_dev, c_my_dev_node, c_n_devs, c_n_devs_node, c_n_nodes, c_n_pes, c_n_pes_node;
uint64_t s_mem[16];
namespace charm { namespace rt { device_state c_rt; } }
suite::app_params g_app;

namespace {

using bytes_t = std::vector<unsigned char>;

struct Stashed {
  bytes_t msg;
  bool ready;
};

// Barrier of one PE block (or warp) that also checks that all threads
// arrive from the same call site.
// Arrivals are counted under a mutex (which also checks the call site);
// waiters spin on the generation word and yield the core (much cheaper than
// waking every thread through a condition variable at each barrier).
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
        fprintf(stderr, "barrier divergence: thread %u at %s:%d, others at %s:%d\n", threadIdx.x, f,
                l, file, line);
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

struct PE {
  std::mutex mu;
  std::deque<bytes_t> inbox;
  charm::chare_proxy_table table;
  std::deque<Stashed> stash;  // arrival order
  SiteBarrier bar;
  // broadcast slots of the block (written by thread 0 before a barrier)
  bytes_t cur;
  int action = 0;
  unsigned char* ubuf = nullptr;
  size_t ucap = 0;
  std::vector<double> red;
  int revive = 0;
  charm::message bmsgs[charm::MSG_BATCH_MAX];  // charm::block_messages() of the block
  alignas(128) unsigned char smem[1 << 20];  // charm::smem_scratch() of the block
#ifdef EMU_MT
  struct Warp {
    SiteBarrier bar;
    unsigned char slot[32][8];
    bool flag[32];
  };
  std::vector<Warp*> warps;
#endif
};

std::vector<PE*> g_pes;
std::atomic<int> g_term{0};
std::atomic<int> g_status{0};
std::atomic<long long> g_progress{0};
int g_err_a = 0, g_err_b = 0;
std::mutex g_err_mu;
SiteBarrier g_grid;  // charm::barrier(): all threads of all PEs

PE& me_pe() { return *g_pes[blockIdx.x]; }

bytes_t make_msg(charm::msgtype type, int chare_id, int idx, int ep, int ref, const void* buf,
    size_t size) {
  size_t total = charm::envelope::alloc_size(type, size);
  bytes_t b(total, 0);
  auto* env = reinterpret_cast<charm::envelope*>(b.data());
  env->type = type;
  env->src_pe = (int)blockIdx.x;
  env->size = total;
  auto* rm = reinterpret_cast<charm::regular_msg*>(b.data() + sizeof(charm::envelope));
  rm->chare_id = chare_id;
  rm->chare_idx = idx;
  rm->ep_id = ep;
  rm->refnum = ref;
  if (size && buf) memcpy(b.data() + 32, buf, size);
  return b;
}

void push(int dst, bytes_t&& b) {
  if (dst < 0 || dst >= (int)g_pes.size()) {
    charm::rt::set_error(CHARMING_ERR_BAD_TARGET, -1, dst);
    return;
  }
  std::lock_guard<std::mutex> lk(g_pes[dst]->mu);
  g_pes[dst]->inbox.push_back(std::move(b));
}

}  // namespace

void emu_sync(const char* file, int line) { me_pe().bar.sync(file, line); }

#ifdef EMU_MT
// ---- warps: the 32 threads of a warp meet at every warp-level call ----------
namespace {
PE::Warp& my_warp() { return *me_pe().warps[threadIdx.x / 32]; }
}  // namespace
void emu_syncwarp(const char* file, int line) { my_warp().bar.sync(file, line); }
bool emu_all_sync(bool p) {
  PE::Warp& w = my_warp();
  unsigned lane = threadIdx.x & 31;
  w.flag[lane] = p;
  w.bar.sync("all_sync", 0);
  bool r = true;
  for (int i = 0; i < 32; i++) r = r && w.flag[i];
  w.bar.sync("all_sync", 1);
  return r;
}
unsigned emu_match_any(long long v) {
  PE::Warp& w = my_warp();
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
  PE::Warp& w = my_warp();
  w.flag[threadIdx.x & 31] = p;
  w.bar.sync("any_sync", 0);
  bool r = false;
  for (int i = 0; i < 32; i++) r = r || w.flag[i];
  w.bar.sync("any_sync", 1);
  return r;
}
void emu_shfl(void* v, unsigned bytes, int mode, int arg) {
  PE::Warp& w = my_warp();
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

// ---- mbarriers and bulk copies ----------------------------------------------
// An mbarrier completes its phase when all expected arrivals happened and
// the transaction count is back to zero; bulk copies run on an engine
// thread, after a random delay, and count their bytes down on completion.
namespace {
struct Mbar {
  int expected = 0, pending = 0;
  long long tx = 0;
  unsigned phase = 0;
  int in_flight = 0;
};
std::mutex g_mb_mu;
std::unordered_map<void*, Mbar> g_mb;
struct Copy {
  void* dst;
  const void* src;
  unsigned bytes;
  void* bar;
};
std::mutex g_q_mu;
std::condition_variable g_q_cv;
std::deque<Copy> g_q;
bool g_q_stop = false;
std::vector<std::pair<const unsigned char*, size_t>> g_src_ranges;  // readable grid buffers

void tma_fail(const char* what, const void* p) {
  fprintf(stderr, "tma model: %s (%p)\n", what, p);
  fflush(stderr);
  _exit(5);
}
Mbar& mb_locked(void* b) {
  auto it = g_mb.find(b);
  if (it == g_mb.end()) tma_fail("mbarrier used before init or after inval", b);
  return it->second;
}
void mb_complete_locked(Mbar& m) {
  if (m.pending == 0 && m.tx == 0) {
    m.phase++;
    m.pending = m.expected;
  }
}
void engine() {
  unsigned rng = 12345;
  while (true) {
    Copy c;
    {
      std::unique_lock<std::mutex> lk(g_q_mu);
      g_q_cv.wait(lk, [] { return g_q_stop || !g_q.empty(); });
      if (g_q.empty()) return;
      c = g_q.front();
      g_q.pop_front();
    }
    rng = rng * 1103515245u + 12345u;
    if ((rng >> 16) % 3 == 0) std::this_thread::sleep_for(std::chrono::microseconds((rng >> 8) % 50));
    memcpy(c.dst, c.src, c.bytes);
    std::lock_guard<std::mutex> lk(g_mb_mu);
    Mbar& m = mb_locked(c.bar);
    m.tx -= c.bytes;
    m.in_flight--;
    if (m.tx < 0) tma_fail("more bytes completed than expected", c.bar);
    mb_complete_locked(m);
  }
}
}  // namespace

namespace jac {
void mbar_init(unsigned long long* b, unsigned count) {
  std::lock_guard<std::mutex> lk(g_mb_mu);
  if (g_mb.count(b)) tma_fail("mbarrier initialised twice without inval", b);
  if (reinterpret_cast<uintptr_t>(b) & 7) tma_fail("mbarrier not 8-byte aligned", b);
  Mbar m;
  m.expected = m.pending = (int)count;
  g_mb[b] = m;
}
void mbar_inval(unsigned long long* b) {
  std::lock_guard<std::mutex> lk(g_mb_mu);
  Mbar& m = mb_locked(b);
  if (m.in_flight || m.tx) tma_fail("mbarrier invalidated with copies in flight", b);
  g_mb.erase(b);
}
void mbar_expect_tx(unsigned long long* b, unsigned bytes) {
  std::lock_guard<std::mutex> lk(g_mb_mu);
  Mbar& m = mb_locked(b);
  m.tx += bytes;
  if (--m.pending < 0) tma_fail("more arrivals than expected", b);
  mb_complete_locked(m);
}
void mbar_arrive(unsigned long long* b) {
  std::lock_guard<std::mutex> lk(g_mb_mu);
  Mbar& m = mb_locked(b);
  if (--m.pending < 0) tma_fail("more arrivals than expected", b);
  mb_complete_locked(m);
}
bool mbar_test_wait(unsigned long long* b, unsigned parity) {
  std::lock_guard<std::mutex> lk(g_mb_mu);
  return (mb_locked(b).phase & 1u) != (parity & 1u);
}
bool mbar_try_wait(unsigned long long* b, unsigned parity) {
  bool ok = mbar_test_wait(b, parity);
  if (!ok) {
    // let the copy-engine thread run even when every block thread waits
    // (the device code bounds these waits by a spin count)
    static thread_local unsigned misses = 0;
    if ((++misses & 63) == 0) std::this_thread::sleep_for(std::chrono::microseconds(20));
    else std::this_thread::yield();
  }
  return ok;
}
void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  if ((reinterpret_cast<uintptr_t>(dst) & 15) || (reinterpret_cast<uintptr_t>(src) & 15) ||
      (bytes & 15) || bytes == 0)
    tma_fail("bulk copy not 16-byte aligned", src);
  PE& pe = me_pe();
  const unsigned char* d = static_cast<const unsigned char*>(dst);
  if (d < pe.smem || d + bytes > pe.smem + sizeof(pe.smem)) tma_fail("bulk copy outside shared memory", dst);
  const unsigned char* s = static_cast<const unsigned char*>(src);
  bool ok = false;
  for (auto& r : g_src_ranges) ok = ok || (s >= r.first && s + bytes <= r.first + r.second);
  if (!ok) tma_fail("bulk copy source outside every grid buffer", src);
  {
    std::lock_guard<std::mutex> lk(g_mb_mu);
    mb_locked(bar).in_flight++;
  }
  std::lock_guard<std::mutex> lk(g_q_mu);
  g_q.push_back(Copy{dst, src, bytes, bar});
  g_q_cv.notify_one();
}
}  // namespace jac
#endif

// ---- the runtime interface the chare code uses ------------------------------
namespace charm {
int my_pe() { return (int)blockIdx.x; }
int n_pes() { return c_n_pes; }
int my_pe_node() { return (int)blockIdx.x; }
int n_pes_node() { return c_n_pes; }
int n_nodes() { return 1; }
void end() { g_term = 1; }
void abort() {}
uint64_t now_ns() {
  // the chare code reads the timer around every sweep and send: the
  // watchdog counts that as progress too (one entry method may sweep long)
  g_progress++;
  return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
             std::chrono::steady_clock::now().time_since_epoch()).count();
}
unsigned int smid() { return blockIdx.x; }
namespace rt {
unsigned long long globaltimer() { return now_ns(); }
}  // namespace rt
void* smem_scratch(size_t* bytes) {
  PE& pe = me_pe();
  if (bytes) *bytes = sizeof(pe.smem);
  return pe.smem;
}
void barrier() { g_grid.sync("grid", 0); }
void barrier_local() { barrier(); }
int device_atoi(const char* s, int n) {
  int v = 0;
  for (int i = 0; i < n; i++) v = v * 10 + (s[i] - '0');
  return v;
}
namespace rt {
void set_error(int code, int a, int b) {
  std::lock_guard<std::mutex> lk(g_err_mu);
  int z = 0;
  if (g_status.compare_exchange_strong(z, code)) {
    g_err_a = a;
    g_err_b = b;
  }
  g_term = 1;
}
}  // namespace rt
namespace detail {
void* pe_alloc(size_t) { return nullptr; }  // the device heap (new) serves every object here
bool pe_owns(const void*) { return false; }
chare_proxy_table& my_proxy_table() { return me_pe().table; }
void cache_proxy(int, chare_proxy_base*) {}
void report_error(int code, int a, int b) { rt::set_error(code, a, b); }
}  // namespace detail

// Block-collective, as on the device: thread 0's buffer is sent.
void send_reg_msg(int chare_id, int chare_idx, int ep, void* buf, size_t size, int dst_pe,
    int refnum) {
  emu_sync(__FILE__, __LINE__);
  if (threadIdx.x == 0) push(dst_pe, make_msg(msgtype::regular, chare_id, chare_idx, ep, refnum, buf, size));
  emu_sync(__FILE__, __LINE__);
}
message* block_messages() { return me_pe().bmsgs; }
// whether msg is in the block's shared array (filled by thread 0 alone)
static bool block_shared(const message& msg) {
  PE& pe = me_pe();
  return &msg >= pe.bmsgs && &msg < pe.bmsgs + MSG_BATCH_MAX;
}
bool alloc_user_msg(message& msg, int dst_pe, size_t size) {
  PE& pe = me_pe();
  if (threadIdx.x == 0) {
    size_t total = envelope::alloc_size(msgtype::user, size);
    pe.ubuf = new unsigned char[total]();
    pe.ucap = total - 32;
  }
  emu_sync(__FILE__, __LINE__);
  unsigned char* got = pe.ubuf;
  if (!block_shared(msg) || threadIdx.x == 0) {
    msg.env = reinterpret_cast<envelope*>(got);
    msg.offset = 0;
    msg.dst_pe = dst_pe;
    msg.cells = 0;
    msg.capacity = pe.ucap;
  }
  emu_sync(__FILE__, __LINE__);
  return got != nullptr;
}
void send_user_msg(int chare_id, int chare_idx, int ep, message& msg, size_t size, int refnum) {
  if (!msg.env) return;
  emu_sync(__FILE__, __LINE__);  // payload writes of all threads are done
  if (threadIdx.x == 0) {
    if (size > msg.capacity) rt::set_error(CHARMING_ERR_MSG_TOO_LARGE, msg.dst_pe, (int)size);
    unsigned char* p = reinterpret_cast<unsigned char*>(msg.env);
    push(msg.dst_pe, make_msg(msgtype::user, chare_id, chare_idx, ep, refnum, p + 32, msg.capacity));
    delete[] p;
  }
  emu_sync(__FILE__, __LINE__);
  if (!block_shared(msg) || threadIdx.x == 0) msg.env = nullptr;
  emu_sync(__FILE__, __LINE__);
}
bool alloc_user_msgs(message* msgs, const int* dst_pes, const size_t* sizes, int n) {
  bool ok = true;
  for (int k = 0; k < n; k++) ok = alloc_user_msg(msgs[k], dst_pes[k], sizes[k]) && ok;
  return ok;
}
void send_user_msgs(int chare_id, const int* chare_idx, int ep, message* msgs, const size_t* sizes,
    const int* refnums, int n) {
  for (int k = 0; k < n; k++) send_user_msg(chare_id, chare_idx[k], ep, msgs[k], sizes[k], refnums ? refnums[k] : -1);
}
void revive_mismatches(int, int, int) { me_pe().revive = 1; }
void send_begin_term_msg() { end(); }
}  // namespace charm

namespace suite {
// Fixed order (thread index) like the device's deterministic block sum.
double block_sum_f64(double v) {
  PE& pe = me_pe();
  if (threadIdx.x == 0) pe.red.assign(blockDim.x, 0.0);
  emu_sync(__FILE__, __LINE__);
  pe.red[threadIdx.x] = v;
  emu_sync(__FILE__, __LINE__);
  double s = 0.0;
  for (unsigned i = 0; i < blockDim.x; i++) s += pe.red[i];
  emu_sync(__FILE__, __LINE__);
  return s;
}
unsigned long long block_sum_u64(unsigned long long v) { return v; }
unsigned long long checksum_block(const void*, unsigned long long n) { return n; }
}  // namespace suite

namespace {

enum { ACT_IDLE = 0, ACT_DELIVER = 1, ACT_STOP = 2 };

// Thread 0: validates the message in pe.cur; returns ACT_DELIVER when its
// refnum matches, else parks it in the stash (ACT_IDLE).
int classify(PE& pe) {
  bytes_t& m = pe.cur;
  auto* env = reinterpret_cast<charm::envelope*>(m.data());
  auto* rm = reinterpret_cast<charm::regular_msg*>(m.data() + sizeof(charm::envelope));
  if (env->size != m.size()) {
    charm::rt::set_error(CHARMING_ERR_BAD_MSG, (int)env->size, (int)m.size());
    return ACT_IDLE;
  }
  if (rm->chare_id < 0 || rm->chare_id >= pe.table.count) {
    charm::rt::set_error(CHARMING_ERR_BAD_TARGET, rm->chare_id, -1);
    return ACT_IDLE;
  }
  charm::chare_proxy_base* p = pe.table.proxies[rm->chare_id];
  if (!p->valid_target(rm->chare_idx, rm->ep_id)) {
    charm::rt::set_error(CHARMING_ERR_BAD_TARGET, rm->chare_id, rm->chare_idx);
    return ACT_IDLE;
  }
  if (!p->refnum_matches(rm->chare_idx, rm->refnum)) {
    pe.stash.push_back(Stashed{std::move(m), false});
    return ACT_IDLE;
  }
  return ACT_DELIVER;
}

void revive(PE& pe) {
  for (auto& s : pe.stash) {
    if (s.ready) continue;
    auto* rm = reinterpret_cast<charm::regular_msg*>(s.msg.data() + sizeof(charm::envelope));
    if (pe.table.proxies[rm->chare_id]->refnum_matches(rm->chare_idx, rm->refnum)) s.ready = true;
  }
}

// Thread 0: next action of the block (ready stash entries first, then the
// inbox head).
int next_action(PE& pe, unsigned& rng) {
  if (g_term) return ACT_STOP;
  if (pe.revive) {
    pe.revive = 0;
    revive(pe);
  }
  auto it = std::find_if(pe.stash.begin(), pe.stash.end(), [](const Stashed& s) { return s.ready; });
  if (it != pe.stash.end()) {
    pe.cur = std::move(it->msg);
    pe.stash.erase(it);
    return classify(pe);
  }
  {
    std::lock_guard<std::mutex> lk(pe.mu);
    if (!pe.inbox.empty()) {
      pe.cur = std::move(pe.inbox.front());
      pe.inbox.pop_front();
    } else {
      pe.cur.clear();
    }
  }
  if (pe.cur.empty()) {
    rng = rng * 1103515245u + 12345u;
    if ((rng >> 16) % 4 == 0) std::this_thread::yield();
    return ACT_IDLE;
  }
  return classify(pe);
}

void pe_thread(int me, int tid, int seed) {
  threadIdx = emu_dim3{(unsigned)tid, 0, 0};
  blockIdx = emu_dim3{(unsigned)me, 0, 0};
  PE& pe = *g_pes[me];
  charm::barrier();
  suite::jacobi2d_main(me);
  charm::barrier();
  unsigned rng = 2654435761u * (unsigned)(me + 1) + (unsigned)seed;
  while (true) {
    if (tid == 0) pe.action = next_action(pe, rng);
    emu_sync(__FILE__, __LINE__);
    int act = pe.action;
    if (act == ACT_STOP) break;
    if (act == ACT_DELIVER) {
      auto* rm = reinterpret_cast<charm::regular_msg*>(pe.cur.data() + sizeof(charm::envelope));
      pe.table.proxies[rm->chare_id]->call(rm->chare_idx, rm->ep_id, pe.cur.data() + 32, rm->refnum);
    }
    emu_sync(__FILE__, __LINE__);
    if (tid == 0 && act == ACT_DELIVER) {
      g_progress++;
      pe.cur.clear();
    }
  }
}

// Initial state as init_kernel: boundary values wherever the ghost zone
// position lies on the global grid, interior 0, both buffers.
template <typename T>
void cell_init(const jac::chare_desc& d, const jac::prob_desc& p, const double* bc) {
  const int D = d.depth;
  for (int r = 1 - D; r <= d.h + D; r++) {
    for (int c = 1 - D; c <= d.w + D; c++) {
      int gy = d.y0 + r, gx = d.x0 + c;
      if (gy < 0 || gy > p.ny + 1 || gx < 0 || gx > p.nx + 1) continue;
      double v = 0.0;
      if (gy == 0) v = bc[0];
      else if (gy == p.ny + 1) v = bc[1];
      else if (gx == 0) v = bc[2];
      else if (gx == p.nx + 1) v = bc[3];
      for (int b = 0; b < 2; b++)
        reinterpret_cast<T*>(d.buf[b])[(long long)r * d.pitch + jac::traits<T>::OFF - 1 + c] = (T)v;
    }
  }
}

template <typename T>
int run(int nx, int ny, int px, int py, int max_sweeps, int K, double tol, int n_pes,
    int halo_mode, const double bc[4], int seed, int threads, int pipeline, int tile_w, int depth,
    int balance) {
  constexpr int V = jac::traits<T>::VEC, OFF = jac::traits<T>::OFF;
  c_n_pes = c_n_pes_node = n_pes;
  c_n_sms = n_pes;
  c_n_nodes = c_n_devs = c_n_devs_node = 1;
  // the decomposition and placement of charming_jacobi2d_create
  charming_jacobi_problem q{};
  q.nx = nx;
  q.ny = ny;
  q.px = px;
  q.py = py;
  q.max_sweeps = max_sweeps;
  q.check_every = K;
  q.tol = tol;
  for (int k = 0; k < 4; k++) q.bc[k] = bc[k];
  jac::layout L;
  std::string err;
  if (!jac::build_layout(&q, 1, 0, balance, depth, pipeline, n_pes, (int)sizeof(T), OFF, V, &L, &err)) {
    fprintf(stderr, "layout: %s\n", err.c_str());
    return 2;
  }
  const int nc = (int)L.chares.size();
  char* grids = static_cast<char*>(aligned_alloc(256, L.total_bytes));
  memset(grids, 0, L.total_bytes);
#ifdef EMU_MT
  g_src_ranges.push_back({reinterpret_cast<const unsigned char*>(grids), L.total_bytes});
#endif
  jac::place_buffers(&L, grids, (int)sizeof(T));
  std::vector<jac::chare_desc>& ch = L.chares;
  jac::prob_desc& pd = L.probs[0];
  for (auto& d : ch) cell_init<T>(d, pd, bc);
  std::vector<int>& block_map = L.block_map;
  jac::prob_result res{};
  unsigned long long done = 0;
  std::vector<int> final_buf(nc, 0);
  std::vector<unsigned long long> sweep_ns(8 * (size_t)n_pes, 0);
  g_app = suite::app_params{};
  g_app.id = suite::APP_JACOBI2D;
  g_app.a[0] = nc;
  g_app.a[1] = 1;
  g_app.a[2] = sizeof(T) == 8 ? CHARMING_F64 : CHARMING_F32;
  g_app.a[3] = pipeline;
  g_app.a[4] = tile_w;
  g_app.a[5] = halo_mode;
  g_app.p[0] = ch.data();
  g_app.p[1] = &pd;
  g_app.p[2] = &res;
  g_app.p[3] = &done;
  g_app.p[4] = final_buf.data();
  g_app.p[5] = block_map.data();
  g_app.p[6] = sweep_ns.data();

  blockDim = emu_dim3{(unsigned)threads, 1, 1};
  gridDim = emu_dim3{(unsigned)n_pes, 1, 1};
  for (int p = 0; p < n_pes; p++) {
    g_pes.push_back(new PE());
    g_pes.back()->bar.n = threads;
#ifdef EMU_MT
    for (int w = 0; w < (threads + 31) / 32; w++) {
      g_pes.back()->warps.push_back(new PE::Warp());
      g_pes.back()->warps.back()->bar.n = 32;
    }
#endif
  }
  g_grid.n = n_pes * threads;
#ifdef EMU_MT
  std::thread tma_engine(engine);
#endif
  std::vector<std::thread> th;
  for (int p = 0; p < n_pes; p++)
    for (int t = 0; t < threads; t++) th.emplace_back(pe_thread, p, t, seed);
  // watchdog: stop when nothing was delivered for 20 s (one entry method
  // may run many passes of a chare without neighbours, slowly under the
  // sanitizers); a block that does not leave its loop 5 s after that is
  // stuck in a barrier
  long long last = -1;
  auto t_last = std::chrono::steady_clock::now();
  while (!g_term) {
    std::this_thread::sleep_for(std::chrono::milliseconds(20));
    long long now_p = g_progress.load();
    if (now_p != last) {
      last = now_p;
      t_last = std::chrono::steady_clock::now();
    } else if (std::chrono::steady_clock::now() - t_last > std::chrono::seconds(20)) {
      charm::rt::set_error(CHARMING_ERR_IDLE_TIMEOUT, 0, 0);
    }
  }
  std::thread([] {
    std::this_thread::sleep_for(std::chrono::seconds(5));
    fprintf(stderr, "blocks did not stop (stuck in a barrier)\n");
    fflush(stderr);
    _exit(4);
  }).detach();
  for (auto& t : th) t.join();
#ifdef EMU_MT
  {
    std::lock_guard<std::mutex> lk(g_q_mu);
    g_q_stop = true;
    g_q_cv.notify_all();
  }
  tma_engine.join();
#endif

  // gather the final grid and compare with the serial oracle
  std::vector<T> grid((size_t)(nx + 2) * (ny + 2)), ref(grid.size());
  for (int gy = 0; gy < ny + 2; gy++) {
    for (int gx = 0; gx < nx + 2; gx++) {
      int iy = std::min(std::max(gy - 1, 0), ny - 1), ix = std::min(std::max(gx - 1, 0), nx - 1);
      int k = L.chare_of[jac::split_owner(ny, py, iy) * px + jac::split_owner(nx, px, ix)];
      const jac::chare_desc& d = ch[k];
      grid[(size_t)gy * (nx + 2) + gx] = reinterpret_cast<T*>(d.buf[final_buf[k]])
          [(long long)(gy - d.y0) * d.pitch + OFF - 1 + (gx - d.x0)];
      double v = 0.0;
      if (gy == 0) v = bc[0];
      else if (gy == ny + 1) v = bc[1];
      else if (gx == 0) v = bc[2];
      else if (gx == nx + 1) v = bc[3];
      ref[(size_t)gy * (nx + 2) + gx] = (T)v;
    }
  }
  if (sizeof(T) == 8) oracle_jacobi2d_f64(reinterpret_cast<double*>(ref.data()), nx, ny, res.sweeps);
  else oracle_jacobi2d_f32(reinterpret_cast<float*>(ref.data()), nx, ny, res.sweeps, 1);
  int exact = memcmp(grid.data(), ref.data(), grid.size() * sizeof(T)) == 0;
  printf("status=%d err=%d,%d sweeps=%d checks=%d res0=%.17g res_last=%.17g exact=%d done=%llu\n",
      g_status.load(), g_err_a, g_err_b, res.sweeps, res.checks, res.res0, res.res_last, exact, done);
  free(grids);
  return g_status.load() == 0 && exact ? 0 : 1;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 11) {
    fprintf(stderr, "usage: %s nx ny px py max_sweeps check_every tol dtype n_pes halo_mode [bc x4] [seed]\n", argv[0]);
    return 2;
  }
  int nx = atoi(argv[1]), ny = atoi(argv[2]), px = atoi(argv[3]), py = atoi(argv[4]);
  int ms = atoi(argv[5]), K = atoi(argv[6]);
  double tol = atof(argv[7]);
  int dtype = atoi(argv[8]), n_pes = atoi(argv[9]), halo = atoi(argv[10]);
  double bc[4] = {1.0, 0.0, 0.0, 0.0};
  if (argc >= 15) for (int k = 0; k < 4; k++) bc[k] = atof(argv[11 + k]);
  int seed = argc >= 16 ? atoi(argv[15]) : 1;
  int threads = argc >= 17 ? atoi(argv[16]) : 1;
  int pipeline = argc >= 18 ? atoi(argv[17]) : 0;
  int tile_w = argc >= 19 ? atoi(argv[18]) : 0;
  int depth = argc >= 20 ? atoi(argv[19]) : 1;
  int balance = argc >= 21 ? atoi(argv[20]) : 0;
#ifdef EMU_MT
  if (n_pes != 1 || threads < 1 || (pipeline && threads % 32)) {
    fprintf(stderr, "the threaded build runs one PE block (n_pes 1); the bulk-copy sweep needs whole warps\n");
    return 2;
  }
#else
  if (threads != 1 || pipeline) {
    fprintf(stderr, "the default build runs one thread per PE and the direct sweep\n");
    return 2;
  }
#endif
  return dtype == 0 ? run<double>(nx, ny, px, py, ms, K, tol, n_pes, halo, bc, seed, threads, pipeline, tile_w, depth, balance)
                    : run<float>(nx, ny, px, py, ms, K, tol, n_pes, halo, bc, seed, threads, pipeline, tile_w, depth, balance);
}
