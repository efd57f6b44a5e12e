// CPU check of the Jacobi2d chare code (TEST INFRASTRUCTURE ONLY).
//
// Compiles charming_b200/csrc/apps/jacobi2d.cu for the host (see
// cuda_host_shim.h) and runs it on an in-process stand-in for the device
// runtime: one host thread per PE, per-PE FIFO inboxes, the refnum stash
// with revive-in-arrival-order, end() as a global flag. Built with
// AddressSanitizer, so any out-of-bounds access of the chare logic (halo
// pack/unpack, tree slots, descriptors) aborts the run. The sweep is the
// direct-load path; the final grid is compared bit for bit with the serial
// oracle (oracle/jacobi_oracle.c).
//
// usage: jacobi_emu nx ny px py max_sweeps check_every tol dtype(0 f64|1 f32)
//                   n_pes halo_mode [bc_top bc_bottom bc_left bc_right]
// prints: status=<code> sweeps=<n> res0=<x> res_last=<x> exact=<0|1>
#include "cuda_host_shim.h"
#include <charming.h>
#include "../../charming_b200/csrc/apps/suite.cuh"
#include "../../charming_b200/csrc/apps/jacobi_types.cuh"
#include "../../charming_b200/csrc/apps/jacobi_sweep.cuh"

#include <barrier>
#include <chrono>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>

extern "C" int oracle_jacobi2d_f64(double* grid, int nx, int ny, int sweeps);
extern "C" int oracle_jacobi2d_f32(float* grid, int nx, int ny, int sweeps, int threads);

thread_local emu_dim3 threadIdx{0, 0, 0};
thread_local emu_dim3 blockIdx{0, 0, 0};
emu_dim3 blockDim{1, 1, 1};
emu_dim3 gridDim{1, 1, 1};
int c_n_sms, c_my_dev, c_my_dev_node, c_n_devs, c_n_devs_node, c_n_nodes, c_n_pes, c_n_pes_node;
thread_local uint64_t s_mem[16];
namespace charm { namespace rt { device_state c_rt; } }
suite::app_params g_app;

namespace {

using bytes_t = std::vector<unsigned char>;

struct Stashed {
  bytes_t msg;
  bool ready;
};

struct PE {
  std::mutex mu;
  std::deque<bytes_t> inbox;
  charm::chare_proxy_table table;
  std::deque<Stashed> stash;  // arrival order
};

std::vector<PE*> g_pes;
std::atomic<int> g_term{0};
std::atomic<int> g_status{0};
std::atomic<long long> g_progress{0};
int g_err_a = 0, g_err_b = 0;
thread_local int tl_revive = 0;
alignas(128) thread_local unsigned char tl_smem[1 << 16];
std::barrier<>* g_barrier = nullptr;

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
  return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
             std::chrono::steady_clock::now().time_since_epoch()).count();
}
unsigned int smid() { return blockIdx.x; }
void* smem_scratch(size_t* bytes) {
  if (bytes) *bytes = sizeof(tl_smem);
  return tl_smem;
}
void barrier() { g_barrier->arrive_and_wait(); }
void barrier_local() { barrier(); }
int device_atoi(const char* s, int n) {
  int v = 0;
  for (int i = 0; i < n; i++) v = v * 10 + (s[i] - '0');
  return v;
}
namespace rt {
void set_error(int code, int a, int b) {
  int z = 0;
  if (g_status.compare_exchange_strong(z, code)) {
    g_err_a = a;
    g_err_b = b;
  }
  g_term = 1;
}
}  // namespace rt
namespace detail {
chare_proxy_table& my_proxy_table() { return g_pes[blockIdx.x]->table; }
void report_error(int code, int a, int b) { rt::set_error(code, a, b); }
}  // namespace detail
void send_reg_msg(int chare_id, int chare_idx, int ep, void* buf, size_t size, int dst_pe,
    int refnum) {
  push(dst_pe, make_msg(msgtype::regular, chare_id, chare_idx, ep, refnum, buf, size));
}
bool alloc_user_msg(message& msg, int dst_pe, size_t size) {
  size_t total = envelope::alloc_size(msgtype::user, size);
  unsigned char* p = new unsigned char[total]();
  msg.env = reinterpret_cast<envelope*>(p);
  msg.offset = 0;
  msg.dst_pe = dst_pe;
  msg.cells = 0;
  msg.capacity = total - 32;
  return true;
}
void send_user_msg(int chare_id, int chare_idx, int ep, message& msg, size_t size, int refnum) {
  if (!msg.env) return;
  if (size > msg.capacity) rt::set_error(CHARMING_ERR_MSG_TOO_LARGE, msg.dst_pe, (int)size);
  unsigned char* p = reinterpret_cast<unsigned char*>(msg.env);
  push(msg.dst_pe, make_msg(msgtype::user, chare_id, chare_idx, ep, refnum, p + 32, msg.capacity));
  delete[] p;
  msg.env = nullptr;
}
void revive_mismatches(int, int, int) { tl_revive = 1; }
void send_begin_term_msg() { end(); }
}  // namespace charm

namespace suite {
double block_sum_f64(double v) { return v; }
unsigned long long block_sum_u64(unsigned long long v) { return v; }
unsigned long long checksum_block(const void*, unsigned long long n) { return n; }
}  // namespace suite

namespace {

// Delivers one message on this PE: refnum check, entry method or stash.
// Returns false when the message was parked.
bool deliver(PE& pe, bytes_t& m) {
  auto* env = reinterpret_cast<charm::envelope*>(m.data());
  auto* rm = reinterpret_cast<charm::regular_msg*>(m.data() + sizeof(charm::envelope));
  if (env->size != m.size()) {
    charm::rt::set_error(CHARMING_ERR_BAD_MSG, (int)env->size, (int)m.size());
    return true;
  }
  if (rm->chare_id < 0 || rm->chare_id >= pe.table.count) {
    charm::rt::set_error(CHARMING_ERR_BAD_TARGET, rm->chare_id, -1);
    return true;
  }
  charm::chare_proxy_base* p = pe.table.proxies[rm->chare_id];
  if (!p->valid_target(rm->chare_idx, rm->ep_id)) {
    charm::rt::set_error(CHARMING_ERR_BAD_TARGET, rm->chare_id, rm->chare_idx);
    return true;
  }
  if (!p->refnum_matches(rm->chare_idx, rm->refnum)) return false;
  p->call(rm->chare_idx, rm->ep_id, m.data() + 32, rm->refnum);
  g_progress++;
  return true;
}

void revive(PE& pe) {
  for (auto& s : pe.stash) {
    if (s.ready) continue;
    auto* rm = reinterpret_cast<charm::regular_msg*>(s.msg.data() + sizeof(charm::envelope));
    if (pe.table.proxies[rm->chare_id]->refnum_matches(rm->chare_idx, rm->refnum)) s.ready = true;
  }
}

void pe_main(int me, int seed) {
  threadIdx = emu_dim3{0, 0, 0};
  blockIdx = emu_dim3{(unsigned)me, 0, 0};
  PE& pe = *g_pes[me];
  charm::barrier();
  suite::jacobi2d_main(me);
  charm::barrier();
  unsigned rng = 2654435761u * (unsigned)(me + 1) + (unsigned)seed;
  while (!g_term) {
    if (tl_revive) {
      tl_revive = 0;
      revive(pe);
    }
    auto it = std::find_if(pe.stash.begin(), pe.stash.end(), [](const Stashed& s) { return s.ready; });
    if (it != pe.stash.end()) {
      bytes_t m = std::move(it->msg);
      pe.stash.erase(it);
      if (!deliver(pe, m)) pe.stash.push_back(Stashed{std::move(m), false});
      continue;
    }
    bytes_t m;
    {
      std::lock_guard<std::mutex> lk(pe.mu);
      if (!pe.inbox.empty()) {
        m = std::move(pe.inbox.front());
        pe.inbox.pop_front();
      }
    }
    if (m.empty()) {
      rng = rng * 1103515245u + 12345u;
      if ((rng >> 16) % 4 == 0) std::this_thread::yield();
      continue;
    }
    if (!deliver(pe, m)) pe.stash.push_back(Stashed{std::move(m), false});
  }
}

template <typename T>
void cell_init(const jac::chare_desc& d, const jac::prob_desc& p, const double* bc) {
  for (int r = 0; r < d.h + 2; r++) {
    for (int c = 0; c < d.w + 2; c++) {
      int gy = d.y0 + r, gx = d.x0 + c;
      double v = 0.0;
      if (gy == 0) v = bc[0];
      else if (gy == p.ny + 1) v = bc[1];
      else if (gx == 0) v = bc[2];
      else if (gx == p.nx + 1) v = bc[3];
      for (int b = 0; b < 2; b++)
        reinterpret_cast<T*>(d.buf[b])[(size_t)r * d.pitch + jac::traits<T>::OFF - 1 + c] = (T)v;
    }
  }
}

template <typename T>
int run(int nx, int ny, int px, int py, int max_sweeps, int K, double tol, int n_pes,
    int halo_mode, const double bc[4], int seed) {
  constexpr int V = jac::traits<T>::VEC, OFF = jac::traits<T>::OFF;
  const int align_el = 128 / (int)sizeof(T);
  c_n_pes = c_n_pes_node = n_pes;
  c_n_sms = n_pes;
  c_n_nodes = c_n_devs = c_n_devs_node = 1;
  int nc = px * py;
  std::vector<jac::chare_desc> ch(nc);
  for (int cy = 0; cy < py; cy++) {
    for (int cx = 0; cx < px; cx++) {
      int r = cy * px + cx;
      jac::chare_desc& d = ch[r];
      d = jac::chare_desc{};
      d.prob = 0;
      d.cx = cx;
      d.cy = cy;
      d.x0 = jac::split_start(nx, px, cx);
      d.y0 = jac::split_start(ny, py, cy);
      d.w = jac::split_start(nx, px, cx + 1) - d.x0;
      d.h = jac::split_start(ny, py, cy + 1) - d.y0;
      d.pitch = (OFF + d.w + 2 * V + align_el - 1) / align_el * align_el;
      d.nbr[jac::TOP] = cy > 0 ? r - px : -1;
      d.nbr[jac::BOTTOM] = cy < py - 1 ? r + px : -1;
      d.nbr[jac::LEFT] = cx > 0 ? r - 1 : -1;
      d.nbr[jac::RIGHT] = cx < px - 1 ? r + 1 : -1;
      d.rank = r;
      d.parent = r > 0 ? (r - 1) / 2 : -1;
      d.child[0] = 2 * r + 1 < nc ? 2 * r + 1 : -1;
      d.child[1] = 2 * r + 2 < nc ? 2 * r + 2 : -1;
      for (int b = 0; b < 2; b++) {
        size_t bytes = ((size_t)d.pitch * (d.h + 2) * sizeof(T) + 255) / 256 * 256;
        d.buf[b] = aligned_alloc(256, bytes);
        memset(d.buf[b], 0, bytes);
      }
    }
  }
  jac::prob_desc pd{};
  pd.nx = nx; pd.ny = ny; pd.px = px; pd.py = py;
  pd.max_sweeps = max_sweeps;
  pd.check_every = K;
  pd.tol = tol;
  pd.root = 0;
  pd.n_chares = nc;
  for (auto& d : ch) cell_init<T>(d, pd, bc);
  // default block map over PEs (include/chare.h placement rule)
  std::vector<int> block_map(n_pes, nc / n_pes);
  for (int p = 0; p < nc % n_pes; p++) block_map[p]++;
  jac::prob_result res{};
  unsigned long long done = 0;
  std::vector<int> final_buf(nc, 0);
  std::vector<unsigned long long> sweep_ns(n_pes, 0);
  g_app = suite::app_params{};
  g_app.id = suite::APP_JACOBI2D;
  g_app.a[0] = nc;
  g_app.a[1] = 1;
  g_app.a[2] = sizeof(T) == 8 ? CHARMING_F64 : CHARMING_F32;
  g_app.a[3] = 0;
  g_app.a[4] = 0;
  g_app.a[5] = halo_mode;
  g_app.p[0] = ch.data();
  g_app.p[1] = &pd;
  g_app.p[2] = &res;
  g_app.p[3] = &done;
  g_app.p[4] = final_buf.data();
  g_app.p[5] = block_map.data();
  g_app.p[6] = sweep_ns.data();

  for (int p = 0; p < n_pes; p++) g_pes.push_back(new PE());
  std::barrier<> bar(n_pes);
  g_barrier = &bar;
  std::vector<std::thread> th;
  for (int p = 0; p < n_pes; p++) th.emplace_back(pe_main, p, seed);
  // watchdog: stop when nothing was delivered for 3 s
  long long last = -1;
  auto t_last = std::chrono::steady_clock::now();
  while (!g_term) {
    std::this_thread::sleep_for(std::chrono::milliseconds(20));
    long long now_p = g_progress.load();
    if (now_p != last) {
      last = now_p;
      t_last = std::chrono::steady_clock::now();
    } else if (std::chrono::steady_clock::now() - t_last > std::chrono::seconds(3)) {
      charm::rt::set_error(CHARMING_ERR_IDLE_TIMEOUT, 0, 0);
    }
  }
  for (auto& t : th) t.join();

  // gather the final grid and compare with the serial oracle
  std::vector<T> grid((size_t)(nx + 2) * (ny + 2)), ref(grid.size());
  for (int gy = 0; gy < ny + 2; gy++) {
    for (int gx = 0; gx < nx + 2; gx++) {
      int iy = std::min(std::max(gy - 1, 0), ny - 1), ix = std::min(std::max(gx - 1, 0), nx - 1);
      int k = jac::split_owner(ny, py, iy) * px + jac::split_owner(nx, px, ix);
      const jac::chare_desc& d = ch[k];
      grid[(size_t)gy * (nx + 2) + gx] = reinterpret_cast<T*>(d.buf[final_buf[k]])
          [(size_t)(gy - d.y0) * d.pitch + OFF - 1 + (gx - d.x0)];
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
  for (auto& d : ch) {
    free(d.buf[0]);
    free(d.buf[1]);
  }
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
  return dtype == 0 ? run<double>(nx, ny, px, py, ms, K, tol, n_pes, halo, bc, seed)
                    : run<float>(nx, ny, px, py, ms, K, tol, n_pes, halo, bc, seed);
}
