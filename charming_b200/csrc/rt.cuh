// Internal device-runtime definitions shared by the scheduler, the transport
// and the built-in programs. Not part of the public API.
//
// Memory layout in HBM (one GPU, n_pes PE thread blocks):
//   tail[pe], head[pe]      ticket counters of PE pe's inbox ring, one 128-B
//                           line each (senders atomicAdd tail; the owner
//                           publishes head with st.release)
//   flags[pe][C]            per-cell sequence word: ticket+1 of the message
//                           that starts in that cell, stored with st.release
//   ring[pe]                C cells of CELL bytes + an overhang of max_msg
//                           bytes, so that a message never wraps: one whose
//                           cells run past the end continues in the overhang
//   stash_keys[pe][S]       descriptors of messages whose refnum mismatched
//   stash_data[pe]          byte arena holding those messages
//   outbox[pe]              sends deferred because their destination's ring
//                           had no space: each holds its ticket and the
//                           whole message, copied into the ring once the
//                           receiver has consumed up to that ticket
//   user_heap[pe]           malloc_user / free_user blocks of the PE
// Cell and flag indices are (ticket mod C); C is a power of two.
//
// A run over several GPUs (one process per GPU, one NVSwitch domain; the
// multi-GPU build of the library, see multi_dev() below): global
// PE p is local PE p % pes_per_dev of GPU p / pes_per_dev. Each GPU's inbox
// side (tail, head, flags, ring, control words, progress stamps) is one
// allocation; the others reach it through device_state::dev[], mapped with
// CUDA IPC. A sender writes straight into the receiver's ring over NVLink:
// no relay PE between GPUs. The ticket atomics, sequence words, heads and
// control words then use system scope.
#pragma once

#include <charming.h>
#include "../../include/charming_c.h"

namespace charm {
namespace rt {

constexpr int CELL = 32;                 // ring cell, bytes
constexpr int HDR = 32;                  // envelope (16) + regular_msg (16)
#ifndef CHARMING_MAX_THREADS
#define CHARMING_MAX_THREADS 512
#endif
constexpr int MAX_THREADS = CHARMING_MAX_THREADS;  // launch bound of the scheduler
constexpr int PROXY_CACHE = 16;          // proxies per PE looked up on chip
constexpr int SMEM_OBJ_MAX = 4096;       // larger objects skip the on-chip arena
constexpr int RQ_MAX = 256;              // ready stash entries listed on chip

struct alignas(128) line_u64 {
  unsigned long long v;
  unsigned long long pad[15];
};

// Stash descriptor, 32 B.
struct stash_key {
  int chare_id;
  int chare_idx;
  int refnum;
  int state;                    // 0 consumed, 1 waiting, 2 ready
  unsigned long long data_off;  // virtual byte offset in the PE's arena
  unsigned int bytes;
  int src_pe;
};

enum : int { KEY_FREE = 0, KEY_WAIT = 1, KEY_READY = 2 };

// Outbox entry header, 32 B; the message (envelope, header, payload) follows.
struct ob_entry {
  int dst;
  int state;                    // OB_FILLING until the send publishes it
  unsigned long long ticket;    // ticket taken in dst's inbox
  unsigned long long bytes;     // message bytes
  unsigned long long span;      // bytes of this entry in the outbox
};
enum : int { OB_FILLING = 0, OB_READY = 1 };
constexpr int OB_HDR = 32;
// A send that found no ring space for this long is moved to the outbox.
constexpr unsigned long long DEFER_AFTER_NS = 20000;

// malloc_user block record (per PE ring of records, oldest first).
struct user_block {
  unsigned long long off;       // virtual offset in the PE's user heap
  unsigned long long span;      // bytes taken, wrap padding included
  unsigned long long start;     // offset of the block's memory in the heap
  int freed;
  int pad;
};

enum : int {
  ST_DELIVERED = 0,   // entry methods run
  ST_SENT,            // messages sent
  ST_STASHED,         // messages parked on refnum mismatch
  ST_REVIVED,         // stashed messages made ready
  ST_BYTES_SENT,      // payload bytes sent
  ST_IDLE_POLLS,      // empty inbox polls
  ST_SPACE_WAITS,     // sends that waited for ring space
  ST_LOOP_NS,         // ns spent in the scheduler loop
  ST_IDLE_CYC,        // SM cycles spent waiting on an empty inbox
  ST_EM_CYC,          // SM cycles spent inside entry methods
  ST_DEFERRED,        // sends moved to the outbox (destination ring full)
  ST_TICKET_NS,       // ns the reserving thread waited for its ticket atomics
  ST_SPACE_NS,        // ns it then waited for ring space (head cache and waits)
  ST_BATCHED,         // deliveries run beside others in a batch of warp-level entry methods
  N_STATS = 14
};

constexpr int MAX_DEVS = 8;  // GPUs of one NVSwitch domain

// The inbox side of one GPU's PEs as this process addresses it: its own
// memory, or a peer GPU's mapped over NVLink.
struct dev_inbox {
  line_u64* tail;                      // [pes_per_dev]
  line_u64* head;                      // [pes_per_dev]
  unsigned long long* flags;           // [pes_per_dev][C]
  unsigned char* ring;                 // [pes_per_dev][ring_stride]
  int* ctrl;                           // [CTRL_WORDS]
  unsigned long long* progress;        // [pes_per_dev]
};

// Device-wide runtime description, copied to __constant__ memory before each
// launch.
struct device_state {
  int n_pes;
  int threads;
  unsigned long long ring_cells;       // C (power of two)
  unsigned long long ring_stride;      // bytes per PE ring region
  unsigned long long max_msg;          // bytes, envelope included
  unsigned long long stash_bytes;      // arena bytes per PE
  int stash_entries;                   // descriptors per PE
  int smem_state_bytes;                // bytes of dynamic smem the runtime keeps
  int smem_arena_bytes;                // then this much for the on-chip object arena
  unsigned long long smem_total;       // dynamic smem bytes per PE
  unsigned long long deadline_ns;      // run limit, relative to kernel start
  unsigned long long idle_timeout_ns;  // no delivery anywhere for this long
  line_u64* tail;
  line_u64* head;
  unsigned long long* flags;
  unsigned char* ring;
  stash_key* stash_keys;
  unsigned char* stash_data;
  chare_proxy_table* proxy_tables;
  int* ctrl;                           // see CTRL_* below
  unsigned long long* progress;        // [n_pes] last delivery (globaltimer)
  unsigned long long* pe_stats;        // [n_pes][N_STATS]
  unsigned long long* pe_times;        // [n_pes][2] loop start / end
  volatile int* host_stop;             // mapped host word, may be null
  int free_chares_at_exit;
  unsigned char* arena;                // [n_pes][arena_bytes]: per-run bump allocator
  unsigned long long arena_bytes;      // per PE
  unsigned char* outbox;               // [n_pes][outbox_stride]: deferred sends
  unsigned long long outbox_bytes;     // ring part per PE (entries may run
                                       // past it into an overhang of max_msg + OB_HDR)
  unsigned long long outbox_stride;
  unsigned char* user_heap;            // [n_pes][user_heap_bytes]: malloc_user
  unsigned long long user_heap_bytes;
  user_block* user_blocks;             // [n_pes][user_blocks_max]
  int user_blocks_max;
  unsigned int idle_sleep_ns;          // pause between inbox polls of a PE idle for 32 polls
  int gpu_level;                       // 1: all blocks form PE 0 (group_state below)
  int n_blocks;                        // thread blocks of the launch (n_pes when 0)
  struct group_state* gl;              // GPU-level mode only
  // several GPUs (n_devs > 1); with one GPU, dev[0] holds the fields above
  int n_devs;                          // GPUs of the run
  int pes_per_dev;                     // PEs on each GPU
  int pe0;                             // global PE of this launch's block 0
  int n_procs;                         // processes (1: GPUs emulated in one launch)
  dev_inbox dev[MAX_DEVS];
};

// GPU-level mode (the reference's default build, src/sched/scheduler.cu:
// 240-333): every thread block of the launch belongs to PE 0. Block 0 runs
// the scheduler; all blocks run each entry method and each collective send
// (the reference's barrier_local() = grid sync between the steps). Thread 0
// of block 0 writes these records before a grid barrier; the other blocks
// read them after it with L1-bypassing loads. Collective calls alternate
// between the two slots, so a slot is rewritten only after every block has
// passed the next call's first barrier.
struct group_slot {
  void* ptr[MSG_BATCH_MAX];                // message starts
  unsigned long long u0[MSG_BATCH_MAX];    // bytes
  unsigned long long u1[MSG_BATCH_MAX];    // tickets
  int i0, i1;
};
struct group_state {
  int act, idx, ep, pad;                   // the scheduler's decision
  void* p;                                 // proxy
  void* arg;                               // entry-method argument
  group_slot slot[2];
};

// Words of device_state::ctrl (each on its own 128-B line).
enum : int {
  CTRL_TERM = 0,        // termination request
  CTRL_STATUS = 32,     // first error code
  CTRL_ERR_PE = 33,
  CTRL_ERR_I0 = 34,
  CTRL_ERR_I1 = 35,
  CTRL_BAR_COUNT = 64,
  CTRL_BAR_GEN = 96,
  CTRL_XBAR = 128,      // GPU 0 only: arrivals at cross-process barriers
  CTRL_WORDS = 160
};

extern __constant__ device_state c_rt;

// Per-PE scheduler state at the start of dynamic shared memory.
struct pe_state {
  int my_pe;
  int term;                 // this PE leaves its loop
  int sent_term;
  int revive_pending;
  unsigned long long head;  // next inbox ticket to consume
  unsigned long long t0;    // kernel start (globaltimer)
  // stash
  unsigned long long key_head, key_tail;
  unsigned long long arena_head, arena_tail;
  int n_waiting, n_ready;
  // the scheduler's decision for the block (written by thread 0 before the
  // loop's first barrier; sends inside entry methods use the b_* slots)
  int d_act;
  int d_idx, d_ep;
  unsigned int d_cells;     // ring cells of the message being delivered
  void* d_p;                // proxy, outbox entry or stash arena destination
  void* d_arg;              // entry-method argument or stash copy source
  unsigned long long d_key; // stash key index of a stash delivery
  unsigned long long d_bytes;
  unsigned long long ready_cursor;  // stash keys before it are not ready
  // ready stashed messages found by the last revive, in key order (offsets
  // from rq_base); rq_over: more than RQ_MAX, scan from ready_cursor instead
  unsigned long long rq_base;
  int rq_n, rq_pos, rq_over;
  unsigned int rq[RQ_MAX];
  // block-collective broadcast slots
  void* b_ptr0;
  const void* b_ptr1;
  unsigned long long b_u0, b_u1;
  int b_i0, b_i1, b_i2, b_i3, b_i4, b_i5;
  int red_i[4];
  unsigned long long red_u[4];
  unsigned long long stats[N_STATS];
  unsigned long long idle_polls_since_check;
  unsigned long long busy_polls;       // messages found waiting (end-of-run checks every 64)
  unsigned long long head_pub;         // head last published to the senders
  unsigned long long arena_top;        // bytes of this PE's arena handed out this run
  unsigned long long sarena_top;       // bytes of the on-chip arena handed out this run
  // outbox (deferred sends): virtual byte offsets, entries in send order
  unsigned long long ob_head, ob_tail;
  int ob_count;
  int ob_lock;                         // held by the thread allocating an entry
  // malloc_user heap: virtual byte offsets and block records
  unsigned long long uh_head, uh_tail;
  unsigned long long ub_head, ub_tail;
  int aw_count;                        // pending async_waits on this PE
  unsigned int gl_seq;                 // GPU-level mode: collective calls of this block
  int bar_ok;                          // the last grid barrier completed
  unsigned long long stamped_delivered;  // deliveries at the last progress stamp
  unsigned long long idle_sum;         // PE 0: sum of all progress counters at the last check
  unsigned long long idle_change_ns;   // PE 0: when that sum last changed
  unsigned long long slow_check_ns;    // last host-stop / idle-timeout check
  unsigned long long idle_checks;
  chare_proxy_base* pcache[PROXY_CACHE];  // proxies[0..PROXY_CACHE) of this PE's table
  // a batch of warp-level deliveries (consecutive inbox messages to
  // different chares, one per warp): thread 0 picks the first, warp 0's
  // scan adds the rest
  int nb;                              // deliveries in the batch
  unsigned int nb_cells;               // ring cells they take from the head
  unsigned long long bkey0;            // chare of the first (array << 32 | index)
  chare_proxy_base* bp[MAX_THREADS / 32];
  void* barg[MAX_THREADS / 32];
  int bidx[MAX_THREADS / 32], bep[MAX_THREADS / 32];
  unsigned long long bstash[MAX_THREADS / 32];  // stash keys of a stash batch
  unsigned long long bkeys[MAX_THREADS / 32];   // its chares
  // the block-shared message array of block_messages() (raw storage: the
  // block's state is never constructed)
  alignas(16) unsigned char bmsg[MSG_BATCH_MAX * sizeof(message)];
  // batched sends (alloc_user_msgs): per message start, ticket, bytes
  void* bm_ptr[MSG_BATCH_MAX];
  unsigned long long bm_tick[MSG_BATCH_MAX];
  unsigned long long bm_bytes[MSG_BATCH_MAX];
  // followed by head_cache[n_pes] (unsigned long long), then scratch
};

__device__ __forceinline__ pe_state* pes() { return reinterpret_cast<pe_state*>(s_mem); }
__device__ __forceinline__ unsigned long long* head_cache() {
  return reinterpret_cast<unsigned long long*>(reinterpret_cast<char*>(s_mem) + sizeof(pe_state));
}

// ---- PTX helpers ----------------------------------------------------------
#ifndef CHARMING_HOST_EMULATION
__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" :: "l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u32(unsigned int* p, unsigned int v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" :: "l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ int ld_relaxed_s32(const int* p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ int ld_sys_s32(const volatile int* p) {
  int v;
  asm volatile("ld.relaxed.sys.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" :: "l"(p), "l"(v) : "memory");
}
// A word of shared memory that other threads of the block update with
// atomics.
__device__ __forceinline__ unsigned long long ld_volatile_shared_u64(const unsigned long long* p) {
  return *reinterpret_cast<const volatile unsigned long long*>(p);
}
// System scope: words in mapped host memory shared with the host.
__device__ __forceinline__ unsigned long long ld_acquire_sys_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.sys.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned long long ld_relaxed_sys_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.sys.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_sys_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.release.sys.global.u64 [%0], %1;" :: "l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed_sys_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.relaxed.sys.global.u64 [%0], %1;" :: "l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned int ld_acquire_sys_u32(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.sys.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
// Acquire side for data published before words read with relaxed loads.
__device__ __forceinline__ void fence_acq_rel_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }
// A signal word polled relaxed, made an acquire by fence_acq_rel_gpu on a hit.
__device__ __forceinline__ unsigned long long ld_signal_u64(const unsigned long long* p) {
  return ld_relaxed_u64(p);
}
__device__ __forceinline__ unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
#else
// The CPU check of the runtime (tests/emu) maps these onto C++ atomics.
inline unsigned long long ld_acquire_u64(const unsigned long long* p) { return __atomic_load_n(p, __ATOMIC_ACQUIRE); }
inline void st_release_u64(unsigned long long* p, unsigned long long v) { __atomic_store_n(p, v, __ATOMIC_RELEASE); }
inline unsigned int ld_acquire_u32(const unsigned int* p) { return __atomic_load_n(p, __ATOMIC_ACQUIRE); }
inline void st_release_u32(unsigned int* p, unsigned int v) { __atomic_store_n(p, v, __ATOMIC_RELEASE); }
inline int ld_relaxed_s32(const int* p) { return __atomic_load_n(p, __ATOMIC_RELAXED); }
inline int ld_sys_s32(const volatile int* p) { return __atomic_load_n(const_cast<const int*>(p), __ATOMIC_RELAXED); }
inline unsigned long long ld_relaxed_u64(const unsigned long long* p) { return __atomic_load_n(p, __ATOMIC_RELAXED); }
inline void st_relaxed_u64(unsigned long long* p, unsigned long long v) { __atomic_store_n(p, v, __ATOMIC_RELAXED); }
inline unsigned long long ld_volatile_shared_u64(const unsigned long long* p) { return __atomic_load_n(p, __ATOMIC_RELAXED); }
inline unsigned long long ld_acquire_sys_u64(const unsigned long long* p) { return __atomic_load_n(p, __ATOMIC_ACQUIRE); }
inline unsigned long long ld_relaxed_sys_u64(const unsigned long long* p) { return __atomic_load_n(p, __ATOMIC_RELAXED); }
inline void st_release_sys_u64(unsigned long long* p, unsigned long long v) { __atomic_store_n(p, v, __ATOMIC_RELEASE); }
inline void st_relaxed_sys_u64(unsigned long long* p, unsigned long long v) { __atomic_store_n(p, v, __ATOMIC_RELAXED); }
inline unsigned int ld_acquire_sys_u32(const unsigned int* p) { return __atomic_load_n(p, __ATOMIC_ACQUIRE); }
inline void fence_acq_rel_gpu() { std::atomic_thread_fence(std::memory_order_acq_rel); }
// ThreadSanitizer does not model fences: the host check polls with acquire
// loads, which give the same ordering as relaxed loads plus the fence.
inline unsigned long long ld_signal_u64(const unsigned long long* p) { return __atomic_load_n(p, __ATOMIC_ACQUIRE); }
unsigned long long globaltimer();
#endif

// Control words of this launch (grid barrier; with one GPU, all of them).
__device__ __forceinline__ int* ctrl(int w) { return c_rt.ctrl + w; }

// ---- several GPUs ----------------------------------------------------------
// Several GPUs need the multi-GPU build of the library (-DCHARMING_MULTI_GPU:
// libcharming_b200_multi.so, libcharming_multi.a). In the default build
// multi_dev() is a compile-time false and the message path carries no test
// of the GPU count: the test cost a one-way pingpong message on one GPU
// about 6 % (4.55 against 4.30 us).
#ifdef CHARMING_MULTI_GPU
__device__ __forceinline__ bool multi_dev() { return c_rt.n_devs > 1; }
#else
__device__ __forceinline__ constexpr bool multi_dev() { return false; }
#endif
__device__ __forceinline__ int dev_of(int pe) { return multi_dev() ? pe / c_rt.pes_per_dev : 0; }
__device__ __forceinline__ int local_of(int pe) { return multi_dev() ? pe % c_rt.pes_per_dev : pe; }
// The GPU the calling block belongs to.
__device__ __forceinline__ int my_dev() {
  return multi_dev() ? (c_rt.pe0 + (int)blockIdx.x) / c_rt.pes_per_dev : 0;
}
__device__ __forceinline__ int* dev_ctrl(int d, int w) { return c_rt.dev[d].ctrl + w; }
// Inbox words other GPUs read or write: system scope when the run has more
// than one GPU.
__device__ __forceinline__ unsigned long long ld_acquire_x(const unsigned long long* p) {
  return multi_dev() ? ld_acquire_sys_u64(p) : ld_acquire_u64(p);
}
__device__ __forceinline__ void st_release_x(unsigned long long* p, unsigned long long v) {
  if (multi_dev()) st_release_sys_u64(p, v);
  else st_release_u64(p, v);
}
__device__ __forceinline__ unsigned long long atomic_add_x(unsigned long long* p, unsigned long long v) {
  return multi_dev() ? atomicAdd_system(p, v) : atomicAdd(p, v);
}

// Error path: first error wins; every PE (of every GPU) stops.
__device__ void set_error(int code, int info0, int info1);
// Every PE of every GPU leaves its loop (end(), a terminate message, the
// host's stop word).
__device__ void raise_term();
__device__ bool terminated_multi();  // out of line, like the other several-GPU lookups
__device__ __forceinline__ bool terminated() {
  if (multi_dev()) return terminated_multi();
  return ld_relaxed_s32(ctrl(CTRL_TERM)) != 0;
}

// Deadline check for bounded waits (thread-local view).
__device__ __forceinline__ bool past_deadline() {
  return globaltimer() - pes()->t0 > c_rt.deadline_ns;
}

__device__ void grid_barrier();
// The same; false (on every thread of the block) when it was left early
// because the run is ending.
__device__ bool grid_barrier_ok();

__device__ __forceinline__ bool gpu_level() { return c_rt.gpu_level != 0; }
// The calling PE's index in this process's per-PE arrays (stash, outbox,
// user heap, proxy tables, arena, statistics), and their length.
__device__ __forceinline__ int local_slot() { return gpu_level() ? 0 : (int)blockIdx.x; }
__device__ __forceinline__ int local_slots() { return gpu_level() ? 1 : c_rt.n_blocks; }
// Loads of the group_state records written by another SM.
__device__ __forceinline__ void* gl_ld_ptr(void* const* p) {
  return reinterpret_cast<void*>(ld_relaxed_u64(reinterpret_cast<const unsigned long long*>(p)));
}

// Invariant checks of the checked build (-DCHARMING_CHECKS): a failed check
// records CHARMING_ERR_APP (or the given code) with two values, and the
// caller skips the access. In the normal build the checks compile away.
#ifdef CHARMING_CHECKS
__device__ __forceinline__ bool verify(bool ok, int code, int a, int b) {
  if (!ok) set_error(code, a, b);
  return ok;
}
#define CHARM_VERIFY(cond, code, a, b) (::charm::rt::verify((cond), (code), (int)(a), (int)(b)))
#else
#define CHARM_VERIFY(cond, code, a, b) (true)
#endif

// Fine-grained timers of the send path (ticket atomics, ring-space waits,
// the phases of the Jacobi halo sends): only in a build with
// -DCHARMING_PROFILE (make VARIANT=_prof EXTRA_NVFLAGS=-DCHARMING_PROFILE,
// selected with CHARMING_LIB); the statistics read 0 otherwise. Their timer
// reads cost the headline launch about 7 %.
#ifdef CHARMING_PROFILE
#define CHARM_PROF(...) __VA_ARGS__
#else
#define CHARM_PROF(...)
#endif

// Message bytes -> ring cells.
__host__ __device__ __forceinline__ unsigned int cells_for(unsigned long long bytes) {
  return (unsigned int)((bytes + CELL - 1) / CELL);
}

} // namespace rt
} // namespace charm
