// Device runtime: the persistent scheduler kernel, the intra-GPU inbox rings,
// the refnum stash, barriers and termination.
//
// Reference counterparts:
//   scheduler kernel / loop      src/sched/scheduler.cu:183-234, :165-171
//   message dispatch             src/sched/scheduler.cu:23-76
//   send                         src/comm/get/get.cu:728-781, :864-914
//   receive + stash              src/comm/get/get.cu:374-465
//   revive                       src/comm/get/get.cu:1316-1345
//   termination                  src/charming.cu:265-267, get.cu:916-988
//   barriers                     src/sched/scheduler.cu:336-350
// What is different, and why:
//   * Each PE owns one multi-producer inbox ring. A sender takes a ticket with
//     one atomicAdd on the ring's tail, writes header and payload straight
//     into the ring, and publishes the ticket with a release store into the
//     cell's sequence word. The receiver consumes tickets in order with
//     acquire loads, so messages from one sender to one receiver are
//     delivered in send order. (The reference picks the lowest free slot of
//     4 per pair and the receiver the lowest occupied index, which reorders.)
//   * The receiver never scans: it polls one sequence word at its head.
//   * A refnum mismatch copies the message to a per-PE stash and frees the
//     ring cells at once, so a parked message never blocks the ring.
//   * Every wait is bounded by the run deadline (%globaltimer); a run that
//     cannot progress ends with an error status instead of spinning forever.
//   * A send that finds no space in its destination's ring does not block its
//     PE for long: after a short wait the whole message goes to the PE's
//     outbox with the ticket it already holds, the send returns, and the
//     scheduler loop copies it into the ring once the receiver has consumed
//     up to that ticket. Two PEs that fill each other's rings from inside
//     entry methods therefore both finish those entry methods and free
//     their rings (the reference spins in the sender, get.cu:241-248).
#include "rt.cuh"

// Execution-environment constants (see include/common.h).
__constant__ int c_n_sms;
__constant__ int c_my_dev;
__constant__ int c_my_dev_node;
__constant__ int c_n_devs;
__constant__ int c_n_devs_node;
__constant__ int c_n_nodes;
__constant__ int c_n_pes;
__constant__ int c_n_pes_node;

namespace charm {
namespace rt {
__constant__ device_state c_rt;
}
}

using namespace charm;
using namespace charm::rt;

// ---------------------------------------------------------------------------
// Errors and termination
// ---------------------------------------------------------------------------
__device__ void charm::rt::set_error(int code, int info0, int info1) {
  const int pe = c_rt.pe0 + (int)blockIdx.x;
  if (!multi_dev()) {
    int prev = atomicCAS(ctrl(CTRL_STATUS), 0, code);
    if (prev == 0) {
      atomicExch(ctrl(CTRL_ERR_PE), pe);
      atomicExch(ctrl(CTRL_ERR_I0), info0);
      atomicExch(ctrl(CTRL_ERR_I1), info1);
    }
    __threadfence();
    atomicExch(ctrl(CTRL_TERM), 1);
    return;
  }
  // Several GPUs: each records the first error it hears of, then all stop.
  for (int d = 0; d < c_rt.n_devs; d++) {
    if (atomicCAS_system(dev_ctrl(d, CTRL_STATUS), 0, code) == 0) {
      atomicExch_system(dev_ctrl(d, CTRL_ERR_PE), pe);
      atomicExch_system(dev_ctrl(d, CTRL_ERR_I0), info0);
      atomicExch_system(dev_ctrl(d, CTRL_ERR_I1), info1);
    }
  }
  __threadfence_system();
  for (int d = 0; d < c_rt.n_devs; d++) atomicExch_system(dev_ctrl(d, CTRL_TERM), 1);
}

__device__ __noinline__ bool charm::rt::terminated_multi() {
  return ld_sys_s32(dev_ctrl(my_dev(), CTRL_TERM)) != 0;
}

__device__ void charm::rt::raise_term() {
  if (!multi_dev()) {
    atomicExch(ctrl(CTRL_TERM), 1);
    return;
  }
  for (int d = 0; d < c_rt.n_devs; d++) atomicExch_system(dev_ctrl(d, CTRL_TERM), 1);
}

__device__ void charm::detail::report_error(int code, int info0, int info1) {
  set_error(code, info0, info1);
}

namespace {
__device__ __forceinline__ unsigned char* smem_arena() {
  return reinterpret_cast<unsigned char*>(s_mem) + c_rt.smem_state_bytes;
}
}  // namespace

__device__ void* charm::detail::pe_alloc(size_t bytes) {
  pe_state* ps = pes();
  // GPU-level mode: every block of the PE reads the objects, so none lives
  // in one block's shared memory
  if (bytes <= (size_t)SMEM_OBJ_MAX && c_rt.smem_arena_bytes > 0 && !gpu_level()) {
    unsigned long long at = (ps->sarena_top + 15) & ~15ULL;
    if (at + bytes <= (unsigned long long)c_rt.smem_arena_bytes) {
      ps->sarena_top = at + bytes;
      return smem_arena() + at;
    }
  }
  if (!c_rt.arena) return nullptr;
  unsigned long long at = (ps->arena_top + 15) & ~15ULL;
  if (at + bytes > c_rt.arena_bytes) return nullptr;
  ps->arena_top = at + bytes;
  return c_rt.arena + (unsigned long long)local_slot() * c_rt.arena_bytes + at;
}

__device__ bool charm::detail::pe_owns(const void* p) {
  const unsigned char* b = static_cast<const unsigned char*>(p);
  if (b >= smem_arena() && b < smem_arena() + c_rt.smem_arena_bytes) return true;
  return c_rt.arena && b >= c_rt.arena && b < c_rt.arena + (unsigned long long)local_slots() * c_rt.arena_bytes;
}

__device__ void charm::detail::cache_proxy(int id, chare_proxy_base* p) {
  if (id >= 0 && id < PROXY_CACHE) pes()->pcache[id] = p;
}

__device__ chare_proxy_table& charm::detail::my_proxy_table() {
  return c_rt.proxy_tables[local_slot()];
}

__device__ void charm::end() {
  if (!terminated()) raise_term();
}

__device__ void charm::send_begin_term_msg() { charm::end(); }

__device__ void charm::abort() {
  // Stops the calling PE only (reference: src/charming.cu:270-277).
  if (threadIdx.x == 0) pes()->term = 1;
  __syncthreads();
}

__device__ int charm::my_pe() { return gpu_level() ? 0 : c_rt.pe0 + (int)blockIdx.x; }
__device__ int charm::n_pes() { return c_n_pes; }
__device__ int charm::my_pe_node() { return charm::my_pe(); }
__device__ int charm::n_pes_node() { return c_n_pes_node; }
__device__ int charm::n_nodes() { return c_n_nodes; }

__device__ int charm::device_atoi(const char* str, int strlen) {
  int v = 0;
  for (int i = 0; i < strlen; i++) v = v * 10 + (str[i] - '0');
  return v;
}

__device__ void* charm::smem_scratch(size_t* bytes) {
  size_t off = (size_t)c_rt.smem_state_bytes + (size_t)c_rt.smem_arena_bytes;
  if (bytes) *bytes = (size_t)c_rt.smem_total - off;
  return reinterpret_cast<char*>(s_mem) + off;
}

__device__ uint64_t charm::now_ns() { return globaltimer(); }

__device__ int charm::pe_thread() {
  return gpu_level() ? (int)(blockIdx.x * blockDim.x + threadIdx.x) : (int)threadIdx.x;
}
__device__ int charm::pe_threads() { return gpu_level() ? (int)(gridDim.x * blockDim.x) : (int)blockDim.x; }
__device__ void charm::pe_sync() {
  if (gpu_level()) grid_barrier();
  else __syncthreads();
}
__device__ bool charm::is_gpu_level() { return gpu_level(); }

__device__ unsigned int charm::smid() {
#ifndef CHARMING_HOST_EMULATION
  unsigned int r;
  asm volatile("mov.u32 %0, %%smid;" : "=r"(r));
  return r;
#else
  return blockIdx.x;
#endif
}

// ---------------------------------------------------------------------------
// Grid barrier (sense by generation counter), bounded by the deadline.
// All PE blocks are co-resident: the host launches cooperatively.
// ---------------------------------------------------------------------------
__device__ bool charm::rt::grid_barrier_ok() {
  pe_state* ps = pes();
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned int* count = reinterpret_cast<unsigned int*>(ctrl(CTRL_BAR_COUNT));
    unsigned int* gen = reinterpret_cast<unsigned int*>(ctrl(CTRL_BAR_GEN));
    unsigned int g = ld_acquire_u32(gen);
    __threadfence();
    unsigned int arrived = atomicAdd(count, 1u);
    int ok = 1;
    if (arrived == (unsigned int)c_rt.n_blocks - 1) {
      atomicExch(count, 0u);
      __threadfence();
      st_release_u32(gen, g + 1);
    } else {
      // Leaves early when the run is ending (an error or end() elsewhere).
      unsigned int spins = 0;
      while (ld_acquire_u32(gen) == g) {
        if ((++spins & 1023) == 0) {
          if (terminated()) {
            ok = 0;
            break;
          }
          if (past_deadline()) {
            set_error(CHARMING_ERR_BARRIER_TIMEOUT, (int)arrived, 0);
            ok = 0;
            break;
          }
        }
      }
    }
    ps->bar_ok = ok;
  }
  __syncthreads();
  return ps->bar_ok != 0;
}

__device__ void charm::rt::grid_barrier() { (void)grid_barrier_ok(); }

// Thread 0 of block 0 of each process: all processes of the run. Arrivals
// take tickets on one counter in GPU 0's control words (never reset within
// a run); the k-th barrier is complete when it reaches (k + 1) * n_procs.
__device__ bool xproc_barrier_ok() {
  unsigned int* cnt = reinterpret_cast<unsigned int*>(dev_ctrl(0, CTRL_XBAR));
  const unsigned int n = (unsigned int)c_rt.n_procs;
  const unsigned int goal = (atomicAdd_system(cnt, 1u) / n + 1) * n;
  unsigned int spins = 0;
  while ((int)(ld_acquire_sys_u32(cnt) - goal) < 0) {
    if ((++spins & 255) == 0) {
      if (terminated()) return false;
      if (past_deadline()) {
        set_error(CHARMING_ERR_BARRIER_TIMEOUT, -1, (int)goal);
        return false;
      }
    }
    __nanosleep(200);
  }
  return true;
}

// All PEs of the run (reference: nvshmem_barrier_all and a grid sync,
// src/sched/scheduler.cu:336-344); barrier_local(): this GPU's launch.
__device__ void charm::barrier() {
  grid_barrier();
  if (c_rt.n_procs > 1) {
    if (blockIdx.x == 0 && threadIdx.x == 0) (void)xproc_barrier_ok();
    grid_barrier();
  }
}
__device__ void charm::barrier_local() { grid_barrier(); }

// ---------------------------------------------------------------------------
// Transport
// ---------------------------------------------------------------------------
namespace {

// PE pe's inbox words and cells (global PE number; with several GPUs, in
// the memory of the GPU it lives on). The several-GPU lookups (a division
// and an indexed table) are out of line, so that the compiler cannot
// evaluate them ahead of the branch on the single-GPU path.
enum : int { W_TAIL = 0, W_HEAD, W_PROGRESS, W_RING, W_FLAGS };
__device__ __noinline__ void* inbox_of_dev(int pe, int what, unsigned long long ticket) {
  const dev_inbox& d = c_rt.dev[pe / c_rt.pes_per_dev];
  const unsigned long long l = (unsigned long long)(pe % c_rt.pes_per_dev);
  const unsigned long long cell = ticket & (c_rt.ring_cells - 1);
  switch (what) {
    case W_TAIL: return &d.tail[l].v;
    case W_HEAD: return &d.head[l].v;
    case W_PROGRESS: return &d.progress[l];
    case W_RING: return d.ring + l * c_rt.ring_stride + cell * CELL;
    default: return d.flags + l * c_rt.ring_cells + cell;
  }
}
__device__ __forceinline__ unsigned char* ring_cell(int pe, unsigned long long ticket) {
  if (multi_dev()) return static_cast<unsigned char*>(inbox_of_dev(pe, W_RING, ticket));
  return c_rt.ring + (unsigned long long)pe * c_rt.ring_stride + (ticket & (c_rt.ring_cells - 1)) * CELL;
}
__device__ __forceinline__ unsigned long long* ring_flag(int pe, unsigned long long ticket) {
  if (multi_dev()) return static_cast<unsigned long long*>(inbox_of_dev(pe, W_FLAGS, ticket));
  return c_rt.flags + (unsigned long long)pe * c_rt.ring_cells + (ticket & (c_rt.ring_cells - 1));
}
__device__ __forceinline__ unsigned long long* tail_of(int pe) {
  if (multi_dev()) return static_cast<unsigned long long*>(inbox_of_dev(pe, W_TAIL, 0));
  return &c_rt.tail[pe].v;
}
__device__ __forceinline__ unsigned long long* head_of(int pe) {
  if (multi_dev()) return static_cast<unsigned long long*>(inbox_of_dev(pe, W_HEAD, 0));
  return &c_rt.head[pe].v;
}
__device__ __forceinline__ unsigned long long* progress_of(int pe) {
  if (multi_dev()) return static_cast<unsigned long long*>(inbox_of_dev(pe, W_PROGRESS, 0));
  return &c_rt.progress[pe];
}

__device__ __forceinline__ unsigned char* outbox_of(int pe) {
  return c_rt.outbox + (unsigned long long)pe * c_rt.outbox_stride;
}
__device__ __forceinline__ bool in_outbox(const unsigned char* m) {
  const unsigned char* b = c_rt.outbox ? outbox_of(blockIdx.x) : nullptr;
  return b && m >= b && m < b + c_rt.outbox_stride;
}

// A new outbox entry for a message of `bytes` that holds `ticket` in dst's
// inbox; returns where the message goes, or nullptr when the outbox is
// full. Any thread (the threads of a batched send may call it at once; a
// block-shared lock orders them). Entries are never allocated while the
// scheduler loop flushes, so only reserving threads race here.
__device__ unsigned char* outbox_put(int dst, unsigned long long ticket, unsigned long long bytes) {
  if (!c_rt.outbox) return nullptr;
  pe_state* ps = pes();
  const unsigned long long span = (OB_HDR + bytes + 15) & ~15ULL;
  while (atomicCAS_block(&ps->ob_lock, 0, 1) != 0) {
  }
  const unsigned long long v = ps->ob_tail;
  const bool ok = v + span - ps->ob_head <= c_rt.outbox_bytes;
  if (ok) ps->ob_tail = v + span;
  __threadfence_block();
  atomicExch_block(&ps->ob_lock, 0);
  if (!ok) return nullptr;
  ob_entry* e = reinterpret_cast<ob_entry*>(outbox_of(blockIdx.x) + v % c_rt.outbox_bytes);
  e->dst = dst;
  e->state = OB_FILLING;
  e->ticket = ticket;
  e->bytes = bytes;
  e->span = span;
  atomicAdd_block(&ps->ob_count, 1);
  atomicAdd_block(&ps->stats[ST_DEFERRED], 1ULL);
  return reinterpret_cast<unsigned char*>(e) + OB_HDR;
}

// Whether a message of `bytes` can go to PE dst (error recorded if not).
__device__ bool send_allowed(int dst, unsigned long long bytes) {
  if (dst < 0 || dst >= c_rt.n_pes) {
    set_error(CHARMING_ERR_BAD_TARGET, -1, dst);
    return false;
  }
  if (bytes > c_rt.max_msg) {
    set_error(CHARMING_ERR_MSG_TOO_LARGE, dst, (int)(bytes > 0x7fffffffULL ? 0x7fffffff : bytes));
    return false;
  }
  if (cells_for(bytes) > c_rt.ring_cells) {  // could never fit
    set_error(CHARMING_ERR_MSG_TOO_LARGE, dst, (int)cells_for(bytes));
    return false;
  }
  return true;
}

__device__ unsigned char* wait_space(int dst, unsigned long long t, unsigned long long bytes,
    unsigned long long* ticket);

// Thread 0 only. Reserves `bytes` in dst's inbox; returns the message start
// (in the ring, or in this PE's outbox when the ring stayed full for
// DEFER_AFTER_NS) or nullptr (error recorded, or the run is ending).
__device__ unsigned char* reserve(int dst, unsigned long long bytes, unsigned long long* ticket) {
  if (!send_allowed(dst, bytes)) return nullptr;
  CHARM_PROF(pe_state* ps = pes(); const unsigned long long t0 = globaltimer();)
  const unsigned long long t = atomic_add_x(tail_of(dst), (unsigned long long)cells_for(bytes));
  CHARM_PROF(const unsigned long long t1 = globaltimer();)
  unsigned char* m = wait_space(dst, t, bytes, ticket);
  CHARM_PROF(atomicAdd_block(&ps->stats[ST_TICKET_NS], t1 - t0);
             atomicAdd_block(&ps->stats[ST_SPACE_NS], globaltimer() - t1);)
  return m;
}

// The caller holds ticket t (cells_for(bytes) cells) in dst's inbox: waits
// until the receiver has consumed enough for it, or moves the message to
// the outbox; returns where the message goes (nullptr: error or the end of
// the run). Any thread.
__device__ unsigned char* wait_space(int dst, unsigned long long t, unsigned long long bytes,
    unsigned long long* ticket) {
  pe_state* ps = pes();
  const unsigned long long C = c_rt.ring_cells;
  const unsigned int cells = cells_for(bytes);
  unsigned long long* hc = head_cache();
  // relaxed read: other threads of the block may raise hc[dst] meanwhile
  if (t + cells - ld_volatile_shared_u64(&hc[dst]) > C) {
    atomicAdd_block(&ps->stats[ST_SPACE_WAITS], 1ULL);
    // This PE publishes its head lazily. Whoever waits for space in this
    // PE's ring meanwhile (itself included) must see all it has consumed:
    // ps->head is stable during an entry method, and the message being
    // processed is not yet counted as consumed, so publishing it is safe
    // (and harmless when repeated).
    st_release_x(head_of(ps->my_pe), ps->head);
    unsigned long long start = globaltimer();
    // A receiver that frees nothing for the idle timeout is taken as stuck.
    unsigned long long limit = c_rt.idle_timeout_ns ? c_rt.idle_timeout_ns : c_rt.deadline_ns;
    unsigned int spins = 0;
    while (true) {
      unsigned long long h = ld_acquire_x(head_of(dst));
      atomicMax(&hc[dst], h);  // monotonic; several threads may reserve at once
      if (t + cells - h <= C) break;
      if ((++spins & 255) == 0) {
        if (terminated()) return nullptr;
        unsigned long long now = globaltimer();
        if (now - start > DEFER_AFTER_NS) {
          unsigned char* ob = outbox_put(dst, t, bytes);
          if (ob) {
            *ticket = t;
            return ob;
          }
        }
        if (now - start > limit || now - ps->t0 > c_rt.deadline_ns) {
          set_error(CHARMING_ERR_RING_FULL, dst, (int)cells);
          return nullptr;
        }
      }
      __nanosleep(100);
    }
  }
  *ticket = t;
  return ring_cell(dst, t);
}

// The release store alone orders the message before its flag: the
// payload written by other threads of the block is ordered before it by
// the barrier the callers pass first (release is cumulative), and a separate
// fence would also invalidate the SM's L1.
//
// Several GPUs: a message to a PE on another GPU is released at system
// scope, one to a PE of the sender's own GPU at GPU scope (the receiver
// acquires at system scope, which pairs with either): a system-scope
// release waits until the sender's writes are visible to every GPU and the
// host, which a message that stays on its GPU does not need.
__device__ __forceinline__ void publish(int dst, unsigned long long ticket) {
  unsigned long long* f = ring_flag(dst, ticket);
  if (multi_dev() && dev_of(dst) != my_dev()) st_release_sys_u64(f, ticket + 1);
  else st_release_u64(f, ticket + 1);
}

// Publishes the message at m (reserved by reserve() for ticket in dst's
// inbox): in the ring, its sequence word; in the outbox, the entry is
// marked complete for the scheduler loop to flush. Callers pass a block
// barrier first.
__device__ __forceinline__ void publish_msg(int dst, unsigned long long ticket, unsigned char* m) {
  if (in_outbox(m)) {
    reinterpret_cast<ob_entry*>(m - OB_HDR)->state = OB_READY;
  } else {
    publish(dst, ticket);
  }
}

// Thread 0: whether the oldest outbox entry is complete and its receiver
// has consumed enough for it to be copied into the ring.
__device__ bool outbox_head_ready() {
  pe_state* ps = pes();
  if (ps->ob_count <= 0) return false;
  const ob_entry* e =
      reinterpret_cast<const ob_entry*>(outbox_of(blockIdx.x) + ps->ob_head % c_rt.outbox_bytes);
  if (e->state != OB_READY) return false;
  const unsigned long long h = ld_acquire_x(head_of(e->dst));
  atomicMax(&head_cache()[e->dst], h);
  return e->ticket + cells_for(e->bytes) - h <= c_rt.ring_cells;
}

// Thread 0: tell the senders how far this PE has consumed its inbox (a
// release store: the reads of the consumed messages are done). Published
// lazily, after an eighth of the ring or before waiting for messages.
__device__ __forceinline__ void publish_head(pe_state* ps, int me) {
  if (ps->head != ps->head_pub) {
    st_release_x(head_of(me), ps->head);
    ps->head_pub = ps->head;
  }
}

// Thread 0: the progress stamp the idle-timeout check reads.
__device__ __forceinline__ void stamp_progress(int me) {
  if (multi_dev()) st_relaxed_sys_u64(progress_of(me), pes()->stats[ST_DELIVERED]);
  else st_relaxed_u64(progress_of(me), pes()->stats[ST_DELIVERED]);
}

} // namespace

// ---------------------------------------------------------------------------
// GPU-level mode: collective sends over all blocks of PE 0 (the reference's
// GPU-level send_reg_msg / send_remote_msg, src/comm/get/get.cu:1224-1273:
// GID 0 takes the space, barrier_local(), the grid copies the payload,
// barrier_local(), GID 0 publishes). Every block calls them in the same
// order with the same arguments.
// ---------------------------------------------------------------------------
namespace {

__device__ __forceinline__ bool gl_lead() { return blockIdx.x == 0 && threadIdx.x == 0; }

// This call's broadcast slot; the block's call count moves on before the
// call's first grid barrier (which begins with a block barrier).
__device__ __forceinline__ group_slot* gl_next_slot() {
  pe_state* ps = pes();
  const unsigned s = ps->gl_seq;
  __syncthreads();
  if (threadIdx.x == 0) ps->gl_seq = s + 1;
  return &c_rt.gl->slot[s & 1];
}

__device__ void group_send_reg_msg(int chare_id, int chare_idx, int ep_id, void* buf, size_t payload_size,
    int dst_pe, int refnum) {
  pe_state* ps = pes();
  group_slot* g = gl_next_slot();
  if (gl_lead()) {
    // taking the space does not read the payload: it overlaps the other
    // blocks' last writes to it
    unsigned long long bytes = envelope::alloc_size(msgtype::regular, payload_size);
    unsigned long long t = 0;
    unsigned char* m = reserve(dst_pe, bytes, &t);
    if (m) {
      envelope* env = reinterpret_cast<envelope*>(m);
      env->type = msgtype::regular;
      env->src_pe = 0;
      env->size = bytes;
      regular_msg* rm = reinterpret_cast<regular_msg*>(m + sizeof(envelope));
      rm->chare_id = chare_id;
      rm->chare_idx = chare_idx;
      rm->ep_id = ep_id;
      rm->refnum = refnum;
      ps->stats[ST_SENT]++;
      ps->stats[ST_BYTES_SENT] += payload_size;
    }
    g->ptr[0] = m;
    g->u0[0] = (m && buf) ? payload_size : 0;
    g->u1[0] = t;
    g->i0 = (buf != nullptr && __isLocal(buf)) ? 1 : 0;
    g->i1 = dst_pe;
  }
  grid_barrier();  // every block's payload writes are done; the space is known
  unsigned char* m = reinterpret_cast<unsigned char*>(gl_ld_ptr(&g->ptr[0]));
  if (m == nullptr) return;
  const size_t n = ld_relaxed_u64(&g->u0[0]);
  const unsigned long long t = ld_relaxed_u64(&g->u1[0]);
  const int dst = ld_relaxed_s32(&g->i1);
  if (n > 0) {
    if (ld_relaxed_s32(&g->i0)) {
      // a thread-local buffer is only addressable by the thread that owns it
      if (gl_lead()) copy_cooperative(m + HDR, buf, n, 0, 1);
    } else {
      copy_cooperative(m + HDR, buf, n, (size_t)charm::pe_thread(), (size_t)charm::pe_threads());
    }
  }
  grid_barrier();  // the payload is complete
  if (gl_lead()) publish_msg(dst, t, m);
}

__device__ bool group_alloc_user_msgs(message* msgs, const int* dst_pes, const size_t* payload_sizes, int n) {
  group_slot* g = gl_next_slot();
  if (gl_lead()) {
    for (int k = 0; k < n; k++) {
      const unsigned long long bytes = envelope::alloc_size(msgtype::user, payload_sizes[k]);
      unsigned long long t = 0;
      g->ptr[k] = reserve(dst_pes[k], bytes, &t);
      g->u0[k] = bytes;
      g->u1[k] = t;
    }
  }
  grid_barrier();
  // a block-shared array (block_messages()) is filled by thread 0 of each block
  const bool fill = !__isShared(msgs) || threadIdx.x == 0;
  bool ok = true;
  for (int k = 0; k < n; k++) {
    envelope* env = reinterpret_cast<envelope*>(gl_ld_ptr(&g->ptr[k]));
    if (fill) {
      msgs[k].env = env;
      msgs[k].offset = ld_relaxed_u64(&g->u1[k]);
      msgs[k].dst_pe = dst_pes[k];
      const unsigned long long bytes = ld_relaxed_u64(&g->u0[k]);
      msgs[k].cells = (int)cells_for(bytes);
      msgs[k].capacity = env ? (size_t)(bytes - HDR) : 0;
    }
    ok = ok && env != nullptr;
  }
  if (__isShared(msgs)) __syncthreads();
  return ok;
}

// Block 0 publishes message k with thread k once every block is done
// writing the payloads.
__device__ void group_send_user_msgs(int chare_id, const int* chare_idx, int ep_id, message* msgs,
    const size_t* payload_sizes, const int* refnums, int n) {
  pe_state* ps = pes();
  grid_barrier();
  if (blockIdx.x == 0) {
    for (int k = (int)threadIdx.x; k < n; k += (int)blockDim.x) {
      if (!msgs[k].env) continue;
      unsigned char* m = reinterpret_cast<unsigned char*>(msgs[k].env);
      envelope* env = msgs[k].env;
      env->type = msgtype::user;
      env->src_pe = 0;
      env->size = (size_t)msgs[k].capacity + HDR;
      regular_msg* rm = reinterpret_cast<regular_msg*>(m + sizeof(envelope));
      rm->chare_id = chare_id;
      rm->chare_idx = chare_idx[k];
      rm->ep_id = ep_id;
      rm->refnum = refnums ? refnums[k] : -1;
      if (payload_sizes[k] > msgs[k].capacity)
        set_error(CHARMING_ERR_MSG_TOO_LARGE, msgs[k].dst_pe, (int)payload_sizes[k]);
      atomicAdd_block(&ps->stats[ST_SENT], 1ULL);
      atomicAdd_block(&ps->stats[ST_BYTES_SENT], (unsigned long long)payload_sizes[k]);
      publish_msg(msgs[k].dst_pe, msgs[k].offset, m);
    }
  }
}

}  // namespace

__device__ void charm::send_reg_msg(int chare_id, int chare_idx, int ep_id, void* buf,
    size_t payload_size, int dst_pe, int refnum) {
  if (gpu_level()) {
    group_send_reg_msg(chare_id, chare_idx, ep_id, buf, payload_size, dst_pe, refnum);
    return;
  }
  pe_state* ps = pes();
  if (threadIdx.x == 0) {
    unsigned long long bytes = envelope::alloc_size(msgtype::regular, payload_size);
    unsigned long long t = 0;
    unsigned char* m = reserve(dst_pe, bytes, &t);
    if (m) {
      envelope* env = reinterpret_cast<envelope*>(m);
      env->type = msgtype::regular;
      env->src_pe = c_rt.pe0 + (int)blockIdx.x;
      env->size = bytes;
      regular_msg* rm = reinterpret_cast<regular_msg*>(m + sizeof(envelope));
      rm->chare_id = chare_id;
      rm->chare_idx = chare_idx;
      rm->ep_id = ep_id;
      rm->refnum = refnum;
      ps->stats[ST_SENT]++;
      ps->stats[ST_BYTES_SENT] += payload_size;
    }
    ps->b_ptr0 = m;
    ps->b_ptr1 = buf;
    ps->b_u0 = (m && buf) ? payload_size : 0;
    ps->b_u1 = t;
    ps->b_i0 = (buf != nullptr && __isLocal(buf)) ? 1 : 0;
    ps->b_i1 = dst_pe;
  }
  __syncthreads();
  unsigned char* m = reinterpret_cast<unsigned char*>(ps->b_ptr0);
  if (m == nullptr) {
    __syncthreads();
    return;
  }
  size_t n = ps->b_u0;
  if (n > 0) {
    if (ps->b_i0) {
      // A thread-local buffer is only addressable by the thread that owns it.
      if (threadIdx.x == 0) copy_cooperative(m + HDR, ps->b_ptr1, n, 0, 1);
    } else {
      copy_cooperative(m + HDR, ps->b_ptr1, n, threadIdx.x, blockDim.x);
    }
  }
  unsigned long long t = ps->b_u1;
  int dst = ps->b_i1;
  __syncthreads();
  if (threadIdx.x == 0) publish_msg(dst, t, m);
}

__device__ bool charm::alloc_user_msg(message& msg, int dst_pe, size_t payload_size) {
  if (gpu_level()) return group_alloc_user_msgs(&msg, &dst_pe, &payload_size, 1);
  pe_state* ps = pes();
  if (threadIdx.x == 0) {
    unsigned long long bytes = envelope::alloc_size(msgtype::user, payload_size);
    unsigned long long t = 0;
    unsigned char* m = reserve(dst_pe, bytes, &t);
    ps->b_ptr0 = m;
    ps->b_u0 = bytes;
    ps->b_u1 = t;
  }
  __syncthreads();
  msg.env = reinterpret_cast<envelope*>(ps->b_ptr0);
  msg.offset = ps->b_u1;
  msg.dst_pe = dst_pe;
  msg.cells = (int)cells_for(ps->b_u0);
  msg.capacity = msg.env ? (size_t)(ps->b_u0 - HDR) : 0;
  __syncthreads();
  return msg.env != nullptr;
}

__device__ void charm::send_user_msg(int chare_id, int chare_idx, int ep_id,
    message& msg, size_t payload_size, int refnum) {
  if (msg.env == nullptr) return;
  if (gpu_level()) {
    group_send_user_msgs(chare_id, &chare_idx, ep_id, &msg, &payload_size, &refnum, 1);
    msg.env = nullptr;
    return;
  }
  pe_state* ps = pes();
  __syncthreads();  // payload writes of all threads are done
  if (threadIdx.x == 0) {
    unsigned char* m = reinterpret_cast<unsigned char*>(msg.env);
    envelope* env = msg.env;
    env->type = msgtype::user;
    env->src_pe = c_rt.pe0 + (int)blockIdx.x;
    // The ring advances by the reserved size, whatever part was filled.
    env->size = (size_t)msg.capacity + HDR;
    regular_msg* rm = reinterpret_cast<regular_msg*>(m + sizeof(envelope));
    rm->chare_id = chare_id;
    rm->chare_idx = chare_idx;
    rm->ep_id = ep_id;
    rm->refnum = refnum;
    if (payload_size > msg.capacity) set_error(CHARMING_ERR_MSG_TOO_LARGE, msg.dst_pe, (int)payload_size);
    ps->stats[ST_SENT]++;
    ps->stats[ST_BYTES_SENT] += payload_size;
    publish_msg(msg.dst_pe, msg.offset, m);
  }
  __syncthreads();
  msg.env = nullptr;
}

__device__ bool charm::alloc_user_msgs(message* msgs, const int* dst_pes,
    const size_t* payload_sizes, int n) {
  if (n > MSG_BATCH_MAX) n = MSG_BATCH_MAX;
  if (gpu_level()) return group_alloc_user_msgs(msgs, dst_pes, payload_sizes, n);
  pe_state* ps = pes();
  if (blockDim.x >= 32) {
    // Warp 0, one lane per message. Lanes whose messages go to the same PE
    // form a group (__match_any_sync): its lowest lane takes the tickets of
    // the whole group with one atomicAdd, and each lane's messages get them
    // in batch order, so one PE's messages to another keep their order.
    // Different PEs' reservations overlap.
    if (threadIdx.x < 32) {
      constexpr unsigned FULL = 0xffffffffu;
      const int k = (int)threadIdx.x;
      const bool act = k < n;
      const unsigned long long bytes = act ? envelope::alloc_size(msgtype::user, payload_sizes[k]) : 0;
      const bool ok = act && send_allowed(dst_pes[k], bytes);
      const unsigned cells = ok ? cells_for(bytes) : 0;
      const unsigned grp = __match_any_sync(FULL, ok ? dst_pes[k] : -1 - k);
      const int leader = __ffs(grp) - 1;
      unsigned pre = 0, tot = 0;
#pragma unroll
      for (int j = 0; j < MSG_BATCH_MAX; j++) {
        const unsigned cj = __shfl_sync(FULL, cells, j);
        if ((grp >> j) & 1u) {
          if (j < k) pre += cj;
          tot += cj;
        }
      }
      unsigned long long base = 0;
      CHARM_PROF(const unsigned long long ta = k == 0 ? globaltimer() : 0;)
      if (ok && k == leader) base = atomic_add_x(tail_of(dst_pes[k]), (unsigned long long)tot);
      base = __shfl_sync(FULL, base, leader);
      CHARM_PROF(__syncwarp(); const unsigned long long tb = k == 0 ? globaltimer() : 0;)
      // A group's lanes wait for ring space in ticket order, one round per
      // message of the group: a message that finds the ring full moves to
      // the outbox, which flushes strictly in entry order, so a group's
      // later ticket must never enter it before an earlier one. Lanes of
      // different groups wait together.
      const int rank = __popc(grp & ((1u << k) - 1));
      int rounds = __popc(grp);
      for (int o = 16; o > 0; o >>= 1) rounds = max(rounds, __shfl_xor_sync(FULL, rounds, o));
      for (int r = 0; r < rounds; r++) {
        if (act && rank == r) {
          unsigned long long t = 0;
          ps->bm_ptr[k] = ok ? wait_space(dst_pes[k], base + pre, bytes, &t) : nullptr;
          ps->bm_tick[k] = t;
          ps->bm_bytes[k] = bytes;
        }
        __syncwarp();
      }
      CHARM_PROF(__syncwarp(); if (k == 0) {
        ps->stats[ST_TICKET_NS] += tb - ta;
        ps->stats[ST_SPACE_NS] += globaltimer() - tb;
      })
    }
  } else {
    // blocks under a warp (host checks): thread by thread, in batch order
    for (int k = (int)threadIdx.x; k < n; k += (int)blockDim.x) {
      unsigned long long bytes = envelope::alloc_size(msgtype::user, payload_sizes[k]);
      unsigned long long t = 0;
      ps->bm_ptr[k] = reserve(dst_pes[k], bytes, &t);
      ps->bm_tick[k] = t;
      ps->bm_bytes[k] = bytes;
    }
  }
  __syncthreads();
  // every thread's own array, or a block-shared one (block_messages()) that
  // thread 0 fills: 512 private copies of the descriptors cost each batch
  // about 300 KB of local-memory stores
  const bool fill = !__isShared(msgs) || threadIdx.x == 0;
  bool ok = true;
  for (int j = 0; j < n; j++) {
    if (fill) {
      msgs[j].env = reinterpret_cast<envelope*>(ps->bm_ptr[j]);
      msgs[j].offset = ps->bm_tick[j];
      msgs[j].dst_pe = dst_pes[j];
      msgs[j].cells = (int)cells_for(ps->bm_bytes[j]);
      msgs[j].capacity = ps->bm_ptr[j] ? (size_t)(ps->bm_bytes[j] - HDR) : 0;
    }
    ok = ok && ps->bm_ptr[j] != nullptr;
  }
  __syncthreads();
  return ok;
}

__device__ charm::message* charm::block_messages() {
  return reinterpret_cast<message*>(pes()->bmsg);
}

__device__ void charm::send_user_msgs(int chare_id, const int* chare_idx, int ep_id,
    message* msgs, const size_t* payload_sizes, const int* refnums, int n) {
  if (n > MSG_BATCH_MAX) n = MSG_BATCH_MAX;
  if (gpu_level()) {
    group_send_user_msgs(chare_id, chare_idx, ep_id, msgs, payload_sizes, refnums, n);
    if (__isShared(msgs)) __syncthreads();  // block 0's publishers are done reading it
    if (!__isShared(msgs) || threadIdx.x == 0)
      for (int j = 0; j < n; j++) msgs[j].env = nullptr;
    return;
  }
  pe_state* ps = pes();
  __syncthreads();  // payload writes of all threads are done
  // one message per thread: the publishing fences overlap
  for (int k = (int)threadIdx.x; k < n; k += (int)blockDim.x) {
    if (!msgs[k].env) continue;
    unsigned char* m = reinterpret_cast<unsigned char*>(msgs[k].env);
    envelope* env = msgs[k].env;
    env->type = msgtype::user;
    env->src_pe = c_rt.pe0 + (int)blockIdx.x;
    env->size = (size_t)msgs[k].capacity + HDR;
    regular_msg* rm = reinterpret_cast<regular_msg*>(m + sizeof(envelope));
    rm->chare_id = chare_id;
    rm->chare_idx = chare_idx[k];
    rm->ep_id = ep_id;
    rm->refnum = refnums ? refnums[k] : -1;
    if (payload_sizes[k] > msgs[k].capacity) set_error(CHARMING_ERR_MSG_TOO_LARGE, msgs[k].dst_pe, (int)payload_sizes[k]);
    atomicAdd_block(&ps->stats[ST_SENT], 1ULL);
    atomicAdd_block(&ps->stats[ST_BYTES_SENT], (unsigned long long)payload_sizes[k]);
    publish_msg(msgs[k].dst_pe, msgs[k].offset, m);
  }
  __syncthreads();
  if (!__isShared(msgs) || threadIdx.x == 0)
    for (int j = 0; j < n; j++) msgs[j].env = nullptr;
}

// ---------------------------------------------------------------------------
// malloc_user / free_user (reference: src/comm/get/get.cu:1348-1362, where
// they take space from the PE's message buffer and free_user returns it
// through the release heap, so space comes back in offset order). Here each
// PE has its own heap region in HBM, handed out as a ring: blocks are taken
// at the tail (a block that would cross the end starts at the beginning),
// and the head moves past the oldest blocks once they are freed, in any
// order. Single-threaded. Blocks live until free_user or the end of the run.
// ---------------------------------------------------------------------------
namespace {
__device__ __forceinline__ user_block* user_blocks_of(int pe) {
  return c_rt.user_blocks + (unsigned long long)pe * c_rt.user_blocks_max;
}
}  // namespace

__device__ void* charm::malloc_user(size_t size, size_t& offset) {
  pe_state* ps = pes();
  const unsigned long long U = c_rt.user_heap_bytes;
  const unsigned long long B = (unsigned long long)c_rt.user_blocks_max;
  const unsigned long long n = (size + 15) & ~15ULL;
  if (!c_rt.user_heap || n == 0 || n > U || ps->ub_tail - ps->ub_head >= B) return nullptr;
  unsigned long long v = ps->uh_tail;
  const unsigned long long p = v % U;
  if (p + n > U) v += U - p;  // does not fit before the end: start over
  if (v + n - ps->uh_head > U) return nullptr;
  user_block* b = user_blocks_of(blockIdx.x) + ps->ub_tail % B;
  b->off = ps->uh_tail;        // the block's share starts where the last one ended
  b->span = v + n - ps->uh_tail;
  b->start = v % U;
  b->freed = 0;
  ps->ub_tail++;
  ps->uh_tail = v + n;
  offset = (size_t)(v % U);
  return c_rt.user_heap + (unsigned long long)blockIdx.x * U + v % U;
}

__device__ void charm::free_user(size_t size, size_t offset) {
  (void)size;  // the block is found by its offset
  pe_state* ps = pes();
  const unsigned long long B = (unsigned long long)c_rt.user_blocks_max;
  user_block* blocks = user_blocks_of(blockIdx.x);
  bool found = false;
  for (unsigned long long i = ps->ub_head; i < ps->ub_tail; i++) {
    user_block* b = blocks + i % B;
    if (!b->freed && b->start == (unsigned long long)offset) {
      b->freed = 1;
      found = true;
      break;
    }
  }
  if (!found) {
    set_error(CHARMING_ERR_BAD_TARGET, -2, (int)offset);
    return;
  }
  while (ps->ub_head < ps->ub_tail && blocks[ps->ub_head % B].freed) ps->ub_head++;
  ps->uh_head = ps->ub_head < ps->ub_tail ? blocks[ps->ub_head % B].off : ps->uh_tail;
}

__device__ void charm::revive_mismatches(int chare_id, int chare_idx, int refnum) {
  // the warps of a batch of warp-level entry methods may set it together
  atomicExch_block(&pes()->revive_pending, 1);
}

__device__ void charm::add_async_wait(int chare_id) { pes()->aw_count++; }

// ---------------------------------------------------------------------------
// Stash (refnum mismatches)
// ---------------------------------------------------------------------------
namespace {

__device__ __forceinline__ stash_key* keys_of(int pe) {
  return c_rt.stash_keys + (unsigned long long)pe * c_rt.stash_entries;
}
__device__ __forceinline__ unsigned char* arena_of(int pe) {
  return c_rt.stash_data + (unsigned long long)pe * c_rt.stash_bytes;
}

// Scheduler actions: thread 0 decides, the block executes (one barrier
// before, one after).
enum : int {
  ACT_NONE = 0,
  ACT_EXIT,         // leave the loop
  ACT_CALL_RING,    // entry method on the message at the inbox head
  ACT_CALL_STASH,   // entry method on a ready stashed message
  ACT_CALL_WAIT,    // entry method of a satisfied async_wait (null argument)
  ACT_STASH_PUT,    // copy the message at the inbox head into the stash
  ACT_FLUSH,        // copy the oldest outbox entry into its destination ring
  ACT_REVIVE,       // mark waiting stashed messages whose refnum now matches
  ACT_CALL_BATCH,   // warp-level entry methods on consecutive inbox messages, one per warp
  ACT_STASH_BATCH,  // warp-level entry methods on ready stashed messages, one per warp
};

// Batches of warp-level deliveries need whole warps and at least two of them.
__device__ __forceinline__ bool batching() { return !gpu_level() && blockDim.x >= 64 && (blockDim.x & 31) == 0; }

__device__ __forceinline__ chare_proxy_base* proxy_of(pe_state* ps, int cid) {
  if (cid >= 0 && cid < PROXY_CACHE) return ps->pcache[cid];  // on chip
  chare_proxy_table& tb = c_rt.proxy_tables[blockIdx.x];
  return (cid >= 0 && cid < tb.count) ? tb.proxies[cid] : nullptr;
}

// Thread 0: a stash descriptor and arena space for a message of `bytes`;
// the arena address, or nullptr (error recorded).
__device__ unsigned char* stash_alloc(unsigned long long bytes, int chare_id, int chare_idx, int refnum,
    int src_pe) {
  pe_state* ps = pes();
  const unsigned long long S = (unsigned long long)c_rt.stash_entries;
  const unsigned long long A = c_rt.stash_bytes;
  bool ok = ps->key_tail - ps->key_head < S;
  unsigned long long v = ps->arena_tail;
  const unsigned long long p = v % A;
  if (p + bytes > A) v += A - p;
  if (v + bytes - ps->arena_head > A) ok = false;
  if (!ok) {
    set_error(CHARMING_ERR_STASH_FULL, (int)(ps->key_tail - ps->key_head), (int)bytes);
    return nullptr;
  }
  stash_key* k = keys_of(blockIdx.x) + (ps->key_tail % S);
  k->chare_id = chare_id;
  k->chare_idx = chare_idx;
  k->refnum = refnum;
  k->state = KEY_WAIT;
  k->data_off = v;
  k->bytes = (unsigned int)bytes;
  k->src_pe = src_pe;
  if (ps->key_tail == ps->key_head) ps->arena_head = v;
  ps->arena_tail = v + bytes;
  ps->key_tail++;
  ps->n_waiting++;
  ps->stats[ST_STASHED]++;
  return arena_of(blockIdx.x) + (v % A);
}

// Thread 0: drop consumed descriptors at the head and release arena bytes.
__device__ void stash_retire() {
  pe_state* ps = pes();
  const unsigned long long S = (unsigned long long)c_rt.stash_entries;
  stash_key* keys = keys_of(blockIdx.x);
  while (ps->key_head < ps->key_tail && keys[ps->key_head % S].state == KEY_FREE) ps->key_head++;
  ps->arena_head = (ps->key_head < ps->key_tail) ? keys[ps->key_head % S].data_off : ps->arena_tail;
  if (ps->ready_cursor < ps->key_head) ps->ready_cursor = ps->key_head;
}

// Block-collective: waiting stashed messages whose refnum now matches become
// ready (counted into red_i[0]), and every ready one goes on the on-chip
// ready list (thread 0 sorts it before the next decision).
__device__ void stash_revive_scan() {
  pe_state* ps = pes();
  const unsigned long long S = (unsigned long long)c_rt.stash_entries;
  stash_key* keys = keys_of(blockIdx.x);
  const unsigned long long kh = ps->key_head, kt = ps->key_tail;
  int cnt = 0;
  for (unsigned long long i = kh + threadIdx.x; i < kt; i += blockDim.x) {
    stash_key* k = keys + (i % S);
    int st = k->state;
    if (st == KEY_WAIT) {
      chare_proxy_base* p = proxy_of(ps, k->chare_id);
      if (p->refnum_matches(k->chare_idx, k->refnum)) {
        k->state = st = KEY_READY;
        cnt++;
      }
    }
    if (st == KEY_READY) {
      const int pos = atomicAdd_block(&ps->rq_n, 1);
      if (pos < RQ_MAX) ps->rq[pos] = (unsigned int)(i - kh);
    }
  }
  if (cnt) atomicAdd_block(&ps->red_i[0], cnt);
}

// Thread 0: the ready list of the last revive in key (arrival) order.
__device__ void ready_list_sort() {
  pe_state* ps = pes();
  if (ps->rq_n > RQ_MAX) {
    ps->rq_over = 1;
    ps->rq_n = RQ_MAX;
  }
  for (int a = 1; a < ps->rq_n; a++) {  // insertion sort: short lists
    const unsigned int v = ps->rq[a];
    int b = a - 1;
    while (b >= 0 && ps->rq[b] > v) {
      ps->rq[b + 1] = ps->rq[b];
      b--;
    }
    ps->rq[b + 1] = v;
  }
  ps->rq_pos = 0;
}

// Thread 0: the oldest ready stashed message, or ~0 when none is left:
// from the ready list, or, when that overflowed, by scanning the keys
// from ready_cursor (keys before it are known not to be ready).
__device__ unsigned long long stash_next_ready() {
  pe_state* ps = pes();
  const unsigned long long S = (unsigned long long)c_rt.stash_entries;
  stash_key* keys = keys_of(blockIdx.x);
  if (!ps->rq_over) {
    while (ps->rq_pos < ps->rq_n) {
      const unsigned long long i = ps->rq_base + ps->rq[ps->rq_pos++];
      if (i >= ps->key_head && i < ps->key_tail && keys[i % S].state == KEY_READY) return i;
    }
    return ~0ULL;
  }
  unsigned long long i = ps->ready_cursor < ps->key_head ? ps->key_head : ps->ready_cursor;
  for (; i < ps->key_tail; i++)
    if (keys[i % S].state == KEY_READY) {
      ps->ready_cursor = i;
      return i;
    }
  ps->ready_cursor = i;
  return ~0ULL;
}

// Thread 0 of PE 0: stop the run when no PE has delivered anything for
// idle_timeout_ns (e.g. a program that never calls end()).
__device__ void check_idle_timeout(unsigned long long now) {
  if (c_rt.idle_timeout_ns == 0) return;
  pe_state* ps = pes();
  unsigned long long sum = 0;
  if (multi_dev()) {
    for (int p = 0; p < c_rt.n_pes; p++) sum += ld_relaxed_sys_u64(progress_of(p));
  } else {
    for (int p = 0; p < c_rt.n_pes; p++) sum += ld_relaxed_u64(&c_rt.progress[p]);
  }
  if (sum != ps->idle_sum) {
    ps->idle_sum = sum;
    ps->idle_change_ns = now;
  } else if (now - ps->idle_change_ns > c_rt.idle_timeout_ns) {
    set_error(CHARMING_ERR_IDLE_TIMEOUT, 0, 0);
  }
}

// ---------------------------------------------------------------------------
// async_wait (reference: check_async_wait, src/comm/get/get.cu:1172-1202,
// called once per scheduler iteration in its GPU-level loop,
// src/sched/scheduler.cu:305).
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool cmp_holds(unsigned long long v, int cmp, unsigned long long x) {
  switch (cmp) {
    case CMP_EQ: return v == x;
    case CMP_NE: return v != x;
    case CMP_GT: return v > x;
    case CMP_LE: return v <= x;
    case CMP_LT: return v < x;
    default: return v >= x;  // CMP_GE
  }
}

// Thread 0: the first satisfied wait (chare arrays in registration order,
// waits in slot order), taken off the list; its proxy, or nullptr. The words
// are read relaxed (no L1 invalidation per check); one acquire fence follows
// a hit, so what their writers published before them is visible.
__device__ chare_proxy_base* take_satisfied_wait(int* idx, int* ep) {
  pe_state* ps = pes();
  chare_proxy_table& tb = c_rt.proxy_tables[blockIdx.x];
  for (int id = 0; id < tb.count; id++) {
    chare_proxy_base* p = proxy_of(ps, id);
    if (p == nullptr || p->async_waits == nullptr) continue;
    for (int i = 0; i < ASYNC_WAIT_MAX; i++) {
      async_wait_t& aw = p->async_waits[i];
      if (!aw.valid) continue;
      bool ok = true;
      for (size_t k = 0; k < aw.nelems && ok; k++)
        ok = cmp_holds(ld_signal_u64(reinterpret_cast<const unsigned long long*>(aw.ivars) + k), aw.cmp,
                       aw.cmp_value);
      if (ok) {
        aw.valid = false;
        ps->aw_count--;
        *idx = aw.idx;
        *ep = aw.ep;
        fence_acq_rel_gpu();
        return p;
      }
    }
  }
  return nullptr;
}

// Thread 0: wait for the message at the inbox head. Returns 1 when it has
// arrived, 2 when deferred sends in the outbox can be flushed or async waits
// are pending (checked every 256 polls), 0 when this PE must leave the loop.
__device__ int poll_inbox() {
  pe_state* ps = pes();
  const int me = ps->my_pe;
  unsigned long long h = ps->head;
  const unsigned long long* f = ring_flag(me, h);
  unsigned int spins = 0;
  unsigned long long idle_t0 = 0;
  while (true) {
    if (ld_acquire_x(f) == h + 1) {
      if (idle_t0) ps->stats[ST_IDLE_CYC] += (unsigned long long)clock64() - idle_t0;
      // a PE that always has a message (a chare that keeps calling itself)
      // still sees the end of the run and its deadline
      if ((++ps->busy_polls & 63) == 0) {
        if (ps->term || terminated()) return 0;
        if (globaltimer() - ps->t0 > c_rt.deadline_ns) {
          set_error(CHARMING_ERR_DEADLINE, 1, 0);
          return 0;
        }
      }
      return 1;
    }
    if (ps->term) {
      publish_head(ps, me);
      return 0;
    }
    if (!idle_t0) {  // about to wait: the senders and the idle check see where we are
      idle_t0 = (unsigned long long)clock64() | 1;
      publish_head(ps, me);
      // deliveries since the last stamp count as progress (a return to the
      // loop for the outbox or async waits does not)
      if (ps->stats[ST_DELIVERED] != ps->stamped_delivered) {
        ps->stamped_delivered = ps->stats[ST_DELIVERED];
        stamp_progress(me);
      }
    }
    ++spins;
    // A PE idle for 32 polls pauses between polls: the polls of many idle
    // PEs slowed the PEs still working (a pingpong on 2 or 4 PEs per SM took
    // 40-100x longer, the batched set on 4 PEs per SM a third longer). The
    // termination word is read every 16th poll, and at every paused one.
    // (not while async waits or deferred sends need the periodic checks below)
    const bool paused = c_rt.idle_sleep_ns && spins > 32 && ps->aw_count == 0 && ps->ob_count == 0;
    if (paused) __nanosleep(c_rt.idle_sleep_ns);
    if ((paused || (spins & 15) == 0) && terminated()) {
      publish_head(ps, me);
      return 0;
    }
    if ((spins & 255) == 0) {
      unsigned long long now = globaltimer();
      if (now - ps->t0 > c_rt.deadline_ns) {
        set_error(CHARMING_ERR_DEADLINE, 0, 0);
        return 0;
      }
      // by time, not by spins: this wait may be cut short by the returns below
      if (now - ps->slow_check_ns > 100000) {
        ps->slow_check_ns = now;
        if (c_rt.host_stop) {
          int hs = ld_sys_s32(c_rt.host_stop);
          if (hs == 1) {
            raise_term();
            return 0;
          } else if (hs > 1) {
            set_error(CHARMING_ERR_HOST_STOP, hs, 0);
            return 0;
          }
        }
        if (me == 0 && ++ps->idle_checks % 10 == 0) check_idle_timeout(now);
      }
      ps->stats[ST_IDLE_POLLS] += 256;
      if ((ps->ob_count > 0 && outbox_head_ready()) || ps->aw_count > 0) {
        ps->stats[ST_IDLE_CYC] += (unsigned long long)clock64() - idle_t0;
        return 2;  // deferred sends can go out, or async waits to check
      }
    }
  }
}

// Thread 0: the thread-0 part that closes the action the block just executed.
__device__ void finish_action() {
  pe_state* ps = pes();
  const int me = ps->my_pe;
  switch (ps->d_act) {
    case ACT_CALL_RING:
    case ACT_STASH_PUT:
      // the block is done with the message: release its cells
      ps->head += ps->d_cells;
      if (ps->head - ps->head_pub >= (c_rt.ring_cells >> 3)) publish_head(ps, me);
      if (ps->d_act == ACT_CALL_RING && (++ps->stats[ST_DELIVERED] & 15) == 0) stamp_progress(me);
      break;
    case ACT_CALL_STASH: {
      const unsigned long long S = (unsigned long long)c_rt.stash_entries;
      keys_of(blockIdx.x)[ps->d_key % S].state = KEY_FREE;
      ps->n_ready--;
      if ((++ps->stats[ST_DELIVERED] & 15) == 0) stamp_progress(me);
      stash_retire();
      break;
    }
    case ACT_CALL_WAIT:
      if ((++ps->stats[ST_DELIVERED] & 15) == 0) stamp_progress(me);
      break;
    case ACT_STASH_BATCH: {
      const unsigned long long S = (unsigned long long)c_rt.stash_entries;
      for (int b = 0; b < ps->nb; b++) keys_of(blockIdx.x)[ps->bstash[b] % S].state = KEY_FREE;
      ps->n_ready -= ps->nb;
      const unsigned long long d0 = ps->stats[ST_DELIVERED];
      ps->stats[ST_DELIVERED] = d0 + (unsigned long long)ps->nb;
      if (ps->nb > 1) ps->stats[ST_BATCHED] += (unsigned long long)ps->nb;
      if ((d0 >> 4) != (ps->stats[ST_DELIVERED] >> 4)) stamp_progress(me);
      stash_retire();
      break;
    }
    case ACT_CALL_BATCH: {
      ps->head += ps->nb_cells;
      if (ps->head - ps->head_pub >= (c_rt.ring_cells >> 3)) publish_head(ps, me);
      const unsigned long long d0 = ps->stats[ST_DELIVERED];
      ps->stats[ST_DELIVERED] = d0 + (unsigned long long)ps->nb;
      if (ps->nb > 1) ps->stats[ST_BATCHED] += (unsigned long long)ps->nb;
      if ((d0 >> 4) != (ps->stats[ST_DELIVERED] >> 4)) stamp_progress(me);
      break;
    }
    case ACT_FLUSH: {
      const ob_entry* e = reinterpret_cast<const ob_entry*>(ps->d_p);
      publish(e->dst, e->ticket);
      ps->ob_head += e->span;
      ps->ob_count--;
      break;
    }
    case ACT_REVIVE: {
      const int c = ps->red_i[0];
      ps->n_ready += c;
      ps->n_waiting -= c;
      ps->stats[ST_REVIVED] += c;
      ready_list_sort();
      break;
    }
    default:
      break;
  }
  ps->d_act = ACT_NONE;
}

// Thread 0: a batch of warp-level deliveries from the ready stashed messages,
// the first (key i) already chosen: the next ready ones in arrival order
// while each is for a warp-level entry method of a chare not yet in the
// batch and its refnum matches (the first that is not is left for the
// next decision, as for inbox batches).
__device__ void stash_batch(chare_proxy_base* p, const stash_key* k, int ep, void* arg, unsigned long long i) {
  pe_state* ps = pes();
  const unsigned long long S = (unsigned long long)c_rt.stash_entries;
  stash_key* keys = keys_of(blockIdx.x);
  const int maxb = (int)(blockDim.x >> 5);
  ps->d_act = ACT_STASH_BATCH;
  ps->nb = 1;
  ps->bp[0] = p;
  ps->bidx[0] = k->chare_idx;
  ps->bep[0] = ep;
  ps->barg[0] = arg;
  ps->bstash[0] = i;
  ps->bkeys[0] = ((unsigned long long)(unsigned)k->chare_id << 32) | (unsigned)k->chare_idx;
  while (ps->nb < maxb && ps->n_ready > ps->nb) {
    const int pos = ps->rq_pos;
    const unsigned long long cur = ps->ready_cursor;
    const unsigned long long j = stash_next_ready();
    bool take = j != ~0ULL;
    const stash_key* kj = take ? keys + (j % S) : nullptr;
    chare_proxy_base* pj = take ? proxy_of(ps, kj->chare_id) : nullptr;
    const unsigned char* env = take ? arena_of(blockIdx.x) + (kj->data_off % c_rt.stash_bytes) : nullptr;
    const int epj = take ? reinterpret_cast<const regular_msg*>(env + sizeof(envelope))->ep_id : 0;
    const unsigned long long key =
        take ? ((unsigned long long)(unsigned)kj->chare_id << 32) | (unsigned)kj->chare_idx : 0;
    take = take && pj->warp_em(epj) && pj->refnum_matches(kj->chare_idx, kj->refnum);
    for (int b = 0; take && b < ps->nb; b++) take = ps->bkeys[b] != key;
    if (!take) {  // leave it for the next decision
      ps->rq_pos = pos;
      ps->ready_cursor = cur;
      break;
    }
    const int n = ps->nb;
    ps->bp[n] = pj;
    ps->bidx[n] = kj->chare_idx;
    ps->bep[n] = epj;
    ps->barg[n] = const_cast<unsigned char*>(env) + HDR;
    ps->bstash[n] = j;
    ps->bkeys[n] = key;
    ps->nb = n + 1;
  }
}

// Thread 0: decides what the block does next (pe_state d_* fields).
__device__ void next_action() {
  pe_state* ps = pes();
  const int me = ps->my_pe;
  const int slot = blockIdx.x;
  const unsigned long long S = (unsigned long long)c_rt.stash_entries;
  while (true) {
    if (ps->term) {
      ps->d_act = ACT_EXIT;
      return;
    }
    // deferred sends whose receivers have room
    if (ps->ob_count > 0 && outbox_head_ready()) {
      ps->d_act = ACT_FLUSH;
      ps->d_p = outbox_of(slot) + ps->ob_head % c_rt.outbox_bytes;
      return;
    }
    // satisfied async waits
    if (ps->aw_count > 0) {
      int idx = 0, ep = 0;
      chare_proxy_base* p = take_satisfied_wait(&idx, &ep);
      if (p) {
        if (terminated()) {
          ps->d_act = ACT_EXIT;
          return;
        }
        ps->d_act = ACT_CALL_WAIT;
        ps->d_p = p;
        ps->d_idx = idx;
        ps->d_ep = ep;
        ps->d_arg = nullptr;
        return;
      }
    }
    // set_refnum since the last look: re-examine the waiting stash entries
    if (ps->revive_pending) {
      ps->revive_pending = 0;
      if (ps->n_waiting > 0) {
        ps->red_i[0] = 0;
        ps->ready_cursor = ps->key_head;
        ps->rq_base = ps->key_head;
        ps->rq_n = 0;
        ps->rq_over = 0;
        ps->d_act = ACT_REVIVE;
        return;
      }
    }
    // ready stashed messages go before new inbox messages, oldest first
    while (ps->n_ready > 0) {
      const unsigned long long i = stash_next_ready();
      if (i == ~0ULL) {
        ps->n_ready = 0;
        break;
      }
      stash_key* k = keys_of(slot) + (i % S);
      chare_proxy_base* p = proxy_of(ps, k->chare_id);
      if (!p->refnum_matches(k->chare_idx, k->refnum)) {  // refnum moved on again
        k->state = KEY_WAIT;
        ps->n_ready--;
        ps->n_waiting++;
        continue;
      }
      if (terminated()) {
        ps->d_act = ACT_EXIT;
        return;
      }
      const unsigned char* env = arena_of(slot) + (k->data_off % c_rt.stash_bytes);
      const regular_msg* rm = reinterpret_cast<const regular_msg*>(env + sizeof(envelope));
      ps->d_act = ACT_CALL_STASH;
      ps->d_p = p;
      ps->d_idx = k->chare_idx;
      ps->d_ep = rm->ep_id;
      ps->d_arg = const_cast<unsigned char*>(env) + HDR;
      ps->d_key = i;
      // (from the on-chip ready list; past RQ_MAX ready ones, one at a time)
      if (p->warp_em(rm->ep_id) && batching() && !ps->rq_over) stash_batch(p, k, rm->ep_id, ps->d_arg, i);
      return;
    }
    // the inbox
    const int got = poll_inbox();
    if (got == 0) {
      ps->term = 1;
      ps->d_act = ACT_EXIT;
      return;
    }
    if (got == 2) continue;
    unsigned char* m = ring_cell(me, ps->head);
    const envelope* env = reinterpret_cast<const envelope*>(m);
    const regular_msg* rm = reinterpret_cast<const regular_msg*>(m + sizeof(envelope));
    unsigned long long size = env->size;
    const int type = (int)env->type;
    ps->d_act = ACT_NONE;
    if (size < HDR || size > c_rt.max_msg || (size & (ALIGN_SIZE - 1))) {
      set_error(CHARMING_ERR_BAD_MSG, env->src_pe, type);
      size = CELL;
    } else if (type == (int)msgtype::regular || type == (int)msgtype::user) {
      const int cid = rm->chare_id;
      chare_proxy_base* p = proxy_of(ps, cid);
      if (p == nullptr || !p->valid_target(rm->chare_idx, rm->ep_id)) {
        set_error(CHARMING_ERR_BAD_TARGET, cid, rm->chare_idx);
      } else if (p->refnum_matches(rm->chare_idx, rm->refnum)) {
        ps->d_act = ACT_CALL_RING;
        ps->d_p = p;
        ps->d_idx = rm->chare_idx;
        ps->d_ep = rm->ep_id;
        ps->d_arg = m + HDR;
        if (p->warp_em(rm->ep_id) && batching()) {
          // the first of a batch; warp 0 looks for more behind it
          ps->d_act = ACT_CALL_BATCH;
          ps->nb = 1;
          ps->nb_cells = cells_for(size);
          ps->bkey0 = ((unsigned long long)(unsigned)cid << 32) | (unsigned)rm->chare_idx;
          ps->bp[0] = p;
          ps->bidx[0] = rm->chare_idx;
          ps->bep[0] = rm->ep_id;
          ps->barg[0] = m + HDR;
        }
      } else {
        unsigned char* dst = stash_alloc(size, cid, rm->chare_idx, rm->refnum, env->src_pe);
        if (dst) {
          ps->d_act = ACT_STASH_PUT;
          ps->d_p = dst;
          ps->d_arg = m;
          ps->d_bytes = size;
        }
      }
    } else if (type == (int)msgtype::do_terminate || type == (int)msgtype::begin_terminate) {
      raise_term();
    } else {
      set_error(CHARMING_ERR_BAD_MSG, env->src_pe, type);
    }
    ps->d_cells = cells_for(size);
    if (ps->d_act != ACT_NONE) return;
    // nothing for the block to do with it: consume it here
    ps->head += ps->d_cells;
    if (ps->head - ps->head_pub >= (c_rt.ring_cells >> 3)) publish_head(ps, me);
  }
}

// Warp 0 (all lanes): extends the batch whose first delivery thread 0
// picked. Lane l reads the sequence words of cells l and l + 32 after the
// first message: where a published message starts the word holds that
// cell's ticket + 1, so one load per lane and window finds every message
// published in the next 64 cells, and one more reads their envelopes.
// Messages follow one another without gaps (each took its cells'
// tickets), so the batch follows the chain from the first message's end
// while each next message is published, is for a warp-level entry method
// of a chare not yet in the batch, and its refnum matches; it stops at the
// first that is not, which the scheduler then takes alone. The batch runs
// after a barrier, so the refnums checked here are the ones the sequential
// order would check: an entry method of the batch changes only its own
// chare's refnum.
struct scan_cell {
  unsigned int cells;
  int ok, idx, ep;
  unsigned long long key, p, arg;
};
__device__ __forceinline__ scan_cell scan_one(pe_state* ps, int me, unsigned long long t) {
  scan_cell c{0, 0, 0, 0, ~0ULL, 0, 0};
  if (ld_acquire_x(ring_flag(me, t)) == t + 1) {
    const unsigned char* m = ring_cell(me, t);
    const envelope* env = reinterpret_cast<const envelope*>(m);
    const regular_msg* rm = reinterpret_cast<const regular_msg*>(m + sizeof(envelope));
    const unsigned long long size = env->size;
    const int type = (int)env->type;
    if (size >= HDR && size <= c_rt.max_msg && !(size & (ALIGN_SIZE - 1)) &&
        (type == (int)msgtype::regular || type == (int)msgtype::user)) {
      chare_proxy_base* q = proxy_of(ps, rm->chare_id);
      c.idx = rm->chare_idx;
      c.ep = rm->ep_id;
      c.ok = q && q->valid_target(c.idx, c.ep) && q->warp_em(c.ep) && q->refnum_matches(c.idx, rm->refnum);
      c.cells = cells_for(size);
      c.key = ((unsigned long long)(unsigned)rm->chare_id << 32) | (unsigned)c.idx;
      c.p = reinterpret_cast<unsigned long long>(q);
      c.arg = reinterpret_cast<unsigned long long>(m + HDR);
    }
  }
  return c;
}

__device__ void batch_extend() {
  constexpr unsigned FULL = 0xffffffffu;
  pe_state* ps = pes();
  const int lane = (int)(threadIdx.x & 31);
  const int me = ps->my_pe;
  const int maxb = (int)(blockDim.x >> 5);
  const unsigned long long t0 = ps->head + ps->nb_cells + (unsigned long long)lane;
  const scan_cell lo = scan_one(ps, me, t0), hi = scan_one(ps, me, t0 + 32);
  // lane j holds the chare of batch member j
  unsigned long long mkey = lane == 0 ? ps->bkey0 : ~0ULL;
  int n = ps->nb, pos = 0;
  unsigned int total = ps->nb_cells;
  while (n < maxb && pos < 64) {  // uniform: every lane computes the same
    const bool w0 = pos < 32;
    const int src = pos & 31;
    if (!__shfl_sync(FULL, w0 ? lo.ok : hi.ok, src)) break;
    const unsigned long long k = __shfl_sync(FULL, w0 ? lo.key : hi.key, src);
    if (__any_sync(FULL, lane < n && mkey == k)) break;
    const unsigned int cl = __shfl_sync(FULL, w0 ? lo.cells : hi.cells, src);
    const unsigned long long bp = __shfl_sync(FULL, w0 ? lo.p : hi.p, src);
    const unsigned long long ba = __shfl_sync(FULL, w0 ? lo.arg : hi.arg, src);
    const int bi = __shfl_sync(FULL, w0 ? lo.idx : hi.idx, src);
    const int be = __shfl_sync(FULL, w0 ? lo.ep : hi.ep, src);
    if (lane == n) mkey = k;
    if (lane == 0) {
      ps->bp[n] = reinterpret_cast<chare_proxy_base*>(bp);
      ps->barg[n] = reinterpret_cast<void*>(ba);
      ps->bidx[n] = bi;
      ps->bep[n] = be;
    }
    n++;
    total += cl;
    pos += (int)cl;
  }
  if (lane == 0) {
    ps->nb = n;
    ps->nb_cells = total;
  }
}

// The loop: thread 0 closes the last action and picks the next; the block
// executes it. Two block barriers per message. In GPU-level mode this is
// block 0's loop: entry methods (and the exit) are handed to the other
// blocks through group_state, with a grid barrier before and after.
__device__ void scheduler_loop() {
  pe_state* ps = pes();
  const bool group = gpu_level();
  if (threadIdx.x == 0) ps->d_act = ACT_NONE;
  while (true) {
    if (threadIdx.x == 0) {
      finish_action();
      next_action();
    }
    __syncthreads();
    const int act = ps->d_act;
    const bool call = act == ACT_CALL_RING || act == ACT_CALL_STASH || act == ACT_CALL_WAIT;
    if (group && (call || act == ACT_EXIT)) {
      if (threadIdx.x == 0) {
        group_state* gs = c_rt.gl;
        gs->act = call ? ACT_CALL_RING : ACT_EXIT;
        gs->p = ps->d_p;
        gs->idx = ps->d_idx;
        gs->ep = ps->d_ep;
        gs->arg = ps->d_arg;
      }
      if (!grid_barrier_ok() || act == ACT_EXIT) break;
    }
    if (act == ACT_EXIT) break;
    chare_proxy_base* p = reinterpret_cast<chare_proxy_base*>(ps->d_p);
    if (call) {
      const long long c0 = clock64();
      // a warp-level entry method outside a batch: warp 0 (of block 0)
      if (!p->warp_em(ps->d_ep) || threadIdx.x < 32) p->em_tab[ps->d_ep](p, ps->d_idx, ps->d_arg);
      if (threadIdx.x == 0) ps->stats[ST_EM_CYC] += (unsigned long long)(clock64() - c0);
      if (group && !grid_barrier_ok()) break;  // every block is done with the message
    } else if (act == ACT_CALL_BATCH || act == ACT_STASH_BATCH) {
      const long long c0 = clock64();
      if (act == ACT_CALL_BATCH) {
        if (threadIdx.x < 32) batch_extend();
        __syncthreads();
      }
      const int w = (int)(threadIdx.x >> 5);
      if (w < ps->nb) {
        chare_proxy_base* q = ps->bp[w];
        q->em_tab[ps->bep[w]](q, ps->bidx[w], ps->barg[w]);
      }
      if (threadIdx.x == 0) ps->stats[ST_EM_CYC] += (unsigned long long)(clock64() - c0);
    } else if (act == ACT_STASH_PUT) {
      copy_cooperative(ps->d_p, ps->d_arg, ps->d_bytes, threadIdx.x, blockDim.x);
    } else if (act == ACT_FLUSH) {
      const ob_entry* e = reinterpret_cast<const ob_entry*>(ps->d_p);
      copy_cooperative(ring_cell(e->dst, e->ticket), reinterpret_cast<const unsigned char*>(e) + OB_HDR,
                       e->bytes, threadIdx.x, blockDim.x);
    } else if (act == ACT_REVIVE) {
      stash_revive_scan();
    }
    __syncthreads();
  }
}

// GPU-level mode, blocks 1..: run each entry method block 0 hands out.
__device__ void helper_loop() {
  const group_state* gs = c_rt.gl;
  while (true) {
    if (!grid_barrier_ok()) break;
    if (ld_relaxed_s32(&gs->act) != ACT_CALL_RING) break;
    chare_proxy_base* p = reinterpret_cast<chare_proxy_base*>(gl_ld_ptr(&gs->p));
    const int ep = ld_relaxed_s32(&gs->ep);
    if (!p->warp_em(ep)) p->em_tab[ep](p, ld_relaxed_s32(&gs->idx), gl_ld_ptr(&gs->arg));  // warp-level: block 0's warp 0
    if (!grid_barrier_ok()) break;
  }
}

} // namespace

// ---------------------------------------------------------------------------
// The persistent scheduler kernel (one launch per run, one block per PE).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(MAX_THREADS, 1)
charming_scheduler_kernel(int argc, char** argv, size_t* argvs) {
  pe_state* ps = pes();
  const int me = charm::my_pe();
  const int slot = local_slot();
  // the block that keeps the PE's state (every block in SM-level mode)
  const bool keeper = !gpu_level() || blockIdx.x == 0;
  if (threadIdx.x == 0) {
    ps->my_pe = me;
    ps->term = 0;
    ps->sent_term = 0;
    ps->revive_pending = 0;
    ps->head = *head_of(me);
    ps->head_pub = ps->head;
    ps->t0 = globaltimer();
    ps->key_head = ps->key_tail = 0;
    ps->arena_head = ps->arena_tail = 0;
    ps->n_waiting = ps->n_ready = 0;
    for (int i = 0; i < N_STATS; i++) ps->stats[i] = 0;
    ps->idle_polls_since_check = 0;
    ps->busy_polls = 0;
    ps->arena_top = 0;
    ps->sarena_top = 0;
    ps->ob_head = ps->ob_tail = 0;
    ps->ob_count = 0;
    ps->ob_lock = 0;
    ps->uh_head = ps->uh_tail = 0;
    ps->ub_head = ps->ub_tail = 0;
    ps->aw_count = 0;
    ps->gl_seq = 0;
    ps->bar_ok = 1;
    ps->ready_cursor = 0;
    ps->d_act = 0;
    ps->rq_base = 0;
    ps->rq_n = ps->rq_pos = 0;
    ps->rq_over = 1;  // no list yet: scan
    ps->stamped_delivered = ~0ULL;
    ps->idle_sum = ~0ULL;
    ps->idle_change_ns = ps->t0;
    ps->slow_check_ns = ps->t0;
    ps->idle_checks = 0;
    for (int i = 0; i < PROXY_CACHE; i++) ps->pcache[i] = nullptr;
  }
  for (int i = threadIdx.x; i < c_rt.n_pes; i += blockDim.x)
    head_cache()[i] = multi_dev() ? ld_relaxed_sys_u64(head_of(i)) : c_rt.head[i].v;
  __syncthreads();

  grid_barrier();
  charm::main(argc, argv, argvs, me);
  grid_barrier();

  const unsigned long long loop_t0 = threadIdx.x == 0 ? globaltimer() : 0;
  if (!terminated() && !ps->term) {
    if (keeper) scheduler_loop();
    else helper_loop();
  }
  const unsigned long long loop_t1 = threadIdx.x == 0 ? globaltimer() : 0;

  if (threadIdx.x == 0 && keeper) {
    ps->stats[ST_LOOP_NS] = loop_t1 - loop_t0;
    for (int i = 0; i < N_STATS; i++) c_rt.pe_stats[(unsigned long long)slot * N_STATS + i] = ps->stats[i];
    c_rt.pe_times[3 * slot] = ps->t0;
    c_rt.pe_times[3 * slot + 1] = loop_t0;
    c_rt.pe_times[3 * slot + 2] = loop_t1;
    if (c_rt.free_chares_at_exit) {
      chare_proxy_table& tb = c_rt.proxy_tables[slot];
      for (int i = tb.count - 1; i >= 0; i--) {
        chare_proxy_base* p = tb.proxies[i];
        if (p) {
          p->release_all();
          delete p;
        }
        tb.proxies[i] = nullptr;
      }
      tb.count = 0;
    }
  }
}

// Resets per-run control words of this launch's GPUs: every inbox restarts
// at its current tail (messages left over from an earlier run are dropped),
// proxy tables empty. With several GPUs, the host runs it on every GPU
// between two host barriers: after every launch of the last run has ended,
// before any of the next starts.
__global__ void charming_reset_kernel() {
  const int n = c_rt.gpu_level ? c_rt.n_pes : c_rt.n_blocks;  // PEs of this launch
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int pe = c_rt.pe0 + i;
    *head_of(pe) = *tail_of(pe);
    *progress_of(pe) = 0;
    c_rt.proxy_tables[i].count = 0;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const int d0 = dev_of(c_rt.pe0), d1 = dev_of(c_rt.pe0 + n - 1);
    for (int d = d0; d <= d1; d++) {
      int* w = c_rt.dev[d].ctrl;
      w[CTRL_TERM] = 0;
      w[CTRL_STATUS] = 0;
      w[CTRL_ERR_PE] = -1;
      w[CTRL_ERR_I0] = 0;
      w[CTRL_ERR_I1] = 0;
      w[CTRL_XBAR] = 0;
    }
    c_rt.ctrl[CTRL_BAR_COUNT] = 0;
  }
}
