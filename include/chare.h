// charming-b200: chares, chare arrays (proxies) and entry methods.
//
// Source-compatible with the reference's include/chare.h:24-270: same
// names, template signatures, placement rule and refnum rule, so that code
// written against it (e.g. examples/hello, refnum, pingpong) compiles
// unchanged. What differs is underneath: a mismatched message is copied into
// a per-PE stash managed by the scheduler instead of a fixed 128-entry table
// per chare type (include/chare.h:12, :51-58), and invalid targets are turned
// into a runtime error status instead of an assert.
#ifndef _CHARE_H_
#define _CHARE_H_

#include "common.h"
#include "message.h"
#include "kernel.h"

#define CHARE_TYPE_CNT_MAX 1024 // Maximum number of chare types per PE
#define EM_CNT_MAX 128          // Maximum number of entry methods per chare type
#define ASYNC_WAIT_MAX 16       // Pending async_waits per chare array per PE
#define MISMATCH_MAX 128        // Kept for source compatibility (stash is per PE)

namespace charm {

struct chare {
  int i;
  int n;

  __device__ chare() : i(-1), n(0) {}
};

template <class C>
struct entry_method_base {
  __device__ virtual void operator()(C& chare, void* arg) = 0;
  __device__ virtual ~entry_method_base() {}
};

template <class C, void Func(C&, void*)>
struct entry_method : entry_method_base<C> {
  __device__ virtual void operator()(C& chare, void* arg) { Func(chare, arg); }
};

struct async_wait_t {
  bool valid;
  uint64_t* ivars;
  size_t nelems;
  int cmp;
  uint64_t cmp_value;
  int idx;
  int ep;
};

struct mismatch_t {
  int found_idx;
  uint64_t comp;
  int chare_idx;
  int refnum;

  __device__ mismatch_t() : found_idx(-1) {}
};

namespace detail {
// Per-PE bump allocator for the runtime's own objects (proxies, chare
// objects, their tables): small objects go to a shared-memory arena of the
// PE block, the rest to a per-PE region of device memory; reset at every
// run, nothing freed one by one. Single-threaded. Returns nullptr when both
// are exhausted (callers fall back to the device heap). Objects in shared
// memory keep their cached state when a gpu-scope acquire (every inbox poll)
// invalidates the SM's L1.
__device__ void* pe_alloc(size_t bytes);
// Whether p came from a PE arena (then it is not handed to free()).
__device__ bool pe_owns(const void* p);
}  // namespace detail

struct chare_proxy_base;
// Entry method `ep` of local chare `idx` on `arg` (all threads of the block).
typedef bool (*proxy_call_fn)(chare_proxy_base* proxy, int idx, int ep, void* arg);
// One registered entry method with the lookup of its chare object: the
// scheduler reaches an entry method with this one indirect call.
typedef void (*em_entry_fn)(chare_proxy_base* proxy, int idx, void* arg);

struct chare_proxy_base {
  int id;        // Chare array ID (registration order on this PE)

  int n_local;   // Number of local chares
  int n_total;   // Total number of chares
  int start_idx; // Starting index of local chares
  int end_idx;   // Ending index of local chares

  int* loc_map;  // Chare -> PE location map

  int em_count;  // Number of registered entry methods

  async_wait_t* async_waits;

  int* refnum;   // Reference numbers of local chares
  mismatch_t* mismatches;

  proxy_call_fn call_fn;  // direct dispatch (no virtual call on the hot path)
  em_entry_fn* em_tab;    // the entry methods, each with its object lookup

  // Entry methods 0..63 registered with add_warp_entry_method (bit ep): one
  // warp runs each of their deliveries.
  unsigned long long warp_ems;

  __device__ chare_proxy_base() : id(-1), n_local(0), n_total(0), start_idx(-1),
  end_idx(-1), loc_map(nullptr), em_count(0), async_waits(nullptr),
  refnum(nullptr), mismatches(nullptr), call_fn(nullptr), em_tab(nullptr), warp_ems(0) {}

  __device__ bool warp_em(int ep) const { return ep >= 0 && ep < 64 && ((warp_ems >> ep) & 1ULL); }

  // Proxies come from the PE arena (shared memory when there is room), so
  // the scheduler's per-message reads of them stay on chip.
  __device__ static void* operator new(size_t bytes) {
    void* p = detail::pe_alloc(bytes);
    return p ? p : malloc(bytes);
  }
  __device__ static void operator delete(void* p) {
    if (p && !detail::pe_owns(p)) free(p);
  }

  // Runs entry method ep of local chare idx on arg (all threads of the PE
  // block). The scheduler decides the refnum match (refnum_matches, the
  // rule of include/chare.h:181-195) in one thread before it calls: the
  // entry method may change the chare's refnum at once, so the threads must
  // not test it again here. Returns true.
  __device__ virtual bool call(int idx, int ep, void* arg, int ref) = 0;
  // Frees the local chares and tables (the runtime calls it when a run ends
  // and then deletes the proxy).
  __device__ virtual void release_all() {}
  __device__ virtual ~chare_proxy_base() {}

  // Target validity, checked by the scheduler before call().
  __device__ bool valid_target(int idx, int ep) const {
    return idx >= start_idx && idx <= end_idx && n_local > 0 && ep >= 0 && ep < em_count;
  }
  __device__ bool refnum_matches(int idx, int ref) const {
    return ref == -1 || ref == refnum[idx - start_idx];
  }
};

struct chare_proxy_table {
  chare_proxy_base* proxies[CHARE_TYPE_CNT_MAX];
  int count;

  __host__ __device__ chare_proxy_table() : count(0) {}
};

namespace detail {
// This PE's proxy table (one per PE thread block).
__device__ chare_proxy_table& my_proxy_table();
// Record a runtime error; the scheduler stops all PEs and the host call
// returns `code` (see charming_c.h for the codes).
__device__ void report_error(int code, int info0, int info1);
enum : int {
  ERR_BAD_TARGET = 3,
  ERR_TOO_MANY_TYPES = 10,
  ERR_TOO_MANY_EMS = 11,
  ERR_NO_MEMORY = 17,
  ERR_TOO_MANY_WAITS = 19,
};
// Registers proxy `id` in the scheduler's on-chip lookup cache.
__device__ void cache_proxy(int id, chare_proxy_base* p);
template <class T>
__device__ T* pe_array(size_t n) {  // trivially constructible T
  void* p = pe_alloc(n * sizeof(T));
  return p ? static_cast<T*>(p) : new T[n];
}
template <class T>
__device__ void pe_free_array(T* p) {
  if (p && !pe_owns(p)) delete[] p;
}
template <class T>
__device__ T* pe_make() {
  void* p = pe_alloc(sizeof(T));
  return p ? new (p) T() : new T();
}
template <class T>
__device__ void pe_destroy(T* p) {
  if (!p) return;
  if (pe_owns(p)) p->~T();
  else delete p;
}
} // namespace detail

__device__ int my_pe();

template <typename C>
struct chare_proxy : chare_proxy_base {
  typedef void (*em_fn_t)(C&, void*);
  C** objects;     // Local chare objects
  // Entry method table (em_tab): per entry method a function that looks up
  // the chare object and calls the entry method, inlined into it (the
  // reference keeps entry_method objects with a virtual call operator; one
  // function pointer per message saves the vtable loads and a second call)

  // Registers this proxy in the calling PE's table (single-threaded).
  __device__ chare_proxy()
    : chare_proxy_base(), objects(nullptr) {
    chare_proxy_table& table = detail::my_proxy_table();
    if (table.count >= CHARE_TYPE_CNT_MAX) {
      detail::report_error(detail::ERR_TOO_MANY_TYPES, table.count, 0);
      return;
    }
    id = table.count++;
    table.proxies[id] = this;
    detail::cache_proxy(id, this);
    call_fn = &chare_proxy<C>::call_static;
    em_tab = detail::pe_array<em_entry_fn>(EM_CNT_MAX);
    if (em_tab == nullptr) detail::report_error(detail::ERR_NO_MEMORY, id, 0);
  }

  template <void Func(C&, void*)>
  __device__ static void em_entry(chare_proxy_base* base, int idx, void* arg) {
    chare_proxy<C>* self = static_cast<chare_proxy<C>*>(base);
    Func(*(self->objects[idx - self->start_idx]), arg);
  }

  // Add entry method to table (single-threaded)
  template <void Func(C&, void*)>
  __device__ void add_entry_method() {
    if (em_tab == nullptr || em_count >= EM_CNT_MAX) {
      detail::report_error(detail::ERR_TOO_MANY_EMS, id, em_count);
      return;
    }
    em_tab[em_count++] = &chare_proxy<C>::em_entry<Func>;
  }

  // Registers an entry method that one warp runs instead of the whole PE
  // block (an extension; the reference has block entry methods only). The
  // scheduler runs consecutive deliveries of such entry methods to different
  // chares together, one per warp of the block. The entry method may use
  // warp-level synchronisation only (no __syncthreads(), and no sends:
  // invoke and the user-message calls are block-collective), indexes its
  // lanes by threadIdx.x % 32, and changes the refnum of its own chare only.
  // Single-threaded, like add_entry_method.
  template <void Func(C&, void*)>
  __device__ void add_warp_entry_method() {
    if (em_count >= 64) {
      detail::report_error(detail::ERR_TOO_MANY_EMS, id, em_count);
      return;
    }
    const int ep = em_count;
    add_entry_method<Func>();
    if (em_count == ep + 1) warp_ems |= 1ULL << ep;
  }

  __device__ static bool call_static(chare_proxy_base* base, int idx, int ep, void* arg) {
    chare_proxy<C>* self = static_cast<chare_proxy<C>*>(base);
    self->em_tab[ep](base, idx, arg);
    return true;
  }

  // Create the chare array on every PE (single-threaded; called by each PE).
  // Default block mapping: n / n_pes per PE, the first n % n_pes PEs get one
  // more; with block_map, block_map[pe] chares go to PE pe, in order
  // (include/chare.h:125-177).
  __device__ void create(int n_chares, int* block_map) {
    int n_pes_ = c_n_pes;
    int me = charm::my_pe();

    loc_map = detail::pe_array<int>(n_chares > 0 ? n_chares : 1);
    if (loc_map == nullptr) {
      detail::report_error(detail::ERR_NO_MEMORY, id, n_chares);
      return;
    }
    n_total = n_chares;

    int n_chares_pe = n_chares / n_pes_;
    int rem = n_chares % n_pes_;
    int start = 0;
    for (int pe = 0; pe < n_pes_; pe++) {
      int n_cur = block_map ? block_map[pe] : n_chares_pe;
      if (!block_map && pe < rem) n_cur++;
      int end = start + n_cur - 1;

      if (pe == me) {
        n_local = n_cur;
        start_idx = start;
        end_idx = end;
        objects = (n_local > 0) ? detail::pe_array<C*>(n_local) : nullptr;
        refnum = (n_local > 0) ? detail::pe_array<int>(n_local) : nullptr;
        if (n_local > 0 && (objects == nullptr || refnum == nullptr)) {
          detail::report_error(detail::ERR_NO_MEMORY, id, n_local);
          n_local = 0;
        }
        for (int k = 0; k < n_local; k++) {
          objects[k] = detail::pe_make<C>();
          if (objects[k] == nullptr) {
            detail::report_error(detail::ERR_NO_MEMORY, id, k);
            n_local = k;
            break;
          }
          objects[k]->i = start_idx + k;
          objects[k]->n = n_total;
          refnum[k] = -1;
        }
      }
      for (int i = start; i <= end && i < n_chares; i++) loc_map[i] = pe;
      start += n_cur;
    }
  }

  inline __device__ void create(int n_chares) { create(n_chares, nullptr); }

  __device__ virtual bool call(int idx, int ep, void* arg, int ref) {
    (void)ref;
    return call_static(this, idx, ep, arg);
  }

  __device__ virtual void release_all() {
    for (int k = 0; k < n_local; k++) detail::pe_destroy(objects[k]);
    detail::pe_free_array(objects);
    detail::pe_free_array(refnum);
    detail::pe_free_array(loc_map);
    detail::pe_free_array(em_tab);
    detail::pe_free_array(async_waits);
    async_waits = nullptr;
    objects = nullptr;
    refnum = nullptr;
    loc_map = nullptr;
    em_tab = nullptr;
    n_local = 0;
    em_count = 0;
  }

  // Local object of chare idx, or nullptr if it lives on another PE.
  __device__ C* local(int idx) const {
    return (idx >= start_idx && idx <= end_idx) ? objects[idx - start_idx] : nullptr;
  }

  // Block-collective sends (include/chare.h:197-210). `buf` is copied before
  // the call returns and may be reused at once.
  inline __device__ void invoke(int idx, int ep) { invoke(idx, ep, nullptr, 0); }
  inline __device__ void invoke(int idx, int ep, void* buf, size_t size) {
    invoke(idx, ep, buf, size, -1);
  }
  inline __device__ void invoke(int idx, int ep, void* buf, size_t size, int ref) {
    if (idx < 0 || idx >= n_total) {
      if (threadIdx.x == 0) detail::report_error(detail::ERR_BAD_TARGET, id, idx);
      return;
    }
    send_reg_msg(id, idx, ep, buf, size, loc_map[idx], ref);
  }

  inline __device__ void invoke_all(int ep) { invoke_all(ep, nullptr, 0); }
  inline __device__ void invoke_all(int ep, void* buf, size_t size) {
    for (int i = 0; i < n_total; i++) invoke(i, ep, buf, size);
  }

  // Zero-copy messages (the reference's TODO user-message API,
  // include/chare.h:255-269). Block-collective.
  inline __device__ bool alloc_msg(message& msg, int idx, size_t size) {
    if (idx < 0 || idx >= n_total) {
      if (threadIdx.x == 0) detail::report_error(detail::ERR_BAD_TARGET, id, idx);
      return false;
    }
    return alloc_user_msg(msg, loc_map[idx], size);
  }
  inline __device__ void invoke(int idx, int ep, message& msg) {
    send_user_msg(id, idx, ep, msg, msg.capacity, -1);
  }
  inline __device__ void invoke(int idx, int ep, message& msg, size_t size) {
    send_user_msg(id, idx, ep, msg, size, -1);
  }
  inline __device__ void invoke(int idx, int ep, message& msg, size_t size, int ref) {
    send_user_msg(id, idx, ep, msg, size, ref);
  }
  // The reference's forms (include/chare.h:257-262) take the message by
  // const reference: the same sends, leaving the caller's copy as it was
  // (it must not be sent again).
  inline __device__ void invoke(int idx, int ep, const message& msg) {
    message m = msg;
    send_user_msg(id, idx, ep, m, m.capacity, -1);
  }
  inline __device__ void invoke(int idx, int ep, const message& msg, size_t size) {
    message m = msg;
    send_user_msg(id, idx, ep, m, size, -1);
  }
  inline __device__ void free_msg(message& msg) {}

  // Batched zero-copy messages to chares idx[0..n) (extension, see
  // alloc_user_msgs in message.h). Block-collective.
  inline __device__ bool alloc_msgs(message* msgs, const int* idx, const size_t* sizes, int n) {
    int pe[MSG_BATCH_MAX];
    for (int k = 0; k < n; k++) {
      if (k >= MSG_BATCH_MAX || idx[k] < 0 || idx[k] >= n_total) {
        if (threadIdx.x == 0) detail::report_error(detail::ERR_BAD_TARGET, id, k < MSG_BATCH_MAX ? idx[k] : k);
        return false;
      }
      pe[k] = loc_map[idx[k]];
    }
    return alloc_user_msgs(msgs, pe, sizes, n);
  }
  inline __device__ void invoke_msgs(const int* idx, int ep, message* msgs, const size_t* sizes,
      const int* refnums, int n) {
    send_user_msgs(id, idx, ep, msgs, sizes, refnums, n);
  }

  // Single-threaded (reference include/chare.h:214-239, built there for its
  // GPU-level mode only). Registers a wait: once each of the nelems 64-bit
  // words at ivars compares true against cmp_value (cmp is one of
  // charm::CMP_*, the NVSHMEM_CMP_* values), the scheduler runs entry method
  // ep of local chare idx once, with a null argument, and forgets the wait.
  // The words are read at device scope, so other PEs publish them with
  // release stores or atomics; what they wrote before is visible to the
  // entry method. Up to ASYNC_WAIT_MAX waits per chare array per PE. A wait
  // that is never satisfied ends the run at the idle timeout.
  inline __device__ void async_wait(uint64_t* ivars, size_t nelems, int cmp, uint64_t cmp_value,
      int idx, int ep) {
    if (idx < start_idx || idx > end_idx || ep < 0 || ep >= em_count || ivars == nullptr ||
        cmp < CMP_EQ || cmp > CMP_GE) {
      detail::report_error(detail::ERR_BAD_TARGET, id, idx);
      return;
    }
    if (async_waits == nullptr) {
      async_waits = detail::pe_array<async_wait_t>(ASYNC_WAIT_MAX);
      if (async_waits == nullptr) {
        detail::report_error(detail::ERR_NO_MEMORY, id, idx);
        return;
      }
      for (int i = 0; i < ASYNC_WAIT_MAX; i++) async_waits[i].valid = false;
    }
    int free_idx = -1;
    for (int i = 0; i < ASYNC_WAIT_MAX; i++) {
      if (!async_waits[i].valid) {
        free_idx = i;
        break;
      }
    }
    if (free_idx < 0) {
      detail::report_error(detail::ERR_TOO_MANY_WAITS, id, idx);
      return;
    }
    async_wait_t& aw = async_waits[free_idx];
    aw.ivars = ivars;
    aw.nelems = nelems;
    aw.cmp = cmp;
    aw.cmp_value = cmp_value;
    aw.idx = idx;
    aw.ep = ep;
    aw.valid = true;
    add_async_wait(id);
  }

  // Single-threaded (include/chare.h:243-253)
  inline __device__ void set_refnum(int idx, int val) {
    if (idx < start_idx || idx > end_idx) {
      detail::report_error(detail::ERR_BAD_TARGET, id, idx);
      return;
    }
    refnum[idx - start_idx] = val;
    revive_mismatches(id, idx, val);
  }
  inline __device__ int get_refnum(int idx) const { return refnum[idx - start_idx]; }
};

} // namespace charm

#endif // _CHARE_H_
