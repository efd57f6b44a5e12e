// charming-b200: message formats and the device-side send interface.
//
// Type and enum names follow the reference's include/message.h:10-95 so that
// user code written against it compiles unchanged. On the wire every message
// in an inbox ring is `envelope` (16 B) + `regular_msg` (16 B) + payload,
// rounded up to 16 B, exactly the reference's envelope::alloc_size
// (include/message.h:61-81). The envelope's padding word carries the sending
// PE, which the reference left unused.
#ifndef _MESSAGE_H_
#define _MESSAGE_H_

#include "common.h"

// Alignment of every message and payload (include/message.h:5)
#define ALIGN_SIZE 16

namespace charm {

// Message types (include/message.h:10-17). request/forward belong to the
// reference's multi-GPU CE path and are accepted by the API but never sent on
// one GPU; begin_terminate/do_terminate are replaced by a device-wide
// termination word (see charm::end()).
enum class msgtype : int {
  regular,
  request,
  forward,
  user,
  begin_terminate,
  do_terminate
};

// Regular message header between chares (include/message.h:20-28)
struct alignas(ALIGN_SIZE) regular_msg {
  int chare_id;
  int chare_idx;
  int ep_id;
  int refnum;

  __device__ regular_msg(int chare_id_, int chare_idx_, int ep_id_, int refnum_)
    : chare_id(chare_id_), chare_idx(chare_idx_), ep_id(ep_id_), refnum(refnum_) {}
};

// Request sent from PE to CE (include/message.h:31-41); kept for source
// compatibility only: there is no CE on a single GPU.
struct alignas(ALIGN_SIZE) request_msg : regular_msg {
  msgtype type;
  void* buf;
  size_t payload_size;
  int dst_pe;

  __device__ request_msg(int chare_id_, int chare_idx_, int ep_id_, msgtype type_,
      void* buf_, size_t payload_size_, int dst_pe_, int refnum_)
    : regular_msg(chare_id_, chare_idx_, ep_id_, refnum_), type(type_),
    buf(buf_), payload_size(payload_size_), dst_pe(dst_pe_) {}
};

// Message forwarded between CEs (include/message.h:44-50); source
// compatibility only.
struct alignas(ALIGN_SIZE) forward_msg : regular_msg {
  int dst_pe;

  __device__ forward_msg(int chare_id_, int chare_idx_, int ep_id_, int dst_pe_,
      int refnum_)
    : regular_msg(chare_id_, chare_idx_, ep_id_, refnum_), dst_pe(dst_pe_) {}
};

// Envelope at the start of every message (include/message.h:53-82).
struct alignas(ALIGN_SIZE) envelope {
  msgtype type;
  int src_pe;   // sending PE (padding in the reference)
  size_t size;  // total message bytes (envelope + header + payload, rounded)

  __device__ envelope(msgtype type_, size_t size_)
    : type(type_), src_pe(-1), size(size_) {}

  // Total size of a message for allocation (include/message.h:61-81)
  static __host__ __device__ inline size_t alloc_size(msgtype type, size_t payload_size) {
    size_t type_size = 0;
    if (type == msgtype::regular || type == msgtype::user) {
      type_size = sizeof(regular_msg);
    } else if (type == msgtype::request) {
      type_size = sizeof(request_msg);
    } else if (type == msgtype::forward) {
      type_size = sizeof(forward_msg);
    }
    size_t s = sizeof(envelope) + type_size + payload_size;
    size_t rem = s % ALIGN_SIZE;
    if (rem != 0) s = s + ALIGN_SIZE - rem;
    return s;
  }
};

// User (zero-copy) message. The reference declares this API but leaves it
// as a TODO (include/message.h:85-95, include/chare.h:255-269). Here it is
// implemented: chare_proxy<C>::alloc_msg() reserves space directly in the
// destination PE's inbox ring, the caller fills payload(), and
// chare_proxy<C>::invoke(idx, ep, msg[, size[, refnum]]) publishes it. The
// payload pointer is valid from alloc_msg until that invoke.
struct alignas(ALIGN_SIZE) message {
  envelope* env;   // start of the reserved ring space
  size_t offset;   // ring ticket (in cells) of the reservation
  int dst_pe;      // destination PE
  int cells;       // reserved ring cells
  size_t capacity; // payload bytes reserved

  __device__ message() : env(nullptr), offset(0), dst_pe(-1), cells(0), capacity(0) {}
  __device__ void* payload() const {
    return env ? (void*)((char*)env + sizeof(envelope) + sizeof(regular_msg)) : nullptr;
  }
};

// Block-collective: every thread of the calling PE block must call these.
// The buffer pointer, size and target are taken from thread 0 (the reference
// does the same through shared memory, src/comm/get/get.cu:866-913), so a
// buffer that only thread 0 holds may be passed.
__device__ void send_reg_msg(int chare_id, int chare_idx, int ep_id, void* buf,
    size_t payload_size, int dst_pe, int refnum);
__device__ void send_begin_term_msg();
__device__ bool alloc_user_msg(message& msg, int dst_pe, size_t payload_size);
__device__ void send_user_msg(int chare_id, int chare_idx, int ep_id,
    message& msg, size_t payload_size, int refnum);

// Several zero-copy messages at once (an extension; the reference sends one
// at a time): n <= MSG_BATCH_MAX messages to PEs dst_pes[k] with
// payload_sizes[k] bytes are reserved by n threads in parallel, and later
// published in parallel, so their ring reservations and publishing fences
// overlap. Block-collective; every thread passes the same arrays. Returns
// false when a reservation failed (error recorded).
constexpr int MSG_BATCH_MAX = 8;
__device__ bool alloc_user_msgs(message* msgs, const int* dst_pes, const size_t* payload_sizes,
    int n);
__device__ void send_user_msgs(int chare_id, const int* chare_idx, int ep_id, message* msgs,
    const size_t* payload_sizes, const int* refnums, int n);
// MSG_BATCH_MAX message descriptors in the calling PE block's shared memory,
// for alloc_user_msgs / send_user_msgs (an extension). Passed one of these,
// the calls fill and clear it from thread 0 alone instead of giving every
// thread its own copy, which saves each batch hundreds of bytes of
// local-memory traffic per thread. One array per block: a batch must be sent
// before the next is reserved.
__device__ message* block_messages();

// Single-threaded (called under threadIdx.x == 0 by set_refnum). Marks the
// PE's stash for re-examination; stashed messages whose refnum now matches
// their chare are delivered, in arrival order, before new inbox messages
// (reference: src/comm/get/get.cu:1316-1345).
__device__ void revive_mismatches(int chare_id, int chare_idx, int refnum);

// Single-threaded (called by chare_proxy<C>::async_wait): tells the
// scheduler that a wait was registered on this PE (reference
// include/message.h:112).
__device__ void add_async_wait(int chare_id);

} // namespace charm

#endif // _MESSAGE_H_
