// Host side of the Jacobi2d solve server, without CUDA calls: admission of
// requests against an HBM budget, request slots and worker chares, the
// decomposition of a request into chares (jacobi_layout.h) bound to
// workers, and the descriptors the device reads. Shared by
// charming_serve_* (serve.cu) and the CPU check of the serving path, so
// both run the same admission and placement.
//
// Request life: submit -> pending (FIFO) -> admitted (slot, workers and
// grid memory taken; descriptors staged; posted to the device ring) ->
// completed (completion record read; slot and workers free again, the grids
// stay resident) -> released (grid memory free).
#pragma once

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <deque>
#include <map>
#include <string>
#include <unordered_map>
#include <vector>

#include "charming_c.h"
#include "jacobi_types.cuh"
#include "jacobi_layout.h"

namespace jserve {

// First-fit allocator over [0, cap) in 256-byte units, free ranges
// coalesced.
class slab {
 public:
  void reset(uint64_t cap) {
    free_.clear();
    cap_ = cap / 256 * 256;
    if (cap_) free_[0] = cap_;
    used_ = peak_ = 0;
  }
  bool alloc(uint64_t n, uint64_t* off) {
    n = (n + 255) / 256 * 256;
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < n) continue;
      *off = it->first;
      uint64_t rest = it->second - n, at = it->first + n;
      free_.erase(it);
      if (rest) free_[at] = rest;
      used_ += n;
      peak_ = std::max(peak_, used_);
      return true;
    }
    return false;
  }
  void release(uint64_t off, uint64_t n) {
    n = (n + 255) / 256 * 256;
    used_ -= n;
    auto it = free_.emplace(off, n).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
  uint64_t used() const { return used_; }
  uint64_t peak() const { return peak_; }
  uint64_t cap() const { return cap_; }

 private:
  std::map<uint64_t, uint64_t> free_;
  uint64_t cap_ = 0, used_ = 0, peak_ = 0;
};

struct request {
  uint64_t tag;
  charming_jacobi_problem prob;
  double submit_s;
};

// An admitted request (active until its completion is read, then done
// until released).
struct admitted {
  uint64_t tag = 0;
  charming_jacobi_problem prob{};
  int slot = -1;
  unsigned gen = 0;
  std::vector<int> workers;             // local chare index -> worker
  std::vector<jac::chare_desc> chares;  // local order, device addresses
  uint64_t off = 0, bytes = 0;          // grid memory in the slab
  double submit_s = 0, admit_s = 0, done_s = 0;
  jac::serve_comp comp{};               // completion record (when done)
  bool done = false;
};

struct params {
  int n_pes = 0;
  int workers_per_pe = 0;
  int max_inflight = 0;
  uint64_t budget = 0;
  int chare_side = 256;
  int depth = 0;                        // 0: the library's default
  int esz = 8, off = 16, vec = 2;       // element bytes, interior column offset, vector width
};

// What admission writes for the device: the worker's descriptor, the
// slot's problem descriptor, then the request record (posted last).
struct sink {
  virtual void stage_desc(int worker, const jac::chare_desc& d) = 0;
  virtual void stage_prob(int slot, const jac::prob_desc& p) = 0;
  virtual void post(int slot, int root_worker, unsigned gen) = 0;
  virtual ~sink() {}
};

class server_state {
 public:
  std::string err;

  void init(const params& p, uintptr_t slab_base) {
    P = p;
    base = slab_base;
    mem.reset(p.budget);
    free_slots.clear();
    for (int s = p.max_inflight - 1; s >= 0; s--) free_slots.push_back(s);
    free_workers.assign(p.n_pes, {});
    for (int pe = 0; pe < p.n_pes; pe++)
      for (int k = p.workers_per_pe - 1; k >= 0; k--) free_workers[pe].push_back(pe * p.workers_per_pe + k);
    pe_load.assign(p.n_pes, 0.0);
    pending.clear();
    by_slot.assign(p.max_inflight, nullptr);
    reqs.clear();
    gen_next = 1;
    n_submitted = n_admitted = n_completed = 0;
    inflight = peak_inflight = 0;
  }

  // Checks a request (size, decomposition, and that it could ever be
  // admitted) and queues it. Returns a status code.
  int submit(const charming_jacobi_problem& q, uint64_t tag, double now) {
    if (reqs.count(tag)) return fail("serve: tag already in use");
    uint64_t bytes = 0;
    int nch = 0;
    jac::layout L;
    if (!plan(q, &L)) return CHARMING_ERR_CONFIG;
    bytes = L.total_bytes;
    nch = (int)L.chares.size();
    if (bytes > mem.cap()) return fail("serve: request larger than the HBM budget");
    if (nch > P.n_pes * P.workers_per_pe) return fail("serve: request needs more chares than workers");
    pending.push_back(request{tag, q, now});
    reqs[tag] = nullptr;
    n_submitted++;
    return CHARMING_OK;
  }

  // Admits pending requests in arrival order while a slot, enough workers
  // and grid memory are free (the head of the queue blocks the rest, so a
  // large request is not starved by smaller ones behind it). Returns the
  // number admitted, or -1 (err set).
  int admit(sink& out, double now) {
    int n = 0;
    while (!pending.empty() && !free_slots.empty()) {
      const request& r = pending.front();
      jac::layout L;
      if (!plan(r.prob, &L)) return -1;
      const int nch = (int)L.chares.size();
      if (free_worker_count() < nch) break;
      uint64_t off = 0;
      if (!mem.alloc(L.total_bytes, &off)) break;
      admitted* a = new admitted();
      a->tag = r.tag;
      a->prob = r.prob;
      a->slot = free_slots.back();
      free_slots.pop_back();
      a->gen = gen_next++;
      a->off = off;
      a->bytes = L.total_bytes;
      a->submit_s = r.submit_s;
      a->admit_s = now;
      place(L, a);
      jac::place_buffers(&L, reinterpret_cast<char*>(base + off), P.esz);
      a->chares.resize(nch);
      for (int k = 0; k < nch; k++) {
        jac::chare_desc d = L.chares[k];
        const int w = a->workers[k];
        for (int q = 0; q < jac::N_DIRS; q++) d.nbr[q] = d.nbr[q] < 0 ? -1 : a->workers[d.nbr[q]];
        d.parent = d.parent < 0 ? -1 : a->workers[d.parent];
        d.child[0] = d.child[0] < 0 ? -1 : a->workers[d.child[0]];
        d.child[1] = d.child[1] < 0 ? -1 : a->workers[d.child[1]];
        d.prob = w;  // each worker keeps its own copy of the problem descriptor
        d.slot = a->slot;
        a->chares[k] = d;
        out.stage_desc(w, d);
      }
      jac::prob_desc pd = L.probs[0];
      pd.root = a->workers[0];
      out.stage_prob(a->slot, pd);
      by_slot[a->slot] = a;
      reqs[a->tag] = a;
      pending.pop_front();
      out.post(a->slot, a->workers[0], a->gen);
      inflight++;
      peak_inflight = std::max(peak_inflight, inflight);
      n_admitted++;
      n++;
    }
    return n;
  }

  // A completion record: frees the request's slot and workers (its grids
  // stay). Returns the request, or null for a record that matches none.
  admitted* complete(const jac::serve_comp& c, double now) {
    if (c.slot < 0 || c.slot >= P.max_inflight) return nullptr;
    admitted* a = by_slot[c.slot];
    if (!a || a->gen != c.gen) return nullptr;
    a->comp = c;
    a->done = true;
    a->done_s = now;
    by_slot[c.slot] = nullptr;
    free_slots.push_back(c.slot);
    for (size_t k = 0; k < a->workers.size(); k++) {
      int w = a->workers[k];
      int pe = w / P.workers_per_pe;
      free_workers[pe].push_back(w);
      pe_load[pe] -= work(a->chares[k]);
    }
    inflight--;
    n_completed++;
    return a;
  }

  // Frees a completed request's grids. Returns a status code.
  int release(uint64_t tag) {
    auto it = reqs.find(tag);
    if (it == reqs.end() || !it->second || !it->second->done) return fail("serve: no completed request with this tag");
    mem.release(it->second->off, it->second->bytes);
    delete it->second;
    reqs.erase(it);
    return CHARMING_OK;
  }

  admitted* find(uint64_t tag) {
    auto it = reqs.find(tag);
    return it == reqs.end() ? nullptr : it->second;
  }
  bool idle() const { return pending.empty() && inflight == 0; }
  ~server_state() {
    for (auto& kv : reqs) delete kv.second;
  }

  params P;
  uint64_t n_submitted = 0, n_admitted = 0, n_completed = 0;
  int inflight = 0, peak_inflight = 0;
  slab mem;

 private:
  int fail(const char* m) {
    err = m;
    return CHARMING_ERR_CONFIG;
  }
  static double work(const jac::chare_desc& d) { return (double)d.w * d.h + 4096.0; }
  int free_worker_count() const {
    int n = 0;
    for (const auto& v : free_workers) n += (int)v.size();
    return n;
  }
  bool plan(const charming_jacobi_problem& q, jac::layout* L) {
    charming_jacobi_problem one = q;
    std::string e;
    if (!jac::build_layout(&one, 1, P.chare_side, 0, P.depth, 0, 1, P.esz, P.off, P.vec, L, &e)) {
      err = e;
      return false;
    }
    return true;
  }
  // Chares (largest first) onto the least-loaded PEs that have a free
  // worker.
  void place(const jac::layout& L, admitted* a) {
    const int nch = (int)L.chares.size();
    std::vector<int> order(nch);
    for (int k = 0; k < nch; k++) order[k] = k;
    std::stable_sort(order.begin(), order.end(),
                     [&](int x, int y) { return work(L.chares[x]) > work(L.chares[y]); });
    a->workers.assign(nch, -1);
    for (int k : order) {
      int best = -1;
      for (int pe = 0; pe < P.n_pes; pe++) {
        if (free_workers[pe].empty()) continue;
        if (best < 0 || pe_load[pe] < pe_load[best]) best = pe;
      }
      a->workers[k] = free_workers[best].back();
      free_workers[best].pop_back();
      pe_load[best] += work(L.chares[k]);
    }
  }

  uintptr_t base = 0;
  std::vector<int> free_slots;
  std::vector<std::vector<int>> free_workers;
  std::vector<double> pe_load;
  std::deque<request> pending;
  std::vector<admitted*> by_slot;
  std::unordered_map<uint64_t, admitted*> reqs;  // tag -> request (null while pending)
  unsigned gen_next = 1;
};

}  // namespace jserve
