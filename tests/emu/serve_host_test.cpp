// Unit check of the solve server's host logic (apps/serve_host.h), TEST
// INFRASTRUCTURE ONLY: the slab allocator, FIFO admission against the HBM
// budget, slots and workers, worker placement, generations, and the
// descriptors handed to the device. Prints "ok" or the first failure.
#include <array>
#include <cstdio>
#include <cstdlib>
#include <set>
#include <vector>

#include "../../charming_b200/csrc/apps/serve_host.h"

#define CHECK(c)                                                          \
  do {                                                                    \
    if (!(c)) {                                                           \
      printf("FAIL %s:%d: %s\n", __FILE__, __LINE__, #c);                 \
      exit(1);                                                            \
    }                                                                     \
  } while (0)

struct Sink : jserve::sink {
  std::vector<jac::chare_desc> d;
  std::vector<jac::prob_desc> p;
  std::vector<std::array<long, 3>> posted;
  Sink(int workers, int slots) : d(workers), p(slots) {}
  void stage_desc(int w, const jac::chare_desc& x) override { d[w] = x; }
  void stage_prob(int s, const jac::prob_desc& x) override { p[s] = x; }
  void post(int slot, int root, unsigned gen) override { posted.push_back({slot, root, (long)gen}); }
};

charming_jacobi_problem prob(int nx, int ny, int sweeps) {
  charming_jacobi_problem q{};
  q.nx = nx;
  q.ny = ny;
  q.max_sweeps = sweeps;
  q.bc[0] = 1.0;
  return q;
}

int main() {
  // slab: first fit, coalescing on release in any order
  {
    jserve::slab s;
    s.reset(10 * 256);
    uint64_t a, b, c, d;
    CHECK(s.alloc(256, &a) && a == 0);
    CHECK(s.alloc(300, &b) && b == 256);  // rounded to 512
    CHECK(s.alloc(1024, &c) && c == 768);
    CHECK(!s.alloc(1024, &d));            // 768 left
    s.release(b, 300);
    CHECK(s.alloc(512, &d) && d == 256);  // the hole is reused
    s.release(a, 256);
    s.release(d, 512);
    s.release(c, 1024);
    CHECK(s.used() == 0);
    CHECK(s.alloc(10 * 256, &a) && a == 0);  // everything coalesced again
    CHECK(s.peak() == 10 * 256);
  }
  // admission
  jserve::params P;
  P.n_pes = 4;
  P.workers_per_pe = 2;
  P.max_inflight = 3;
  P.chare_side = 16;
  P.esz = 8;
  P.off = 16;
  P.vec = 2;
  jac::layout L1;
  std::string e;
  charming_jacobi_problem big = prob(48, 32, 10);  // 3 x 2 chares
  CHECK(jac::build_layout(&big, 1, 16, 0, 0, 0, 1, 8, 16, 2, &L1, &e));
  P.budget = 2 * L1.total_bytes + 16384;            // two of these at once, plus a small one
  jserve::server_state st;
  const uintptr_t base = 1u << 20;
  st.init(P, base);
  Sink sk(8, 3);
  CHECK(st.submit(prob(200, 200, 1), 1, 0.0) != CHARMING_OK);  // 13 x 13 chares > 8 workers
  CHECK(st.submit(big, 10, 0.0) == CHARMING_OK);
  CHECK(st.submit(big, 10, 0.0) != CHARMING_OK);               // tag in use
  CHECK(st.submit(big, 11, 0.0) == CHARMING_OK);
  CHECK(st.submit(prob(8, 8, 3), 12, 0.0) == CHARMING_OK);     // 1 chare, but behind a blocked head
  CHECK(st.submit(big, 13, 0.0) == CHARMING_OK);
  CHECK(st.admit(sk, 1.0) == 1);  // 6 of 8 workers taken: the second 6-chare request waits
  CHECK(st.inflight == 1 && sk.posted.size() == 1);
  // the admitted request: 6 workers, one or two per PE, balanced
  jserve::admitted* a = st.find(10);
  CHECK(a && a->workers.size() == 6 && a->slot >= 0 && a->gen == 1);
  std::vector<int> per_pe(4, 0);
  std::set<int> ws(a->workers.begin(), a->workers.end());
  CHECK(ws.size() == 6);
  for (int w : a->workers) per_pe[w / 2]++;
  for (int k = 0; k < 4; k++) CHECK(per_pe[k] >= 1 && per_pe[k] <= 2);
  // descriptors: neighbours and tree in worker ids, own prob copy, slot,
  // buffers inside the slab
  for (size_t k = 0; k < a->workers.size(); k++) {
    const jac::chare_desc& d = sk.d[a->workers[k]];
    CHECK(d.prob == a->workers[k] && d.slot == a->slot);
    for (int q = 0; q < jac::N_DIRS; q++) CHECK(d.nbr[q] == -1 || ws.count(d.nbr[q]));
    CHECK(d.parent == -1 || ws.count(d.parent));
    CHECK((uintptr_t)d.buf[0] >= base && (uintptr_t)d.buf[1] < base + P.budget);
  }
  CHECK(sk.p[a->slot].root == a->workers[0] && sk.p[a->slot].n_chares == 6);
  CHECK(sk.posted[0][0] == a->slot && sk.posted[0][1] == a->workers[0]);
  // completion frees the workers and the slot (not the memory): the next
  // two requests fit now (11 in memory, 12 behind it)
  jac::serve_comp c{};
  c.slot = a->slot;
  c.gen = 99;
  CHECK(st.complete(c, 2.0) == nullptr);  // wrong generation: ignored
  c.gen = a->gen;
  CHECK(st.complete(c, 2.0) == a && a->done);
  CHECK(st.admit(sk, 2.0) == 2);          // 11 (6 workers) and 12 (1 worker); 13 waits
  CHECK(st.find(11)->gen == 2 && st.find(12)->gen == 3);
  CHECK(st.release(11) != CHARMING_OK);   // not completed yet
  CHECK(st.release(10) == CHARMING_OK);   // memory of 10 free: 13 still needs workers
  CHECK(st.admit(sk, 3.0) == 0);
  jac::serve_comp c2{};
  c2.slot = st.find(11)->slot;
  c2.gen = 2;
  CHECK(st.complete(c2, 3.0));
  CHECK(st.admit(sk, 3.0) == 1 && st.find(13)->gen == 4);
  CHECK(st.mem.peak() <= P.budget);
  CHECK(st.peak_inflight == 2 && st.n_admitted == 4 && st.n_completed == 2);
  printf("ok\n");
  return 0;
}
