// Jacobi2d chares: the scenario of the reference's examples/jacobi2d
// (jacobi2d.cu:93-279) on this runtime, for many problems at once.
//
// Per chare and exchange ("pass"): receive one halo per neighbour, run the
// pass's sweeps on the block (jacobi_sweep.cuh), then pack the new boundary
// rows/columns straight into the neighbours' inbox rings (zero-copy
// messages). Halos carry their pass number, which closes the reference's
// ghost race (jacobi2d.cu:171-190 / :222): a halo of pass p lands in the
// ghost zone of buffer p & 1. A pass is one sweep with ghost depth 1 (the
// reference's scheme) or up to `depth` sweeps with a ghost zone that deep,
// corners included (temporal blocking: same arithmetic per point, fewer
// exchanges and one read + one write of the block per pass).
// Optional FP64 residual every `check_every` sweeps: each chare's partial
// goes up a binary tree over the problem's chares (fixed summation order, so
// the norm is bit-reproducible) and the stop decision comes back down. The
// decision for the check taken at sweep cK is applied at sweep (c+1)K, which
// leaves K sweeps for the round trip.
//
// Serving (g_app.a[6] != 0): the same chares form a pool of reusable
// workers, created once for a long-lived scheduler run; a server chare on
// PE 0 polls a request ring in mapped host memory and starts each admitted
// request at its root worker (the start travels down the residual tree).
// Every message carries the request's generation; the first one of a new
// generation resets the worker, copies its descriptor from the host's
// staging table and initialises its grids. The request's last chare to
// finish writes a completion record into mapped host memory.
#include "suite.cuh"
#include "jacobi_types.cuh"
#include "jacobi_sweep.cuh"

namespace {

enum : int { EP_START = 0, EP_HALO = 1, EP_CONT = 2, EP_PARTIAL = 3, EP_DECISION = 4 };
enum : int { EP_POLL = 0 };  // server chare

// g_app fields of this program.
struct japp {
  __device__ static int n_chares() { return (int)g_app.a[0]; }
  __device__ static int dtype() { return (int)g_app.a[2]; }
  __device__ static int pipeline() { return (int)g_app.a[3]; }
  __device__ static int tile_w() { return (int)g_app.a[4]; }
  __device__ static int halo_mode() { return (int)g_app.a[5]; }
  // multi-sweep passes: 0 phase-split items, 1 the single-loop items
  __device__ static bool deep_lean() { return g_app.a[9] == 0; }
  __device__ static const jac::chare_desc* chares() {
    return reinterpret_cast<const jac::chare_desc*>(g_app.p[0]);
  }
  __device__ static const jac::prob_desc* probs() {
    return reinterpret_cast<const jac::prob_desc*>(g_app.p[1]);
  }
  __device__ static jac::prob_result* results() {
    return reinterpret_cast<jac::prob_result*>(g_app.p[2]);
  }
  __device__ static unsigned long long* done_counter() {
    return reinterpret_cast<unsigned long long*>(g_app.p[3]);
  }
  __device__ static int* final_buf() { return reinterpret_cast<int*>(g_app.p[4]); }
  __device__ static const int* block_map() { return reinterpret_cast<const int*>(g_app.p[5]); }
  // per-PE nanoseconds of the run: [4 * pe + k], k = 0 sweeps, 1 sending
  // halos, 2 halo entry methods (unpack and what follows)
  __device__ static unsigned long long* pe_ns() {
    return reinterpret_cast<unsigned long long*>(g_app.p[6]);
  }
  // serving
  __device__ static bool serving() { return g_app.a[6] != 0; }
  __device__ static int serve_q() { return (int)g_app.a[7]; }   // request ring entries
  __device__ static int serve_cq() { return (int)g_app.a[8]; }  // completion ring entries
  __device__ static jac::serve_req* serve_reqs() { return reinterpret_cast<jac::serve_req*>(g_app.p[7]); }
  __device__ static const jac::chare_desc* stage_descs() {
    return reinterpret_cast<const jac::chare_desc*>(g_app.p[8]);
  }
  __device__ static const jac::prob_desc* stage_probs() {
    return reinterpret_cast<const jac::prob_desc*>(g_app.p[9]);
  }
  __device__ static jac::serve_comp* serve_comps() { return reinterpret_cast<jac::serve_comp*>(g_app.p[10]); }
  // [0] requests started and not completed, [1] completion tickets
  __device__ static unsigned long long* serve_ctr() { return reinterpret_cast<unsigned long long*>(g_app.p[11]); }
  __device__ static unsigned int* serve_done() { return reinterpret_cast<unsigned int*>(g_app.p[12]); }
  __device__ static const int* serve_ctl() { return reinterpret_cast<const int*>(g_app.p[13]); }  // [0] stop
  __device__ static const int* server_map() { return reinterpret_cast<const int*>(g_app.p[14]); }
};

struct JBlock : charm::chare {
  int iter;          // sweeps completed; buf[cur] holds u_iter
  int pass;          // passes completed (cur == pass & 1)
  int cur;
  int sent;          // last pass whose boundary went to the neighbours
  int started;       // the start message has been processed
  int got[2];        // halos received for the pass of each parity
  int gotx[2];       // of which left/right halos (two-phase exchange)
  int nbr_count;     // halos per pass
  int nbx;           // of which left/right (two-phase exchange)
  int sent_y;        // last pass whose top/bottom halos went out (two-phase)
  int done;
  int waiting;       // parked until the decision of check iter/K - 1 arrives
  // residual tree state for the check in progress
  int have_own;
  int child_got[2];
  double own;
  double child_val[2];
  int decided;       // highest check with a known decision (-1: none)
  int stop_check;    // check whose decision was "stop" (-1: none)
  double res0, res_last;
  int checks;
  unsigned gen;      // request generation (serving; 0 otherwise)
  // The chare's own copies of its block and problem descriptors: chare
  // objects live in the PE's on-chip arena, so the entry methods read these
  // without a trip to memory after every inbox acquire.
  jac::chare_desc desc;
  jac::prob_desc prob;
  __device__ JBlock() { reset(0); }
  __device__ void reset(unsigned g) {
    iter = pass = cur = 0;
    sent = -1;
    started = nbr_count = done = waiting = have_own = 0;
    own = 0.0;
    decided = stop_check = -1;
    res0 = res_last = 0.0;
    checks = 0;
    gen = g;
    got[0] = got[1] = 0;
    gotx[0] = gotx[1] = 0;
    nbx = 0;
    sent_y = -1;
    child_got[0] = child_got[1] = 0;
    child_val[0] = child_val[1] = 0.0;
  }
};

// The server chare of a serving run (one, on PE 0): next request ticket.
struct JServer : charm::chare {
  unsigned long long next;
  __device__ JServer() : next(0) {}
};

__shared__ charm::chare_proxy<JBlock>* jproxy;
// This PE's phase timers (ns: sweeps, halo sending, halo entry methods),
// kept on chip and stored through to japp::pe_ns() after every update (a
// store only: no read of global memory on the message path).
// Slots: 0 sweeps, 1 halo sends (all of send_halos), 2 halo entry methods,
// 3 of the sends: up to the ring space taken, 4 of the sends: publishing,
// 5 of the sends: up to the reservation call.
constexpr int PE_NS_SLOTS = 8;
__shared__ unsigned long long s_pe_ns[6];
// The phase timers count SM cycles (clock64, a register read, instead of
// the %globaltimer reads of the run-level checks); the host converts them
// with the SM clock rate.
__device__ __forceinline__ unsigned long long pe_clock() { return (unsigned long long)clock64(); }
__device__ __forceinline__ void add_pe_cyc(int k, unsigned long long cyc) {
  s_pe_ns[k] += cyc;
  japp::pe_ns()[PE_NS_SLOTS * blockIdx.x + k] = s_pe_ns[k];
}
__shared__ charm::chare_proxy<JServer>* sproxy;

template <typename T>
__device__ jac::block_view<T> view(const jac::chare_desc& d, int b) {
  return jac::block_view<T>{reinterpret_cast<T*>(d.buf[b]), d.pitch};
}

// Sweeps per pass: the ghost depth, cut at the next residual check and at
// max_sweeps, so checks fall on pass boundaries.
__device__ int pass_len(const jac::chare_desc& d, const jac::prob_desc& p, int iter) {
  int L = d.depth;
  if (p.max_sweeps - iter < L) L = p.max_sweeps - iter;
  if (p.check_every > 0) {
    int to_check = p.check_every - iter % p.check_every;
    if (to_check < L) L = to_check;
  }
  return L < 1 ? 1 : L;
}

// One pass of L sweeps buf[cur] -> buf[cur^1]; returns the block's residual
// sum of the pass's first sweep (FP64, deterministic) when resid is set.
// All threads.
template <typename T>
__device__ double sweep_block(const jac::chare_desc& d, int cur, bool resid, int L) {
  jac::block_view<T> in = view<T>(d, cur), out = view<T>(d, cur ^ 1);
  double acc = 0.0;
  bool done = false;
  if (!CHARM_VERIFY(d.w > 0 && d.h > 0 && d.buf[0] && d.buf[1] && (cur == 0 || cur == 1) &&
                        L >= 1 && L <= d.depth,
                    CHARMING_ERR_APP, 8000 + cur, d.w))
    return 0.0;
  // phase timers: thread 0 alone reads the clock
  const unsigned long long t0 = threadIdx.x == 0 ? pe_clock() : 0;
  if (L > 1) {
    int fixed = (d.nbr[jac::TOP] < 0 ? 1 : 0) | (d.nbr[jac::BOTTOM] < 0 ? 2 : 0) |
                (d.nbr[jac::LEFT] < 0 ? 4 : 0) | (d.nbr[jac::RIGHT] < 0 ? 8 : 0);
    __syncthreads();
    acc = resid ? jac::sweep_deep<T, true>(in, out, d.w, d.h, L, fixed, japp::deep_lean())
                : jac::sweep_deep<T, false>(in, out, d.w, d.h, L, fixed, japp::deep_lean());
    __syncthreads();
    done = true;
  }
#if !defined(CHARMING_HOST_EMULATION) || defined(CHARMING_HOST_EMULATION_TMA)
  if (!done && japp::pipeline()) {
    size_t sb = 0;
    void* sm = charm::smem_scratch(&sb);
    jac::tma_plan P;
    if (jac::make_plan<T>(d.w, blockDim.x, sb, japp::tile_w(), &P)) {
      if (resid) jac::sweep_tma<T, true>(in, out, d.w, d.h, sm, sb, P, &acc);
      else jac::sweep_tma<T, false>(in, out, d.w, d.h, sm, sb, P, &acc);
      done = true;
    }
  }
#endif
  if (!done) {
    __syncthreads();
    acc = resid ? jac::sweep_direct<T, true>(in, out, d.w, d.h)
                : jac::sweep_direct<T, false>(in, out, d.w, d.h);
    __syncthreads();
  }
  if (threadIdx.x == 0) add_pe_cyc(0, pe_clock() - t0);
  return resid ? suite::block_sum_f64(acc) : 0.0;
}

// Copies up to N_DIRS rectangles between a chare grid and packed row-major
// buffers (to_grid: buffers -> grid) in one pass over all their cells. A
// rectangle whose rows start on 16-byte boundaries on both sides and hold
// whole vectors moves in 16-byte vectors, the others element by element.
// Each thread loads a batch of B units before it stores any, so the loads of
// all rectangles are in flight together instead of one rectangle (or row)
// after another. All threads.
template <typename T>
__device__ void copy_rects(jac::block_view<T> g, const jac::region* e, T* const* bufs, int n, bool to_grid) {
  using VT = typename jac::vec_of<T>::type;
  constexpr int V = jac::traits<T>::VEC, B = 8;
  int start[jac::N_DIRS + 1], unit[jac::N_DIRS];
  start[0] = 0;
  for (int k = 0; k < n; k++) {
    const bool vec = (e[k].nc % V) == 0 &&
                     (reinterpret_cast<uintptr_t>(g.at(e[k].r0, e[k].c0)) & 15) == 0 &&
                     (reinterpret_cast<uintptr_t>(bufs[k]) & 15) == 0;
    unit[k] = vec ? V : 1;
    start[k + 1] = start[k] + e[k].nr * e[k].nc / unit[k];
  }
  const int total = start[n];
  const int stride = (int)blockDim.x;
  for (int base = (int)threadIdx.x; base < total; base += B * stride) {
    VT v[B];
    T* dst[B];
    int u[B];
#pragma unroll
    for (int b = 0; b < B; b++) {
      const int i = base + b * stride;
      dst[b] = nullptr;
      u[b] = 1;
      if (i < total) {
        int k = 0;
        while (k + 1 < n && i >= start[k + 1]) k++;
        const int nu = e[k].nc / unit[k];        // units per row
        const int j = i - start[k];
        const int r = j / nu, cu = j - r * nu;
        T* gp = g.at(e[k].r0 + r, e[k].c0 + cu * unit[k]);
        T* bp = bufs[k] + (size_t)r * e[k].nc + cu * unit[k];
        T* src = to_grid ? bp : gp;
        dst[b] = to_grid ? gp : bp;
        u[b] = unit[k];
        if (unit[k] == V) v[b] = *reinterpret_cast<const VT*>(src);
        else reinterpret_cast<T*>(&v[b])[0] = *src;
      }
    }
#pragma unroll
    for (int b = 0; b < B; b++) {
      if (!dst[b]) continue;
      if (u[b] == V) *reinterpret_cast<VT*>(dst[b]) = v[b];
      else *dst[b] = reinterpret_cast<const T*>(&v[b])[0];
    }
  }
}

// Thread 0: the chare's halo counts per pass (all its neighbours; with the
// two-phase exchange the corner directions have none).
__device__ void count_nbrs(JBlock& c, const jac::chare_desc& d) {
  int n = 0, nx = 0;
  for (int k = 0; k < jac::N_DIRS; k++) {
    if (d.nbr[k] < 0) continue;
    n++;
    if (d.ext > 0 && (k == jac::LEFT || k == jac::RIGHT)) nx++;
  }
  c.nbr_count = n;
  c.nbx = nx;
}

// Packs the boundary regions of buf[cur] for every neighbour straight into
// their inbox rings (zero-copy) and publishes them together: the ring
// reservations, the packing loads and the publishing fences of the messages
// overlap (refnum = pass in halo_mode 1). phase 0: every neighbour (the
// one-phase exchange); 1: left and right; 2: top and bottom, with the ghost
// columns the left/right halos of this pass filled. All threads.
// The halos of one batch: one copy per block, written by thread 0 (a
// private copy in every thread was local memory, about 350 bytes per thread
// per batch).
struct halo_batch {
  int idx[jac::N_DIRS], dirs[jac::N_DIRS], refs[jac::N_DIRS];
  size_t bytes[jac::N_DIRS];
  jac::region e[jac::N_DIRS];
  void* vals[jac::N_DIRS];
  int n;
};
__shared__ halo_batch s_halos;

template <typename T>
__device__ void send_halos(JBlock& c, const jac::chare_desc& d, int phase = 0) {
  const unsigned long long t0 = threadIdx.x == 0 ? pe_clock() : 0;
  halo_batch& b = s_halos;
  __syncthreads();  // every thread is done with the last batch's record
  if (threadIdx.x == 0) {
    int n = 0;
    const bool tagged = japp::halo_mode() == 1;
    for (int dir = 0; dir < jac::N_DIRS; dir++) {
      if (d.nbr[dir] < 0) continue;
      if (phase == 1 && dir != jac::LEFT && dir != jac::RIGHT) continue;
      if (phase == 2 && dir != jac::TOP && dir != jac::BOTTOM) continue;
      b.e[n] = jac::halo_edge(dir, d);
      b.idx[n] = d.nbr[dir];
      b.dirs[n] = dir;
      b.refs[n] = tagged ? c.pass : -1;
      b.bytes[n] = sizeof(jac::halo_hdr) + (size_t)b.e[n].nr * b.e[n].nc * sizeof(T);
      n++;
    }
    b.n = n;
  }
  __syncthreads();
  const int n = b.n;
  static_assert(jac::N_DIRS <= charm::MSG_BATCH_MAX, "one batch holds every halo of a phase");
  charm::message* msg = charm::block_messages();  // one copy per block, in shared memory
  CHARM_PROF(if (threadIdx.x == 0) add_pe_cyc(5, pe_clock() - t0);)
  const bool got = n > 0 && jproxy->alloc_msgs(msg, b.idx, b.bytes, n);
  CHARM_PROF(if (threadIdx.x == 0) add_pe_cyc(3, pe_clock() - t0);)
  if (got) {
    for (int k = (int)threadIdx.x; k < n; k += (int)blockDim.x) {  // one header per thread
      jac::halo_hdr* hh = reinterpret_cast<jac::halo_hdr*>(msg[k].payload());
      hh->dir = jac::opposite(b.dirs[k]);
      hh->len = b.e[k].nr * b.e[k].nc;
      hh->pass = c.pass;
      hh->gen = c.gen;
      b.vals[k] = reinterpret_cast<char*>(msg[k].payload()) + sizeof(jac::halo_hdr);
    }
    __syncthreads();
    copy_rects<T>(view<T>(d, c.cur), b.e, reinterpret_cast<T* const*>(b.vals), n, false);
    CHARM_PROF(const unsigned long long tp = threadIdx.x == 0 ? pe_clock() : 0;)
    jproxy->invoke_msgs(b.idx, EP_HALO, msg, b.bytes, b.refs, n);
    CHARM_PROF(if (threadIdx.x == 0) add_pe_cyc(4, pe_clock() - tp);)
  }
  if (threadIdx.x == 0) add_pe_cyc(1, pe_clock() - t0);
}

// Halo of pass hh->pass -> ghost zone of buf[pass & 1]. All threads.
template <typename T>
__device__ void unpack_halo(JBlock& c, const jac::chare_desc& d, const void* arg) {
  const jac::halo_hdr* hh = reinterpret_cast<const jac::halo_hdr*>(arg);
  T* vals = const_cast<T*>(reinterpret_cast<const T*>(reinterpret_cast<const char*>(arg) + sizeof(jac::halo_hdr)));
  jac::region gr = jac::halo_ghost(hh->dir, d);
  copy_rects<T>(view<T>(d, hh->pass & 1), &gr, &vals, 1, true);
}


// Serving, thread 0 of the request's last chare: completion record into the
// mapped host ring (fields first, then seq with a system-scope release).
// The ring has as many entries as request slots and the host frees a slot
// only after reading its record, so an entry is never overwritten unread.
__device__ void serve_complete(const JBlock& c, const jac::chare_desc& d) {
  using namespace charm::rt;
  unsigned long long t = atomicAdd(&japp::serve_ctr()[1], 1ULL);
  jac::serve_comp* r = japp::serve_comps() + t % (unsigned long long)japp::serve_cq();
  r->slot = d.slot;
  r->gen = c.gen;
  r->sweeps = c.iter;
  r->checks = c.checks;
  r->final_buf = c.cur;
  r->status = 0;
  r->res0 = c.res0;
  r->res_last = c.res_last;
  r->t_ns = globaltimer();
  __threadfence_system();
  st_release_sys_u64(&r->seq, t + 1);
  atomicAdd(&japp::serve_ctr()[0], ~0ULL);  // one request fewer in flight
}

// All threads. Marks the chare done; the last chare of all problems ends the
// run (the reference counts "end" messages at chare 0, jacobi2d.cu:274-279).
// Serving: the last chare of the request reports its completion instead.
__device__ void finish(JBlock& c, const jac::chare_desc& d) {
  __shared__ int s_last;
  if (threadIdx.x == 0 && japp::serving()) {
    c.done = 1;
    const jac::prob_desc& p = c.prob;
    __threadfence();
    unsigned n = atomicAdd(&japp::serve_done()[d.slot], 1u) + 1;
    if (n == (unsigned)p.n_chares) serve_complete(c, d);
    s_last = 0;
  } else if (threadIdx.x == 0) {
    c.done = 1;
    japp::final_buf()[c.i] = c.cur;
    const jac::prob_desc& p = c.prob;
    if (p.root == c.i) {
      jac::prob_result& r = japp::results()[d.prob];
      r.sweeps = c.iter;
      r.checks = c.checks;
      r.res0 = c.res0;
      r.res_last = c.res_last;
    }
    __threadfence();
    unsigned long long n = atomicAdd(japp::done_counter(), 1ULL) + 1;
    s_last = (n == (unsigned long long)japp::n_chares()) ? 1 : 0;
  }
  __syncthreads();
  if (s_last) charm::end();
}

// Serving, all threads: the first message of a new request generation
// resets the worker, copies its descriptor and its request's problem
// descriptor from the host's staging tables (mapped host memory, read at
// system scope) into the worker's own entries, and writes both grids: the
// boundary ring where the block touches it, 0 everywhere else (ghost cells
// beyond the ring included, so nothing of a previous request survives).
// Generations grow with every admission. Returns 0 for a message of an
// older generation, which the caller drops: with residual checks none can
// arrive (a chare finishes only after the last decision of its tree, so
// nothing of a completed request is in flight), without them a start that
// went down the tree after its chare had finished can.
template <typename T>
__device__ int ensure_gen(JBlock& c, unsigned gen) {
  using namespace charm::rt;
  if (!japp::serving()) return 1;
  __shared__ int s_new;
  if (threadIdx.x == 0) s_new = gen > c.gen ? 1 : gen == c.gen ? 0 : -1;
  __syncthreads();
  const int fresh = s_new;
  __syncthreads();
  if (fresh <= 0) return fresh + 1;
  static_assert(sizeof(jac::chare_desc) % 8 == 0 && sizeof(jac::prob_desc) % 8 == 0, "word copies");
  constexpr int WD = sizeof(jac::chare_desc) / 8, WP = sizeof(jac::prob_desc) / 8;
  {
    const unsigned long long* src = reinterpret_cast<const unsigned long long*>(japp::stage_descs() + c.i);
    unsigned long long* dst = reinterpret_cast<unsigned long long*>(&c.desc);
    for (int k = threadIdx.x; k < WD; k += blockDim.x) dst[k] = ld_relaxed_sys_u64(src + k);
  }
  __syncthreads();
  const jac::chare_desc& d = c.desc;
  {
    const unsigned long long* src = reinterpret_cast<const unsigned long long*>(japp::stage_probs() + d.slot);
    unsigned long long* dst = reinterpret_cast<unsigned long long*>(&c.prob);
    for (int k = threadIdx.x; k < WP; k += blockDim.x) dst[k] = ld_relaxed_sys_u64(src + k);
  }
  __syncthreads();
  const jac::prob_desc& p = c.prob;
  if (CHARM_VERIFY(d.w > 0 && d.h > 0 && d.depth >= 1 && d.depth <= jac::DEPTH_MAX && d.prob == c.i,
                   CHARMING_ERR_APP, 9000 + d.depth, c.i)) {
    const int D = d.depth, rows = d.h + 2 * D;
    const long long n = (long long)rows * d.pitch;
    for (int b = 0; b < 2; b++) {
      T* base = reinterpret_cast<T*>(d.buf[b]) + (long long)(1 - D) * d.pitch;
      for (long long x = threadIdx.x; x < n; x += blockDim.x) {
        const int r = (int)(x / d.pitch) + 1 - D, col = (int)(x % d.pitch) - jac::traits<T>::OFF + 1;
        const int gy = d.y0 + r, gx = d.x0 + col;
        double v = 0.0;
        if (gy >= 0 && gy <= p.ny + 1 && gx >= 0 && gx <= p.nx + 1) {
          if (gy == 0) v = p.bc[0];
          else if (gy == p.ny + 1) v = p.bc[1];
          else if (gx == 0) v = p.bc[2];
          else if (gx == p.nx + 1) v = p.bc[3];
        }
        base[x] = (T)v;
      }
    }
  }
  if (threadIdx.x == 0) {
    c.reset(gen);
    count_nbrs(c, d);
    c.started = 1;
  }
  __syncthreads();
  return 1;
}

#include "jacobi_chare.cuh"

// Serving, server chare: takes up to 4 posted requests from the mapped ring
// per call, starts each at its root worker, and calls itself again; ends the
// run when the host asked to stop and no request is in flight. All threads.
__device__ void em_poll(JServer& s, void* arg) {
  using namespace charm::rt;
  constexpr int MAXN = 4;
  __shared__ int s_n, s_stop;
  __shared__ jac::start_msg s_m[MAXN];
  __shared__ int s_root[MAXN];
  if (threadIdx.x == 0) {
    int n = 0;
    while (n < MAXN) {
      jac::serve_req* q = japp::serve_reqs() + s.next % (unsigned long long)japp::serve_q();
      if (ld_acquire_sys_u64(&q->seq) != s.next + 1) break;
      unsigned long long w1 = ld_relaxed_sys_u64(reinterpret_cast<const unsigned long long*>(q) + 1);
      unsigned long long w2 = ld_relaxed_sys_u64(reinterpret_cast<const unsigned long long*>(q) + 2);
      s_m[n].slot = (int)(unsigned)(w1 & 0xffffffffu);
      s_root[n] = (int)(unsigned)(w1 >> 32);
      s_m[n].gen = (unsigned)(w2 & 0xffffffffu);
      atomicExch(&japp::serve_done()[s_m[n].slot], 0u);
      atomicAdd(&japp::serve_ctr()[0], 1ULL);
      s.next++;
      n++;
    }
    __threadfence();
    s_n = n;
    // 1: the host asked to stop and nothing is in flight; 2: the run is
    // ending anyway (an error elsewhere, or past its deadline)
    s_stop = n == 0 && ld_sys_s32(japp::serve_ctl()) != 0 &&
             ld_relaxed_u64(&japp::serve_ctr()[0]) == 0;
    if (terminated()) {
      s_stop = 2;
    } else if (past_deadline()) {
      set_error(CHARMING_ERR_DEADLINE, 2, 0);
      s_stop = 2;
    }
  }
  __syncthreads();
  const int n = s_n, stop = s_stop;
  for (int k = 0; k < n; k++) {
    jac::start_msg m = s_m[k];
    jproxy->invoke(s_root[k], EP_START, &m, sizeof(m));
  }
  __syncthreads();
  if (stop) {
    if (stop == 1) charm::end();
    return;
  }
  sproxy->invoke(0, EP_POLL);
}

__device__ void em_start(JBlock& c, void* arg) {
  if (japp::dtype() == CHARMING_F32) em_start_t<float>(c, arg); else em_start_t<double>(c, arg);
}
__device__ void em_halo(JBlock& c, void* arg) {
  if (japp::dtype() == CHARMING_F32) em_halo_t<float>(c, arg); else em_halo_t<double>(c, arg);
}
__device__ void em_cont(JBlock& c, void* arg) {
  if (japp::dtype() == CHARMING_F32) em_cont_t<float>(c); else em_cont_t<double>(c);
}
__device__ void em_partial(JBlock& c, void* arg) {
  if (japp::dtype() == CHARMING_F32) em_partial_t<float>(c, arg); else em_partial_t<double>(c, arg);
}
__device__ void em_decision(JBlock& c, void* arg) {
  if (japp::dtype() == CHARMING_F32) em_decision_t<float>(c, arg); else em_decision_t<double>(c, arg);
}

}  // namespace

__device__ void suite::jacobi2d_main(int pe) {
  if (threadIdx.x == 0) {
    for (int k = 0; k < 6; k++) s_pe_ns[k] = 0;
    jproxy = new charm::chare_proxy<JBlock>();
    jproxy->add_entry_method<&em_start>();
    jproxy->add_entry_method<&em_halo>();
    jproxy->add_entry_method<&em_cont>();
    jproxy->add_entry_method<&em_partial>();
    jproxy->add_entry_method<&em_decision>();
    jproxy->create(japp::n_chares(), const_cast<int*>(japp::block_map()));
    if (!japp::serving()) {
      // each chare keeps its own descriptors (serving workers copy theirs
      // per request)
      for (int i = jproxy->start_idx; i <= jproxy->end_idx && jproxy->n_local > 0; i++) {
        JBlock* c = jproxy->local(i);
        if (!c) continue;
        c->desc = japp::chares()[i];
        c->prob = japp::probs()[c->desc.prob];
      }
    }
    if (japp::serving()) {
      sproxy = new charm::chare_proxy<JServer>();
      sproxy->add_entry_method<&em_poll>();
      sproxy->create(1, const_cast<int*>(japp::server_map()));
    }
  }
  __syncthreads();
  if (japp::serving()) {
    if (pe == 0) sproxy->invoke(0, EP_POLL);
  } else if (jproxy->n_local > 0) {
    for (int i = jproxy->start_idx; i <= jproxy->end_idx; i++) jproxy->invoke(i, EP_START);
  }
}
