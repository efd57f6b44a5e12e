// Jacobi2d solve server: C ABI charming_serve_*.
//
// One long-lived scheduler launch runs a pool of worker chares (the
// Jacobi2d chares of jacobi2d.cu in serving mode) and a server chare on
// PE 0. The host side (serve_host.h) admits requests against an HBM budget,
// decomposes each into chares bound to free workers, writes their
// descriptors into staging tables in mapped host memory and posts the
// request into a ring there; the server chare starts it. Requests admitted
// while others run share the PEs with them (continuous batching). The last
// chare of a request writes a completion record into a second mapped ring,
// which charming_serve_poll reads; the grids stay in HBM until
// charming_serve_release, and charming_serve_fetch copies one out with the
// copy engine while the scheduler keeps running.
#include <chrono>
#include <cstring>
#include <thread>
#include <vector>

#include "suite.cuh"
#include "jacobi_types.cuh"
#include "jacobi_sweep.cuh"
#include "serve_host.h"
#include "../host.cuh"

__device__ void suite::serve_main(int pe) {
  // the server runs inside the Jacobi2d program (g_app.a[6] != 0)
  if (threadIdx.x == 0 && pe == 0) charm::end();
}

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

template <typename T>
T* host_mapped(size_t n, cudaError_t* e) {
  void* p = nullptr;
  if (*e == cudaSuccess) *e = cudaHostAlloc(&p, n * sizeof(T) + 64, cudaHostAllocMapped);
  if (*e == cudaSuccess) memset(p, 0, n * sizeof(T) + 64);
  return reinterpret_cast<T*>(p);
}

struct Server : jserve::sink {
  jserve::server_state st;
  charming_serve_config cfg{};
  int n_workers = 0, Q = 0, CQ = 0;
  size_t esz = 4;
  int off_el = 32;
  // device
  char* d_slab = nullptr;
  unsigned long long* d_ctr = nullptr;
  unsigned int* d_done = nullptr;
  int* d_block_map = nullptr;
  int* d_server_map = nullptr;
  int* d_final = nullptr;
  unsigned long long* d_pe_ns = nullptr;
  // mapped host memory
  jac::serve_req* h_req = nullptr;
  jac::chare_desc* h_desc = nullptr;
  jac::prob_desc* h_prob = nullptr;
  jac::serve_comp* h_comp = nullptr;
  int* h_ctl = nullptr;
  suite::app_params* h_params = nullptr;
  unsigned long long req_ticket = 0, comp_next = 0;
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int run_status = CHARMING_OK;
  bool launched = false, ended = false;

  void stage_desc(int w, const jac::chare_desc& d) override { h_desc[w] = d; }
  void stage_prob(int slot, const jac::prob_desc& p) override { h_prob[slot] = p; }
  void post(int slot, int root, unsigned gen) override {
    jac::serve_req* r = h_req + req_ticket % (unsigned long long)Q;
    r->slot = slot;
    r->root = root;
    r->gen = gen;
    __atomic_store_n(&r->seq, req_ticket + 1, __ATOMIC_RELEASE);
    req_ticket++;
  }

  // The scheduler launch ended (normally only after stop): its status.
  int check_running() {
    if (ended) return run_status;
    cudaError_t q = cudaEventQuery(ev1);
    if (q == cudaErrorNotReady) return CHARMING_OK;
    ended = true;
    float ms = 0.f;
    if (q == cudaSuccess) cudaEventElapsedTime(&ms, ev0, ev1);
    run_status = q == cudaSuccess ? charm_host::collect_run(ms) : charm_host::cuda_fail(q, "serve run");
    if (run_status == CHARMING_OK) run_status = CHARMING_ERR_CONFIG;  // ended before stop
    return run_status;
  }

  // Reads ready completion records (at most max_n into out, if given).
  int drain(charming_serve_completion* out, int max_n) {
    int k = 0;
    while (!out || k < max_n) {
      jac::serve_comp* r = h_comp + comp_next % (unsigned long long)CQ;
      if (__atomic_load_n(&r->seq, __ATOMIC_ACQUIRE) != comp_next + 1) break;
      jac::serve_comp c = *r;
      comp_next++;
      jserve::admitted* a = st.complete(c, now_s());
      if (!a) {
        charm_host::set_error_text("serve: completion record of no request");
        return -CHARMING_ERR_APP;
      }
      if (out) {
        charming_serve_completion& o = out[k];
        o.tag = a->tag;
        o.status = c.status;
        o.sweeps = c.sweeps;
        o.res0 = c.res0;
        o.res_last = c.res_last;
        o.submit_s = a->submit_s;
        o.admit_s = a->admit_s;
        o.done_s = a->done_s;
      }
      k++;
    }
    return k;
  }

  int admit() {
    int n = st.admit(*this, now_s());
    if (n < 0) {
      charm_host::set_error_text(st.err);
      return CHARMING_ERR_CONFIG;
    }
    return CHARMING_OK;
  }

  void free_all() {
    cudaFree(d_slab);
    cudaFree(d_ctr);
    cudaFree(d_done);
    cudaFree(d_block_map);
    cudaFree(d_server_map);
    cudaFree(d_final);
    cudaFree(d_pe_ns);
    cudaFreeHost(h_req);
    cudaFreeHost(h_desc);
    cudaFreeHost(h_prob);
    cudaFreeHost(h_comp);
    cudaFreeHost(h_ctl);
    cudaFreeHost(h_params);
    if (copy_stream) cudaStreamDestroy(copy_stream);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
  }
};

Server* g_server = nullptr;  // one server at a time (it holds every PE)

int fail(int code, const char* msg) {
  charm_host::set_error_text(msg);
  return code;
}

}  // namespace

extern "C" int charming_serve_start(const charming_serve_config* cfg, void** server) {
  int rc = charm_host::ensure_init();
  if (rc) return rc;
  if (!cfg || !server) return fail(CHARMING_ERR_CONFIG, "serve: bad arguments");
  if (g_server) return fail(CHARMING_ERR_CONFIG, "serve: a server is already running");
  if (cfg->dtype != CHARMING_F32 && cfg->dtype != CHARMING_F64) return fail(CHARMING_ERR_CONFIG, "serve: dtype");
  if (cfg->max_inflight < 1 || cfg->workers_per_pe < 1 || cfg->hbm_budget_bytes < 4096 || cfg->deadline_s <= 0)
    return fail(CHARMING_ERR_CONFIG, "serve: config");
  const int n_pes = charm_host::info().n_pes;
  Server* s = new Server();
  s->cfg = *cfg;
  s->n_workers = n_pes * cfg->workers_per_pe;
  s->Q = s->CQ = cfg->max_inflight;
  const bool f64 = cfg->dtype == CHARMING_F64;
  s->esz = f64 ? 8 : 4;
  s->off_el = f64 ? jac::traits<double>::OFF : jac::traits<float>::OFF;
  jserve::params P;
  P.n_pes = n_pes;
  P.workers_per_pe = cfg->workers_per_pe;
  P.max_inflight = cfg->max_inflight;
  P.budget = cfg->hbm_budget_bytes;
  // default: large chares (fewer halo messages per point); requests far
  // apart in size still spread over many PEs because many run at once
  P.chare_side = cfg->chare_side > 0 ? cfg->chare_side : 2048;
  P.depth = 0;
  P.esz = (int)s->esz;
  P.off = s->off_el;
  P.vec = f64 ? jac::traits<double>::VEC : jac::traits<float>::VEC;

  cudaError_t e = cudaMalloc(&s->d_slab, cfg->hbm_budget_bytes);
  if (e == cudaSuccess) e = cudaMalloc(&s->d_ctr, 128);
  if (e == cudaSuccess) e = cudaMalloc(&s->d_done, sizeof(unsigned) * s->Q);
  if (e == cudaSuccess) e = cudaMalloc(&s->d_block_map, sizeof(int) * n_pes);
  if (e == cudaSuccess) e = cudaMalloc(&s->d_server_map, sizeof(int) * n_pes);
  if (e == cudaSuccess) e = cudaMalloc(&s->d_final, sizeof(int) * s->n_workers);
  if (e == cudaSuccess) e = cudaMalloc(&s->d_pe_ns, 64 * (size_t)n_pes);
  if (e == cudaSuccess) e = cudaMemset(s->d_ctr, 0, 128);
  if (e == cudaSuccess) e = cudaMemset(s->d_done, 0, sizeof(unsigned) * s->Q);
  if (e == cudaSuccess) e = cudaMemset(s->d_pe_ns, 0, 64 * (size_t)n_pes);
  s->h_req = host_mapped<jac::serve_req>(s->Q, &e);
  s->h_desc = host_mapped<jac::chare_desc>(s->n_workers, &e);
  s->h_prob = host_mapped<jac::prob_desc>(s->Q, &e);
  s->h_comp = host_mapped<jac::serve_comp>(s->CQ, &e);
  s->h_ctl = host_mapped<int>(32, &e);
  if (e == cudaSuccess) e = cudaHostAlloc(&s->h_params, sizeof(suite::app_params), cudaHostAllocDefault);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&s->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&s->ev1);
  if (e == cudaSuccess) {
    std::vector<int> bm(n_pes, cfg->workers_per_pe), sm(n_pes, 0);
    sm[0] = 1;
    e = cudaMemcpy(s->d_block_map, bm.data(), sizeof(int) * n_pes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(s->d_server_map, sm.data(), sizeof(int) * n_pes, cudaMemcpyHostToDevice);
  }
  if (e != cudaSuccess) {
    rc = charm_host::cuda_fail(e, "serve: allocation");
    s->free_all();
    delete s;
    return rc;
  }
  s->st.init(P, reinterpret_cast<uintptr_t>(s->d_slab));

  suite::app_params& ap = *s->h_params;
  memset(&ap, 0, sizeof(ap));
  ap.id = suite::APP_JACOBI2D;
  ap.a[0] = s->n_workers;
  ap.a[2] = cfg->dtype;
  ap.a[6] = 1;
  ap.a[7] = s->Q;
  ap.a[8] = s->CQ;
  // p[0], p[1] (descriptor tables) stay null: each worker copies its
  // descriptors from the staging tables into its own chare object
  ap.p[4] = s->d_final;
  ap.p[5] = s->d_block_map;
  ap.p[6] = s->d_pe_ns;
  ap.p[7] = s->h_req;
  ap.p[8] = s->h_desc;
  ap.p[9] = s->h_prob;
  ap.p[10] = s->h_comp;
  ap.p[11] = s->d_ctr;
  ap.p[12] = s->d_done;
  ap.p[13] = s->h_ctl;
  ap.p[14] = s->d_server_map;

  rc = charm_host::set_deadline(cfg->deadline_s);
  cudaStream_t st = charm_host::stream();
  charm_host::request_stop(0);
  if (rc == CHARMING_OK) {
    e = cudaMemcpyToSymbolAsync(g_app, s->h_params, sizeof(suite::app_params), 0, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaEventRecord(s->ev0, st);
    rc = charm_host::cuda_fail(e, "serve: launch setup");
  }
  if (rc == CHARMING_OK) rc = charm_host::enqueue_scheduler(st);
  if (rc == CHARMING_OK) rc = charm_host::cuda_fail(cudaEventRecord(s->ev1, st), "serve: launch");
  if (rc != CHARMING_OK) {
    cudaStreamSynchronize(st);
    charm_host::set_deadline(-1.0);
    s->free_all();
    delete s;
    return rc;
  }
  s->launched = true;
  g_server = s;
  *server = s;
  return CHARMING_OK;
}

extern "C" int charming_serve_submit(void* server, const charming_jacobi_problem* req, uint64_t tag) {
  Server* s = reinterpret_cast<Server*>(server);
  if (!s || s != g_server || !req) return fail(CHARMING_ERR_CONFIG, "serve: bad arguments");
  int rc = s->check_running();
  if (rc) return rc;
  rc = s->st.submit(*req, tag, now_s());
  if (rc) return fail(rc, s->st.err.c_str());
  return s->admit();
}

extern "C" int charming_serve_poll(void* server, charming_serve_completion* out, int max_n, int* n_out) {
  Server* s = reinterpret_cast<Server*>(server);
  if (!s || s != g_server || (max_n > 0 && !out) || !n_out) return fail(CHARMING_ERR_CONFIG, "serve: bad arguments");
  *n_out = 0;
  int k = s->drain(out, max_n);
  if (k < 0) return -k;
  *n_out = k;
  int rc = s->admit();
  if (rc) return rc;
  return k > 0 ? CHARMING_OK : s->check_running();
}

extern "C" int charming_serve_fetch(void* server, uint64_t tag, void* host_grid) {
  Server* s = reinterpret_cast<Server*>(server);
  if (!s || s != g_server || !host_grid) return fail(CHARMING_ERR_CONFIG, "serve: bad arguments");
  jserve::admitted* a = s->st.find(tag);
  if (!a || !a->done) return fail(CHARMING_ERR_CONFIG, "serve: no completed request with this tag");
  const charming_jacobi_problem& q = a->prob;
  const size_t es = s->esz, row = (size_t)(q.nx + 2) * es;
  char* g = reinterpret_cast<char*>(host_grid);
  // interior of each chare from its final buffer (copy engine: the
  // scheduler keeps running)
  cudaError_t e = cudaSuccess;
  for (const jac::chare_desc& d : a->chares) {
    const char* src = reinterpret_cast<const char*>(d.buf[a->comp.final_buf]) +
                      ((size_t)d.pitch + s->off_el) * es;
    char* dst = g + (size_t)(d.y0 + 1) * row + (size_t)(d.x0 + 1) * es;
    e = cudaMemcpy2DAsync(dst, row, src, (size_t)d.pitch * es, (size_t)d.w * es, d.h, cudaMemcpyDeviceToHost,
                          s->copy_stream);
    if (e != cudaSuccess) break;
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->copy_stream);
  if (e != cudaSuccess) return charm_host::cuda_fail(e, "serve: fetch");
  // the fixed boundary ring, as the workers wrote it
  auto put = [&](int gy, int gx, double v) {
    char* p = g + (size_t)gy * row + (size_t)gx * es;
    if (es == 8) memcpy(p, &v, 8);
    else {
      float f = (float)v;
      memcpy(p, &f, 4);
    }
  };
  for (int gy = 1; gy <= q.ny; gy++) {
    put(gy, 0, q.bc[2]);
    put(gy, q.nx + 1, q.bc[3]);
  }
  for (int gx = 0; gx <= q.nx + 1; gx++) {
    put(0, gx, q.bc[0]);
    put(q.ny + 1, gx, q.bc[1]);
  }
  return CHARMING_OK;
}

extern "C" int charming_serve_release(void* server, uint64_t tag) {
  Server* s = reinterpret_cast<Server*>(server);
  if (!s || s != g_server) return fail(CHARMING_ERR_CONFIG, "serve: bad arguments");
  int rc = s->st.release(tag);
  if (rc) return fail(rc, s->st.err.c_str());
  return s->admit();
}

// Stops admitting, waits (within the run deadline) for the requests in
// flight, lets the server chare end the run, and frees everything. Pending
// requests that were never admitted are dropped.
extern "C" int charming_serve_stop(void* server, charming_serve_stats* stats) {
  Server* s = reinterpret_cast<Server*>(server);
  if (!s || s != g_server) return fail(CHARMING_ERR_CONFIG, "serve: bad arguments");
  int rc = CHARMING_OK;
  const double t_end = now_s() + s->cfg.deadline_s;
  while (s->st.inflight > 0 && !s->ended && now_s() < t_end) {
    int k = s->drain(nullptr, 0);
    if (k < 0) {
      rc = -k;
      break;
    }
    if (k == 0) {
      if (s->check_running()) break;
      std::this_thread::sleep_for(std::chrono::microseconds(200));
    }
  }
  __atomic_store_n(s->h_ctl, 1, __ATOMIC_RELEASE);
  cudaError_t e = cudaStreamSynchronize(charm_host::stream());
  if (!s->ended) {
    s->ended = true;
    float ms = 0.f;
    if (e == cudaSuccess) cudaEventElapsedTime(&ms, s->ev0, s->ev1);
    s->run_status = e == cudaSuccess ? charm_host::collect_run(ms) : charm_host::cuda_fail(e, "serve run");
  }
  if (rc == CHARMING_OK) rc = s->run_status;
  if (rc == CHARMING_OK && s->st.inflight > 0) rc = fail(CHARMING_ERR_DEADLINE, "serve: requests still in flight at stop");
  if (stats) {
    stats->submitted = s->st.n_submitted;
    stats->admitted = s->st.n_admitted;
    stats->completed = s->st.n_completed;
    stats->peak_bytes = s->st.mem.peak();
    stats->peak_inflight = s->st.peak_inflight;
    float ms = 0.f;
    if (e == cudaSuccess) cudaEventElapsedTime(&ms, s->ev0, s->ev1);
    stats->busy_s = ms * 1e-3;
  }
  charm_host::set_deadline(-1.0);
  s->free_all();
  g_server = nullptr;
  delete s;
  return rc;
}
