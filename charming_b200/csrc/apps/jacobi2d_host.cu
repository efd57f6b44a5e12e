// Host side of the Jacobi2d program: decomposition into chares, placement on
// PEs, chare grids in HBM, init/load/store kernels and the run (optionally
// replayed from a captured CUDA graph). C ABI: charming_jacobi2d_*.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <queue>
#include <vector>
#include "suite.cuh"
#include "jacobi_types.cuh"
#include "jacobi_sweep.cuh"
#include "jacobi_layout.h"
#include "../host.cuh"

namespace {

struct JHandle {
  std::vector<charming_jacobi_problem> probs;
  charming_jacobi_options opt{};
  int n_chares = 0;
  size_t esz = 8;
  std::vector<jac::chare_desc> chares;     // placed order
  std::vector<int> block_map;              // chares per PE
  std::vector<int> chare_of;               // [prob offset + cy*px + cx] -> chare
  std::vector<size_t> chare_of_off;
  std::vector<int> px, py;
  jac::chare_desc* d_chares = nullptr;
  jac::prob_desc* d_probs = nullptr;
  jac::prob_result* d_results = nullptr;
  unsigned long long* d_done = nullptr;
  int* d_final = nullptr;
  int* d_block_map = nullptr;
  int* d_chare_of = nullptr;
  unsigned long long* d_sweep_ns = nullptr;
  char* d_grid = nullptr;
  size_t grid_bytes = 0;
  void* d_stage = nullptr;
  size_t stage_bytes = 0;
  // charming_jacobi2d_solve_stream: two input and two output staging
  // buffers, copy streams and their events
  void* d_pipe = nullptr;
  size_t pipe_bytes = 0;
  int* d_latch = nullptr;
  cudaStream_t s_h2d = nullptr, s_d2h = nullptr;
  cudaEvent_t in_ready[2] = {}, in_free[2] = {}, out_ready[2] = {}, out_free[2] = {};
  suite::app_params* h_params = nullptr;   // pinned
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double last_ms = 0.0;
  int max_per_pe = 0;
  uint64_t points = 0, halo_msgs = 0;
};

template <typename T>
__device__ __forceinline__ T* cell(const jac::chare_desc& d, int b, int r, int c) {
  return reinterpret_cast<T*>(d.buf[b]) + (size_t)r * d.pitch + jac::traits<T>::OFF - 1 + c;
}

// Initial state: boundary ring from bc (top/bottom rows include the corners),
// interior 0; written to both buffers over the whole ghost zone wherever the
// position lies on the global grid (ghost cells on the domain boundary must
// hold boundary values for the multi-sweep pass). One block per chare.
template <typename T>
__global__ void init_kernel(const jac::chare_desc* ch, const jac::prob_desc* pr, const double* bc) {
  const jac::chare_desc d = ch[blockIdx.x];
  const jac::prob_desc p = pr[d.prob];
  const double* b = bc + 4 * d.prob;
  const int D = d.depth, W = d.w + 2 * D;
  long long n = (long long)(d.h + 2 * D) * W;
  for (long long x = threadIdx.x; x < n; x += blockDim.x) {
    int r = (int)(x / W) + 1 - D, c = (int)(x % W) + 1 - D;
    int gy = d.y0 + r, gx = d.x0 + c;
    if (gy < 0 || gy > p.ny + 1 || gx < 0 || gx > p.nx + 1) continue;
    double v = 0.0;
    if (gy == 0) v = b[0];
    else if (gy == p.ny + 1) v = b[1];
    else if (gx == 0) v = b[2];
    else if (gx == p.nx + 1) v = b[3];
    *cell<T>(d, 0, r, c) = (T)v;
    *cell<T>(d, 1, r, c) = (T)v;
  }
}

// Global grid (ny+2) x (nx+2) in `stage` -> blocks of one problem (whole
// ghost zone, as init_kernel).
template <typename T>
__global__ void scatter_kernel(const jac::chare_desc* ch, const int* chare_of, int nx, int ny,
    const T* stage) {
  const jac::chare_desc d = ch[chare_of[blockIdx.x]];
  const int D = d.depth, W = d.w + 2 * D;
  long long n = (long long)(d.h + 2 * D) * W;
  for (long long x = threadIdx.x; x < n; x += blockDim.x) {
    int r = (int)(x / W) + 1 - D, c = (int)(x % W) + 1 - D;
    int gy = d.y0 + r, gx = d.x0 + c;
    if (gy < 0 || gy > ny + 1 || gx < 0 || gx > nx + 1) continue;
    T v = stage[(size_t)gy * (nx + 2) + gx];
    *cell<T>(d, 0, r, c) = v;
    *cell<T>(d, 1, r, c) = v;
  }
}

// Blocks of one problem -> global grid: interior cells from their owner,
// ring cells from the ghost ring of the edge chare next to them.
template <typename T>
__global__ void gather_kernel(const jac::chare_desc* ch, const int* chare_of, const int* final_buf,
    int nx, int ny, int px, int py, T* stage) {
  long long n = (long long)(nx + 2) * (ny + 2);
  for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < n;
       x += (long long)gridDim.x * blockDim.x) {
    int gy = (int)(x / (nx + 2)), gx = (int)(x % (nx + 2));
    int iy = min(max(gy - 1, 0), ny - 1), ix = min(max(gx - 1, 0), nx - 1);
    int cy = jac::split_owner(ny, py, iy), cx = jac::split_owner(nx, px, ix);
    int k = chare_of[cy * px + cx];
    const jac::chare_desc& d = ch[k];
    stage[x] = *cell<T>(d, final_buf[k], gy - d.y0, gx - d.x0);
  }
}

int fail(int code, const char* msg) {
  charm_host::set_error_text(msg);
  return code;
}

int check_cuda(cudaError_t e, const char* what) { return charm_host::cuda_fail(e, what); }

}  // namespace

extern "C" int charming_jacobi2d_create(const charming_jacobi_problem* probs, int n,
    const charming_jacobi_options* opt, void** handle) {
  int rc = charm_host::ensure_init();
  if (rc) return rc;
  if (!probs || n <= 0 || !opt || !handle) return fail(CHARMING_ERR_CONFIG, "jacobi2d: bad arguments");
  if (opt->dtype != CHARMING_F64 && opt->dtype != CHARMING_F32)
    return fail(CHARMING_ERR_CONFIG, "jacobi2d: dtype");
  const int n_pes = charm_host::info().n_pes;
  JHandle* h = new JHandle();
  h->probs.assign(probs, probs + n);
  h->opt = *opt;
  h->esz = opt->dtype == CHARMING_F64 ? 8 : 4;
  const int V = opt->dtype == CHARMING_F64 ? jac::traits<double>::VEC : jac::traits<float>::VEC;
  const int OFF = opt->dtype == CHARMING_F64 ? jac::traits<double>::OFF : jac::traits<float>::OFF;

  // decomposition, tree, neighbours, placement, grid offsets
  jac::layout L;
  std::string err;
  if (!jac::build_layout(probs, n, opt->chare_side, opt->balance, opt->depth, opt->pipeline, n_pes,
                         (int)h->esz, OFF, V, &L, &err)) {
    delete h;
    return fail(CHARMING_ERR_CONFIG, err.c_str());
  }
  const int nch = (int)L.chares.size();
  h->n_chares = nch;
  h->px = L.px;
  h->py = L.py;
  h->block_map = L.block_map;
  h->chare_of = L.chare_of;
  h->chare_of_off = L.chare_of_off;
  h->max_per_pe = L.max_per_pe;
  h->points = L.points;
  h->halo_msgs = L.halo_msgs;
  h->grid_bytes = L.total_bytes;
  std::vector<jac::prob_desc>& pd = L.probs;
  cudaError_t e = cudaMalloc(&h->d_grid, L.total_bytes);
  if (e != cudaSuccess) {
    delete h;
    return charm_host::cuda_fail(e, "jacobi2d grids");
  }
  // zero everything once: ghost cells beyond the boundary ring are read
  // (never used) by the multi-sweep pass
  e = cudaMemset(h->d_grid, 0, L.total_bytes);
  if (e != cudaSuccess) {
    cudaFree(h->d_grid);
    delete h;
    return charm_host::cuda_fail(e, "jacobi2d grids");
  }
  jac::place_buffers(&L, h->d_grid, (int)h->esz);
  h->chares = L.chares;
  e = cudaMalloc(&h->d_chares, sizeof(jac::chare_desc) * nch);
  if (e == cudaSuccess) e = cudaMalloc(&h->d_probs, sizeof(jac::prob_desc) * n);
  if (e == cudaSuccess) e = cudaMalloc(&h->d_results, sizeof(jac::prob_result) * n);
  if (e == cudaSuccess) e = cudaMalloc(&h->d_done, 64);
  if (e == cudaSuccess) e = cudaMalloc(&h->d_final, sizeof(int) * nch);
  if (e == cudaSuccess) e = cudaMalloc(&h->d_block_map, sizeof(int) * n_pes);
  if (e == cudaSuccess) e = cudaMalloc(&h->d_chare_of, sizeof(int) * h->chare_of.size());
  if (e == cudaSuccess) e = cudaMalloc(&h->d_sweep_ns, 64 * (size_t)n_pes);
  if (e == cudaSuccess) e = cudaMemcpy(h->d_chares, h->chares.data(), sizeof(jac::chare_desc) * nch, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(h->d_probs, pd.data(), sizeof(jac::prob_desc) * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(h->d_results, 0, sizeof(jac::prob_result) * n);
  if (e == cudaSuccess) e = cudaMemset(h->d_final, 0, sizeof(int) * nch);
  if (e == cudaSuccess) e = cudaMemcpy(h->d_block_map, h->block_map.data(), sizeof(int) * n_pes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(h->d_chare_of, h->chare_of.data(), sizeof(int) * h->chare_of.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaHostAlloc(&h->h_params, sizeof(suite::app_params), cudaHostAllocDefault);
  if (e == cudaSuccess) e = cudaEventCreate(&h->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&h->ev1);
  if (e != cudaSuccess) {
    rc = charm_host::cuda_fail(e, "jacobi2d descriptors");
    charming_jacobi2d_destroy(h);
    return rc;
  }
  suite::app_params& ap = *h->h_params;
  memset(&ap, 0, sizeof(ap));
  ap.id = suite::APP_JACOBI2D;
  ap.a[0] = nch;
  ap.a[1] = n;
  ap.a[2] = opt->dtype;
  ap.a[3] = opt->pipeline;
  ap.a[4] = opt->tile_w;
  ap.a[5] = opt->halo_mode;
  // CHARMING_DEEP_CHAINED=1: multi-sweep passes on the single-loop items
  // (the phase-split ones are the default; both give the same bits)
  ap.a[9] = getenv("CHARMING_DEEP_CHAINED") && atoi(getenv("CHARMING_DEEP_CHAINED")) ? 1 : 0;
  ap.p[0] = h->d_chares;
  ap.p[1] = h->d_probs;
  ap.p[2] = h->d_results;
  ap.p[3] = h->d_done;
  ap.p[4] = h->d_final;
  ap.p[5] = h->d_block_map;
  ap.p[6] = h->d_sweep_ns;
  *handle = h;
  return charming_jacobi2d_init(h);
}

extern "C" int charming_jacobi2d_init(void* handle) {
  JHandle* h = reinterpret_cast<JHandle*>(handle);
  if (!h) return CHARMING_ERR_CONFIG;
  int n = (int)h->probs.size();
  std::vector<double> bc(4 * n);
  for (int p = 0; p < n; p++)
    for (int k = 0; k < 4; k++) bc[4 * p + k] = h->probs[p].bc[k];
  double* d_bc = nullptr;
  cudaError_t e = cudaMalloc(&d_bc, sizeof(double) * bc.size());
  if (e == cudaSuccess) e = cudaMemcpy(d_bc, bc.data(), sizeof(double) * bc.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    if (h->esz == 8) init_kernel<double><<<h->n_chares, 256>>>(h->d_chares, h->d_probs, d_bc);
    else init_kernel<float><<<h->n_chares, 256>>>(h->d_chares, h->d_probs, d_bc);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  cudaFree(d_bc);
  if (e == cudaSuccess) e = cudaMemset(h->d_final, 0, sizeof(int) * h->n_chares);
  return check_cuda(e, "jacobi2d init");
}

static int ensure_stage(JHandle* h, size_t bytes) {
  if (h->stage_bytes >= bytes) return CHARMING_OK;
  if (h->d_stage) cudaFree(h->d_stage);
  h->d_stage = nullptr;
  h->stage_bytes = 0;
  cudaError_t e = cudaMalloc(&h->d_stage, bytes);
  if (e != cudaSuccess) return check_cuda(e, "jacobi2d staging buffer");
  h->stage_bytes = bytes;
  return CHARMING_OK;
}

extern "C" int charming_jacobi2d_load(void* handle, int prob, const void* host_grid) {
  JHandle* h = reinterpret_cast<JHandle*>(handle);
  if (!h || prob < 0 || prob >= (int)h->probs.size() || !host_grid) return CHARMING_ERR_CONFIG;
  const charming_jacobi_problem& q = h->probs[prob];
  size_t bytes = (size_t)(q.nx + 2) * (q.ny + 2) * h->esz;
  int rc = ensure_stage(h, bytes);
  if (rc) return rc;
  cudaStream_t s = charm_host::stream();
  cudaError_t e = cudaMemcpyAsync(h->d_stage, host_grid, bytes, cudaMemcpyHostToDevice, s);
  int nc = h->px[prob] * h->py[prob];
  const int* co = h->d_chare_of + h->chare_of_off[prob];
  if (e == cudaSuccess) {
    if (h->esz == 8) scatter_kernel<double><<<nc, 256, 0, s>>>(h->d_chares, co, q.nx, q.ny, (const double*)h->d_stage);
    else scatter_kernel<float><<<nc, 256, 0, s>>>(h->d_chares, co, q.nx, q.ny, (const float*)h->d_stage);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemsetAsync(h->d_final, 0, sizeof(int) * h->n_chares, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  return check_cuda(e, "jacobi2d load");
}

extern "C" int charming_jacobi2d_store(void* handle, int prob, void* host_grid) {
  JHandle* h = reinterpret_cast<JHandle*>(handle);
  if (!h || prob < 0 || prob >= (int)h->probs.size() || !host_grid) return CHARMING_ERR_CONFIG;
  const charming_jacobi_problem& q = h->probs[prob];
  size_t cells = (size_t)(q.nx + 2) * (q.ny + 2);
  size_t bytes = cells * h->esz;
  int rc = ensure_stage(h, bytes);
  if (rc) return rc;
  cudaStream_t s = charm_host::stream();
  const int* co = h->d_chare_of + h->chare_of_off[prob];
  int blocks = (int)std::min<size_t>((cells + 255) / 256, 4096);
  if (h->esz == 8)
    gather_kernel<double><<<blocks, 256, 0, s>>>(h->d_chares, co, h->d_final, q.nx, q.ny,
        h->px[prob], h->py[prob], (double*)h->d_stage);
  else
    gather_kernel<float><<<blocks, 256, 0, s>>>(h->d_chares, co, h->d_final, q.nx, q.ny,
        h->px[prob], h->py[prob], (float*)h->d_stage);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(host_grid, h->d_stage, bytes, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  return check_cuda(e, "jacobi2d store");
}

// Work of one run on stream s: counters, program parameters, scheduler.
static int enqueue_run(JHandle* h, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(h->d_done, 0, 64, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->d_results, 0, sizeof(jac::prob_result) * h->probs.size(), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->d_sweep_ns, 0, 64 * h->block_map.size(), s);
  if (e == cudaSuccess)
    e = cudaMemcpyToSymbolAsync(g_app, h->h_params, sizeof(suite::app_params), 0,
                                cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return check_cuda(e, "jacobi2d run setup");
  return charm_host::enqueue_scheduler(s);
}

extern "C" int charming_jacobi2d_run(void* handle) {
  JHandle* h = reinterpret_cast<JHandle*>(handle);
  if (!h) return CHARMING_ERR_CONFIG;
  cudaStream_t s = charm_host::stream();
  charm_host::request_stop(0);
  int rc;
  cudaError_t e;
  if (h->opt.use_graph) {
    if (!h->graph_exec) {
      e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
      if (e != cudaSuccess) return check_cuda(e, "graph capture begin");
      rc = enqueue_run(h, s);
      e = cudaStreamEndCapture(s, &h->graph);
      if (rc) return rc;
      if (e != cudaSuccess) return check_cuda(e, "graph capture end");
      e = cudaGraphInstantiate(&h->graph_exec, h->graph, 0);
      if (e != cudaSuccess) return check_cuda(e, "graph instantiate");
    }
    cudaEventRecord(h->ev0, s);
    e = cudaGraphLaunch(h->graph_exec, s);
    if (e != cudaSuccess) return check_cuda(e, "graph launch");
    cudaEventRecord(h->ev1, s);
  } else {
    cudaEventRecord(h->ev0, s);
    rc = enqueue_run(h, s);
    if (rc) return rc;
    cudaEventRecord(h->ev1, s);
  }
  e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return check_cuda(e, "jacobi2d run");
  float ms = 0.f;
  cudaEventElapsedTime(&ms, h->ev0, h->ev1);
  h->last_ms = ms;
  return charm_host::collect_run(ms);
}

extern "C" int charming_jacobi2d_run_n(void* handle, int n_runs, double* total_ms) {
  JHandle* h = reinterpret_cast<JHandle*>(handle);
  if (!h || n_runs < 1) return CHARMING_ERR_CONFIG;
  cudaStream_t s = charm_host::stream();
  charm_host::request_stop(0);
  cudaError_t e = cudaSuccess;
  if (!h->d_latch) e = cudaMalloc(&h->d_latch, 4 * sizeof(int));
  if (e == cudaSuccess) e = cudaMemsetAsync(h->d_latch, 0, 4 * sizeof(int), s);
  if (e == cudaSuccess) e = cudaEventRecord(h->ev0, s);
  if (e != cudaSuccess) return check_cuda(e, "jacobi2d runs");
  int rc;
  for (int k = 0; k < n_runs; k++) {
    if (h->opt.use_graph && h->graph_exec) {
      e = cudaGraphLaunch(h->graph_exec, s);
      if (e != cudaSuccess) return check_cuda(e, "graph launch");
    } else if ((rc = enqueue_run(h, s))) {
      return rc;
    }
    if ((rc = charm_host::enqueue_status_latch(h->d_latch, s))) return rc;
  }
  e = cudaEventRecord(h->ev1, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return check_cuda(e, "jacobi2d runs");
  float ms = 0.f;
  cudaEventElapsedTime(&ms, h->ev0, h->ev1);
  if (total_ms) *total_ms = ms;
  h->last_ms = ms / n_runs;
  int latch[4] = {0, 0, 0, 0};
  e = cudaMemcpy(latch, h->d_latch, sizeof(latch), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return check_cuda(e, "jacobi2d run status");
  rc = charm_host::collect_run(h->last_ms);
  return latch[0] ? latch[0] : rc;
}

// Device-side work of load (staged grid -> chare blocks) and store (chare
// blocks -> staged grid) on stream s, without the host copies.
static void enqueue_scatter(JHandle* h, int prob, const void* stage, cudaStream_t s) {
  const charming_jacobi_problem& q = h->probs[prob];
  const int nc = h->px[prob] * h->py[prob];
  const int* co = h->d_chare_of + h->chare_of_off[prob];
  if (h->esz == 8) scatter_kernel<double><<<nc, 256, 0, s>>>(h->d_chares, co, q.nx, q.ny, (const double*)stage);
  else scatter_kernel<float><<<nc, 256, 0, s>>>(h->d_chares, co, q.nx, q.ny, (const float*)stage);
}
static void enqueue_gather(JHandle* h, int prob, void* stage, cudaStream_t s) {
  const charming_jacobi_problem& q = h->probs[prob];
  const size_t cells = (size_t)(q.nx + 2) * (q.ny + 2);
  const int* co = h->d_chare_of + h->chare_of_off[prob];
  const int blocks = (int)std::min<size_t>((cells + 255) / 256, 4096);
  if (h->esz == 8)
    gather_kernel<double><<<blocks, 256, 0, s>>>(h->d_chares, co, h->d_final, q.nx, q.ny, h->px[prob],
                                                 h->py[prob], (double*)stage);
  else
    gather_kernel<float><<<blocks, 256, 0, s>>>(h->d_chares, co, h->d_final, q.nx, q.ny, h->px[prob],
                                                h->py[prob], (float*)stage);
}

static int ensure_pipe(JHandle* h, size_t bytes) {
  cudaError_t e = cudaSuccess;
  if (h->pipe_bytes < bytes) {
    if (h->d_pipe) cudaFree(h->d_pipe);
    h->d_pipe = nullptr;
    h->pipe_bytes = 0;
    e = cudaMalloc(&h->d_pipe, 4 * bytes);
    if (e != cudaSuccess) return check_cuda(e, "jacobi2d stream staging");
    h->pipe_bytes = bytes;
  }
  if (!h->d_latch) e = cudaMalloc(&h->d_latch, 4 * sizeof(int));
  if (e == cudaSuccess && !h->s_h2d) e = cudaStreamCreateWithFlags(&h->s_h2d, cudaStreamNonBlocking);
  if (e == cudaSuccess && !h->s_d2h) e = cudaStreamCreateWithFlags(&h->s_d2h, cudaStreamNonBlocking);
  for (int b = 0; b < 2 && e == cudaSuccess; b++) {
    if (!h->in_ready[b]) e = cudaEventCreateWithFlags(&h->in_ready[b], cudaEventDisableTiming);
    if (e == cudaSuccess && !h->in_free[b]) e = cudaEventCreateWithFlags(&h->in_free[b], cudaEventDisableTiming);
    if (e == cudaSuccess && !h->out_ready[b]) e = cudaEventCreateWithFlags(&h->out_ready[b], cudaEventDisableTiming);
    if (e == cudaSuccess && !h->out_free[b]) e = cudaEventCreateWithFlags(&h->out_free[b], cudaEventDisableTiming);
  }
  return check_cuda(e, "jacobi2d stream setup");
}

// n solves of problem prob, host_in[k] -> host_out[k], pipelined: the copy
// of solve k+1's input (one stream) and of solve k-1's result (another)
// overlap solve k on the runtime's stream, through two input and two
// output staging buffers on the device. Each solve is exactly load, run,
// store of that grid; the other problems of the handle are run too and left
// where they end. Returns the first failing run's status.
extern "C" int charming_jacobi2d_solve_stream(void* handle, int prob, int n, const void* const* host_in,
    void* const* host_out, double* out_ms) {
  JHandle* h = reinterpret_cast<JHandle*>(handle);
  if (!h || prob < 0 || prob >= (int)h->probs.size() || n < 0 || (n > 0 && (!host_in || !host_out)))
    return CHARMING_ERR_CONFIG;
  const charming_jacobi_problem& q = h->probs[prob];
  const size_t bytes = (size_t)(q.nx + 2) * (q.ny + 2) * h->esz;
  int rc = ensure_pipe(h, bytes);
  if (rc) return rc;
  char* stage_in[2] = {static_cast<char*>(h->d_pipe), static_cast<char*>(h->d_pipe) + bytes};
  char* stage_out[2] = {static_cast<char*>(h->d_pipe) + 2 * bytes, static_cast<char*>(h->d_pipe) + 3 * bytes};
  cudaStream_t s = charm_host::stream();
  charm_host::request_stop(0);
  cudaError_t e = cudaMemsetAsync(h->d_latch, 0, 4 * sizeof(int), s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaEventRecord(h->ev0, h->s_h2d);
  for (int k = 0; k < n && e == cudaSuccess; k++) {
    const int b = k & 1;
    // input k into stage_in[b] once solve k-2 has scattered it
    if (k >= 2) e = cudaStreamWaitEvent(h->s_h2d, h->in_free[b], 0);
    if (e == cudaSuccess) e = cudaMemcpyAsync(stage_in[b], host_in[k], bytes, cudaMemcpyHostToDevice, h->s_h2d);
    if (e == cudaSuccess) e = cudaEventRecord(h->in_ready[b], h->s_h2d);
    // solve k
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s, h->in_ready[b], 0);
    if (e == cudaSuccess) {
      enqueue_scatter(h, prob, stage_in[b], s);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaEventRecord(h->in_free[b], s);
    if (e == cudaSuccess) e = cudaMemsetAsync(h->d_final, 0, sizeof(int) * h->n_chares, s);
    if (e != cudaSuccess) break;
    if (h->opt.use_graph && h->graph_exec) e = cudaGraphLaunch(h->graph_exec, s);
    else if ((rc = enqueue_run(h, s))) return rc;
    if (e == cudaSuccess && (rc = charm_host::enqueue_status_latch(h->d_latch, s))) return rc;
    // result k into stage_out[b] once the copy of result k-2 has left it
    if (e == cudaSuccess && k >= 2) e = cudaStreamWaitEvent(s, h->out_free[b], 0);
    if (e == cudaSuccess) {
      enqueue_gather(h, prob, stage_out[b], s);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaEventRecord(h->out_ready[b], s);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(h->s_d2h, h->out_ready[b], 0);
    if (e == cudaSuccess) e = cudaMemcpyAsync(host_out[k], stage_out[b], bytes, cudaMemcpyDeviceToHost, h->s_d2h);
    if (e == cudaSuccess) e = cudaEventRecord(h->out_free[b], h->s_d2h);
  }
  if (e == cudaSuccess) e = cudaEventRecord(h->ev1, h->s_d2h);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->s_d2h);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  float ms = 0.f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, h->ev0, h->ev1);
  if (out_ms) *out_ms = ms;
  int latch[4] = {0, 0, 0, 0};
  if (e == cudaSuccess) e = cudaMemcpy(latch, h->d_latch, sizeof(latch), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return check_cuda(e, "jacobi2d solve stream");
  return latch[0];
}

extern "C" int charming_jacobi2d_result(void* handle, int prob, charming_jacobi_result* out) {
  JHandle* h = reinterpret_cast<JHandle*>(handle);
  if (!h || !out || prob < 0 || prob >= (int)h->probs.size()) return CHARMING_ERR_CONFIG;
  jac::prob_result r;
  cudaError_t e = cudaMemcpy(&r, h->d_results + prob, sizeof(r), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return check_cuda(e, "jacobi2d result");
  out->sweeps = r.sweeps;
  out->checks = r.checks;
  out->res0 = r.res0;
  out->res_last = r.res_last;
  return CHARMING_OK;
}

extern "C" int charming_jacobi2d_get_info(void* handle, charming_jacobi_info* out) {
  JHandle* h = reinterpret_cast<JHandle*>(handle);
  if (!h || !out) return CHARMING_ERR_CONFIG;
  out->n_problems = (int)h->probs.size();
  out->n_chares = h->n_chares;
  out->max_chares_per_pe = h->max_per_pe;
  out->interior_points = h->points;
  out->grid_bytes = h->grid_bytes;
  out->halo_msgs_per_sweep = h->halo_msgs;
  out->last_run_ms = h->last_ms;
  // the per-PE phase timers count SM cycles
  std::vector<unsigned long long> ns(8 * h->block_map.size());
  cudaError_t e = cudaMemcpy(ns.data(), h->d_sweep_ns, 8 * ns.size(), cudaMemcpyDeviceToHost);
  int dev = 0, khz = 0;
  if (e == cudaSuccess) e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, dev);
  if (e != cudaSuccess) return check_cuda(e, "jacobi2d info");
  const double ms_per = khz > 0 ? 1.0 / khz : 0.0;
  double mx = 0, sum[6] = {0, 0, 0, 0, 0, 0};
  int busy = 0;
  for (size_t p = 0; p < h->block_map.size(); p++) {
    mx = std::max(mx, (double)ns[8 * p]);
    if (h->block_map[p] > 0) {
      for (int k = 0; k < 6; k++) sum[k] += (double)ns[8 * p + k];
      busy++;
    }
  }
  out->send_reserve_ms_mean = busy ? sum[3] / busy * ms_per : 0.0;
  out->send_publish_ms_mean = busy ? sum[4] / busy * ms_per : 0.0;
  out->send_setup_ms_mean = busy ? sum[5] / busy * ms_per : 0.0;
  out->sweep_ms_max = mx * ms_per;
  out->sweep_ms_mean = busy ? sum[0] / busy * ms_per : 0.0;
  out->send_ms_mean = busy ? sum[1] / busy * ms_per : 0.0;
  out->halo_ms_mean = busy ? sum[2] / busy * ms_per : 0.0;
  return CHARMING_OK;
}

extern "C" int charming_jacobi2d_destroy(void* handle) {
  JHandle* h = reinterpret_cast<JHandle*>(handle);
  if (!h) return CHARMING_OK;
  cudaDeviceSynchronize();
  if (h->graph_exec) cudaGraphExecDestroy(h->graph_exec);
  if (h->graph) cudaGraphDestroy(h->graph);
  cudaFree(h->d_grid);
  cudaFree(h->d_chares);
  cudaFree(h->d_probs);
  cudaFree(h->d_results);
  cudaFree(h->d_done);
  cudaFree(h->d_final);
  cudaFree(h->d_block_map);
  cudaFree(h->d_chare_of);
  cudaFree(h->d_sweep_ns);
  cudaFree(h->d_stage);
  cudaFree(h->d_pipe);
  cudaFree(h->d_latch);
  if (h->s_h2d) cudaStreamDestroy(h->s_h2d);
  if (h->s_d2h) cudaStreamDestroy(h->s_d2h);
  for (int b = 0; b < 2; b++) {
    if (h->in_ready[b]) cudaEventDestroy(h->in_ready[b]);
    if (h->in_free[b]) cudaEventDestroy(h->in_free[b]);
    if (h->out_ready[b]) cudaEventDestroy(h->out_ready[b]);
    if (h->out_free[b]) cudaEventDestroy(h->out_free[b]);
  }
  if (h->h_params) cudaFreeHost(h->h_params);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  delete h;
  return CHARMING_OK;
}
