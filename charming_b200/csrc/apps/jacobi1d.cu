// Jacobi1d chares: the scenario of the reference's examples/jacobi1d
// (jacobi1d.cu:62-170): n chares of `width` points with 2 ghost points per
// side, boundary ghosts 10 and interior 0, 5-point window
// sum = 0; sum += t[i-2..i+2]; new = sum / 5. Ghosts travel as 32-byte
// messages tagged refnum = sweep (the reference sends them untagged and
// ends the run when the first chare finishes, jacobi1d.cu:120-139; here the
// last chare to finish calls end()).
#include "suite.cuh"
#include "../host.cuh"
#include <vector>

namespace {

constexpr int GHOST = 2;

struct J1Block : charm::chare {
  int iter, cur, got, nbrs;
  __device__ J1Block() : iter(0), cur(0), got(0), nbrs(0) {}
};

struct ghost_msg {
  int dir;  // 0: goes to the receiver's left ghosts, 1: right ghosts
  int iter;
  double data[GHOST];
};

__shared__ charm::chare_proxy<J1Block>* j1proxy;

// g_app: a[0] n chares, a[1] width, a[2] sweeps; p[0] slab of 2 buffers of
// (width + 4) doubles per chare (stride a[3] doubles); p[1] done counter;
// p[2] final buffer index per chare.
__device__ double* j1buf(int chare, int b) {
  long long stride = g_app.a[3];
  return reinterpret_cast<double*>(g_app.p[0]) + (size_t)chare * 2 * stride + (size_t)b * stride;
}

__device__ void j1_send(J1Block& c) {
  int n = (int)g_app.a[0], w = (int)g_app.a[1];
  double* a = j1buf(c.i, c.cur);
  ghost_msg m;
  m.iter = c.iter;
  if (c.i > 0) {  // my first two interior points -> left neighbour's right ghosts
    m.dir = 1;
    m.data[0] = a[GHOST];
    m.data[1] = a[GHOST + 1];
    j1proxy->invoke(c.i - 1, 1, &m, sizeof(m), c.iter);
  }
  if (c.i < n - 1) {
    m.dir = 0;
    m.data[0] = a[w];
    m.data[1] = a[w + 1];
    j1proxy->invoke(c.i + 1, 1, &m, sizeof(m), c.iter);
  }
}

__device__ void j1_step(J1Block& c) {
  int w = (int)g_app.a[1], sweeps = (int)g_app.a[2];
  while (true) {
    __shared__ int s_done;
    if (threadIdx.x == 0) s_done = (c.iter >= sweeps) ? 1 : 0;
    __syncthreads();
    if (s_done) {
      __shared__ int s_last;
      if (threadIdx.x == 0) {
        reinterpret_cast<int*>(g_app.p[2])[c.i] = c.cur;
        __threadfence();
        unsigned long long k = atomicAdd(reinterpret_cast<unsigned long long*>(g_app.p[1]), 1ULL) + 1;
        s_last = (k == (unsigned long long)g_app.a[0]) ? 1 : 0;
      }
      __syncthreads();
      if (s_last) charm::end();
      return;
    }
    if (c.nbrs > 0) {
      if (threadIdx.x == 0) j1proxy->set_refnum(c.i, c.iter);
      __syncthreads();
      j1_send(c);
      return;
    }
    // single chare: sweep in place without messages
    const double* a = j1buf(c.i, c.cur);
    double* b = j1buf(c.i, c.cur ^ 1);
    for (int i = GHOST + threadIdx.x; i < w + GHOST; i += blockDim.x) {
      double s = 0;
      for (int j = -GHOST; j <= GHOST; j++) s = __dadd_rn(s, a[i + j]);
      b[i] = __ddiv_rn(s, (double)(1 + 2 * GHOST));
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      c.cur ^= 1;
      c.iter++;
    }
    __syncthreads();
  }
}

__device__ void j1_start(J1Block& c, void* arg) {
  int n = (int)g_app.a[0];
  if (threadIdx.x == 0) c.nbrs = (c.i > 0) + (c.i < n - 1);
  __syncthreads();
  j1_step(c);
}

__device__ void j1_ghost(J1Block& c, void* arg) {
  int w = (int)g_app.a[1];
  const ghost_msg* m = reinterpret_cast<const ghost_msg*>(arg);
  __shared__ int s_go;
  if (threadIdx.x == 0) {
    double* a = j1buf(c.i, c.cur);
    int base = m->dir == 0 ? 0 : w + GHOST;
    a[base] = m->data[0];
    a[base + 1] = m->data[1];
    s_go = (++c.got == c.nbrs) ? 1 : 0;
  }
  __syncthreads();
  if (!s_go) return;
  const double* a = j1buf(c.i, c.cur);
  double* b = j1buf(c.i, c.cur ^ 1);
  for (int i = GHOST + threadIdx.x; i < w + GHOST; i += blockDim.x) {
    double s = 0;
    for (int j = -GHOST; j <= GHOST; j++) s = __dadd_rn(s, a[i + j]);
    b[i] = __ddiv_rn(s, (double)(1 + 2 * GHOST));
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    c.cur ^= 1;
    c.iter++;
    c.got = 0;
  }
  __syncthreads();
  j1_step(c);
}

}  // namespace

__device__ void suite::jacobi1d_main(int pe) {
  if (threadIdx.x == 0) {
    j1proxy = new charm::chare_proxy<J1Block>();
    j1proxy->add_entry_method<&j1_start>();
    j1proxy->add_entry_method<&j1_ghost>();
    j1proxy->create((int)g_app.a[0]);
  }
  __syncthreads();
  if (j1proxy->n_local > 0) {
    for (int i = j1proxy->start_idx; i <= j1proxy->end_idx; i++) j1proxy->invoke(i, 0);
  }
}

__global__ void j1_init_kernel(double* slab, int n, int w, long long stride) {
  long long total = (long long)n * 2 * stride;
  for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < total;
       x += (long long)gridDim.x * blockDim.x) {
    long long k = x / (2 * stride), i = x % stride;
    double v = 0.0;
    if ((k == 0 && i < GHOST) || (k == n - 1 && i >= w + GHOST && i < w + 2 * GHOST)) v = 10.0;
    slab[x] = v;
  }
}

extern "C" int charming_jacobi1d(int n_chares, int width, int sweeps, double* host_out,
    double* out_ms) {
  int rc = charm_host::ensure_init();
  if (rc) return rc;
  if (n_chares < 1 || width < GHOST || sweeps < 0 || !host_out) return CHARMING_ERR_CONFIG;
  long long stride = ((long long)width + 2 * GHOST + 15) / 16 * 16;
  double* slab = nullptr;
  unsigned long long* ctr = nullptr;
  int* fin = nullptr;
  cudaError_t e = cudaMalloc(&slab, sizeof(double) * n_chares * 2 * stride);
  if (e == cudaSuccess) e = cudaMalloc(&ctr, 64);
  if (e == cudaSuccess) e = cudaMalloc(&fin, sizeof(int) * n_chares);
  if (e != cudaSuccess) {
    cudaFree(slab);
    cudaFree(ctr);
    return charm_host::cuda_fail(e, "jacobi1d buffers");
  }
  j1_init_kernel<<<1024, 256>>>(slab, n_chares, width, stride);
  cudaMemset(ctr, 0, 64);
  cudaMemset(fin, 0, sizeof(int) * n_chares);
  cudaDeviceSynchronize();
  suite::app_params p{};
  p.id = suite::APP_JACOBI1D;
  p.a[0] = n_chares;
  p.a[1] = width;
  p.a[2] = sweeps;
  p.a[3] = stride;
  p.p[0] = slab;
  p.p[1] = ctr;
  p.p[2] = fin;
  rc = suite_run(p);
  std::vector<int> hf(n_chares);
  std::vector<double> hb((size_t)n_chares * 2 * stride);
  cudaMemcpy(hf.data(), fin, sizeof(int) * n_chares, cudaMemcpyDeviceToHost);
  cudaMemcpy(hb.data(), slab, sizeof(double) * hb.size(), cudaMemcpyDeviceToHost);
  // global array: 2 left boundary ghosts, all interiors, 2 right ghosts
  const double* first = &hb[(size_t)hf[0] * stride];
  host_out[0] = first[0];
  host_out[1] = first[1];
  for (int k = 0; k < n_chares; k++) {
    const double* a = &hb[(size_t)k * 2 * stride + (size_t)hf[k] * stride];
    for (int i = 0; i < width; i++) host_out[2 + (size_t)k * width + i] = a[GHOST + i];
  }
  const double* last = &hb[(size_t)(n_chares - 1) * 2 * stride + (size_t)hf[n_chares - 1] * stride];
  host_out[2 + (size_t)n_chares * width] = last[width + GHOST];
  host_out[3 + (size_t)n_chares * width] = last[width + GHOST + 1];
  charming_stats st;
  charming_last_stats(&st);
  if (out_ms) *out_ms = st.kernel_ms;
  cudaFree(slab);
  cudaFree(ctr);
  cudaFree(fin);
  return rc;
}
